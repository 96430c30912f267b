// Minimal stand-in for the parts of Onika's operator API (onika/scg) that a hippoLBM plugin
// uses: OperatorNode, ADD_SLOT, OperatorNodeFactory, make_simple_operator, ONIKA_AUTORUN_INIT.
// Test infrastructure only: it lets tests/cpp compile and run hippolbm_b200/host/onika_plugin.cpp
// without Onika (which is not part of this project).  Slots resolve by name, first in the
// operator's own configuration (what a deck's YAML gives that operator), then in the graph's
// shared slots (what operators exchange: the reference's `fields`, here the `hlbm` handle).
#pragma once
#include <any>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>

namespace onika {
namespace scg {

enum SlotMode { INPUT, OUTPUT, INPUT_OUTPUT, PRIVATE };
enum SlotRequirement { REQUIRED, OPTIONAL };
struct DocString {
  const char* text = "";
};

// the graph's shared slots (one graph per process in this stand-in)
inline std::map<std::string, std::any>& shared_slots() {
  static std::map<std::string, std::any> m;
  return m;
}

class OperatorNode {
 public:
  virtual ~OperatorNode() = default;
  virtual void execute() = 0;
  // what a deck gives this operator (its own slot values)
  template <class T>
  void configure(const std::string& slot, T value) {
    local_[slot] = std::move(value);
  }
  std::any* find_local(const std::string& slot) {
    auto it = local_.find(slot);
    return it == local_.end() ? nullptr : &it->second;
  }

 private:
  std::map<std::string, std::any> local_;
};

template <class T>
class OperatorSlot {
 public:
  OperatorSlot(OperatorNode* owner, const char* name, SlotMode mode, SlotRequirement req, DocString = {})
      : owner_(owner), name_(name), mode_(mode), required_(req == REQUIRED) {}
  OperatorSlot(OperatorNode* owner, const char* name, SlotMode mode, T default_value, DocString = {})
      : owner_(owner), name_(name), mode_(mode), required_(false), default_(std::move(default_value)), has_default_(true) {}
  bool has_value() const { return lookup(false) != nullptr; }
  T* operator->() const { return lookup(true); }
  T& operator*() const { return *lookup(true); }

 private:
  T* lookup(bool create) const {
    if (std::any* a = owner_->find_local(name_)) return std::any_cast<T>(a);
    auto& g = shared_slots();
    auto it = g.find(name_);
    if (it != g.end()) return std::any_cast<T>(&it->second);
    if (!create) return nullptr;
    if (has_default_) return std::any_cast<T>(&(g[name_] = default_));
    if (mode_ == OUTPUT || mode_ == INPUT_OUTPUT || !required_) return std::any_cast<T>(&(g[name_] = T{}));
    throw std::runtime_error("required slot '" + name_ + "' has no value");
  }
  OperatorNode* owner_;
  std::string name_;
  SlotMode mode_;
  bool required_;
  T default_{};
  bool has_default_ = false;
};

#define ADD_SLOT(type, name, mode, ...) ::onika::scg::OperatorSlot<type> name{this, #name, ::onika::scg::mode, __VA_ARGS__}

class OperatorNodeFactory {
 public:
  using Maker = std::function<std::shared_ptr<OperatorNode>()>;
  static OperatorNodeFactory* instance() {
    static OperatorNodeFactory f;
    return &f;
  }
  void register_factory(const std::string& name, Maker make) { makers_[name] = std::move(make); }
  std::shared_ptr<OperatorNode> make_operator(const std::string& name) const {
    auto it = makers_.find(name);
    if (it == makers_.end()) throw std::runtime_error("no operator named '" + name + "'");
    return it->second();
  }

 private:
  std::map<std::string, Maker> makers_;
};

template <class T>
std::shared_ptr<OperatorNode> make_simple_operator() {
  return std::make_shared<T>();
}

}  // namespace scg
}  // namespace onika

#define ONIKA_AUTORUN_INIT(tag)                                       \
  static void onika_autorun_##tag();                                  \
  static const int onika_autorun_reg_##tag = (onika_autorun_##tag(), 0); \
  static void onika_autorun_##tag()
