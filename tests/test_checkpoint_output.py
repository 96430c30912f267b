"""Checkpoint / restore of the carried state and the ParaView writer.

A lattice restored from a checkpoint of the same deck continues bit for bit in every tier (the
image holds the populations exactly as stored, plus the step count that salts stochastic
rounding).  The ParaView writer emits the reference's P / U / OBST point fields."""
import numpy as np
import pytest

from hippolbm_b200.deck import couette_case, sphere_channel_case
from hippolbm_b200.output import read_vtr, write_vtr


def test_vtr_roundtrip(tmp_path):
    rng = np.random.default_rng(3)
    n = (5, 4, 3)
    p = rng.random(60).astype(np.float32)
    u = rng.random((60, 3)).astype(np.float32)
    path = str(tmp_path / "a.vtr")
    write_vtr(path, 0.5, [("P", p), ("U", u)], n)
    back = read_vtr(path)
    assert np.array_equal(back["P"], p) and np.array_equal(back["U"], u)
    assert np.allclose(back["X"], np.arange(5) * 0.5) and back["Z"].size == 3
    head = open(path, "rb").read().split(b"<AppendedData")[0].decode()
    assert 'WholeExtent="0 4 0 3 0 2"' in head and 'Name="U" NumberOfComponents="3"' in head


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64_strict", "f32", "f16", "bf16"])
def test_restart_continues_bit_for_bit(precision, tmp_path):
    """The image carries the storage parameters and the step count: a context restored from it
    needs nothing but the deck."""
    from hippolbm_b200.lattice import Lattice

    case = sphere_channel_case((40, 18, 16), (10.0, 9.0, 8.0), 3.0, steps=30, collision="mrt")
    with Lattice.from_case(case, precision) as a:
        a.step(13)
        path = str(tmp_path / "ckpt.bin")
        a.save_checkpoint(path)
        a.step(17)
        f_ref = a.populations()
    with Lattice.from_case(case, precision) as b:
        b.load_checkpoint(path)
        assert b.info()["steps"] == 13
        b.step(17)
        assert np.array_equal(b.populations(), f_ref)


@pytest.mark.gpu
def test_storage_reencode_on_the_device():
    """Changing the storage scale or the collision (which sets the MRT rest reference) re-encodes
    the 16-bit state on the device: the populations move by at most one storage quantum."""
    from hippolbm_b200.lattice import Lattice

    case = sphere_channel_case((32, 16, 16), (8.0, 8.0, 8.0), 3.0, steps=40, collision="bgk")
    with Lattice.from_case(case, "f16") as lat:
        lat.step(40)
        f0 = lat.populations()
        dev = np.abs(f0 - np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)[:, None, None, None]).max()
        lat.L.hlbm_storage_scale(lat.h, 1.0, 4096.0)
        f1 = lat.populations()
        lat.L.hlbm_collision(lat.h, 1, None)  # MRT: the rest reference moves by up to 0.15
        f2 = lat.populations()
    assert np.abs(f1 - f0).max() <= dev * 2.0 ** -10
    assert np.abs(f2 - f1).max() <= (dev + 0.15) * 2.0 ** -10


@pytest.mark.gpu
def test_restore_rejects_another_shape():
    from hippolbm_b200 import capi
    from hippolbm_b200.lattice import Lattice

    with Lattice.from_case(couette_case(16, 0.7, 0.05, 1), "f32") as a, \
            Lattice.from_case(couette_case(12, 0.7, 0.05, 1), "f32") as b:
        img = a.checkpoint()
        with pytest.raises(capi.HlbmError):
            b.restore(img)
        with pytest.raises(capi.HlbmError):
            b.restore(img[:100])


@pytest.mark.gpu
def test_write_paraview_fields(tmp_path):
    from hippolbm_b200.lattice import Lattice
    from hippolbm_b200.output import write_paraview

    case = sphere_channel_case((32, 16, 16), (8.0, 8.0, 8.0), 3.0, steps=20, collision="bgk")
    with Lattice.from_case(case, "f64") as lat:
        lat.step(20)
        pvtr = write_paraview(lat, 20, str(tmp_path), distributions=True)
        rho, u = lat.macro()
        flags = lat.flags().reshape(-1)
        f = lat.populations()
        prm = lat.parameters()
    assert pvtr.endswith("hippoLBM_0000000020.pvtr")
    d = read_vtr(str(tmp_path / "ParaviewOutput" / "hippoLBM_0000000020" / "000000.vtr"))
    fluid = flags == -1
    p_ref = np.where(fluid, prm["celerity"] ** 2 * prm["avg_rho"] / 3.0 * (rho.reshape(-1) - 1.0), 0.0)
    p_ref = p_ref.astype(np.float32)
    assert np.array_equal(d["P"], p_ref)
    assert np.array_equal(d["OBST"], flags.astype(np.float32))
    u_ref = u.reshape(3, -1).T.copy()
    u_ref[~fluid] = 0
    assert np.array_equal(d["U"], u_ref.astype(np.float32))
    assert np.array_equal(d["Fi"], f.reshape(19, -1).T.astype(np.float32))
