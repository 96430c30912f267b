"""ParaView output of a lattice (`write_paraview`, write_paraview.cpp:71-80 / write_paraview.hpp).

Same directory layout, file names and point fields as the reference writer:
<output_directory>/ParaviewOutput/<filename % timestep>.pvtr, pointing at
<output_directory>/ParaviewOutput/<filename % timestep>/000000.vtr, with
  P    = c^2 * avg_rho / 3 * (rho - 1) on fluid nodes, 0 elsewhere (writer.hpp:54-62),
  U    = dx / dtLB * u on fluid nodes, 0 elsewhere (writer.hpp:41-51),
  OBST = the flag value,
  Fi   = the 19 populations when `distributions` is set (write_paraview.cpp:73-76),
all Float32, over the real nodes with coordinates x * dx.  The reference writes ASCII; this writer
stores the arrays as raw appended binary (the same VTK XML schema), which ParaView reads the same
way and which is what makes whole-lattice output affordable at 10^8 nodes.
"""
from __future__ import annotations

import os

import numpy as np


def _array_header(name: str, comps: int, offset: int) -> str:
    return (f'          <DataArray type="Float32" Name="{name}" NumberOfComponents="{comps}" '
            f'format="appended" offset="{offset}"/>\n')


def write_vtr(path: str, dx: float, fields: list[tuple[str, np.ndarray]], n: tuple[int, int, int]):
    """fields: (name, float32 array of shape (nodes,) or (nodes, comps)) in x-fastest node order."""
    nx, ny, nz = n
    coords = [("X", (np.arange(nx) * dx).astype(np.float32)), ("Y", (np.arange(ny) * dx).astype(np.float32)),
              ("Z", (np.arange(nz) * dx).astype(np.float32))]
    blocks, offset, head = [], 0, []
    extent = f"0 {nx - 1} 0 {ny - 1} 0 {nz - 1}"
    head.append('<?xml version="1.0"?>\n')
    head.append('<VTKFile type="RectilinearGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">\n')
    head.append(f' <RectilinearGrid WholeExtent="{extent}">\n')
    head.append(f'  <Piece Extent="{extent}">\n')
    head.append('   <Coordinates>\n')
    for name, a in coords:
        head.append(_array_header(name, 1, offset))
        blocks.append(a)
        offset += 8 + a.nbytes
    head.append('   </Coordinates>\n')
    head.append('   <PointData>\n')
    for name, a in fields:
        comps = 1 if a.ndim == 1 else a.shape[1]
        head.append(_array_header(name, comps, offset))
        blocks.append(a)
        offset += 8 + a.nbytes
    head.append('   </PointData>\n  </Piece>\n </RectilinearGrid>\n <AppendedData encoding="raw">\n_')
    with open(path, "wb") as fh:
        fh.write("".join(head).encode())
        for a in blocks:
            a = np.ascontiguousarray(a, dtype="<f4")
            fh.write(np.uint64(a.nbytes).tobytes())
            fh.write(a.tobytes())
        fh.write(b"\n </AppendedData>\n</VTKFile>\n")


def write_pvtr(path: str, piece: str, fields: list[tuple[str, int]], n: tuple[int, int, int]):
    nx, ny, nz = n
    extent = f"0 {nx - 1} 0 {ny - 1} 0 {nz - 1}"
    with open(path, "w") as fh:
        fh.write('<?xml version="1.0"?>\n<VTKFile type="PRectilinearGrid" version="1.0" byte_order="LittleEndian">\n')
        fh.write(f' <PRectilinearGrid WholeExtent="{extent}" GhostLevel="0">\n')
        fh.write(f'  <Piece Extent="{extent}" Source="{piece}"/>\n')
        fh.write('  <PCoordinates>\n')
        for name in "XYZ":
            fh.write(f'   <PDataArray type="Float32" Name="{name}"/>\n')
        fh.write('  </PCoordinates>\n  <PPointData Scalars="P OBST" Vectors="U">\n')
        for name, comps in fields:
            fh.write(f'   <PDataArray Name="{name}" type="Float32" NumberOfComponents="{comps}"/>\n')
        fh.write('  </PPointData>\n </PRectilinearGrid>\n</VTKFile>\n')


def write_paraview(lat, timestep: int, output_directory: str = "hippoLBMOutputDir",
                   filename: str = "hippoLBM_%010d", distributions: bool = False) -> str:
    """Write one time step of `lat` (a `Lattice`); returns the .pvtr path."""
    prm = lat.parameters()
    info = lat.info()
    n = (info["nx"], info["ny"], info["nz"])
    dx = prm["celerity"] * prm["dtLB"]
    rho, u = lat.macro()
    flags = lat.flags().reshape(-1)
    fluid = flags == -1
    p = np.where(fluid, prm["celerity"] ** 2 * prm["avg_rho"] / 3.0 * (rho.reshape(-1) - 1.0), 0.0)
    uu = u.reshape(3, -1).T * (dx / prm["dtLB"])
    uu[~fluid] = 0.0
    fields = [("P", p.astype(np.float32)), ("OBST", flags.astype(np.float32)), ("U", uu.astype(np.float32))]
    if distributions:
        f = lat.populations().reshape(19, -1).T
        fields.append(("Fi", f.astype(np.float32)))
    base = os.path.join(output_directory, "ParaviewOutput")
    name = filename % timestep
    os.makedirs(os.path.join(base, name), exist_ok=True)
    write_vtr(os.path.join(base, name, "000000.vtr"), dx, fields, n)
    pvtr = os.path.join(base, name + ".pvtr")
    write_pvtr(pvtr, f"{name}/000000.vtr", [(k, 1 if a.ndim == 1 else a.shape[1]) for k, a in fields], n)
    return pvtr


def read_vtr(path: str) -> dict:
    """Arrays of a .vtr written by `write_vtr` (raw appended Float32), by name."""
    with open(path, "rb") as fh:
        data = fh.read()
    split = data.index(b'<AppendedData encoding="raw">')
    head = data[:split].decode()
    start = data.index(b"_", split) + 1
    out = {}
    import re

    for m in re.finditer(r'Name="(\w+)" NumberOfComponents="(\d+)" format="appended" offset="(\d+)"', head):
        name, comps, off = m.group(1), int(m.group(2)), int(m.group(3))
        nbytes = int(np.frombuffer(data, np.uint64, 1, start + off)[0])
        a = np.frombuffer(data, "<f4", nbytes // 4, start + off + 8)
        out[name] = a.reshape(-1, comps) if comps > 1 else a
    return out
