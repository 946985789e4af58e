"""TEST INFRASTRUCTURE ONLY (the oracle): a restatement, in numpy, of zephyr's
VTU and PVD writers (io/vtu_file.cpp, io/pvd_file.cpp, io/vtk_type.*) for
2-D adaptive meshes written as quadrilaterals (VtuStructure::
fill_adaptive_hex_2D, vtu_file.cpp:186-201), the default of PvdFile and
VtuFile.  It checks the CUDA library's writer byte for byte; the reference's
own writer pins it (tests/golden/vtu_*.npz).

A variable is (name, vtk type, components, array of n cells x components).
"""
from __future__ import annotations

import numpy as np

VTK_QUAD = 9
# VtkType names of the numpy types the writer uses (vtk_type.cpp:70-95)
_VTK = {np.dtype(np.int8): "Int8", np.dtype(np.int32): "Int32", np.dtype(np.uint8): "UInt8",
        np.dtype(np.uint32): "UInt32", np.dtype(np.float32): "Float32", np.dtype(np.float64): "Float64"}


def quad_points(map_x, map_y):
    """The four corners vs<-1,-1>, vs<+1,-1>, vs<+1,+1>, vs<-1,+1> of every
    cell (map points 0, 2, 8, 6 of 9), as (4 n, 3) doubles with z = 0."""
    mx = np.asarray(map_x, dtype=np.float64).reshape(-1, 9)
    my = np.asarray(map_y, dtype=np.float64).reshape(-1, 9)
    n = mx.shape[0]
    pts = np.zeros((n, 4, 3))
    for k, q in enumerate((0, 2, 8, 6)):
        pts[:, k, 0] = mx[:, q]
        pts[:, k, 1] = my[:, q]
    return pts.reshape(-1, 3)


def cell_variable(name, cells):
    """The named variables of io/variable.cpp:11-160 from per-cell arrays
    (dict with level, flag, b_idx, z_idx, cx, cy)."""
    n = len(cells["cx"])
    if name == "rank":
        return (name, np.zeros(n, np.int32))
    if name == "index":
        return (name, np.arange(n, dtype=np.int32))
    if name == "level":
        return (name, np.asarray(cells["level"]).astype(np.int8))
    if name == "flag":
        return (name, np.asarray(cells["flag"]).astype(np.int8))
    if name == "b_idx":
        return (name, np.asarray(cells["b_idx"]).astype(np.int32))
    if name == "z_idx":
        return (name, np.asarray(cells["z_idx"]).astype(np.int32))
    if name in ("center", "coords"):
        c = np.zeros((n, 3), np.float32)
        c[:, 0] = np.asarray(cells["cx"], dtype=np.float64).astype(np.float32)
        c[:, 1] = np.asarray(cells["cy"], dtype=np.float64).astype(np.float32)
        return (name, c)
    raise ValueError(f"unknown variable '{name}'")


def vtu_bytes(points, variables):
    """VtuStructure::write_header + write_primitives + write_cells_data
    (vtu_file.cpp:439-530) of quadrilateral cells with the given corner
    points ((4 n, 3) doubles) and (name, array) variables."""
    points = np.ascontiguousarray(points, dtype=np.float64)
    n_points = points.shape[0]
    n_cells = n_points // 4
    conn = np.arange(n_points, dtype=np.uint32)
    offsets = (4 * (np.arange(n_cells, dtype=np.uint32) + 1)).astype(np.uint32)
    types = np.full(n_cells, VTK_QUAD, np.uint8)
    head = []
    head.append('<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">\n')
    head.append("  <UnstructuredGrid>\n")
    head.append(f'    <Piece NumberOfPoints="{n_points}" NumberOfCells="{n_cells}">\n')
    off = 0
    head.append("      <Points>\n")
    head.append(f'        <DataArray type="Float64" Name="Points" NumberOfComponents="3" format="appended" '
                f'offset="{off}"/>\n')
    head.append("      </Points>\n")
    off += 4 + points.nbytes
    head.append("      <Cells>\n")
    for arr, nm in ((conn, "connectivity"), (offsets, "offsets"), (types, "types")):
        head.append(f'        <DataArray type="{_VTK[arr.dtype]}" Name="{nm}" format="appended" offset="{off}"/>\n')
        off += 4 + arr.nbytes
    head.append("      </Cells>\n")
    head.append("      <CellData>\n")
    blobs = []
    for name, arr in variables:
        arr = np.ascontiguousarray(arr)
        comps = 1 if arr.ndim == 1 else arr.shape[1]
        line = f'        <DataArray type="{_VTK[arr.dtype]}" Name="{name}'
        if comps >= 2:
            line += f'" NumberOfComponents="{comps}'
        line += f'" format="appended" offset="{off}"/>\n'
        head.append(line)
        off += 4 + n_cells * comps * arr.dtype.itemsize
        blobs.append(arr)
    head.append("      </CellData>\n")
    head.append("    </Piece>\n")
    head.append("  </UnstructuredGrid>\n")
    out = bytearray("".join(head).encode())
    out += b'  <AppendedData encoding="raw">\n_'
    for arr in (points, conn, offsets, types, *blobs):
        out += np.uint32(arr.nbytes).tobytes() + arr.tobytes()
    return bytes(out)


def pvd_text(filename, datasets):
    """PvdFile::open + update_pvd (pvd_file.cpp:89-211), one rank: the file
    `filename`.pvd after saves at the given timesteps."""
    lines = ['<?xml version="1.0"?>\n', '<VTKFile type="Collection" version="0.1" byte_order="LittleEndian">\n',
             "    <Collection>\n"]
    for k, t in enumerate(datasets):
        lines.append(f'        <DataSet timestep="{t:.15e}" part="0" file="{filename}_{k}.vtu"/>\n')
    lines += ["    </Collection>\n", "</VTKFile>\n"]
    return "".join(lines)
