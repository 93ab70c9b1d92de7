"""Exodus II test files written with scipy's NetCDF classic writer (an
implementation independent of the library's reader), with the dimension and
variable names the Exodus library uses: coordinates, element blocks with
elem_type, elemental variables of one time step, named side sets."""
import numpy as np
from scipy.io import netcdf_file

LEN_NAME = 33


def _names(strings):
    out = np.zeros((len(strings), LEN_NAME), dtype="S1")
    for i, s in enumerate(strings):
        for k, ch in enumerate(s.encode()):
            out[i, k] = bytes([ch])
    return out


def write(path, coords, blocks, elem_type, elem_vars=None, side_sets=None, version=2,
          split_coords=True):
    """coords [n][dim]; blocks: list of 1-based connectivity arrays in Exodus
    node order; elem_vars: {name: [n_elem] values over the concatenated
    blocks}; side_sets: {name: (elem ids 1-based, side ids 1-based)}."""
    elem_vars = elem_vars or {}
    side_sets = side_sets or {}
    n, dim = coords.shape
    f = netcdf_file(path, "w", version=version)
    f.api_version = np.float32(5.22)
    f.version = np.float32(5.22)
    f.floating_point_word_size = np.int32(8)
    f.title = b"salvus test mesh"
    # (scipy's writer takes the record dimension first only)
    f.createDimension("time_step", None)
    f.createDimension("len_string", LEN_NAME)
    f.createDimension("len_name", LEN_NAME)
    f.createDimension("four", 4)
    f.createDimension("num_dim", dim)
    f.createDimension("num_nodes", n)
    f.createDimension("num_elem", sum(len(b) for b in blocks))
    f.createDimension("num_el_blk", len(blocks))
    t = f.createVariable("time_whole", "d", ("time_step",))
    t[0] = 0.0
    ids = f.createVariable("eb_prop1", "i", ("num_el_blk",))
    ids.name = b"ID"
    ids[:] = np.arange(1, len(blocks) + 1, dtype=np.int32)
    if split_coords:
        for a, nm in enumerate(["coordx", "coordy", "coordz"][:dim]):
            v = f.createVariable(nm, "d", ("num_nodes",))
            v[:] = coords[:, a]
    else:
        v = f.createVariable("coord", "d", ("num_dim", "num_nodes"))
        v[:] = coords.T
    for b, conn in enumerate(blocks, start=1):
        f.createDimension(f"num_el_in_blk{b}", len(conn))
        f.createDimension(f"num_nod_per_el{b}", conn.shape[1])
        c = f.createVariable(f"connect{b}", "i", (f"num_el_in_blk{b}", f"num_nod_per_el{b}"))
        c.elem_type = elem_type.encode()
        c[:] = conn.astype(np.int32)
    if elem_vars:
        names = list(elem_vars)
        f.createDimension("num_elem_var", len(names))
        nv = f.createVariable("name_elem_var", "c", ("num_elem_var", "len_name"))
        nv[:] = _names(names)
        off = 0
        for b, conn in enumerate(blocks, start=1):
            for k, nm in enumerate(names, start=1):
                v = f.createVariable(f"vals_elem_var{k}eb{b}", "d", ("time_step", f"num_el_in_blk{b}"))
                v[0, :] = np.asarray(elem_vars[nm])[off:off + len(conn)]
            off += len(conn)
    if side_sets:
        names = list(side_sets)
        f.createDimension("num_side_sets", len(names))
        sn = f.createVariable("ss_names", "c", ("num_side_sets", "len_name"))
        sn[:] = _names(names)
        sp = f.createVariable("ss_prop1", "i", ("num_side_sets",))
        sp[:] = np.arange(1, len(names) + 1, dtype=np.int32)
        for s, nm in enumerate(names, start=1):
            el, sd = side_sets[nm]
            f.createDimension(f"num_side_ss{s}", len(el))
            e = f.createVariable(f"elem_ss{s}", "i", (f"num_side_ss{s}",))
            e[:] = np.asarray(el, dtype=np.int32)
            d = f.createVariable(f"side_ss{s}", "i", (f"num_side_ss{s}",))
            d[:] = np.asarray(sd, dtype=np.int32)
    f.close()


def box_side_sets(coords, cells_exo, sides, lo, hi, axes="xyz"):
    """Side sets x0, x1, y0, y1 (, z0, z1) of an axis-aligned box: every
    element side (Exodus local node lists `sides`) whose nodes all lie on the
    plane."""
    out = {}
    dim = coords.shape[1]
    for a in range(dim):
        for tag, val in (("0", lo[a]), ("1", hi[a])):
            el, sd = [], []
            for e, cell in enumerate(cells_exo):
                for s, loc in enumerate(sides):
                    if np.all(np.abs(coords[cell[list(loc)] - 1, a] - val) < 1e-9):
                        el.append(e + 1)
                        sd.append(s + 1)
            out[axes[a] + tag] = (el, sd)
    return out


QUAD_SIDES = [(0, 1), (1, 2), (2, 3), (3, 0)]
TRI_SIDES = [(0, 1), (1, 2), (2, 0)]
HEX_SIDES = [(0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (0, 4, 7, 3), (0, 3, 2, 1), (4, 5, 6, 7)]
TET_SIDES = [(0, 1, 3), (1, 2, 3), (0, 3, 2), (0, 2, 1)]
# library vertex i = Exodus node ORDER[i]; Exodus node j = library vertex INV[j]
ORDER = {"QUAD4": [0, 1, 2, 3], "TRI3": [0, 1, 2], "HEX8": [0, 3, 2, 1, 4, 5, 6, 7],
         "TET4": [0, 2, 1, 3]}


def to_exodus(cells_lib, elem_type):
    """1-based Exodus connectivity from 0-based library-order cells."""
    order = ORDER[elem_type]
    out = np.zeros_like(cells_lib)
    for i, j in enumerate(order):
        out[:, j] = cells_lib[:, i]
    return out + 1
