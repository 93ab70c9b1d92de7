"""CPU-only checks of the C-ABI library: it loads, exports every entry point
declared in include/*.h, and its host-side mesh flattening (topological GLL
numbering, Mesh::setupGlobalDof semantics) agrees with the oracle's
independent coordinate-keyed numbering."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import pyoracle as po
from salvus_b200 import configs, core, meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names.update(re.findall(r"\b(salvus_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 25
    L = ctypes.CDLL(core.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the ctypes signature table covers the header
    from salvus_b200 import serving
    bound = {n for n, _, _ in core.SIGNATURES} | {n for n, _ in serving.SERVER_SIGNATURES}
    assert set(names) <= bound, sorted(set(names) - bound)


def test_version_string():
    assert b"sm_100a" in core.lib().salvus_version()


def _host_mesh(cfg):
    return core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"], device=-1)


def _match(xa, xb, scale):
    """Index map a -> b by rounded coordinates."""
    key = lambda x: [tuple(r) for r in np.round(x / scale * 1e6).astype(np.int64)]
    kb = {k: i for i, k in enumerate(key(xb))}
    return np.array([kb[k] for k in key(xa)])


@pytest.mark.parametrize("order", [1, 2, 4, 7])
def test_quad_numbering_matches_oracle(order):
    cfg = configs.standing_wave_2d(nel=5, order=order)
    m = _host_mesh(cfg)
    assert m.n_nodes == (5 * order + 1) ** 2
    o = po.Problem(cfg["shape"], order, cfg["physics"], cfg["vertices"], cfg["cells"], cfg["params"])
    xm, xo = m.node_coords(), o.coords()
    idx = _match(xm, xo, cfg["L"])
    assert len(set(idx)) == m.n_nodes
    conn = m.connectivity()
    # connectivity: element-local tensor order, nodes at the P1-mapped GLL points
    x, _ = po.gll(order)
    n = order + 1
    V, C = cfg["vertices"], cfg["cells"]
    for e in [0, 7, 24]:
        v = V[C[e]]
        for p in range(n * n):
            r, s = x[p % n], x[p // n]
            w = np.array([(1 - r) * (1 - s), (1 + r) * (1 - s), (1 + r) * (1 + s), (1 - r) * (1 + s)]) / 4
            np.testing.assert_allclose(xm[conn[e, p]], w @ v, atol=1e-9)


@pytest.mark.parametrize("order", [1, 2, 4])
def test_hex_numbering_matches_oracle(order):
    V, C = meshgen.structured_hex(3, 2, 2, 3.0, 2.0, 2.0)
    par = np.full((1, len(C), 8), 1.0)
    cfg = dict(shape=core.HEX, order=order, physics=core.ACOUSTIC, vertices=V, cells=C, params=par)
    m = _host_mesh(cfg)
    assert m.n_nodes == (3 * order + 1) * (2 * order + 1) ** 2
    o = po.Problem(core.HEX, order, core.ACOUSTIC, V, C, par)
    assert o.G == m.n_nodes
    idx = _match(m.node_coords(), o.coords(), 3.0)
    assert len(set(idx)) == m.n_nodes


def test_hex_numbering_rotated_cells():
    # shared faces seen with different local orientations must still match
    V, C = meshgen.structured_hex(2, 2, 1, 2.0, 2.0, 1.0)
    # re-express element 1 with its vertices rotated about t (still right-handed)
    c = C[1].copy()
    C[1] = [c[1], c[2], c[3], c[0], c[7], c[4], c[5], c[6]]
    par = np.full((1, len(C), 8), 1.0)
    cfg = dict(shape=core.HEX, order=4, physics=core.ACOUSTIC, vertices=V, cells=C, params=par)
    m = _host_mesh(cfg)
    assert m.n_nodes == 9 * 9 * 5
    xm = m.node_coords()
    conn = m.connectivity()
    # every element's local node p sits where its own P1 map puts it
    x, _ = po.gll(4)
    signs = np.array([[-1, -1, -1], [-1, 1, -1], [1, 1, -1], [1, -1, -1],
                      [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
    for e in range(len(C)):
        v = V[C[e]]
        for p in range(125):
            ref = np.array([x[p % 5], x[(p // 5) % 5], x[p // 25]])
            w = np.prod(1 + signs * ref, axis=1) / 8
            np.testing.assert_allclose(xm[conn[e, p]], w @ v, atol=1e-9)


def _first_hull_element(shape, V, C, x):
    for e in range(len(C)):
        if po.check_hull(shape, V[C[e]], x) == 1:
            return e
    return -1


@pytest.mark.parametrize("which", ["ring2d", "elastic3d"])
def test_point_location_matches_oracle(which):
    if which == "ring2d":
        cfg = configs.ricker_2d(nel=40, order=4)
        pts = list(cfg["receivers"]) + [s["location"] for s in cfg["sources"]] + [(2500.0, 2500.0)]
    else:
        cfg = configs.elastic_hex(nel=6, order=4, n_receivers=10)
        pts = list(cfg["receivers"]) + [s["location"] for s in cfg["sources"]]
    m = _host_mesh(cfg)
    V, C = cfg["vertices"], cfg["cells"]
    for x in pts:
        e, ref = m.locate(x)
        assert e == _first_hull_element(cfg["shape"], V, C, np.asarray(x, float))
        np.testing.assert_allclose(ref, po.inverse_map(cfg["shape"], V[C[e]], x), atol=1e-6)
        # the product's reference coordinates map back to the point exactly
        d = len(ref)
        signs = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], float) if d == 2 else np.array(
            [[-1, -1, -1], [-1, 1, -1], [1, 1, -1], [1, -1, -1],
             [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
        w = np.prod(1 + signs * ref, axis=1) / 2 ** d
        np.testing.assert_allclose(w @ V[C[e]], x, rtol=1e-12, atol=1e-8)
    with pytest.raises(core.SalvusError):
        m.locate([-1.0] * m.dim)


def test_invalid_meshes_rejected():
    V, C = meshgen.structured_quad(2, 2, 1.0, 1.0)
    par = np.ones((1, len(C), 4))
    bad = C.copy()
    bad[0] = bad[0][::-1]  # left-handed
    with pytest.raises(core.SalvusError):
        core.Mesh(core.QUAD, 4, core.ACOUSTIC, V, bad, par, device=-1)
    bad = C.copy()
    bad[1, 2] = 999
    with pytest.raises(core.SalvusError):
        core.Mesh(core.QUAD, 4, core.ACOUSTIC, V, bad, par, device=-1)
    with pytest.raises(core.SalvusError):
        core.Mesh(core.QUAD, 11, core.ACOUSTIC, V, C, par, device=-1)
    with pytest.raises(core.SalvusError):
        core.Mesh(core.QUAD, 4, core.ELASTIC3D, V, C, np.ones((3, len(C), 4)), device=-1)
    with pytest.raises(core.SalvusError):
        core.Mesh(core.QUAD, 4, core.ACOUSTIC, V, C, par * np.nan, device=-1)
    m = core.Mesh(core.QUAD, 4, core.ACOUSTIC, V, C, par, device=-1)
    with pytest.raises(core.SalvusError):
        core.Problem(m)


def test_invalid_physics_meshes_rejected():
    """2-D elastic and fluid-solid physics need quadrilaterals; the fluid flag
    must be 0 or 1 and the same at all four vertices of an element."""
    V, C = meshgen.structured_quad(3, 3, 3.0, 3.0)
    E = len(C)
    with pytest.raises(core.SalvusError):
        Vh, Ch = meshgen.structured_hex(1, 1, 1, 1.0, 1.0, 1.0)
        core.Mesh(core.HEX, 2, core.ELASTIC2D, Vh, Ch, np.ones((5, 1, 8)), device=-1)
    Vt, Ct = meshgen.delaunay_tri(3, 3, 3.0, 3.0, seed=1)
    with pytest.raises(core.SalvusError):
        core.Mesh(core.TRI, 3, core.COUPLED2D, Vt, Ct, np.ones((7, len(Ct), 3)), device=-1)
    par = np.ones((7, E, 4))
    par[0] = 0.0
    par[0][4] = 1.0
    m = core.Mesh(core.QUAD, 3, core.COUPLED2D, V, C, par, device=-1)  # one fluid element
    assert m.n_components == 3
    m.close()
    half = par.copy()
    half[0][2] = 0.5
    with pytest.raises(core.SalvusError, match="FLUID"):
        core.Mesh(core.QUAD, 3, core.COUPLED2D, V, C, half, device=-1)
    mixed = par.copy()
    mixed[0][3, 1] = 1.0
    with pytest.raises(core.SalvusError, match="FLUID"):
        core.Mesh(core.QUAD, 3, core.COUPLED2D, V, C, mixed, device=-1)
    with pytest.raises(core.SalvusError):
        core.Mesh(core.QUAD, 3, 7, V, C, par, device=-1)


def test_interior_node_lists_on_the_host():
    """The fused steps gather every node except the element-interior ones:
    G - E (N-1)^d for acoustic quads and parallelepiped elastic hexahedra,
    all G otherwise (order 1, distorted or acoustic hexahedra, per-point
    geometry requested)."""
    def layout(cfg, flags=0):
        m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                      cfg["params"], device=-1, flags=flags)
        return m.layout(), m.n_nodes, len(cfg["cells"])

    (aff, gathered), G, E = layout(configs.standing_wave_2d(nel=10, order=4))
    assert not aff and G == 41 * 41 and gathered == G - E * 9
    (aff, gathered), G, E = layout(configs.standing_wave_2d(nel=6, order=1))
    assert gathered == G
    (aff, gathered), G, E = layout(configs.elastic_hex(nel=3, order=4, n_receivers=2))
    assert aff and G == 13 ** 3 and gathered == G - E * 27
    (aff, gathered), G, E = layout(configs.elastic_hex(nel=3, order=4, n_receivers=2),
                                   flags=core.MESH_PER_POINT_GEOMETRY)
    assert not aff and gathered == G
    (aff, gathered), G, E = layout(configs.acoustic_hex(nel=3, order=4))
    assert not aff and gathered == G
    cfg = configs.elastic_hex(nel=3, order=3, n_receivers=2)
    V = cfg["vertices"].copy()
    inner = np.all((V > 1.0) & (V < cfg["L"] - 1.0), axis=1)
    V[inner] += 37.0
    cfg["vertices"] = V
    (aff, gathered), G, E = layout(cfg)
    assert not aff and gathered == G
