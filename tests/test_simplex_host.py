"""P3 simplices without a GPU: the oracle's and the product's reference
elements against the reference's own sympy-generated tables (golden
fixtures from p3_triangle.c / p3_tetrahedra.c), basis and quadrature
properties, the product's host-side node numbering against the oracle's,
point location, and the oracle's physics on small meshes."""
import itertools
import json
import math
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from salvus_b200 import configs, core, meshgen

import simplex_cases as sc

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "ref_tables.json")))

# The reference tables were produced by numpy.linalg.solve on a Vandermonde
# matrix (condition ~3e2 triangle, ~6e5 tetrahedron), so they carry their own
# rounding: about 1e-13 (triangle) and 1e-12 (tetrahedron) absolute.
CASES = [(po.TRI, core.TRI, "tri_p3", 12, 2e-13), (po.TET, core.TET, "tet_p3", 50, 2e-12)]


def golden(key, P, dim):
    g = GOLD[key]
    x = np.stack([g["rst"[k]] for k in range(dim)], axis=1)
    # out[a*P + b] = d phi_b / d xi (node a)  ->  D[k][i][q]
    D = np.stack([np.array(g[n]).reshape(P, P).T for n in ("dphi_dr", "dphi_ds", "dphi_dt")[:dim]])
    return x, np.array(g["w"]), D


@pytest.mark.parametrize("oshape,pshape,key,P,tol", CASES)
def test_oracle_tables_match_reference(oshape, pshape, key, P, tol):
    x, w, D = po.simplex_tables(oshape)
    gx, gw, gD = golden(key, P, x.shape[1])
    assert np.abs(x - gx).max() <= 1e-15
    assert np.abs(w - gw).max() <= 1e-15
    assert np.abs(D - gD).max() <= tol


@pytest.mark.parametrize("oshape,pshape,key,P,tol", CASES)
def test_product_tables_match_reference_and_oracle(oshape, pshape, key, P, tol):
    x, w, D = core.element_tables(pshape, 3)
    gx, gw, gD = golden(key, P, x.shape[1])
    assert np.abs(x - gx).max() <= 1e-15
    assert np.abs(w - gw).max() <= 1e-15
    assert np.abs(D - gD).max() <= tol
    # the product builds the same interpolant from a different generating set
    assert np.abs(D - po.simplex_tables(oshape)[2]).max() <= tol


def test_product_tensor_tables_match_reference_gll():
    for N in (1, 4, 7):
        x, w, D = core.element_tables(core.QUAD, N)
        g = GOLD["quad"][str(N)]
        n = N + 1
        gx = np.array(g["points"])
        assert np.abs(x[:n, 0] - gx).max() <= 1e-13
        ww = np.outer(g["weights"], g["weights"]).ravel()
        assert np.abs(w - ww).max() <= 1e-13
        # d phi_(j,0) / d r at point (i,0) = l_j'(xi_i) = grad[i][j]
        grad = np.array(g["grad"])
        assert np.abs(D[0][:n, :n].T - grad).max() <= 1e-11


@pytest.mark.parametrize("shape", [po.TRI, po.TET])
def test_basis_properties(shape):
    x, w, D = po.simplex_tables(shape)
    P, d = x.shape
    rng = np.random.default_rng(7)
    for _ in range(5):
        lam = rng.dirichlet(np.ones(d + 1))
        ref = (-1 + 2 * lam[1:]) if shape == po.TRI else lam[1:]
        phi, dphi = po.simplex_basis(shape, ref)
        assert abs(phi.sum() - 1) < 1e-12
        assert np.abs(dphi.sum(axis=0)).max() < 1e-11
        # cubic reproduction: sum_i phi_i(x) p(x_i) = p(x)
        p = lambda y: 1 + 2 * y[..., 0] ** 3 - y[..., 0] * y[..., 1] + 0.5 * y[..., -1] ** 2
        assert abs(phi @ p(x) - p(ref)) < 1e-11
    # Kronecker property at the nodes
    for q in (0, P // 2, P - 1):
        phi, _ = po.simplex_basis(shape, x[q])
        assert np.abs(phi - np.eye(P)[q]).max() < 1e-12
    # derivative rows annihilate constants
    assert np.abs(D.sum(axis=1)).max() < 1e-10


def test_quadrature_exactness():
    # tetrahedron: the 50-point rule integrates polynomials of degree <= 5
    # exactly (weights normalised to sum 1 = 6 x volume)
    x, w, _ = po.simplex_tables(po.TET)
    for deg in range(6):
        for e in itertools.product(range(deg + 1), repeat=3):
            if sum(e) != deg:
                continue
            exact = 6 * math.factorial(e[0]) * math.factorial(e[1]) * math.factorial(e[2]) / \
                math.factorial(deg + 3)
            assert abs(np.sum(w * np.prod(x ** np.array(e), axis=1)) - exact) < 1e-14
    # triangle: the reference's 4-digit node coordinates leave the 12-point
    # rule exact to degree 1 and accurate to ~2e-5 up to degree 5 (weights sum
    # 1 = area / 2 of the (-1,-1) (1,-1) (-1,1) triangle)
    x, w, _ = po.simplex_tables(po.TRI)
    from scipy import integrate
    for deg in range(6):
        for e in itertools.product(range(deg + 1), repeat=2):
            if sum(e) != deg:
                continue
            exact = integrate.dblquad(lambda s, r: r ** e[0] * s ** e[1], -1, 1, lambda r: -1,
                                      lambda r: -r)[0] / 2
            err = abs(np.sum(w * np.prod(x ** np.array(e), axis=1)) - exact)
            assert err < (1e-15 if deg <= 1 else 3e-5)


@pytest.mark.parametrize("which", ["tri", "tet"])
def test_host_numbering_matches_oracle(which):
    cfg = sc.small_tri() if which == "tri" else sc.small_tet(core.ACOUSTIC)
    mesh, _, orc, idx = sc.build_pair(cfg, core.FP64, None, device=-1)
    assert mesh.n_nodes == orc.G
    assert len(set(idx.tolist())) == orc.G  # bijection
    xm = mesh.node_coords()
    assert np.abs(xm - orc.coords()[idx]).max() <= 1e-9 * cfg["L"]
    # connectivity reproduces the P1 map of every reference node
    conn = mesh.connectivity()
    ref_nodes, _, _ = core.element_tables(cfg["shape"], 3)
    V, C = cfg["vertices"], cfg["cells"]
    for e in (0, len(C) // 2, len(C) - 1):
        v = V[C[e]]
        for q in range(conn.shape[1]):
            r = ref_nodes[q]
            if which == "tri":
                lam = [-(r[0] + r[1]) / 2, (r[0] + 1) / 2, (r[1] + 1) / 2]
            else:
                lam = [1 - r.sum(), r[1], r[0], r[2]]
            assert np.abs(xm[conn[e, q]] - np.dot(lam, v)).max() <= 1e-9 * cfg["L"]
    # every element shares its vertex nodes with its neighbours: the number of
    # distinct nodes equals the count from the mesh topology
    P = conn.shape[1]
    nv = C.shape[1]
    nvert = len(np.unique(C))
    edges = set()
    faces = set()
    for c in C:
        for a, b in itertools.combinations(sorted(c), 2):
            edges.add((a, b))
        if nv == 4:
            for f in itertools.combinations(sorted(c), 3):
                faces.add(f)
    expect = nvert + 2 * len(edges) + (6 * len(faces) + 10 * len(C) if nv == 4 else 3 * len(C))
    assert mesh.n_nodes == expect


@pytest.mark.parametrize("which", ["tri", "tet"])
def test_locate_point(which):
    cfg = sc.small_tri() if which == "tri" else sc.small_tet(core.ACOUSTIC)
    mesh = core.Mesh(cfg["shape"], 3, cfg["physics"], cfg["vertices"], cfg["cells"], cfg["params"],
                     device=-1)
    rng = np.random.default_rng(3)
    dim = mesh.dim
    L = np.array([2e4, 1e4] if which == "tri" else [1e4] * 3)
    for _ in range(10):
        x = rng.uniform(0.01, 0.99, size=dim) * L
        e, ref = mesh.locate(x)
        v = cfg["vertices"][cfg["cells"][e]]
        if which == "tri":
            lam = np.array([-(ref[0] + ref[1]) / 2, (ref[0] + 1) / 2, (ref[1] + 1) / 2])
        else:
            lam = np.array([1 - ref.sum(), ref[1], ref[0], ref[2]])
        assert lam.min() >= -1e-12
        assert np.abs(lam @ v - x).max() <= 1e-8 * L.max()
        oe = po.Problem  # oracle locates by the same first-element rule
    with pytest.raises(core.SalvusError):
        mesh.locate(-L * 0.1)


def test_oracle_triangle_standing_wave():
    lx, ly, vp = 2.0e4, 1.0e4, 4000.0
    V, C = meshgen.delaunay_tri(24, 12, lx, ly, seed=5)
    p = po.Problem(po.TRI, 3, po.ACOUSTIC, V, C, np.full((1, len(C), 3), vp))
    xyz = p.coords()
    dt = 0.4 * 2 / np.sqrt(p.max_eigenvalue(300))
    om = np.pi * vp * np.sqrt(1 / lx ** 2 + 1 / ly ** 2)
    u0 = np.cos(np.pi * xyz[:, 0] / lx) * np.cos(np.pi * xyz[:, 1] / ly)
    p.set_field("u", u0[:, None])
    e0 = p.energy()
    n = int(round(2 * np.pi / om / dt))
    p.run(n, dt)
    u = p.get_field("u")[:, 0]
    # the reference's P3 triangle eigenfunction bound is 1.936e-3
    # (test_Scalar_2D.cpp:376) on its own mesh
    assert np.abs(u - u0 * np.cos(om * n * dt)).max() < 1e-4
    assert abs(p.energy() / e0 - 1) < 1e-4


def test_oracle_tet_elastic_energy_and_rigid_motion():
    cfg = sc.small_tet(core.ELASTIC3D)
    p = sc.oracle_problem(cfg)
    # rigid translation and rotation are in the kernel of K
    X = p.coords()
    for u in (np.tile([1.0, -2.0, 0.5], (p.G, 1)),
              np.stack([-X[:, 1], X[:, 0], np.zeros(p.G)], axis=1)):
        p.set_field("u", u)
        a = p.acceleration(0.0)
        assert np.abs(a).max() < 1e-9 * np.abs(u).max()
    rng = np.random.default_rng(1)
    p.set_field("u", rng.standard_normal((p.G, 3)) * 1e-3)
    p.set_field("v", np.zeros((p.G, 3)))
    e0 = p.energy()
    dt = sc.oracle_dt(cfg, 0.3)
    p.run(50, dt)
    assert abs(p.energy() / e0 - 1) < 0.05


@pytest.mark.parametrize("which", ["quad", "hex", "tri", "tet"])
def test_boundary_nodes(which):
    """Outer-boundary nodes: exactly the nodes on the box surface."""
    if which == "quad":
        V, C = meshgen.structured_quad(6, 5, 6e3, 5e3)
        m = core.Mesh(core.QUAD, 4, core.ACOUSTIC, V, C, np.full((1, len(C), 4), 3e3), device=-1)
        L = np.array([6e3, 5e3])
    elif which == "hex":
        V, C = meshgen.structured_hex(3, 4, 2, 3e3, 4e3, 2e3)
        m = core.Mesh(core.HEX, 3, core.ACOUSTIC, V, C, np.full((1, len(C), 8), 3e3), device=-1)
        L = np.array([3e3, 4e3, 2e3])
    elif which == "tri":
        cfg = sc.small_tri()
        m = core.Mesh(core.TRI, 3, core.ACOUSTIC, cfg["vertices"], cfg["cells"], cfg["params"], device=-1)
        L = np.array([2e4, 1e4])
    else:
        cfg = sc.small_tet(core.ACOUSTIC)
        m = core.Mesh(core.TET, 3, core.ACOUSTIC, cfg["vertices"], cfg["cells"], cfg["params"], device=-1)
        L = np.array([1e4] * 3)
    X = m.node_coords()
    tol = 1e-9 * L.max()
    on_box = np.any((np.abs(X) < tol) | (np.abs(X - L) < tol), axis=1)
    b = m.boundary_nodes()
    assert np.array_equal(np.sort(b), np.flatnonzero(on_box))
