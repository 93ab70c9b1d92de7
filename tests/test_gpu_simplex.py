"""GPU parity for the P3 simplices (12-node triangles, 50-node tetrahedra,
acoustic and elastic) through the C ABI, against the FP64 oracle.

Tolerances: FP64 GPU vs FP64 oracle rel-L2 <= 1e-10 (operation order only);
FP32 GPU vs FP64 oracle seismogram rel-L2 <= 1e-4 (the stated FP32 target).
"""
import numpy as np
import pytest

from salvus_b200 import configs, core

import simplex_cases as sc

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-4

CASES = {
    "tri": lambda: sc.small_tri(),
    "tet_acoustic": lambda: sc.small_tet(core.ACOUSTIC),
    "tet_elastic": lambda: sc.small_tet(core.ELASTIC3D),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    cfg = CASES[request.param]()
    cfg["dt"] = sc.oracle_dt(cfg)
    cfg["name"] = request.param
    return cfg


def test_inverse_mass(case):
    mesh, prob, orc, idx = sc.build_pair(case, core.FP64, case["dt"])
    assert sc.rel_l2(mesh.inverse_mass(), orc.inverse_mass()[idx]) <= 1e-13


@pytest.mark.parametrize("precision,tol", [(core.FP64, 1e-12), (core.FP32, 4e-6)])
def test_acceleration(case, precision, tol):
    """a = M^-1 (f - K u) for a random u: one assemble + inverse mass."""
    mesh, prob, orc, idx = sc.build_pair(case, precision, case["dt"])
    c = mesh.n_components
    rng = np.random.default_rng(11)
    u = rng.standard_normal((mesh.n_nodes, c))
    prob.set_field("u", u)
    inv = np.argsort(idx)
    orc.set_field("u", u[inv])
    prob.assembleIntoGlobalDof()
    prob.applyInverseMassMatrix()
    a = prob.get_field("a")
    ao = orc.acceleration(0.0)[idx]
    assert sc.rel_l2(a, ao) <= tol


@pytest.mark.parametrize("precision,tol", [(core.FP64, TOL64), (core.FP32, TOL32)])
def test_seismograms(case, precision, tol):
    mesh, prob, orc, idx = sc.build_pair(case, precision, case["dt"])
    n = 300
    prob.set_seismogram_capacity(n)
    prob.run(n)
    s_g = prob.seismograms()
    s_o = orc.run(n, case["dt"])
    assert np.abs(s_o).max() > 0
    assert sc.rel_l2(s_g, s_o) <= tol
    u_g = prob.get_field("u")
    u_o = orc.get_field("u")[idx]
    assert sc.rel_l2(u_g, u_o) <= tol


def test_graph_equals_plain(case):
    runs = []
    for mode in (core.RUN_PLAIN, core.RUN_GRAPH):
        mesh, prob, orc, idx = sc.build_pair(case, core.FP32, case["dt"])
        prob.set_seismogram_capacity(80)
        prob.run(80, mode)
        runs.append((prob.seismograms(), prob.get_field("u")))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


def test_triangle_standing_wave_fp32():
    """Neumann eigenmode on a Delaunay P3 triangle mesh, one period, FP32."""
    from salvus_b200 import meshgen
    lx, ly, vp = 2.0e4, 1.0e4, 4000.0
    V, C = meshgen.delaunay_tri(32, 16, lx, ly, seed=8)
    mesh = core.Mesh(core.TRI, 3, core.ACOUSTIC, V, C, np.full((1, len(C), 3), vp))
    dt = 0.4 * mesh.critical_dt(300)
    prob = core.Problem(mesh, core.FP32, dt=dt)
    X = mesh.node_coords()
    u0 = np.cos(np.pi * X[:, 0] / lx) * np.cos(np.pi * X[:, 1] / ly)
    prob.set_field("u", u0)
    om = np.pi * vp * np.sqrt(1 / lx ** 2 + 1 / ly ** 2)
    n = int(round(2 * np.pi / om / dt))
    prob.run(n)
    u = prob.get_field("u")[:, 0]
    assert np.abs(u - u0 * np.cos(om * n * dt)).max() < 1e-4


@pytest.mark.parametrize("physics,n", [(core.ACOUSTIC, 15), (core.ELASTIC3D, 12)])
def test_tensor_core_kernel_matches_cuda_cores(physics, n, monkeypatch):
    """FP32 tetrahedra: the tcgen05 kernel (split-TF32 contractions, several
    tiles per CTA at these sizes) against the CUDA-core FP32 kernel, both
    against the FP64 kernel, on one assemble of a random field."""
    cfg = sc.small_tet(physics, n=n)
    out = {}
    for name, kern, prec in (("tc", "tensor", core.FP32), ("cuda", "cuda", core.FP32),
                             ("fp64", "cuda", core.FP64)):
        monkeypatch.setenv("SALVUS_TET_KERNEL", kern)
        mesh = core.Mesh(cfg["shape"], 3, cfg["physics"], cfg["vertices"], cfg["cells"],
                         cfg["params"])
        prob = core.Problem(mesh, prec, dt=1e-3)
        rng = np.random.default_rng(5)
        prob.set_field("u", rng.standard_normal((mesh.n_nodes, mesh.n_components)))
        prob.assembleIntoGlobalDof()
        out[name] = prob.get_field("a")
        prob.close()
        mesh.close()
    # split-TF32 products drop the lo x lo term and round the lo parts to TF32:
    # a few 1e-7 per product, about 1e-6 relative on the assembled residual
    assert sc.rel_l2(out["tc"], out["fp64"]) <= 5e-6
    assert sc.rel_l2(out["cuda"], out["fp64"]) <= 2e-6
    assert sc.rel_l2(out["tc"], out["cuda"]) <= 6e-6


def test_triangle_tensor_core_kernel_matches_cuda_cores(monkeypatch):
    """FP32 triangles: the optional tcgen05 kernel (SALVUS_TRI_KERNEL=tc,
    split-TF32 contractions, several tiles per CTA) against the default
    CUDA-core FP32 kernel, both against the FP64 kernel, on one assemble of a
    random field."""
    cfg = configs.simplex_tri(nx=120, ny=60, n_receivers=4, seed=7)
    out = {}
    for name, kern, prec in (("tc", "tc", core.FP32), ("cuda", "cuda", core.FP32),
                             ("fp64", "cuda", core.FP64)):
        monkeypatch.setenv("SALVUS_TRI_KERNEL", kern)
        mesh = core.Mesh(cfg["shape"], 3, cfg["physics"], cfg["vertices"], cfg["cells"],
                         cfg["params"])
        prob = core.Problem(mesh, prec, dt=1e-3)
        rng = np.random.default_rng(5)
        prob.set_field("u", rng.standard_normal((mesh.n_nodes, 1)))
        prob.assembleIntoGlobalDof()
        out[name] = prob.get_field("a")
        prob.close()
        mesh.close()
    assert sc.rel_l2(out["tc"], out["fp64"]) <= 5e-6
    assert sc.rel_l2(out["cuda"], out["fp64"]) <= 2e-6
    assert sc.rel_l2(out["tc"], out["cuda"]) <= 6e-6
