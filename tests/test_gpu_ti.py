"""Transversely isotropic Elastic3D on the GPU against the FP64 oracle.

The reference builds its elastic constants from six per-vertex parameters,
RHO VPV VPH VSV VSH ETA (Elastic3D.cpp:33-54), and applies all nine of them
in computeStress (Elastic3D.cpp:106-118).  Meshes created with
SALVUS_MESH_ELASTIC_TI take those six parameters; a model that is not
isotropic runs five-constant records in the hexahedron kernels (FP32 column
kernel, FP64 / FP32 classic kernel) and the CUDA-core tetrahedron kernel.

Tolerances: FP64 <= 1e-10, FP32 <= 1e-4 rel-L2 on seismograms and fields.
A six-parameter model that happens to be isotropic must give bitwise the
result of the three-parameter form (the isotropic kernels are kept).
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from salvus_b200 import configs, core

pytestmark = pytest.mark.gpu

TOL64, TOL32 = 1e-10, 1e-4


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def oracle_of(cfg):
    return po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                      configs.oracle_params(cfg))


def pair(cfg, precision, dt):
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"])
    prob = core.Problem(mesh, precision, dt=dt)
    orc = oracle_of(cfg)
    for s in cfg["sources"]:
        prob.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                        moment_tensor=s["moment_tensor"])
        orc.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                       s["moment_tensor"], kind=1)
    for r in cfg["receivers"]:
        prob.add_receiver(r)
        orc.add_receiver(r)
    scale = cfg["L"]
    key = lambda x: [tuple(k) for k in np.round(x / scale * 1e7).astype(np.int64)]
    ko = {k: i for i, k in enumerate(key(orc.coords()))}
    idx = np.array([ko[k] for k in key(mesh.node_coords())])
    return mesh, prob, orc, idx


@pytest.fixture(scope="module")
def hex_ti():
    cfg = configs.elastic_hex(nel=5, order=4, n_receivers=10, anisotropy=configs.VTI)
    cfg["dt"] = 0.4 * 2.0 / np.sqrt(oracle_of(cfg).max_eigenvalue(200))
    return cfg


@pytest.mark.parametrize("precision,tol", [(core.FP64, TOL64), (core.FP32, TOL32)])
def test_hex_ti_seismograms_and_field(hex_ti, precision, tol):
    mesh, prob, orc, idx = pair(hex_ti, precision, hex_ti["dt"])
    n = 400
    prob.run(n, core.RUN_GRAPH)
    s_o = orc.run(n, hex_ti["dt"])
    assert np.abs(s_o).max() > 0
    assert rel_l2(prob.seismograms(), s_o) <= tol
    assert rel_l2(prob.get_field("u"), orc.get_field("u")[idx]) <= tol


def test_hex_ti_differs_from_isotropic(hex_ti):
    """The anisotropy is large enough to matter: the isotropic model with
    the vertical velocities gives seismograms several percent away."""
    iso = dict(hex_ti)
    p = hex_ti["params"]
    iso["params"] = np.stack([p[0], p[1], p[3]])
    _, a, _, _ = pair(hex_ti, core.FP64, hex_ti["dt"])
    _, b, _, _ = pair(iso, core.FP64, hex_ti["dt"])
    a.run(300)
    b.run(300)
    assert rel_l2(a.seismograms(), b.seismograms()) > 1e-2


@pytest.mark.parametrize("order", [1, 2, 3, 5, 6])
@pytest.mark.parametrize("precision,tol", [(core.FP64, 1e-12), (core.FP32, 4e-6)])
def test_hex_ti_stiffness_action_every_order(order, precision, tol):
    """One assembly without sources: a = -K u against the oracle's -K u."""
    cfg = configs.elastic_hex(nel=3, order=order, n_receivers=2, anisotropy=configs.VTI)
    cfg["sources"] = []
    mesh, prob, orc, idx = pair(cfg, precision, 1e-3)
    rng = np.random.default_rng(order)
    u = rng.standard_normal((mesh.n_nodes, 3))
    prob.set_field("u", u)
    prob.assembleIntoGlobalDof()
    orc_u = np.empty_like(u)
    orc_u[idx] = u
    assert rel_l2(prob.get_field("a"), orc.apply_stiffness(orc_u)[idx]) <= tol


def test_hex_ti_classic_kernel(hex_ti, monkeypatch):
    monkeypatch.setenv("SALVUS_HEX_KERNEL", "classic")
    mesh, prob, orc, idx = pair(hex_ti, core.FP32, hex_ti["dt"])
    prob.run(300)
    assert rel_l2(prob.seismograms(), orc.run(300, hex_ti["dt"])) <= TOL32


@pytest.mark.parametrize("precision", [core.FP32, core.FP64])
def test_isotropic_six_parameter_model_is_the_three_parameter_one(precision):
    cfg = configs.elastic_hex(nel=4, order=4, n_receivers=4)
    rho, vp, vs = cfg["params"]
    six = dict(cfg)
    six["params"] = np.stack([rho, vp, vp, vs, vs, np.ones_like(rho)])
    out = []
    for c in (cfg, six):
        mesh = core.Mesh(c["shape"], c["order"], c["physics"], c["vertices"], c["cells"],
                         c["params"])
        p = core.Problem(mesh, precision, dt=1e-3)
        s = c["sources"][0]
        p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                     moment_tensor=s["moment_tensor"])
        for r in c["receivers"]:
            p.add_receiver(r)
        p.run(100, core.RUN_GRAPH)
        out.append((p.seismograms(), p.get_field("u")))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("precision,tol", [(core.FP64, TOL64), (core.FP32, TOL32)])
def test_tet_ti_seismograms(precision, tol):
    cfg = configs.simplex_tet(n=3, physics=core.ELASTIC3D, n_receivers=5, anisotropy=configs.VTI)
    dt = 0.4 * 2.0 / np.sqrt(oracle_of(cfg).max_eigenvalue(300))
    mesh, prob, orc, idx = pair(cfg, precision, dt)
    n = 300
    prob.run(n, core.RUN_GRAPH)
    s_o = orc.run(n, dt)
    assert np.abs(s_o).max() > 0
    assert rel_l2(prob.seismograms(), s_o) <= tol
    assert rel_l2(prob.get_field("u"), orc.get_field("u")[idx]) <= tol
