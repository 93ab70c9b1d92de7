"""GPU parity for meshes of fluid and solid quadrilaterals (Scalar and
Elastic2D elements coupled by the ElasticToAcoustic2D / AcousticToElastic2D
surface integrals, fields [u, ux, uy]) against the FP64 oracle's restatement
of the reference's coupling: FP64 rel-L2 <= 1e-10, FP32 <= 1e-4, on an
interface with a fluid notch, with Dirichlet boundaries, and single-class
meshes bitwise equal to the single-physics problems."""
import numpy as np
import pytest

from salvus_b200 import configs, core

from test_gpu_parity import build_pair, oracle_dt, rel_l2
from test_oracle_coupled import notched

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg():
    c = configs.coupled_2d(nel=24, order=4, n_receivers=12)
    c["params"] = notched(c)
    c["dt"] = oracle_dt(c)
    return c


@pytest.mark.parametrize("precision,tol", [(core.FP64, 1e-10), (core.FP32, 1e-4)])
def test_coupled_sources_receivers(cfg, precision, tol):
    mesh, prob, orc, idx = build_pair(cfg, precision, cfg["dt"])
    assert prob.c == 3
    n = 1200
    prob.set_seismogram_capacity(n)
    prob.run(n)
    s_o = orc.run(n, cfg["dt"])
    s_g = prob.seismograms()
    assert s_g.shape == (12, 3, n)
    # both media carry signal: fluid u and solid ux, uy
    assert np.abs(s_o[:, 0]).max() > 0 and np.abs(s_o[:, 1:]).max() > 0
    assert rel_l2(s_g, s_o) <= tol
    u_o = orc.get_field("u")[idx]
    for k in range(3):
        assert rel_l2(prob.get_field("u")[:, k], u_o[:, k]) <= tol


@pytest.mark.parametrize("precision,tol", [(core.FP64, 1e-10), (core.FP32, 1e-4)])
def test_coupled_dirichlet(cfg, precision, tol):
    mesh, prob, orc, idx = build_pair(cfg, precision, cfg["dt"])
    b = mesh.boundary_nodes()
    prob.set_dirichlet(b)
    orc.set_dirichlet(idx[b])
    n = 600
    prob.set_seismogram_capacity(n)
    prob.run(n)
    s_o = orc.run(n, cfg["dt"])
    assert rel_l2(prob.seismograms(), s_o) <= tol
    assert np.abs(prob.get_field("u")[b]).max() == 0.0


@pytest.mark.parametrize("kind", ["fluid", "solid"])
def test_single_class_mesh_equals_single_physics(kind):
    c = configs.coupled_2d(nel=16, order=4)
    par = c["params"].copy()
    par[0][:] = 1.0 if kind == "fluid" else 0.0
    phys, sub, comp = ((core.ACOUSTIC, par[1:2], [0]) if kind == "fluid"
                       else (core.ELASTIC2D, par[2:7], [1, 2]))
    m3 = core.Mesh(c["shape"], c["order"], c["physics"], c["vertices"], c["cells"], par)
    m1 = core.Mesh(c["shape"], c["order"], phys, c["vertices"], c["cells"], sub)
    dt = 0.4 * m1.critical_dt(iterations=60)
    p3, p1 = core.Problem(m3, core.FP32, dt=dt), core.Problem(m1, core.FP32, dt=dt)
    X = m3.node_coords()
    u0 = np.zeros((len(X), 3))
    for k in comp:
        u0[:, k] = np.exp(-((X[:, 0] - 4000 - 300 * k) ** 2 + (X[:, 1] - 5200) ** 2) / 1e6)
    p3.set_field("u", u0)
    p1.set_field("u", u0[:, comp])
    p3.run(200)
    p1.run(200)
    assert np.array_equal(p3.get_field("u")[:, comp], p1.get_field("u"))


def test_coupled_source_kinds(cfg):
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"])
    p = core.Problem(mesh, core.FP32, dt=cfg["dt"])
    fluid_pt = cfg["sources"][1]["location"]
    with pytest.raises(core.SalvusError):
        p.add_source(fluid_pt, 2.0, 0.6, 1.0, moment_tensor=[1.0, 1.0, 0.0])
    with pytest.raises(core.SalvusError):
        core.Problem(mesh, core.FP32, dt=cfg["dt"], n_shots=4)
