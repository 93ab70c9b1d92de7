"""Homogeneous Dirichlet boundaries (HomogeneousDirichlet.cpp): stiffness rows
of boundary points zeroed, sources kept.  GPU vs the FP64 oracle with the same
boundary nodes (FP64 rel-L2 <= 1e-10, FP32 <= 1e-4), and the Dirichlet
eigenmode sin(pi x/L) sin(pi y/L) against its analytic solution.  The 3-D
cases move their receivers below the clamped top surface and keep one on it,
whose trace must stay exactly zero."""
import numpy as np
import pytest

from salvus_b200 import configs, core

import simplex_cases as sc
from test_gpu_parity import build_pair, oracle_dt, rel_l2

pytestmark = pytest.mark.gpu


def sink_receivers(cfg):
    """receivers at 70% depth, plus the first one left on the top surface"""
    r = np.asarray(cfg["receivers"], dtype=np.float64)
    inner = r.copy()
    inner[:, 2] = 0.7 * cfg["L"]
    cfg["receivers"] = np.concatenate([r[:1], inner])
    return cfg


def with_dirichlet(mesh, prob, orc, idx):
    b = mesh.boundary_nodes()
    prob.set_dirichlet(b)
    orc.set_dirichlet(idx[b])
    return b


@pytest.mark.parametrize("precision,tol", [(core.FP64, 1e-10), (core.FP32, 1e-4)])
def test_quad_dirichlet_eigenmode(precision, tol):
    cfg = configs.ricker_2d(nel=20, order=4)
    cfg.pop("sources")
    dt = oracle_dt(cfg)
    mesh, prob, orc, idx = build_pair(cfg, precision, dt)
    b = with_dirichlet(mesh, prob, orc, idx)
    X = mesh.node_coords()
    L = cfg["L"]
    u0 = np.sin(np.pi * X[:, 0] / L) * np.sin(np.pi * X[:, 1] / L)
    u0[b] = 0.0  # sin(pi) is not exactly zero in floating point
    prob.set_field("u", u0)
    orc.set_field("u", u0[np.argsort(idx)])
    n = int(round(2 * np.pi / cfg["omega"] / dt))
    prob.run(n)
    s_o = orc.run(n, dt)
    assert rel_l2(prob.seismograms(), s_o) <= tol
    u = prob.get_field("u")[:, 0]
    assert rel_l2(u, orc.get_field("u")[idx, 0]) <= tol
    # boundary stays at rest; the field follows the analytic mode (bound of
    # the free-boundary standing-wave test: first-order Newmark start)
    assert np.abs(u[b]).max() == 0.0
    exact = u0 * np.cos(cfg["omega"] * n * dt)
    assert np.abs(u - exact).max() < 0.6 * cfg["omega"] * dt + 1e-3


@pytest.mark.parametrize("precision,tol", [(core.FP64, 1e-10), (core.FP32, 1e-4)])
def test_hex_elastic_dirichlet_source(precision, tol):
    cfg = sink_receivers(configs.elastic_hex(nel=4, order=3, n_receivers=6, seed=3))
    dt = oracle_dt(cfg)
    mesh, prob, orc, idx = build_pair(cfg, precision, dt)
    with_dirichlet(mesh, prob, orc, idx)
    n = 400
    prob.set_seismogram_capacity(n)
    prob.run(n)
    s_o = orc.run(n, dt)
    s_g = prob.seismograms()
    assert np.abs(s_o[1:]).max() > 0
    assert np.abs(s_g[0]).max() == 0.0
    assert rel_l2(s_g[1:], s_o[1:]) <= tol


def test_tet_acoustic_dirichlet_tensor_cores():
    cfg = sink_receivers(sc.small_tet(core.ACOUSTIC))
    dt = sc.oracle_dt(cfg)
    mesh, prob, orc, idx = sc.build_pair(cfg, core.FP32, dt)
    with_dirichlet(mesh, prob, orc, idx)
    n = 300
    prob.set_seismogram_capacity(n)
    prob.run(n)
    s_o = orc.run(n, dt)
    s_g = prob.seismograms()
    assert np.abs(s_o[1:]).max() > 0
    # P3 simplex basis functions of off-face nodes vanish on the face only to
    # rounding (Vandermonde inverse), unlike the tensor Lagrange factors
    assert np.abs(s_g[0]).max() <= 1e-12 * np.abs(s_g[1:]).max()
    assert sc.rel_l2(s_g[1:], s_o[1:]) <= 1e-4


@pytest.mark.parametrize("precision,tol", [(core.FP64, 1e-10), (core.FP32, 1e-4)])
def test_elastic2d_dirichlet(precision, tol):
    """HomogeneousDirichlet<Elastic2D<TensorQuad<QuadP1>>> (HomogeneousDirichlet.cpp:118-121)"""
    cfg = configs.elastic_2d(nel=12, order=4, n_receivers=6)
    dt = oracle_dt(cfg)
    mesh, prob, orc, idx = build_pair(cfg, precision, dt)
    b = with_dirichlet(mesh, prob, orc, idx)
    n = 600
    prob.set_seismogram_capacity(n)
    prob.run(n)
    s_o = orc.run(n, dt)
    assert np.abs(s_o).max() > 0
    assert rel_l2(prob.seismograms(), s_o) <= tol
    u = prob.get_field("u")
    assert np.abs(u[b]).max() == 0.0
    assert rel_l2(u, orc.get_field("u")[idx]) <= tol
