"""GPU parity: the CUDA path (through the C ABI) against the FP64 oracle.

Tolerances: FP64 GPU vs FP64 oracle rel-L2 <= 1e-10 (operation order only);
FP32 GPU vs FP64 oracle seismogram rel-L2 <= 1e-4 (the stated FP32 target).
"""
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from salvus_b200 import configs, core

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL32 = 1e-4


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def build_pair(cfg, precision, dt, flags=0):
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"])
    prob = core.Problem(mesh, precision, dt=dt)
    orc = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     configs.oracle_params(cfg), flags=flags)
    for s in cfg.get("sources", []):
        if "moment_tensor" in s:
            prob.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                            moment_tensor=s["moment_tensor"])
            orc.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                           s["moment_tensor"], kind=1)
        else:
            prob.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                            direction=s["direction"])
            orc.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                           s["direction"])
    for r in cfg.get("receivers", []):
        prob.add_receiver(r)
        orc.add_receiver(r)
    # product node i <-> oracle node idx[i]
    scale = cfg.get("L", 1.0)
    key = lambda x: [tuple(k) for k in np.round(x / scale * 1e7).astype(np.int64)]
    ko = {k: i for i, k in enumerate(key(orc.coords()))}
    idx = np.array([ko[k] for k in key(mesh.node_coords())])
    return mesh, prob, orc, idx


def oracle_dt(cfg, frac=0.4):
    o = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                   configs.oracle_params(cfg))
    return frac * 2.0 / np.sqrt(o.max_eigenvalue(200))


@pytest.fixture(scope="module")
def cfg0():
    cfg = configs.ricker_2d(nel=40, order=4)
    cfg["dt"] = oracle_dt(cfg)
    return cfg


@pytest.mark.parametrize("precision,tol", [(core.FP64, TOL64), (core.FP32, TOL32)])
def test_standing_wave_cfg0a(cfg0, precision, tol):
    cfg = dict(cfg0)
    cfg.pop("sources")
    mesh, prob, orc, idx = build_pair(cfg, precision, cfg0["dt"])
    X = mesh.node_coords()
    u0 = configs.standing_wave_initial(X, cfg["L"])
    prob.set_field("u", u0)
    orc.set_field("u", u0[np.argsort(idx)])
    n = 2000
    prob.run(n)
    s_o = orc.run(n, cfg0["dt"])
    s_g = prob.seismograms()
    assert rel_l2(s_g, s_o) <= tol
    u_g = prob.get_field("u")[:, 0]
    u_o = orc.get_field("u")[idx, 0]
    assert rel_l2(u_g, u_o) <= tol
    exact = u0 * np.cos(cfg["omega"] * n * cfg0["dt"])
    err_max = float(np.abs(u_g - exact).max())
    log_path = os.environ.get("SALVUS_ACCURACY_LOG")
    if log_path:
        with open(log_path, "a") as f:
            f.write(json.dumps(dict(
                workload="standing wave 40x40 quads order 4, 2000 steps",
                precision=["fp32", "fp64"][precision], reference="analytic eigenmode",
                max_abs_error=err_max, rel_l2_error=rel_l2(u_g, exact),
                rel_l2_vs_oracle=rel_l2(u_g, u_o), omega_dt=cfg["omega"] * cfg0["dt"])) + "\n")
    # analytic check with the reference's first-order Newmark start
    assert err_max < 0.6 * cfg["omega"] * cfg0["dt"] + 1e-3


@pytest.mark.parametrize("precision,tol", [(core.FP64, TOL64), (core.FP32, TOL32)])
def test_ricker_receivers_cfg0b(cfg0, precision, tol):
    mesh, prob, orc, idx = build_pair(cfg0, precision, cfg0["dt"])
    n = 2000
    prob.run(n)
    s_o = orc.run(n, cfg0["dt"])
    s_g = prob.seismograms()
    assert s_g.shape == (16, 1, n)
    assert np.abs(s_o).max() > 0
    assert rel_l2(s_g, s_o) <= tol


@pytest.mark.parametrize("precision,tol", [(core.FP64, TOL64), (core.FP32, TOL32)])
def test_acoustic_hex(precision, tol):
    cfg = configs.acoustic_hex(nel=4, order=4)
    cfg["sources"] = [dict(location=(4123.0, 5301.0, 4777.0), center_freq=1.0, time_delay=1.2,
                           amplitude=1.0, direction=[1.0])]
    cfg["receivers"] = [(1000.0 + 700 * k, 8000.0 - 500 * k, 3000.0 + 300 * k) for k in range(8)]
    dt = oracle_dt(cfg)
    mesh, prob, orc, idx = build_pair(cfg, precision, dt)
    X = mesh.node_coords()
    u0 = configs.standing_wave_initial(X, cfg["L"])
    prob.set_field("u", u0)
    orc.set_field("u", u0[np.argsort(idx)])
    n = 300
    prob.run(n)
    s_o = orc.run(n, dt)
    assert rel_l2(prob.seismograms(), s_o) <= tol
    assert rel_l2(prob.get_field("u")[:, 0], orc.get_field("u")[idx, 0]) <= tol


@pytest.fixture(scope="module")
def cfg1_small():
    cfg = configs.elastic_hex(nel=5, order=4, n_receivers=12)
    cfg["dt"] = oracle_dt(cfg)
    return cfg


@pytest.mark.parametrize("precision,tol", [(core.FP64, TOL64), (core.FP32, TOL32)])
def test_elastic_hex_moment_tensor(cfg1_small, precision, tol):
    cfg = cfg1_small
    mesh, prob, orc, idx = build_pair(cfg, precision, cfg["dt"])
    n = 400
    prob.run(n)
    s_o = orc.run(n, cfg["dt"])
    s_g = prob.seismograms()
    assert s_g.shape == (12, 3, n)
    assert np.abs(s_o).max() > 0
    assert rel_l2(s_g, s_o) <= tol
    assert rel_l2(prob.get_field("u"), orc.get_field("u")[idx]) <= tol


def test_elastic_force_source_fp64(cfg1_small):
    cfg = dict(cfg1_small)
    cfg["sources"] = [dict(location=(511.0, 497.0, 523.0), center_freq=1.5, time_delay=0.8,
                           amplitude=1e10, direction=[0.3, -0.5, 0.8])]
    mesh, prob, orc, idx = build_pair(cfg, core.FP64, cfg["dt"])
    prob.run(200)
    s_o = orc.run(200, cfg["dt"])
    assert rel_l2(prob.seismograms(), s_o) <= TOL64


@pytest.mark.parametrize("precision", [core.FP32, core.FP64])
def test_three_call_sequence_equals_fused_step(cfg0, precision):
    """assembleIntoGlobalDof -> applyInverseMassMatrix -> takeTimeStep gives
    bitwise the same wavefield as the fused step and the graph replay."""
    cfgs = [build_pair(cfg0, precision, cfg0["dt"]) for _ in range(3)]
    n = 70
    p_lit, p_fused, p_graph = cfgs[0][1], cfgs[1][1], cfgs[2][1]
    for _ in range(n):
        p_lit.assembleIntoGlobalDof()
        p_lit.applyInverseMassMatrix()
        p_lit.takeTimeStep()
    for _ in range(n):
        p_fused.step()
    p_graph.run(n, core.RUN_GRAPH)
    a, b, c = (p.get_field("u") for p in (p_lit, p_fused, p_graph))
    assert np.array_equal(a, b)
    assert np.array_equal(b, c)
    assert np.array_equal(p_lit.seismograms(), p_graph.seismograms())


def test_run_with_overlapped_receivers_equals_single_steps(cfg1_small):
    """salvus_run samples the receivers of each step on a second stream,
    overlapped with the next step's stiffness launch; the seismograms and
    the wavefield equal those of single salvus_step calls (receivers on the
    problem's own stream), bitwise, in graph and plain runs."""
    probs = [build_pair(cfg1_small, core.FP32, cfg1_small["dt"])[1] for _ in range(3)]
    n = 77
    for _ in range(n):
        probs[0].step()
    probs[1].run(n, core.RUN_GRAPH)
    probs[2].run(n, core.RUN_PLAIN)
    s0 = probs[0].seismograms()
    for q in probs[1:]:
        assert np.array_equal(s0, q.seismograms())
        assert np.array_equal(probs[0].get_field("u"), q.get_field("u"))


def test_deterministic_rerun(cfg1_small):
    outs = []
    for _ in range(2):
        mesh, prob, orc, idx = build_pair(cfg1_small, core.FP32, cfg1_small["dt"])
        prob.run(150)
        outs.append(prob.seismograms())
    assert np.array_equal(outs[0], outs[1])


def test_inverse_mass_matches_oracle(cfg1_small):
    mesh, prob, orc, idx = build_pair(cfg1_small, core.FP64, cfg1_small["dt"])
    np.testing.assert_allclose(mesh.inverse_mass(), orc.inverse_mass()[idx], rtol=1e-13)


def test_gpu_eigenvalue_matches_oracle():
    cfg = configs.standing_wave_2d(nel=8, order=4)
    m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                  cfg["params"])
    o = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                   cfg["params"])
    lg, lo = m.max_eigenvalue(400), o.max_eigenvalue(400)
    assert abs(lg - lo) / lo < 2e-2


def test_errors_are_loud():
    cfg = configs.standing_wave_2d(nel=4, order=4)
    m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                  cfg["params"])
    p = core.Problem(m, core.FP32)
    p.add_receiver((100.0, 100.0))
    with pytest.raises(core.SalvusError):
        p.step()  # no dt
    p.set_dt(1e-3)
    with pytest.raises(core.SalvusError):
        p.add_receiver((-5.0, 1.0))  # outside the mesh
    with pytest.raises(core.SalvusError):
        p.add_source((100.0, 100.0), 1.0, 1.0, moment_tensor=[1, 0, 0, 0, 0, 0])
    p.step()
    with pytest.raises(core.SalvusError):
        p.seismograms(0, 5)  # only one step held


@pytest.mark.parametrize("precision", [core.FP64, core.FP32])
def test_large_field_round_trip(precision):
    """Fields larger than the pinned bounce chunks (4.2 M nodes x 3 x 8 B =
    100 MB) round-trip through set_field / get_field: exactly in FP64, as the
    FP32 rounding of the input in FP32."""
    cfg = configs.elastic_hex(nel=40, order=4, n_receivers=1)
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"])
    prob = core.Problem(mesh, precision, dt=1e-3)
    rng = np.random.default_rng(11)
    x = rng.standard_normal((mesh.n_nodes, 3))
    assert x.nbytes > 64 << 20
    for name in ("u", "v"):
        prob.set_field(name, x)
        y = prob.get_field(name)
        want = x if precision == core.FP64 else x.astype(np.float32).astype(np.float64)
        assert np.array_equal(y, want)
    prob.close()
    mesh.close()
