"""Shot-batched problems (many Ricker shots on one mesh, one launch sequence
per step): each shot's seismograms must match the FP64 oracle run for that
shot alone (FP32 tolerance 1e-4) and the single-shot GPU path (1e-5)."""
import numpy as np
import pytest

from oracle import pyoracle as po
from salvus_b200 import configs, core

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


@pytest.fixture(scope="module")
def setup():
    cfg = configs.batched_quad(nel=24, order=4, n_shots=40, n_receivers=8, seed=5)
    o = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                   cfg["params"])
    dt = 0.4 * 2.0 / np.sqrt(o.max_eigenvalue(200))
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"])
    return cfg, dt, mesh


def batched(cfg, dt, mesh, nsteps, mode=core.RUN_GRAPH):
    S = len(cfg["sources"])
    p = core.Problem(mesh, core.FP32, dt=dt, n_shots=S)
    for s in cfg["sources"]:
        p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                     direction=s["direction"], shot=s["shot"])
    for r in cfg["receivers"]:
        p.add_receiver(r)
    p.run(nsteps, mode)
    return p


def test_batched_matches_oracle_per_shot(setup):
    cfg, dt, mesh = setup
    n = 600
    p = batched(cfg, dt, mesh, n)
    seis = p.seismograms()
    assert seis.shape == (40, 8, 1, n)
    for k in [0, 7, 23, 39]:
        s = cfg["sources"][k]
        o = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                       cfg["params"])
        o.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"], s["direction"])
        for r in cfg["receivers"]:
            o.add_receiver(r)
        ref = o.run(n, dt)
        assert np.abs(ref).max() > 0
        assert rel_l2(seis[k], ref) <= 1e-4, k


def test_batched_matches_single_shot_gpu(setup):
    cfg, dt, mesh = setup
    n = 400
    seis = batched(cfg, dt, mesh, n).seismograms()
    for k in [3, 31]:
        s = cfg["sources"][k]
        q = core.Problem(mesh, core.FP32, dt=dt)
        q.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                     direction=s["direction"])
        for r in cfg["receivers"]:
            q.add_receiver(r)
        q.run(n)
        assert rel_l2(seis[k], q.seismograms()) <= 1e-5


def test_batched_graph_equals_plain_and_is_deterministic(setup):
    cfg, dt, mesh = setup
    a = batched(cfg, dt, mesh, 100, core.RUN_GRAPH).seismograms()
    b = batched(cfg, dt, mesh, 100, core.RUN_PLAIN).seismograms()
    c = batched(cfg, dt, mesh, 100, core.RUN_GRAPH).seismograms()
    assert np.array_equal(a, b)
    assert np.array_equal(a, c)


def test_batched_fields_and_tuning(setup):
    cfg, dt, mesh = setup
    p = core.Problem(mesh, core.FP32, dt=dt, n_shots=5)
    sc, epc, gsc, gn = p.autotune()
    assert sc in (32, 64, 128, 256) and epc >= 1 and gsc >= 32 and gn >= 1
    X = mesh.node_coords()
    u0 = configs.standing_wave_initial(X, cfg["L"])
    p.set_field("u", u0, shot=2)
    assert np.allclose(p.get_field("u", shot=2)[:, 0], u0, rtol=1e-6, atol=1e-7)
    assert np.all(p.get_field("u", shot=1) == 0)
    with pytest.raises(core.SalvusError):
        p.get_field("u", shot=5)
    with pytest.raises(core.SalvusError):
        p.assembleIntoGlobalDof()
    # free oscillation of shot 2 only; the other shots stay at rest
    p.run(50)
    assert np.abs(p.get_field("u", shot=2)).max() > 0.5
    assert np.all(p.get_field("u", shot=4) == 0)


@pytest.mark.parametrize("order", [2, 4, 6])
def test_fused_batched_step_equals_unfused(order, monkeypatch):
    """The fused batched step (interior nodes advanced in the stiffness
    kernel, edge nodes gathered) gives bitwise the wavefields and
    seismograms of the unfused sequence (stiffness, sources, gather)."""
    cfg = configs.batched_quad(nel=16, order=order, n_shots=40, n_receivers=6, seed=7)
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"])
    dt = 0.4 * mesh.critical_dt(iterations=100)
    a = batched(cfg, dt, mesh, 120)
    monkeypatch.setenv("SALVUS_BATCH_STEP", "unfused")
    b = batched(cfg, dt, mesh, 120)
    assert np.abs(a.seismograms()).max() > 0
    assert np.array_equal(a.seismograms(), b.seismograms())
    for shot in (0, 17, 39):
        assert np.array_equal(a.get_field("u", shot=shot), b.get_field("u", shot=shot))
        assert np.array_equal(a.get_field("v", shot=shot), b.get_field("v", shot=shot))
