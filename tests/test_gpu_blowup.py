"""Blow-up detection: a finite check of the displacement field after every 32
steps sets the problem's status word, which salvus_problem_status,
salvus_synchronize, salvus_problem_get_field and salvus_get_seismograms
report as SALVUS_E_NONFINITE (the reference's failures surface as
exceptions caught in main, Main.cpp:70-74).  The failures are made on the
host: a NaN written into u through salvus_problem_set_field, or a time step
far beyond the stability limit.  Nothing here faults the GPU.
"""
import numpy as np
import pytest

from salvus_b200 import configs, core, serving

pytestmark = pytest.mark.gpu


def problem(cfg, precision=core.FP32, dt=1.5e-3):
    m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                  cfg["params"])
    p = core.Problem(m, precision, dt=dt)
    for s in cfg.get("sources", []):
        kw = ({"moment_tensor": s["moment_tensor"]} if "moment_tensor" in s
              else {"direction": s["direction"]})
        p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"], **kw)
    for r in cfg.get("receivers", []):
        p.add_receiver(r)
    return p


@pytest.mark.parametrize("mode", [core.RUN_GRAPH, core.RUN_PLAIN])
@pytest.mark.parametrize("precision", [core.FP32, core.FP64])
def test_nan_injected_on_the_host_is_reported(mode, precision):
    cfg = configs.ricker_2d(nel=12, order=4, n_receivers=4)
    p = problem(cfg, precision)
    u = np.zeros((p.mesh.n_nodes, 1))
    u[p.mesh.n_nodes // 3, 0] = np.nan
    p.set_field("u", u)
    p.run(64, mode)
    with pytest.raises(core.SalvusError) as e:
        p.status()
    assert e.value.code == core.E_NONFINITE
    with pytest.raises(core.SalvusError):
        p.synchronize()
    # cleared, with finite fields the same problem runs normally again
    with pytest.raises(core.SalvusError):
        p.status(clear=True)
    for f in ("u", "v", "a", "a_"):
        p.set_field(f, np.zeros((p.mesh.n_nodes, 1)))
    p.run(64, mode)
    p.status()
    assert np.all(np.isfinite(p.get_field("u")))


def test_unstable_time_step_is_reported():
    cfg = configs.elastic_hex(nel=3, order=4, n_receivers=2)
    m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                  cfg["params"])
    dt = 8.0 * m.critical_dt(iterations=100)
    p = core.Problem(m, core.FP32, dt=dt)
    s = cfg["sources"][0]
    p.add_source(s["location"], s["center_freq"], 0.0, s["amplitude"],
                 moment_tensor=s["moment_tensor"])
    p.run(2048, core.RUN_GRAPH)
    with pytest.raises(core.SalvusError) as e:
        p.status()
    assert e.value.code == core.E_NONFINITE


def test_stable_run_reports_ok():
    cfg = configs.elastic_hex(nel=3, order=4, n_receivers=2)
    p = problem(cfg, dt=1e-3)
    p.run(256, core.RUN_GRAPH)
    p.status()


def test_group_member_blow_up_leaves_the_others_alone():
    cfgs = [configs.ricker_2d(nel=10 + 2 * k, order=4, n_receivers=3, seed=k) for k in range(3)]
    probs = [problem(c) for c in cfgs]
    u = np.zeros((probs[1].mesh.n_nodes, 1))
    u[5, 0] = np.inf
    probs[1].set_field("u", u)
    g = core.Group(probs)
    g.run(64)
    with pytest.raises(core.SalvusError) as e:
        g.synchronize()  # reports the members' status
    assert e.value.code == core.E_NONFINITE
    probs[0].status()
    probs[2].status()
    with pytest.raises(core.SalvusError) as e:
        probs[1].status()
    assert e.value.code == core.E_NONFINITE
    g.close()


def test_serving_fails_the_diverging_job_and_finishes_the_rest():
    srv = serving.Server(budget_bytes=8 * 10**9, max_running=4, chunk_steps=32)
    good = [configs.serving_job("quad", 16 + 4 * k, 40 + k) for k in range(3)]
    bad = configs.serving_job("quad", 20, 77)
    ids = [srv.submit(c, 1.5e-3, 200) for c in good[:2]]
    jb = srv.submit(bad, 0.2, 2000)  # far beyond the stability limit of a 500 m mesh
    ids.append(srv.submit(good[2], 1.5e-3, 200))
    for j in ids:
        srv.wait(j, 300)
    with pytest.raises(core.SalvusError, match="non-finite"):
        srv.wait(jb, 300)  # a failed job's wait returns its error
    st, done, _ = srv.poll(jb)
    assert st == serving.FAILED
    assert b"non-finite" in core.lib().salvus_last_error()
    for j, c in zip(ids, good):
        assert srv.poll(j)[0] == serving.DONE
        ref = problem(c)
        ref.set_seismogram_capacity(208)
        ref.run(200)
        assert np.array_equal(srv.seismograms(j), ref.seismograms())
    srv.close()
