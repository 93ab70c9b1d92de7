"""Serving (continuous batching of forward-modelling jobs): each job's
seismograms are bitwise the same alone (a plain Problem) and in the mix; the
scheduler streams samples back while jobs run, honours cancellation and the
device-memory budget."""
import time

import numpy as np
import pytest

from salvus_b200 import configs, core, serving

pytestmark = pytest.mark.gpu

DT = {"quad": 1.5e-3, "hex": 8.0e-4}


def alone(cfg, dt, n):
    m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                  cfg["params"])
    p = core.Problem(m, core.FP32, dt=dt)
    for s in cfg["sources"]:
        if "moment_tensor" in s:
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                         moment_tensor=s["moment_tensor"])
        else:
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                         direction=s["direction"])
    for r in cfg["receivers"]:
        p.add_receiver(r)
    p.set_seismogram_capacity(n + 8)
    p.run(n)
    return p.seismograms()


def test_results_identical_alone_and_in_the_mix():
    stream = configs.serving_stream(10, seed=11, quad_edges=(10, 24), hex_edges=(3, 6),
                                    steps=(60, 200))
    srv = serving.Server(budget_bytes=8 * 10**9, max_running=4, chunk_steps=32)
    jobs = []
    for kind, edge, seed, n, _ in stream:
        cfg = configs.serving_job(kind, edge, seed)
        jobs.append((srv.submit(cfg, DT[kind], n), cfg, kind, n))
    for jid, cfg, kind, n in jobs:
        srv.wait(jid, 300)
        assert srv.poll(jid)[0] == serving.DONE
    for jid, cfg, kind, n in jobs:
        mix = srv.seismograms(jid)
        ref = alone(cfg, DT[kind], n)
        assert mix.shape == ref.shape
        assert np.abs(ref).max() > 0
        assert np.array_equal(mix, ref), (kind, cfg["cells"].shape)
    st = srv.stats()
    assert st["completed"] == 10 and st["failed"] == 0
    assert st["p99_latency_s"] >= st["p50_latency_s"] > 0
    srv.close()


def test_streaming_cancel_and_budget():
    srv = serving.Server(budget_bytes=1 * 10**9, max_running=2, chunk_steps=16)
    big = configs.serving_job("quad", 40, 5)
    jid = srv.submit(big, DT["quad"], 4000)
    # samples stream back while the job runs
    deadline = time.time() + 60
    while srv.poll(jid)[1] < 64 and time.time() < deadline:
        time.sleep(0.01)
    st, done, G = srv.poll(jid)
    assert done >= 64 and G > 0
    early = srv.seismograms(jid, 0, 64)
    srv.cancel(jid)
    srv.wait(jid, 60)
    assert srv.poll(jid)[0] == serving.CANCELLED
    assert np.array_equal(early, alone(big, DT["quad"], 64))
    # a job that can never fit the budget is refused at submit
    huge = configs.serving_job("hex", 40, 6)
    with pytest.raises(core.SalvusError):
        srv.submit(huge, DT["hex"], 10)
    # a job whose source lies outside its mesh fails without disturbing others
    bad = configs.serving_job("quad", 12, 7)
    bad["sources"][0]["location"] = (-5.0, 10.0)
    good = configs.serving_job("quad", 12, 8)
    jb, jg = srv.submit(bad, DT["quad"], 50), srv.submit(good, DT["quad"], 50)
    with pytest.raises(core.SalvusError):
        srv.wait(jb, 60)
    srv.wait(jg, 60)
    assert srv.poll(jb)[0] == serving.FAILED and srv.poll(jg)[0] == serving.DONE
    assert np.array_equal(srv.seismograms(jg), alone(good, DT["quad"], 50))
    srv.close()
