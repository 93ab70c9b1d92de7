"""Problem groups: meshes of uneven size advanced together (one persistent
work-queue launch per step, one cooperative member-partitioned launch per
step, or one launch per stage) must give every member
exactly (bitwise) the seismograms and fields it gets alone, for acoustic quads and elastic hexahedra, with members that have
no receivers, across graph-replayed chunks and remainders, and over several
group runs."""
import numpy as np
import pytest

from salvus_b200 import configs, core

pytestmark = pytest.mark.gpu

DT = {"quad": 1.5e-3, "hex": 8.0e-4}


def make(kind, edge, seed, receivers=True):
    cfg = configs.serving_job(kind, edge, seed)
    m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                  cfg["params"])
    p = core.Problem(m, core.FP32, dt=DT[kind])
    for s in cfg["sources"]:
        if "moment_tensor" in s:
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                         moment_tensor=s["moment_tensor"])
        else:
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                         direction=s["direction"])
    if receivers:
        for r in cfg["receivers"]:
            p.add_receiver(r)
    p.set_seismogram_capacity(256)
    return m, p


@pytest.mark.parametrize("form", ["persistent", "partitioned", "stages"])
@pytest.mark.parametrize("kind,edges", [("quad", (10, 17, 24, 13)), ("hex", (3, 5, 4))])
def test_group_matches_solo_bitwise(kind, edges, form, monkeypatch):
    """persistent: one work-queue launch per step; partitioned: one cooperative
    launch per step, each member on its own CTAs; stages: one launch per stage."""
    monkeypatch.setenv("SALVUS_GROUP_STEP", form)
    runs = (75, 40)  # two chunks + remainder, then one chunk + remainder
    solo = []
    for k, edge in enumerate(edges):
        m, p = make(kind, edge, 100 + k, receivers=(k != 1))
        p.run(sum(runs), core.RUN_GRAPH)
        solo.append((p.seismograms(), p.get_field("u"), p.get_field("v")))
    keep = [make(kind, edge, 100 + k, receivers=(k != 1)) for k, edge in enumerate(edges)]
    group = core.Group([p for _, p in keep])
    for n in runs:
        group.run(n)
    group.synchronize()
    for k, (_, p) in enumerate(keep):
        s, u, v = solo[k]
        assert p.step_index == sum(runs)
        if k != 1:
            assert np.abs(s).max() > 0
        assert np.array_equal(p.seismograms(), s), (kind, k)
        assert np.array_equal(p.get_field("u"), u), (kind, k)
        assert np.array_equal(p.get_field("v"), v), (kind, k)
    group.close()


def test_group_rejects_mixed_classes():
    _, pq = make("quad", 8, 1)
    _, ph = make("hex", 3, 2)
    with pytest.raises(core.SalvusError):
        core.Group([pq, ph])
    with pytest.raises(core.SalvusError):
        core.Group([pq, pq])
