"""Bounded device waits, exercised: the tensor-core tetrahedron / triangle
kernels' worker warps are made to wait first on a barrier that nothing
arrives on (salvus_problem_hold_device_waits) under a short wait limit, and
a one-cycle limit makes the member barriers of the partitioned group step
give up.  The kernels
record the wait's code, return cleanly (the MMA issuer drains its own MMAs
under the default bound before tensor memory is freed) and the host reports
SALVUS_E_TIMEOUT.  After the status is cleared and the default limit is
restored, the same problem (group) runs normally and reproduces a fresh
run bitwise.  No GPU is faulted: every wait here is bounded and ends.
"""
import numpy as np
import pytest

from salvus_b200 import configs, core

pytestmark = pytest.mark.gpu


def mesh_of(cfg):
    return core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"])


def smooth_field(mesh, seed):
    x = mesh.node_coords()
    k = np.random.default_rng(seed).uniform(1.0, 3.0, size=(mesh.n_components, mesh.dim))
    L = x.max(axis=0) - x.min(axis=0)
    return np.stack([np.prod(np.cos(np.pi * k[c] * x / L), axis=1)
                     for c in range(mesh.n_components)], axis=1)


def start(p, u0):
    zero = np.zeros_like(u0)
    p.set_field("u", u0)
    for f in ("v", "a", "a_"):
        p.set_field(f, zero)


@pytest.mark.parametrize("which", ["tet_elastic", "tet_acoustic", "tri_tc"])
def test_tensor_core_wait_gives_up_and_recovers(which, monkeypatch):
    if which == "tri_tc":
        monkeypatch.setenv("SALVUS_TRI_KERNEL", "tc")
        cfg = configs.simplex_tri(nx=24, ny=12, n_receivers=2)
    else:
        phys = core.ELASTIC3D if which == "tet_elastic" else core.ACOUSTIC
        cfg = configs.simplex_tet(n=4, physics=phys, n_receivers=2)
    mesh = mesh_of(cfg)
    dt = 0.2 * mesh.critical_dt(iterations=60)
    u0 = 1e-3 * smooth_field(mesh, 1)
    ref = core.Problem(mesh, core.FP32, dt=dt)
    start(ref, u0)
    ref.run(40, core.RUN_GRAPH)
    ref.status()
    p = core.Problem(mesh, core.FP32, dt=dt)
    # the workers first wait on a barrier nothing arrives on: every launch
    # runs out of a ~2 ms wait limit and takes the timeout path
    p.set_wait_limit(1 << 22)
    p.hold_device_waits(True)
    start(p, u0)
    p.run(40, core.RUN_GRAPH)
    with pytest.raises(core.SalvusError) as e:
        p.status(clear=True)
    assert e.value.code == core.E_TIMEOUT
    assert "code 1" in str(e.value)  # wait codes 1000-1199
    p.status()  # cleared
    p.hold_device_waits(False)
    p.set_wait_limit(0)
    start(p, u0)
    p.run(40, core.RUN_GRAPH)
    p.status()
    for f in ("u", "v", "a_"):
        assert np.array_equal(p.get_field(f), ref.get_field(f))


def test_partitioned_group_wait_gives_up_and_recovers(monkeypatch):
    monkeypatch.setenv("SALVUS_GROUP_STEP", "partitioned")
    cfgs = [configs.ricker_2d(nel=40 + 8 * k, order=4, n_receivers=3, seed=k) for k in range(3)]
    meshes = [mesh_of(c) for c in cfgs]
    u0 = [1e-3 * smooth_field(m, k) for k, m in enumerate(meshes)]

    dt = 0.4 * min(m.critical_dt(iterations=60) for m in meshes)

    def members():
        ps = [core.Problem(m, core.FP32, dt=dt) for m in meshes]
        for p, u in zip(ps, u0):
            start(p, u)
        return ps

    ref = members()
    g0 = core.Group(ref)
    g0.run(64)
    g0.synchronize()
    ps = members()
    g = core.Group(ps)
    g.set_wait_limit(1)
    g.run(64)
    with pytest.raises(core.SalvusError) as e:
        g.synchronize()
    assert e.value.code == core.E_TIMEOUT
    g.clear_status()
    g.set_wait_limit(0)
    for p, u in zip(ps, u0):
        start(p, u)
    g.run(64)
    g.synchronize()
    for p, q in zip(ps, ref):
        assert np.array_equal(p.get_field("u"), q.get_field("u"))
    g.close()
    g0.close()
