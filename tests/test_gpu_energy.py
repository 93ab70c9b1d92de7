"""GPU energy 1/2 v^T M v + 1/2 u^T K u (FP64 compensated sums) against the
oracle's FP64 energy on the same state, for acoustic quads, elastic hexes and
fluid-solid quads, in FP64 and FP32; run-to-run bitwise; bounded over a
source-free standing-wave run."""
import numpy as np
import pytest

from oracle import pyoracle as po
from salvus_b200 import configs, core

from test_gpu_parity import build_pair, oracle_dt

pytestmark = pytest.mark.gpu


def _state(mesh, orc, idx, c, seed):
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((mesh.n_nodes, c))
    v = rng.standard_normal((mesh.n_nodes, c))
    inv = np.argsort(idx)
    orc.set_field("u", u[inv])
    orc.set_field("v", v[inv])
    return u, v


@pytest.mark.parametrize("kind", ["quad", "hex", "coupled"])
@pytest.mark.parametrize("precision,tol", [(core.FP64, 1e-11), (core.FP32, 2e-6)])
def test_energy_matches_oracle(kind, precision, tol):
    cfg = {"quad": lambda: configs.ricker_2d(nel=16, order=4),
           "hex": lambda: configs.elastic_hex(nel=4, order=4, n_receivers=2),
           "coupled": lambda: configs.coupled_2d(nel=12, order=4)}[kind]()
    cfg.pop("sources", None)
    mesh, prob, orc, idx = build_pair(cfg, precision, 1e-3)
    u, v = _state(mesh, orc, idx, prob.c, 3)
    prob.set_field("u", u)
    prob.set_field("v", v)
    k, e = prob.energy()
    ref = orc.energy()
    assert abs((k + e) - ref) <= tol * abs(ref)
    assert (k, e) == prob.energy()  # same bits on a second call


def test_energy_bounded_standing_wave_fp32():
    cfg = configs.standing_wave_2d(nel=20, order=4)
    dt = oracle_dt(cfg)
    mesh, prob, orc, idx = build_pair(cfg, core.FP32, dt)
    X = mesh.node_coords()
    prob.set_field("u", configs.standing_wave_initial(X, cfg["L"]))
    e0 = sum(prob.energy())
    es = []
    for _ in range(10):
        prob.run(100)
        es.append(sum(prob.energy()))
    # Newmark without sources: the energy oscillates within O(dt^2), no drift
    assert max(abs(e - e0) for e in es) < 0.05 * e0
