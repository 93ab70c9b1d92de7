"""Every polynomial order of the tensor-product elements against the FP64
oracle: acoustic quadrilaterals 1-10 and acoustic / elastic hexahedra 1-6, the
orders whose GLL tables the reference generates (Quad/Autogen/order{1..10}_
square.c, Hex/Autogen/order{1..6}_hex.c).  Each case runs a Ricker point
source long enough for the wavelet to reach the receivers; FP64 GPU vs FP64
oracle rel-L2 <= 1e-10 (operation order only), FP32 <= 1e-4."""
import numpy as np
import pytest

from salvus_b200 import configs, core

from test_gpu_parity import TOL32, TOL64, build_pair, oracle_dt, rel_l2

pytestmark = pytest.mark.gpu

_ORACLE = {}


def _case(kind, order):
    if kind == "quad":
        cfg = configs.ricker_2d(nel=8, order=order, n_receivers=6, radius=1.5e3, seed=order)
        horizon = 1.2  # s: wavelet peak 0.6 s + 1.5 km at 4 km/s
    elif kind == "hex":
        cfg = configs.acoustic_hex(nel=3, order=order)
        cfg["sources"] = [dict(location=(4123.0, 5301.0, 4777.0), center_freq=1.0, time_delay=1.2,
                               amplitude=1.0, direction=[1.0])]
        cfg["receivers"] = [(2500.0 + 900 * k, 7000.0 - 600 * k, 3500.0 + 500 * k) for k in range(6)]
        horizon = 2.0
    else:
        cfg = configs.elastic_hex(nel=3, order=order, n_receivers=6, seed=order)
        horizon = 1.0
    return cfg, horizon


def _run(kind, order, precision):
    cfg, horizon = _case(kind, order)
    if (kind, order) not in _ORACLE:
        _ORACLE[(kind, order)] = oracle_dt(cfg)
    dt = _ORACLE[(kind, order)]
    n = int(min(3000, max(200, np.ceil(horizon / dt))))
    mesh, prob, orc, idx = build_pair(cfg, precision, dt)
    prob.set_seismogram_capacity(n)
    prob.run(n)
    s_o = orc.run(n, dt)
    out = (prob.seismograms(), s_o, prob.get_field("u"), orc.get_field("u")[idx])
    prob.close()
    mesh.close()
    return out


@pytest.mark.parametrize("precision,tol", [(core.FP64, TOL64), (core.FP32, TOL32)])
@pytest.mark.parametrize("order", list(range(1, 11)))
def test_acoustic_quad_every_order(order, precision, tol):
    s_g, s_o, u_g, u_o = _run("quad", order, precision)
    assert np.abs(s_o).max() > 0
    assert rel_l2(s_g, s_o) <= tol
    assert rel_l2(u_g, u_o) <= tol


@pytest.mark.parametrize("precision,tol", [(core.FP64, TOL64), (core.FP32, TOL32)])
@pytest.mark.parametrize("kind", ["hex", "elastic_hex"])
@pytest.mark.parametrize("order", list(range(1, 7)))
def test_hexahedra_every_order(order, kind, precision, tol):
    s_g, s_o, u_g, u_o = _run(kind, order, precision)
    assert np.abs(s_o).max() > 0
    assert rel_l2(s_g, s_o) <= tol
    assert rel_l2(u_g, u_o) <= tol
