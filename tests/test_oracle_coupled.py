"""Fluid-solid quadrilateral meshes in the oracle (CPU): element classes reduce
to the single-physics problems, the reference's coupling (ElasticToAcoustic2D /
AcousticToElastic2D with the single summed mass) moves energy across the
interface and stays bounded, each consistency switch K1-K4 changes the
result, and the fully consistent velocity coupling is unstable under the
explicit Newmark step -- the reason the product keeps the reference's form."""
import numpy as np
import pytest

from oracle import pyoracle as po
from salvus_b200 import configs


def problem(cfg, params=None, physics=None, flags=0):
    par = cfg["params"] if params is None else params
    return po.Problem(cfg["shape"], cfg["order"], cfg["physics"] if physics is None else physics,
                      cfg["vertices"], cfg["cells"], par, flags=flags)


def bump(X, x0, y0, r=1000.0):
    return np.exp(-((X[:, 0] - x0) ** 2 + (X[:, 1] - y0) ** 2) / r ** 2)


@pytest.mark.parametrize("kind", ["fluid", "solid"])
def test_single_class_meshes_equal_single_physics(kind):
    cfg = configs.coupled_2d(nel=8, order=3, std=0.0)
    par = cfg["params"].copy()
    par[0][:] = 1.0 if kind == "fluid" else 0.0
    pc = problem(cfg, par)
    if kind == "fluid":
        ps = problem(cfg, par[1:2], po.ACOUSTIC)
        comp = [0]
    else:
        ps = problem(cfg, par[2:7], po.ELASTIC2D)
        comp = [1, 2]
    X = pc.coords()
    u0 = np.zeros((pc.G, 3))
    for k in comp:
        u0[:, k] = bump(X, 4000.0 + 300 * k, 5200.0)
    dt = 0.4 * 2.0 / np.sqrt(ps.max_eigenvalue(200))
    pc.set_field("u", u0)
    ps.set_field("u", u0[:, comp])
    pc.run(150, dt)
    ps.run(150, dt)
    uc = pc.get_field("u")
    assert np.array_equal(uc[:, comp], ps.get_field("u"))
    others = [k for k in range(3) if k not in comp]
    assert np.abs(uc[:, others]).max() == 0.0


def notched(cfg):
    """the interface with a one-element fluid notch into the solid, so that a
    coupled fluid element borders an uncoupled fluid element (K3 acts there;
    on a straight interface the extra fluid-fluid edge terms cancel)"""
    nel = int(round(np.sqrt(len(cfg["cells"]))))
    ctr = cfg["vertices"][cfg["cells"]].mean(axis=1)
    top_solid = np.where(cfg["params"][0][:, 0] == 0.0, ctr[:, 1], -np.inf).max()
    e = int(np.argmin(np.abs(ctr[:, 0] - ctr[:, 0].mean()) + np.abs(ctr[:, 1] - top_solid)))
    par = cfg["params"].copy()
    par[0][e] = 1.0
    par[2][e] = par[2][e + nel]  # fluid density of the element above
    return par


def run_bump(flags, steps=800):
    cfg = configs.coupled_2d(nel=12, order=4, std=0.0)
    p = problem(cfg, notched(cfg), flags=flags)
    X = p.coords()
    u0 = np.zeros((p.G, 3))
    u0[:, 2] = bump(X, 5000.0, cfg["interface_y"] - 800.0)
    dt = 0.4 * 2.0 / np.sqrt(p.max_eigenvalue(300))
    p.set_field("u", u0)
    norms = []
    for _ in range(steps // 100):
        p.run(100, dt)
        norms.append(np.abs(p.get_field("u")).max(axis=0))
    return np.array(norms), p


def test_reference_coupling_transfers_and_stays_bounded():
    norms, _ = run_bump(0)
    assert np.all(np.isfinite(norms))
    assert norms[:, 0].max() > 0          # the fluid field is driven by the solid
    assert norms[:, 1:].max() < 2.0       # the unit solid pulse does not grow


@pytest.mark.parametrize("flag", [po.K1_SPLIT_MASS, po.K2_SOLID_NORMAL, po.K3_INTERFACE_EDGES,
                                  po.K4_FLUID_VP2])
def test_each_consistency_switch_changes_the_result(flag):
    a, _ = run_bump(0, steps=200)
    b, _ = run_bump(flag, steps=200)
    assert not np.allclose(a, b, rtol=1e-9, atol=0)


def test_consistent_velocity_coupling_is_unstable():
    # explicit Newmark with the lagged velocities of a physically scaled
    # (vp^2, normal) coupling: growth by orders of magnitude at the dt that is
    # stable for either medium alone
    norms, _ = run_bump(po.COUPLING_CONSISTENT)
    assert not np.all(np.isfinite(norms)) or norms[-1].max() > 1e3
