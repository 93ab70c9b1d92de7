"""Elastic2D oracle (Elastic2D.cpp:29-127) on CPU: traction-free eigenmodes
with C13 = 0, whose frequencies pick out C11 (x mode) and C33 (y mode) and
so check the stress convention; energy stays bounded; moment-tensor and
force sources inject what their definitions say."""
import numpy as np
import pytest

from oracle import pyoracle as po
from salvus_b200 import configs, meshgen


def homogeneous(nel=8, order=4, L=1.0e4, rho=2000.0, c11=3.0e10, c33=2.0e10, c55=1.0e10,
                jitter=0.0, seed=1):
    V, C = meshgen.structured_quad(nel, nel, L, L)
    if jitter > 0:
        h = L / nel
        rng = np.random.default_rng(seed)
        inner = np.all((V > 0.5 * h) & (V < L - 0.5 * h), axis=1)
        V = V.copy()
        V[inner] += rng.uniform(-jitter * h, jitter * h, size=(inner.sum(), 2))
    vals = (rho, c11, 0.0, c33, c55)  # C13 = 0: the cos modes are traction-free
    par = np.stack([np.full((len(C), 4), v) for v in vals])
    return po.Problem(po.QUAD, order, po.ELASTIC2D, V, C, par), L, rho, c11, c33


@pytest.mark.parametrize("axis,jitter", [(0, 0.0), (1, 0.0), (0, 0.2)])
def test_free_eigenmode(axis, jitter):
    p, L, rho, c11, c33 = homogeneous(jitter=jitter)
    assert p.c == 2
    X = p.coords()
    u0 = np.zeros((p.G, 2))
    u0[:, axis] = np.cos(np.pi * X[:, axis] / L)
    omega = np.pi / L * np.sqrt((c11 if axis == 0 else c33) / rho)
    dt = 0.4 * 2.0 / np.sqrt(p.max_eigenvalue(300))
    p.set_field("u", u0)
    e0 = p.energy()
    n = int(round(1.3 * np.pi / omega / dt))
    p.run(n, dt)
    u = p.get_field("u")
    exact = u0 * np.cos(omega * n * dt)
    tol = 0.6 * omega * dt + (2e-3 if jitter else 1e-4)
    assert np.abs(u - exact).max() < tol
    assert abs(p.energy() - e0) / e0 < 0.05


def _nodal_force(cfg, src, kind):
    p = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                   configs.oracle_params(cfg))
    comp = src["moment_tensor"] if kind == 1 else src["direction"]
    p.add_source(src["location"], src["center_freq"], src["time_delay"], src["amplitude"], comp,
                 kind=kind)
    # u = 0: a = M^-1 f at the Ricker peak t = delay (stf = amplitude)
    f = p.acceleration(src["time_delay"]) / p.inverse_mass()[:, None]
    return f, p.coords()


def test_force_source_integrates_to_amplitude():
    cfg = configs.elastic_2d(nel=10, order=3, n_receivers=5)
    src = cfg["sources"][1]
    f, _ = _nodal_force(cfg, src, 0)
    amp = src["amplitude"]
    assert abs(f[:, 0].sum()) < 1e-9 * amp
    assert abs(f[:, 1].sum() - amp) < 1e-9 * amp


def test_moment_tensor_source_moments():
    # f_{i,a} = sum_b M_ab dphi_i/dx_b: no net force, first moment
    # sum_i x_{i,c} f_{i,a} = M_ac (the bilinear map lies in the GLL basis)
    cfg = configs.elastic_2d(nel=10, order=3, n_receivers=5, jitter=0.2)
    src = cfg["sources"][0]
    f, X = _nodal_force(cfg, src, 1)
    amp = src["amplitude"]
    mxx, myy, mxy = src["moment_tensor"]
    M = amp * np.array([[mxx, mxy], [mxy, myy]])
    assert np.abs(f.sum(axis=0)).max() < 1e-6 * np.abs(M).max()
    first = np.einsum("ic,ia->ac", X, f)
    assert np.abs(first - M).max() < 1e-9 * np.abs(M).max()
