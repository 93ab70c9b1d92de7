"""Pin the FP64 oracle against the reference's own golden tables and KATs.

Golden vectors: tests/golden/ref_tables.json, generated by
tests/golden/make_golden.py from the reference's sympy-generated Autogen C
sources.  KATs restate the reference's element tests
(src/cxx/Testing/test_TensorQuad.cpp, test_TensorHex.cpp, test_source.cpp,
test_QuadP1.cpp, test_HexP1.cpp) as properties.
"""
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as po

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_tables.json")))

QUAD_REF = np.array([[-1, -1], [1, -1], [1, 1], [-1, 1]], float)
HEX_REF = np.array([[-1, -1, -1], [-1, 1, -1], [1, 1, -1], [1, -1, -1],
                    [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)


@pytest.mark.parametrize("N", range(1, 11))
def test_gll_points_weights_derivative(N):
    # order4_square.c:131-149 tables carry 15 significant digits (quirk Q13)
    g = GOLD["quad"][str(N)]
    x, w = po.gll(N)
    np.testing.assert_allclose(x, g["points"], atol=2e-15)
    np.testing.assert_allclose(w, g["weights"], rtol=1e-13, atol=1e-14)
    D = po.deriv_matrix(N)
    np.testing.assert_allclose(D, np.array(g["grad"]), atol=1e-12 * N * N)


@pytest.mark.parametrize("N", range(1, 11))
def test_quad_lagrange_tables(N):
    g = GOLD["quad"][str(N)]
    n = N + 1
    for smp in g["samples"]:
        r, s = smp["ref"]
        lr, dr = po.lagrange(N, r)
        ls, ds = po.lagrange(N, s)
        # tensor order p = i + n j (r fastest)
        l = np.outer(ls, lr).ravel()
        np.testing.assert_allclose(l, smp["l"], atol=1e-11)
        np.testing.assert_allclose(np.outer(ls, dr).ravel(), smp["dr"], atol=1e-10 * n)
        np.testing.assert_allclose(np.outer(ds, lr).ravel(), smp["ds"], atol=1e-10 * n)


@pytest.mark.parametrize("N", range(1, 7))
def test_hex_lagrange_tables(N):
    g = GOLD["hex"][str(N)]
    n = N + 1
    for smp in g["samples"]:
        r, s, t = smp["ref"]
        lr, dr = po.lagrange(N, r)
        ls, ds = po.lagrange(N, s)
        lt, dt = po.lagrange(N, t)
        tens = lambda a, b, c: np.einsum("k,j,i->kji", c, b, a).ravel()
        np.testing.assert_allclose(tens(lr, ls, lt), smp["l"], atol=1e-11)
        np.testing.assert_allclose(tens(dr, ls, lt), smp["dr"], atol=1e-10 * n)
        np.testing.assert_allclose(tens(lr, ds, lt), smp["ds"], atol=1e-10 * n)
        np.testing.assert_allclose(tens(lr, ls, dt), smp["dt"], atol=1e-10 * n)


def test_ricker_closed_form():
    # test_source.cpp:263-291: fire(t) == A (1 - 2 pi^2 f^2 tau^2) exp(-pi^2 f^2 tau^2)
    for amp, t0, f in [(10, 0.1, 50), (20, 0.01, 60)]:
        for j in range(1000):
            t = j * 1e-3
            fac = np.pi ** 2 * f ** 2 * (t - t0) ** 2
            assert po.ricker(t, f, t0, amp) == pytest.approx(amp * (1 - 2 * fac) * np.exp(-fac),
                                                             rel=1e-14, abs=1e-14)


@pytest.mark.parametrize("N", [1, 3, 4, 7, 10])
def test_quad_element_kats(N):
    # test_TensorQuad.cpp:68-206 on the reference square
    n = N + 1
    P = n * n
    g = GOLD["quad"][str(N)]
    pts = np.array(g["points"])
    for p in range(P):
        u = np.zeros(P)
        u[p] = 1.0
        grad = po.element_gradient(po.QUAD, N, QUAD_REF, u)
        # gradient of basis p at every point p' equals the sympy derivative table
        for q in range(P):
            i, j = q % n, q // n
            lr, dr = po.lagrange(N, pts[i])
            ls, ds = po.lagrange(N, pts[j])
            assert grad[q, 0] == pytest.approx(np.outer(ls, dr).ravel()[p], abs=1e-10 * n * n)
        f = np.zeros((P, 2))
        f[p] = 1.0
        assert po.element_grad_test(po.QUAD, N, QUAD_REF, f).sum() == pytest.approx(0.0, abs=1e-10)
    delta = po.element_delta(po.QUAD, N, QUAD_REF, [0.0, 0.0])
    assert po.element_test(po.QUAD, N, QUAD_REF, delta).sum() == pytest.approx(1.0, rel=1e-12)
    assert po.element_par(po.QUAD, N, np.ones(4)).sum() == pytest.approx(P, rel=1e-13)


@pytest.mark.parametrize("N", [1, 3, 4])
def test_hex_element_kats(N):
    # test_TensorHex.cpp:63-240 on the reference cube
    n = N + 1
    P = n ** 3
    for p in range(0, P, max(1, P // 17)):
        f = np.zeros((P, 3))
        f[p] = 1.0
        assert po.element_grad_test(po.HEX, N, HEX_REF, f).sum() == pytest.approx(0.0, abs=1e-10)
        u = np.zeros(P)
        u[p] = 1.0
        grad = po.element_gradient(po.HEX, N, HEX_REF, u)
        assert np.abs(grad.sum(axis=0)).max() < 1e3  # finite
    delta = po.element_delta(po.HEX, N, HEX_REF, [0.0, 0.0, 0.0])
    assert po.element_test(po.HEX, N, HEX_REF, delta).sum() == pytest.approx(1.0, rel=1e-12)
    assert po.element_par(po.HEX, N, np.ones(8)).sum() == pytest.approx(P, rel=1e-13)
    # gradient of a linear field is exact and constant
    x, _ = po.gll(N)
    X = np.array([[x[p % n], x[(p // n) % n], x[p // (n * n)]] for p in range(P)])
    lin = 2.0 * X[:, 0] - 3.0 * X[:, 1] + 0.5 * X[:, 2]
    np.testing.assert_allclose(po.element_gradient(po.HEX, N, HEX_REF, lin),
                               np.tile([2.0, -3.0, 0.5], (P, 1)), atol=1e-11)


def test_p1_inverse_map_and_hull():
    # test_QuadP1.cpp / test_HexP1.cpp: inverse map recovers reference coords
    rng = np.random.default_rng(3)
    quad = np.array([[0, 0], [2, 0.1], [2.2, 1.9], [-0.1, 2]], float)
    hexv = HEX_REF * np.array([1.5, 2.0, 0.7]) + np.array([10.0, -3.0, 2.0])
    for shape, vtx, d in [(po.QUAD, quad, 2), (po.HEX, hexv, 3)]:
        for _ in range(20):
            ref = rng.uniform(-0.95, 0.95, d)
            w = []
            nv = 4 if d == 2 else 8
            signs = QUAD_REF if d == 2 else HEX_REF
            w = np.prod(1 + signs * ref, axis=1) / 2 ** d
            x = w @ vtx
            assert po.check_hull(shape, vtx, x) == 1
            np.testing.assert_allclose(po.inverse_map(shape, vtx, x), ref, atol=1e-6)
        far = vtx.mean(axis=0) + 100.0
        assert po.check_hull(shape, vtx, far) == 0


def test_literal_quirks_agree_on_affine_cells():
    # Q3 (J^-1 at output point) and Q17 (swapped dN/dr, dN/ds arguments) are
    # exact on parallelograms: literal and corrected forms agree there.
    N, n = 4, 5
    vtx = np.array([[0, 0], [2, 0.5], [2.7, 2.5], [0.7, 2.0]], float)  # parallelogram
    rng = np.random.default_rng(1)
    f = rng.standard_normal((n * n, 2))
    a = po.element_grad_test(po.QUAD, N, vtx, f)
    b = po.element_grad_test(po.QUAD, N, vtx, f, flags=po.Q3_QUAD_INVJ_AT_OUTPUT | po.Q17_QUAD_SWAPPED_JAC)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)
    # and differ on a general quad, where the reference's quirks change the result
    vtx2 = np.array([[0, 0], [2, 0.1], [2.2, 1.9], [-0.1, 2.0]], float)
    c = po.element_grad_test(po.QUAD, N, vtx2, f)
    d = po.element_grad_test(po.QUAD, N, vtx2, f, flags=po.Q3_QUAD_INVJ_AT_OUTPUT | po.Q17_QUAD_SWAPPED_JAC)
    assert np.abs(c - d).max() > 1e-6


def test_standing_wave_oracle():
    # Neumann analogue of test_Scalar_2D.cpp:62-89 (cos mode, omega = sqrt2 pi vp/L)
    from salvus_b200 import configs
    cfg = configs.standing_wave_2d(nel=10, order=4)
    p = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                   cfg["params"])
    assert p.G == 41 * 41
    X = p.coords()
    dt = 0.4 * 2.0 / np.sqrt(p.max_eigenvalue(300))
    p.set_field("u", configs.standing_wave_initial(X, cfg["L"]))
    e0 = p.energy()
    nsteps = 300
    p.run(nsteps, dt)
    exact = configs.standing_wave_initial(X, cfg["L"]) * np.cos(cfg["omega"] * nsteps * dt)
    err = np.abs(p.get_field("u")[:, 0] - exact).max()
    # the reference's Newmark start (a_ = 0, Order2Newmark.cpp:99-108) is first
    # order: error ~ (omega dt / 2) |sin(omega t)|
    assert err < 0.6 * cfg["omega"] * dt + 1e-4
    assert abs(p.energy() - e0) / e0 < 0.05


def test_delta_source_integrates_to_amplitude():
    # test_source.cpp:319-331: the source term of the owning element sums to
    # the Ricker amplitude at t = delay; other elements see nothing.
    from salvus_b200 import configs
    cfg = configs.standing_wave_2d(nel=6, order=3)
    p = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                   cfg["params"])
    p.add_source((3210.0, 4870.0), 2.0, 0.5, 10.0, [1.0])
    a = p.acceleration(0.5) / p.inverse_mass()[:, None]
    assert a.sum() == pytest.approx(10.0, rel=1e-12)
