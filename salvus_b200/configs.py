"""Seeded synthetic workloads for the headline configurations.

All inputs are synthetic (no datasets): structured meshes, Gaussian random
field models and seeded source / receiver positions.  Sizes are parameters so
that tests can run the same physics at reduced size.
"""
import numpy as np

from . import meshgen
from .core import ACOUSTIC, COUPLED2D, ELASTIC2D, ELASTIC3D, HEX, QUAD, TET, TRI


def standing_wave_2d(nel=40, order=4, L=1.0e4, vp=4000.0):
    """2-D acoustic quad mesh of an L x L square, homogeneous vp, free
    (Neumann) boundaries.  Initial condition u = cos(pi x/L) cos(pi y/L)."""
    V, C = meshgen.structured_quad(nel, nel, L, L)
    par = np.full((1, len(C), 4), vp)
    return dict(shape=QUAD, order=order, physics=ACOUSTIC, vertices=V, cells=C, params=par,
                L=L, vp=vp, omega=np.sqrt(2.0) * np.pi * vp / L)


def standing_wave_initial(xyz, L):
    return np.prod(np.cos(np.pi * xyz / L), axis=1)


def ricker_2d(nel=40, order=4, L=1.0e4, vp=4000.0, f0=2.0, n_receivers=16, radius=3.0e3, seed=0):
    """Point Ricker source at the centre and a seeded ring of receivers."""
    cfg = standing_wave_2d(nel, order, L, vp)
    center = (L / 2, L / 2)
    cfg.update(
        sources=[dict(location=center, center_freq=f0, time_delay=1.2 / f0, amplitude=1.0,
                      direction=[1.0])],
        receivers=meshgen.ring_positions(center, radius, n_receivers, seed),
    )
    return cfg


def ti_params(rho, vp, vs, C, anisotropy):
    """The reference's six Elastic3D parameters per element vertex
    (Elastic3D.cpp:33-54), [6][E][nv] RHO VPV VPH VSV VSH ETA, for a vertical
    symmetry axis: VPV = vp, VPH = vp sqrt(1 + 2 eps), VSV = vs,
    VSH = vs sqrt(1 + 2 gamma), ETA = eta (Thomsen-style parameters from the
    `anisotropy` dict eps, gamma, eta)."""
    eps, gam, eta = anisotropy["eps"], anisotropy["gamma"], anisotropy["eta"]
    pe = lambda x: meshgen.per_element_vertex(x, C)
    return np.stack([pe(rho), pe(vp), pe(vp * np.sqrt(1 + 2 * eps)), pe(vs),
                     pe(vs * np.sqrt(1 + 2 * gam)), pe(np.full_like(rho, eta))])


VTI = dict(eps=0.08, gamma=0.06, eta=0.9)  # a moderately anisotropic layer


def elastic_hex(nel=64, order=4, h=200.0, vp=6000.0, vs=3464.0, rho=2700.0, std=0.05,
                corr=1000.0, f0=1.5, n_receivers=64, seed=1, anisotropy=None):
    """3-D elastic hex cube with a Gaussian random-field perturbation of
    vp, vs and rho, a moment-tensor Ricker source at the centre and receivers
    at seeded positions on the top surface.  anisotropy (dict eps, gamma,
    eta) makes the material transversely isotropic: six parameters per
    vertex (ti_params)."""
    L = nel * h
    V, C = meshgen.structured_hex(nel, nel, nel, L, L, L)
    grf = meshgen.gaussian_random_field((nel + 1,) * 3, h, corr, seed)  # [z][y][x]
    pert = 1.0 + std * grf.ravel()
    vpv, vsv, rhov = vp * pert, vs * pert, rho * pert
    if anisotropy is not None:
        params = ti_params(rhov, vpv, vsv, C, anisotropy)
    else:
        params = np.stack([meshgen.per_element_vertex(rhov, C), meshgen.per_element_vertex(vpv, C),
                           meshgen.per_element_vertex(vsv, C)])
    rng = np.random.default_rng(seed)
    mt = rng.standard_normal(6)
    rec_xy = rng.uniform(0.02 * L, 0.98 * L, size=(n_receivers, 2))
    receivers = np.concatenate([rec_xy, np.full((n_receivers, 1), L)], axis=1)
    return dict(shape=HEX, order=order, physics=ELASTIC3D, vertices=V, cells=C, params=params,
                L=L, sources=[dict(location=(L / 2 + 0.37 * h, L / 2 - 0.21 * h, L / 2 + 0.13 * h),
                                   center_freq=f0, time_delay=1.2 / f0, amplitude=1.0e13,
                                   moment_tensor=mt)],
                receivers=receivers)


def acoustic_hex(nel=8, order=4, L=1.0e4, vp=4000.0):
    V, C = meshgen.structured_hex(nel, nel, nel, L, L, L)
    par = np.full((1, len(C), 8), vp)
    return dict(shape=HEX, order=order, physics=ACOUSTIC, vertices=V, cells=C, params=par, L=L,
                vp=vp, omega=np.sqrt(3.0) * np.pi * vp / L)


def batched_quad(nel=200, order=4, L=1.0e4, vmin=2500.0, vmax=5500.0, corr=800.0, n_shots=256,
                 n_receivers=16, seed=2):
    """Smooth random velocity model on an nel x nel quad mesh and n_shots
    Ricker sources (f0 uniform in 1.5-3 Hz, positions uniform in the interior)."""
    V, C = meshgen.structured_quad(nel, nel, L, L)
    h = L / nel
    grf = meshgen.gaussian_random_field((nel + 1, nel + 1), h, corr, seed).ravel()
    lo, hi = grf.min(), grf.max()
    vpv = vmin + (vmax - vmin) * (grf - lo) / (hi - lo)
    par = meshgen.per_element_vertex(vpv, C)[None]
    rng = np.random.default_rng(seed)
    f0 = rng.uniform(1.5, 3.0, n_shots)
    pos = rng.uniform(0.1 * L, 0.9 * L, size=(n_shots, 2))
    sources = [dict(location=tuple(pos[s]), center_freq=f0[s], time_delay=1.2 / f0[s],
                    amplitude=1.0, direction=[1.0], shot=s) for s in range(n_shots)]
    receivers = meshgen.ring_positions((L / 2, L / 2), 0.35 * L, n_receivers, seed)
    return dict(shape=QUAD, order=order, physics=ACOUSTIC, vertices=V, cells=C, params=par, L=L,
                sources=sources, receivers=receivers)


def serving_job(kind, edge, seed, order=4, n_receivers=8):
    """One forward-modelling job of the serving stream: a 2-D acoustic quad
    job on a 10 km square (edge x edge elements, vp GRF in 2500-5500 m/s) or
    a 3-D elastic hex job on a cube of 200 m hexes (vp, vs, rho with a 5 %
    GRF), each with its own seeded model, Ricker source and receivers."""
    rng = np.random.default_rng(seed)
    if kind == "quad":
        L = 1.0e4
        cfg = batched_quad(nel=edge, order=order, n_shots=1, n_receivers=n_receivers, seed=seed)
        src = cfg["sources"][0]
        cfg["sources"] = [dict(location=src["location"], center_freq=src["center_freq"],
                               time_delay=src["time_delay"], amplitude=1.0, direction=[1.0])]
        cfg["h"] = L / edge
        cfg["vmax"] = 5500.0
        return cfg
    cfg = elastic_hex(nel=edge, order=order, n_receivers=n_receivers, seed=seed,
                      f0=float(rng.uniform(1.0, 2.0)))
    cfg["h"] = 200.0
    cfg["vmax"] = 6000.0 * 1.25
    return cfg


def serving_stream(n_jobs, seed=4, quad_edges=(50, 400), hex_edges=(16, 48), steps=(1000, 6000),
                   rate_hz=1.0):
    """Seeded job stream: half quads (edge ~ U{quad_edges}), half hexes (edge
    ~ U{hex_edges}), steps ~ U{steps}, Poisson arrivals at rate_hz.  Returns
    (kind, edge, seed, n_steps, arrival_s) tuples; meshes are built on demand."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n_jobs):
        t += rng.exponential(1.0 / rate_hz)
        kind = "quad" if rng.random() < 0.5 else "hex"
        lo, hi = quad_edges if kind == "quad" else hex_edges
        out.append((kind, int(rng.integers(lo, hi + 1)), int(seed * 100003 + k),
                    int(rng.integers(steps[0], steps[1] + 1)), t))
    return out


def elastic_2d(nel=200, order=4, L=1.0e4, vp=4000.0, vs=2300.0, rho=2500.0, eps=0.1, std=0.05,
               corr=800.0, f0=2.0, n_receivers=16, jitter=0.0, seed=5):
    """2-D elastic quads (Elastic2D physics) on an L x L square: Gaussian
    random-field perturbation of vp, vs and rho, weak VTI anisotropy
    C11 = (1 + 2 eps) C33, C33 = rho vp^2, C55 = rho vs^2, C13 = C33 - 2 C55;
    a seeded moment-tensor source and a vertical force near the centre,
    receivers on a seeded ring.  jitter moves interior vertices by up to
    jitter * h (general quadrilaterals)."""
    V, C = meshgen.structured_quad(nel, nel, L, L)
    h = L / nel
    rng = np.random.default_rng(seed)
    if jitter > 0:
        inner = np.all((V > 0.5 * h) & (V < L - 0.5 * h), axis=1)
        V = V.copy()
        V[inner] += rng.uniform(-jitter * h, jitter * h, size=(inner.sum(), 2))
    grf = meshgen.gaussian_random_field((nel + 1, nel + 1), h, corr, seed).ravel()
    pert = 1.0 + std * grf
    rv, pv, sv = rho * pert, vp * pert, vs * pert
    c33 = rv * pv * pv
    c55 = rv * sv * sv
    c11 = (1.0 + 2.0 * eps) * c33
    c13 = c33 - 2.0 * c55
    params = np.stack([meshgen.per_element_vertex(x, C) for x in (rv, c11, c13, c33, c55)])
    center = (L / 2 + 0.31 * h, L / 2 - 0.17 * h)
    mt = rng.standard_normal(3)
    return dict(shape=QUAD, order=order, physics=ELASTIC2D, vertices=V, cells=C, params=params,
                L=L, vp=vp, vs=vs,
                sources=[dict(location=center, center_freq=f0, time_delay=1.2 / f0, amplitude=1.0e10,
                              moment_tensor=mt),
                         dict(location=(L / 2 - 1.3 * h, L / 2 + 0.6 * h), center_freq=f0,
                              time_delay=1.4 / f0, amplitude=1.0e9, direction=[0.0, 1.0])],
                receivers=meshgen.ring_positions((L / 2, L / 2), 0.3 * L, n_receivers, seed))


def coupled_2d(nel=40, order=4, L=1.0e4, depth=0.4, vp_f=1500.0, rho_f=1000.0, vp=4000.0,
               vs=2300.0, rho=2600.0, std=0.05, corr=800.0, f0=2.0, n_receivers=16, seed=6):
    """2-D fluid over solid (ocean over crust) on nel x nel quads of an L x L
    square: elements whose centre lies in the top `depth` fraction are fluid
    (homogeneous vp_f, rho_f), the rest solid (isotropic elastic, 5 % GRF).
    params [7][E][4] = FLUID, VP, RHO, C11, C13, C33, C55.  A moment-tensor
    source in the solid, a pressure source in the fluid, receivers on a ring
    crossing the interface.  Fields per node [u (fluid), ux, uy]."""
    V, C = meshgen.structured_quad(nel, nel, L, L)
    h = L / nel
    grf = meshgen.gaussian_random_field((nel + 1, nel + 1), h, corr, seed).ravel()
    pert = 1.0 + std * grf
    rv, pv, sv = rho * pert, vp * pert, vs * pert
    c33 = rv * pv * pv
    c55 = rv * sv * sv
    c13 = c33 - 2.0 * c55
    ctr = V[C].mean(axis=1)
    fluid = (ctr[:, 1] > (1.0 - depth) * L).astype(np.float64)
    fl = fluid[:, None] * np.ones((1, 4))
    pe = lambda x: meshgen.per_element_vertex(x, C)
    rho_e = np.where(fl > 0, rho_f, pe(rv))
    params = np.stack([fl, np.full_like(fl, vp_f), rho_e, pe(c33), pe(c13), pe(c33), pe(c55)])
    rng = np.random.default_rng(seed)
    y_if = (1.0 - depth) * L
    return dict(shape=QUAD, order=order, physics=COUPLED2D, vertices=V, cells=C, params=params,
                L=L, interface_y=y_if,
                sources=[dict(location=(L / 2 + 0.31 * h, 0.5 * y_if + 0.13 * h), center_freq=f0,
                              time_delay=1.2 / f0, amplitude=1.0e10,
                              moment_tensor=rng.standard_normal(3)),
                         dict(location=(0.3 * L + 0.2 * h, y_if + 0.5 * depth * L + 0.4 * h),
                              center_freq=f0, time_delay=1.5 / f0, amplitude=1.0e4,
                              direction=[1.0, 0.0, 0.0])],
                receivers=meshgen.ring_positions((L / 2, y_if), 0.25 * L, n_receivers, seed))


def simplex_tri(nx=448, ny=224, lx=2.0e4, ly=1.0e4, vp=4000.0, std=0.05, corr=1000.0, f0=1.0,
                n_receivers=16, seed=3):
    """2-D acoustic P3 triangles: seeded Delaunay mesh of a jittered
    (nx+1) x (ny+1) point lattice over lx x ly (about 2 nx ny triangles),
    vp homogeneous times (1 + std GRF), Ricker f0 at the centre, a seeded
    receiver ring of radius 0.3 ly."""
    V, C = meshgen.delaunay_tri(nx, ny, lx, ly, seed=seed)
    h = lx / nx
    grf = meshgen.gaussian_random_field((ny + 1, nx + 1), h, corr, seed).ravel()
    vpv = vp * (1.0 + std * grf)
    par = meshgen.per_element_vertex(vpv, C)[None]
    center = (lx / 2 + 0.31 * h, ly / 2 - 0.17 * h)
    return dict(shape=TRI, order=3, physics=ACOUSTIC, vertices=V, cells=C, params=par, L=lx,
                sources=[dict(location=center, center_freq=f0, time_delay=1.2 / f0, amplitude=1.0,
                              direction=[1.0])],
                receivers=meshgen.ring_positions(center, 0.3 * ly, n_receivers, seed))


def simplex_tet(n=44, L=1.0e4, physics=ELASTIC3D, vp=6000.0, vs=3464.0, rho=2700.0, std=0.05,
                corr=1000.0, f0=1.0, n_receivers=64, seed=3, anisotropy=None, mesh="delaunay"):
    """3-D P3 tetrahedra over an L cube: a seeded Delaunay tetrahedralisation
    of a jittered body-centred cubic point set on n^3 cells (about 12 n^3
    elements; n = 44 gives 176k points and ~1.02M tetrahedra), or with
    mesh="kuhn" a jittered lattice whose cells are split into 6 tetrahedra
    each; material homogeneous times (1 + std GRF);
    elastic: seeded moment-tensor Ricker source, acoustic: pressure source;
    receivers at seeded positions on the top surface."""
    h = L / n
    if mesh == "kuhn":
        V, C = meshgen.kuhn_tet(n, n, n, L, L, L, seed=seed)
        grf = meshgen.gaussian_random_field((n + 1,) * 3, h, corr, seed).ravel()
    else:
        V, C = meshgen.delaunay_tet(n, n, n, L, L, L, seed=seed)
        # the field on the doubled lattice: cell corners at even, cell
        # centres at odd indices (the point order of delaunay_tet)
        g2 = meshgen.gaussian_random_field((2 * n + 1,) * 3, h / 2, corr, seed)
        grf = np.concatenate([g2[::2, ::2, ::2].ravel(), g2[1::2, 1::2, 1::2].ravel()])
    pert = 1.0 + std * grf
    rng = np.random.default_rng(seed)
    rec_xy = rng.uniform(0.02 * L, 0.98 * L, size=(n_receivers, 2))
    receivers = np.concatenate([rec_xy, np.full((n_receivers, 1), L)], axis=1)
    loc = (L / 2 + 0.37 * h, L / 2 - 0.21 * h, L / 2 + 0.13 * h)
    if physics == ACOUSTIC:
        par = meshgen.per_element_vertex(vp * pert, C)[None]
        src = dict(location=loc, center_freq=f0, time_delay=1.2 / f0, amplitude=1.0, direction=[1.0])
    else:
        if anisotropy is not None:
            par = ti_params(rho * pert, vp * pert, vs * pert, C, anisotropy)
        else:
            par = np.stack([meshgen.per_element_vertex(rho * pert, C),
                            meshgen.per_element_vertex(vp * pert, C),
                            meshgen.per_element_vertex(vs * pert, C)])
        src = dict(location=loc, center_freq=f0, time_delay=1.2 / f0, amplitude=1.0e13,
                   moment_tensor=rng.standard_normal(6))
    return dict(shape=TET, order=3, physics=physics, vertices=V, cells=C, params=par, L=L,
                sources=[src], receivers=receivers)


def oracle_params(cfg):
    """Parameter array in the oracle's layout (elastic: RHO VPV VPH VSV VSH ETA)."""
    p = cfg["params"]
    if cfg["physics"] in (ACOUSTIC, ELASTIC2D, COUPLED2D) or len(p) == 6:
        return p
    rho, vp, vs = p
    return np.stack([rho, vp, vp, vs, vs, np.ones_like(rho)])
