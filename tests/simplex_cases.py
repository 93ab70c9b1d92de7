"""Shared builders for the P3 simplex parity tests: a product problem and an
oracle problem on the same seeded mesh, with the product -> oracle node map
(by coordinates)."""
import numpy as np

from oracle import pyoracle as po
from salvus_b200 import configs, core


def small_tri(seed=3):
    return configs.simplex_tri(nx=16, ny=8, n_receivers=6, seed=seed)


def small_tet(physics, n=3, seed=3):
    return configs.simplex_tet(n=n, physics=physics, n_receivers=5, seed=seed)


def oracle_problem(cfg):
    return po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                      configs.oracle_params(cfg))


def oracle_dt(cfg, frac=0.4):
    return frac * 2.0 / np.sqrt(oracle_problem(cfg).max_eigenvalue(300))


def add_sources(prob, orc, cfg):
    for s in cfg["sources"]:
        if "moment_tensor" in s:
            prob.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                            moment_tensor=s["moment_tensor"])
            orc.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                           s["moment_tensor"], kind=1)
        else:
            prob.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                            direction=s["direction"])
            orc.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                           s["direction"])
    for r in cfg["receivers"]:
        prob.add_receiver(r)
        orc.add_receiver(r)


def node_map(mesh_xyz, orc_xyz, scale):
    """idx with product node i <-> oracle node idx[i]."""
    key = lambda x: [tuple(k) for k in np.round(x / scale * 1e7).astype(np.int64)]
    ko = {k: i for i, k in enumerate(key(orc_xyz))}
    return np.array([ko[k] for k in key(mesh_xyz)])


def build_pair(cfg, precision, dt, device=0):
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"], device=device)
    orc = oracle_problem(cfg)
    idx = node_map(mesh.node_coords(), orc.coords(), cfg["L"])
    if device < 0:
        return mesh, None, orc, idx
    prob = core.Problem(mesh, precision, dt=dt)
    add_sources(prob, orc, cfg)
    return mesh, prob, orc, idx


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))
