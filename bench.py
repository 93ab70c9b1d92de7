"""Benchmark: GLL-point updates/s of the explicit spectral-element time step.

Workload (default): 3-D elastic Hexahedron<Elastic3D>, 64^3 hexes of 200 m,
order 4 (125 GLL points per element, G = 257^3 = 16,974,593 nodes, 3
components), FP32 fields with FP64-computed geometry, Gaussian random-field
model, moment-tensor Ricker source, 64 surface receivers.  A step is one time
step of the whole mesh.  Per-step inputs (~3.6 GB of geometry, material and
wavefields) exceed the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs an independent replica on its own GPU (the
path does not shard: replicas only); value = total updates / max rank time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GLL-point updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--repeats", type=int, default=5,
                    help="time the K-step region this many times; report the median")
    ap.add_argument("--nel", type=int, default=64)
    ap.add_argument("--order", type=int, default=4)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-shots", action="store_true", help="skip the batched-shots leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-simplex", action="store_true", help="skip the P3 simplex leg")
    ap.add_argument("--no-elastic2d", action="store_true", help="skip the 2-D elastic quad leg")
    ap.add_argument("--no-general", action="store_true",
                    help="skip timing the per-point-geometry stiffness kernel")
    ap.add_argument("--profile-leg", default=None,
                    choices=["quad", "elastic2d", "coupled", "tri", "tet", "shots", "group"],
                    help="set up one workload and run --steps plain steps (for ncu captures)")
    ap.add_argument("--elastic2d-only", action="store_true",
                    help="run only the 2-D elastic quad leg (profiling)")
    ap.add_argument("--e2d-nel", type=int, default=720,
                    help="2-D elastic leg: nel x nel quads (default 720, ~8.3M nodes)")
    ap.add_argument("--simplex-only", action="store_true",
                    help="run only the P3 simplex leg (profiling / quick checks)")
    ap.add_argument("--tet-n", type=int, default=44,
                    help="tetrahedral mesh cells per side (Delaunay of a jittered BCC point "
                         "set, ~12 n^3 elements; 44 -> ~1.02M)")
    ap.add_argument("--serving-jobs", type=int, default=24)
    ap.add_argument("--serving-max-running", type=int, default=32,
                    help="serving leg: jobs admitted at once (running or being prepared)")
    ap.add_argument("--serving-only", action="store_true",
                    help="run only the serving leg (e.g. --serving-jobs 500) and print its JSON")
    ap.add_argument("--serving-no-serial", action="store_true",
                    help="serving leg: skip the serial plain runs (latency percentiles of a "
                         "long stream only; no throughput ratio)")
    ap.add_argument("--profile-only", action="store_true",
                    help="run a few steps only (for ncu captures); prints no JSON")
    ap.add_argument("--per-point-geometry", action="store_true",
                    help="build the hexahedron mesh with per-point geometry records "
                         "(profiling the general layout with --profile-only)")
    return ap.parse_args()


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def max_over_ranks(x, dist=None, device="cuda"):
    """The largest of each rank's x (every rank gets it); x itself without a
    process group.  Replicas time the same work, so the job's time is the
    slowest rank's."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(nodes, steps, ms, world):
    """Whole-job GLL-point updates/s of `world` replicas that each advanced
    `nodes` nodes `steps` steps, from the max-over-ranks time in ms."""
    return world * nodes * steps / (ms / 1e3)


def workload(args):
    return {"workload": f"elastic3d hex {args.nel}^3 order {args.order}, 64 receivers, "
                        f"moment-tensor Ricker, GRF model",
            "shape": "Hexahedron<Elastic3D>", "elements": args.nel ** 3, "order": args.order,
            "fields": "fp32 (geometry computed fp64)", "l2": "inputs larger than L2 (no flush)"}


def arm_config(args, world=1):
    """The `config` object of both arms' JSON lines: the workload and the
    replica count (the reference arm is one CPU instance, so world = 1)."""
    return dict(workload(args), parallelism=f"replicas x{world}")


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_leg(args, nel_sample, steps, warm, target_s=10.0):
    """Time the FP64 CPU oracle in reference-faithful mode (per-point Jacobian
    rebuilds, Hexahedra.cpp:600,702) on a bounded sample of the workload."""
    from oracle import pyoracle as po
    from salvus_b200 import configs
    thr = cpu_threads()
    cfg = configs.elastic_hex(nel=nel_sample, order=args.order)
    o = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                   configs.oracle_params(cfg), flags=po.FAITHFUL_RECOMPUTE, threads=thr)
    s = cfg["sources"][0]
    o.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                 s["moment_tensor"], kind=1)
    for r in cfg["receivers"]:
        o.add_receiver(r)
    dt = 1e-3
    t0 = time.perf_counter()
    if warm > 0:
        o.run(warm, dt)  # warm-up, also sizes the sample
    per_step = (time.perf_counter() - t0) / max(1, warm)
    if steps is None:  # about target_s of CPU work, 2..200 steps
        steps = int(min(200, max(2, target_s / max(per_step, 1e-6))))
    t0 = time.perf_counter()
    o.run(steps, dt)
    el = time.perf_counter() - t0
    rate = o.G * steps / el
    sample = (f"oracle (FP64 reference-faithful restatement, OpenMP over element colours) on "
              f"{nel_sample}^3 elements (G={o.G}) x {steps} steps after {warm} warm-up; "
              f"{el:.2f} s")
    return rate, thr, sample, el


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None

    def start(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        self.proc.wait()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        busy = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": float(np.median(busy)) if busy else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def shots_leg(core, configs, timed, steps, n_shots=256, nel=200, device=0):
    """Config 2: n_shots Ricker shots on a nel x nel order-4 quad mesh with a
    seeded smooth velocity model.  Batched form (one graph-replayed launch
    sequence per step for all shots) against the plain form (one shot, one
    host-launched step at a time) on the same mesh."""
    cfg = configs.batched_quad(nel=nel, order=4, n_shots=n_shots)
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"], device=device)
    dt = 0.4 * mesh.critical_dt(iterations=60)
    G = mesh.n_nodes
    p = core.Problem(mesh, core.FP32, dt=dt, n_shots=n_shots)
    for s in cfg["sources"]:
        p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                     direction=s["direction"], shot=s["shot"])
    for r in cfg["receivers"]:
        p.add_receiver(r)
    p.set_seismogram_capacity(steps + 64)
    tune = p.autotune()
    p.run(5, core.RUN_GRAPH)
    p.prepare_run(steps)
    p.synchronize()
    ms_b = timed(p, lambda: p.run(steps, core.RUN_GRAPH))
    # per-kernel device times of the same step (host-launched, event-timed):
    # what a single launch per step could save is at most the graph step
    # minus their sum
    p.profile(True)
    p.run(min(steps, 50), core.RUN_PLAIN)
    kern = {k: v[0] / max(v[1], 1) for k, v in p.profile_read().items()}
    p.profile(False)
    q = core.Problem(mesh, core.FP32, dt=dt)
    s = cfg["sources"][0]
    q.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                 direction=s["direction"])
    for r in cfg["receivers"]:
        q.add_receiver(r)
    q.set_seismogram_capacity(2 * steps + 128)
    q.run(5, core.RUN_PLAIN)
    q.synchronize()
    ms_p = timed(q, lambda: q.run(steps, core.RUN_PLAIN))
    # the same single shot with its time loop replayed from a CUDA graph
    q.run(64, core.RUN_GRAPH)
    q.prepare_run(steps)
    q.synchronize()
    ms_g = timed(q, lambda: q.run(steps, core.RUN_GRAPH))
    batched = G * n_shots * steps / (ms_b / 1e3)
    plain = G * steps / (ms_p / 1e3)
    return {"workload": f"acoustic quad {nel}^2 order 4, {n_shots} Ricker shots, GRF model, "
                        f"{len(cfg['receivers'])} receivers",
            "value": batched, "unit": METRIC, "ms_per_step": ms_b / steps,
            "plain_value": plain, "plain_ms_per_step": ms_p / steps,
            "single_graph_value": G * steps / (ms_g / 1e3), "single_graph_ms_per_step": ms_g / steps,
            "form": "fused batched step (interior nodes in the stiffness kernel), CUDA graph",
            "shot_throughput_ratio": batched / plain, "steps": steps,
            "kernels_ms": kern,
            "launch_gaps_ms_per_step": ms_b / steps - sum(kern.values()),
            "tuning": {"stiffness_shot_lanes": tune[0], "stiffness_elements_per_cta": tune[1],
                       "gather_shot_lanes": tune[2], "gather_nodes_per_cta": tune[3]}}


def simplex_leg(core, configs, timed, steps, device=0, tet_n=55):
    """Config 3: P3 simplices in FP32 -- acoustic triangles (Delaunay, ~200k
    elements over 20 x 10 km) and elastic tetrahedra (~1M elements over a
    10 km cube), homogeneous + 5 % GRF, Ricker f0 = 1 Hz.  Each is timed as
    graph-replayed steps; the stiffness kernel is timed per launch."""
    out = {}
    for name, cfg in (("tri_acoustic", configs.simplex_tri()),
                      ("tet_elastic", configs.simplex_tet(n=tet_n, physics=core.ELASTIC3D))):
        mesh = core.Mesh(cfg["shape"], 3, cfg["physics"], cfg["vertices"], cfg["cells"],
                         cfg["params"], device=device)
        dt = 0.4 * mesh.critical_dt(iterations=40)
        p = core.Problem(mesh, core.FP32, dt=dt)
        for s in cfg["sources"]:
            if "moment_tensor" in s:
                p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                             moment_tensor=s["moment_tensor"])
            else:
                p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                             direction=s["direction"])
        for r in cfg["receivers"]:
            p.add_receiver(r)
        p.set_seismogram_capacity(steps + 64)
        p.run(5, core.RUN_GRAPH)
        p.prepare_run(steps)
        p.synchronize()
        ms = timed(p, lambda: p.run(steps, core.RUN_GRAPH))
        p.profile(True)
        p.run(min(steps, 50), core.RUN_PLAIN)
        prof = p.profile_read()
        p.profile(False)
        G, E, P, c = mesh.n_nodes, mesh.n_elements, mesh.points_per_element, mesh.n_components
        k_ms, k_n = prof.get("stiffness", (0.0, 1))
        st_ms = k_ms / max(k_n, 1)
        # useful FLOPs of the factored operator per element: gradient and
        # divergence contractions, 2 x (dim x P x P) multiply-adds per component
        dim = mesh.dim
        flops = E * c * 2 * 2 * dim * P * P
        out[name] = {"elements": E, "nodes": G, "components": c, "dt": dt, "steps": steps,
                     "value": G * steps / (ms / 1e3), "unit": METRIC,
                     "ms_per_step": ms / steps,
                     "kernels_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items()},
                     "stiffness_tflops": flops / (st_ms / 1e3) / 1e12 if st_ms > 0 else None}
        p.close()
        mesh.close()
    return out


def elastic2d_leg(core, configs, timed, steps, device=0, nel=720, peak=None):
    """2-D elastic quads (Elastic2D physics): FP32, order 4,
    nel^2 undistorted structured quads over 10 x 10 km, 5 % GRF, weak VTI
    anisotropy, moment-tensor + force Ricker sources, 16 receivers.  Timed as
    graph-replayed steps; the stiffness kernel per launch against HBM."""
    cfg = configs.elastic_2d(nel=nel, order=4)
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"], device=device)
    dt = 0.4 * mesh.critical_dt(iterations=40)
    p = core.Problem(mesh, core.FP32, dt=dt)
    for s in cfg["sources"]:
        if "moment_tensor" in s:
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                         moment_tensor=s["moment_tensor"])
        else:
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                         direction=s["direction"])
    for r in cfg["receivers"]:
        p.add_receiver(r)
    p.set_seismogram_capacity(steps + 64)
    p.run(5, core.RUN_GRAPH)
    p.prepare_run(steps)
    p.synchronize()
    ms = timed(p, lambda: p.run(steps, core.RUN_GRAPH))
    p.profile(True)
    p.run(min(steps, 50), core.RUN_PLAIN)
    prof = p.profile_read()
    p.profile(False)
    G, E, P = mesh.n_nodes, mesh.n_elements, mesh.points_per_element
    k_ms, k_n = prof.get("stiffness", (0.0, 1))
    st_ms = k_ms / max(k_n, 1)
    # algorithmic bytes per stiffness launch: per point 32 B record (invJ 4,
    # C11 C13 C33 C55 x w detJ) + 4 B connectivity + 8 B residual write, plus
    # the compulsory u read of 8 B per node
    b_stiff = E * P * (32 + 4 + 8) + G * 8
    ach = b_stiff / (st_ms / 1e3) / 1e9 if st_ms > 0 else None
    out = {"elements": E, "nodes": G, "components": 2, "dt": dt, "steps": steps,
           "value": G * steps / (ms / 1e3), "unit": METRIC, "ms_per_step": ms / steps,
           "kernels_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items()},
           "roofline": {"bound": "hbm", "kernel": "elastic2d_stiffness", "achieved": ach,
                        "peak": peak, "unit": "GB/s",
                        "frac": (ach / peak) if (ach and peak) else None,
                        "algorithmic_bytes": b_stiff}}
    p.close()
    mesh.close()
    return out


def profile_leg(core, configs, name, steps, device=0):
    """One workload at a capture-friendly size (inputs larger than L2, a few
    GB at most), `steps` host-launched plain steps, nothing timed: the command
    that ncu captures.  quad: 1000^2 acoustic quads N=4; elastic2d / coupled:
    720^2 quads N=4; tri: 1400 x 700 x 2 P3 triangles; tet: ~393k elastic
    P3 tetrahedra (Delaunay, 32^3 BCC cells); shots: 200^2 quads x 256 shots; group: 12 acoustic quad
    meshes of 100^2..320^2 in one problem group."""
    def populate(p, cfg, shots=False):
        for s in cfg.get("sources", []):
            kw = ({"moment_tensor": s["moment_tensor"]} if "moment_tensor" in s
                  else {"direction": s["direction"]})
            if shots:
                kw["shot"] = s["shot"]
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"], **kw)
        for r in cfg.get("receivers", []):
            p.add_receiver(r)
        p.set_seismogram_capacity(steps + 8)

    def build(cfg, **kw):
        return core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"],
                         cfg["cells"], cfg["params"], device=device, **kw)

    if name == "group":
        probs = []
        for k, edge in enumerate(range(100, 340, 20)):
            cfg = configs.ricker_2d(nel=edge, order=4, n_receivers=4, seed=k)
            m = build(cfg)
            p = core.Problem(m, core.FP32, dt=1e-4)
            populate(p, cfg)
            probs.append((m, p))
        g = core.Group([p for _, p in probs])
        g.run(steps)
        g.synchronize()
        return
    cfg = {"quad": lambda: configs.ricker_2d(nel=1000, order=4),
           "elastic2d": lambda: configs.elastic_2d(nel=720, order=4),
           "coupled": lambda: configs.coupled_2d(nel=720, order=4),
           "tri": lambda: configs.simplex_tri(nx=1400, ny=700),
           "tet": lambda: configs.simplex_tet(n=32, physics=core.ELASTIC3D),
           "shots": lambda: configs.batched_quad(nel=200, order=4, n_shots=256)}[name]()
    mesh = build(cfg)
    shots = name == "shots"
    p = core.Problem(mesh, core.FP32, dt=1e-4, n_shots=256 if shots else 1)
    populate(p, cfg, shots)
    p.run(steps, core.RUN_PLAIN)
    p.synchronize()


def unit_dt(core, meshgen, kind, order=4):
    """Critical step of a unit mesh (h = 1, vp_max = 1) for this element
    family; dt_crit(h, vp) = unit_dt * h / vp (lambda_max scales as (vp/h)^2)."""
    if kind == "quad":
        V, C = meshgen.structured_quad(6, 6, 6.0, 6.0)
        m = core.Mesh(core.QUAD, order, core.ACOUSTIC, V, C, np.ones((1, len(C), 4)))
    else:
        V, C = meshgen.structured_hex(4, 4, 4, 4.0, 4.0, 4.0)
        E = len(C)
        par = np.stack([np.full((E, 8), 1.0), np.full((E, 8), 1.0), np.full((E, 8), 0.5773)])
        m = core.Mesh(core.HEX, order, core.ELASTIC3D, V, C, par)
    return m.critical_dt(iterations=300)


def class_rate(core, configs, kind, device=0, steps=64):
    """Graph-replayed FP32 rate (GLL-point updates/s) of one large mesh of a
    serving job class: 64^3 elastic hexahedra or 1000^2 acoustic quads,
    order 4 -- the per-node rates behind the serving leg's device-time
    floor."""
    import torch
    cfg = (configs.elastic_hex(nel=64, order=4) if kind == "hex"
           else configs.batched_quad(nel=1000, order=4, n_shots=1))
    m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                  cfg["params"], device=device)
    p = core.Problem(m, core.FP32, dt=1e-5)
    p.run(32, core.RUN_GRAPH)
    p.synchronize()
    stream = torch.cuda.ExternalStream(p.stream_handle())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    p.run(steps, core.RUN_GRAPH)
    b.record(stream)
    torch.cuda.synchronize()
    rate = m.n_nodes * steps / (a.elapsed_time(b) / 1e3)
    p.close()
    m.close()
    return rate


def serving_leg(core, configs, meshgen, n_jobs=24, seed=4, load=0.8, hex_rate=None,
                quad_rate=None, max_running=32, serial=True):
    """Config 4 (bounded sample): a seeded stream of n_jobs jobs, half 2-D
    acoustic quads (edge U{50..400}), half 3-D elastic hexes (edge
    U{16..48}), order 4, own model and source each, steps U{1000..6000}.
    First every job runs alone, one after the other (plain form, mesh
    preparation included); then the same jobs arrive as a Poisson stream at
    load x the serial service rate and the server runs them.

    hex_rate and quad_rate (GLL-point updates/s of a 64^3 hexahedron and a
    1000^2 quadrilateral mesh on this GPU, graph-replayed) give a
    device-time floor: the jobs' updates need at least sum(G * steps) /
    rate of their class seconds of device time, so no served form can beat
    serial_s / that floor.  serial=False skips the serial runs (long
    streams measured for their latency percentiles only)."""
    from salvus_b200 import serving
    ud = {k: unit_dt(core, meshgen, k) for k in ("quad", "hex")}
    stream = configs.serving_stream(n_jobs, seed=seed)
    jobs = []
    for kind, edge, s, n, _ in stream:
        cfg = configs.serving_job(kind, edge, s)
        dt = 0.4 * ud[kind] * cfg["h"] / cfg["vmax"]
        jobs.append((kind, cfg, dt, n))
    # serial plain runs
    t0 = time.perf_counter()
    serial_updates = 0.0
    for kind, cfg, dt, n in (jobs if serial else []):
        m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                      cfg["params"])
        p = core.Problem(m, core.FP32, dt=dt)
        s = cfg["sources"][0]
        if "moment_tensor" in s:
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                         moment_tensor=s["moment_tensor"])
        else:
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                         direction=s["direction"])
        for r in cfg["receivers"]:
            p.add_receiver(r)
        p.set_seismogram_capacity(n + 8)
        p.run(n, core.RUN_PLAIN)
        p.seismograms()
        serial_updates += m.n_nodes * n
        p.close()
        m.close()
    serial_s = time.perf_counter() - t0 if serial else None
    # capacity: all jobs submitted at once
    srv = serving.Server(budget_bytes=150 * 10**9, max_running=max_running, chunk_steps=64)
    t0 = time.perf_counter()
    ids = [srv.submit(cfg, dt, n) for kind, cfg, dt, n in jobs]
    for j in ids:
        srv.wait(j, 3600)
    burst_s = time.perf_counter() - t0
    burst_stats = srv.stats()
    burst_updates = burst_stats["gll_point_updates"]
    srv.close()
    # served stream at `load` times the measured capacity
    rng = np.random.default_rng(seed + 1)
    gaps = rng.exponential(burst_s / n_jobs / load, size=n_jobs)
    srv = serving.Server(budget_bytes=150 * 10**9, max_running=max_running, chunk_steps=64)
    t0 = time.perf_counter()
    ids = []
    for (kind, cfg, dt, n), gap in zip(jobs, gaps):
        time.sleep(gap)
        ids.append(srv.submit(cfg, dt, n))
    for j in ids:
        srv.wait(j, 3600)
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    floor = None
    if hex_rate and quad_rate:
        # G of an edge^d mesh of order N: (N edge + 1)^d nodes
        order = jobs[0][1]["order"]
        upd = {"hex": 0, "quad": 0}
        for kind, edge, _, n, _ in stream:
            upd[kind] += (order * edge + 1) ** (3 if kind == "hex" else 2) * n
        fl = upd["hex"] / hex_rate + upd["quad"] / quad_rate
        floor = {"hex_updates": upd["hex"], "quad_updates": upd["quad"],
                 "hex_rate_64cube": hex_rate, "quad_rate_1000sq": quad_rate,
                 "device_floor_s": fl, "ratio_ceiling": serial_s / fl if serial else None,
                 "makespan_over_floor": burst_s / fl,
                 "form": "each class's updates at the graph-replayed per-node rate of one large "
                         "mesh of that class (a lower bound on the device time of any served "
                         "form, so serial_s / floor bounds the throughput ratio)"}
    return {"workload": f"{n_jobs} jobs: 2-D acoustic quads 50^2-400^2 and 3-D elastic hexes "
                        f"16^3-48^3, order 4, 1000-6000 steps; latency under Poisson arrivals at "
                        f"{load:.0%} of the measured capacity "
                        + ("(the 2000-job stream)" if n_jobs >= 2000
                           else "(bounded sample of the 2000-job stream)"),
            "p50_latency_s": st["p50_latency_s"], "p99_latency_s": st["p99_latency_s"],
            "mean_latency_s": st["mean_latency_s"], "completed": st["completed"],
            "failed": st["failed"], "value": burst_updates / burst_s, "unit": METRIC,
            "value_form": "all jobs submitted at once; total G*steps / makespan (preparation included)",
            "makespan_s": burst_s, "stream_updates_per_s": st["gll_point_updates"] / st["busy_seconds"],
            "stream_wall_s": wall,
            "serial_value": serial_updates / serial_s if serial else None, "serial_s": serial_s,
            "serial_form": "each job alone, one after the other, plain host-launched steps, "
                           "preparation included",
            "throughput_ratio": ((burst_updates / burst_s) / (serial_updates / serial_s)
                                 if serial else None),
            "peak_device_bytes": st["peak_device_bytes"],
            "prep_seconds_burst": burst_stats["prep_seconds"],
            "prep_seconds_stream": st["prep_seconds"], "max_running": max_running,
            "device_floor": floor}


REFERENCE_BUDGET_S = 150.0  # timed CPU work of the reference arm, at most


def reference_arm(args, rank, world):
    """The reference's CPU path (the FP64 oracle port in reference-faithful
    mode, all host threads) on the SAME mesh as the GPU arm: every step is a
    full step of the nel^3 workload.  --warmup steps untimed, then --steps
    steps timed; when --steps full steps would exceed REFERENCE_BUDGET_S the
    first ones that fit are timed (the per-step cost does not depend on the
    step index) and `timed_steps` says how many."""
    if rank != 0:
        return
    from oracle import pyoracle as po  # fails loudly if the oracle is not built
    from salvus_b200 import configs
    K, W = max(1, args.steps), max(1, args.warmup)
    thr = cpu_threads()
    t_setup = time.perf_counter()
    cfg = configs.elastic_hex(nel=args.nel, order=args.order)
    o = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                   configs.oracle_params(cfg), flags=po.FAITHFUL_RECOMPUTE, threads=thr)
    s = cfg["sources"][0]
    o.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                 s["moment_tensor"], kind=1)
    for r in cfg["receivers"]:
        o.add_receiver(r)
    setup_s = time.perf_counter() - t_setup
    # the workload's step (0.4 of the critical step of the 64^3 mesh); the
    # CPU cost of a step does not depend on dt
    dt = 1.2546e-3
    t0 = time.perf_counter()
    o.run(W, dt)
    per_step = (time.perf_counter() - t0) / W
    k_run = K if K * per_step <= REFERENCE_BUDGET_S else max(1, int(REFERENCE_BUDGET_S / per_step))
    t0 = time.perf_counter()
    o.run(k_run, dt)
    el = time.perf_counter() - t0
    rate = o.G * k_run / el
    sample = (f"oracle (FP64 reference-faithful restatement, per-point Jacobian rebuilds, OpenMP "
              f"over element colours, {thr} threads) on the full {args.nel}^3-element mesh "
              f"(G={o.G}): {k_run} of {K} steps timed after {W} warm-up steps, {el:.1f} s; "
              f"setup {setup_s:.0f} s untimed")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC,
            "n_gpus": args.gpus, "steps": K, "warmup": W, "timed_steps": k_run,
            "higher_is_better": True,
            "ms_per_step": 1e3 * el / k_run, "dtype": "f64", "data": "synthetic",
            "scaling": "weak", "vs_baseline": None,
            "config": arm_config(args),
            "cpu_baseline": {"value": rate, "unit": METRIC, "cores": thr, "kind": "port",
                             "sample": sample},
            "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the reference needs PETSc/Eigen/HDF5/Exodus (absent); its CPU path is "
                    "timed through the oracle port, which restates it and keeps its per-point "
                    "Jacobian rebuild cost; each step is one full step of the same mesh as the "
                    "GPU arm"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = env_rank()
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return

    import torch
    from salvus_b200 import configs, core

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.profile_leg:
        profile_leg(core, configs, args.profile_leg, args.steps, device=local)
        return

    if args.serving_only:
        from salvus_b200 import meshgen
        out = {"serving": serving_leg(core, configs, meshgen, n_jobs=args.serving_jobs,
                                      hex_rate=class_rate(core, configs, "hex", local),
                                      quad_rate=class_rate(core, configs, "quad", local),
                                      max_running=args.serving_max_running,
                                      serial=not args.serving_no_serial)}
        if rank == 0:
            print(json.dumps(out), flush=True)
        return

    if args.simplex_only or args.elastic2d_only:
        def timed_simple(prob, fn):
            stream = torch.cuda.ExternalStream(prob.stream_handle())
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            return a.elapsed_time(b)
        if args.elastic2d_only:
            peaks = measured_peaks()
            out = {"elastic2d": elastic2d_leg(core, configs, timed_simple, steps=args.steps,
                                              device=local, nel=args.e2d_nel,
                                              peak=peaks["hbm_gbs"] if peaks else 6650.0)}
        else:
            out = {"simplices": simplex_leg(core, configs, timed_simple, steps=args.steps,
                                            device=local, tet_n=args.tet_n)}
        if rank == 0:
            print(json.dumps(out), flush=True)
        return

    cfg = configs.elastic_hex(nel=args.nel, order=args.order)
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"], device=local,
                     flags=core.MESH_PER_POINT_GEOMETRY if args.per_point_geometry else 0)
    G = mesh.n_nodes
    # profile-only runs (ncu captures) skip the power iteration to keep the
    # launch list short
    dt = 1e-3 if args.profile_only else 0.4 * mesh.critical_dt(iterations=60)

    def make_problem():
        p = core.Problem(mesh, core.FP32, dt=dt)
        s = cfg["sources"][0]
        p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                     moment_tensor=s["moment_tensor"])
        for r in cfg["receivers"]:
            p.add_receiver(r)
        p.set_seismogram_capacity(args.steps + args.warmup + 64)
        return p

    p = make_problem()
    if args.profile_only:
        p.run(max(args.steps, 3), core.RUN_PLAIN)
        p.synchronize()
        return
    def barrier():
        if dist:
            dist.barrier()

    def timed_on(prob, fn):
        """CUDA events on the problem's own stream around fn(); max over ranks."""
        stream = torch.cuda.ExternalStream(prob.stream_handle())
        barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(a.elapsed_time(b), dist, "cuda")

    def timed(fn):
        return timed_on(p, fn)

    clocks = Clocks(local)
    # warm-up steps, then the capture of the graphs a K-step run replays
    # (nothing runs in the capture)
    p.run(args.warmup, core.RUN_GRAPH)
    p.prepare_run(args.steps)
    p.synchronize()
    # the K-step region is timed R times back to back; value = the median
    R = max(1, args.repeats)
    clocks.start()
    l0 = core.launch_count()
    runs = [timed(lambda: p.run(args.steps, core.RUN_GRAPH)) for _ in range(R)]
    launches = (core.launch_count() - l0) // R
    ck = clocks.stop()
    ms = float(np.median(runs))
    value = replica_rate(G, args.steps, ms, world)

    # plain form: one host launch sequence per step
    kp = min(args.steps, 200)
    ms_plain = timed(lambda: p.run(kp, core.RUN_PLAIN))
    plain = replica_rate(G, kp, ms_plain, world)

    # per-kernel device time (events around each launch, plain form)
    p.profile(True)
    p.run(min(args.steps, 100), core.RUN_PLAIN)
    prof = p.profile_read()
    p.profile(False)

    E, P = mesh.n_elements, mesh.points_per_element
    affine, n_gather = mesh.layout()
    form, epc = p.step_config()  # the hexahedron autotuner's choice
    fused = affine and form == core.STEP_FUSED_INTERIOR
    n_int = G - n_gather  # element-interior nodes (advanced in the stiffness kernel when fused)
    if fused:
        # parallelepiped layout, fused step: per point conn 4 B + lambda' mu'
        # 8 B; per element invJ 36 B; u read 12 B/node; residual write
        # 12 B/point for the points on element faces; interior nodes: inverse
        # mass 4 B + (v, a_) read 24 B + (u, v, a_) write 36 B
        b_stiff = E * P * 12 + E * 36 + G * 12 + (E * P - n_int) * 12 + n_int * 64
        # shared-node gather: node list + offsets 8 B/node, residual 12 B +
        # incidence index 4 B per face point, inverse mass 4 B + (u, v, a_)
        # read and write 72 B per node
        b_upd = n_gather * 8 + (E * P - n_int) * 16 + n_gather * 76
        layout = "per-element inverse Jacobian, interior nodes advanced in the stiffness kernel"
    elif affine:
        # parallelepiped layout (default): per point conn 4 B + lambda' mu'
        # 8 B; per element invJ 36 B; u read 12 B/node; the element-local
        # residual write 12 B/point
        b_stiff = E * P * 12 + E * 36 + G * 12 + E * P * 12
        b_upd = E * P * 16 + G * (4 + 72 + 4)
        layout = "per-element inverse Jacobian (parallelepiped elements)"
    else:
        # per-point records: 48 B (invJ 9, lambda', mu', conn) + u read
        # 12 B/node + the element-local residual write 12 B/point
        b_stiff = E * P * 48 + G * 12 + E * P * 12
        # gather/update: residual read 12 B/point + incidence index 4 B/point +
        # offsets 4 B/node + (u, v, a_) read and write 72 B/node + inverse mass 4 B/node
        b_upd = E * P * 16 + G * (4 + 72 + 4)
        layout = "per-point inverse Jacobians"
    # what bounds the kernel (ncu at 32^3, same kernels): the per-point
    # layout streams 48 B of records per point and is HBM-bound; the
    # parallelepiped layout reads 2.2x fewer DRAM bytes and is held by the
    # L1 / shared-memory pipe instead (its tensor-product contractions read
    # 60 shared-memory words per point)
    limiter = ("L1/shared-memory pipe (ncu l1tex throughput 86 % of peak, DRAM ~34 %): with "
               "the per-element Jacobian the kernel moves 2.2x fewer bytes than the per-point "
               "layout and is no longer HBM-bound" if affine and not fused else
               "HBM (DRAM bytes equal the algorithmic bytes)" if not affine else
               "L1/shared-memory pipe and occupancy (80 registers)")
    # the canonical step bytes of a per-GLL-point geometry layout (isotropic
    # elastic: d = 3, m = 2 material words; c = 3): the compulsory traffic a
    # straightforward implementation of the step moves
    b_canon_step = 4 * P * E * (1 + 9 + 1 + 2) + 8 * 3 * G + (28 * 3 + 4) * G
    peaks = measured_peaks()
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    k_ms, k_n = prof.get("stiffness", (0.0, 1))
    u_ms, u_n = prof.get("gather_update", (0.0, 1))
    st_ms = k_ms / max(k_n, 1)
    up_ms = u_ms / max(u_n, 1)
    ach = b_stiff / (st_ms / 1e3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic_elastic_hex_stiffness.txt")
    if os.path.exists(tf):
        key = "dram_bytes_per_launch_fullsize_affine=" if affine else "dram_bytes_per_launch_fullsize="
        for line in open(tf):
            if line.startswith(key):
                traffic = float(line.split("=")[1])

    # the per-point-geometry kernel on the same workload (the layout whose
    # canonical bytes are B_K = 4 P E (1 + 10 + 2) + 8 c G): its own launch
    # time and fraction of HBM
    general = None
    if affine and not args.no_general:
        mesh_g = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"],
                           cfg["cells"], cfg["params"], device=local,
                           flags=core.MESH_PER_POINT_GEOMETRY)
        pg = core.Problem(mesh_g, core.FP32, dt=dt)
        pg.run(3, core.RUN_PLAIN)
        pg.profile(True)
        pg.run(min(args.steps, 50), core.RUN_PLAIN)
        prof_g = pg.profile_read()
        pg.profile(False)
        gk_ms, gk_n = prof_g.get("stiffness", (0.0, 1))
        g_ms = gk_ms / max(gk_n, 1)
        b_g = E * P * 48 + G * 12 + E * P * 12
        b_canon = 4 * P * E * (1 + 10 + 2) + 8 * 3 * G
        general = {"kernel": "elastic_hex_stiffness (per-point records)", "ms": g_ms,
                   "achieved": b_g / (g_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                   "frac": b_g / (g_ms / 1e3) / 1e9 / peak, "algorithmic_bytes": b_g,
                   "canonical_bytes": b_canon,
                   "frac_canonical": b_canon / (g_ms / 1e3) / 1e9 / peak}
        pg.close()
        mesh_g.close()

    # end-to-end through the public API with host buffers: initial state from
    # host (u0, v0 FP64), K steps, seismograms back to the host
    p2 = make_problem()
    p2.set_seismogram_capacity(max(args.warmup, 32) + max(1, args.repeats) * args.steps + 64)
    rng = np.random.default_rng(7)
    u0 = (1e-6 * rng.standard_normal((G, 3)))
    v0 = np.zeros((G, 3))
    seis_holder = {}

    def e2e_job(k, first):
        p2.set_field("u", u0)
        p2.set_field("v", v0)
        p2.run(k, core.RUN_GRAPH)
        seis_holder["s"] = p2.seismograms(first, k)

    # one untimed warm-up job (pinned staging buffers, graph capture), then
    # the timed job
    w_e2e = max(args.warmup, 32)
    e2e_job(w_e2e, 0)
    p2.prepare_run(args.steps)
    p2.synchronize()
    # the job is timed R times (each one uploads u0 / v0 again); the median
    e2e_runs = [timed_on(p2, lambda i=i: e2e_job(args.steps, w_e2e + i * args.steps))
                for i in range(R)]
    ms_e2e = float(np.median(e2e_runs))
    e2e = replica_rate(G, args.steps, ms_e2e, world)
    # u0 and v0 cross PCIe as FP32 (converted on the host threads from the
    # caller's FP64 arrays), amortised over the K steps of the job
    h2d = 2 * G * 3 * 4 / args.steps
    d2h = len(cfg["receivers"]) * 3 * 8

    shots = None
    if not args.no_shots:
        shots = shots_leg(core, configs, timed_on, steps=min(args.steps, 300), device=local)
    serve = None
    if not args.no_serving and rank == 0 and world == 1:
        from salvus_b200 import meshgen
        serve = serving_leg(core, configs, meshgen, n_jobs=args.serving_jobs,
                            hex_rate=(value if args.nel == 64 and args.order == 4
                                      else class_rate(core, configs, "hex", local)),
                            quad_rate=class_rate(core, configs, "quad", local),
                            max_running=args.serving_max_running)

    simplex = None
    if not args.no_simplex:
        simplex = simplex_leg(core, configs, timed_on, steps=min(args.steps, 200), device=local,
                              tet_n=args.tet_n)

    e2d = None
    if not args.no_elastic2d:
        e2d = elastic2d_leg(core, configs, timed_on, steps=min(args.steps, 300), device=local,
                            nel=args.e2d_nel, peak=peak)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, thr, sample, _ = cpu_leg(args, min(args.nel, 32), None, 1)
        cpu = {"value": rate, "unit": METRIC, "cores": thr, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded GRF model, structured hex mesh)",
            "config": arm_config(args, world),
            "form": "graph-replayed fused step",
            "plain": {"value": plain, "unit": METRIC, "steps": kp, "ms_per_step": ms_plain / kp,
                      "form": "host-launched fused step"},
            "kernels_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items()},
            "roofline": {"bound": "hbm", "kernel": "elastic_hex_stiffness", "layout": layout,
                         "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "limiter": limiter,
                         "traffic": traffic, "algorithmic_bytes": b_stiff,
                         "kernel_ms": st_ms, "elements_per_cta": epc,
                         "peak_source": "measured" if peaks else "fallback"},
            "roofline_update": {"kernel": "gather_update", "achieved": b_upd / (up_ms / 1e3) / 1e9,
                                "peak": peak, "unit": "GB/s", "algorithmic_bytes": b_upd,
                                "kernel_ms": up_ms,
                                "frac": b_upd / (up_ms / 1e3) / 1e9 / peak},
            "roofline_step": {"bytes_per_step": b_stiff + b_upd, "ms_per_step": ms / args.steps,
                              "achieved": (b_stiff + b_upd) / (ms / args.steps / 1e3) / 1e9,
                              "peak": peak, "unit": "GB/s",
                              "frac": (b_stiff + b_upd) / (ms / args.steps / 1e3) / 1e9 / peak,
                              "canonical_bytes": b_canon_step,
                              "frac_canonical": b_canon_step / (ms / args.steps / 1e3) / 1e9 / peak,
                              "canonical_form": "per-GLL-point geometry layout: B_K = 4 P E (1 + "
                                                "d^2 + 1 + m) + 8 c G, B_U = (28 c + 4) G"},
            "roofline_per_point_geometry": general,
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "host_input_bytes": 2 * G * 3 * 8,
                    "repeats": {"n": len(e2e_runs), "ms_median": ms_e2e,
                                "ms_min": min(e2e_runs), "ms_max": max(e2e_runs)},
                    "form": "C-ABI job: FP64 host u0/v0 (converted to FP32 on host threads, "
                            "pinned DMA), K graph-replayed steps, seismogram read-back; h2d "
                            "amortised over K"},
            "repeats": {"n": R, "ms_per_step_median": ms / args.steps,
                        "ms_per_step_min": min(runs) / args.steps,
                        "ms_per_step_max": max(runs) / args.steps},
            "gpu_launches": launches,
            "clocks": ck,
            "cpu_baseline": cpu,
            "shots_batched": shots,
            "serving": serve,
            "simplices": simplex,
            "elastic2d": e2d,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
