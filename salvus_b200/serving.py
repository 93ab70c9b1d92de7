"""Python binding of the serving entry points (salvus_server_* in
include/salvus_b200.h): a continuous-batching request loop for
forward-modelling jobs of different mesh sizes and step counts on one GPU."""
import ctypes

import numpy as np

from .core import (_D, _DP, _I32, _I64, _VP, ACOUSTIC, COUPLED2D, ELASTIC2D, ELASTIC3D,
                   MESH_ELASTIC_TI, MeshDesc, SalvusError, SourceDesc, _check, _dp, lib)

QUEUED, RUNNING, DONE, FAILED, CANCELLED = range(5)


class JobDesc(ctypes.Structure):
    _fields_ = [("mesh", MeshDesc), ("precision", _I32), ("n_sources", _I32),
                ("sources", ctypes.POINTER(SourceDesc)), ("n_receivers", _I32), ("reserved", _I32),
                ("receivers", _DP), ("dt", _D), ("n_steps", _I64)]


class Stats(ctypes.Structure):
    _fields_ = [("submitted", _I64), ("completed", _I64), ("failed", _I64), ("running", _I64),
                ("queued", _I64), ("p50_latency_s", _D), ("p99_latency_s", _D),
                ("mean_latency_s", _D), ("gll_point_updates", _D), ("busy_seconds", _D),
                ("peak_device_bytes", _I64), ("prep_seconds", _D)]


_BOUND = False

# (name, argtypes) of the serving entry points; all return int status
SERVER_SIGNATURES = [
        ("salvus_server_create", [ctypes.c_int, _I64, _I32, _I32, ctypes.POINTER(_VP)]),
        ("salvus_server_submit", [_VP, ctypes.POINTER(JobDesc), ctypes.POINTER(_I64)]),
        ("salvus_server_poll", [_VP, _I64, ctypes.POINTER(_I32), ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
        ("salvus_server_seismograms", [_VP, _I64, _I64, _I64, _DP]),
        ("salvus_server_wait", [_VP, _I64, _D]),
        ("salvus_server_cancel", [_VP, _I64]),
        ("salvus_server_release", [_VP, _I64]),
        ("salvus_server_stats_read", [_VP, ctypes.POINTER(Stats)]),
        ("salvus_server_destroy", [_VP]),
]


def _bind():
    global _BOUND
    if _BOUND:
        return lib()
    L = lib()
    for name, args in SERVER_SIGNATURES:
        f = getattr(L, name)
        f.restype = ctypes.c_int
        f.argtypes = args
    _BOUND = True
    return L


class Server:
    def __init__(self, device=0, budget_bytes=150 * 10**9, max_running=16, chunk_steps=32):
        L = _bind()
        h = _VP()
        _check(L.salvus_server_create(device, int(budget_bytes), max_running, chunk_steps, ctypes.byref(h)))
        self.h = h
        self._meta = {}

    def close(self):
        if getattr(self, "h", None):
            lib().salvus_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, cfg, dt, n_steps, precision=0):
        """cfg: dict with shape/order/physics/vertices/cells/params, sources
        (location, center_freq, time_delay, amplitude, direction | moment_tensor),
        receivers."""
        v = np.ascontiguousarray(cfg["vertices"], dtype=np.float64)
        c = np.ascontiguousarray(cfg["cells"], dtype=np.int64)
        p = np.ascontiguousarray(cfg["params"], dtype=np.float64)
        srcs = (SourceDesc * max(1, len(cfg.get("sources", []))))()
        for k, s in enumerate(cfg.get("sources", [])):
            loc = list(s["location"]) + [0.0] * (3 - len(s["location"]))
            srcs[k].location[:] = loc
            srcs[k].center_freq, srcs[k].time_delay = s["center_freq"], s["time_delay"]
            srcs[k].amplitude = s.get("amplitude", 1.0)
            if "moment_tensor" in s:
                srcs[k].kind = 1
                srcs[k].comp[:] = list(s["moment_tensor"])
            else:
                d = list(np.atleast_1d(s.get("direction", [1.0])))
                srcs[k].comp[:] = d + [0.0] * (6 - len(d))
        rec = np.zeros((max(1, len(cfg.get("receivers", []))), 3))
        for k, r in enumerate(cfg.get("receivers", [])):
            rec[k, : len(r)] = r
        rec = np.ascontiguousarray(rec)
        flags = MESH_ELASTIC_TI if cfg["physics"] == ELASTIC3D and p.shape[0] == 6 else 0
        m = MeshDesc(cfg["shape"], cfg["order"], cfg["physics"], flags, v.shape[0], _dp(v),
                     c.shape[0], c.ctypes.data_as(ctypes.POINTER(_I64)), _dp(p))
        d = JobDesc(m, precision, len(cfg.get("sources", [])), srcs, len(cfg.get("receivers", [])), 0,
                    _dp(rec), float(dt), int(n_steps))
        jid = _I64()
        _check(lib().salvus_server_submit(self.h, ctypes.byref(d), ctypes.byref(jid)))
        comps = {ACOUSTIC: 1, ELASTIC3D: 3, ELASTIC2D: 2, COUPLED2D: 3}[cfg["physics"]]
        self._meta[jid.value] = (len(cfg.get("receivers", [])), comps, n_steps)
        return jid.value

    def poll(self, job):
        st, done, G = _I32(), _I64(), _I64()
        _check(lib().salvus_server_poll(self.h, job, ctypes.byref(st), ctypes.byref(done), ctypes.byref(G)))
        return st.value, done.value, G.value

    def wait(self, job, timeout=600.0):
        _check(lib().salvus_server_wait(self.h, job, float(timeout)))

    def seismograms(self, job, first=0, count=None):
        R, c, n = self._meta[job]
        if count is None:
            count = self.poll(job)[1] - first
        out = np.zeros((R, c, count))
        if R and count:
            _check(lib().salvus_server_seismograms(self.h, job, first, count, _dp(out)))
        return out

    def cancel(self, job):
        _check(lib().salvus_server_cancel(self.h, job))

    def release(self, job):
        _check(lib().salvus_server_release(self.h, job))

    def stats(self):
        s = Stats()
        _check(lib().salvus_server_stats_read(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}
