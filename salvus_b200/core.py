"""ctypes binding of libsalvus_b200.so with the reference's vocabulary.

The reference's time loop (src/cxx/Main.cpp:45-66) is

    elements, fields = problem.assembleIntoGlobalDof(elements, fields, time, time_idx, ...)
    fields = problem.applyInverseMassMatrix(fields)
    fields, time = problem.takeTimeStep(fields, time, options)

`Problem` below keeps those three method names (the element list and the
field dictionary live on the GPU, so they are not passed around), plus fused
`step()` / `run()` forms.  Errors raise `SalvusError` with the library's
message, as the reference throws std::runtime_error.
"""
import ctypes
import weakref
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsalvus_b200.so")

QUAD, HEX, TRI, TET = 0, 1, 2, 3
ACOUSTIC, ELASTIC3D, ELASTIC2D, COUPLED2D = 0, 1, 2, 3
FP32, FP64 = 0, 1
E_INVALID, E_OOM, E_CUDA, E_TIMEOUT, E_NONFINITE, E_STATE, E_UNSUPPORTED = -1, -2, -3, -4, -5, -6, -7
STEP_PLAIN, STEP_FUSED_INTERIOR = 0, 1  # salvus_problem_step_config forms
MESH_FP32_ONLY = 1  # salvus_mesh_desc.flags: build only the FP32 stiffness records
MESH_ELASTIC_TI = 2  # salvus_mesh_desc.flags: elastic3d params RHO VPV VPH VSV VSH ETA
MESH_PER_POINT_GEOMETRY = 4  # salvus_mesh_desc.flags: per-point Jacobians for parallelepipeds too
FIELD_U, FIELD_V, FIELD_A, FIELD_A_PREV = 0, 1, 2, 3
FORCE, MOMENT_TENSOR = 0, 1
RUN_PLAIN, RUN_GRAPH = 0, 1

_FIELDS = {"u": FIELD_U, "v": FIELD_V, "a": FIELD_A, "a_": FIELD_A_PREV}

_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_VP = ctypes.c_void_p


class SalvusError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class MeshDesc(ctypes.Structure):
    _fields_ = [("shape", _I32), ("order", _I32), ("physics", _I32), ("reserved", _I32),
                ("n_vertices", _I64), ("vertices", _DP), ("n_elements", _I64),
                ("cells", ctypes.POINTER(_I64)), ("params", _DP)]


class SourceDesc(ctypes.Structure):
    _fields_ = [("location", _D * 3), ("center_freq", _D), ("time_delay", _D), ("amplitude", _D),
                ("kind", _I32), ("shot", _I32), ("comp", _D * 6)]


# (name, restype, argtypes) of every entry point declared in include/salvus_b200.h
SIGNATURES = [
    ("salvus_last_error", ctypes.c_char_p, []),
    ("salvus_version", ctypes.c_char_p, []),
    ("salvus_element_tables", ctypes.c_int, [_I32, _I32, ctypes.POINTER(_I32), _DP, _DP, _DP]),
    ("salvus_mesh_create", ctypes.c_int, [ctypes.POINTER(MeshDesc), ctypes.c_int, ctypes.POINTER(_VP)]),
    ("salvus_mesh_destroy", ctypes.c_int, [_VP]),
    ("salvus_mesh_info", ctypes.c_int, [_VP, ctypes.POINTER(_I64), ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
    ("salvus_mesh_node_coords", ctypes.c_int, [_VP, _DP]),
    ("salvus_problem_status", ctypes.c_int, [_VP, _I32]),
    ("salvus_problem_set_wait_limit", ctypes.c_int, [_VP, _I64]),
    ("salvus_problem_hold_device_waits", ctypes.c_int, [_VP, _I32]),
    ("salvus_group_set_wait_limit", ctypes.c_int, [_VP, _I64]),
    ("salvus_group_clear_status", ctypes.c_int, [_VP]),
    ("salvus_mesh_layout", ctypes.c_int, [_VP, ctypes.POINTER(_I32), ctypes.POINTER(_I64)]),
    ("salvus_mesh_connectivity", ctypes.c_int, [_VP, ctypes.POINTER(_I64)]),
    ("salvus_mesh_locate_point", ctypes.c_int, [_VP, _DP, ctypes.POINTER(_I64), _DP]),
    ("salvus_mesh_inverse_mass", ctypes.c_int, [_VP, _DP]),
    ("salvus_mesh_boundary_nodes", ctypes.c_int, [_VP, ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
    ("salvus_problem_set_dirichlet", ctypes.c_int, [_VP, _I64, ctypes.POINTER(_I64)]),
    ("salvus_problem_energy", ctypes.c_int, [_VP, _DP, _DP]),
    ("salvus_exodus_open", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_VP)]),
    ("salvus_exodus_close", ctypes.c_int, [_VP]),
    ("salvus_exodus_info", ctypes.c_int, [_VP, ctypes.POINTER(_I32), ctypes.POINTER(_I32),
                                          ctypes.POINTER(_I64), ctypes.POINTER(_I64),
                                          ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
    ("salvus_exodus_mesh", ctypes.c_int, [_VP, _DP, ctypes.POINTER(_I64)]),
    ("salvus_exodus_variable_name", ctypes.c_int, [_VP, _I32, ctypes.c_char_p, _I32]),
    ("salvus_exodus_variable", ctypes.c_int, [_VP, ctypes.c_char_p, _DP]),
    ("salvus_exodus_params", ctypes.c_int, [_VP, _I32, _DP]),
    ("salvus_exodus_elastic3d_params", ctypes.c_int, [_VP, _DP]),
    ("salvus_exodus_side_set_name", ctypes.c_int, [_VP, _I32, ctypes.c_char_p, _I32]),
    ("salvus_exodus_side_set_nodes", ctypes.c_int, [_VP, _VP, ctypes.c_char_p,
                                                    ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
    ("salvus_mesh_max_eigenvalue", ctypes.c_int, [_VP, _I32, ctypes.c_uint64, _DP]),
    ("salvus_group_create", ctypes.c_int, [ctypes.POINTER(_VP), _I32, ctypes.POINTER(_VP)]),
    ("salvus_group_run", ctypes.c_int, [_VP, _I64]),
    ("salvus_group_synchronize", ctypes.c_int, [_VP]),
    ("salvus_group_destroy", ctypes.c_int, [_VP]),
    ("salvus_problem_create", ctypes.c_int, [_VP, _I32, _I32, ctypes.POINTER(_VP)]),
    ("salvus_problem_destroy", ctypes.c_int, [_VP]),
    ("salvus_problem_set_dt", ctypes.c_int, [_VP, _D]),
    ("salvus_problem_add_source", ctypes.c_int, [_VP, ctypes.POINTER(SourceDesc)]),
    ("salvus_problem_add_receiver", ctypes.c_int, [_VP, _DP]),
    ("salvus_problem_set_seismogram_capacity", ctypes.c_int, [_VP, _I64]),
    ("salvus_problem_set_field", ctypes.c_int, [_VP, _I32, _I32, _DP]),
    ("salvus_problem_get_field", ctypes.c_int, [_VP, _I32, _I32, _DP]),
    ("salvus_assemble", ctypes.c_int, [_VP]),
    ("salvus_apply_inverse_mass", ctypes.c_int, [_VP]),
    ("salvus_take_time_step", ctypes.c_int, [_VP]),
    ("salvus_step", ctypes.c_int, [_VP]),
    ("salvus_run", ctypes.c_int, [_VP, _I64, _I32]),
    ("salvus_problem_prepare_run", ctypes.c_int, [_VP, _I64]),
    ("salvus_synchronize", ctypes.c_int, [_VP]),
    ("salvus_problem_step_index", _I64, [_VP]),
    ("salvus_problem_stream", ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    ("salvus_get_seismograms", ctypes.c_int, [_VP, _I64, _I64, _DP]),
    ("salvus_problem_info", ctypes.c_int, [_VP, ctypes.POINTER(_I32), ctypes.POINTER(_I32), ctypes.POINTER(_I32)]),
    ("salvus_profile_enable", ctypes.c_int, [_VP, _I32]),
    ("salvus_profile_read", ctypes.c_int, [_VP, _I32, ctypes.POINTER(ctypes.c_char_p), _DP,
                                           ctypes.POINTER(_I64), ctypes.POINTER(_I32)]),
    ("salvus_launch_count", _I64, []),
    ("salvus_apply_stiffness_noalloc", ctypes.c_int, [_VP, _I32, _VP, _VP, _VP]),
    ("salvus_problem_autotune", ctypes.c_int, [_VP] + [ctypes.POINTER(_I32)] * 4),
    ("salvus_problem_step_config", ctypes.c_int, [_VP] + [ctypes.POINTER(_I32)] * 2),
]

_LIB = None


def lib():
    """Load the in-tree CUDA library; fails loudly when it is missing."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise SalvusError(-7, f"{LIB_PATH} is not built (python -m salvus_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def _check(rc):
    if rc != 0:
        raise SalvusError(rc, lib().salvus_last_error().decode())


def _dp(a):
    return a.ctypes.data_as(_DP)


def element_tables(shape, order):
    """(points [P][dim], weights [P], dphi [dim][P][P]) of a reference element,
    dphi[k][i][q] = d phi_i / d xi_k at point q (no GPU needed)."""
    dim = 2 if shape in (QUAD, TRI) else 3
    P = _I32()
    _check(lib().salvus_element_tables(shape, order, ctypes.byref(P), None, None, None))
    P = P.value
    x, w, D = np.zeros((P, dim)), np.zeros(P), np.zeros((dim, P, P))
    _check(lib().salvus_element_tables(shape, order, None, _dp(x), _dp(w), _dp(D)))
    return x, w, D


class Mesh:
    """Flattened mesh resident on one GPU (DMPlex mesh + Exodus model + the
    per-element precomputation of the reference, done once)."""

    def __init__(self, shape, order, physics, vertices, cells, params, device=0, flags=0):
        self.shape, self.order, self.physics = shape, order, physics
        self._v = np.ascontiguousarray(vertices, dtype=np.float64)
        self._c = np.ascontiguousarray(cells, dtype=np.int64)
        self._p = np.ascontiguousarray(params, dtype=np.float64)
        if physics == ELASTIC3D and self._p.shape[0] == 6:
            flags |= MESH_ELASTIC_TI  # RHO VPV VPH VSV VSH ETA
        d = MeshDesc(shape, order, physics, flags, self._v.shape[0], _dp(self._v), self._c.shape[0],
                     self._c.ctypes.data_as(ctypes.POINTER(_I64)), _dp(self._p))
        h = _VP()
        _check(lib().salvus_mesh_create(ctypes.byref(d), device, ctypes.byref(h)))
        self.h = h
        self._problems = weakref.WeakSet()
        G, c, P = _I64(), _I32(), _I32()
        _check(lib().salvus_mesh_info(self.h, ctypes.byref(G), ctypes.byref(c), ctypes.byref(P)))
        self.n_nodes, self.n_components, self.points_per_element = G.value, c.value, P.value
        self.dim = 2 if shape in (QUAD, TRI) else 3
        self.n_elements = self._c.shape[0]

    def close(self):
        # problems on this mesh first (when both are found unreachable in a
        # reference cycle, the collector may finalise the mesh first)
        for p in list(getattr(self, "_problems", ())):
            p.close()
        if getattr(self, "h", None):
            lib().salvus_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def layout(self):
        """(per_element_jacobian, gathered_nodes): whether one inverse
        Jacobian per element is stored, and how many nodes the fused FP32
        step assembles by node gather."""
        a, g = _I32(), _I64()
        _check(lib().salvus_mesh_layout(self.h, ctypes.byref(a), ctypes.byref(g)))
        return bool(a.value), g.value

    def node_coords(self):
        x = np.zeros((self.n_nodes, self.dim))
        _check(lib().salvus_mesh_node_coords(self.h, _dp(x)))
        return x

    def connectivity(self):
        c = np.zeros((self.n_elements, self.points_per_element), dtype=np.int64)
        _check(lib().salvus_mesh_connectivity(self.h, c.ctypes.data_as(ctypes.POINTER(_I64))))
        return c

    def locate(self, xyz):
        """(element, reference coordinates) of a physical point."""
        x = np.zeros(3)
        x[: len(xyz)] = xyz
        e, r = _I64(), np.zeros(3)
        _check(lib().salvus_mesh_locate_point(self.h, _dp(x), ctypes.byref(e), _dp(r)))
        return e.value, r[: self.dim]

    def boundary_nodes(self):
        """Global ids of the nodes on the outer boundary (ascending)."""
        n = _I64()
        _check(lib().salvus_mesh_boundary_nodes(self.h, ctypes.byref(n), None))
        out = np.zeros(n.value, dtype=np.int64)
        _check(lib().salvus_mesh_boundary_nodes(self.h, ctypes.byref(n),
                                                out.ctypes.data_as(ctypes.POINTER(_I64))))
        return out

    def inverse_mass(self):
        m = np.zeros(self.n_nodes)
        _check(lib().salvus_mesh_inverse_mass(self.h, _dp(m)))
        return m

    def max_eigenvalue(self, iterations=200, seed=1):
        out = _D()
        _check(lib().salvus_mesh_max_eigenvalue(self.h, iterations, seed, ctypes.byref(out)))
        return out.value

    def critical_dt(self, iterations=200, seed=1):
        return 2.0 / np.sqrt(self.max_eigenvalue(iterations, seed))


class Problem:
    """One wavefield on a mesh: Order2Newmark with sources and receivers."""

    def __init__(self, mesh, precision=FP32, dt=None, n_shots=1):
        self.mesh = mesh
        h = _VP()
        _check(lib().salvus_problem_create(mesh.h, precision, n_shots, ctypes.byref(h)))
        self.h = h
        mesh._problems.add(self)
        self.n_shots = n_shots
        self.precision = precision
        self.c = mesh.n_components
        self.n_receivers = 0
        if dt is not None:
            self.set_dt(dt)

    def close(self):
        if getattr(self, "h", None):
            lib().salvus_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_dt(self, dt):
        self.dt = float(dt)
        _check(lib().salvus_problem_set_dt(self.h, self.dt))

    def add_source(self, location, center_freq, time_delay, amplitude=1.0, direction=None,
                   moment_tensor=None, shot=0):
        s = SourceDesc()
        loc = list(location) + [0.0] * (3 - len(location))
        s.location[:] = loc
        s.center_freq, s.time_delay, s.amplitude = center_freq, time_delay, amplitude
        s.shot = shot
        if moment_tensor is not None:
            s.kind = MOMENT_TENSOR
            mt = [float(x) for x in moment_tensor]
            s.comp[:] = mt + [0.0] * (6 - len(mt))
        else:
            s.kind = FORCE
            d = [1.0] if direction is None else list(np.atleast_1d(direction))
            s.comp[:] = d + [0.0] * (6 - len(d))
        _check(lib().salvus_problem_add_source(self.h, ctypes.byref(s)))

    def add_receiver(self, location):
        x = np.zeros(3)
        x[: len(location)] = location
        _check(lib().salvus_problem_add_receiver(self.h, _dp(x)))
        self.n_receivers += 1

    def set_dirichlet(self, nodes):
        """Homogeneous Dirichlet on these global nodes (HomogeneousDirichlet)."""
        nodes = np.ascontiguousarray(nodes, dtype=np.int64)
        _check(lib().salvus_problem_set_dirichlet(self.h, len(nodes),
                                                  nodes.ctypes.data_as(ctypes.POINTER(_I64))))

    def energy(self):
        """(kinetic, strain) energy of the current state, FP64 compensated sums."""
        k, e = ctypes.c_double(), ctypes.c_double()
        _check(lib().salvus_problem_energy(self.h, ctypes.byref(k), ctypes.byref(e)))
        return k.value, e.value

    def set_seismogram_capacity(self, steps):
        _check(lib().salvus_problem_set_seismogram_capacity(self.h, int(steps)))

    def set_field(self, name, values, shot=0):
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(self.mesh.n_nodes, self.c)
        _check(lib().salvus_problem_set_field(self.h, _FIELDS[name], shot, _dp(v)))

    def get_field(self, name, shot=0):
        out = np.zeros((self.mesh.n_nodes, self.c))
        _check(lib().salvus_problem_get_field(self.h, _FIELDS[name], shot, _dp(out)))
        return out

    # -- the reference's three per-step calls
    def assembleIntoGlobalDof(self):
        _check(lib().salvus_assemble(self.h))

    def applyInverseMassMatrix(self):
        _check(lib().salvus_apply_inverse_mass(self.h))

    def takeTimeStep(self):
        _check(lib().salvus_take_time_step(self.h))

    # -- fused forms
    def step(self):
        _check(lib().salvus_step(self.h))

    def prepare_run(self, n_steps):
        """Capture the graphs a graph run of n_steps replays (nothing runs)."""
        _check(lib().salvus_problem_prepare_run(self.h, n_steps))

    def run(self, n_steps, mode=RUN_GRAPH):
        _check(lib().salvus_run(self.h, int(n_steps), mode))

    def set_wait_limit(self, cycles):
        """Bound (SM cycles) of the device waits of this problem's kernels;
        <= 0 restores the default (about a second)."""
        _check(lib().salvus_problem_set_wait_limit(self.h, int(cycles)))

    def hold_device_waits(self, enable=True):
        """Test hook: the tensor-core simplex kernels' workers wait on a
        barrier nothing arrives on, so launches time out (SALVUS_E_TIMEOUT)."""
        _check(lib().salvus_problem_hold_device_waits(self.h, 1 if enable else 0))

    def status(self, clear=False):
        """Raise SalvusError for a non-finite wavefield (SALVUS_E_NONFINITE) or
        a bounded device wait that gave up; clear=True resets the status
        word after reading it."""
        rc = lib().salvus_problem_status(self.h, 1 if clear else 0)
        if rc:
            raise SalvusError(rc, lib().salvus_last_error().decode())

    def synchronize(self):
        _check(lib().salvus_synchronize(self.h))

    def stream_handle(self):
        """cudaStream_t of this problem (an integer address)."""
        s = _VP()
        _check(lib().salvus_problem_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    @property
    def step_index(self):
        return lib().salvus_problem_step_index(self.h)

    def seismograms(self, first=0, count=None):
        """FP64 samples of u after steps first..first+count-1: [n_receivers][c][count]
        for one shot, [n_shots][n_receivers][c][count] for a batched problem."""
        if count is None:
            count = self.step_index - first
        out = np.zeros((self.n_shots, self.n_receivers, self.c, count))
        if self.n_receivers and count:
            _check(lib().salvus_get_seismograms(self.h, first, count, _dp(out)))
        return out[0] if self.n_shots == 1 else out

    def autotune(self):
        """(stiffness shot lanes, elements per CTA, gather shot lanes, nodes per CTA)."""
        v = [_I32() for _ in range(4)]
        _check(lib().salvus_problem_autotune(self.h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def step_config(self):
        """(form, elements per CTA) the autotuners chose: form STEP_PLAIN or
        STEP_FUSED_INTERIOR (bitwise the same fields); runs the tuning first
        if needed."""
        v = [_I32() for _ in range(2)]
        _check(lib().salvus_problem_step_config(self.h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def profile(self, enable=True):
        _check(lib().salvus_profile_enable(self.h, 1 if enable else 0))

    def profile_read(self):
        n = 16
        names = (ctypes.c_char_p * n)()
        ms = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int64)
        k = _I32()
        _check(lib().salvus_profile_read(self.h, n, names, _dp(ms), cnt.ctypes.data_as(ctypes.POINTER(_I64)),
                                         ctypes.byref(k)))
        return {names[i].decode(): (ms[i], int(cnt[i])) for i in range(k.value)}


class Group:
    """FP32 single-shot problems of one element class (acoustic quads or
    elastic hexahedra of one order) advanced together, one launch per step
    stage for all members; each member's result is bitwise its solo result."""

    def __init__(self, problems):
        self.problems = list(problems)
        arr = (_VP * len(self.problems))(*[p.h for p in self.problems])
        h = _VP()
        _check(lib().salvus_group_create(arr, len(self.problems), ctypes.byref(h)))
        self.h = h

    def run(self, n_steps):
        _check(lib().salvus_group_run(self.h, int(n_steps)))

    def synchronize(self):
        _check(lib().salvus_group_synchronize(self.h))

    def set_wait_limit(self, cycles):
        _check(lib().salvus_group_set_wait_limit(self.h, int(cycles)))

    def clear_status(self):
        _check(lib().salvus_group_clear_status(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().salvus_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def launch_count():
    return lib().salvus_launch_count()
