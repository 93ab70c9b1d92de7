"""ctypes binding of the FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline legs import
this module; the product package never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

QUAD, HEX, TRI, TET = 0, 1, 2, 3
ACOUSTIC, ELASTIC3D, ELASTIC2D, COUPLED2D = 0, 1, 2, 3
Q1_Z_NOT_ADVANCED = 1 << 0
Q2_ELASTIC_SRC_UNSCALED = 1 << 1
Q3_QUAD_INVJ_AT_OUTPUT = 1 << 2
Q17_QUAD_SWAPPED_JAC = 1 << 3
FAITHFUL_RECOMPUTE = 1 << 4
K1_SPLIT_MASS = 1 << 5
K2_SOLID_NORMAL = 1 << 6
K3_INTERFACE_EDGES = 1 << 7
K4_FLUID_VP2 = 1 << 8
COUPLING_CONSISTENT = K1_SPLIT_MASS | K2_SOLID_NORMAL | K3_INTERFACE_EDGES | K4_FLUID_VP2
LITERAL = Q1_Z_NOT_ADVANCED | Q2_ELASTIC_SRC_UNSCALED | Q3_QUAD_INVJ_AT_OUTPUT | Q17_QUAD_SWAPPED_JAC

_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.c_int64


class _Desc(ctypes.Structure):
    _fields_ = [
        ("shape", ctypes.c_int), ("order", ctypes.c_int), ("physics", ctypes.c_int),
        ("n_vertices", _I64), ("vertices", _DP),
        ("n_elements", _I64), ("cells", ctypes.POINTER(_I64)),
        ("params", _DP), ("flags", ctypes.c_uint), ("threads", ctypes.c_int),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = ctypes.CDLL(path)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(_Desc)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_num_nodes.restype = _I64
        L.orc_num_nodes.argtypes = [ctypes.c_void_p]
        L.orc_num_components.argtypes = [ctypes.c_void_p]
        L.orc_node_coords.argtypes = [ctypes.c_void_p, _DP]
        L.orc_add_source.argtypes = [ctypes.c_void_p, _DP, _D, _D, _D, ctypes.c_int, _DP]
        L.orc_add_receiver.argtypes = [ctypes.c_void_p, _DP]
        L.orc_set_dirichlet.argtypes = [ctypes.c_void_p, _I64, ctypes.POINTER(_I64)]
        L.orc_set_field.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
        L.orc_get_field.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
        L.orc_inverse_mass.argtypes = [ctypes.c_void_p, _DP]
        L.orc_inverse_mass_c.argtypes = [ctypes.c_void_p, _DP]
        L.orc_apply_stiffness.argtypes = [ctypes.c_void_p, _DP, _DP]
        L.orc_run.argtypes = [ctypes.c_void_p, _I64, _D, _DP]
        L.orc_acceleration.argtypes = [ctypes.c_void_p, _D, _DP]
        L.orc_max_eigenvalue.restype = _D
        L.orc_max_eigenvalue.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64]
        L.orc_energy.restype = _D
        L.orc_energy.argtypes = [ctypes.c_void_p]
        L.orc_step_index.restype = _I64
        L.orc_step_index.argtypes = [ctypes.c_void_p]
        L.orc_gll.argtypes = [ctypes.c_int, _DP, _DP]
        L.orc_deriv_matrix.argtypes = [ctypes.c_int, _DP]
        L.orc_lagrange.argtypes = [ctypes.c_int, _D, _DP, _DP]
        L.orc_ricker.restype = _D
        L.orc_ricker.argtypes = [_D, _D, _D, _D]
        L.orc_p1_jacobian.argtypes = [ctypes.c_int, _DP, _DP, ctypes.c_uint, _DP, _DP]
        L.orc_check_hull.argtypes = [ctypes.c_int, _DP, _DP]
        L.orc_inverse_map.argtypes = [ctypes.c_int, _DP, _DP, _DP]
        for name in ("orc_element_gradient", "orc_element_grad_test", "orc_element_test",
                     "orc_element_delta"):
            getattr(L, name).argtypes = [ctypes.c_int, ctypes.c_int, _DP, ctypes.c_uint, _DP, _DP]
        L.orc_element_par.argtypes = [ctypes.c_int, ctypes.c_int, _DP, _DP]
        L.orc_simplex_tables.argtypes = [ctypes.c_int, _DP, _DP, _DP]
        L.orc_simplex_basis.argtypes = [ctypes.c_int, _DP, _DP, _DP]
        _LIB = L
    return _LIB


def _dim(shape):
    return 2 if shape in (QUAD, TRI) else 3


def _npts(shape, order):
    if shape == TRI:
        return 12
    if shape == TET:
        return 50
    return (order + 1) ** _dim(shape)


def _p(a):
    return a.ctypes.data_as(_DP)


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def gll(order):
    n = order + 1
    x, w = np.zeros(n), np.zeros(n)
    assert lib().orc_gll(order, _p(x), _p(w)) == 0
    return x, w


def deriv_matrix(order):
    n = order + 1
    D = np.zeros((n, n))
    assert lib().orc_deriv_matrix(order, _p(D)) == 0
    return D


def lagrange(order, xi):
    n = order + 1
    l, dl = np.zeros(n), np.zeros(n)
    assert lib().orc_lagrange(order, float(xi), _p(l), _p(dl)) == 0
    return l, dl


def ricker(t, f0, t0, amp):
    return lib().orc_ricker(float(t), float(f0), float(t0), float(amp))


def simplex_tables(shape):
    """(nodes [P][dim], weights [P], D [dim][P][P]) with D[k][i][q] = dphi_i/dxi_k (x_q)."""
    P, d = _npts(shape, 3), _dim(shape)
    x, w, D = np.zeros((P, 3)), np.zeros(P), np.zeros((d, P, P))
    assert lib().orc_simplex_tables(shape, _p(x), _p(w), _p(D)) == 0
    return x[:, :d], w, D


def simplex_basis(shape, ref):
    P, d = _npts(shape, 3), _dim(shape)
    r = np.zeros(3)
    r[:d] = ref
    phi, dphi = np.zeros(P), np.zeros((P, d))
    assert lib().orc_simplex_basis(shape, _p(r), _p(phi), _p(dphi)) == 0
    return phi, dphi


def _elem(fn, shape, order, vtx, flags, inp, out_shape):
    vtx, inp = _c(vtx), _c(inp)
    out = np.zeros(out_shape)
    rc = getattr(lib(), fn)(shape, order, _p(vtx), flags, _p(inp), _p(out))
    if rc:
        raise RuntimeError(lib().orc_last_error().decode())
    return out


def element_gradient(shape, order, vtx, u, flags=0):
    return _elem("orc_element_gradient", shape, order, vtx, flags, u,
                 (_npts(shape, order), _dim(shape)))


def element_grad_test(shape, order, vtx, f, flags=0):
    return _elem("orc_element_grad_test", shape, order, vtx, flags, f, (_npts(shape, order),))


def element_test(shape, order, vtx, f, flags=0):
    return _elem("orc_element_test", shape, order, vtx, flags, f, (_npts(shape, order),))


def element_delta(shape, order, vtx, ref, flags=0):
    return _elem("orc_element_delta", shape, order, vtx, flags, ref, (_npts(shape, order),))


def element_par(shape, order, par_vtx):
    par_vtx = _c(par_vtx)
    out = np.zeros(_npts(shape, order))
    assert lib().orc_element_par(shape, order, _p(par_vtx), _p(out)) == 0
    return out


def check_hull(shape, vtx, x):
    vtx, x = _c(vtx), _c(x)
    return lib().orc_check_hull(shape, _p(vtx), _p(x))


def inverse_map(shape, vtx, x):
    vtx, x = _c(vtx), _c(x)
    ref = np.zeros(3)
    rc = lib().orc_inverse_map(shape, _p(vtx), _p(x), _p(ref))
    if rc:
        raise RuntimeError(lib().orc_last_error().decode())
    return ref[: _dim(shape)]


def p1_jacobian(shape, vtx, ref, flags=0):
    d = _dim(shape)
    vtx, ref3 = _c(vtx), np.zeros(3)
    ref3[:d] = ref
    det, inv = np.zeros(1), np.zeros((d, d))
    lib().orc_p1_jacobian(shape, _p(vtx), _p(ref3), flags, _p(det), _p(inv))
    return det[0], inv


class Problem:
    """FP64 reference-restatement problem on a conforming quad / hex mesh."""

    def __init__(self, shape, order, physics, vertices, cells, params, flags=0, threads=1):
        self._keep = [_c(vertices), _c(cells, np.int64), _c(params)]
        d = _Desc()
        d.shape, d.order, d.physics = shape, order, physics
        d.n_vertices = self._keep[0].shape[0]
        d.vertices = _p(self._keep[0])
        d.n_elements = self._keep[1].shape[0]
        d.cells = self._keep[1].ctypes.data_as(ctypes.POINTER(_I64))
        d.params = _p(self._keep[2])
        d.flags, d.threads = flags, threads
        self.h = lib().orc_create(ctypes.byref(d))
        if not self.h:
            raise RuntimeError(lib().orc_last_error().decode())
        self.dim = _dim(shape)
        self.G = lib().orc_num_nodes(self.h)
        self.c = lib().orc_num_components(self.h)
        self.nrec = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def coords(self):
        x = np.zeros((self.G, self.dim))
        lib().orc_node_coords(self.h, _p(x))
        return x

    def add_source(self, x, f0, t0, amp, comp, kind=0):
        x3 = np.zeros(3)
        x3[: len(x)] = x
        comp = _c(np.atleast_1d(comp))
        rc = lib().orc_add_source(self.h, _p(x3), f0, t0, amp, kind, _p(comp))
        if rc < 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return rc

    def add_receiver(self, x):
        x3 = np.zeros(3)
        x3[: len(x)] = x
        rc = lib().orc_add_receiver(self.h, _p(x3))
        if rc < 0:
            raise RuntimeError(lib().orc_last_error().decode())
        self.nrec += 1
        return rc

    def set_dirichlet(self, nodes):
        nodes = np.ascontiguousarray(nodes, dtype=np.int64)
        assert lib().orc_set_dirichlet(self.h, len(nodes), nodes.ctypes.data_as(ctypes.POINTER(_I64))) == 0

    def set_field(self, which, vals):
        vals = _c(vals).reshape(self.G, self.c)
        assert lib().orc_set_field(self.h, {"u": 0, "v": 1}[which], _p(vals)) == 0

    def get_field(self, which):
        out = np.zeros((self.G, self.c))
        assert lib().orc_get_field(self.h, {"u": 0, "v": 1, "a": 2}[which], _p(out)) == 0
        return out

    def inverse_mass(self):
        out = np.zeros(self.G)
        lib().orc_inverse_mass(self.h, _p(out))
        return out

    def inverse_mass_components(self):
        out = np.zeros((self.G, self.c))
        lib().orc_inverse_mass_c(self.h, _p(out))
        return out

    def apply_stiffness(self, u):
        """-K u (no sources, no coupling terms)."""
        u = _c(u).reshape(self.G, self.c)
        out = np.zeros((self.G, self.c))
        lib().orc_apply_stiffness(self.h, _p(u), _p(out))
        return out

    def acceleration(self, t):
        out = np.zeros((self.G, self.c))
        lib().orc_acceleration(self.h, float(t), _p(out))
        return out

    def run(self, nsteps, dt):
        seis = np.zeros((max(self.nrec, 1), self.c, nsteps))
        rc = lib().orc_run(self.h, int(nsteps), float(dt), _p(seis))
        if rc:
            raise RuntimeError(lib().orc_last_error().decode())
        return seis[: self.nrec]

    def max_eigenvalue(self, iters=200, seed=1):
        return lib().orc_max_eigenvalue(self.h, iters, seed)

    def energy(self):
        return lib().orc_energy(self.h)
