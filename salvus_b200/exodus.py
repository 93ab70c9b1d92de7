"""Exodus II meshes and models through the library's own reader (NetCDF
classic container, no Exodus / NetCDF library): the mesh, the material
parameters of a physics and side-set nodes for Dirichlet boundaries, as the
reference's Mesh::read / ExodusModel::read provide them (Mesh.cpp:53-86,
ExodusModel.cpp:37-81)."""
import ctypes

import numpy as np

from . import core
from .core import _check, _dp, lib

_NV = {core.QUAD: 4, core.HEX: 8, core.TRI: 3, core.TET: 4}
_NPAR = {core.ACOUSTIC: 1, core.ELASTIC3D: 3, core.ELASTIC2D: 5, core.COUPLED2D: 7}


class ExodusFile:
    def __init__(self, path):
        h = ctypes.c_void_p()
        _check(lib().salvus_exodus_open(str(path).encode(), ctypes.byref(h)))
        self.h = h
        sh, dim, nes, nss = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        nvtx, nel = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().salvus_exodus_info(self.h, ctypes.byref(sh), ctypes.byref(dim),
                                        ctypes.byref(nvtx), ctypes.byref(nel),
                                        ctypes.byref(nes), ctypes.byref(nss)))
        self.shape, self.dim = sh.value, dim.value
        self.n_vertices, self.n_elements = nvtx.value, nel.value
        self.nv = _NV[self.shape]
        self.variable_names = [self._name(lib().salvus_exodus_variable_name, i)
                               for i in range(nes.value)]
        self.side_set_names = [self._name(lib().salvus_exodus_side_set_name, i)
                               for i in range(nss.value)]

    def _name(self, fn, i):
        buf = ctypes.create_string_buffer(256)
        _check(fn(self.h, i, buf, 256))
        return buf.value.decode()

    def close(self):
        if self.h:
            lib().salvus_exodus_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mesh_arrays(self):
        """(vertices [n_vertices][dim], cells [n_elements][nv]) in the library's
        vertex orders, 0-based."""
        v = np.zeros((self.n_vertices, self.dim))
        c = np.zeros((self.n_elements, self.nv), dtype=np.int64)
        _check(lib().salvus_exodus_mesh(self.h, _dp(v), c.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return v, c

    def variable(self, name):
        out = np.zeros(self.n_elements)
        _check(lib().salvus_exodus_variable(self.h, name.encode(), _dp(out)))
        return out

    def params(self, physics):
        """Parameter array [npar][n_elements][nv] of salvus_mesh_desc for a physics."""
        out = np.zeros((_NPAR[physics], self.n_elements, self.nv))
        _check(lib().salvus_exodus_params(self.h, physics, _dp(out)))
        return out

    def elastic3d_params(self):
        """The reference's six Elastic3D parameters [6][n_elements][nv]
        RHO VPV VPH VSV VSH ETA (transversely isotropic models)."""
        out = np.zeros((6, self.n_elements, self.nv))
        _check(lib().salvus_exodus_elastic3d_params(self.h, _dp(out)))
        return out

    def mesh(self, physics, order, device=0):
        """The file's mesh and model; elastic 3-D reads the six reference
        parameters, so transversely isotropic models run as such (isotropic
        ones keep the isotropic kernels)."""
        v, c = self.mesh_arrays()
        par = self.elastic3d_params() if physics == core.ELASTIC3D else self.params(physics)
        return core.Mesh(self.shape, order, physics, v, c, par, device=device)

    def side_set_nodes(self, mesh, name):
        n = ctypes.c_int64()
        _check(lib().salvus_exodus_side_set_nodes(self.h, mesh.h, name.encode(), ctypes.byref(n), None))
        out = np.zeros(n.value, dtype=np.int64)
        _check(lib().salvus_exodus_side_set_nodes(self.h, mesh.h, name.encode(), ctypes.byref(n),
                                                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return out
