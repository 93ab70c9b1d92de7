"""The allocation-free stiffness entry point (salvus_apply_stiffness_noalloc).

It serves callers that cannot allocate device memory while they run (a host
framework that owns all device memory through its own pool, or code that
must not touch the allocator mid-run): they pass their own device buffers for
u and a, and the library keeps its element-local residual in a fixed array
instead of allocating one.  Checked here through the C ABI against the
ordinary path (salvus_assemble on a problem, which allocates its own
buffers): a = f - K u with no sources is -K u.  Two calls in a row, with
different inputs, must each match, since every call reuses the same array.
Meshes that the entry point cannot serve (FP64 on an FP32-only mesh,
fluid-solid meshes) are rejected before anything is launched; those checks
use host-only meshes and need no GPU.
This file is collected last so that a failure here stops a -x run only after
every other test has run.
"""
import ctypes

import numpy as np
import pytest

from salvus_b200 import configs, core

TOL = {core.FP32: 1e-4, core.FP64: 1e-10}


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def existing_path(mesh, precision, u):
    p = core.Problem(mesh, precision, dt=1e-3)
    p.set_field("u", u)
    p.assembleIntoGlobalDof()
    a = p.get_field("a")
    p.close()
    return a


def call(mesh_h, precision, u_ptr, a_ptr, stream):
    return core.lib().salvus_apply_stiffness_noalloc(mesh_h, precision, ctypes.c_void_p(u_ptr),
                                                    ctypes.c_void_p(a_ptr), ctypes.c_void_p(stream))


def no_alloc_path(mesh, precision, u):
    import torch
    dtype = torch.float32 if precision == core.FP32 else torch.float64
    ud = torch.tensor(u, dtype=dtype, device="cuda")
    ad = torch.full_like(ud, float("nan"))
    stream = torch.cuda.current_stream().cuda_stream
    rc = call(mesh.h, precision, ud.data_ptr(), ad.data_ptr(), stream)
    if rc:
        raise core.SalvusError(rc, core.lib().salvus_last_error().decode())
    torch.cuda.synchronize()
    return ad.double().cpu().numpy()


def make_cfg(which):
    if which == "elastic":
        return configs.elastic_hex(nel=4, order=4, n_receivers=2)
    if which == "acoustic2d":
        return configs.standing_wave_2d(nel=12, order=4)
    if which == "tet_elastic":  # FP32: the tensor-core kernel with bounded waits
        return configs.simplex_tet(n=3, physics=core.ELASTIC3D, n_receivers=2)
    if which == "tri":
        return configs.simplex_tri(nx=16, ny=8, n_receivers=2)
    raise ValueError(which)


def mesh_of(cfg, device=0, flags=0):
    return core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"], device=device, flags=flags)


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["elastic", "acoustic2d", "tet_elastic", "tri"])
@pytest.mark.parametrize("precision", [core.FP32, core.FP64])
def test_matches_existing_entry_point_twice(which, precision):
    mesh = mesh_of(make_cfg(which))
    rng = np.random.default_rng(11)
    for k in range(2):
        u = rng.standard_normal((mesh.n_nodes, mesh.n_components))
        ref = existing_path(mesh, precision, u)
        got = no_alloc_path(mesh, precision, u)
        assert np.all(np.isfinite(got)), f"call {k}: unwritten output"
        assert rel_l2(got, ref) <= TOL[precision], f"call {k}"


@pytest.mark.gpu
def test_fp32_only_mesh_serves_fp32_and_rejects_fp64_without_launching():
    import torch
    mesh = mesh_of(make_cfg("elastic"), flags=core.MESH_FP32_ONLY)
    rng = np.random.default_rng(5)
    u = rng.standard_normal((mesh.n_nodes, 3))
    got = no_alloc_path(mesh, core.FP32, u)
    ref = existing_path(mesh_of(make_cfg("elastic")), core.FP32, u)
    assert rel_l2(got, ref) <= TOL[core.FP32]
    ud = torch.zeros((mesh.n_nodes, 3), dtype=torch.float64, device="cuda")
    ad = torch.zeros_like(ud)
    before = core.launch_count()
    rc = call(mesh.h, core.FP64, ud.data_ptr(), ad.data_ptr(), 0)
    assert rc == -6  # SALVUS_E_STATE
    assert core.launch_count() == before


@pytest.mark.gpu
def test_rejects_meshes_beyond_the_scratch_limit():
    # 30^3 order-4 elastic hexes need 27000 * 125 * 3 * 4 B = 40.5 MB > 32 MiB
    import torch
    mesh = mesh_of(configs.elastic_hex(nel=30, order=4, n_receivers=2))
    ud = torch.zeros((mesh.n_nodes, 3), dtype=torch.float32, device="cuda")
    ad = torch.zeros_like(ud)
    rc = call(mesh.h, core.FP32, ud.data_ptr(), ad.data_ptr(), 0)
    assert rc == -1
    assert b"at most" in core.lib().salvus_last_error()


def test_rejects_fp64_on_fp32_only_mesh_on_the_host():
    mesh = mesh_of(make_cfg("elastic"), device=-1, flags=core.MESH_FP32_ONLY)
    dummy = np.zeros(8)
    before = core.launch_count()
    rc = call(mesh.h, core.FP64, dummy.ctypes.data, dummy.ctypes.data, 0)
    assert rc == -6  # SALVUS_E_STATE, decided before any device work
    assert b"FP32_ONLY" in core.lib().salvus_last_error()
    assert core.launch_count() == before


def test_rejects_fluid_solid_meshes_on_the_host():
    mesh = mesh_of(configs.coupled_2d(nel=6, order=2, n_receivers=2), device=-1)
    dummy = np.zeros(8)
    rc = call(mesh.h, core.FP32, dummy.ctypes.data, dummy.ctypes.data, 0)
    assert rc == -7  # SALVUS_E_UNSUPPORTED
    assert b"velocity" in core.lib().salvus_last_error()
