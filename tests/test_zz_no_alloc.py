"""The allocation-free stiffness entry point (salvus_apply_stiffness_noalloc).

It serves callers that cannot allocate device memory while they run (a host
framework that owns all device memory through its own pool, or code that
must not touch the allocator mid-run): they pass their own device buffers for
u and a, and the library keeps its element-local residual in a fixed array
instead of allocating one.  Checked here through the C ABI against the
ordinary path (salvus_assemble on a problem, which allocates its own
buffers): a = f - K u with no sources is -K u.  Two calls in a row, with
different inputs, must each match, since every call reuses the same array.
This file is collected last so that a failure here stops a -x run only after
every other test has run.
"""
import ctypes

import numpy as np
import pytest

from salvus_b200 import configs, core

pytestmark = pytest.mark.gpu

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


def no_alloc_path(mesh, precision, u):
    import torch
    dtype = torch.float32 if precision == core.FP32 else torch.float64
    ud = torch.tensor(u, dtype=dtype, device="cuda")
    ad = torch.full_like(ud, float("nan"))
    stream = torch.cuda.current_stream().cuda_stream
    rc = core.lib().salvus_apply_stiffness_noalloc(mesh.h, precision, ctypes.c_void_p(ud.data_ptr()),
                                                  ctypes.c_void_p(ad.data_ptr()),
                                                  ctypes.c_void_p(stream))
    if rc:
        raise core.SalvusError(rc, core.lib().salvus_last_error().decode())
    torch.cuda.synchronize()
    return ad.double().cpu().numpy()


@pytest.mark.parametrize("which,precision", [("elastic", core.FP32), ("elastic", core.FP64),
                                             ("acoustic2d", core.FP32), ("acoustic2d", core.FP64)])
def test_matches_existing_entry_point_twice(which, precision):
    cfg = (configs.elastic_hex(nel=4, order=4, n_receivers=2) if which == "elastic"
           else configs.standing_wave_2d(nel=12, order=4))
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"])
    rng = np.random.default_rng(11)
    for call in range(2):
        u = rng.standard_normal((mesh.n_nodes, mesh.n_components))
        ref = existing_path(mesh, precision, u)
        got = no_alloc_path(mesh, precision, u)
        assert np.all(np.isfinite(got)), f"call {call}: unwritten output"
        assert rel_l2(got, ref) <= TOL[precision], f"call {call}"


def test_rejects_meshes_beyond_the_scratch_limit():
    # 30^3 order-4 elastic hexes need 27000 * 125 * 3 * 4 B = 40.5 MB > 32 MiB
    cfg = configs.elastic_hex(nel=30, order=4, n_receivers=2)
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"])
    import torch
    ud = torch.zeros((mesh.n_nodes, 3), dtype=torch.float32, device="cuda")
    ad = torch.zeros_like(ud)
    rc = core.lib().salvus_apply_stiffness_noalloc(mesh.h, core.FP32, ctypes.c_void_p(ud.data_ptr()),
                                                  ctypes.c_void_p(ad.data_ptr()), None)
    assert rc == -1
    assert b"at most" in core.lib().salvus_last_error()
