"""The header-only C++ facade (include/salvus/salvus.hpp) keeps the
reference's template vocabulary (Quad<Acoustic>, Hexahedron<Elastic3D>,
Order2Newmark, Ricker, Receiver, the Element::Factory-style string factory).
tests/cpp/facade_demo.cpp drives it like Main.cpp:45-66; its seismograms
must equal the Python path's bitwise (same C ABI, same kernels)."""
import json
import os
import subprocess

import numpy as np
import pytest

from salvus_b200 import core, meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def compile_demo(out):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "facade_demo.cpp"),
           "-L" + os.path.join(ROOT, "salvus_b200"), "-lsalvus_b200", "-L/usr/local/cuda/lib64",
           "-lcudart", "-Wl,-rpath," + os.path.join(ROOT, "salvus_b200"), "-o", out]
    subprocess.check_call(cmd)


def test_facade_compiles(tmp_path):
    compile_demo(str(tmp_path / "facade_demo"))
    assert os.path.exists(tmp_path / "facade_demo")


@pytest.mark.gpu
def test_facade_matches_python_path(tmp_path):
    exe = str(tmp_path / "facade_demo")
    compile_demo(exe)
    got = json.loads(subprocess.check_output([exe]).decode())

    V, C = meshgen.structured_quad(8, 8, 1e4, 1e4)
    m = core.Mesh(core.QUAD, 4, core.ACOUSTIC, V, C, np.full((1, len(C), 4), 4000.0))
    p = core.Problem(m, core.FP32, dt=2e-3)
    p.add_source((5123.0, 4987.0), 4.0, 0.3, 1.0, direction=[1.0])
    p.add_receiver((2000.0, 3000.0))
    p.add_receiver((7000.0, 6100.0))
    for _ in range(150):
        p.assembleIntoGlobalDof()
        p.applyInverseMassMatrix()
        p.takeTimeStep()
    assert np.array_equal(np.array(got["quad_acoustic"]), p.seismograms().ravel())

    V, C = meshgen.structured_hex(3, 3, 3, 600.0, 600.0, 600.0)
    E = len(C)
    par = np.stack([np.full((E, 8), x) for x in (2700.0, 6000.0, 3464.0)])
    m = core.Mesh(core.HEX, 4, core.ELASTIC3D, V, C, par)
    p = core.Problem(m, core.FP32, dt=1e-3)
    p.add_source((311.0, 287.0, 305.0), 8.0, 0.15, 1e10,
                 moment_tensor=[1.0, -0.5, 0.3, 0.2, 0.1, -0.4])
    p.add_receiver((100.0, 500.0, 600.0))
    p.run(120, core.RUN_GRAPH)
    s = p.seismograms()
    assert np.abs(s).max() > 0
    assert np.array_equal(np.array(got["hex_elastic"]), s.ravel())

    V, C = meshgen.kuhn_tet(2, 2, 2, 600.0, 600.0, 600.0, jitter=0.0)
    E = len(C)
    par = np.stack([np.full((E, 4), x) for x in (2700.0, 6000.0, 3464.0)])
    m = core.Mesh(core.TET, 3, core.ELASTIC3D, V, C, par)
    p = core.Problem(m, core.FP32, dt=5e-4)
    p.add_source((311.0, 287.0, 305.0), 8.0, 0.15, 1e10,
                 moment_tensor=[1.0, -0.5, 0.3, 0.2, 0.1, -0.4])
    p.add_receiver((100.0, 500.0, 600.0))
    p.run(120, core.RUN_GRAPH)
    s = p.seismograms()
    assert np.abs(s).max() > 0
    assert np.array_equal(np.array(got["tet_elastic"]), s.ravel())

    # fluid over solid quads with Dirichlet sides, graph replay
    V, C = meshgen.structured_quad(8, 8, 1e4, 1e4)
    E = len(C)
    fluid = (np.arange(E) // 8 >= 5).astype(np.float64)
    vals = [fluid, np.full(E, 1500.0), np.where(fluid > 0, 1000.0, 2600.0), np.full(E, 4.16e10),
            np.full(E, 1.408e10), np.full(E, 4.16e10), np.full(E, 1.376e10)]
    par = np.stack([np.repeat(x[:, None], 4, axis=1) for x in vals])
    m = core.Mesh(core.QUAD, 4, core.COUPLED2D, V, C, par)
    p = core.Problem(m, core.FP32, dt=4e-3)
    p.set_dirichlet(m.boundary_nodes())
    p.add_source((5123.0, 3987.0), 4.0, 0.3, 1e10, moment_tensor=[1.0, -0.5, 0.3])
    p.add_receiver((4000.0, 7500.0))
    p.add_receiver((6000.0, 2500.0))
    p.run(200, core.RUN_GRAPH)
    s = p.seismograms()
    assert np.abs(s[0, 0]).max() > 0 and np.abs(s[1, 1:]).max() > 0
    assert np.array_equal(np.array(got["fluid_solid"]), s.ravel())
