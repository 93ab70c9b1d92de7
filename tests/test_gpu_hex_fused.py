"""The FP32 step of elastic hexahedra that are all parallelepipeds.

Such meshes keep one inverse Jacobian per element and per-point material
records only.  The fused step (picked by the hexahedron autotuner when it is
the faster form on the problem, forced by SALVUS_HEX_STEP=fused) advances
each element's interior nodes in the stiffness kernel (one-term assembly,
inverse mass, Newmark; elements holding a source are finished by the source
kernel) while the node gather handles the shared nodes.  Checked here:
  * both step forms == three-call sequence == graph replay, bitwise (the
    interior arithmetic repeats the unfused order exactly), also with
    sources inside an element and with more sources than the fused kernel
    scans (the plain sequence then runs);
  * the fused step == the default step, bitwise;
  * parallelepiped records against per-point records
    (SALVUS_MESH_PER_POINT_GEOMETRY): same physics, FP32 rounding only;
  * a mesh of distorted hexahedra (per-point records, the column kernel)
    against the FP64 oracle;
  * every configuration the autotuner chooses between (form x CTA width)
    pinned in turn == the tuned default, bitwise.
"""
import numpy as np
import pytest

from oracle import pyoracle as po
from salvus_b200 import configs, core

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def problem(cfg, precision=core.FP32, dt=2e-3, flags=0, sources=None):
    mesh = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     cfg["params"], flags=flags)
    p = core.Problem(mesh, precision, dt=dt)
    for s in (cfg["sources"] if sources is None else sources):
        if "moment_tensor" in s:
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                         moment_tensor=s["moment_tensor"])
        else:
            p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                         direction=s["direction"])
    for r in cfg["receivers"]:
        p.add_receiver(r)
    return p


def three_call(p, n):
    for _ in range(n):
        p.assembleIntoGlobalDof()
        p.applyInverseMassMatrix()
        p.takeTimeStep()


def state(p):
    return [p.get_field(f) for f in ("u", "v", "a_")] + [p.seismograms()]


def assert_same(a, b):
    for x, y in zip(state(a), state(b)):
        assert np.array_equal(x, y)


@pytest.fixture(params=["default", "fused"])
def step_form(request, monkeypatch):
    if request.param == "fused":
        monkeypatch.setenv("SALVUS_HEX_STEP", "fused")
    return request.param


@pytest.mark.parametrize("order", [2, 4, 6])
def test_fused_equals_three_call_and_graph(order, step_form):
    cfg = configs.elastic_hex(nel=3, order=order, n_receivers=6)
    n = 70
    m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                  cfg["params"])
    dt = 0.4 * m.critical_dt(iterations=100)
    pa, pb, pc = problem(cfg, dt=dt), problem(cfg, dt=dt), problem(cfg, dt=dt)
    three_call(pa, n)
    for _ in range(n):
        pb.step()
    pc.run(n, core.RUN_GRAPH)
    assert np.abs(pa.seismograms()).max() > 0
    assert_same(pa, pb)
    assert_same(pa, pc)


def test_source_inside_an_element_interior(step_form):
    """A force at an interior GLL point's neighbourhood: the source element's
    interior nodes get their source terms in the stiffness kernel."""
    cfg = configs.elastic_hex(nel=3, order=4, n_receivers=4)
    h = cfg["L"] / 3
    src = [dict(location=(1.5 * h + 1.0, 1.5 * h - 2.0, 1.5 * h + 3.0), center_freq=1.5,
                time_delay=0.4, amplitude=1e12, direction=[0.2, -0.7, 0.4]),
           dict(location=(1.5 * h + 9.0, 1.5 * h + 5.0, 1.5 * h - 4.0), center_freq=2.0,
                time_delay=0.5, amplitude=3e11, direction=[0.0, 0.0, 1.0])]
    pa, pb = problem(cfg, sources=src), problem(cfg, sources=src)
    three_call(pa, 80)
    pb.run(80, core.RUN_GRAPH)
    assert_same(pa, pb)


def test_many_sources_run_the_plain_sequence(step_form):
    cfg = configs.elastic_hex(nel=3, order=4, n_receivers=4)
    rng = np.random.default_rng(3)
    src = [dict(location=tuple(rng.uniform(0.1, 0.9, 3) * cfg["L"]), center_freq=1.5,
                time_delay=0.5, amplitude=1e11, direction=list(rng.standard_normal(3)))
           for _ in range(20)]
    pa, pb = problem(cfg, sources=src), problem(cfg, sources=src)
    three_call(pa, 50)
    pb.run(50, core.RUN_GRAPH)
    assert_same(pa, pb)


def test_fused_switch_is_bitwise_equal(monkeypatch):
    cfg = configs.elastic_hex(nel=4, order=4, n_receivers=4)
    pa = problem(cfg)
    pa.run(60, core.RUN_PLAIN)
    monkeypatch.setenv("SALVUS_HEX_STEP", "fused")
    pb = problem(cfg)
    pb.run(60, core.RUN_PLAIN)
    assert_same(pa, pb)


@pytest.mark.parametrize("aniso", [None, configs.VTI])
def test_parallelepiped_records_match_per_point_records(aniso):
    cfg = configs.elastic_hex(nel=4, order=4, n_receivers=8, anisotropy=aniso)
    pa = problem(cfg)
    pb = problem(cfg, flags=core.MESH_PER_POINT_GEOMETRY)
    pa.run(300)
    pb.run(300)
    assert rel_l2(pa.seismograms(), pb.seismograms()) <= 1e-5
    assert rel_l2(pa.get_field("u"), pb.get_field("u")) <= 1e-5


def distorted_hex(nel=4, order=3, seed=9):
    cfg = configs.elastic_hex(nel=nel, order=order, n_receivers=6)
    V = cfg["vertices"].copy()
    h = cfg["L"] / nel
    inner = np.all((V > 0.5 * h) & (V < cfg["L"] - 0.5 * h), axis=1)
    V[inner] += np.random.default_rng(seed).uniform(-0.15 * h, 0.15 * h, size=(inner.sum(), 3))
    cfg["vertices"] = V
    # source and receivers at cell centres: on distorted hexahedra a point
    # close to a face can fall outside both neighbours' hull tests (the
    # reference's HexP1::checkHull, HexP1.cpp:8-84, restated)
    L = cfg["L"]
    cfg["sources"][0]["location"] = (L / 2 + 0.5 * h, L / 2 - 0.5 * h, L / 2 + 0.5 * h)
    cfg["receivers"] = [((i + 0.5) * h, (j + 0.5) * h, L - 0.5 * h)
                        for i, j in ((0, 1), (1, 3), (2, 0), (3, 2), (1, 1), (2, 2))]
    return cfg


# FP64: the reference's inverse map stops at a 1e-6 m residual
# (HexP1.cpp:135-187), so on distorted elements the oracle's source and
# receiver reference coordinates sit ~1e-9 off the converged ones the
# product uses; 1e-8 bounds that, well below the FP32 1e-4.
@pytest.mark.parametrize("precision,tol", [(core.FP64, 1e-8), (core.FP32, 1e-4)])
def test_distorted_hexahedra_against_oracle(precision, tol):
    cfg = distorted_hex()
    orc = po.Problem(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                     configs.oracle_params(cfg))
    dt = 0.4 * 2.0 / np.sqrt(orc.max_eigenvalue(200))
    p = problem(cfg, precision, dt)
    s = cfg["sources"][0]
    orc.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                   s["moment_tensor"], kind=1)
    for r in cfg["receivers"]:
        orc.add_receiver(r)
    n = 300
    p.run(n)
    s_o = orc.run(n, dt)
    assert np.abs(s_o).max() > 0
    assert rel_l2(p.seismograms(), s_o) <= tol


def test_fp32_field_upload_rounds_like_a_float32_cast():
    """salvus_problem_set_field converts FP64 host values to FP32 on host
    threads in pinned chunks; the bits equal a float32 cast of each value
    (round to nearest even), across chunk boundaries (86 MB of FP32 here)."""
    cfg = configs.elastic_hex(nel=48, order=4, n_receivers=2)
    p = problem(cfg)
    G = p.mesh.n_nodes
    vals = np.random.default_rng(4).standard_normal((G, 3)) * 10.0 ** np.random.default_rng(5).integers(-30, 30, (G, 3))
    vals[::997, 1] = 1.0 + 2.0 ** -24  # a tie: rounds to even (1.0)
    p.set_field("v", vals)
    got = p.get_field("v")
    assert np.array_equal(got, vals.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("order", [2, 4])
def test_autotuned_configurations_agree_bitwise(order, monkeypatch):
    """The hexahedron autotuner times the plain and fused forms with CTAs of
    128 / (N+1)^2 elements and twice that; every one of the four,
    pinned through SALVUS_HEX_CONFIG, gives the tuned default's fields and
    seismograms bitwise, and step_config reports what was pinned."""
    monkeypatch.delenv("SALVUS_HEX_STEP", raising=False)
    cfg = configs.elastic_hex(nel=4, order=order, n_receivers=5)
    m = core.Mesh(cfg["shape"], cfg["order"], cfg["physics"], cfg["vertices"], cfg["cells"],
                  cfg["params"])
    dt = 0.4 * m.critical_dt(iterations=100)
    ref = problem(cfg, dt=dt)
    form, epc = ref.step_config()
    e1 = 128 // (order + 1) ** 2
    assert form in (core.STEP_PLAIN, core.STEP_FUSED_INTERIOR) and epc in (e1, 2 * e1)
    ref.run(80, core.RUN_GRAPH)
    for f in (0, 1):
        for w in (0, 1):
            monkeypatch.setenv("SALVUS_HEX_CONFIG", f"{f},{w}")
            p = problem(cfg, dt=dt)  # a new mesh: the CTA width belongs to the mesh
            assert p.step_config() == (f, e1 * (1 + w))
            p.run(80, core.RUN_GRAPH)
            assert_same(p, ref)
