"""Exodus II reader (no GPU): files written by scipy's independent NetCDF
classic writer with the Exodus library's names are read back bitwise --
coordinates (split and joined), multi-block connectivity converted to the
library's vertex orders (valid meshes of every shape), per-vertex parameters
NAME_<i> of each physics with the reference's VP <-> VPV fallback, the fluid
flag, side sets equal to the mesh boundary -- in CDF-1 and CDF-2; NetCDF-4
and malformed files fail loudly."""
import numpy as np
import pytest

from salvus_b200 import core, meshgen
from salvus_b200.exodus import ExodusFile

import exodus_files as xf


def per_vertex(cells, vertices, fn):
    """[E][nv] values of fn at each element's library-order vertices"""
    return fn(vertices[cells])


def vars_of(name, vals):
    return {f"{name}_{i}": vals[:, i] for i in range(vals.shape[1])}


@pytest.mark.parametrize("version", [1, 2])
@pytest.mark.parametrize("split", [True, False])
def test_quad_mesh_params_and_side_sets(tmp_path, version, split):
    V, C = meshgen.structured_quad(6, 4, 600.0, 400.0)
    exo = xf.to_exodus(C, "QUAD4")
    vp = per_vertex(C, V, lambda x: 3000.0 + x[..., 0] + 2 * x[..., 1])
    rho = per_vertex(C, V, lambda x: 2000.0 + 0.5 * x[..., 0])
    fluid = (V[C].mean(axis=1)[:, 1] > 200.0).astype(float)
    ev = {**vars_of("VP", vp), **vars_of("RHO", rho), "fluid": fluid}
    for k, nm in enumerate(["C11", "C13", "C33", "C55"]):
        ev.update(vars_of(nm, rho * (10.0 + k)))
    ss = xf.box_side_sets(V, exo, xf.QUAD_SIDES, (0, 0), (600, 400))
    path = str(tmp_path / "quad.e")
    xf.write(path, V, [exo[:10], exo[10:]], "QUAD4", ev, ss, version=version, split_coords=split)
    f = ExodusFile(path)
    assert (f.shape, f.dim, f.n_vertices, f.n_elements) == (core.QUAD, 2, len(V), len(C))
    assert f.side_set_names == ["x0", "x1", "y0", "y1"]
    v, c = f.mesh_arrays()
    assert np.array_equal(v, V) and np.array_equal(c, C)
    assert np.array_equal(f.params(core.ACOUSTIC)[0], vp)
    p2 = f.params(core.ELASTIC2D)
    assert np.array_equal(p2[0], rho) and np.array_equal(p2[4], rho * 13.0)
    pc = f.params(core.COUPLED2D)
    assert np.array_equal(pc[0], np.repeat(fluid[:, None], 4, axis=1))
    assert np.array_equal(pc[1], vp) and np.array_equal(pc[6], rho * 13.0)
    assert np.array_equal(f.variable("fluid"), fluid)
    # side sets: x0 lies on x = 0, all four together are the outer boundary
    m = f.mesh(core.ACOUSTIC, 3, device=-1)
    X = m.node_coords()
    x0 = f.side_set_nodes(m, "x0")
    assert len(x0) == 4 * 3 + 1 and np.all(X[x0, 0] == 0.0)
    allb = np.unique(np.concatenate([f.side_set_nodes(m, s) for s in f.side_set_names]))
    assert np.array_equal(allb, m.boundary_nodes())
    f.close()


def test_hex_mesh_vertex_order_and_isotropic_elastic(tmp_path):
    V, C = meshgen.structured_hex(3, 2, 2, 300.0, 200.0, 200.0)
    exo = xf.to_exodus(C, "HEX8")
    vp = per_vertex(C, V, lambda x: 6000.0 + x[..., 0] - x[..., 2])
    vs = vp / 1.8
    rho = per_vertex(C, V, lambda x: 2700.0 + x[..., 1])
    ev = {**vars_of("RHO", rho), **vars_of("VPV", vp), **vars_of("VPH", vp),
          **vars_of("VSV", vs), **vars_of("VSH", vs), **vars_of("ETA", np.ones_like(vp))}
    ss = xf.box_side_sets(V, exo, xf.HEX_SIDES, (0, 0, 0), (300, 200, 200))
    path = str(tmp_path / "hex.e")
    xf.write(path, V, [exo], "HEX8", ev, ss)
    f = ExodusFile(path)
    v, c = f.mesh_arrays()
    assert np.array_equal(c, C)
    p = f.params(core.ELASTIC3D)  # VP, VS fall back to VPV, VSV
    assert np.array_equal(p[0], rho) and np.array_equal(p[1], vp) and np.array_equal(p[2], vs)
    m = f.mesh(core.ELASTIC3D, 2, device=-1)  # right-hand orientation checked at creation
    allb = np.unique(np.concatenate([f.side_set_nodes(m, s) for s in f.side_set_names]))
    assert np.array_equal(allb, m.boundary_nodes())
    z1 = f.side_set_nodes(m, "z1")
    assert np.all(m.node_coords()[z1, 2] == 200.0) and len(z1) == 7 * 5


def test_anisotropic_elastic_model(tmp_path):
    """An anisotropic Elastic3D model: the isotropic reader refuses it, the
    six-parameter reader returns RHO VPV VPH VSV VSH ETA (ETA defaulting to
    1 when absent), and mesh() builds a transversely isotropic mesh."""
    V, C = meshgen.structured_hex(1, 1, 1, 1.0, 1.0, 1.0)
    ones = np.ones((1, 8))
    ev = {**vars_of("RHO", ones), **vars_of("VPV", ones), **vars_of("VPH", 2 * ones),
          **vars_of("VSV", ones), **vars_of("VSH", 1.5 * ones)}
    path = str(tmp_path / "aniso.e")
    xf.write(path, V, [xf.to_exodus(C, "HEX8")], "HEX8", ev)
    f = ExodusFile(path)
    with pytest.raises(core.SalvusError, match="anisotropic"):
        f.params(core.ELASTIC3D)
    p6 = f.elastic3d_params()
    want = np.stack([ones, ones, 2 * ones, ones, 1.5 * ones, ones])
    assert np.array_equal(p6, want)
    m = f.mesh(core.ELASTIC3D, 2, device=-1)
    assert m.n_nodes == 27


def test_isotropic_file_six_parameters(tmp_path):
    """VP / VS only: the six-parameter form repeats them as VPV = VPH and
    VSV = VSH with ETA = 1."""
    V, C = meshgen.structured_hex(1, 1, 1, 1.0, 1.0, 1.0)
    ones = np.ones((1, 8))
    ev = {**vars_of("RHO", 3 * ones), **vars_of("VP", 2 * ones), **vars_of("VS", ones)}
    path = str(tmp_path / "iso.e")
    xf.write(path, V, [xf.to_exodus(C, "HEX8")], "HEX8", ev)
    p6 = ExodusFile(path).elastic3d_params()
    assert np.array_equal(p6, np.stack([3 * ones, 2 * ones, 2 * ones, ones, ones, ones]))


@pytest.mark.parametrize("kind", ["tri", "tet"])
def test_simplex_meshes(tmp_path, kind):
    if kind == "tri":
        V, C = meshgen.delaunay_tri(6, 4, 600.0, 400.0, seed=2)
        et, shape, sides, hi = "TRI3", core.TRI, xf.TRI_SIDES, (600.0, 400.0)
    else:
        V, C = meshgen.kuhn_tet(2, 2, 2, 200.0, 200.0, 200.0, seed=2)
        et, shape, sides, hi = "TET4", core.TET, xf.TET_SIDES, (200.0, 200.0, 200.0)
    exo = xf.to_exodus(C, et)
    vp = per_vertex(C, V, lambda x: 4000.0 + x[..., 0])
    ss = xf.box_side_sets(V, exo, sides, (0.0,) * len(hi), hi)
    path = str(tmp_path / f"{kind}.e")
    xf.write(path, V, [exo], et, vars_of("VP", vp), ss)
    f = ExodusFile(path)
    assert f.shape == shape
    v, c = f.mesh_arrays()
    assert np.array_equal(c, C)
    assert np.array_equal(f.params(core.ACOUSTIC)[0], vp)
    m = f.mesh(core.ACOUSTIC, 3, device=-1)
    allb = np.unique(np.concatenate([f.side_set_nodes(m, s) for s in f.side_set_names]))
    assert np.array_equal(allb, m.boundary_nodes())


def test_bad_files(tmp_path):
    p4 = tmp_path / "nc4.e"
    p4.write_bytes(b"\x89HDF\r\n\x1a\n" + b"\0" * 64)
    with pytest.raises(core.SalvusError, match="HDF5"):
        ExodusFile(str(p4))
    junk = tmp_path / "junk.e"
    junk.write_bytes(b"CDF\x02" + b"\xff" * 20)
    with pytest.raises(core.SalvusError):
        ExodusFile(str(junk))
    with pytest.raises(core.SalvusError):
        ExodusFile(str(tmp_path / "missing.e"))
    V, C = meshgen.structured_quad(2, 2, 1.0, 1.0)
    path = str(tmp_path / "novars.e")
    xf.write(path, V, [xf.to_exodus(C, "QUAD4")], "QUAD4")
    f = ExodusFile(path)
    with pytest.raises(core.SalvusError, match="VP"):
        f.params(core.ACOUSTIC)
    with pytest.raises(core.SalvusError, match="fluid"):
        f.params(core.COUPLED2D)


@pytest.mark.gpu
def test_exodus_mesh_drives_the_gpu_path(tmp_path):
    """A fluid-over-solid model read from Exodus (fluid flag, per-vertex
    parameters, a Dirichlet side set) runs bitwise like the same arrays."""
    from salvus_b200 import configs
    cfg = configs.coupled_2d(nel=12, order=4)
    V, C = cfg["vertices"], cfg["cells"]
    names = ["VP", "RHO", "C11", "C13", "C33", "C55"]
    ev = {"fluid": cfg["params"][0][:, 0]}
    for k, nm in enumerate(names):
        ev.update(vars_of(nm, cfg["params"][k + 1]))
    exo = xf.to_exodus(C, "QUAD4")
    ss = xf.box_side_sets(V, exo, xf.QUAD_SIDES, (0, 0), (cfg["L"], cfg["L"]))
    path = str(tmp_path / "coupled.e")
    xf.write(path, V, [exo], "QUAD4", ev, ss)
    f = ExodusFile(path)
    runs = []
    for m in (f.mesh(core.COUPLED2D, 4),
              core.Mesh(core.QUAD, 4, core.COUPLED2D, V, C, cfg["params"])):
        p = core.Problem(m, core.FP32, dt=2e-3)
        p.set_dirichlet(f.side_set_nodes(m, "y0"))
        s = cfg["sources"][0]
        p.add_source(s["location"], s["center_freq"], s["time_delay"], s["amplitude"],
                     moment_tensor=s["moment_tensor"])
        for r in cfg["receivers"]:
            p.add_receiver(r)
        p.run(300)
        runs.append((p.seismograms(), p.get_field("u")))
    assert np.abs(runs[0][0]).max() > 0
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
