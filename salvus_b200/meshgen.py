"""Seeded synthetic meshes and material models (file-free, like the
reference's in-memory cell-list meshes, Mesh.cpp:31-51).

Vertex order inside a cell follows the reference's right-hand (PETSc) rule:
  quad  v0(-,-) v1(+,-) v2(+,+) v3(-,+)                (QuadP1.h:98-108)
  hex   v0(-,-,-) v1(-,+,-) v2(+,+,-) v3(+,-,-)
        v4(-,-,+) v5(+,-,+) v6(+,+,+) v7(-,+,+)       (HexP1.cpp:86-122)

  tri   v0 -> (-1,-1), v1 -> (1,-1), v2 -> (-1,1), counter-clockwise (TriP1.cpp:56-94)
  tet   v0 -> (0,0,0), v1 -> (0,1,0), v2 -> (1,0,0), v3 -> (0,0,1), with
        det[v2-v0; v1-v0; v3-v0] > 0                  (TetP1.cpp:91-150)

Material follows the ExodusModel convention: one value per element vertex
(NAME_0 .. NAME_k, ExodusModel.cpp:455-470), P1-interpolated to GLL points.
"""
import numpy as np


def structured_quad(nx, ny, lx, ly, x0=0.0, y0=0.0):
    """Returns (vertices [nv,2] f64, cells [ne,4] i64) in element order x-fastest."""
    xs = x0 + np.linspace(0.0, lx, nx + 1)
    ys = y0 + np.linspace(0.0, ly, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    vertices = np.stack([X.ravel(), Y.ravel()], axis=1)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    i, j = i.ravel(), j.ravel()
    vid = lambda ii, jj: jj * (nx + 1) + ii
    cells = np.stack([vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)], axis=1)
    return vertices, cells.astype(np.int64)


def structured_hex(nx, ny, nz, lx, ly, lz, origin=(0.0, 0.0, 0.0)):
    """Returns (vertices [nv,3] f64, cells [ne,8] i64), element order x fastest."""
    xs = origin[0] + np.linspace(0.0, lx, nx + 1)
    ys = origin[1] + np.linspace(0.0, ly, ny + 1)
    zs = origin[2] + np.linspace(0.0, lz, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    vertices = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()

    def vid(ii, jj, kk):
        return (kk * (ny + 1) + jj) * (nx + 1) + ii

    # (r,s,t) = (x,y,z); signs per vertex as in HexP1::interpolateAtPoint
    cells = np.stack([
        vid(i, j, k), vid(i, j + 1, k), vid(i + 1, j + 1, k), vid(i + 1, j, k),
        vid(i, j, k + 1), vid(i + 1, j, k + 1), vid(i + 1, j + 1, k + 1), vid(i, j + 1, k + 1),
    ], axis=1)
    return vertices, cells.astype(np.int64)


def gaussian_random_field(shape, spacing, corr_len, seed):
    """Zero-mean, unit-std Gaussian random field on a regular vertex lattice by
    FFT synthesis with a Gaussian covariance of correlation length corr_len."""
    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in shape)
    # pad to avoid periodic wrap-around correlation
    pad = tuple(int(s + 2 * np.ceil(3 * corr_len / spacing)) for s in shape)
    noise = rng.standard_normal(pad)
    k2 = np.zeros(pad)
    for ax, n in enumerate(pad):
        k = 2 * np.pi * np.fft.fftfreq(n, d=spacing)
        sh = [1] * len(pad)
        sh[ax] = n
        k2 = k2 + (k.reshape(sh)) ** 2
    spec = np.exp(-k2 * corr_len ** 2 / 8.0)  # sqrt of a Gaussian PSD
    field = np.real(np.fft.ifftn(np.fft.fftn(noise) * spec))
    sl = tuple(slice(0, s) for s in shape)
    field = field[sl]
    field = (field - field.mean()) / field.std()
    return field


def per_element_vertex(values_at_vertices, cells):
    """Per-element, per-vertex parameter array [ne, nv] from global vertex values."""
    return np.ascontiguousarray(values_at_vertices[cells])


def ring_positions(center, radius, count, seed):
    rng = np.random.default_rng(seed)
    phi = rng.uniform(0.0, 2.0 * np.pi)
    th = 2.0 * np.pi * np.arange(count) / count + phi
    return np.stack([center[0] + radius * np.cos(th), center[1] + radius * np.sin(th)], axis=1)


def _jittered_lattice(counts, lengths, jitter, rng):
    """Regular vertex lattice with interior vertices moved by up to
    jitter x spacing (boundary vertices slide along their faces only)."""
    axes = [np.linspace(0.0, l, n + 1) for n, l in zip(counts, lengths)]
    grids = np.meshgrid(*axes[::-1], indexing="ij")[::-1]  # x fastest
    pts = np.stack([g.ravel() for g in grids], axis=1)
    h = np.array([l / n for n, l in zip(counts, lengths)])
    d = rng.uniform(-jitter, jitter, size=pts.shape) * h
    for k, l in enumerate(lengths):
        on_edge = (np.abs(pts[:, k]) < 1e-9 * l) | (np.abs(pts[:, k] - l) < 1e-9 * l)
        d[on_edge, k] = 0.0
    return pts + d


def delaunay_tri(nx, ny, lx, ly, jitter=0.3, seed=3):
    """Seeded Delaunay triangulation (scipy) of a jittered (nx+1) x (ny+1)
    point lattice over [0,lx] x [0,ly]: about 2 nx ny triangles, returned
    counter-clockwise in TriP1 vertex order."""
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    pts = _jittered_lattice((nx, ny), (lx, ly), jitter, rng)
    tri = Delaunay(pts)
    cells = tri.simplices.astype(np.int64)
    v = pts[cells]
    det = (v[:, 1, 0] - v[:, 0, 0]) * (v[:, 2, 1] - v[:, 0, 1]) - \
        (v[:, 1, 1] - v[:, 0, 1]) * (v[:, 2, 0] - v[:, 0, 0])
    neg = det < 0
    cells[neg, 1], cells[neg, 2] = cells[neg, 2].copy(), cells[neg, 1].copy()
    keep = np.abs(det) > 1e-12 * (lx * ly / (nx * ny))
    return pts, np.ascontiguousarray(cells[keep])


def delaunay_tet(nx, ny, nz, lx, ly, lz, jitter=0.06, seed=3):
    """Seeded Delaunay tetrahedralisation (scipy / qhull) of a jittered
    body-centred cubic point set over [0,lx] x [0,ly] x [0,lz]: the
    (nx+1) x (ny+1) x (nz+1) cell-corner lattice (boundary points slide along
    their faces only) plus the nx ny nz cell centres, each moved by up to
    jitter x spacing.  Its Delaunay tetrahedra stay well shaped (no slivers,
    unlike a Delaunay of a jittered cubic lattice, whose near-cospherical
    corner sets give near-flat tetrahedra and a tiny stable time step); about
    12 tetrahedra per cell, in qhull's element order.  Flat tetrahedra on the
    boundary faces (coplanar boundary points) are dropped; cells are returned
    in TetP1 order with positive orientation."""
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    corners = _jittered_lattice((nx, ny, nz), (lx, ly, lz), jitter, rng)
    h = np.array([lx / nx, ly / ny, lz / nz])
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    centres = (np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1) + 0.5) * h
    centres += rng.uniform(-jitter, jitter, size=centres.shape) * h
    pts = np.concatenate([corners, centres])
    cells = Delaunay(pts).simplices.astype(np.int64)
    v = pts[cells]
    det = np.einsum("ij,ij->i", v[:, 2] - v[:, 0], np.cross(v[:, 1] - v[:, 0], v[:, 3] - v[:, 0]))
    neg = det < 0
    cells[neg, 1], cells[neg, 2] = cells[neg, 2].copy(), cells[neg, 1].copy()
    keep = np.abs(det) > 1e-9 * float(np.prod(h))
    return pts, np.ascontiguousarray(cells[keep])


# Kuhn (Freudenthal) split of a cube into 6 tetrahedra along the main
# diagonal 0 -> 7 (corner index = i + 2 j + 4 k).
_KUHN = [(0, 1, 3, 7), (0, 1, 5, 7), (0, 2, 3, 7), (0, 2, 6, 7), (0, 4, 5, 7), (0, 4, 6, 7)]


def kuhn_tet(nx, ny, nz, lx, ly, lz, jitter=0.15, seed=3):
    """Seeded tetrahedral mesh of [0,lx] x [0,ly] x [0,lz]: a jittered vertex
    lattice whose cells are split into 6 tetrahedra each (no slivers, unlike
    a Delaunay of random points).  Cells are returned in TetP1 order with
    positive orientation."""
    rng = np.random.default_rng(seed)
    pts = _jittered_lattice((nx, ny, nz), (lx, ly, lz), jitter, rng)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()

    def vid(c):
        return ((k + (c >> 2)) * (ny + 1) + (j + ((c >> 1) & 1))) * (nx + 1) + (i + (c & 1))

    cells = np.concatenate([np.stack([vid(a), vid(b), vid(c), vid(d)], axis=1)
                            for (a, b, c, d) in _KUHN], axis=0)
    # interleave so that the 6 tetrahedra of one cube are consecutive
    cells = cells.reshape(6, -1, 4).transpose(1, 0, 2).reshape(-1, 4).astype(np.int64)
    v = pts[cells]
    det = np.einsum("ij,ij->i", v[:, 2] - v[:, 0],
                    np.cross(v[:, 1] - v[:, 0], v[:, 3] - v[:, 0]))
    neg = det < 0
    cells[neg, 1], cells[neg, 2] = cells[neg, 2].copy(), cells[neg, 1].copy()
    return pts, np.ascontiguousarray(cells)
