"""Seeded synthetic meshes and material models (file-free, like the
reference's in-memory cell-list meshes, Mesh.cpp:31-51).

Vertex order inside a cell follows the reference's right-hand (PETSc) rule:
  quad  v0(-,-) v1(+,-) v2(+,+) v3(-,+)                (QuadP1.h:98-108)
  hex   v0(-,-,-) v1(-,+,-) v2(+,+,-) v3(+,-,-)
        v4(-,-,+) v5(+,-,+) v6(+,+,+) v7(-,+,+)       (HexP1.cpp:86-122)

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
