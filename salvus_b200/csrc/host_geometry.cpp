// host_geometry.cpp -- FP64 host math: GLL basis, P1 element maps, point
// location.  Used once at setup; the per-step arithmetic runs on the GPU.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "internal.h"

namespace salvus {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

const char *last_error() { return g_err; }

// Legendre P_N and its first two derivatives at x (Bonnet recurrence; the
// second derivative from the Legendre ODE away from x = +-1).
static void legendre3(int N, double x, double *p, double *dp, double *d2p) {
  double pm1 = 1.0, pc = x, dpm1 = 0.0, dpc = 1.0;
  if (N == 0) {
    *p = 1.0; *dp = 0.0; *d2p = 0.0;
    return;
  }
  for (int k = 1; k < N; ++k) {
    double pn = ((2 * k + 1) * x * pc - k * pm1) / (k + 1);
    double dpn = dpm1 + (2 * k + 1) * pc;  // P'_{k+1} = P'_{k-1} + (2k+1) P_k
    pm1 = pc; pc = pn;
    dpm1 = dpc; dpc = dpn;
  }
  *p = pc;
  *dp = dpc;
  *d2p = (2 * x * dpc - N * (N + 1.0) * pc) / (1 - x * x);
}

// GLL nodes: +-1 and the roots of P_N'; Newton on P_N' with P_N'' from the
// Legendre ODE.  Weights 2 / (N (N+1) P_N(x)^2).  D from the closed form
// D_ij = P_N(x_i) / (P_N(x_j) (x_i - x_j)), D_00 = -N(N+1)/4, D_NN = -D_00.
int make_basis(int shape, int order, Basis *b) {
  if (is_simplex(shape)) return make_simplex_basis(shape, order, b);
  if (shape != SALVUS_QUAD && shape != SALVUS_HEX)
    return fail(SALVUS_E_UNSUPPORTED, "unknown element shape %d", shape);
  const int dim = (shape == SALVUS_QUAD) ? 2 : 3;
  const int maxo = dim == 2 ? kMaxQuadOrder : kMaxHexOrder;
  if (order < 1 || order > maxo)
    return fail(SALVUS_E_UNSUPPORTED, "polynomial order %d not supported for %s (1..%d)", order,
                dim == 2 ? "quad" : "hex", maxo);
  const int N = order, n = N + 1;
  b->shape = shape; b->simplex = false;
  b->order = N; b->n = n; b->dim = dim;
  b->P = dim == 2 ? n * n : n * n * n;
  b->nv = dim == 2 ? 4 : 8;
  b->xi.assign(n, 0.0);
  b->w.assign(n, 0.0);
  b->D.assign(n * n, 0.0);
  b->xi[0] = -1.0;
  b->xi[N] = 1.0;
  for (int i = 1; i < N; ++i) {
    // Chebyshev-Gauss-Lobatto start, refined
    double x = -std::cos(M_PI * i / N);
    for (int it = 0; it < 60; ++it) {
      double p, dp, d2p;
      legendre3(N, x, &p, &dp, &d2p);
      double dx = dp / d2p;
      x -= dx;
      if (std::fabs(dx) <= 1e-16 * (1 + std::fabs(x))) break;
    }
    b->xi[i] = x;
  }
  for (int i = 0; i < n / 2; ++i) {  // enforce exact symmetry
    double m = 0.5 * (b->xi[n - 1 - i] - b->xi[i]);
    b->xi[i] = -m;
    b->xi[n - 1 - i] = m;
  }
  if (n % 2) b->xi[n / 2] = 0.0;
  std::vector<double> PN(n);
  for (int i = 0; i < n; ++i) {
    double p, dp, d2p;
    double x = b->xi[i];
    // P_N at the end points is (+-1)^N; avoid the ODE division there
    if (i == 0 || i == N) {
      p = (i == 0 && (N % 2)) ? -1.0 : 1.0;
    } else {
      legendre3(N, x, &p, &dp, &d2p);
    }
    PN[i] = p;
    b->w[i] = 2.0 / (N * (N + 1.0) * p * p);
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double v;
      if (i != j) v = PN[i] / (PN[j] * (b->xi[i] - b->xi[j]));
      else if (i == 0) v = -N * (N + 1.0) / 4.0;
      else if (i == N) v = N * (N + 1.0) / 4.0;
      else v = 0.0;
      b->D[i * n + j] = v;
    }
  return SALVUS_OK;
}

// Barycentric Lagrange values and derivatives on the GLL nodes.
void lagrange_1d(const Basis &b, double x, double *l, double *dl) {
  const int n = b.n;
  for (int j = 0; j < n; ++j) {
    double v = 1.0, dv = 0.0;
    for (int k = 0; k < n; ++k) {
      if (k == j) continue;
      double den = b.xi[j] - b.xi[k];
      dv = dv * (x - b.xi[k]) / den + v / den;
      v *= (x - b.xi[k]) / den;
    }
    l[j] = v;
    if (dl) dl[j] = dv;
  }
}

void point_ref(const Basis &b, int p, double *ref) {
  if (b.simplex) {
    for (int a = 0; a < 3; ++a) ref[a] = b.nodes[(size_t)p * 3 + a];
    return;
  }
  const int n = b.n;
  ref[0] = b.xi[p % n];
  ref[1] = b.xi[(p / n) % n];
  ref[2] = b.dim == 3 ? b.xi[p / (n * n)] : 0.0;
}

double point_weight(const Basis &b, int p) {
  if (b.simplex) return b.sw[p];
  const int n = b.n;
  double w = b.w[p % n] * b.w[(p / n) % n];
  return b.dim == 3 ? w * b.w[p / (n * n)] : w;
}

void basis_at(const Basis &b, const double *ref, double *phi, double *dphi) {
  if (b.simplex) {
    simplex_basis_at(b, ref, phi, dphi);
    return;
  }
  const int n = b.n, P = b.P;
  std::vector<double> l(3 * n, 1.0), dl(3 * n, 0.0);
  for (int a = 0; a < b.dim; ++a) lagrange_1d(b, ref[a], &l[a * n], &dl[a * n]);
  for (int q = 0; q < P; ++q) {
    const int i = q % n, j = (q / n) % n, k = b.dim == 3 ? q / (n * n) : 0;
    const double lz = b.dim == 3 ? l[2 * n + k] : 1.0, dz = b.dim == 3 ? dl[2 * n + k] : 0.0;
    phi[q] = l[i] * l[n + j] * lz;
    if (dphi) {
      dphi[q * 3 + 0] = dl[i] * l[n + j] * lz;
      dphi[q * 3 + 1] = l[i] * dl[n + j] * lz;
      dphi[q * 3 + 2] = l[i] * l[n + j] * dz;
    }
  }
}

static const double kQuadSign[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
static const double kHexSign[8][3] = {{-1, -1, -1}, {-1, 1, -1}, {1, 1, -1}, {1, -1, -1},
                                      {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

static void inverse3(const double *J, double *detJ, double *invJ);

// J[i][k] = dx_k / dxi_i; gradient = invJ * reference gradient.
void p1_jacobian(int shape, const double *vtx, const double *ref, double *detJ, double *invJ) {
  const int dim = shape_dim(shape);
  if (shape == SALVUS_TRI) {
    // reference triangle (-1,-1) (1,-1) (-1,1): rows (v1 - v0)/2, (v2 - v0)/2
    const double J[4] = {0.5 * (vtx[2] - vtx[0]), 0.5 * (vtx[3] - vtx[1]),
                         0.5 * (vtx[4] - vtx[0]), 0.5 * (vtx[5] - vtx[1])};
    const double d = J[0] * J[3] - J[1] * J[2];
    *detJ = d;
    if (invJ) {
      invJ[0] = J[3] / d; invJ[1] = -J[1] / d;
      invJ[2] = -J[2] / d; invJ[3] = J[0] / d;
    }
    return;
  }
  if (shape == SALVUS_TET) {
    // reference tetrahedron v0 (0,0,0) v1 (0,1,0) v2 (1,0,0) v3 (0,0,1):
    // rows d/dr = v2 - v0, d/ds = v1 - v0, d/dt = v3 - v0
    double J[9];
    for (int m = 0; m < 3; ++m) {
      J[m] = vtx[6 + m] - vtx[m];
      J[3 + m] = vtx[3 + m] - vtx[m];
      J[6 + m] = vtx[9 + m] - vtx[m];
    }
    inverse3(J, detJ, invJ);
    return;
  }
  if (dim == 2) {
    double J[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; ++k) {
      double dr = 0.25 * kQuadSign[k][0] * (1 + kQuadSign[k][1] * ref[1]);
      double ds = 0.25 * kQuadSign[k][1] * (1 + kQuadSign[k][0] * ref[0]);
      J[0] += dr * vtx[2 * k];
      J[1] += dr * vtx[2 * k + 1];
      J[2] += ds * vtx[2 * k];
      J[3] += ds * vtx[2 * k + 1];
    }
    double d = J[0] * J[3] - J[1] * J[2];
    *detJ = d;
    if (invJ) {
      invJ[0] = J[3] / d; invJ[1] = -J[1] / d;
      invJ[2] = -J[2] / d; invJ[3] = J[0] / d;
    }
    return;
  }
  double J[9] = {0};
  for (int k = 0; k < 8; ++k) {
    const double *sg = kHexSign[k];
    double a = 1 + sg[0] * ref[0], bb = 1 + sg[1] * ref[1], c = 1 + sg[2] * ref[2];
    double d0 = 0.125 * sg[0] * bb * c, d1 = 0.125 * sg[1] * a * c, d2 = 0.125 * sg[2] * a * bb;
    for (int m = 0; m < 3; ++m) {
      J[m] += d0 * vtx[3 * k + m];
      J[3 + m] += d1 * vtx[3 * k + m];
      J[6 + m] += d2 * vtx[3 * k + m];
    }
  }
  inverse3(J, detJ, invJ);
}

static void inverse3(const double *J, double *detJ, double *invJ) {
  double m00 = J[4] * J[8] - J[5] * J[7], m01 = J[5] * J[6] - J[3] * J[8],
         m02 = J[3] * J[7] - J[4] * J[6];
  double d = J[0] * m00 + J[1] * m01 + J[2] * m02;
  *detJ = d;
  if (invJ) {
    double id = 1.0 / d;
    invJ[0] = m00 * id;
    invJ[1] = (J[2] * J[7] - J[1] * J[8]) * id;
    invJ[2] = (J[1] * J[5] - J[2] * J[4]) * id;
    invJ[3] = m01 * id;
    invJ[4] = (J[0] * J[8] - J[2] * J[6]) * id;
    invJ[5] = (J[2] * J[3] - J[0] * J[5]) * id;
    invJ[6] = m02 * id;
    invJ[7] = (J[1] * J[6] - J[0] * J[7]) * id;
    invJ[8] = (J[0] * J[4] - J[1] * J[3]) * id;
  }
}

// Vertex weights of the P1 map: QuadP1.h:98-108, HexP1.cpp:242-298,
// TriP1::interpolateAtPoint TriP1.cpp:96-109 ([-r/2-s/2, r/2+1/2, s/2+1/2]),
// TetP1::interpolateAtPoint TetP1.cpp:45-60 ([1-r-s-t, s, r, t]).
void p1_weights(int shape, const double *ref, double *w) {
  switch (shape) {
    case SALVUS_QUAD:
      for (int k = 0; k < 4; ++k)
        w[k] = 0.25 * (1 + kQuadSign[k][0] * ref[0]) * (1 + kQuadSign[k][1] * ref[1]);
      break;
    case SALVUS_HEX:
      for (int k = 0; k < 8; ++k)
        w[k] = 0.125 * (1 + kHexSign[k][0] * ref[0]) * (1 + kHexSign[k][1] * ref[1]) *
               (1 + kHexSign[k][2] * ref[2]);
      break;
    case SALVUS_TRI:
      w[0] = -0.5 * (ref[0] + ref[1]);
      w[1] = 0.5 * (ref[0] + 1.0);
      w[2] = 0.5 * (ref[1] + 1.0);
      break;
    default:
      w[0] = 1.0 - ref[0] - ref[1] - ref[2];
      w[1] = ref[1];
      w[2] = ref[0];
      w[3] = ref[2];
      break;
  }
}

void p1_map(int shape, const double *vtx, const double *ref, double *x) {
  const int dim = shape_dim(shape), nv = shape_nv(shape);
  double w[8];
  p1_weights(shape, ref, w);
  for (int m = 0; m < dim; ++m) x[m] = 0.0;
  for (int k = 0; k < nv; ++k)
    for (int m = 0; m < dim; ++m) x[m] += w[k] * vtx[dim * k + m];
}

// Same inclusion rule as QuadP1::checkHull (QuadP1.cpp:8-39: all edge cross
// products of one sign, zeros count for both) and HexP1::checkHull
// (HexP1.cpp:8-84: no outward face normal sees the point).
//
// Simplices: barycentric coordinates of the point all >= -1e-12.  (The
// reference's TriP1::checkHull / TetP1::checkHull, TriP1.cpp:6-34 /
// TetP1.cpp:6-43, end with a "fabs(1-(l1+l2+l3)) < 1e-8 -> outside" test that
// is always true for triangles and rejects a whole face of every
// tetrahedron; the barycentric part is kept, that test is not.)
int check_hull(int shape, const double *vtx, const double *x) {
  const int dim = shape_dim(shape);
  double det, zero[3] = {0, 0, 0};
  p1_jacobian(shape, vtx, zero, &det, nullptr);
  if (!(det > 0)) return fail(SALVUS_E_INVALID, "poorly behaved element (detJ <= 0)");
  if (is_simplex(shape)) {
    double ref[3] = {0, 0, 0}, w[4];
    int rc = inverse_map(shape, vtx, x, ref);
    if (rc) return rc;
    p1_weights(shape, ref, w);
    for (int k = 0; k < shape_nv(shape); ++k)
      if (w[k] < -1e-12) return 0;
    return 1;
  }
  if (dim == 2) {
    int nneg = 0, npos = 0;
    for (int i = 0; i < 4; ++i) {
      const double *p0 = vtx + 2 * i, *p1 = vtx + 2 * ((i + 1) % 4);
      double cr = (p1[0] - p0[0]) * (x[1] - p0[1]) - (p1[1] - p0[1]) * (x[0] - p0[0]);
      if (cr < 0) ++nneg;
      else if (cr > 0) ++npos;
      else { ++nneg; ++npos; }
    }
    return (nneg == 4 || npos == 4) ? 1 : 0;
  }
  // (a, b, d) corners of each face; normal = (b - a) x (d - a) points outward
  static const int face[6][3] = {{0, 1, 3}, {4, 5, 7}, {0, 3, 4}, {2, 1, 6}, {0, 4, 1}, {2, 6, 3}};
  for (int f = 0; f < 6; ++f) {
    const double *a = vtx + 3 * face[f][0], *b = vtx + 3 * face[f][1], *d = vtx + 3 * face[f][2];
    double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    double v[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
    double nn[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    double s = nn[0] * (x[0] - a[0]) + nn[1] * (x[1] - a[1]) + nn[2] * (x[2] - a[2]);
    if (s > 0) return 0;
  }
  return 1;
}

// Newton inverse of the P1 map, iterated to machine precision (the reference
// stops at a 1e-6 physical residual, which on affine cells is already exact
// after the first step).
int inverse_map(int shape, const double *vtx, const double *x, double *ref) {
  const int dim = shape_dim(shape);
  double r[3] = {0, 0, 0};
  double prev = INFINITY;
  int stalled = 0, floor_steps = 0;
  for (int it = 0; it < 60; ++it) {
    double X[3] = {0, 0, 0}, det, inv[9];
    p1_map(shape, vtx, r, X);
    p1_jacobian(shape, vtx, r, &det, inv);
    double step_norm = 0.0;
    double dr[3] = {0, 0, 0};
    for (int a = 0; a < dim; ++a) {
      for (int b = 0; b < dim; ++b) dr[a] += inv[b * dim + a] * (x[b] - X[b]);
      step_norm = std::fmax(step_norm, std::fabs(dr[a]));
    }
    for (int a = 0; a < dim; ++a) r[a] += dr[a];
    // quadratic convergence until the step reaches the rounding floor of the
    // physical coordinates; stop once it no longer shrinks, or after three
    // steps below 1e-10 (steps at the rounding floor fluctuate)
    stalled = (step_norm >= 0.5 * prev) ? stalled + 1 : 0;
    prev = step_norm;
    floor_steps = step_norm < 1e-10 ? floor_steps + 1 : 0;
    // affine simplices: the first Newton step is exact, the second polishes
    const bool affine_done = is_simplex(shape) && it >= 1;
    if (step_norm < 1e-14 || (step_norm < 1e-10 && stalled >= 2) || floor_steps >= 3 ||
        affine_done) {
      for (int a = 0; a < dim; ++a) ref[a] = r[a];
      return SALVUS_OK;
    }
  }
  return fail(SALVUS_E_INVALID, "inverse coordinate transform did not converge");
}

int record_words(int shape, int physics, int fp64, bool ti) {
  // simplices: one record per element (affine geometry), see kernels_simplex.cuh
  if (shape == SALVUS_TRI) return 16;                        // G(3) pad s[12]
  if (shape == SALVUS_TET) return physics == SALVUS_ELASTIC3D ? (ti ? 280 : 120) : 64;
  // invJ(9) lambda' mu' [conn]; transversely isotropic invJ(9) A' C' [conn] F' L' N' [0]
  if (physics == SALVUS_ELASTIC3D) return ti ? (fp64 ? 14 : 16) : (fp64 ? 11 : 12);
  if (physics == SALVUS_ELASTIC2D) return 8;                // invJ(4) C11' C13' C33' C55'
  if (physics == SALVUS_COUPLED2D) return 8;                // per class: fluid 4 | 3, solid 8
  if (shape == SALVUS_QUAD) return fp64 ? 3 : 4;          // G00 G01 G11 [conn]
  return fp64 ? 6 : 8;                                    // G(6) [conn pad]
}

int DeviceBuffer::alloc(size_t n) {
  release();
  if (n == 0) n = 16;
  cudaError_t e = cudaMalloc(&ptr, n);
  if (e != cudaSuccess) {
    ptr = nullptr;
    return fail(SALVUS_E_OOM, "cudaMalloc(%zu bytes) failed: %s", n, cudaGetErrorString(e));
  }
  bytes = n;
  return SALVUS_OK;
}

void DeviceBuffer::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

}  // namespace salvus
