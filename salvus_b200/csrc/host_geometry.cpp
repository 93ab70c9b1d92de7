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
  const int dim = (shape == SALVUS_QUAD) ? 2 : 3;
  const int maxo = dim == 2 ? kMaxQuadOrder : kMaxHexOrder;
  if (order < 1 || order > maxo)
    return fail(SALVUS_E_UNSUPPORTED, "polynomial order %d not supported for %s (1..%d)", order,
                dim == 2 ? "quad" : "hex", maxo);
  const int N = order, n = N + 1;
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

static const double kQuadSign[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
static const double kHexSign[8][3] = {{-1, -1, -1}, {-1, 1, -1}, {1, 1, -1}, {1, -1, -1},
                                      {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

// J[i][k] = dx_k / dxi_i; gradient = invJ * reference gradient.
void p1_jacobian(int dim, const double *vtx, const double *ref, double *detJ, double *invJ) {
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

void p1_map(int dim, const double *vtx, const double *ref, double *x) {
  const int nv = dim == 2 ? 4 : 8;
  for (int m = 0; m < dim; ++m) x[m] = 0.0;
  for (int k = 0; k < nv; ++k) {
    double wk = dim == 2 ? 0.25 * (1 + kQuadSign[k][0] * ref[0]) * (1 + kQuadSign[k][1] * ref[1])
                         : 0.125 * (1 + kHexSign[k][0] * ref[0]) * (1 + kHexSign[k][1] * ref[1]) *
                               (1 + kHexSign[k][2] * ref[2]);
    for (int m = 0; m < dim; ++m) x[m] += wk * vtx[dim * k + m];
  }
}

// Same inclusion rule as QuadP1::checkHull (QuadP1.cpp:8-39: all edge cross
// products of one sign, zeros count for both) and HexP1::checkHull
// (HexP1.cpp:8-84: no outward face normal sees the point).
int check_hull(int dim, const double *vtx, const double *x) {
  double det, zero[3] = {0, 0, 0};
  p1_jacobian(dim, vtx, zero, &det, nullptr);
  if (!(det > 0)) return fail(SALVUS_E_INVALID, "poorly behaved element (detJ <= 0)");
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
int inverse_map(int dim, const double *vtx, const double *x, double *ref) {
  double r[3] = {0, 0, 0};
  double prev = INFINITY;
  int stalled = 0;
  for (int it = 0; it < 60; ++it) {
    double X[3] = {0, 0, 0}, det, inv[9];
    p1_map(dim, vtx, r, X);
    p1_jacobian(dim, vtx, r, &det, inv);
    double step_norm = 0.0;
    double dr[3] = {0, 0, 0};
    for (int a = 0; a < dim; ++a) {
      for (int b = 0; b < dim; ++b) dr[a] += inv[b * dim + a] * (x[b] - X[b]);
      step_norm = std::fmax(step_norm, std::fabs(dr[a]));
    }
    for (int a = 0; a < dim; ++a) r[a] += dr[a];
    // quadratic convergence until the step reaches the rounding floor of the
    // physical coordinates; stop once it no longer shrinks
    stalled = (step_norm >= 0.5 * prev) ? stalled + 1 : 0;
    prev = step_norm;
    if (step_norm < 1e-14 || (step_norm < 1e-10 && stalled >= 2)) {
      for (int a = 0; a < dim; ++a) ref[a] = r[a];
      return SALVUS_OK;
    }
  }
  return fail(SALVUS_E_INVALID, "inverse coordinate transform did not converge");
}

int record_words(int shape, int physics, int fp64) {
  if (physics == SALVUS_ELASTIC3D) return fp64 ? 11 : 12;  // invJ(9) lambda' mu' [conn]
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
