/*
 * oracle.c -- FP64 CPU restatement of the Salvus spectral-element time step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  The CUDA product never links,
 * loads or calls this file.  Each function cites the reference lines it
 * restates; reference paths are relative to the reference project root.
 *
 * Parity is pinned by (a) the reference's own sympy-generated GLL / Lagrange
 * tables (golden fixtures produced from the reference sources), (b) the
 * reference's element KATs restated as properties, (c) the Ricker closed
 * form, and (d) the analytic Neumann standing wave.
 */
#include "oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* quads up to order 10 (TensorQuad.h:69), hexes up to order 6 (the
 * reference's order7_hex.c is missing, Hexahedra.h:14-17). */
#define ORC_MAX_N 11
#define ORC_MAX_P 343

static __thread char g_err[512];
static void set_err(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}
const char *orc_last_error(void) { return g_err; }

/* ------------------------------------------------------------------------ */
/* Legendre polynomial P_N(x) and P_{N-1}(x) by the three-term recurrence.   */
static void legendre(int N, double x, double *pn, double *pnm1) {
  double p0 = 1.0, p1 = x;
  if (N == 0) { *pn = 1.0; *pnm1 = 0.0; return; }
  for (int k = 2; k <= N; ++k) {
    double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  *pn = p1;
  *pnm1 = p0;
}

/* GLL points = roots of (1-x^2) P_N'(x); weights 2/(N(N+1) P_N(x_i)^2).
 * Restates quadrature_points_weights.py:55-93 (the generator of
 * gll_coordinates_orderN_square / gll_weights_orderN_square,
 * src/cxx/Element/HyperCube/Quad/Autogen/order4_square.c:131-149). */
int orc_gll(int order, double *pts, double *wts) {
  if (order < 1 || order >= ORC_MAX_N) { set_err("order %d unsupported", order); return -1; }
  const int N = order, n = N + 1;
  for (int i = 0; i < n; ++i) {
    double x = -cos(M_PI * i / N);
    if (i > 0 && i < N) {
      /* Newton on q(x) = P_{N+1} - P_{N-1}; q' = (2N+1) P_N. */
      for (int it = 0; it < 100; ++it) {
        double pn, pnm1, pnp1, dummy;
        legendre(N, x, &pn, &pnm1);
        legendre(N + 1, x, &pnp1, &dummy);
        double dx = (pnp1 - pnm1) / ((2.0 * N + 1.0) * pn);
        x -= dx;
        if (fabs(dx) < 1e-17) break;
      }
    }
    pts[i] = x;
  }
  /* exact antisymmetry */
  for (int i = 0; i < n / 2; ++i) {
    double m = 0.5 * (pts[n - 1 - i] - pts[i]);
    pts[i] = -m;
    pts[n - 1 - i] = m;
  }
  if (n % 2) pts[n / 2] = 0.0;
  pts[0] = -1.0;
  pts[N] = 1.0;
  if (wts) {
    for (int i = 0; i < n; ++i) {
      double pn, pnm1;
      legendre(N, pts[i], &pn, &pnm1);
      wts[i] = 2.0 / (N * (N + 1.0) * pn * pn);
    }
  }
  return 0;
}

/* D[i][j] = l_j'(xi_i) -- the layout of mGrd (TensorQuad.cpp:107-142,
 * Hexahedra.cpp:535-577).  Barycentric form; diagonal = minus row sum. */
int orc_deriv_matrix(int order, double *D) {
  double x[ORC_MAX_N], lam[ORC_MAX_N];
  if (orc_gll(order, x, NULL)) return -1;
  const int n = order + 1;
  for (int j = 0; j < n; ++j) {
    double prod = 1.0;
    for (int k = 0; k < n; ++k)
      if (k != j) prod *= (x[j] - x[k]);
    lam[j] = 1.0 / prod;
  }
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) {
      if (i == j) continue;
      double v = (lam[j] / lam[i]) / (x[i] - x[j]);
      D[i * n + j] = v;
      s += v;
    }
    D[i * n + i] = -s;
  }
  return 0;
}

/* 1-D Lagrange basis on GLL nodes and its derivative at xi
 * (code_generator.py:13-43, interpolate_orderN_square). */
int orc_lagrange(int order, double xi, double *l, double *dl) {
  double x[ORC_MAX_N];
  if (orc_gll(order, x, NULL)) return -1;
  const int n = order + 1;
  for (int j = 0; j < n; ++j) {
    double v = 1.0;
    for (int k = 0; k < n; ++k)
      if (k != j) v *= (xi - x[k]) / (x[j] - x[k]);
    l[j] = v;
    if (dl) {
      double d = 0.0;
      for (int m = 0; m < n; ++m) {
        if (m == j) continue;
        double t = 1.0 / (x[j] - x[m]);
        for (int k = 0; k < n; ++k)
          if (k != j && k != m) t *= (xi - x[k]) / (x[j] - x[k]);
        d += t;
      }
      dl[j] = d;
    }
  }
  return 0;
}

/* Ricker::fire, src/cxx/Source/Ricker.cpp:27-33. */
double orc_ricker(double t, double f0, double t0, double amp) {
  const double factor = M_PI * M_PI * f0 * f0 * (t - t0) * (t - t0);
  return amp * ((1 - 2 * factor) * exp(-1 * factor));
}

/* ------------------------------------------------------------------------ */
/* P3 simplex tables.                                                        */
/* Nodal basis of the mass-lumped P3 triangle (P3 + cubic bubble x P1, 12
 * nodes) and tetrahedron (P3 + face bubbles x P2 + interior bubble x P2, 50
 * nodes): phi_i(x) = sum_m mono_m(x) C[m][i] with C = V^-1, V[q][m] =
 * mono_m(x_q), exactly as p3ElementPolynomials builds it
 * (triangle_points_weights_polys.py:62-97, tetrahedra_points_weights_polys.py:55-105),
 * and the derivative tables are d mono / d xi at the nodes times C
 * (genP3code, ...:133-160 / :200-225). */
#define ORC_SP 50
typedef struct {
  int P, dim;
  double x[ORC_SP][3];
  double w[ORC_SP];
  double D[3][ORC_SP * ORC_SP]; /* D[k][i*P+q] = d phi_i / d xi_k (x_q) */
  double C[ORC_SP * ORC_SP];    /* C[m*P+i] */
} stab_t;
static stab_t g_stab[2];        /* [0] triangle, [1] tetrahedron */
static int g_stab_ok[2];

/* value and gradient of a polynomial factor */
typedef struct { double v, d[3]; } dual_t;
static dual_t dl_var(double x, int k) { dual_t r = {x, {0, 0, 0}}; r.d[k] = 1; return r; }
static dual_t dl_const(double c) { dual_t r = {c, {0, 0, 0}}; return r; }
static dual_t dl_mul(dual_t a, dual_t b) {
  dual_t r = {a.v * b.v, {0, 0, 0}};
  for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
static dual_t dl_add(dual_t a, dual_t b) {
  dual_t r = {a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}};
  return r;
}
static dual_t dl_scale(dual_t a, double c) {
  dual_t r = {a.v * c, {a.d[0] * c, a.d[1] * c, a.d[2] * c}};
  return r;
}
static dual_t dl_pow(dual_t a, int e) {
  dual_t r = dl_const(1);
  for (int i = 0; i < e; ++i) r = dl_mul(r, a);
  return r;
}

/* Monomial list of the triangle generator (triangle_points_weights_polys.py:63-69):
 * P3 = [1, r, s, rs, r^2, s^2, r^3, s^3, r^2 s, r s^2], then b [r, s] with
 * b = (-r-s)(s+1)(r+1). */
static void tri_monomials(const double *x, dual_t *m) {
  dual_t r = dl_var(x[0], 0), s = dl_var(x[1], 1), one = dl_const(1);
  dual_t b = dl_mul(dl_mul(dl_add(dl_scale(r, -1), dl_scale(s, -1)), dl_add(s, one)), dl_add(r, one));
  m[0] = one; m[1] = r; m[2] = s; m[3] = dl_mul(r, s);
  m[4] = dl_pow(r, 2); m[5] = dl_pow(s, 2); m[6] = dl_pow(r, 3); m[7] = dl_pow(s, 3);
  m[8] = dl_mul(dl_pow(r, 2), s); m[9] = dl_mul(r, dl_pow(s, 2));
  m[10] = dl_mul(r, b); m[11] = dl_mul(s, b);
}

/* Monomial list of the tetrahedron generator (tetrahedra_points_weights_polys.py:55-83). */
static void tet_monomials(const double *x, dual_t *m) {
  dual_t r = dl_var(x[0], 0), s = dl_var(x[1], 1), t = dl_var(x[2], 2), one = dl_const(1);
  dual_t l0 = dl_add(one, dl_scale(dl_add(dl_add(r, s), t), -1)); /* 1 - r - s - t */
  dual_t b1 = dl_mul(dl_mul(r, s), l0), b2 = dl_mul(dl_mul(r, t), l0), b3 = dl_mul(dl_mul(t, s), l0);
  dual_t b4 = dl_mul(dl_mul(r, s), t), bt = dl_mul(b4, l0);
  dual_t rr = dl_add(one, dl_scale(dl_add(r, t), -1)), ss = dl_add(one, dl_scale(dl_add(s, t), -1));
  int k = 0;
  /* P3 */
  m[k++] = one; m[k++] = r; m[k++] = dl_pow(r, 2); m[k++] = dl_pow(r, 3);
  m[k++] = s; m[k++] = dl_pow(s, 2); m[k++] = dl_pow(s, 3);
  m[k++] = t; m[k++] = dl_pow(t, 2); m[k++] = dl_pow(t, 3);
  m[k++] = dl_mul(r, s); m[k++] = dl_mul(dl_pow(r, 2), s); m[k++] = dl_mul(r, dl_pow(s, 2));
  m[k++] = dl_mul(r, t); m[k++] = dl_mul(dl_pow(r, 2), t); m[k++] = dl_mul(r, dl_pow(t, 2));
  m[k++] = dl_mul(s, t); m[k++] = dl_mul(dl_pow(s, 2), t); m[k++] = dl_mul(s, dl_pow(t, 2));
  m[k++] = dl_mul(dl_mul(r, s), t);
  /* interior bubble x [1, r, s, t, rs, rt, st, r^2, s^2, t^2] */
  dual_t p1t[10] = {one, r, s, t, dl_mul(r, s), dl_mul(r, t), dl_mul(s, t),
                    dl_pow(r, 2), dl_pow(s, 2), dl_pow(t, 2)};
  for (int i = 0; i < 10; ++i) m[k++] = dl_mul(bt, p1t[i]);
  /* face bubbles x P2 pieces */
  dual_t f1[5] = {r, s, dl_mul(r, s), dl_pow(r, 2), dl_pow(s, 2)};
  dual_t f2[5] = {r, t, dl_mul(r, t), dl_pow(r, 2), dl_pow(t, 2)};
  dual_t f3[5] = {t, s, dl_mul(t, s), dl_pow(t, 2), dl_pow(s, 2)};
  dual_t f4[5] = {rr, ss, dl_mul(rr, ss), dl_pow(rr, 2), dl_pow(ss, 2)};
  for (int i = 0; i < 5; ++i) m[k++] = dl_mul(b1, f1[i]);
  for (int i = 0; i < 5; ++i) m[k++] = dl_mul(b2, f2[i]);
  for (int i = 0; i < 5; ++i) m[k++] = dl_mul(b3, f3[i]);
  for (int i = 0; i < 5; ++i) m[k++] = dl_mul(b4, f4[i]);
}

/* Reference nodes in PETSc closure order (face, edges, vertices) of
 * p3ReferenceNodes (triangle_points_weights_polys.py:26-47), 4-digit values
 * as the generator states them; weights of p3QuadratureWeights (:14-24). */
static void tri_nodes(stab_t *t) {
  static const double rs[12][2] = {
      {-0.5853, -0.5853}, {0.1706, -0.5853}, {-0.5853, 0.1706}, {-0.413, -1.0},
      {0.413, -1.0},      {0.413, -0.413},   {-0.413, 0.413},   {-1.0, 0.413},
      {-1.0, -0.413},     {-1.0, -1.0},      {1.0, -1.0},       {-1.0, 1.0}};
  const double s7 = sqrt(7.0);
  const double ws = 2 * (919 * s7 + 2471) / (124080 * s7 + 330960);
  const double wa = 2 * (s7 * pow(2 + s7, 4)) / (25280 + 9520 * s7);
  const double wb = 2 * (147 + 42 * s7) / (400 * s7 + 1280);
  for (int q = 0; q < 12; ++q) {
    t->x[q][0] = rs[q][0]; t->x[q][1] = rs[q][1]; t->x[q][2] = 0;
    t->w[q] = q < 3 ? wb : q < 9 ? wa : ws;
  }
}

/* BuildNodesTetrahedraP3 (BuildNodesTetrahedraP3.py:10-313): interior
 * orbits (gamma, delta), two face orbits per face (beta1, beta2), two points
 * per edge (alpha), then the corners; the constants and weights (x6 for the
 * unit-volume normalisation) are those of Chin-Joe-Kong, Mulder and Van
 * Veldhuizen (1999) as quoted in p3QuadratureWeights
 * (tetrahedra_points_weights_polys.py:15-45). */
static void tet_nodes(stab_t *t) {
  const double beta1 = 0.1972862280257976, beta2 = 0.4256461243139345;
  const double alpha = 0.2928294047674109, gamma = 0.9503775858394107e-01;
  const double delta = 0.1252462362578136;
  static const double O[3] = {0, 0, 0}, X[3] = {1, 0, 0}, Y[3] = {0, 1, 0}, Z[3] = {0, 0, 1};
  const double *R[4] = {O, X, Y, Z};
  int k = 0;
  /* interior A: corner pulled towards the opposite face centroid */
  for (int c = 0; c < 4; ++c) {
    for (int m = 0; m < 3; ++m) {
      double cen = 0;
      for (int o = 0; o < 4; ++o)
        if (o != c) cen += R[o][m];
      t->x[k][m] = (1 - 3 * gamma) * R[c][m] + 3 * gamma * (cen / 3.0);
    }
    ++k;
  }
  /* interior B: between opposite edge midpoints */
  static const int pairs[6][4] = {{0, 3, 1, 2}, {0, 1, 2, 3}, {0, 2, 1, 3},
                                  {1, 2, 0, 3}, {2, 3, 0, 1}, {1, 3, 0, 2}};
  for (int i = 0; i < 6; ++i, ++k)
    for (int m = 0; m < 3; ++m) {
      double a = 0.5 * (R[pairs[i][0]][m] + R[pairs[i][1]][m]);
      double b = 0.5 * (R[pairs[i][2]][m] + R[pairs[i][3]][m]);
      t->x[k][m] = (1 - 2 * delta) * a + 2 * delta * b;
    }
  /* faces: (O,Y,X) (O,Z,Y) (O,X,Z) (X,Y,Z), beta1 orbit then beta2 orbit */
  const double *F[4][3] = {{O, Y, X}, {O, Z, Y}, {O, X, Z}, {X, Y, Z}};
  for (int f = 0; f < 4; ++f)
    for (int o = 0; o < 2; ++o) {
      const double beta = o == 0 ? beta1 : beta2;
      for (int i = 0; i < 3; ++i, ++k)
        for (int m = 0; m < 3; ++m) {
          double mid = 0.5 * (F[f][(i + 1) % 3][m] + F[f][(i + 2) % 3][m]);
          t->x[k][m] = (1 - 2 * beta) * F[f][i][m] + 2 * beta * mid;
        }
    }
  /* edges */
  const double *Ed[6][2] = {{O, Y}, {Y, X}, {X, O}, {O, Z}, {Z, Y}, {X, Z}};
  for (int e = 0; e < 6; ++e)
    for (int o = 0; o < 2; ++o, ++k)
      for (int m = 0; m < 3; ++m) {
        double a = o == 0 ? 1 - alpha : alpha;
        t->x[k][m] = a * Ed[e][0][m] + (1 - a) * Ed[e][1][m];
      }
  /* corners v0..v3 = (0,0,0) (0,1,0) (1,0,0) (0,0,1) (TetP1.cpp:153-199 map) */
  const double *Cn[4] = {O, Y, X, Z};
  for (int c = 0; c < 4; ++c, ++k)
    for (int m = 0; m < 3; ++m) t->x[k][m] = Cn[c][m];
  const double w0 = 0.2143608668049743e-03 * 6, wa = 0.8268179517797114e-03 * 6;
  const double wb1 = 0.1840177904191860e-02 * 6, wb2 = 0.1831324329245650e-02 * 6;
  const double wg = 0.7542468904648131e-02 * 6, wd = 0.1360991755970793e-01 * 6;
  for (int q = 0; q < 50; ++q) {
    double w;
    if (q < 4) w = wg;
    else if (q < 10) w = wd;
    else if (q < 34) w = ((q - 10) % 6) < 3 ? wb1 : wb2;
    else if (q < 46) w = wa;
    else w = w0;
    t->w[q] = w;
  }
}

/* In-place inverse by Gauss-Jordan elimination with partial pivoting
 * (extended precision). */
static int invert_ld(int n, long double *A) {
  long double *I = (long double *)calloc((size_t)n * n, sizeof(long double));
  if (!I) return -1;
  for (int i = 0; i < n; ++i) I[i * n + i] = 1;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (fabsl(A[r * n + c]) > fabsl(A[piv * n + c])) piv = r;
    if (A[piv * n + c] == 0) { free(I); return -1; }
    if (piv != c)
      for (int k = 0; k < n; ++k) {
        long double x = A[c * n + k]; A[c * n + k] = A[piv * n + k]; A[piv * n + k] = x;
        x = I[c * n + k]; I[c * n + k] = I[piv * n + k]; I[piv * n + k] = x;
      }
    long double d = A[c * n + c];
    for (int k = 0; k < n; ++k) { A[c * n + k] /= d; I[c * n + k] /= d; }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      long double f = A[r * n + c];
      if (f == 0) continue;
      for (int k = 0; k < n; ++k) { A[r * n + k] -= f * A[c * n + k]; I[r * n + k] -= f * I[c * n + k]; }
    }
  }
  memcpy(A, I, sizeof(long double) * (size_t)n * n);
  free(I);
  return 0;
}

static void simplex_monomials(int tet, const double *x, dual_t *m) {
  if (tet) tet_monomials(x, m);
  else tri_monomials(x, m);
}

static int build_stab(int tet) {
  stab_t *t = &g_stab[tet];
  t->P = tet ? 50 : 12;
  t->dim = tet ? 3 : 2;
  const int P = t->P;
  if (tet) tet_nodes(t);
  else tri_nodes(t);
  long double *V = (long double *)malloc(sizeof(long double) * P * P);
  if (!V) return -1;
  dual_t m[ORC_SP];
  for (int q = 0; q < P; ++q) {
    simplex_monomials(tet, t->x[q], m);
    for (int j = 0; j < P; ++j) V[q * P + j] = m[j].v;
  }
  if (invert_ld(P, V)) { free(V); return -1; }
  for (int i = 0; i < P * P; ++i) t->C[i] = (double)V[i];
  for (int q = 0; q < P; ++q) {
    simplex_monomials(tet, t->x[q], m);
    for (int k = 0; k < t->dim; ++k)
      for (int i = 0; i < P; ++i) {
        long double s = 0;
        for (int j = 0; j < P; ++j) s += (long double)m[j].d[k] * V[j * P + i];
        t->D[k][i * P + q] = (double)s;
      }
  }
  free(V);
  return 0;
}

__attribute__((constructor)) static void init_simplex_tables(void) {
  g_stab_ok[0] = build_stab(0) == 0;
  g_stab_ok[1] = build_stab(1) == 0;
}

static const stab_t *stab_for(int shape) {
  int k = shape == ORC_TRI ? 0 : shape == ORC_TET ? 1 : -1;
  if (k < 0 || !g_stab_ok[k]) return NULL;
  return &g_stab[k];
}

int orc_simplex_tables(int shape, double *nodes, double *weights, double *D) {
  const stab_t *t = stab_for(shape);
  if (!t) { set_err("no simplex tables for shape %d", shape); return -1; }
  const int P = t->P;
  for (int q = 0; q < P; ++q) {
    if (nodes) for (int m = 0; m < 3; ++m) nodes[q * 3 + m] = t->x[q][m];
    if (weights) weights[q] = t->w[q];
  }
  if (D) for (int k = 0; k < t->dim; ++k) memcpy(D + (size_t)k * P * P, t->D[k], sizeof(double) * P * P);
  return 0;
}

int orc_simplex_basis(int shape, const double *ref, double *phi, double *dphi) {
  const stab_t *t = stab_for(shape);
  if (!t) { set_err("no simplex tables for shape %d", shape); return -1; }
  const int P = t->P;
  dual_t m[ORC_SP];
  simplex_monomials(shape == ORC_TET, ref, m);
  for (int i = 0; i < P; ++i) {
    long double v = 0, d[3] = {0, 0, 0};
    for (int j = 0; j < P; ++j) {
      long double c = t->C[j * P + i];
      v += c * m[j].v;
      for (int k = 0; k < t->dim; ++k) d[k] += c * m[j].d[k];
    }
    if (phi) phi[i] = (double)v;
    if (dphi) for (int k = 0; k < t->dim; ++k) dphi[i * t->dim + k] = (double)d[k];
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* P1 geometry.                                                              */
/* Quad vertex signs (QuadP1.h:98-108): v0(-,-) v1(+,-) v2(+,+) v3(-,+).     */
static const double QS[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
/* Hex vertex signs (HexP1.cpp:86-122, 242-298): PETSc right-hand order.    */
static const double HS[8][3] = {{-1, -1, -1}, {-1, 1, -1}, {1, 1, -1}, {1, -1, -1},
                                {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

/* TriP1::interpolateAtPoint TriP1.cpp:96-109 (reference triangle
 * (-1,-1) (1,-1) (-1,1)); TetP1::interpolateAtPoint TetP1.cpp:45-60
 * (v0 -> (0,0,0), v1 -> (0,1,0), v2 -> (1,0,0), v3 -> (0,0,1)). */
static int shape_dim(int shape) { return shape == ORC_QUAD || shape == ORC_TRI ? 2 : 3; }
static int shape_nv(int shape) {
  return shape == ORC_QUAD ? 4 : shape == ORC_HEX ? 8 : shape == ORC_TRI ? 3 : 4;
}
static int is_simplex(int shape) { return shape == ORC_TRI || shape == ORC_TET; }

int orc_p1_interpolate(int shape, const double *ref, double *w) {
  if (shape == ORC_TRI) {
    w[0] = -ref[0] / 2.0 - ref[1] / 2.0;
    w[1] = ref[0] / 2.0 + 1.0 / 2.0;
    w[2] = ref[1] / 2.0 + 1.0 / 2.0;
  } else if (shape == ORC_TET) {
    w[0] = -ref[0] - ref[1] - ref[2] + 1;
    w[1] = ref[1];
    w[2] = ref[0];
    w[3] = ref[2];
  } else if (shape == ORC_QUAD) {
    for (int k = 0; k < 4; ++k)
      w[k] = 0.25 * (1 + QS[k][0] * ref[0]) * (1 + QS[k][1] * ref[1]);
  } else {
    for (int k = 0; k < 8; ++k)
      w[k] = 0.125 * (1 + HS[k][0] * ref[0]) * (1 + HS[k][1] * ref[1]) * (1 + HS[k][2] * ref[2]);
  }
  return 0;
}

static int inv2(const double J[4], double *det, double *inv) {
  double d = J[0] * J[3] - J[1] * J[2];
  *det = d;
  if (inv) {
    inv[0] = J[3] / d; inv[1] = -J[1] / d;
    inv[2] = -J[2] / d; inv[3] = J[0] / d;
  }
  return 0;
}
static int inv3(const double J[9], double *det, double *inv) {
  double c00 = J[4] * J[8] - J[5] * J[7];
  double c01 = J[5] * J[6] - J[3] * J[8];
  double c02 = J[3] * J[7] - J[4] * J[6];
  double d = J[0] * c00 + J[1] * c01 + J[2] * c02;
  *det = d;
  if (inv) {
    double id = 1.0 / d;
    inv[0] = c00 * id;
    inv[1] = (J[2] * J[7] - J[1] * J[8]) * id;
    inv[2] = (J[1] * J[5] - J[2] * J[4]) * id;
    inv[3] = c01 * id;
    inv[4] = (J[0] * J[8] - J[2] * J[6]) * id;
    inv[5] = (J[2] * J[3] - J[0] * J[5]) * id;
    inv[6] = c02 * id;
    inv[7] = (J[1] * J[6] - J[0] * J[7]) * id;
    inv[8] = (J[0] * J[4] - J[1] * J[3]) * id;
  }
  return 0;
}

/* Jacobian J[i][k] = d x_k / d xi_i (rows = reference directions), its
 * determinant and inverse; gradient = invJ * reference gradient.
 * QuadP1::inverseJacobianAtPoint QuadP1.h:79-90; HexP1::inverseJacobianAtPoint
 * HexP1.cpp:189-240. */
int orc_p1_jacobian(int shape, const double *vtx, const double *ref, unsigned flags,
                    double *detJ, double *invJ) {
  if (shape == ORC_TRI) {
    /* TriP1::inverseJacobian TriP1.cpp:56-94: rows d/dr = (v1 - v0)/2,
     * d/ds = (v2 - v0)/2 */
    double J[4] = {(vtx[2] - vtx[0]) / 2, (vtx[3] - vtx[1]) / 2,
                   (vtx[4] - vtx[0]) / 2, (vtx[5] - vtx[1]) / 2};
    return inv2(J, detJ, invJ);
  }
  if (shape == ORC_TET) {
    /* TetP1::inverseJacobian TetP1.cpp:91-150: rows d/dr = v2 - v0,
     * d/ds = v1 - v0, d/dt = v3 - v0 */
    double J[9];
    for (int m = 0; m < 3; ++m) {
      J[0 + m] = vtx[6 + m] - vtx[m];
      J[3 + m] = vtx[3 + m] - vtx[m];
      J[6 + m] = vtx[9 + m] - vtx[m];
    }
    return inv3(J, detJ, invJ);
  }
  if (shape == ORC_QUAD) {
    double J[4] = {0, 0, 0, 0};
    double r = ref[0], s = ref[1];
    for (int k = 0; k < 4; ++k) {
      double dr, ds;
      if (flags & ORC_Q17_QUAD_SWAPPED_JAC) {
        /* QuadP1.h:20-27 evaluate dN/dr at r and dN/ds at s. */
        dr = 0.25 * QS[k][0] * (1 + QS[k][1] * r);
        ds = 0.25 * QS[k][1] * (1 + QS[k][0] * s);
      } else {
        dr = 0.25 * QS[k][0] * (1 + QS[k][1] * s);
        ds = 0.25 * QS[k][1] * (1 + QS[k][0] * r);
      }
      J[0] += dr * vtx[2 * k + 0];
      J[1] += dr * vtx[2 * k + 1];
      J[2] += ds * vtx[2 * k + 0];
      J[3] += ds * vtx[2 * k + 1];
    }
    return inv2(J, detJ, invJ);
  } else {
    double J[9] = {0};
    for (int k = 0; k < 8; ++k) {
      double a = 1 + HS[k][0] * ref[0], b = 1 + HS[k][1] * ref[1], c = 1 + HS[k][2] * ref[2];
      double d0 = 0.125 * HS[k][0] * b * c;
      double d1 = 0.125 * HS[k][1] * a * c;
      double d2 = 0.125 * HS[k][2] * a * b;
      for (int m = 0; m < 3; ++m) {
        J[0 + m] += d0 * vtx[3 * k + m];
        J[3 + m] += d1 * vtx[3 * k + m];
        J[6 + m] += d2 * vtx[3 * k + m];
      }
    }
    return inv3(J, detJ, invJ);
  }
}

static void p1_map(int shape, const double *vtx, const double *ref, double *x) {
  double w[8];
  orc_p1_interpolate(shape, ref, w);
  int nv = shape_nv(shape), d = shape_dim(shape);
  for (int m = 0; m < d; ++m) {
    double s = 0;
    for (int k = 0; k < nv; ++k) s += w[k] * vtx[d * k + m];
    x[m] = s;
  }
}

/* QuadP1::checkHull QuadP1.cpp:8-39; HexP1::checkHull HexP1.cpp:8-84. */
int orc_check_hull(int shape, const double *vtx, const double *x) {
  double det, ref0[3] = {0, 0, 0};
  orc_p1_jacobian(shape, vtx, ref0, 0, &det, NULL);
  if (det <= 0) { set_err("poorly behaved element (detJ <= 0)"); return -1; }
  if (is_simplex(shape)) {
    /* Barycentric test of TriP1::checkHull TriP1.cpp:6-34 /
     * TetP1::checkHull TetP1.cpp:6-43, corrected: the reference's final
     * "fabs(1-(l1+l2+l3)) < 1e-8" rejection is identically true for
     * triangles (l3 = 1-l1-l2) and rejects every point of the face opposite
     * the last vertex for tetrahedra; here all barycentrics >= -1e-12. */
    double ref[3], w[4];
    if (orc_inverse_map(shape, vtx, x, ref)) return -1;
    orc_p1_interpolate(shape, ref, w);
    for (int k = 0; k < shape_nv(shape); ++k)
      if (w[k] < -1e-12) return 0;
    return 1;
  }
  if (shape == ORC_QUAD) {
    int nneg = 0, npos = 0;
    static const int em[5] = {0, 1, 2, 3, 0};
    for (int i = 0; i < 4; ++i) {
      const double *p0 = vtx + 2 * em[i], *p1 = vtx + 2 * em[i + 1];
      double vx = p1[0] - p0[0], vy = p1[1] - p0[1];
      double px = x[0] - p0[0], py = x[1] - p0[1];
      double x0 = vx * py - vy * px;
      if (x0 < 0) nneg++;
      else if (x0 > 0) npos++;
      else { npos++; nneg++; }
    }
    return (nneg == 4 || npos == 4) ? 1 : 0;
  } else {
    static const int sides[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 3, 5, 4},
                                    {2, 1, 7, 6}, {0, 4, 7, 1}, {2, 6, 5, 3}};
    for (int sd = 0; sd < 6; ++sd) {
      const double *a = vtx + 3 * sides[sd][0], *b = vtx + 3 * sides[sd][1],
                   *dd = vtx + 3 * sides[sd][3];
      double l1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
      double l2[3] = {dd[0] - a[0], dd[1] - a[1], dd[2] - a[2]};
      double nrm[3] = {l1[1] * l2[2] - l1[2] * l2[1], l1[2] * l2[0] - l1[0] * l2[2],
                       l1[0] * l2[1] - l1[1] * l2[0]};
      double dot = nrm[0] * (x[0] - a[0]) + nrm[1] * (x[1] - a[1]) + nrm[2] * (x[2] - a[2]);
      if (dot > 0) return 0;
    }
    return 1;
  }
}

/* Newton inverse map, tol 1e-6 on the physical residual, <= 10 iterations:
 * QuadP1::inverseCoordinateTransform QuadP1.cpp:41-92,
 * HexP1::inverseCoordinateTransform HexP1.cpp:135-187. */
int orc_inverse_map(int shape, const double *vtx, const double *x, double *ref) {
  /* affine simplices (TriP1.cpp:36-54, TetP1.cpp:62-89 closed forms) need
   * a single Newton step from the origin */
  const int d = shape_dim(shape);
  double sol[3] = {0, 0, 0};
  for (int it = 0;; ++it) {
    double X[3], det, inv[9];
    p1_map(shape, vtx, sol, X);
    double obj[3] = {x[0] - X[0], x[1] - X[1], d == 3 ? x[2] - X[2] : 0.0};
    int ok = 1;
    for (int m = 0; m < d; ++m)
      if (!(fabs(obj[m]) < 1e-6)) ok = 0;
    if (ok) break;
    /* dx/dxi = J^T, so the Newton step is (J^T)^-1 obj = invJ^T obj. */
    orc_p1_jacobian(shape, vtx, sol, 0, &det, inv);
    for (int a = 0; a < d; ++a) {
      double s = 0;
      for (int b = 0; b < d; ++b) s += inv[b * d + a] * obj[b];
      sol[a] += s;
    }
    if (it > 10) { set_err("inverse map failed to converge after 10 iterations"); return -1; }
  }
  for (int m = 0; m < d; ++m) ref[m] = sol[m];
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Tensor element operators (single element).                                */
typedef struct {
  int shape, dim, n, P, nv;
  double xi[ORC_MAX_N], w[ORC_MAX_N], D[ORC_MAX_N * ORC_MAX_N];
  const stab_t *sx; /* simplex tables (NULL for tensor elements) */
} basis_t;

static int basis_init(basis_t *b, int shape, int order) {
  b->shape = shape;
  b->dim = shape_dim(shape);
  b->nv = shape_nv(shape);
  b->n = order + 1;
  b->sx = NULL;
  if (is_simplex(shape)) {
    /* P3 only (Triangle.cpp:24-39, Tetrahedra.cpp:66-84) */
    if (order != 3) { set_err("simplices are built for order 3 only (got %d)", order); return -1; }
    b->sx = stab_for(shape);
    if (!b->sx) { set_err("simplex tables unavailable"); return -1; }
    b->P = b->sx->P;
    return 0;
  }
  b->P = b->dim == 2 ? b->n * b->n : b->n * b->n * b->n;
  if (b->P > ORC_MAX_P) { set_err("order %d unsupported for this shape", order); return -1; }
  if (orc_gll(order, b->xi, b->w)) return -1;
  return orc_deriv_matrix(order, b->D);
}

static inline void point_ref(const basis_t *b, int p, double *ref) {
  if (b->sx) {
    ref[0] = b->sx->x[p][0]; ref[1] = b->sx->x[p][1]; ref[2] = b->sx->x[p][2];
    return;
  }
  int n = b->n;
  ref[0] = b->xi[p % n];
  ref[1] = b->xi[(p / n) % n];
  ref[2] = b->dim == 3 ? b->xi[p / (n * n)] : 0.0;
}
static inline double point_w(const basis_t *b, int p) {
  if (b->sx) return b->sx->w[p];
  int n = b->n;
  double w = b->w[p % n] * b->w[(p / n) % n];
  if (b->dim == 3) w *= b->w[p / (n * n)];
  return w;
}

/* Reference-direction gradient at every point.  TensorQuad.cpp:198-201,
 * Hexahedra.cpp:611-616. */
static void ref_gradient(const basis_t *b, const double *u, double *gr /* [P][dim] */) {
  const int n = b->n, d = b->dim;
  if (b->sx) {
    /* reference gradient at node q: sum_j dphi_j/dxi_k (x_q) u_j
     * (Triangle::computeGradient Triangle.cpp:365-385; the tetrahedron's
     * mGradientPhi_dx of Tetrahedra.cpp:396-407 folds J^-1 into the same sum) */
    const int P = b->P;
    for (int q = 0; q < P; ++q)
      for (int k = 0; k < d; ++k) {
        double s = 0;
        for (int j = 0; j < P; ++j) s += b->sx->D[k][j * P + q] * u[j];
        gr[q * d + k] = s;
      }
    return;
  }
  for (int p = 0; p < b->P; ++p) {
    int r = p % n, s = (p / n) % n, t = p / (n * n);
    double g0 = 0, g1 = 0, g2 = 0;
    for (int i = 0; i < n; ++i) {
      g0 += b->D[r * n + i] * u[i + s * n + t * n * n];
      g1 += b->D[s * n + i] * u[r + i * n + t * n * n];
      if (d == 3) g2 += b->D[t * n + i] * u[r + s * n + i * n * n];
    }
    gr[p * d + 0] = g0;
    gr[p * d + 1] = g1;
    if (d == 3) gr[p * d + 2] = g2;
  }
}

/* Per-point geometry of one element: detJ[P], invJ[P][d*d]. */
static void element_geometry(const basis_t *b, const double *vtx, unsigned flags,
                             double *detJ, double *invJ) {
  for (int p = 0; p < b->P; ++p) {
    double ref[3];
    point_ref(b, p, ref);
    orc_p1_jacobian(b->shape, vtx, ref, flags, &detJ[p], &invJ[p * b->dim * b->dim]);
  }
}

/* computeGradient: physical gradient = invJ * ref gradient. */
static void grad_from_geom(const basis_t *b, const double *invJ, const double *u, double *g) {
  double gr[ORC_MAX_P * 3];
  const int d = b->dim;
  ref_gradient(b, u, gr);
  for (int p = 0; p < b->P; ++p) {
    const double *iJ = invJ + p * d * d;
    for (int a = 0; a < d; ++a) {
      double s = 0;
      for (int k = 0; k < d; ++k) s += iJ[a * d + k] * gr[p * d + k];
      g[p * d + a] = s;
    }
  }
}

/* Gradient-test integral, per-quadrature-point form (Hexahedra.cpp:689-754;
 * corrected 2-D form).  F = invJ^T f at each point, then D^T sums weighted
 * by w detJ. */
static void grad_test_from_geom(const basis_t *b, const double *detJ, const double *invJ,
                                const double *f, double *out) {
  const int n = b->n, d = b->dim;
  double F[ORC_MAX_P * 3];
  for (int p = 0; p < b->P; ++p) {
    const double *iJ = invJ + p * d * d;
    for (int k = 0; k < d; ++k) {
      double s = 0;
      for (int a = 0; a < d; ++a) s += iJ[a * d + k] * f[p * d + a];
      F[p * d + k] = s * detJ[p];
    }
  }
  if (b->sx) {
    /* out_i = sum_q w_q detJ sum_k dphi_i/dxi_k (x_q) F_k(q)
     * (Tetrahedra::applyGradTestAndIntegrate Tetrahedra.cpp:248-275,
     * Triangle::applyGradTestAndIntegrate Triangle.cpp:323-346) */
    const int P = b->P;
    for (int i = 0; i < P; ++i) {
      double s = 0;
      for (int q = 0; q < P; ++q) {
        double t = 0;
        for (int k = 0; k < d; ++k) t += F[q * d + k] * b->sx->D[k][i * P + q];
        s += b->sx->w[q] * t;
      }
      out[i] = s;
    }
    return;
  }
  for (int p = 0; p < b->P; ++p) {
    int r = p % n, s = (p / n) % n, t = p / (n * n);
    double sr = 0, ss = 0, st = 0;
    for (int i = 0; i < n; ++i) {
      int ri = i + s * n + t * n * n, si = r + i * n + t * n * n, ti = r + s * n + i * n * n;
      sr += F[ri * d + 0] * b->D[i * n + r] * b->w[i];
      ss += F[si * d + 1] * b->D[i * n + s] * b->w[i];
      if (d == 3) st += F[ti * d + 2] * b->D[i * n + t] * b->w[i];
    }
    if (d == 2) {
      out[p] = sr * b->w[s] + ss * b->w[r];
    } else {
      out[p] = sr * b->w[s] * b->w[t] + ss * b->w[r] * b->w[t] + st * b->w[r] * b->w[s];
    }
  }
}

/* 2-D reference-literal gradient-test (TensorQuad.cpp:351-397): sums use
 * detJ at the quadrature points, J^-1 is applied at the output point. */
static void grad_test_quad_literal(const basis_t *b, const double *vtx, unsigned flags,
                                   const double *detJ, const double *f, double *out) {
  const int n = b->n;
  for (int p = 0; p < b->P; ++p) {
    int r = p % n, s = p / n;
    double dfx0 = 0, dfx1 = 0, dfy0 = 0, dfy1 = 0;
    for (int i = 0; i < n; ++i) {
      int ri = i + s * n, si = r + i * n;
      dfx0 += detJ[ri] * f[ri * 2 + 0] * b->D[i * n + r] * b->w[i];
      dfx1 += detJ[si] * f[si * 2 + 0] * b->D[i * n + s] * b->w[i];
      dfy0 += detJ[ri] * f[ri * 2 + 1] * b->D[i * n + r] * b->w[i];
      dfy1 += detJ[si] * f[si * 2 + 1] * b->D[i * n + s] * b->w[i];
    }
    dfx0 *= b->w[s]; dfx1 *= b->w[r]; dfy0 *= b->w[s]; dfy1 *= b->w[r];
    double ref[3], dj, iJ[4];
    point_ref(b, p, ref);
    orc_p1_jacobian(b->shape, vtx, ref, flags, &dj, iJ);
    out[p] = iJ[0] * dfx0 + iJ[1] * dfx1 + iJ[2] * dfy0 + iJ[3] * dfy1;
  }
}

int orc_element_gradient(int shape, int order, const double *vtx, unsigned flags,
                         const double *u, double *grad) {
  basis_t b;
  if (basis_init(&b, shape, order)) return -1;
  double detJ[ORC_MAX_P], invJ[ORC_MAX_P * 9];
  element_geometry(&b, vtx, flags, detJ, invJ);
  grad_from_geom(&b, invJ, u, grad);
  return 0;
}

int orc_element_grad_test(int shape, int order, const double *vtx, unsigned flags,
                          const double *f, double *out) {
  basis_t b;
  if (basis_init(&b, shape, order)) return -1;
  double detJ[ORC_MAX_P], invJ[ORC_MAX_P * 9];
  element_geometry(&b, vtx, flags, detJ, invJ);
  if (shape == ORC_QUAD && (flags & ORC_Q3_QUAD_INVJ_AT_OUTPUT))
    grad_test_quad_literal(&b, vtx, flags, detJ, f, out);
  else
    grad_test_from_geom(&b, detJ, invJ, f, out);
  return 0;
}

/* applyTestAndIntegrate TensorQuad.cpp:326-348, Hexahedra.cpp:659-686. */
int orc_element_test(int shape, int order, const double *vtx, unsigned flags,
                     const double *f, double *out) {
  basis_t b;
  if (basis_init(&b, shape, order)) return -1;
  for (int p = 0; p < b.P; ++p) {
    double ref[3], dj;
    point_ref(&b, p, ref);
    orc_p1_jacobian(shape, vtx, ref, flags, &dj, NULL);
    out[p] = f[p] * dj * point_w(&b, p);
  }
  return 0;
}

static void tensor_lagrange(const basis_t *b, const double *ref, double *l, double *dl /* [P][d] or NULL */) {
  if (b->sx) {
    orc_simplex_basis(b->shape, ref, l, dl);
    return;
  }
  double lr[ORC_MAX_N], ls[ORC_MAX_N], lt[ORC_MAX_N], dr[ORC_MAX_N], ds[ORC_MAX_N], dt[ORC_MAX_N];
  const int n = b->n;
  orc_lagrange(n - 1, ref[0], lr, dr);
  orc_lagrange(n - 1, ref[1], ls, ds);
  if (b->dim == 3) orc_lagrange(n - 1, ref[2], lt, dt);
  for (int p = 0; p < b->P; ++p) {
    int r = p % n, s = (p / n) % n, t = p / (n * n);
    if (b->dim == 2) {
      l[p] = lr[r] * ls[s];
      if (dl) { dl[p * 2 + 0] = dr[r] * ls[s]; dl[p * 2 + 1] = lr[r] * ds[s]; }
    } else {
      l[p] = lr[r] * ls[s] * lt[t];
      if (dl) {
        dl[p * 3 + 0] = dr[r] * ls[s] * lt[t];
        dl[p * 3 + 1] = lr[r] * ds[s] * lt[t];
        dl[p * 3 + 2] = lr[r] * ls[s] * dt[t];
      }
    }
  }
}

/* getDeltaFunctionCoefficients TensorQuad.cpp:287-306, Hexahedra.cpp:467-490. */
int orc_element_delta(int shape, int order, const double *vtx, unsigned flags,
                      const double *ref, double *out) {
  basis_t b;
  if (basis_init(&b, shape, order)) return -1;
  tensor_lagrange(&b, ref, out, NULL);
  for (int p = 0; p < b.P; ++p) {
    double pr[3], dj;
    point_ref(&b, p, pr);
    orc_p1_jacobian(shape, vtx, pr, flags, &dj, NULL);
    out[p] /= (point_w(&b, p) * dj);
  }
  return 0;
}

/* ParAtIntPts TensorQuad.cpp:309-323, Hexahedra.cpp:635-656. */
int orc_element_par(int shape, int order, const double *par_vtx, double *out) {
  basis_t b;
  if (basis_init(&b, shape, order)) return -1;
  for (int p = 0; p < b.P; ++p) {
    double ref[3], w[8];
    point_ref(&b, p, ref);
    orc_p1_interpolate(shape, ref, w);
    double s = 0;
    for (int k = 0; k < b.nv; ++k) s += w[k] * par_vtx[k];
    out[p] = s;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Problem.                                                                  */
typedef struct {
  int64_t elem;
  double ref[3];
  double f0, t0, amp;
  double *wts; /* [P][c] nodal weights multiplied by the source time function */
} src_t;

typedef struct {
  int64_t elem;
  double *l; /* [P] Lagrange weights */
} rec_t;

/* One edge point of a fluid-solid coupling surface integral. kind 0: fluid
 * element point, a_u += cx vx + cy vy; kind 1: solid element point,
 * a_ux += cx v, a_uy += cy v (v: the fluid velocity field). */
typedef struct {
  int64_t e;
  int q, kind;
  double cx, cy;
} cpl_t;

struct orc_problem {
  orc_desc d;
  basis_t b;
  int c, npar;
  int64_t E, G;
  double *vtx;     /* [E][nv][dim] */
  double *par;     /* [npar][E][nv] */
  int64_t *conn;   /* [E][P] */
  double *xyz;     /* [G][dim] */
  /* cached per-point data (not used in faithful mode) */
  double *detJ, *invJ, *mat; /* mat: acoustic vp^2 [E][P]; elastic 9 c_ij [E][9][P] */
  double *mi;      /* [G][c] inverse diagonal mass per component (0: none) */
  double *Ke;      /* triangles: dense element stiffness [E][P][P] */
  char *dirichlet; /* [G] node flags (NULL: none) */
  char *fluid;     /* coupled meshes: [E] 1 for fluid elements */
  cpl_t *cpl;      /* coupled meshes: edge-point coupling terms, element order */
  int64_t ncpl;
  double *u, *v, *a, *a_; /* [G][c] */
  int64_t step;
  /* colouring for threaded assembly */
  int ncolours;
  int64_t *col_off, *col_elems;
  src_t *src; int nsrc;
  rec_t *rec; int nrec;
};

static void *xcalloc(size_t n, size_t s) {
  void *p = calloc(n ? n : 1, s);
  if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
  return p;
}

/* -- coordinate-keyed node numbering (independent of the product's
 *    topological numbering; semantics of Mesh::setupGlobalDof Mesh.cpp:361-452) */
typedef struct { int64_t k[3]; int64_t id; } hent_t;

static uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

static int number_nodes(orc_problem *p) {
  const basis_t *b = &p->b;
  const int d = b->dim;
  /* tolerance: 1e-7 of the smallest element-vertex spacing */
  double hmin = INFINITY;
  for (int64_t e = 0; e < p->E; ++e) {
    const double *v = p->vtx + e * b->nv * d;
    for (int k = 1; k < b->nv; ++k) {
      double s = 0;
      for (int m = 0; m < d; ++m) s += (v[k * d + m] - v[m]) * (v[k * d + m] - v[m]);
      if (s > 0 && sqrt(s) < hmin) hmin = sqrt(s);
    }
  }
  const double tol = 1e-7 * hmin;
  size_t cap = 1024;
  while (cap < (size_t)(p->E * b->P)) cap <<= 1;
  hent_t *tab = (hent_t *)malloc(cap * sizeof(hent_t));
  if (!tab) { set_err("oom"); return -1; }
  for (size_t i = 0; i < cap; ++i) tab[i].id = -1;
  p->conn = (int64_t *)xcalloc((size_t)(p->E * b->P), sizeof(int64_t));
  double *xyz = (double *)xcalloc((size_t)(p->E * b->P) * d, sizeof(double));
  int64_t G = 0;
  for (int64_t e = 0; e < p->E; ++e) {
    const double *v = p->vtx + e * b->nv * d;
    for (int q = 0; q < b->P; ++q) {
      double ref[3], x[3] = {0, 0, 0};
      point_ref(b, q, ref);
      p1_map(b->shape, v, ref, x);
      int64_t key[3];
      for (int m = 0; m < 3; ++m) key[m] = (m < d) ? (int64_t)llround(x[m] / tol) : 0;
      uint64_t h = mix64((uint64_t)key[0] ^ mix64((uint64_t)key[1] ^ mix64((uint64_t)key[2])));
      size_t i = h & (cap - 1);
      for (;;) {
        if (tab[i].id < 0) {
          tab[i].k[0] = key[0]; tab[i].k[1] = key[1]; tab[i].k[2] = key[2];
          tab[i].id = G;
          for (int m = 0; m < d; ++m) xyz[G * d + m] = x[m];
          p->conn[e * b->P + q] = G++;
          break;
        }
        if (tab[i].k[0] == key[0] && tab[i].k[1] == key[1] && tab[i].k[2] == key[2]) {
          p->conn[e * b->P + q] = tab[i].id;
          break;
        }
        i = (i + 1) & (cap - 1);
      }
    }
  }
  free(tab);
  p->G = G;
  p->xyz = (double *)realloc(xyz, (size_t)G * d * sizeof(double));
  return 0;
}

static void colour_elements(orc_problem *p) {
  const int P = p->b.P;
  uint64_t *mask = (uint64_t *)xcalloc((size_t)p->G, sizeof(uint64_t));
  int *col = (int *)xcalloc((size_t)p->E, sizeof(int));
  int nc = 0;
  for (int64_t e = 0; e < p->E; ++e) {
    uint64_t used = 0;
    for (int q = 0; q < P; ++q) used |= mask[p->conn[e * P + q]];
    int c = 0;
    while (c < 64 && (used >> c) & 1) ++c;
    if (c >= 64) { fprintf(stderr, "oracle: colouring overflow\n"); abort(); }
    col[e] = c;
    if (c + 1 > nc) nc = c + 1;
    for (int q = 0; q < P; ++q) mask[p->conn[e * P + q]] |= (1ull << c);
  }
  p->ncolours = nc;
  p->col_off = (int64_t *)xcalloc((size_t)nc + 1, sizeof(int64_t));
  p->col_elems = (int64_t *)xcalloc((size_t)p->E, sizeof(int64_t));
  for (int64_t e = 0; e < p->E; ++e) p->col_off[col[e] + 1]++;
  for (int c = 0; c < nc; ++c) p->col_off[c + 1] += p->col_off[c];
  int64_t *fill = (int64_t *)xcalloc((size_t)nc, sizeof(int64_t));
  for (int64_t e = 0; e < p->E; ++e) p->col_elems[p->col_off[col[e]] + fill[col[e]]++] = e;
  free(fill); free(col); free(mask);
}

/* Material words per GLL point: acoustic vp^2; elastic 3-D 9 c_ij;
 * elastic 2-D c11 c13 c33 c55. */
static int mat_words(int physics) {
  return physics == ORC_ACOUSTIC ? 1 : (physics == ORC_ELASTIC3D ? 9 : 4);
}

/* Physics of element e: coupled meshes hold fluid (Scalar) and solid
 * (Elastic2D) elements, chosen per element by the model's fluid flag
 * (ExodusModel::getElementType ExodusModel.cpp:473-520). */
static int elem_physics(const orc_problem *p, int64_t e) {
  if (p->d.physics != ORC_COUPLED2D) return p->d.physics;
  return p->fluid[e] ? ORC_ACOUSTIC : ORC_ELASTIC2D;
}

/* Material at GLL points of element e: acoustic vp^2 (Scalar.cpp:45);
 * elastic c_ij (Elastic3D.cpp:42-53, c11 c12 c13 c22 c23 c33 c44 c55 c66);
 * elastic 2-D C11 C13 C33 C55 (Elastic2D.cpp:57-60; its c13 / c23 slots stay
 * zero, Elastic2D.cpp:16-21,55-56). */
static void element_material(const orc_problem *p, int64_t e, double *m, double *rho) {
  const basis_t *b = &p->b;
  const int P = b->P, nv = b->nv;
  double tmp[8][ORC_MAX_P];
  for (int k = 0; k < p->npar; ++k)
    orc_element_par(b->shape, b->n - 1, p->par + ((size_t)k * p->E + e) * nv, tmp[k]);
  if (p->d.physics == ORC_COUPLED2D) {
    /* FLUID VP RHO C11 C13 C33 C55 */
    for (int q = 0; q < P; ++q) {
      if (p->fluid[e]) {
        m[q] = pow(tmp[1][q], 2);
        for (int k = 1; k < 4; ++k) m[k * P + q] = 0.0;
        if (rho) rho[q] = 1.0;
      } else {
        for (int k = 0; k < 4; ++k) m[k * P + q] = tmp[k + 3][q];
        if (rho) rho[q] = tmp[2][q];
      }
    }
  } else if (p->d.physics == ORC_ACOUSTIC) {
    for (int q = 0; q < P; ++q) m[q] = pow(tmp[0][q], 2);
    if (rho) for (int q = 0; q < P; ++q) rho[q] = 1.0;
  } else if (p->d.physics == ORC_ELASTIC2D) {
    for (int q = 0; q < P; ++q) {
      for (int k = 0; k < 4; ++k) m[k * P + q] = tmp[k + 1][q];
      if (rho) rho[q] = tmp[0][q];
    }
  } else {
    for (int q = 0; q < P; ++q) {
      double r = tmp[0][q], vpv = tmp[1][q], vph = tmp[2][q], vsv = tmp[3][q], vsh = tmp[4][q],
             eta = tmp[5][q];
      double c11 = r * pow(vph, 2), c22 = r * pow(vph, 2), c33 = r * pow(vpv, 2);
      double c44 = r * pow(vsv, 2), c55 = r * pow(vsv, 2), c66 = r * pow(vsh, 2);
      double c12 = c11 - 2 * c66, c13 = eta * (c11 - 2 * c44), c23 = eta * (c11 - 2 * c44);
      m[0 * P + q] = c11; m[1 * P + q] = c12; m[2 * P + q] = c13;
      m[3 * P + q] = c22; m[4 * P + q] = c23; m[5 * P + q] = c33;
      m[6 * P + q] = c44; m[7 * P + q] = c55; m[8 * P + q] = c66;
      if (rho) rho[q] = r;
    }
  }
}

/* Element stiffness K_e u_e, [P][c] in and out.
 * Scalar::computeStiffnessTerm Scalar.cpp:58-71 / computeStress :42-55;
 * Elastic3D::computeStiffnessTerm Elastic3D.cpp:70-103 / computeStress :106-118. */
static void element_stiffness_phys(const orc_problem *p, int64_t e, int phys, const double *ue,
                                   double *ke) {
  const basis_t *b = &p->b;
  const int P = b->P, d = b->dim;
  const unsigned fl = p->d.flags;
  const double *vtx = p->vtx + e * b->nv * d;
  double detJ_l[ORC_MAX_P], invJ_l[ORC_MAX_P * 9], mat_l[9 * ORC_MAX_P];
  const double *detJ, *invJ, *mat;
  const int faithful = (fl & ORC_FAITHFUL_RECOMPUTE) != 0;
  if (faithful) {
    element_geometry(b, vtx, fl, detJ_l, invJ_l);
    detJ = detJ_l; invJ = invJ_l;
    if (p->d.physics != ORC_ELASTIC3D) {
      /* Scalar::computeStress / Elastic2D::computeStress re-interpolate the
       * material every call (Scalar.cpp:45, Elastic2D.cpp:57-60) */
      element_material(p, e, mat_l, NULL);
      mat = mat_l;
    } else {
      /* Elastic3D caches c_ij per element at attach time (Elastic3D.cpp:33-54) */
      mat = p->mat + e * P * 9;
    }
  } else {
    detJ = p->detJ + e * P;
    invJ = p->invJ + e * P * d * d;
    mat = p->mat + e * P * mat_words(p->d.physics);
  }
  if (b->shape == ORC_TRI) {
    /* ScalarTri::computeStiffnessTerm ScalarTri.cpp:12-17: K_e u_e */
    const double *K = p->Ke + e * P * P;
    for (int i = 0; i < P; ++i) {
      double s = 0;
      for (int j = 0; j < P; ++j) s += K[i * P + j] * ue[j];
      ke[i] = s;
    }
    return;
  }
  if (phys == ORC_ACOUSTIC) {
    double g[ORC_MAX_P * 3];
    grad_from_geom(b, invJ, ue, g);
    for (int q = 0; q < P; ++q)
      for (int a = 0; a < d; ++a) g[q * d + a] *= mat[q];
    if (b->shape == ORC_QUAD && (fl & ORC_Q3_QUAD_INVJ_AT_OUTPUT)) {
      grad_test_quad_literal(b, vtx, fl, detJ, g, ke);
    } else {
      if (faithful) element_geometry(b, vtx, fl, detJ_l, invJ_l); /* Hexahedra.cpp:702 */
      grad_test_from_geom(b, detJ, invJ, g, ke);
    }
    return;
  }
  if (phys == ORC_ELASTIC2D) {
    /* Elastic2D::computeStiffnessTerm Elastic2D.cpp:84-107: strain
     * (ux_x, ux_y, uy_x, uy_y), stress Elastic2D.cpp:62-78 */
    double ux[ORC_MAX_P] = {0}, uy[ORC_MAX_P] = {0}, gx[ORC_MAX_P * 2], gy[ORC_MAX_P * 2];
    for (int q = 0; q < P; ++q) { ux[q] = ue[q * 2]; uy[q] = ue[q * 2 + 1]; }
    grad_from_geom(b, invJ, ux, gx);
    if (faithful) element_geometry(b, vtx, fl, detJ_l, invJ_l);
    grad_from_geom(b, invJ, uy, gy);
    double fx[ORC_MAX_P * 2], fy[ORC_MAX_P * 2];
    for (int q = 0; q < P; ++q) {
      const double exx = gx[q * 2 + 0], eyy = gy[q * 2 + 1];
      const double exy = gx[q * 2 + 1] + gy[q * 2 + 0];
      const double c11 = mat[0 * P + q], c13 = mat[1 * P + q], c33 = mat[2 * P + q],
                   c55 = mat[3 * P + q];
      const double sxx = c11 * exx + c13 * eyy, syy = c13 * exx + c33 * eyy, sxy = c55 * exy;
      fx[q * 2 + 0] = sxx; fx[q * 2 + 1] = sxy;
      fy[q * 2 + 0] = sxy; fy[q * 2 + 1] = syy;
    }
    double kx[ORC_MAX_P], ky[ORC_MAX_P];
    if (fl & ORC_Q3_QUAD_INVJ_AT_OUTPUT) {
      grad_test_quad_literal(b, vtx, fl, detJ, fx, kx);
      grad_test_quad_literal(b, vtx, fl, detJ, fy, ky);
    } else {
      if (faithful) element_geometry(b, vtx, fl, detJ_l, invJ_l);
      grad_test_from_geom(b, detJ, invJ, fx, kx);
      if (faithful) element_geometry(b, vtx, fl, detJ_l, invJ_l);
      grad_test_from_geom(b, detJ, invJ, fy, ky);
    }
    for (int q = 0; q < P; ++q) { ke[q * 2] = kx[q]; ke[q * 2 + 1] = ky[q]; }
    return;
  }
  /* elastic 3-D */
  double ux[ORC_MAX_P] = {0}, uy[ORC_MAX_P] = {0}, uz[ORC_MAX_P] = {0};
  for (int q = 0; q < P; ++q) { ux[q] = ue[q * 3]; uy[q] = ue[q * 3 + 1]; uz[q] = ue[q * 3 + 2]; }
  double gx[ORC_MAX_P * 3], gy[ORC_MAX_P * 3], gz[ORC_MAX_P * 3];
  grad_from_geom(b, invJ, ux, gx);
  if (faithful) element_geometry(b, vtx, fl, detJ_l, invJ_l);
  grad_from_geom(b, invJ, uy, gy);
  if (faithful) element_geometry(b, vtx, fl, detJ_l, invJ_l);
  grad_from_geom(b, invJ, uz, gz);
  double sx[ORC_MAX_P * 3], sy[ORC_MAX_P * 3], sz[ORC_MAX_P * 3];
  for (int q = 0; q < P; ++q) {
    double e0 = gx[q * 3 + 0], e1 = gy[q * 3 + 1], e2 = gz[q * 3 + 2];
    double e3 = gy[q * 3 + 2] + gz[q * 3 + 1];
    double e4 = gx[q * 3 + 2] + gz[q * 3 + 0];
    double e5 = gx[q * 3 + 1] + gy[q * 3 + 0];
    double c11 = mat[0 * P + q], c12 = mat[1 * P + q], c13 = mat[2 * P + q];
    double c22 = mat[3 * P + q], c23 = mat[4 * P + q], c33 = mat[5 * P + q];
    double c44 = mat[6 * P + q], c55 = mat[7 * P + q], c66 = mat[8 * P + q];
    double s0 = c11 * e0 + c12 * e1 + c13 * e2;
    double s1 = c12 * e0 + c22 * e1 + c23 * e2;
    double s2 = c13 * e0 + c23 * e1 + c33 * e2;
    double s3 = c44 * e3, s4 = c55 * e4, s5 = c66 * e5;
    sx[q * 3 + 0] = s0; sx[q * 3 + 1] = s5; sx[q * 3 + 2] = s4;
    sy[q * 3 + 0] = s5; sy[q * 3 + 1] = s1; sy[q * 3 + 2] = s3;
    sz[q * 3 + 0] = s4; sz[q * 3 + 1] = s3; sz[q * 3 + 2] = s2;
  }
  double kx[ORC_MAX_P], ky[ORC_MAX_P], kz[ORC_MAX_P];
  if (faithful) element_geometry(b, vtx, fl, detJ_l, invJ_l);
  grad_test_from_geom(b, detJ, invJ, sx, kx);
  if (faithful) element_geometry(b, vtx, fl, detJ_l, invJ_l);
  grad_test_from_geom(b, detJ, invJ, sy, ky);
  if (faithful) element_geometry(b, vtx, fl, detJ_l, invJ_l);
  grad_test_from_geom(b, detJ, invJ, sz, kz);
  for (int q = 0; q < P; ++q) { ke[q * 3] = kx[q]; ke[q * 3 + 1] = ky[q]; ke[q * 3 + 2] = kz[q]; }
}

/* Coupled meshes: the element's own physics on its components of [u, ux, uy]
 * (fluid: u; solid: ux, uy); the others stay zero. */
static void element_stiffness(const orc_problem *p, int64_t e, const double *ue, double *ke) {
  if (p->d.physics != ORC_COUPLED2D) {
    element_stiffness_phys(p, e, p->d.physics, ue, ke);
    return;
  }
  const int P = p->b.P;
  double us[ORC_MAX_P * 2] = {0}, ks[ORC_MAX_P * 2];
  for (int i = 0; i < P * 3; ++i) ke[i] = 0.0;
  if (p->fluid[e]) {
    for (int q = 0; q < P; ++q) us[q] = ue[q * 3];
    element_stiffness_phys(p, e, ORC_ACOUSTIC, us, ks);
    for (int q = 0; q < P; ++q) ke[q * 3] = ks[q];
  } else {
    for (int q = 0; q < P; ++q) { us[q * 2] = ue[q * 3 + 1]; us[q * 2 + 1] = ue[q * 3 + 2]; }
    element_stiffness_phys(p, e, ORC_ELASTIC2D, us, ks);
    for (int q = 0; q < P; ++q) { ke[q * 3 + 1] = ks[q * 2]; ke[q * 3 + 2] = ks[q * 2 + 1]; }
  }
}

typedef struct { int64_t a, b, e; int i; } edge_t;
static int edge_cmp(const void *x, const void *y) {
  const edge_t *p = (const edge_t *)x, *q = (const edge_t *)y;
  if (p->a != q->a) return p->a < q->a ? -1 : 1;
  if (p->b != q->b) return p->b < q->b ? -1 : 1;
  return p->e < q->e ? -1 : (p->e > q->e);
}

/* Coupling surface integrals of the fluid-solid interface, per element in
 * element order, per local edge i (vertex i -> i+1, TensorQuad.cpp:476-516:
 * edge "Jacobian" |v_{i+1} - v_i| / 2, GLL weights along the edge, outward
 * normal (dy, -dx) / |.| of TensorQuad::getEdgeNormal TensorQuad.cpp:400-418).
 * Elements couple when an edge neighbour has the other physics
 * (Mesh::CouplingFields Mesh.cpp:480-503 via TotalCouplingFields).
 *   fluid element (ElasticToAcoustic.cpp:17-41): a_u += int phi (v_s . n_f)
 *     on every edge with a neighbour (K3: solid neighbours only; K4: times
 *     vp^2 at the point, the natural boundary term of int vp^2 grad . grad);
 *   solid element (AcousticToElastic2D.cpp:18-60): a_ux, a_uy -= rho0 int
 *     phi v on edges with a fluid neighbour, rho0 = mean vertex RHO of that
 *     neighbour (AcousticToElastic2D.cpp:33-46); K2: -rho0 int phi v n_f,a
 *     = rho0 int phi v n_s,a. */
static void build_coupling(orc_problem *p) {
  const int n = p->b.n, E4 = (int)(p->E * 4);
  edge_t *ed = (edge_t *)xcalloc((size_t)E4, sizeof(edge_t));
  for (int64_t e = 0; e < p->E; ++e)
    for (int i = 0; i < 4; ++i) {
      int64_t va = p->d.cells[e * 4 + i], vb = p->d.cells[e * 4 + (i + 1) % 4];
      edge_t *x = &ed[e * 4 + i];
      x->a = va < vb ? va : vb; x->b = va < vb ? vb : va; x->e = e; x->i = i;
    }
  qsort(ed, (size_t)E4, sizeof(edge_t), edge_cmp);
  int64_t *nbr = (int64_t *)xcalloc((size_t)E4, sizeof(int64_t));
  for (int k = 0; k < E4; ++k) nbr[ed[k].e * 4 + ed[k].i] = -1;
  for (int k = 0; k + 1 < E4; ++k)
    if (ed[k].a == ed[k + 1].a && ed[k].b == ed[k + 1].b) {
      nbr[ed[k].e * 4 + ed[k].i] = ed[k + 1].e;
      nbr[ed[k + 1].e * 4 + ed[k + 1].i] = ed[k].e;
    }
  free(ed);
  const unsigned fl = p->d.flags;
  p->cpl = (cpl_t *)xcalloc((size_t)E4 * n, sizeof(cpl_t));
  p->ncpl = 0;
  for (int64_t e = 0; e < p->E; ++e) {
    const int fe = p->fluid[e];
    int has_other = 0;
    for (int i = 0; i < 4; ++i) {
      int64_t f = nbr[e * 4 + i];
      if (f >= 0 && p->fluid[f] != fe) has_other = 1;
    }
    if (!has_other) continue;
    for (int i = 0; i < 4; ++i) {
      const int64_t f = nbr[e * 4 + i];
      if (f < 0) continue;
      if (p->fluid[f] == fe && !(fe && !(fl & ORC_K3_INTERFACE_EDGES))) continue;
      const double *v0 = p->vtx + (e * 4 + i) * 2, *v1 = p->vtx + (e * 4 + (i + 1) % 4) * 2;
      const double dx = v1[0] - v0[0], dy = v1[1] - v0[1];
      const double len = sqrt(dx * dx + dy * dy);
      const double d = len / 2.0, nx = dy / len, ny = -dx / len;
      double rho0 = 0.0, vp[ORC_MAX_P];
      if (fe) orc_element_par(ORC_QUAD, n - 1, p->par + ((size_t)1 * p->E + e) * 4, vp);
      if (!fe) {
        for (int a = 0; a < 4; ++a) rho0 += p->par[((size_t)2 * p->E + f) * 4 + a];
        rho0 /= 4;
      }
      for (int j = 0; j < n; ++j) {
        int q;
        switch (i) {
          case 0: q = j; break;
          case 1: q = (n - 1) + n * j; break;
          case 2: q = n * n - 1 - j; break;
          default: q = n * (n - 1) - n * j; break;
        }
        cpl_t *c = &p->cpl[p->ncpl++];
        c->e = e; c->q = q; c->kind = fe ? 0 : 1;
        const double wd = p->b.w[j] * d;
        if (fe) {
          const double s2 = (fl & ORC_K4_FLUID_VP2) ? vp[q] * vp[q] : 1.0;
          c->cx = s2 * wd * nx; c->cy = s2 * wd * ny;
        } else if (fl & ORC_K2_SOLID_NORMAL) {
          c->cx = rho0 * wd * nx; c->cy = rho0 * wd * ny;
        } else {
          c->cx = -rho0 * wd; c->cy = -rho0 * wd;
        }
      }
    }
  }
  free(nbr);
}

orc_problem *orc_create(const orc_desc *d) {
  if (!d || d->shape < ORC_QUAD || d->shape > ORC_TET) { set_err("bad shape"); return NULL; }
  if (d->physics == ORC_ELASTIC3D && d->shape != ORC_HEX && d->shape != ORC_TET) {
    set_err("elastic 3-D physics needs hexahedra or tetrahedra");
    return NULL;
  }
  if ((d->physics == ORC_ELASTIC2D || d->physics == ORC_COUPLED2D) && d->shape != ORC_QUAD) {
    set_err("2-D elastic and coupled physics need quadrilaterals");
    return NULL;
  }
  if (d->physics < ORC_ACOUSTIC || d->physics > ORC_COUPLED2D) { set_err("bad physics"); return NULL; }
  orc_problem *p = (orc_problem *)xcalloc(1, sizeof(orc_problem));
  p->d = *d;
  if (p->d.threads < 1) p->d.threads = 1;
  if (basis_init(&p->b, d->shape, d->order)) { free(p); return NULL; }
  const basis_t *b = &p->b;
  const int dim = b->dim, nv = b->nv, P = b->P;
  p->c = d->physics == ORC_ACOUSTIC ? 1 : (d->physics == ORC_ELASTIC2D ? 2 : 3);
  p->npar = d->physics == ORC_ACOUSTIC ? 1 : (d->physics == ORC_ELASTIC2D ? 5 :
            (d->physics == ORC_COUPLED2D ? 7 : 6));
  p->E = d->n_elements;
  p->vtx = (double *)xcalloc((size_t)(p->E * nv * dim), sizeof(double));
  for (int64_t e = 0; e < p->E; ++e)
    for (int k = 0; k < nv; ++k) {
      int64_t vi = d->cells[e * nv + k];
      if (vi < 0 || vi >= d->n_vertices) { set_err("cell vertex out of range"); orc_destroy(p); return NULL; }
      for (int m = 0; m < dim; ++m) p->vtx[(e * nv + k) * dim + m] = d->vertices[vi * dim + m];
    }
  p->par = (double *)xcalloc((size_t)(p->npar * p->E * nv), sizeof(double));
  memcpy(p->par, d->params, sizeof(double) * (size_t)(p->npar * p->E * nv));
  if (d->physics == ORC_COUPLED2D) {
    p->fluid = (char *)xcalloc((size_t)p->E, 1);
    for (int64_t e = 0; e < p->E; ++e) {
      const double f0 = p->par[e * nv];
      for (int a = 0; a < nv; ++a)
        if (p->par[e * nv + a] != f0 || (f0 != 0.0 && f0 != 1.0)) {
          set_err("element %lld: fluid flag must be 0 or 1 at every vertex", (long long)e);
          orc_destroy(p);
          return NULL;
        }
      p->fluid[e] = f0 == 1.0;
    }
  }
  /* element sanity (checkHull's right-hand-rule check) */
  for (int64_t e = 0; e < p->E; ++e) {
    double det, ref0[3] = {0, 0, 0};
    orc_p1_jacobian(b->shape, p->vtx + e * nv * dim, ref0, 0, &det, NULL);
    if (!(det > 0)) { set_err("element %lld has detJ <= 0", (long long)e); orc_destroy(p); return NULL; }
  }
  if (number_nodes(p)) { orc_destroy(p); return NULL; }
  /* simplices: vertex valences exceed the 64-colour mask; their threaded
   * assembly buffers element results and scatters them in element order */
  if (!is_simplex(d->shape)) colour_elements(p);
  const int nm = mat_words(d->physics);
  const int faithful = (d->flags & ORC_FAITHFUL_RECOMPUTE) != 0;
  if (!faithful) {
    p->detJ = (double *)xcalloc((size_t)(p->E * P), sizeof(double));
    p->invJ = (double *)xcalloc((size_t)(p->E * P * dim * dim), sizeof(double));
    for (int64_t e = 0; e < p->E; ++e)
      element_geometry(b, p->vtx + e * nv * dim, d->flags, p->detJ + e * P, p->invJ + e * P * dim * dim);
  }
  if (!faithful || d->physics == ORC_ELASTIC3D) {
    /* (coupled meshes keep 4 words for fluid and solid elements alike) */
    p->mat = (double *)xcalloc((size_t)(p->E * P * nm), sizeof(double));
    for (int64_t e = 0; e < p->E; ++e) element_material(p, e, p->mat + e * P * nm, NULL);
  }
  if (d->shape == ORC_TRI) {
    /* Triangle::buildStiffnessMatrix Triangle.cpp:194-241:
     * K_ij = detJ sum_q w_q vp_q^2 (dphi_i/dx dphi_j/dx + dphi_i/dz dphi_j/dz) */
    p->Ke = (double *)xcalloc((size_t)(p->E * P * P), sizeof(double));
    double dx[12 * 12], dz[12 * 12];
    for (int64_t e = 0; e < p->E; ++e) {
      double det, iJ[4], ref0[3] = {0, 0, 0}, vp2[12];
      orc_p1_jacobian(ORC_TRI, p->vtx + e * nv * dim, ref0, 0, &det, iJ);
      element_material(p, e, vp2, NULL);
      for (int i = 0; i < P; ++i)
        for (int q = 0; q < P; ++q) {
          const double dr = b->sx->D[0][i * P + q], ds = b->sx->D[1][i * P + q];
          dx[i * P + q] = dr * iJ[0] + ds * iJ[1];
          dz[i * P + q] = dr * iJ[2] + ds * iJ[3];
        }
      double *K = p->Ke + e * P * P;
      for (int i = 0; i < P; ++i)
        for (int j = 0; j < P; ++j) {
          double sx = 0, sz = 0;
          for (int q = 0; q < P; ++q) {
            sx += b->sx->w[q] * (vp2[q] * dx[i * P + q] * dx[j * P + q]);
            sz += b->sx->w[q] * (vp2[q] * dz[i * P + q] * dz[j * P + q]);
          }
          K[i * P + j] = det * sx + det * sz;
        }
    }
  }
  /* Diagonal mass: Scalar.cpp:34-39 (no rho), Elastic3D.cpp:63-67 (rho);
   * summed in element order then reciprocal (Order2Newmark.cpp:32-66). */
  /* One mass summed over every element, shared by all components
   * (Order2Newmark.cpp:38-52); K1 on coupled meshes: fluid elements add to
   * u's mass only, solid elements to ux's and uy's. */
  const int cc = p->c;
  p->mi = (double *)xcalloc((size_t)(p->G * cc), sizeof(double));
  for (int64_t e = 0; e < p->E; ++e) {
    double m[9 * ORC_MAX_P], rho[ORC_MAX_P], me[ORC_MAX_P];
    element_material(p, e, m, rho);
    orc_element_test(b->shape, b->n - 1, p->vtx + e * nv * dim, d->flags, rho, me);
    int k0 = 0, k1 = cc;
    if (d->physics == ORC_COUPLED2D && (d->flags & ORC_K1_SPLIT_MASS)) {
      k0 = p->fluid[e] ? 0 : 1;
      k1 = p->fluid[e] ? 1 : 3;
    }
    for (int q = 0; q < P; ++q)
      for (int k = k0; k < k1; ++k) p->mi[p->conn[e * P + q] * cc + k] += me[q];
  }
  for (int64_t i = 0; i < p->G * cc; ++i) p->mi[i] = p->mi[i] > 0 ? 1.0 / p->mi[i] : 0.0;
  if (d->physics == ORC_COUPLED2D) build_coupling(p);
  size_t nf = (size_t)(p->G * p->c);
  p->u = (double *)xcalloc(nf, sizeof(double));
  p->v = (double *)xcalloc(nf, sizeof(double));
  p->a = (double *)xcalloc(nf, sizeof(double));
  p->a_ = (double *)xcalloc(nf, sizeof(double));
  return p;
}

void orc_destroy(orc_problem *p) {
  if (!p) return;
  free(p->vtx); free(p->par); free(p->conn); free(p->xyz);
  free(p->detJ); free(p->invJ); free(p->mat); free(p->mi); free(p->Ke); free(p->dirichlet);
  free(p->fluid); free(p->cpl);
  free(p->u); free(p->v); free(p->a); free(p->a_);
  free(p->col_off); free(p->col_elems);
  for (int i = 0; i < p->nsrc; ++i) free(p->src[i].wts);
  for (int i = 0; i < p->nrec; ++i) free(p->rec[i].l);
  free(p->src); free(p->rec);
  free(p);
}

int64_t orc_num_nodes(const orc_problem *p) { return p->G; }
int orc_num_components(const orc_problem *p) { return p->c; }
int64_t orc_step_index(const orc_problem *p) { return p->step; }
int orc_node_coords(const orc_problem *p, double *xyz) {
  memcpy(xyz, p->xyz, sizeof(double) * (size_t)(p->G * p->b.dim));
  return 0;
}

/* First element (in element order) whose hull holds x, as in
 * Problem::initializeElements Problem.cpp:77-109 (rank-0 attach rule). */
static int64_t locate(const orc_problem *p, const double *x, double *ref) {
  const int nv = p->b.nv, d = p->b.dim;
  for (int64_t e = 0; e < p->E; ++e) {
    int h = orc_check_hull(p->b.shape, p->vtx + e * nv * d, x);
    if (h < 0) return -2;
    if (h == 1) {
      if (orc_inverse_map(p->b.shape, p->vtx + e * nv * d, x, ref)) return -2;
      return e;
    }
  }
  set_err("point (%g, %g, %g) is outside the mesh", x[0], x[1], d == 3 ? x[2] : 0.0);
  return -1;
}

int orc_add_source(orc_problem *p, const double *x, double f0, double t0, double amp,
                   int kind, const double *comp) {
  const basis_t *b = &p->b;
  const int P = b->P, c = p->c, d = b->dim;
  if (kind == 1 && p->d.physics == ORC_ACOUSTIC) { set_err("moment tensor needs elastic physics"); return -1; }
  double ref[3] = {0, 0, 0};
  int64_t e = locate(p, x, ref);
  if (e < 0) return -1;
  /* components this element's physics pushes: coupled fluid u, solid ux uy */
  int k0 = 0, k1 = c;
  if (p->d.physics == ORC_COUPLED2D) {
    k0 = p->fluid[e] ? 0 : 1;
    k1 = p->fluid[e] ? 1 : 3;
    if (kind == 1 && p->fluid[e]) { set_err("moment tensor source in a fluid element"); return -1; }
  }
  p->src = (src_t *)realloc(p->src, sizeof(src_t) * (size_t)(p->nsrc + 1));
  src_t *s = &p->src[p->nsrc];
  s->elem = e; s->f0 = f0; s->t0 = t0; s->amp = amp;
  memcpy(s->ref, ref, sizeof ref);
  s->wts = (double *)xcalloc((size_t)(P * c), sizeof(double));
  const double *vtx = p->vtx + e * b->nv * d;
  if (kind == 0) {
    /* delta coefficients l_p/(w_p detJ_p) (getDeltaFunctionCoefficients),
     * times direction (Ricker::fire), then x w_p detJ_p
     * (applyTestAndIntegrate, Scalar.cpp:87) -- omitted for elastic in the
     * reference-literal mode (Elastic3D.cpp:126-133, quirk Q2). */
    double delta[ORC_MAX_P], integ[ORC_MAX_P];
    orc_element_delta(b->shape, b->n - 1, vtx, p->d.flags, ref, delta);
    int scale = !(p->d.physics == ORC_ELASTIC3D && (p->d.flags & ORC_Q2_ELASTIC_SRC_UNSCALED));
    if (scale) orc_element_test(b->shape, b->n - 1, vtx, p->d.flags, delta, integ);
    for (int q = 0; q < P; ++q)
      for (int a = k0; a < k1; ++a)
        s->wts[q * c + a] = (scale ? integ[q] : delta[q]) * comp[a];
  } else {
    /* moment tensor: f_{q,a} = sum_b M_ab dphi_q/dx_b (x_s);
     * 3-D comp = [Mxx Myy Mzz Myz Mxz Mxy], 2-D comp = [Mxx Myy Mxy] */
    double l[ORC_MAX_P], dl[ORC_MAX_P * 3], det, iJ[9];
    tensor_lagrange(b, ref, l, dl);
    orc_p1_jacobian(b->shape, vtx, ref, p->d.flags, &det, iJ);
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (d == 2) {
      M[0][0] = comp[0]; M[1][1] = comp[1]; M[0][1] = M[1][0] = comp[2];
    } else {
      M[0][0] = comp[0]; M[1][1] = comp[1]; M[2][2] = comp[2];
      M[1][2] = M[2][1] = comp[3]; M[0][2] = M[2][0] = comp[4]; M[0][1] = M[1][0] = comp[5];
    }
    for (int q = 0; q < P; ++q) {
      double gx[3] = {0, 0, 0};
      for (int a = 0; a < d; ++a) {
        double sacc = 0;
        for (int k = 0; k < d; ++k) sacc += iJ[a * d + k] * dl[q * d + k];
        gx[a] = sacc;
      }
      for (int a = 0; a < d; ++a) {
        double f = 0;
        for (int k = 0; k < d; ++k) f += M[a][k] * gx[k];
        s->wts[q * c + k0 + a] = f;
      }
    }
  }
  return p->nsrc++;
}

int orc_add_receiver(orc_problem *p, const double *x) {
  double ref[3] = {0, 0, 0};
  int64_t e = locate(p, x, ref);
  if (e < 0) return -1;
  p->rec = (rec_t *)realloc(p->rec, sizeof(rec_t) * (size_t)(p->nrec + 1));
  rec_t *r = &p->rec[p->nrec];
  r->elem = e;
  r->l = (double *)xcalloc((size_t)p->b.P, sizeof(double));
  tensor_lagrange(&p->b, ref, r->l, NULL);
  return p->nrec++;
}

int orc_set_field(orc_problem *p, int which, const double *vals) {
  double *f = which == 0 ? p->u : which == 1 ? p->v : NULL;
  if (!f) { set_err("bad field"); return -1; }
  memcpy(f, vals, sizeof(double) * (size_t)(p->G * p->c));
  return 0;
}

int orc_get_field(const orc_problem *p, int which, double *vals) {
  const double *f = which == 0 ? p->u : which == 1 ? p->v : which == 2 ? p->a : NULL;
  if (!f) { set_err("bad field"); return -1; }
  memcpy(vals, f, sizeof(double) * (size_t)(p->G * p->c));
  return 0;
}

int orc_inverse_mass(const orc_problem *p, double *mi) {
  for (int64_t g = 0; g < p->G; ++g) mi[g] = p->mi[g * p->c];
  return 0;
}

int orc_inverse_mass_c(const orc_problem *p, double *mi) {
  memcpy(mi, p->mi, sizeof(double) * (size_t)(p->G * p->c));
  return 0;
}

int orc_set_dirichlet(orc_problem *p, int64_t n, const int64_t *nodes) {
  free(p->dirichlet);
  p->dirichlet = NULL;
  if (n <= 0) return 0;
  p->dirichlet = (char *)xcalloc((size_t)p->G, 1);
  for (int64_t k = 0; k < n; ++k) {
    if (nodes[k] < 0 || nodes[k] >= p->G) { set_err("node out of range"); return -1; }
    p->dirichlet[nodes[k]] = 1;
  }
  return 0;
}

/* HomogeneousDirichlet::computeStiffnessTerm (HomogeneousDirichlet.cpp:65-73) */
static void zero_dirichlet_rows(const orc_problem *p, int64_t e, double *ke) {
  if (!p->dirichlet) return;
  const int P = p->b.P, c = p->c;
  for (int q = 0; q < P; ++q)
    if (p->dirichlet[p->conn[e * P + q]])
      for (int k = 0; k < c; ++k) ke[q * c + k] = 0.0;
}

/* a = f(t) - K u, assembled.  Problem::assembleIntoGlobalDof Problem.cpp:143-214. */
static void assemble(orc_problem *p, const double *u, double t, double *a, int with_src) {
  const int P = p->b.P, c = p->c;
  memset(a, 0, sizeof(double) * (size_t)(p->G * c));
  if (p->d.threads <= 1) {
    double ue[ORC_MAX_P * 3], ke[ORC_MAX_P * 3];
    for (int64_t e = 0; e < p->E; ++e) {
      const int64_t *cn = p->conn + e * P;
      for (int q = 0; q < P; ++q)
        for (int k = 0; k < c; ++k) ue[q * c + k] = u[cn[q] * c + k];
      element_stiffness(p, e, ue, ke);
      zero_dirichlet_rows(p, e, ke);
      for (int q = 0; q < P; ++q)
        for (int k = 0; k < c; ++k) a[cn[q] * c + k] += -ke[q * c + k];
    }
  } else if (p->ncolours == 0) {
    double *buf = (double *)xcalloc((size_t)(p->E * P * c), sizeof(double));
#pragma omp parallel for num_threads(p->d.threads) schedule(static)
    for (int64_t e = 0; e < p->E; ++e) {
      double ue[ORC_MAX_P * 3];
      const int64_t *cn = p->conn + e * P;
      for (int q = 0; q < P; ++q)
        for (int k = 0; k < c; ++k) ue[q * c + k] = u[cn[q] * c + k];
      element_stiffness(p, e, ue, buf + e * P * c);
      zero_dirichlet_rows(p, e, buf + e * P * c);
    }
    for (int64_t e = 0; e < p->E; ++e) {
      const int64_t *cn = p->conn + e * P;
      for (int q = 0; q < P; ++q)
        for (int k = 0; k < c; ++k) a[cn[q] * c + k] += -buf[(e * P + q) * c + k];
    }
    free(buf);
  } else {
    for (int col = 0; col < p->ncolours; ++col) {
      const int64_t lo = p->col_off[col], hi = p->col_off[col + 1];
#pragma omp parallel for num_threads(p->d.threads) schedule(static)
      for (int64_t i = lo; i < hi; ++i) {
        double ue[ORC_MAX_P * 3], ke[ORC_MAX_P * 3];
        const int64_t e = p->col_elems[i];
        const int64_t *cn = p->conn + e * P;
        for (int q = 0; q < P; ++q)
          for (int k = 0; k < c; ++k) ue[q * c + k] = u[cn[q] * c + k];
        element_stiffness(p, e, ue, ke);
        zero_dirichlet_rows(p, e, ke);
        for (int q = 0; q < P; ++q)
          for (int k = 0; k < c; ++k) a[cn[q] * c + k] += -ke[q * c + k];
      }
    }
  }
  if (with_src && p->ncpl) {
    /* computeSurfaceIntegral (Problem.cpp:191-198) with the velocity field */
    for (int64_t i = 0; i < p->ncpl; ++i) {
      const cpl_t *k = &p->cpl[i];
      const int64_t g = p->conn[k->e * P + k->q];
      if (k->kind == 0) {
        a[g * 3] += k->cx * p->v[g * 3 + 1] + k->cy * p->v[g * 3 + 2];
      } else {
        a[g * 3 + 1] += k->cx * p->v[g * 3];
        a[g * 3 + 2] += k->cy * p->v[g * 3];
      }
    }
  }
  if (with_src) {
    /* computeSourceTerm at time t (Problem.cpp:196; Scalar.cpp:79-88;
     * Elastic3D.cpp:126-133), sources in attach order. */
    for (int i = 0; i < p->nsrc; ++i) {
      const src_t *s = &p->src[i];
      double stf = orc_ricker(t, s->f0, s->t0, s->amp);
      const int64_t *cn = p->conn + s->elem * P;
      for (int q = 0; q < P; ++q)
        for (int k = 0; k < c; ++k) a[cn[q] * c + k] += s->wts[q * c + k] * stf;
    }
  }
}

int orc_apply_stiffness(orc_problem *p, const double *u, double *ku) {
  assemble(p, u, 0.0, ku, 0);
  return 0;
}

int orc_acceleration(orc_problem *p, double t, double *a) {
  assemble(p, p->u, t, a, 1);
  const int c = p->c;
  for (int64_t g = 0; g < p->G; ++g)
    for (int k = 0; k < c; ++k) a[g * c + k] *= p->mi[g * c + k];
  return 0;
}

int orc_run(orc_problem *p, int64_t nsteps, double dt, double *seis) {
  const int c = p->c, P = p->b.P;
  const int64_t G = p->G;
  const double acl = 0.5 * dt, dsp = 0.5 * dt * dt;
  /* components advanced by takeTimeStep: Order2Newmark.cpp:93-96 lists
   * {"ax","ay","ax","a"} (2-D and 3-D elastic: x twice, z never);
   * corrected mode advances each component once. */
  int comps[4], ncomp = 0;
  if (c == 1) {
    comps[ncomp++] = 0;
  } else if ((p->d.flags & ORC_Q1_Z_NOT_ADVANCED) && p->d.physics == ORC_COUPLED2D) {
    comps[ncomp++] = 1; comps[ncomp++] = 2; comps[ncomp++] = 1; comps[ncomp++] = 0;
  } else if (p->d.flags & ORC_Q1_Z_NOT_ADVANCED) {
    comps[ncomp++] = 0; comps[ncomp++] = 1; comps[ncomp++] = 0;
  } else {
    for (int k = 0; k < c; ++k) comps[ncomp++] = k;
  }
  for (int64_t n = 0; n < nsteps; ++n) {
    const double t = (double)p->step * dt; /* integer step count (quirk Q11) */
    assemble(p, p->u, t, p->a, 1);
    /* applyInverseMassMatrix Order2Newmark.cpp:68-83 */
    for (int64_t g = 0; g < G; ++g)
      for (int k = 0; k < c; ++k) p->a[g * c + k] *= p->mi[g * c + k];
    /* takeTimeStep Order2Newmark.cpp:85-114 (VecAXPBYPCZ twice + VecCopy) */
    for (int ci = 0; ci < ncomp; ++ci) {
      const int k = comps[ci];
      for (int64_t g = 0; g < G; ++g) {
        const int64_t i = g * c + k;
        p->v[i] = acl * p->a[i] + acl * p->a_[i] + 1.0 * p->v[i];
        p->u[i] = dt * p->v[i] + dsp * p->a[i] + 1.0 * p->u[i];
        p->a_[i] = p->a[i];
      }
    }
    p->step++;
    if (seis) {
      for (int r = 0; r < p->nrec; ++r) {
        const rec_t *rc = &p->rec[r];
        const int64_t *cn = p->conn + rc->elem * P;
        for (int k = 0; k < c; ++k) {
          /* Kahan-compensated FP64 sum */
          double s = 0, comp = 0;
          for (int q = 0; q < P; ++q) {
            double y = rc->l[q] * p->u[cn[q] * c + k] - comp;
            double tt = s + y;
            comp = (tt - s) - y;
            s = tt;
          }
          seis[((int64_t)r * c + k) * nsteps + n] = s;
        }
      }
    }
  }
  return 0;
}

double orc_max_eigenvalue(orc_problem *p, int iters, uint64_t seed) {
  const int c = p->c;
  const int64_t N = p->G * c;
  double *x = (double *)xcalloc((size_t)N, sizeof(double));
  double *y = (double *)xcalloc((size_t)N, sizeof(double));
  uint64_t st = seed ? seed : 1;
  for (int64_t i = 0; i < N; ++i) {
    st = mix64(st);
    x[i] = ((st >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
  }
  double lam = 0;
  for (int it = 0; it < iters; ++it) {
    /* y = M^-1 K x  (assemble gives -K x) */
    assemble(p, x, 0.0, y, 0);
    double num = 0, den = 0;
    for (int64_t g = 0; g < p->G; ++g)
      for (int k = 0; k < c; ++k) {
        int64_t i = g * c + k;
        if (p->mi[i] == 0.0) { y[i] = 0.0; continue; }
        y[i] = -y[i] * p->mi[i];
        num += y[i] * y[i] / p->mi[i];
        den += x[i] * y[i] / p->mi[i];
      }
    lam = num / den;
    double nrm = 0;
    for (int64_t i = 0; i < N; ++i) nrm = fmax(nrm, fabs(y[i]));
    for (int64_t i = 0; i < N; ++i) x[i] = y[i] / nrm;
  }
  free(x); free(y);
  return lam;
}

double orc_energy(orc_problem *p) {
  const int c = p->c;
  const int64_t N = p->G * c;
  double *ku = (double *)xcalloc((size_t)N, sizeof(double));
  assemble(p, p->u, 0.0, ku, 0); /* -K u */
  double ek = 0, ep = 0;
  for (int64_t g = 0; g < p->G; ++g)
    for (int k = 0; k < c; ++k) {
      int64_t i = g * c + k;
      if (p->mi[i] != 0.0) ek += 0.5 * p->v[i] * p->v[i] / p->mi[i];
      ep += -0.5 * p->u[i] * ku[i];
    }
  free(ku);
  return ek + ep;
}
