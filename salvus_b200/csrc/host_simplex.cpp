// host_simplex.cpp -- the P3 mass-lumped simplex reference elements and the
// flattening of triangle / tetrahedron meshes.
//
// Reference elements (Triangle.cpp:24-107, Tetrahedra.cpp:66-151 with the
// tables of the sympy generators triangle_points_weights_polys.py and
// tetrahedra_points_weights_polys.py / BuildNodesTetrahedraP3.py):
//   triangle     12 nodes: 3 interior, 2 per edge, 3 vertices; space
//                P3 + b P1 (b the cubic bubble);
//   tetrahedron  50 nodes: 10 interior, 6 per face, 2 per edge, 4 vertices;
//                space P3 + b_T P2 + sum_f b_f P2 (b_T the quartic interior
//                bubble, b_f the cubic face bubbles).
// The nodes are the reference's, in its closure order (interior, faces,
// edges, vertices); the quadrature weights are the nodal weights of the
// mass-lumped rule.  The nodal basis is the unique interpolant in that
// space; here it is built from barycentric generators of the space (cubic
// barycentric monomials, bubbles times barycentric quadratics) and a
// Vandermonde inverse in extended precision.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <unordered_map>

#include "internal.h"

namespace salvus {

namespace {

// Barycentric coordinates as affine functions of the reference point:
// lambda_v(ref) = L0[v] + sum_k L1[v][k] ref_k (the P1 vertex weights).
struct Affine {
  int nv;
  double c0[4];
  double c1[4][3];
};

Affine barycentric(int shape) {
  Affine a{};
  a.nv = shape_nv(shape);
  double zero[3] = {0, 0, 0}, w0[4], w[4];
  p1_weights(shape, zero, w0);
  for (int v = 0; v < a.nv; ++v) a.c0[v] = w0[v];
  for (int k = 0; k < shape_dim(shape); ++k) {
    double e[3] = {0, 0, 0};
    e[k] = 1;
    p1_weights(shape, e, w);
    for (int v = 0; v < a.nv; ++v) a.c1[v][k] = w[v] - w0[v];
  }
  return a;
}

// Exponent vectors of the generators (products of barycentric powers).
std::vector<std::array<int, 4>> generators(int shape) {
  std::vector<std::array<int, 4>> g;
  const int nv = shape_nv(shape);
  // all cubic barycentric monomials (span P3)
  for (int a = 0; a <= 3; ++a)
    for (int b = 0; b <= 3 - a; ++b)
      for (int c = 0; c <= 3 - a - b; ++c) {
        int d = 3 - a - b - c;
        if (nv == 3 && d != 0) continue;
        g.push_back({a, b, c, nv == 3 ? 0 : d});
      }
  if (shape == SALVUS_TRI) {
    // cubic bubble l0 l1 l2 times l1 and l2 (with P3, spans P3 + b P1)
    g.push_back({1, 2, 1, 0});
    g.push_back({1, 1, 2, 0});
    return g;
  }
  // interior bubble l0 l1 l2 l3 times every barycentric quadratic
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) {
      std::array<int, 4> e = {1, 1, 1, 1};
      e[i]++;
      e[j]++;
      g.push_back(e);
    }
  // face bubble (product over the face's vertices) times five quadratics of
  // the face's barycentrics (the sixth is dependent modulo P3 and b_T P2)
  for (int opp = 0; opp < 4; ++opp) {
    int f[3], k = 0;
    for (int v = 0; v < 4; ++v)
      if (v != opp) f[k++] = v;
    const int mult[5][2] = {{f[0], f[0]}, {f[1], f[1]}, {f[2], f[2]}, {f[0], f[1]}, {f[0], f[2]}};
    for (auto &m : mult) {
      std::array<int, 4> e = {1, 1, 1, 1};
      e[opp] = 0;
      e[m[0]]++;
      e[m[1]]++;
      g.push_back(e);
    }
  }
  return g;
}

// Generator values (and reference gradients) at a reference point.
void eval_generators(int shape, const std::vector<std::array<int, 4>> &gen, const double *ref,
                     long double *val, long double *grad /* [m][3] or null */) {
  const Affine A = barycentric(shape);
  const int dim = shape_dim(shape);
  long double lam[4];
  for (int v = 0; v < A.nv; ++v) {
    long double s = A.c0[v];
    for (int k = 0; k < dim; ++k) s += (long double)A.c1[v][k] * ref[k];
    lam[v] = s;
  }
  for (size_t m = 0; m < gen.size(); ++m) {
    const auto &e = gen[m];
    long double p = 1;
    for (int v = 0; v < A.nv; ++v)
      for (int r = 0; r < e[v]; ++r) p *= lam[v];
    val[m] = p;
    if (!grad) continue;
    for (int k = 0; k < 3; ++k) grad[m * 3 + k] = 0;
    for (int v = 0; v < A.nv; ++v) {
      if (e[v] == 0) continue;
      long double d = e[v];
      for (int u = 0; u < A.nv; ++u)
        for (int r = 0; r < e[u] - (u == v ? 1 : 0); ++r) d *= lam[u];
      for (int k = 0; k < dim; ++k) grad[m * 3 + k] += d * A.c1[v][k];
    }
  }
}

// Gauss-Jordan inverse with partial pivoting.
bool invert(int n, std::vector<long double> &A) {
  std::vector<long double> I((size_t)n * n, 0);
  for (int i = 0; i < n; ++i) I[(size_t)i * n + i] = 1;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (fabsl(A[(size_t)r * n + c]) > fabsl(A[(size_t)piv * n + c])) piv = r;
    if (A[(size_t)piv * n + c] == 0) return false;
    for (int k = 0; k < n && piv != c; ++k) {
      std::swap(A[(size_t)c * n + k], A[(size_t)piv * n + k]);
      std::swap(I[(size_t)c * n + k], I[(size_t)piv * n + k]);
    }
    const long double inv = 1 / A[(size_t)c * n + c];
    for (int k = 0; k < n; ++k) {
      A[(size_t)c * n + k] *= inv;
      I[(size_t)c * n + k] *= inv;
    }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const long double f = A[(size_t)r * n + c];
      if (f == 0) continue;
      for (int k = 0; k < n; ++k) {
        A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
        I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
      }
    }
  }
  A.swap(I);
  return true;
}

// Reference nodes.  Triangle: the 4-digit node table of the reference
// generator (p3ReferenceNodes), closure order interior (0-2), edges (3-8),
// vertices (9-11).
const double kTriNodes[12][2] = {
    {-0.5853, -0.5853}, {0.1706, -0.5853}, {-0.5853, 0.1706}, {-0.413, -1.0},
    {0.413, -1.0},      {0.413, -0.413},   {-0.413, 0.413},   {-1.0, 0.413},
    {-1.0, -0.413},     {-1.0, -1.0},      {1.0, -1.0},       {-1.0, 1.0}};

// Tetrahedron: orbits of the Chin-Joe-Kong / Mulder / Van Veldhuizen (1999)
// rule, written as barycentric weights on the reference corners O X Y Z
// (= vertices v0 v2 v1 v3 of the TetP1 map), in the reference's order:
// 4 corner-pulled interior points, 6 edge-pair interior points, per face
// (O,Y,X) (O,Z,Y) (O,X,Z) (X,Y,Z) the beta1 then beta2 orbits, 2 points per
// edge (O,Y) (Y,X) (X,O) (O,Z) (Z,Y) (X,Z), then corners O Y X Z.
void tet_nodes(double (*x)[3]) {
  const double b1 = 0.1972862280257976, b2 = 0.4256461243139345, al = 0.2928294047674109;
  const double ga = 0.9503775858394107e-01, de = 0.1252462362578136;
  const double corner[4][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};  // O X Y Z
  enum { O = 0, X = 1, Y = 2, Z = 3 };
  int k = 0;
  auto put = [&](const double *wt) {
    for (int m = 0; m < 3; ++m) {
      double s = 0;
      for (int c = 0; c < 4; ++c) s += wt[c] * corner[c][m];
      x[k][m] = s;
    }
    ++k;
  };
  for (int c = 0; c < 4; ++c) {
    double wt[4] = {ga, ga, ga, ga};
    wt[c] = 1 - 3 * ga;
    put(wt);
  }
  // (1-2 delta) * midpoint(a,b) + 2 delta * midpoint(c,d)
  const int pr[6][4] = {{O, Z, X, Y}, {O, X, Y, Z}, {O, Y, X, Z},
                        {X, Y, O, Z}, {Y, Z, O, X}, {X, Z, O, Y}};
  for (auto &p : pr) {
    double wt[4] = {0, 0, 0, 0};
    wt[p[0]] += 0.5 * (1 - 2 * de);
    wt[p[1]] += 0.5 * (1 - 2 * de);
    wt[p[2]] += de;
    wt[p[3]] += de;
    put(wt);
  }
  const int face[4][3] = {{O, Y, X}, {O, Z, Y}, {O, X, Z}, {X, Y, Z}};
  for (auto &f : face)
    for (double be : {b1, b2})
      for (int i = 0; i < 3; ++i) {
        double wt[4] = {0, 0, 0, 0};
        wt[f[i]] = 1 - 2 * be;
        wt[f[(i + 1) % 3]] = be;
        wt[f[(i + 2) % 3]] = be;
        put(wt);
      }
  const int edge[6][2] = {{O, Y}, {Y, X}, {X, O}, {O, Z}, {Z, Y}, {X, Z}};
  for (auto &e : edge)
    for (int o = 0; o < 2; ++o) {
      double wt[4] = {0, 0, 0, 0};
      wt[e[0]] = o == 0 ? 1 - al : al;
      wt[e[1]] = o == 0 ? al : 1 - al;
      put(wt);
    }
  for (int c : {O, Y, X, Z}) {
    double wt[4] = {0, 0, 0, 0};
    wt[c] = 1;
    put(wt);
  }
}

}  // namespace

int make_simplex_basis(int shape, int order, Basis *b) {
  if (order != 3)
    return fail(SALVUS_E_UNSUPPORTED, "%s elements are built for order 3 only (got %d)",
                shape == SALVUS_TRI ? "triangle" : "tetrahedron", order);
  const bool tet = shape == SALVUS_TET;
  const int P = tet ? 50 : 12, dim = tet ? 3 : 2;
  b->shape = shape;
  b->simplex = true;
  b->order = 3;
  b->n = 4;
  b->dim = dim;
  b->P = P;
  b->nv = dim + 1;
  b->nodes.assign((size_t)P * 3, 0.0);
  b->sw.assign(P, 0.0);
  if (tet) {
    double x[50][3];
    tet_nodes(x);
    for (int q = 0; q < P; ++q)
      for (int m = 0; m < 3; ++m) b->nodes[(size_t)q * 3 + m] = x[q][m];
    // nodal weights x6 (unit-volume normalisation of the reference rule)
    const double w0 = 0.2143608668049743e-03, wa = 0.8268179517797114e-03;
    const double wb1 = 0.1840177904191860e-02, wb2 = 0.1831324329245650e-02;
    const double wg = 0.7542468904648131e-02, wd = 0.1360991755970793e-01;
    for (int q = 0; q < P; ++q) {
      double w = q < 4 ? wg : q < 10 ? wd : q < 34 ? (((q - 10) % 6) < 3 ? wb1 : wb2) : q < 46 ? wa : w0;
      b->sw[q] = 6.0 * w;
    }
  } else {
    for (int q = 0; q < P; ++q) {
      b->nodes[(size_t)q * 3 + 0] = kTriNodes[q][0];
      b->nodes[(size_t)q * 3 + 1] = kTriNodes[q][1];
    }
    // closed-form weights of the 12-point rule (sum 1)
    const double r7 = std::sqrt(7.0);
    const double wi = (84 * r7 + 294) / (400 * r7 + 1280);
    const double we = 2 * r7 * std::pow(2 + r7, 4) / (9520 * r7 + 25280);
    const double wv = (1838 * r7 + 4942) / (124080 * r7 + 330960);
    for (int q = 0; q < P; ++q) b->sw[q] = q < 3 ? wi : q < 9 ? we : wv;
  }
  const auto gen = generators(shape);
  if ((int)gen.size() != P) return fail(SALVUS_E_INVALID, "simplex generator count mismatch");
  std::vector<long double> V((size_t)P * P), g(P), dg((size_t)P * 3);
  for (int q = 0; q < P; ++q) {
    eval_generators(shape, gen, &b->nodes[(size_t)q * 3], g.data(), nullptr);
    for (int m = 0; m < P; ++m) V[(size_t)q * P + m] = g[m];
  }
  if (!invert(P, V)) return fail(SALVUS_E_INVALID, "singular simplex Vandermonde matrix");
  b->C.assign((size_t)P * P, 0.0);
  for (size_t i = 0; i < V.size(); ++i) b->C[i] = (double)V[i];
  b->SD.assign((size_t)dim * P * P, 0.0);
  for (int q = 0; q < P; ++q) {
    eval_generators(shape, gen, &b->nodes[(size_t)q * 3], g.data(), dg.data());
    for (int k = 0; k < dim; ++k)
      for (int j = 0; j < P; ++j) {
        long double s = 0;
        for (int m = 0; m < P; ++m) s += dg[(size_t)m * 3 + k] * V[(size_t)m * P + j];
        b->SD[((size_t)k * P + j) * P + q] = (double)s;
      }
  }
  return SALVUS_OK;
}

void simplex_basis_at(const Basis &b, const double *ref, double *phi, double *dphi) {
  const int P = b.P;
  static thread_local std::vector<std::array<int, 4>> gen_tri, gen_tet;
  auto &gen = b.shape == SALVUS_TRI ? gen_tri : gen_tet;
  if (gen.empty()) gen = generators(b.shape);
  std::vector<long double> g(P), dg((size_t)P * 3);
  eval_generators(b.shape, gen, ref, g.data(), dphi ? dg.data() : nullptr);
  for (int i = 0; i < P; ++i) {
    long double v = 0, d[3] = {0, 0, 0};
    for (int m = 0; m < P; ++m) {
      const long double c = b.C[(size_t)m * P + i];
      v += c * g[m];
      if (dphi)
        for (int k = 0; k < 3; ++k) d[k] += c * dg[(size_t)m * 3 + k];
    }
    phi[i] = (double)v;
    if (dphi)
      for (int k = 0; k < 3; ++k) dphi[i * 3 + k] = (double)d[k];
  }
}

// Node sharing on simplices: a node of element e with barycentric
// coordinates lambda (w.r.t. the element's vertices) is identified by the
// global ids of the vertices where lambda > 0 together with the quantised
// lambda values, sorted by global vertex id.  Edge and face nodes therefore
// match across elements whatever the local vertex order; interior nodes are
// private to their element.  (Mesh::setupGlobalDof, Mesh.cpp:361-452, shares
// DOFs on vertices / edges / faces through the DMPlex section.)
int flatten_simplex(salvus_mesh *m, const int64_t *cells, int64_t n_vertices) {
  const int P = m->P, nv = m->nv;
  const int64_t E = m->E;
  struct Key {
    std::array<int64_t, 6> k;
    bool operator==(const Key &o) const { return k == o.k; }
  };
  struct KeyHash {
    size_t operator()(const Key &x) const {
      uint64_t h = 1469598103934665603ull;
      for (int64_t v : x.k) {
        h ^= (uint64_t)v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
        h *= 1099511628211ull;
      }
      return (size_t)h;
    }
  };
  // per local node: support vertices and quantised weights
  std::vector<int> nsup(P);
  std::vector<std::array<int, 4>> sup(P);
  std::vector<std::array<int64_t, 4>> qw(P);
  int n_interior = 0;
  for (int q = 0; q < P; ++q) {
    double ref[3], w[4];
    point_ref(m->basis, q, ref);
    p1_weights(m->shape, ref, w);
    nsup[q] = 0;
    for (int v = 0; v < nv; ++v)
      if (w[v] > 1e-9) {
        sup[q][nsup[q]] = v;
        qw[q][nsup[q]] = (int64_t)std::llround(w[v] * 1e9);
        nsup[q]++;
      }
    if (nsup[q] == nv) n_interior++;
  }
  m->conn.assign((size_t)(E * P), -1);
  std::vector<int64_t> vtx_id(n_vertices, -1);
  std::unordered_map<Key, int64_t, KeyHash> shared;
  shared.reserve((size_t)(E * (nv == 3 ? 3 : 12)));
  int64_t G = 0;
  for (int64_t e = 0; e < E; ++e) {
    const int64_t *cv = cells + e * nv;
    int64_t interior_base = G;
    G += n_interior;
    int interior_k = 0;
    for (int q = 0; q < P; ++q) {
      int64_t gid;
      if (nsup[q] == nv) {
        gid = interior_base + interior_k++;
      } else if (nsup[q] == 1) {
        const int64_t v = cv[sup[q][0]];
        if (v < 0 || v >= n_vertices) return fail(SALVUS_E_INVALID, "cell vertex out of range");
        if (vtx_id[v] < 0) vtx_id[v] = G++;
        gid = vtx_id[v];
      } else {
        std::array<std::pair<int64_t, int64_t>, 3> pr;
        const int ns = nsup[q];
        for (int i = 0; i < ns; ++i) pr[i] = {cv[sup[q][i]], qw[q][i]};
        std::sort(pr.begin(), pr.begin() + ns);
        Key key;
        key.k.fill(-1);
        for (int i = 0; i < ns; ++i) {
          key.k[2 * i] = pr[i].first;
          key.k[2 * i + 1] = pr[i].second;
        }
        auto it = shared.find(key);
        if (it == shared.end()) {
          gid = G++;
          shared.emplace(key, gid);
        } else {
          gid = it->second;
        }
      }
      if (gid >= 2147483647) return fail(SALVUS_E_UNSUPPORTED, "too many nodes for int32");
      m->conn[(size_t)(e * P + q)] = (int32_t)gid;
    }
  }
  m->G = G;
  return SALVUS_OK;
}

}  // namespace salvus
