// host_mesh.cpp -- one-time flattening of a conforming quad / hex mesh (and,
// through flatten_simplex, triangle / tetrahedron meshes) into
// GLL connectivity and the node -> element-point incidence used by the
// deterministic assembly.  Semantics of Mesh::setupGlobalDof (Mesh.cpp:361-452:
// DMPlexCreateSection + spectral closure permutation): nodes on shared
// vertices, edges and faces are shared; element-local order is the tensor
// order r + n s + n^2 t (identity closure, TensorQuad.cpp:41, Hexahedra.cpp:57).
//
// Shared entities are keyed topologically by global vertex ids, so the
// numbering needs no coordinates and no tolerances.
#include <algorithm>
#include <cmath>
#include <array>
#include <cstring>
#include <unordered_map>

#include "internal.h"

namespace salvus {

namespace {

// local corner bits (ci, cj[, ck]) -> element vertex (PETSc right-hand order)
const int kQuadCorner[2][2] = {{0, 3}, {1, 2}};  // [ci][cj]
const int kHexCorner[2][2][2] = {{{0, 4}, {1, 7}}, {{3, 5}, {2, 6}}};  // [ci][cj][ck]

struct Key4 {
  std::array<int64_t, 4> v;
  bool operator==(const Key4 &o) const { return v == o.v; }
};
struct Key4Hash {
  size_t operator()(const Key4 &k) const {
    uint64_t h = 1469598103934665603ull;
    for (int64_t x : k.v) {
      h ^= (uint64_t)x + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
      h *= 1099511628211ull;
    }
    return (size_t)h;
  }
};

}  // namespace

int flatten_simplex(salvus_mesh *m, const int64_t *cells, int64_t n_vertices);
static int flatten_tensor(salvus_mesh *m, const int64_t *cells, int64_t n_vertices);

int flatten_mesh(salvus_mesh *m, const int64_t *cells, int64_t n_vertices) {
  const int dim = m->dim, P = m->P;
  const int64_t E = m->E;
  if ((double)E * P >= 2147483647.0)
    return fail(SALVUS_E_UNSUPPORTED, "mesh too large: E*P = %lld exceeds int32 incidence",
                (long long)(E * P));
  int rc = is_simplex(m->shape) ? flatten_simplex(m, cells, n_vertices)
                                : flatten_tensor(m, cells, n_vertices);
  if (rc) return rc;
  const int64_t G = m->G;
  // node -> incident element points, ascending element order
  m->inc_off.assign((size_t)G + 1, 0);
  for (int64_t i = 0; i < E * P; ++i) m->inc_off[(size_t)m->conn[i] + 1]++;
  for (int64_t g = 0; g < G; ++g) m->inc_off[g + 1] += m->inc_off[g];
  m->inc_idx.assign((size_t)(E * P), 0);
  std::vector<int32_t> fill(m->inc_off.begin(), m->inc_off.end() - 1);
  for (int64_t i = 0; i < E * P; ++i) m->inc_idx[(size_t)fill[m->conn[i]]++] = (int32_t)i;
  // node coordinates (P1 map of the element points)
  m->xyz.assign((size_t)(G * dim), 0.0);
  for (int64_t e = 0; e < E; ++e) {
    const double *v = m->vtx.data() + e * m->nv * dim;
    for (int p = 0; p < P; ++p) {
      double ref[3], x[3];
      point_ref(m->basis, p, ref);
      p1_map(m->shape, v, ref, x);
      int64_t g = m->conn[(size_t)(e * P + p)];
      for (int d = 0; d < dim; ++d) m->xyz[(size_t)(g * dim + d)] = x[d];
    }
  }
  return SALVUS_OK;
}

static int flatten_tensor(salvus_mesh *m, const int64_t *cells, int64_t n_vertices) {
  const int dim = m->dim, n = m->n, N = n - 1, P = m->P;
  const int64_t E = m->E;
  m->conn.assign((size_t)(E * P), -1);
  std::vector<int64_t> vtx_id(n_vertices, -1);
  std::unordered_map<uint64_t, int64_t> edges;
  std::unordered_map<Key4, int64_t, Key4Hash> faces;
  edges.reserve((size_t)(E * (dim == 2 ? 2 : 3) + 16));
  if (dim == 3) faces.reserve((size_t)(E * 3 + 16));
  int64_t G = 0;
  const int nloc = dim == 2 ? 4 : 8;
  for (int64_t e = 0; e < E; ++e) {
    const int64_t *cv = cells + e * nloc;
    auto corner_gid = [&](int ci, int cj, int ck) -> int64_t {
      return dim == 2 ? cv[kQuadCorner[ci][cj]] : cv[kHexCorner[ci][cj][ck]];
    };
    int64_t interior_base = G;
    if (N >= 2) {
      int64_t nint = 1;
      for (int d = 0; d < dim; ++d) nint *= (N - 1);
      G += nint;
    }
    for (int p = 0; p < P; ++p) {
      int idx[3] = {p % n, (p / n) % n, dim == 3 ? p / (n * n) : 0};
      int fixed[3], freed[3], nfix = 0, nfree = 0;
      for (int d = 0; d < dim; ++d) {
        if (idx[d] == 0 || idx[d] == N) fixed[nfix++] = d;
        else freed[nfree++] = d;
      }
      int64_t gid;
      if (nfree == dim) {
        // element interior: a private block reserved when the element starts
        int64_t ii = 0, mul = 1;
        for (int d = 0; d < dim; ++d) { ii += (idx[d] - 1) * mul; mul *= (N - 1); }
        gid = interior_base + ii;
      } else {
        // corners of the entity: fixed dims at their side, free dims at 0/1
        int cb[3];
        for (int d = 0; d < dim; ++d) cb[d] = idx[d] == N ? 1 : 0;
        if (nfree == 0) {
          int64_t v = corner_gid(cb[0], cb[1], cb[2]);
          if (v < 0 || v >= n_vertices) return fail(SALVUS_E_INVALID, "cell vertex out of range");
          if (vtx_id[v] < 0) vtx_id[v] = G++;
          gid = vtx_id[v];
        } else if (nfree == 1) {
          const int a = freed[0];
          int c0[3] = {cb[0], cb[1], cb[2]}, c1[3] = {cb[0], cb[1], cb[2]};
          c0[a] = 0; c1[a] = 1;
          int64_t g0 = corner_gid(c0[0], c0[1], c0[2]), g1 = corner_gid(c1[0], c1[1], c1[2]);
          int t = idx[a];
          if (g0 > g1) { std::swap(g0, g1); t = N - t; }
          uint64_t key = ((uint64_t)g0 << 32) | (uint64_t)g1;
          auto it = edges.find(key);
          int64_t base;
          if (it == edges.end()) { base = G; G += N - 1; edges.emplace(key, base); }
          else base = it->second;
          gid = base + (t - 1);
        } else {
          const int a = freed[0], b = freed[1];
          int64_t cg[2][2];
          for (int sa = 0; sa < 2; ++sa)
            for (int sb = 0; sb < 2; ++sb) {
              int cc[3] = {cb[0], cb[1], cb[2]};
              cc[a] = sa; cc[b] = sb;
              cg[sa][sb] = corner_gid(cc[0], cc[1], cc[2]);
            }
          int oa = 0, ob = 0;
          for (int sa = 0; sa < 2; ++sa)
            for (int sb = 0; sb < 2; ++sb)
              if (cg[sa][sb] < cg[oa][ob]) { oa = sa; ob = sb; }
          const bool axis_a = cg[1 - oa][ob] < cg[oa][1 - ob];
          int da = oa ? N - idx[a] : idx[a];
          int db = ob ? N - idx[b] : idx[b];
          int x = axis_a ? da : db, y = axis_a ? db : da;
          Key4 key{{cg[0][0], cg[0][1], cg[1][0], cg[1][1]}};
          std::sort(key.v.begin(), key.v.end());
          auto it = faces.find(key);
          int64_t base;
          if (it == faces.end()) {
            base = G;
            G += (int64_t)(N - 1) * (N - 1);
            faces.emplace(key, base);
          } else {
            base = it->second;
          }
          gid = base + (x - 1) + (int64_t)(N - 1) * (y - 1);
        }
      }
      if (gid >= 2147483647) return fail(SALVUS_E_UNSUPPORTED, "too many nodes for int32");
      m->conn[(size_t)(e * P + p)] = (int32_t)gid;
    }
  }
  m->G = G;
  return SALVUS_OK;
}

// First element in element order whose hull holds x (the rank-0 attach rule
// of Problem::initializeElements, Problem.cpp:77-109), then the inverse map.
int locate_point(const salvus_mesh *m, const double *x, int64_t *elem, double *ref) {
  const int dim = m->dim, nv = m->nv;
  for (int64_t e = 0; e < m->E; ++e) {
    const double *v = m->vtx.data() + e * nv * dim;
    // cheap bounding-box reject before the reference hull rule
    bool out = false;
    for (int d = 0; d < dim && !out; ++d) {
      double lo = v[d], hi = v[d];
      for (int k = 1; k < nv; ++k) {
        lo = std::min(lo, v[k * dim + d]);
        hi = std::max(hi, v[k * dim + d]);
      }
      double pad = 1e-9 * (hi - lo);
      if (x[d] < lo - pad || x[d] > hi + pad) out = true;
    }
    if (out) continue;
    int h = check_hull(m->shape, v, x);
    if (h < 0) return h;
    if (h == 1) {
      *elem = e;
      return inverse_map(m->shape, v, x, ref);
    }
  }
  return fail(SALVUS_E_NOT_FOUND, "point (%g, %g, %g) lies outside the mesh", x[0], x[1],
              dim == 3 ? x[2] : 0.0);
}

// Nodes on the outer boundary: element faces (edges in 2-D) that belong to a
// single element, keyed by their sorted global vertex ids; a point lies on a
// face when its P1 weights vanish on every vertex off the face.
int boundary_nodes(const salvus_mesh *m, std::vector<int64_t> &out) {
  const int nv = m->nv, P = m->P, dim = m->dim;
  // faces of the reference element as vertex lists
  std::vector<std::vector<int>> faces;
  if (is_simplex(m->shape)) {
    for (int opp = 0; opp < nv; ++opp) {
      std::vector<int> f;
      for (int v = 0; v < nv; ++v)
        if (v != opp) f.push_back(v);
      faces.push_back(f);
    }
  } else {
    // vertex v lies on face (d, side) when its reference coordinate d is side
    std::vector<std::array<double, 3>> vref(nv);
    for (int v = 0; v < nv; ++v) {
      // the vertex is the point where its own P1 weight is 1: probe corners
      for (int c = 0; c < (1 << dim); ++c) {
        double ref[3] = {0, 0, 0}, w[8];
        for (int d = 0; d < dim; ++d) ref[d] = ((c >> d) & 1) ? 1.0 : -1.0;
        p1_weights(m->shape, ref, w);
        if (w[v] > 0.5) vref[v] = {ref[0], ref[1], ref[2]};
      }
    }
    for (int d = 0; d < dim; ++d)
      for (double side : {-1.0, 1.0}) {
        std::vector<int> f;
        for (int v = 0; v < nv; ++v)
          if (vref[v][d] == side) f.push_back(v);
        faces.push_back(f);
      }
  }
  // local points of each face
  std::vector<std::vector<int>> face_pts(faces.size());
  for (size_t f = 0; f < faces.size(); ++f)
    for (int q = 0; q < P; ++q) {
      double ref[3], w[8];
      point_ref(m->basis, q, ref);
      p1_weights(m->shape, ref, w);
      bool on = true;
      for (int v = 0; v < nv && on; ++v)
        if (std::find(faces[f].begin(), faces[f].end(), v) == faces[f].end() &&
            std::fabs(w[v]) > 1e-12)
          on = false;
      if (on) face_pts[f].push_back(q);
    }
  // count faces by sorted global vertex keys (vertex ids read back from the
  // connectivity of the element's vertex points)
  std::vector<int> vpt(nv, -1);
  for (int v = 0; v < nv; ++v)
    for (int q = 0; q < P; ++q) {
      double ref[3], w[8];
      point_ref(m->basis, q, ref);
      p1_weights(m->shape, ref, w);
      if (std::fabs(w[v] - 1.0) < 1e-12) vpt[v] = q;
    }
  std::unordered_map<Key4, int, Key4Hash> count;
  count.reserve((size_t)(m->E * faces.size()));
  auto key_of = [&](int64_t e, const std::vector<int> &f) {
    Key4 k{{-1, -1, -1, -1}};
    for (size_t a = 0; a < f.size(); ++a) k.v[a] = m->conn[(size_t)(e * P + vpt[f[a]])];
    std::sort(k.v.begin(), k.v.begin() + f.size());
    return k;
  };
  for (int64_t e = 0; e < m->E; ++e)
    for (auto &f : faces) count[key_of(e, f)]++;
  std::vector<char> flag((size_t)m->G, 0);
  for (int64_t e = 0; e < m->E; ++e)
    for (size_t f = 0; f < faces.size(); ++f)
      if (count[key_of(e, faces[f])] == 1)
        for (int q : face_pts[f]) flag[(size_t)m->conn[(size_t)(e * P + q)]] = 1;
  out.clear();
  for (int64_t g = 0; g < m->G; ++g)
    if (flag[(size_t)g]) out.push_back(g);
  return SALVUS_OK;
}

}  // namespace salvus
