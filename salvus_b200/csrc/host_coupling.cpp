// host_coupling.cpp -- meshes of fluid and solid quadrilaterals
// (SALVUS_COUPLED2D): element classes and the per-point coefficients of the
// fluid-solid coupling surface integrals, built once at mesh creation.
//
// Reference semantics restated:
//  * element class from the model's per-element fluid flag
//    (ExodusModel::getElementType ExodusModel.cpp:473-520): fluid elements run
//    Scalar physics on u, solid ones Elastic2D on ux, uy;
//  * an element couples when an edge neighbour has the other class
//    (Mesh::setupTopology Mesh.cpp:313-350 tags edges with their elements'
//    types, Mesh::TotalCouplingFields Mesh.cpp:505-521, Element::Factory
//    Element.cpp:153-171);
//  * coupled fluid element (ElasticToAcoustic2D, ElasticToAcoustic.cpp:17-41):
//    on EVERY edge that has a neighbour (Mesh::CouplingFields Mesh.cpp:480-503
//    lists them all), a_u += int_edge phi (v_s . n), n the element's outward
//    normal (TensorQuad::getEdgeNormal TensorQuad.cpp:400-418);
//  * coupled solid element (AcousticToElastic2D, AcousticToElastic2D.cpp:
//    18-60): on edges with a fluid neighbour, a_ux and a_uy both get
//    -rho0 int_edge phi v, rho0 the mean vertex RHO of that neighbour;
//  * edge integral (TensorQuad::applyTestAndIntegrateEdge TensorQuad.cpp:
//    476-516): f at the edge's GLL points times the GLL weight times
//    |v_{i+1} - v_i| / 2 for local edge i from vertex i to vertex i + 1.
// The integrals act on the velocity field and add to the element-local
// residual after the stiffness (a = f - K u + s, Problem.cpp:188-198); the
// coefficients of one element point are summed over its coupled edges.
#include <algorithm>
#include <cmath>
#include <map>
#include <unordered_map>

#include "internal.h"

namespace salvus {

int setup_coupled(salvus_mesh *m, const int64_t *cells) {
  const int64_t E = m->E;
  const int n = m->n, P = m->P;
  // classes: FLUID flag per element vertex, 0 or 1, equal at all vertices
  std::vector<char> fluid((size_t)E);
  for (int64_t e = 0; e < E; ++e) {
    const double f0 = m->par[(size_t)e * 4];
    for (int a = 0; a < 4; ++a) {
      const double f = m->par[(size_t)e * 4 + a];
      if (f != f0 || (f != 0.0 && f != 1.0))
        return fail(SALVUS_E_INVALID, "element %lld: FLUID must be 0 or 1 at every vertex",
                    (long long)e);
    }
    fluid[(size_t)e] = f0 == 1.0;
  }
  m->elist.clear();
  m->cls_k.assign((size_t)E, 0);
  for (int pass = 1; pass >= 0; --pass)
    for (int64_t e = 0; e < E; ++e)
      if (fluid[(size_t)e] == pass) {
        m->cls_k[(size_t)e] = (int32_t)(pass ? m->elist.size() : m->elist.size() - m->n_fluid);
        m->elist.push_back((int32_t)e);
        if (pass) m->n_fluid++;
      }
  // edge neighbours: elements sharing the (unordered) global vertex pair
  struct PairHash {
    size_t operator()(const std::pair<int64_t, int64_t> &k) const {
      return (size_t)((uint64_t)k.first * 0x9E3779B97F4A7C15ull ^
                      ((uint64_t)k.second + 0x632BE59BD9B4E019ull));
    }
  };
  std::unordered_map<std::pair<int64_t, int64_t>, int64_t, PairHash> first;  // pair -> e*4+i
  first.reserve((size_t)(2 * E + 16));
  std::vector<int64_t> nbr((size_t)(4 * E), -1);
  for (int64_t e = 0; e < E; ++e)
    for (int i = 0; i < 4; ++i) {
      int64_t a = cells[e * 4 + i], b = cells[e * 4 + (i + 1) % 4];
      if (a > b) std::swap(a, b);
      auto it = first.find({a, b});
      if (it == first.end()) {
        first.emplace(std::make_pair(a, b), e * 4 + i);
      } else {
        nbr[(size_t)(e * 4 + i)] = it->second / 4;
        nbr[(size_t)it->second] = e;
      }
    }
  // per element point: summed coefficients, fluid points then solid points
  std::map<int64_t, std::pair<double, double>> fl, so;
  for (int64_t e = 0; e < E; ++e) {
    const bool fe = fluid[(size_t)e];
    bool other = false;
    for (int i = 0; i < 4; ++i) {
      const int64_t f = nbr[(size_t)(e * 4 + i)];
      if (f >= 0 && fluid[(size_t)f] != fe) other = true;
    }
    if (!other) continue;
    const double *vtx = m->vtx.data() + e * 8;
    for (int i = 0; i < 4; ++i) {
      const int64_t f = nbr[(size_t)(e * 4 + i)];
      if (f < 0) continue;
      if (!fe && fluid[(size_t)f] != 1) continue;  // solid: fluid neighbours only
      const double *v0 = vtx + 2 * i, *v1 = vtx + 2 * ((i + 1) % 4);
      const double dx = v1[0] - v0[0], dy = v1[1] - v0[1];
      const double len = std::sqrt(dx * dx + dy * dy), d = len / 2.0;
      const double nx = dy / len, ny = -dx / len;
      double rho0 = 0.0;
      if (!fe) {
        for (int a = 0; a < 4; ++a) rho0 += m->par[((size_t)2 * E + f) * 4 + a];
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
        const double wd = m->basis.w[j] * d;
        const int64_t ep = e * P + q;
        if (fe) {
          auto &c = fl[ep];
          c.first += wd * nx;
          c.second += wd * ny;
        } else {
          auto &c = so[ep];
          c.first += -rho0 * wd;
          c.second += -rho0 * wd;
        }
      }
    }
  }
  m->n_cpl_fluid = (int64_t)fl.size();
  m->n_cpl = (int64_t)(fl.size() + so.size());
  m->cpl_pts.clear();
  m->cpl_coef.clear();
  for (auto *mp : {&fl, &so})
    for (auto &kv : *mp) {
      m->cpl_pts.push_back((int32_t)kv.first);
      m->cpl_pts.push_back(m->conn[(size_t)kv.first]);
      m->cpl_coef.push_back(kv.second.first);
      m->cpl_coef.push_back(kv.second.second);
    }
  return SALVUS_OK;
}

}  // namespace salvus
