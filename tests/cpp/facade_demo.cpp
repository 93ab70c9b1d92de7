// Drives the C++ plugin facade the way the reference's Main.cpp:45-66 drives
// its Problem: assembleIntoGlobalDof -> applyInverseMassMatrix ->
// takeTimeStep, for Quad<Acoustic>, Hexahedron<Elastic3D>,
// Tetrahedron<Elastic3D> and Quad<FluidSolid2D> (with Dirichlet sides), and prints
// the seismograms as JSON for comparison with the Python path.
#include <cstdio>
#include <vector>

#include "salvus/salvus.hpp"

using namespace salvus;

static void quad_mesh(int n, double L, std::vector<double> &v, std::vector<int64_t> &c) {
  for (int j = 0; j <= n; ++j)
    for (int i = 0; i <= n; ++i) { v.push_back(L * i / n); v.push_back(L * j / n); }
  auto id = [&](int i, int j) { return (int64_t)j * (n + 1) + i; };
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      c.push_back(id(i, j)); c.push_back(id(i + 1, j)); c.push_back(id(i + 1, j + 1)); c.push_back(id(i, j + 1));
    }
}

static void hex_mesh(int n, double L, std::vector<double> &v, std::vector<int64_t> &c) {
  for (int k = 0; k <= n; ++k)
    for (int j = 0; j <= n; ++j)
      for (int i = 0; i <= n; ++i) { v.push_back(L * i / n); v.push_back(L * j / n); v.push_back(L * k / n); }
  auto id = [&](int i, int j, int k) { return ((int64_t)k * (n + 1) + j) * (n + 1) + i; };
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        int64_t q[8] = {id(i, j, k), id(i, j + 1, k), id(i + 1, j + 1, k), id(i + 1, j, k),
                        id(i, j, k + 1), id(i + 1, j, k + 1), id(i + 1, j + 1, k + 1), id(i, j + 1, k + 1)};
        c.insert(c.end(), q, q + 8);
      }
}

// Lattice of n^3 cubes, each split into 6 tetrahedra along its main diagonal
// (the construction of salvus_b200.meshgen.kuhn_tet with no jitter),
// positively oriented in TetP1 vertex order.
static void tet_mesh(int n, double L, std::vector<double> &v, std::vector<int64_t> &c) {
  for (int k = 0; k <= n; ++k)
    for (int j = 0; j <= n; ++j)
      for (int i = 0; i <= n; ++i) { v.push_back(L * i / n); v.push_back(L * j / n); v.push_back(L * k / n); }
  const int kuhn[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7}, {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        for (auto &t : kuhn) {
          int64_t q[4];
          for (int a = 0; a < 4; ++a) {
            const int cc = t[a];
            q[a] = ((int64_t)(k + (cc >> 2)) * (n + 1) + (j + ((cc >> 1) & 1))) * (n + 1) + (i + (cc & 1));
          }
          const double *p0 = &v[3 * q[0]], *p1 = &v[3 * q[1]], *p2 = &v[3 * q[2]], *p3 = &v[3 * q[3]];
          double a[3], b[3], d[3];
          for (int m = 0; m < 3; ++m) { a[m] = p2[m] - p0[m]; b[m] = p1[m] - p0[m]; d[m] = p3[m] - p0[m]; }
          const double det = a[0] * (b[1] * d[2] - b[2] * d[1]) - a[1] * (b[0] * d[2] - b[2] * d[0]) +
                             a[2] * (b[0] * d[1] - b[1] * d[0]);
          if (det < 0) std::swap(q[1], q[2]);
          c.insert(c.end(), q, q + 4);
        }
}

static void print(const char *name, const std::vector<double> &s, bool last) {
  std::printf("\"%s\": [", name);
  for (size_t i = 0; i < s.size(); ++i) std::printf("%s%.17g", i ? "," : "", s[i]);
  std::printf("]%s\n", last ? "" : ",");
}

int main() {
  std::printf("{\n");
  {  // Quad<Acoustic>, literal three-call loop
    std::vector<double> v; std::vector<int64_t> c;
    quad_mesh(8, 1e4, v, c);
    std::vector<double> vp(c.size(), 4000.0);
    Mesh<Quad<Acoustic>> mesh(4, v, c, vp);
    Order2Newmark<Quad<Acoustic>> problem(mesh, 2e-3);
    Ricker src; src.location = {5123.0, 4987.0, 0.0}; src.center_freq = 4.0; src.time_delay = 0.3;
    problem.addSource(src);
    Receiver r1; r1.location = {2000.0, 3000.0, 0.0}; problem.addReceiver(r1);
    Receiver r2; r2.location = {7000.0, 6100.0, 0.0}; problem.addReceiver(r2);
    for (int n = 0; n < 150; ++n) {
      problem.assembleIntoGlobalDof();
      problem.applyInverseMassMatrix();
      problem.takeTimeStep();
    }
    print("quad_acoustic", problem.seismograms(), false);
  }
  {  // Hexahedron<Elastic3D> through the string factory, graph replay
    std::vector<double> v; std::vector<int64_t> c;
    hex_mesh(3, 600.0, v, c);
    const size_t E = c.size() / 8;
    std::vector<double> par;
    for (double val : {2700.0, 6000.0, 3464.0}) par.insert(par.end(), E * 8, val);
    Simulation sim = makeProblem("hex", "3delastic", 4, v, c, par, 1e-3);
    Ricker src; src.location = {311.0, 287.0, 305.0}; src.center_freq = 8.0; src.time_delay = 0.15;
    src.amplitude = 1e10; src.moment_tensor = {1.0, -0.5, 0.3, 0.2, 0.1, -0.4};
    sim.problem->addSource(src);
    Receiver r; r.location = {100.0, 500.0, 600.0}; sim.problem->addReceiver(r);
    sim.problem->run(120, true);
    print("hex_elastic", sim.problem->seismograms(), false);
  }
  {  // Tetrahedron<Elastic3D> (P3, tensor-core stiffness) through the factory
    std::vector<double> v; std::vector<int64_t> c;
    tet_mesh(2, 600.0, v, c);
    const size_t E = c.size() / 4;
    std::vector<double> par;
    for (double val : {2700.0, 6000.0, 3464.0}) par.insert(par.end(), E * 4, val);
    Simulation sim = makeProblem("tet", "3delastic", 3, v, c, par, 5e-4);
    Ricker src; src.location = {311.0, 287.0, 305.0}; src.center_freq = 8.0; src.time_delay = 0.15;
    src.amplitude = 1e10; src.moment_tensor = {1.0, -0.5, 0.3, 0.2, 0.1, -0.4};
    sim.problem->addSource(src);
    Receiver r; r.location = {100.0, 500.0, 600.0}; sim.problem->addReceiver(r);
    sim.problem->run(120, true);
    print("tet_elastic", sim.problem->seismograms(), false);
  }
  {  // fluid over solid quads (Quad<FluidSolid2D>) with Dirichlet sides
    std::vector<double> v; std::vector<int64_t> c;
    quad_mesh(8, 1e4, v, c);
    const size_t E = c.size() / 4;
    std::vector<double> par(7 * E * 4);
    for (size_t e = 0; e < E; ++e) {
      const bool fluid = e / 8 >= 5;  // top three element rows
      const double vals[7] = {fluid ? 1.0 : 0.0, 1500.0, fluid ? 1000.0 : 2600.0,
                              4.16e10, 1.408e10, 4.16e10, 1.376e10};
      for (int k = 0; k < 7; ++k)
        for (int a = 0; a < 4; ++a) par[(k * E + e) * 4 + a] = vals[k];
    }
    Mesh<Quad<FluidSolid2D>> mesh(4, v, c, par);
    Order2Newmark<Quad<FluidSolid2D>> problem(mesh, 4e-3);
    problem.setDirichlet(mesh.boundaryNodes());
    Ricker src; src.location = {5123.0, 3987.0, 0.0}; src.center_freq = 4.0; src.time_delay = 0.3;
    src.amplitude = 1e10; src.moment_tensor = {1.0, -0.5, 0.3};
    problem.addSource(src);
    Receiver r1; r1.location = {4000.0, 7500.0, 0.0}; problem.addReceiver(r1);
    Receiver r2; r2.location = {6000.0, 2500.0, 0.0}; problem.addReceiver(r2);
    problem.run(200, true);
    print("fluid_solid", problem.seismograms(), true);
  }
  std::printf("}\n");
  return 0;
}
