// salvus.hpp -- header-only C++ plugin facade over the C ABI (salvus_b200.h)
// that keeps the reference's element / physics / problem vocabulary:
//
//   reference (src/cxx)                          here
//   Scalar<TensorQuad<QuadP1>>                   Quad<Acoustic>
//   Scalar<Hexahedra<HexP1>>                     Hexahedron<Acoustic>
//   Elastic3D<Hexahedra<HexP1>>                  Hexahedron<Elastic3D>
//   ScalarTri<Scalar<Triangle<TriP1>>>           Triangle<Acoustic>
//   Scalar<Tetrahedra<TetP1>>                    Tetrahedron<Acoustic>
//   (no reference element)                       Tetrahedron<Elastic3D>
//   Elastic2D<TensorQuad<QuadP1>>                Quad<Elastic2D>
//   Scalar / Elastic2D quads of one mesh with    Quad<FluidSolid2D>
//     ElasticToAcoustic2D / AcousticToElastic2D
//   Element::Factory("quad"|"hex"|"tri"|"tet", {"fluid"|"2delastic"|"3delastic"})
//                                                (Element.cpp:117-304)
//                                                makeProblem(shape, physics, ...)
//   Problem / Order2Newmark                      Problem<Element> (= Order2Newmark<Element>)
//     assembleIntoGlobalDof (Problem.cpp:143-214)    assembleIntoGlobalDof()
//     applyInverseMassMatrix (Order2Newmark.cpp:68-83) applyInverseMassMatrix()
//     takeTimeStep (Order2Newmark.cpp:85-114)    takeTimeStep()
//   Ricker (Ricker.cpp:9-33), Receiver (Receiver.cpp:27-42)
//
// Errors throw std::runtime_error with the library's message, as the
// reference does (caught in Main.cpp:70-74).
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../salvus_b200.h"

namespace salvus {

inline void check(int rc) {
  if (rc != SALVUS_OK) throw std::runtime_error(salvus_last_error());
}

// ---- physics tags (Physics mixins of the reference) ----
struct Acoustic {  // Scalar<...>, Scalar.cpp
  static constexpr int physics = SALVUS_ACOUSTIC;
  static constexpr int components = 1;
  static constexpr const char *name = "fluid";
};
struct Elastic3D {  // Elastic3D<...>, Elastic3D.cpp
  static constexpr int physics = SALVUS_ELASTIC3D;
  static constexpr int components = 3;
  static constexpr const char *name = "3delastic";
};
struct Elastic2D {  // Elastic2D<...>, Elastic2D.cpp
  static constexpr int physics = SALVUS_ELASTIC2D;
  static constexpr int components = 2;
  static constexpr const char *name = "2delastic";
};
// fluid and solid quadrilaterals in one mesh, element class from the FLUID
// parameter, coupled through ElasticToAcoustic2D / AcousticToElastic2D;
// fields [u, ux, uy]
struct FluidSolid2D {
  static constexpr int physics = SALVUS_COUPLED2D;
  static constexpr int components = 3;
  static constexpr const char *name = "fluid,2delastic";
};

// ---- element shapes (TensorQuad<QuadP1>, Hexahedra<HexP1>) ----
template <class Physics>
struct Quad {
  static_assert(Physics::physics == SALVUS_ACOUSTIC || Physics::physics == SALVUS_ELASTIC2D ||
                    Physics::physics == SALVUS_COUPLED2D,
                "quads carry acoustic, 2-D elastic or coupled fluid-solid physics");
  using physics_type = Physics;
  static constexpr int shape = SALVUS_QUAD;
  static constexpr int dim = 2;
  static constexpr int vertices = 4;
  static constexpr int max_order = 10;  // TensorQuad.h:69
};
template <class Physics>
struct Hexahedron {
  using physics_type = Physics;
  static constexpr int shape = SALVUS_HEX;
  static constexpr int dim = 3;
  static constexpr int vertices = 8;
  static constexpr int max_order = 6;  // Hexahedra.h:14-17 (order7_hex.c missing)
};

// ---- P3 simplices (Triangle<TriP1>, Tetrahedra<TetP1>; order 3 only) ----
template <class Physics>
struct Triangle {
  static_assert(Physics::physics == SALVUS_ACOUSTIC,
                "triangles carry acoustic physics (ScalarTri, Element.cpp:202-227)");
  using physics_type = Physics;
  static constexpr int shape = SALVUS_TRI;
  static constexpr int dim = 2;
  static constexpr int vertices = 3;
  static constexpr int max_order = 3;  // Triangle.cpp:24-39
};
template <class Physics>
struct Tetrahedron {
  using physics_type = Physics;
  static constexpr int shape = SALVUS_TET;
  static constexpr int dim = 3;
  static constexpr int vertices = 4;
  static constexpr int max_order = 3;  // Tetrahedra.cpp:66-84
};

// ---- sources and receivers ----
struct Ricker {
  std::array<double, 3> location{0, 0, 0};
  double center_freq = 1.0, time_delay = 1.0, amplitude = 1.0;
  std::vector<double> direction{1.0};      // force direction (c components)
  std::vector<double> moment_tensor;       // Mxx Myy Mzz Myz Mxz Mxy, or Mxx Myy Mxy in 2-D
  int shot = 0;
  salvus_source desc() const {
    salvus_source s{};
    for (int a = 0; a < 3; ++a) s.location[a] = location[a];
    s.center_freq = center_freq;
    s.time_delay = time_delay;
    s.amplitude = amplitude;
    s.shot = shot;
    if (!moment_tensor.empty()) {
      if (moment_tensor.size() != 6 && moment_tensor.size() != 3)
        throw std::runtime_error("moment tensor needs 6 (3-D) or 3 (2-D) components");
      s.kind = SALVUS_SOURCE_MOMENT_TENSOR;
      for (size_t a = 0; a < moment_tensor.size(); ++a) s.comp[a] = moment_tensor[a];
    } else {
      s.kind = SALVUS_SOURCE_FORCE;
      for (size_t a = 0; a < direction.size() && a < 6; ++a) s.comp[a] = direction[a];
    }
    return s;
  }
};

struct Receiver {
  std::array<double, 3> location{0, 0, 0};
  std::string name;
};

// ---- mesh: DMPlex mesh + Exodus model + per-element precomputation ----
template <class Element>
class Mesh {
 public:
  // vertices [n_vertices][dim]; cells [n_elements][nv] (PETSc right-hand
  // order for quads / hexes, TriP1 / TetP1 order for simplices); params per
  // element vertex: acoustic VP [E][nv], elastic RHO, VP, VS [3][E][nv] or
  // the reference's six RHO, VPV, VPH, VSV, VSH, ETA [6][E][nv]
  // (Elastic3D.cpp:33-54; transversely isotropic), 2-D elastic RHO, C11,
  // C13, C33, C55 [5][E][4], fluid-solid FLUID, VP, RHO, C11, C13, C33, C55
  // [7][E][4].
  Mesh(int order, const std::vector<double> &vertices, const std::vector<int64_t> &cells,
       const std::vector<double> &params, int device = 0) {
    if (order < 1 || order > Element::max_order)
      throw std::runtime_error("Polynomial order " + std::to_string(order) + " not supported");
    salvus_mesh_desc d{};
    d.shape = Element::shape;
    d.order = order;
    d.physics = Element::physics_type::physics;
    d.n_vertices = (int64_t)(vertices.size() / Element::dim);
    d.vertices = vertices.data();
    d.n_elements = (int64_t)(cells.size() / Element::vertices);
    d.cells = cells.data();
    d.params = params.data();
    if (d.physics == SALVUS_ELASTIC3D &&
        params.size() == (size_t)(6 * d.n_elements * Element::vertices))
      d.reserved |= SALVUS_MESH_ELASTIC_TI;
    salvus_mesh *m = nullptr;
    check(salvus_mesh_create(&d, device, &m));
    mesh_.reset(m);
    int32_t c = 0, P = 0;
    check(salvus_mesh_info(m, &nodes_, &c, &P));
    elements_ = d.n_elements;
    points_ = P;
  }
  int64_t numNodes() const { return nodes_; }
  int64_t numElements() const { return elements_; }
  int pointsPerElement() const { return points_; }
  std::vector<double> nodeCoords() const {
    std::vector<double> x((size_t)nodes_ * Element::dim);
    check(salvus_mesh_node_coords(mesh_.get(), x.data()));
    return x;
  }
  // nodes of the outer boundary (for HomogeneousDirichlet on every side)
  std::vector<int64_t> boundaryNodes() const {
    int64_t n = 0;
    check(salvus_mesh_boundary_nodes(mesh_.get(), &n, nullptr));
    std::vector<int64_t> out((size_t)n);
    if (n) check(salvus_mesh_boundary_nodes(mesh_.get(), &n, out.data()));
    return out;
  }
  double criticalDt(int iterations = 200) const {
    double lam = 0;
    check(salvus_mesh_max_eigenvalue(mesh_.get(), iterations, 1, &lam));
    return 2.0 / std::sqrt(lam);
  }
  salvus_mesh *handle() const { return mesh_.get(); }

 private:
  struct Del {
    void operator()(salvus_mesh *m) const { salvus_mesh_destroy(m); }
  };
  std::unique_ptr<salvus_mesh, Del> mesh_;
  int64_t nodes_ = 0, elements_ = 0;
  int points_ = 0;
};

// ---- runtime-polymorphic problem (what Element::Factory + Problem::Factory
// hand to the time loop) ----
class ProblemBase {
 public:
  virtual ~ProblemBase() = default;
  virtual void addSource(const Ricker &r) = 0;
  virtual void addReceiver(const Receiver &r) = 0;
  virtual void assembleIntoGlobalDof() = 0;
  virtual void applyInverseMassMatrix() = 0;
  virtual void takeTimeStep() = 0;
  virtual void step() = 0;
  virtual void run(int64_t steps, bool graph = true) = 0;
  virtual int64_t stepIndex() const = 0;
  virtual std::vector<double> seismograms() = 0;
  virtual std::vector<double> getField(const std::string &name) = 0;
  virtual void setField(const std::string &name, const std::vector<double> &v) = 0;
  // HomogeneousDirichlet (HomogeneousDirichlet.cpp:14-78) on these nodes
  virtual void setDirichlet(const std::vector<int64_t> &nodes) = 0;
  // {kinetic, strain} energy of the current state (FP64 compensated sums)
  virtual std::array<double, 2> energy() = 0;
};

// Order2Newmark over one element type (Order2Newmark.h:6-26).
template <class Element>
class Problem : public ProblemBase {
 public:
  Problem(const Mesh<Element> &mesh, double dt, int precision = SALVUS_FP32) : mesh_(&mesh) {
    salvus_problem *p = nullptr;
    check(salvus_problem_create(mesh.handle(), precision, 1, &p));
    p_.reset(p);
    check(salvus_problem_set_dt(p, dt));
  }
  void addSource(const Ricker &r) override {
    salvus_source s = r.desc();
    check(salvus_problem_add_source(p_.get(), &s));
  }
  void addReceiver(const Receiver &r) override {
    check(salvus_problem_add_receiver(p_.get(), r.location.data()));
    ++receivers_;
  }
  std::array<double, 2> energy() override {
    std::array<double, 2> e{0, 0};
    check(salvus_problem_energy(p_.get(), &e[0], &e[1]));
    return e;
  }
  void setDirichlet(const std::vector<int64_t> &nodes) override {
    check(salvus_problem_set_dirichlet(p_.get(), (int64_t)nodes.size(), nodes.data()));
  }
  void assembleIntoGlobalDof() override { check(salvus_assemble(p_.get())); }
  void applyInverseMassMatrix() override { check(salvus_apply_inverse_mass(p_.get())); }
  void takeTimeStep() override { check(salvus_take_time_step(p_.get())); }
  void step() override { check(salvus_step(p_.get())); }
  void run(int64_t steps, bool graph = true) override {
    check(salvus_run(p_.get(), steps, graph ? SALVUS_RUN_GRAPH : SALVUS_RUN_PLAIN));
  }
  int64_t stepIndex() const override { return salvus_problem_step_index(p_.get()); }
  // [receivers][c][steps] of u sampled after every step
  std::vector<double> seismograms() override {
    const int64_t n = stepIndex();
    std::vector<double> out((size_t)receivers_ * Element::physics_type::components * n);
    if (receivers_ && n) check(salvus_get_seismograms(p_.get(), 0, n, out.data()));
    return out;
  }
  std::vector<double> getField(const std::string &name) override {
    std::vector<double> v((size_t)mesh_->numNodes() * Element::physics_type::components);
    check(salvus_problem_get_field(p_.get(), field_id(name), 0, v.data()));
    return v;
  }
  void setField(const std::string &name, const std::vector<double> &v) override {
    if (v.size() != (size_t)mesh_->numNodes() * Element::physics_type::components)
      throw std::runtime_error("field " + name + " has the wrong size");
    check(salvus_problem_set_field(p_.get(), field_id(name), 0, v.data()));
  }

 private:
  static int field_id(const std::string &n) {
    if (n == "u" || n == "ux") return SALVUS_FIELD_U;
    if (n == "v" || n == "vx") return SALVUS_FIELD_V;
    if (n == "a" || n == "ax") return SALVUS_FIELD_A;
    if (n == "a_" || n == "ax_") return SALVUS_FIELD_A_PREV;
    throw std::runtime_error("You are attempting to use field " + n + " which is not registered.");
  }
  struct Del {
    void operator()(salvus_problem *p) const { salvus_problem_destroy(p); }
  };
  const Mesh<Element> *mesh_;
  std::unique_ptr<salvus_problem, Del> p_;
  int receivers_ = 0;
};

template <class Element>
using Order2Newmark = Problem<Element>;

// String factory in the spirit of Element::Factory (Element.cpp:26-304):
// shape "quad" | "hex" | "tri" | "tet", physics "fluid" | "2delastic" |
// "3delastic" | "fluid,2delastic" (quads of both kinds in one mesh).
struct Simulation {
  std::shared_ptr<void> mesh;
  std::unique_ptr<ProblemBase> problem;
};

namespace detail {
template <class Element>
Simulation make(int order, const std::vector<double> &v, const std::vector<int64_t> &c,
                const std::vector<double> &p, double dt, int precision, int device) {
  auto mesh = std::make_shared<Mesh<Element>>(order, v, c, p, device);
  Simulation s;
  s.problem.reset(new Problem<Element>(*mesh, dt, precision));
  s.mesh = mesh;
  return s;
}
}  // namespace detail

inline Simulation makeProblem(const std::string &shape, const std::string &physics, int order,
                              const std::vector<double> &vertices,
                              const std::vector<int64_t> &cells,
                              const std::vector<double> &params, double dt,
                              int precision = SALVUS_FP32, int device = 0) {
  if (shape == "quad" && physics == "fluid")
    return detail::make<Quad<Acoustic>>(order, vertices, cells, params, dt, precision, device);
  if (shape == "quad" && physics == "2delastic")
    return detail::make<Quad<Elastic2D>>(order, vertices, cells, params, dt, precision, device);
  if (shape == "quad" && physics == "fluid,2delastic")
    return detail::make<Quad<FluidSolid2D>>(order, vertices, cells, params, dt, precision, device);
  if (shape == "hex" && physics == "fluid")
    return detail::make<Hexahedron<Acoustic>>(order, vertices, cells, params, dt, precision, device);
  if (shape == "hex" && physics == "3delastic")
    return detail::make<Hexahedron<Elastic3D>>(order, vertices, cells, params, dt, precision, device);
  if (shape == "tri" && physics == "fluid")
    return detail::make<Triangle<Acoustic>>(order, vertices, cells, params, dt, precision, device);
  if (shape == "tet" && physics == "fluid")
    return detail::make<Tetrahedron<Acoustic>>(order, vertices, cells, params, dt, precision, device);
  if (shape == "tet" && physics == "3delastic")
    return detail::make<Tetrahedron<Elastic3D>>(order, vertices, cells, params, dt, precision, device);
  throw std::runtime_error("Element type " + shape + " with physics " + physics +
                           " not supported on this path");
}

}  // namespace salvus
