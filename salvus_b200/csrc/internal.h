// internal.h -- host-side structures of the B200 spectral-element library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/salvus_b200.h"

namespace salvus {

// Largest supported polynomial orders (reference limits: TensorQuad.h:69 for
// quads, Hexahedra.h:14-17 with order7_hex.c missing for hexes).
constexpr int kMaxQuadOrder = 10;
constexpr int kMaxHexOrder = 6;
// Default bound of every device-side wait, in SM clock cycles (~1 s).
constexpr long long kDefaultWaitLimit = 1ll << 31;

void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);
#define SALVUS_CUDA(call)                                                       \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess)                                                     \
      return ::salvus::fail(SALVUS_E_CUDA, "%s failed: %s (%s:%d)", #call,     \
                            cudaGetErrorString(e_), __FILE__, __LINE__);       \
  } while (0)

// Reference element of one shape.  Tensor shapes: the 1-D GLL basis of
// order N (xi, w, D[i*n+j] = l_j'(xi_i)).  Simplices (P3 only): the nodal
// tables of the mass-lumped 12-node triangle / 50-node tetrahedron.
struct Basis {
  int shape = 0, order = 0, n = 0, dim = 0, P = 0, nv = 0;
  bool simplex = false;
  std::vector<double> xi, w, D;  // tensor: 1-D GLL nodes, weights, derivative matrix
  std::vector<double> nodes;     // simplex: [P][3] reference coordinates
  std::vector<double> sw;        // simplex: [P] quadrature weights
  std::vector<double> SD;        // simplex: [dim][P][P], SD[(k*P + j)*P + q] = d phi_j/d xi_k (x_q)
  std::vector<double> C;         // simplex: [P][P] phi_i = sum_m g_m C[m*P + i]
};
int make_basis(int shape, int order, Basis *b);
int make_simplex_basis(int shape, int order, Basis *b);
void lagrange_1d(const Basis &b, double x, double *l, double *dl);
// Basis values phi[P] and reference gradients dphi[P][3] (may be null) at a
// reference point, for any shape.
void basis_at(const Basis &b, const double *ref, double *phi, double *dphi);
void simplex_basis_at(const Basis &b, const double *ref, double *phi, double *dphi);
// Reference coordinates and quadrature weight of element point p.
void point_ref(const Basis &b, int p, double *ref);
double point_weight(const Basis &b, int p);

// P1 geometry of one element: vertex signs of QuadP1.h:98-108 / HexP1.cpp,
// affine maps of TriP1.cpp:56-94 / TetP1.cpp:91-150.
void p1_jacobian(int shape, const double *vtx, const double *ref, double *detJ, double *invJ);
void p1_map(int shape, const double *vtx, const double *ref, double *x);
void p1_weights(int shape, const double *ref, double *w);  // vertex weights [nv]
int check_hull(int shape, const double *vtx, const double *x);  // 1 in, 0 out, <0 error
int inverse_map(int shape, const double *vtx, const double *x, double *ref);
inline int shape_dim(int shape) { return (shape == SALVUS_QUAD || shape == SALVUS_TRI) ? 2 : 3; }
inline int shape_nv(int shape) {
  return shape == SALVUS_QUAD ? 4 : shape == SALVUS_HEX ? 8 : shape == SALVUS_TRI ? 3 : 4;
}
inline bool is_simplex(int shape) { return shape == SALVUS_TRI || shape == SALVUS_TET; }
// field components per node and material parameters per element vertex
inline int physics_components(int physics) {
  return (physics == SALVUS_ELASTIC3D || physics == SALVUS_COUPLED2D) ? 3
                                                                      : (physics == SALVUS_ELASTIC2D ? 2 : 1);
}
// (flags: salvus_mesh_desc.reserved; SALVUS_MESH_ELASTIC_TI selects the six
// transversely isotropic elastic 3-D parameters)
inline int physics_params(int physics, int flags = 0) {
  return physics == SALVUS_ELASTIC3D ? ((flags & SALVUS_MESH_ELASTIC_TI) ? 6 : 3)
         : physics == SALVUS_ELASTIC2D ? 5 : physics == SALVUS_COUPLED2D ? 7 : 1;
}

struct DeviceBuffer {
  void *ptr = nullptr;
  size_t bytes = 0;
  int alloc(size_t n);
  void release();
  ~DeviceBuffer() { release(); }
  template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Number of float / double words per element-point record in the stiffness
// kernels (geometry + folded material [+ packed connectivity for FP32]);
// ti: transversely isotropic elastic material (five constants per point).
int record_words(int shape, int physics, int fp64, bool ti = false);

}  // namespace salvus

// Server support (server.cpp): non-blocking chunk collection.  Enqueues on
// the problem's stream, without synchronising, a copy of the seismogram ring
// ([shots][receivers][c][capacity] doubles, step s at column s % capacity)
// and of the status word into host buffers (page-locked for overlap);
// reports the ring's rows and capacity.  status_error turns a status word
// read that way into the error salvus_problem_status would return.
struct salvus_problem;
namespace salvus {
int enqueue_seis_copy(salvus_problem *p, double *ring, int *status);
void seis_ring_shape(const salvus_problem *p, int64_t *rows, int64_t *capacity);
int status_error(const salvus_problem *p, int status);
}  // namespace salvus

// stream of a problem group (server scheduling)
cudaStream_t salvus_group_stream_internal(const salvus_group *g);

struct salvus_mesh {
  int device = 0;
  int sm_count = 148;
  bool host_only = false;
  bool fp32_only = false;
  bool ti = false;  // elastic 3-D with transversely isotropic material (6 parameters)
  int shape = 0, order = 0, physics = 0, dim = 0, nv = 0, n = 0, P = 0, c = 0, npar = 0;
  int64_t E = 0, G = 0;
  salvus::Basis basis;
  std::vector<double> vtx;        // [E][nv][dim]
  std::vector<double> par;        // [npar][E][nv]
  std::vector<int32_t> conn;      // [E][P]
  std::vector<double> xyz;        // [G][dim]
  std::vector<int32_t> inc_off;   // [G+1]   node -> incident element points
  std::vector<int32_t> inc_idx;   // [E*P]   e*P + p, sorted by element
  std::vector<double> mi;         // [G] inverse mass (FP64, host copy)
  // meshes of fluid and solid quadrilaterals (SALVUS_COUPLED2D)
  int64_t n_fluid = 0;            // fluid elements; they come first in elist
  std::vector<int32_t> elist;     // [E] fluid elements ascending, then solid ones
  std::vector<int32_t> cls_k;     // [E] index of each element within its class
  std::vector<int32_t> cpl_pts;   // [n_cpl][2] coupled element point e*P + p, its node
  std::vector<double> cpl_coef;   // [n_cpl][2] coupling coefficients (cx, cy)
  int64_t n_cpl = 0, n_cpl_fluid = 0;  // fluid points first
  // device
  salvus::DeviceBuffer d_conn, d_inc_off, d_inc_idx, d_vtx, d_par;
  salvus::DeviceBuffer d_mi64, d_mi32;
  salvus::DeviceBuffer d_rec32, d_rec64;  // stiffness records per precision
  // elastic hexahedra that are all parallelepipeds: d_rec32 holds material
  // planes [NM][E*P], d_jac32 the per-element invJ [E][9]; d_gnodes lists
  // the nodes that are not interior to an element (fused steps' gather)
  bool affine = false;
  // parallelepiped hexahedron kernels: CTAs of 128 / (N+1)^2 elements (0) or
  // twice that (1), set by the hexahedron autotuner
  int hex_wide = 0;
  salvus::DeviceBuffer d_jac32, d_gnodes;
  std::vector<int32_t> gnodes;  // host copy of d_gnodes
  int64_t n_gnodes = 0;
  salvus::DeviceBuffer d_sd32, d_sd64;    // simplex derivative tables [dim][P][P]
  salvus::DeviceBuffer d_tc_tab;          // tetrahedra: tensor-core operand image (hi | lo)
  salvus::DeviceBuffer d_elist, d_cls_k, d_cpl_pts, d_cpl32, d_cpl64;
  int tet_kernel = 0;                     // FP32 tetrahedra: 0 tensor cores, 1 CUDA cores
  int tri_kernel = 1;                     // triangles: 0 tensor cores (FP32), 1 constant-table, 2 shared-table
  cudaStream_t stream = nullptr;
};

struct salvus_problem {
  salvus_mesh *mesh = nullptr;
  int device = 0;  // the mesh's device, kept for teardown after the mesh is gone
  int prec = SALVUS_FP32;
  int shots = 1;
  int c = 1;
  double dt = 0.0;
  bool dt_set = false;
  int64_t step = 0;
  size_t rsize = 4;  // sizeof(real)
  salvus::DeviceBuffer d_u, d_v, d_a, d_ap, d_r;
  salvus::DeviceBuffer d_step;   // int64 device step counter
  salvus::DeviceBuffer d_stage;  // FP64 staging for host field copies
  salvus::DeviceBuffer d_escr, d_epart;  // energy: -K u scratch, block partials
  // pinned host bounce buffers for field copies (two chunks, allocated on
  // the first large copy) and the events that guard their reuse
  void *h_pin[2] = {nullptr, nullptr};
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  salvus::DeviceBuffer d_err;    // int: device-side status word (bounded waits, finite check)
  long long wait_limit = salvus::kDefaultWaitLimit;  // bound of device waits, SM cycles
  int hold_waits = 0;  // test hook: tensor-core workers wait on a barrier nothing arrives on
  // homogeneous Dirichlet: element-local points (e*P + p) whose stiffness
  // rows are zeroed
  salvus::DeviceBuffer d_dir_pts;
  int64_t n_dir_pts = 0;
  // sources (host mirror + device)
  struct Src {
    salvus_source desc;
    int64_t elem;
    double ref[3];
    std::vector<double> wts;  // [P][c]
  };
  std::vector<Src> srcs;
  salvus::DeviceBuffer d_src_elem, d_src_par, d_src_wts;
  salvus::DeviceBuffer d_src_uelem;  // distinct source elements (fused hexahedron step)
  int n_src_uelem = 0;
  bool src_dirty = true;
  // receivers
  struct Rec {
    double xyz[3];
    int64_t elem;
    double ref[3];
    std::vector<double> l;  // [P]
  };
  std::vector<Rec> recs;
  salvus::DeviceBuffer d_rec_elem, d_rec_l, d_seis;
  int64_t seis_cap = 4096;
  bool rec_dirty = true;
  // shot batching (shots > 1): fields are [G][c][S_pad]; d_v holds the
  // half-step velocity w = v + dt/2 a_; sources grouped by shot
  int shots_pad = 1;
  salvus::DeviceBuffer d_shot_off;
  int tune_stiff = -1, tune_gather = -1;  // autotuner choices (indices)
  int hex_form = -1;  // hexahedron step form: 0 plain, 1 fused interior update (-1 untuned)
  // graphs
  cudaGraphExec_t graph_exec = nullptr;
  int graph_steps = 0;
  int64_t graph_launches = 0;  // kernel launches in one replay of graph_exec
  // the graph of the last remainder length (a run's steps after its whole
  // 32-step replays, when at least 8)
  cudaGraphExec_t tail_exec = nullptr;
  int tail_steps = 0;
  int64_t tail_launches = 0;
  cudaStream_t stream = nullptr;
  // receivers of the fused step on a second stream inside salvus_run
  // (overlapped with the next step's stiffness launch): the stream, the
  // fork / join events, whether a launch is still to be joined, and whether
  // the current call allows the overlap
  cudaStream_t rec_stream = nullptr;
  cudaEvent_t ev_updated = nullptr, ev_recorded = nullptr;
  bool rec_pending = false, rec_overlap = false;
  // profiling
  bool profiling = false;
  struct Ev {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<Ev> events;
  std::vector<double> prof_ms;
  std::vector<int64_t> prof_n;
};
