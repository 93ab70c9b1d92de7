// abi.cu -- extern "C" entry points (include/salvus_b200.h): mesh flattening,
// device residency, and the per-step launch sequence
//   stiffness (element-local residual) -> sources -> node gather + inverse
//   mass + Newmark -> receivers.
#include <cuda_runtime.h>

#include <unistd.h>

#include <atomic>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#include "internal.h"
#include "kernels_setup.cuh"
#include "kernels_stiffness.cuh"
#include "kernels_step.cuh"
#include "kernels_hex_v2.cuh"
#include "kernels_hex_affine.cuh"
#include "kernels_batch.cuh"
#include "kernels_simplex.cuh"
#include "kernels_simplex_tc.cuh"
#include "kernels_tri_tc.cuh"
#include "kernels_elastic2d.cuh"
#include "kernels_quad_col.cuh"
#include "kernels_group.cuh"
#include <algorithm>
#include <cstdlib>
#include <type_traits>

namespace salvus {
const char *last_error();
int flatten_mesh(salvus_mesh *m, const int64_t *cells, int64_t n_vertices);
int locate_point(const salvus_mesh *m, const double *x, int64_t *elem, double *ref);
int boundary_nodes(const salvus_mesh *m, std::vector<int64_t> &out);
int setup_coupled(salvus_mesh *m, const int64_t *cells);

static std::atomic<int64_t> g_launches{0};

enum Kind { K_STIFF = 0, K_SRC, K_UPDATE, K_REC, K_GATHER, K_MINV, K_NEWMARK, K_GRAPH, K_NKINDS };
static const char *kKindNames[K_NKINDS] = {"stiffness", "source",        "gather_update",
                                           "receivers", "gather",        "inverse_mass",
                                           "newmark",   "graph_replay"};

struct ProfScope {
  salvus_problem *p;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(salvus_problem *p_, int k) : p(p_), kind(k) {
    if (p && p->profiling) {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, p->stream);
    }
  }
  ~ProfScope() {
    if (a) {
      cudaEventRecord(b, p->stream);
      p->events.push_back({kind, a, b});
    }
  }
};

static inline unsigned blocks_for(int64_t n, int threads) {
  return (unsigned)((n + threads - 1) / threads);
}

template <typename real>
static DMatrix<real> dmatrix(const Basis &b) {
  DMatrix<real> d{};
  for (int i = 0; i < b.n * b.n; ++i) d.d[i] = (real)b.D[i];
  return d;
}

static int check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SALVUS_E_CUDA, "%s launch failed: %s", what, cudaGetErrorString(e));
  return SALVUS_OK;
}

// Calls fn(std::integral_constant<int, C>) for the field's component count
// (1 acoustic, 2 elastic 2-D, 3 elastic 3-D).
template <typename Fn>
static int by_components(int c, Fn &&fn) {
  switch (c) {
    case 1: return fn(std::integral_constant<int, 1>{});
    case 2: return fn(std::integral_constant<int, 2>{});
    case 3: return fn(std::integral_constant<int, 3>{});
  }
  return fail(SALVUS_E_UNSUPPORTED, "no kernels for %d field components", c);
}

// ---------------------------------------------------------------------------
// stiffness dispatch
template <int DIM, int N, typename real>
static int launch_acoustic(const salvus_mesh *m, const real *rec, const real *u, real *r,
                           cudaStream_t st) {
  using S = AcousticShape<DIM, N>;
  const unsigned grid = blocks_for(m->E, S::EPB);
  acoustic_stiffness_kernel<DIM, N, real><<<grid, S::THREADS, 0, st>>>(
      m->E, rec, m->d_conn.as<int32_t>(), u, r, dmatrix<real>(m->basis));
  g_launches++;
  return check_launch("acoustic stiffness");
}

// FP32 elastic hexahedra: the column-threaded kernel with 32-bit shared
// planes and 128-thread CTAs (whole warps: 5 order-4 elements, 6 CTAs per
// SM) by default; SALVUS_HEX_KERNEL=classic selects the register / shared-
// memory kernel that also serves FP64 (read at every launch).
static bool hex_classic() {
  const char *s = std::getenv("SALVUS_HEX_KERNEL");
  return s && std::strcmp(s, "classic") == 0;
}

template <int N, bool TI>
static int launch_elastic_v2(const salvus_mesh *m, const float *rec, const float *u, float *r,
                             cudaStream_t st) {
  constexpr int n2 = (N + 1) * (N + 1), EPB = 128 / n2 > 0 ? 128 / n2 : 1;
  using T = ElasticV2Shape<N, EPB, TI>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(elastic_hex_stiffness_v2_kernel<N, EPB, TI>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
    attr = true;
  }
  elastic_hex_stiffness_v2_kernel<N, EPB, TI><<<blocks_for(m->E, EPB), T::THREADS, T::SMEM, st>>>(
      m->E, rec, u, r, dmatrix<float>(m->basis));
  g_launches++;
  return check_launch("elastic stiffness");
}

template <int N, typename real, bool TI>
static int launch_elastic_classic(const salvus_mesh *m, const real *rec, const real *u, real *r,
                                  cudaStream_t st) {
  using S = ElasticShape<N, real>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(elastic_hex_stiffness_kernel<N, real, TI>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
    attr_set = true;
  }
  elastic_hex_stiffness_kernel<N, real, TI><<<blocks_for(m->E, S::EPB), S::THREADS, S::SMEM, st>>>(
      m->E, rec, m->d_conn.as<int32_t>(), u, r, dmatrix<real>(m->basis));
  g_launches++;
  return check_launch("elastic stiffness");
}

// Parallelepiped meshes (m->affine): per-element inverse Jacobian, material
// planes; kFuse also advances the interior nodes (kernels_hex_affine.cuh).
// CTAs hold EPB elements: 128 / (N+1)^2 or, when the hexahedron autotuner
// found it faster on this mesh (m->hex_wide), twice as many.
template <int N, int EPB, bool TI, bool kFuse>
static int launch_elastic_affine_epb(const salvus_mesh *m, const float *mat, float *u, float *r,
                                     cudaStream_t st, const HexInteriorUpdate &iu) {
  using T = HexAffineShape<N, EPB, TI>;
  auto kern = kFuse ? elastic_hex_affine_fused_kernel<N, EPB, TI>
                    : elastic_hex_affine_kernel<N, EPB, TI>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
    attr = true;
  }
  kern<<<blocks_for(m->E, EPB), T::THREADS, T::SMEM, st>>>(
      m->E, m->d_jac32.as<float>(), mat, m->d_conn.as<int32_t>(), u, r, dmatrix<float>(m->basis),
      iu);
  g_launches++;
  return check_launch(kFuse ? "elastic stiffness (fused interior)" : "elastic stiffness");
}
template <int N, bool TI, bool kFuse>
static int launch_elastic_affine(const salvus_mesh *m, const float *mat, float *u, float *r,
                                 cudaStream_t st, const HexInteriorUpdate &iu) {
  constexpr int n2 = (N + 1) * (N + 1), EPB = 128 / n2 > 0 ? 128 / n2 : 1;
  return m->hex_wide ? launch_elastic_affine_epb<N, 2 * EPB, TI, kFuse>(m, mat, u, r, st, iu)
                     : launch_elastic_affine_epb<N, EPB, TI, kFuse>(m, mat, u, r, st, iu);
}

template <int N, typename real>
static int launch_elastic(const salvus_mesh *m, const real *rec, const real *u, real *r,
                          cudaStream_t st) {
  if constexpr (std::is_same<real, float>::value) {
    if (m->affine) {
      HexInteriorUpdate none{};
      return m->ti ? launch_elastic_affine<N, true, false>(m, rec, const_cast<float *>(u), r, st, none)
                   : launch_elastic_affine<N, false, false>(m, rec, const_cast<float *>(u), r, st, none);
    }
    if (!hex_classic())
      return m->ti ? launch_elastic_v2<N, true>(m, rec, u, r, st)
                   : launch_elastic_v2<N, false>(m, rec, u, r, st);
  }
  return m->ti ? launch_elastic_classic<N, real, true>(m, rec, u, r, st)
               : launch_elastic_classic<N, real, false>(m, rec, u, r, st);
}

// Quadrilateral stiffness: column-threaded kernels (kernels_quad_col.cuh) by
// default; SALVUS_QUAD_KERNEL=point selects the point-threaded ones (read at
// every launch).
static bool quad_point_kernels() {
  const char *v = std::getenv("SALVUS_QUAD_KERNEL");
  return v && std::strcmp(v, "point") == 0;
}
template <int N, typename real>
static int acoustic2(const salvus_mesh *m, const real *rec, const real *u, real *r, cudaStream_t s) {
  // (FP64 elastic columns of order 9-10 exceed the register file: point kernels)
  if (!quad_point_kernels() && (sizeof(real) == 4 || N <= 8)) {
    constexpr int EPB = quad_col_epb<N>();
    using S = QuadColShape<N, EPB>;
    const DMatrix<real> D = dmatrix<real>(m->basis);
    const int32_t *cn = m->d_conn.as<int32_t>();
    if (m->physics == SALVUS_ACOUSTIC) {
      acoustic_quad_col_kernel<N, EPB, real><<<blocks_for(m->E, EPB), S::THREADS, 0, s>>>(
          m->E, rec, cn, u, r, D);
      g_launches++;
      return check_launch("acoustic quad stiffness");
    }
    if (m->physics == SALVUS_ELASTIC2D) {
      elastic2d_col_kernel<N, EPB, real, 2, 0><<<blocks_for(m->E, EPB), S::THREADS, 0, s>>>(
          m->E, nullptr, rec, cn, u, r, D);
      g_launches++;
      return check_launch("elastic 2-D stiffness");
    }
    // fluid elements (u) then solid elements (ux, uy), class-compact records
    const int64_t Ef = m->n_fluid, Es = m->E - m->n_fluid;
    const int32_t *el = m->d_elist.as<int32_t>();
    if (Ef > 0) {
      acoustic_quad_col_list_kernel<N, EPB, real><<<blocks_for(Ef, EPB), S::THREADS, 0, s>>>(
          Ef, el, rec, cn, u, r, D);
      g_launches++;
      int rc = check_launch("fluid stiffness");
      if (rc) return rc;
    }
    if (Es > 0) {
      const real *rs = rec + Ef * m->P * (sizeof(real) == 4 ? 4 : 3);
      elastic2d_col_kernel<N, EPB, real, 3, 1><<<blocks_for(Es, EPB), S::THREADS, 0, s>>>(
          Es, el + Ef, rs, cn, u, r, D);
      g_launches++;
      return check_launch("solid stiffness");
    }
    return SALVUS_OK;
  }
  if (m->physics == SALVUS_COUPLED2D) {
    // fluid elements (u) then solid elements (ux, uy), class-compact records
    const int64_t Ef = m->n_fluid, Es = m->E - m->n_fluid;
    const int32_t *el = m->d_elist.as<int32_t>();
    if (Ef > 0) {
      using S = AcousticShape<2, N>;
      acoustic_list_kernel<N, real><<<blocks_for(Ef, S::EPB), S::THREADS, 0, s>>>(
          Ef, el, rec, m->d_conn.as<int32_t>(), u, r, dmatrix<real>(m->basis));
      g_launches++;
      int rc = check_launch("fluid stiffness");
      if (rc) return rc;
    }
    if (Es > 0) {
      using S = Elastic2DShape<N>;
      const real *rs = rec + Ef * m->P * (sizeof(real) == 4 ? 4 : 3);
      elastic2d_stiffness_kernel<N, real, 3, 1><<<blocks_for(Es, S::EPB), S::THREADS, 0, s>>>(
          Es, el + Ef, rs, m->d_conn.as<int32_t>(), u, r, dmatrix<real>(m->basis));
      g_launches++;
      return check_launch("solid stiffness");
    }
    return SALVUS_OK;
  }
  if (m->physics == SALVUS_ELASTIC2D) {
    // CTA shape: SALVUS_E2D_EPB elements per CTA (read at every launch; 0 or
    // unset: as many as fit 256 threads)
    const char *ev = std::getenv("SALVUS_E2D_EPB");
    const int epb = ev ? std::atoi(ev) : 0;
    auto go = [&](auto tag) {
      constexpr int EPB = decltype(tag)::value;
      using S = Elastic2DShape<N, EPB>;
      elastic2d_stiffness_kernel<N, real, 2, 0, EPB><<<blocks_for(m->E, S::EPB), S::THREADS, 0, s>>>(
          m->E, nullptr, rec, m->d_conn.as<int32_t>(), u, r, dmatrix<real>(m->basis));
      g_launches++;
      return check_launch("elastic 2-D stiffness");
    };
    switch (epb) {
      case 2: return go(std::integral_constant<int, 2>{});
      case 4: return go(std::integral_constant<int, 4>{});
      case 5: return go(std::integral_constant<int, 5>{});
      case 8: return go(std::integral_constant<int, 8>{});
      default: return go(std::integral_constant<int, 0>{});
    }
  }
  return launch_acoustic<2, N, real>(m, rec, u, r, s);
}
template <int N, typename real>
static int acoustic3(const salvus_mesh *m, const real *rec, const real *u, real *r, cudaStream_t s) {
  return launch_acoustic<3, N, real>(m, rec, u, r, s);
}

// P3 simplices on CUDA cores
template <typename real>
static const real *simplex_tables(const salvus_mesh *m) {
  return sizeof(real) == 4 ? (const real *)m->d_sd32.ptr : (const real *)m->d_sd64.ptr;
}

template <typename real, int C, bool TI = false>
static int launch_tet(const salvus_mesh *m, const real *rec, const real *u, real *r,
                      cudaStream_t st) {
  using S = TetShape<real, C, TI>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(tet_stiffness_kernel<real, C, TI>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
    attr = true;
  }
  tet_stiffness_kernel<real, C, TI><<<blocks_for(m->E, S::EPB), S::THREADS, S::SMEM, st>>>(
      m->E, rec, m->d_conn.as<int32_t>(), simplex_tables<real>(m), u, r);
  g_launches++;
  return check_launch("tetrahedron stiffness");
}

// FP32 tetrahedra on the tensor cores (tcgen05, split TF32)
template <int C>
static int launch_tet_tc(const salvus_mesh *m, const float *rec, const float *u, float *r,
                         cudaStream_t st, int *err, long long wlim, int hold) {
  using S = TetTcShape<C>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(tet_tc_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)S::SMEM);
    attr = true;
  }
  const int64_t tiles = (m->E + S::NE - 1) / S::NE;
  const unsigned grid = (unsigned)(tiles < m->sm_count ? tiles : m->sm_count);
  tet_tc_kernel<C><<<grid, S::THREADS, S::SMEM, st>>>(
      m->E, rec, m->d_conn.as<int32_t>(), m->d_tc_tab.as<uint4>(), u, r, err, wlim, hold);
  g_launches++;
  return check_launch("tetrahedron stiffness (tensor cores)");
}

static int launch_tri_tc(const salvus_mesh *m, const float *rec, const float *u, float *r,
                         cudaStream_t st, int *err, long long wlim, int hold) {
  using S = TriTcShape;
  static int per_sm = 0;
  if (!per_sm) {
    cudaFuncSetAttribute(tri_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
    SALVUS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tri_tc_kernel, S::THREADS,
                                                              S::SMEM));
    if (per_sm < 1) per_sm = 1;
  }
  const int64_t tiles = (m->E + S::NE - 1) / S::NE;
  const int64_t slots = (int64_t)per_sm * m->sm_count;
  const unsigned grid = (unsigned)(tiles < slots ? tiles : slots);
  tri_tc_kernel<<<grid, S::THREADS, S::SMEM, st>>>(m->E, rec, m->d_conn.as<int32_t>(),
                                                   m->d_tc_tab.as<uint4>(), u, r, err, wlim, hold);
  g_launches++;
  return check_launch("triangle stiffness (tensor cores)");
}

template <typename real>
static int launch_simplex(const salvus_mesh *m, const real *rec, const real *u, real *r,
                          cudaStream_t st, int *err, long long wlim, int hold) {
  if constexpr (std::is_same<real, float>::value) {
    if (m->shape == SALVUS_TRI && m->tri_kernel == 0)
      return launch_tri_tc(m, rec, u, r, st, err, wlim, hold);
    if (m->shape == SALVUS_TET && m->tet_kernel == 0) {
      if (m->physics == SALVUS_ELASTIC3D)
        return launch_tet_tc<3>(m, rec, u, r, st, err, wlim, hold);
      return launch_tet_tc<1>(m, rec, u, r, st, err, wlim, hold);
    }
  }
  if (m->shape == SALVUS_TRI) {
    if (m->tri_kernel == 2)
      tri_acoustic_kernel<real><<<blocks_for(m->E, 128), 128, 0, st>>>(
          m->E, rec, m->d_conn.as<int32_t>(), simplex_tables<real>(m), u, r);
    else
      tri_acoustic_const_kernel<real><<<blocks_for(m->E, 128), 128, 0, st>>>(
          m->E, rec, m->d_conn.as<int32_t>(), u, r);
    g_launches++;
    return check_launch("triangle stiffness");
  }
  if (m->physics == SALVUS_ELASTIC3D)
    return m->ti ? launch_tet<real, 3, true>(m, rec, u, r, st) : launch_tet<real, 3>(m, rec, u, r, st);
  return launch_tet<real, 1>(m, rec, u, r, st);
}

template <typename real>
static int launch_stiffness(const salvus_mesh *m, const real *rec, const real *u, real *r,
                            cudaStream_t st, int *err = nullptr,
                            long long wlim = salvus::kDefaultWaitLimit, int hold = 0) {
  if (is_simplex(m->shape)) return launch_simplex<real>(m, rec, u, r, st, err, wlim, hold);
  if (m->physics == SALVUS_ELASTIC3D) {
    switch (m->order) {
      case 1: return launch_elastic<1, real>(m, rec, u, r, st);
      case 2: return launch_elastic<2, real>(m, rec, u, r, st);
      case 3: return launch_elastic<3, real>(m, rec, u, r, st);
      case 4: return launch_elastic<4, real>(m, rec, u, r, st);
      case 5: return launch_elastic<5, real>(m, rec, u, r, st);
      case 6: return launch_elastic<6, real>(m, rec, u, r, st);
    }
  } else if (m->shape == SALVUS_QUAD) {
    switch (m->order) {
      case 1: return acoustic2<1, real>(m, rec, u, r, st);
      case 2: return acoustic2<2, real>(m, rec, u, r, st);
      case 3: return acoustic2<3, real>(m, rec, u, r, st);
      case 4: return acoustic2<4, real>(m, rec, u, r, st);
      case 5: return acoustic2<5, real>(m, rec, u, r, st);
      case 6: return acoustic2<6, real>(m, rec, u, r, st);
      case 7: return acoustic2<7, real>(m, rec, u, r, st);
      case 8: return acoustic2<8, real>(m, rec, u, r, st);
      case 9: return acoustic2<9, real>(m, rec, u, r, st);
      case 10: return acoustic2<10, real>(m, rec, u, r, st);
    }
  } else {
    switch (m->order) {
      case 1: return acoustic3<1, real>(m, rec, u, r, st);
      case 2: return acoustic3<2, real>(m, rec, u, r, st);
      case 3: return acoustic3<3, real>(m, rec, u, r, st);
      case 4: return acoustic3<4, real>(m, rec, u, r, st);
      case 5: return acoustic3<5, real>(m, rec, u, r, st);
      case 6: return acoustic3<6, real>(m, rec, u, r, st);
    }
  }
  return fail(SALVUS_E_UNSUPPORTED, "no stiffness kernel for shape %d order %d", m->shape, m->order);
}

// ---------------------------------------------------------------------------
// mesh setup
template <typename real>
static int build_simplex_records(salvus_mesh *m, DeviceBuffer &out, DeviceBuffer &sd,
                                 DeviceBuffer &mass_local) {
  const int rw = record_words(m->shape, m->physics, sizeof(real) == 8, m->ti);
  int rc = out.alloc(sizeof(real) * (size_t)m->E * rw);
  if (rc) return rc;
  SimplexTable tab{};
  for (int q = 0; q < m->P; ++q) {
    for (int a = 0; a < 3; ++a) tab.x[q][a] = m->basis.nodes[(size_t)q * 3 + a];
    tab.w[q] = m->basis.sw[q];
  }
  simplex_geometry_kernel<real><<<blocks_for(m->E, 128), 128, 0, m->stream>>>(
      m->E, m->shape, m->physics, m->P, rw, m->d_vtx.as<double>(), m->d_par.as<double>(), tab,
      out.as<real>(), mass_local.as<double>(), m->ti);
  g_launches++;
  if ((rc = check_launch("simplex geometry"))) return rc;
  std::vector<real> t(m->basis.SD.size());
  for (size_t i = 0; i < t.size(); ++i) t[i] = (real)m->basis.SD[i];
  if ((rc = sd.alloc(sizeof(real) * t.size()))) return rc;
  SALVUS_CUDA(cudaMemcpyAsync(sd.ptr, t.data(), sizeof(real) * t.size(), cudaMemcpyHostToDevice,
                              m->stream));
  if (m->shape == SALVUS_TRI) {
    // the reference triangle's table, identical for every mesh: constant
    // memory of this device (tri_acoustic_const_kernel)
    if (sizeof(real) == 4)
      SALVUS_CUDA(cudaMemcpyToSymbolAsync(c_tri_sd32, t.data(), sizeof(real) * t.size(), 0,
                                          cudaMemcpyHostToDevice, m->stream));
    else
      SALVUS_CUDA(cudaMemcpyToSymbolAsync(c_tri_sd64, t.data(), sizeof(real) * t.size(), 0,
                                          cudaMemcpyHostToDevice, m->stream));
  }
  if (sizeof(real) == 4 && m->shape == SALVUS_TRI) {
    // tensor-core operand images (kernels_tri_tc.cuh), K-major no-swizzle
    // core-matrix order, TF32 hi part and FP32 remainder, zero padding:
    //   B1[kappa = 16 k + q][j] = dphi_j/dxi_k (x_q)   32 x 16
    //   B2[i][kappa = 16 k + q] = dphi_i/dxi_k (x_q)    16 x 32
    constexpr int P = 12;
    constexpr size_t B = 32 * 16;
    std::vector<float> img(4 * B, 0.f);
    auto off = [](int row, int k, int kdim) {
      return (size_t)(((row >> 3) * (kdim / 4) * 128 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4) / 4);
    };
    for (int k = 0; k < 2; ++k)
      for (int q = 0; q < P; ++q)
        for (int j = 0; j < P; ++j) {
          const double v = m->basis.SD[((size_t)k * P + j) * P + q];
          const float f = (float)v;
          uint32_t bits;
          std::memcpy(&bits, &f, 4);
          bits = (bits + 0x1000u) & 0xFFFFE000u;  // nearest TF32 (ties away from zero)
          float hi, lo;
          std::memcpy(&hi, &bits, 4);
          lo = (float)(v - (double)hi);
          const int kap = 16 * k + q;
          img[off(kap, j, 16)] = hi;
          img[B + off(kap, j, 16)] = lo;
          img[2 * B + off(j, kap, 32)] = hi;
          img[3 * B + off(j, kap, 32)] = lo;
        }
    if ((rc = m->d_tc_tab.alloc(sizeof(float) * img.size()))) return rc;
    SALVUS_CUDA(cudaMemcpyAsync(m->d_tc_tab.ptr, img.data(), sizeof(float) * img.size(),
                                cudaMemcpyHostToDevice, m->stream));
  }
  if (sizeof(real) == 4 && m->shape == SALVUS_TET) {
    // tensor-core operand images, K-major no-swizzle core-matrix order, each
    // as a TF32 hi part and an FP32 remainder:
    //   B1[kappa = 56 k + q][j] = dphi_j/dxi_k (x_q)   176 x 56
    //   B2[i][kappa = 56 k + q] = dphi_i/dxi_k (x_q)    64 x 168
    constexpr int P = 50;
    constexpr size_t B1 = 176 * 56, B2 = 64 * 168;
    std::vector<float> img(2 * B1 + 2 * B2, 0.f);
    auto off = [](int row, int k, int kdim) {
      return (size_t)(((row >> 3) * (kdim / 4) * 128 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4) / 4);
    };
    auto split = [](double v, float &hi, float &lo) {
      // nearest TF32 value (round half away from zero on the 13 dropped bits)
      const float f = (float)v;
      uint32_t bits;
      std::memcpy(&bits, &f, 4);
      bits = (bits + 0x1000u) & 0xFFFFE000u;
      std::memcpy(&hi, &bits, 4);
      lo = (float)(v - (double)hi);
    };
    for (int k = 0; k < 3; ++k)
      for (int q = 0; q < P; ++q)
        for (int j = 0; j < P; ++j) {
          float hi, lo;
          split(m->basis.SD[((size_t)k * P + j) * P + q], hi, lo);
          const int kap = 56 * k + q;
          img[off(kap, j, 56)] = hi;
          img[B1 + off(kap, j, 56)] = lo;
          img[2 * B1 + off(j, kap, 168)] = hi;
          img[2 * B1 + B2 + off(j, kap, 168)] = lo;
        }
    if ((rc = m->d_tc_tab.alloc(sizeof(float) * img.size()))) return rc;
    SALVUS_CUDA(cudaMemcpyAsync(m->d_tc_tab.ptr, img.data(), sizeof(float) * img.size(),
                                cudaMemcpyHostToDevice, m->stream));
  }
  SALVUS_CUDA(cudaStreamSynchronize(m->stream));
  return SALVUS_OK;
}

template <typename real, bool kPack>
static int build_records(salvus_mesh *m, DeviceBuffer &out, DeviceBuffer &mass_local) {
  if (is_simplex(m->shape))
    return build_simplex_records<real>(m, out, sizeof(real) == 4 ? m->d_sd32 : m->d_sd64,
                                       mass_local);
  const int rw = record_words(m->shape, m->physics, sizeof(real) == 8, m->ti);
  int rc = out.alloc(sizeof(real) * (size_t)(m->E * m->P) * rw);
  if (rc) return rc;
  GllTable gll{};
  for (int i = 0; i < m->n; ++i) {
    gll.xi[i] = m->basis.xi[i];
    gll.w[i] = m->basis.w[i];
  }
  const int64_t total = m->E * m->P;
  geometry_kernel<real, kPack><<<blocks_for(total, 128), 128, 0, m->stream>>>(
      m->E, m->dim, m->n, m->P, m->physics, rw, m->d_vtx.as<double>(), m->d_par.as<double>(),
      m->d_conn.as<int32_t>(), gll, out.as<real>(), mass_local.as<double>(),
      m->d_cls_k.as<int32_t>(), m->n_fluid, m->ti);
  g_launches++;
  return check_launch("geometry");
}

// Nodes the fused step (parallelepiped elastic hexahedra) and the fused
// batched step (acoustic quadrilaterals) gather: all but the element-interior
// ones (every local index in 1..N-1), which those steps advance in the
// stiffness kernel.  Host-side, ascending node ids.
static void interior_free_nodes(salvus_mesh *m) {
  m->gnodes.clear();
  m->n_gnodes = 0;
  const bool quad = m->shape == SALVUS_QUAD && m->physics == SALVUS_ACOUSTIC;
  if (m->order < 2 || !(m->affine || quad)) return;
  const int n = m->n;
  std::vector<char> interior((size_t)m->G, 0);
  for (int64_t e = 0; e < m->E; ++e) {
    const int32_t *cn = m->conn.data() + e * m->P;
    if (m->dim == 2) {
      for (int j = 1; j < n - 1; ++j)
        for (int i = 1; i < n - 1; ++i) interior[(size_t)cn[i + n * j]] = 1;
    } else {
      for (int k = 1; k < n - 1; ++k)
        for (int j = 1; j < n - 1; ++j)
          for (int i = 1; i < n - 1; ++i) interior[(size_t)cn[i + n * j + n * n * k]] = 1;
    }
  }
  m->gnodes.reserve((size_t)m->G);
  for (int64_t g = 0; g < m->G; ++g)
    if (!interior[(size_t)g]) m->gnodes.push_back((int32_t)g);
  m->n_gnodes = (int64_t)m->gnodes.size();
}

static int mesh_setup_device(salvus_mesh *m) {
  int rc;
  SALVUS_CUDA(cudaSetDevice(m->device));
  SALVUS_CUDA(cudaDeviceGetAttribute(&m->sm_count, cudaDevAttrMultiProcessorCount, m->device));
  SALVUS_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  const int64_t EP = m->E * m->P;
  if ((rc = m->d_conn.alloc(sizeof(int32_t) * EP))) return rc;
  if ((rc = m->d_inc_off.alloc(sizeof(int32_t) * (m->G + 1)))) return rc;
  if ((rc = m->d_inc_idx.alloc(sizeof(int32_t) * EP))) return rc;
  if ((rc = m->d_vtx.alloc(sizeof(double) * m->vtx.size()))) return rc;
  if ((rc = m->d_par.alloc(sizeof(double) * m->par.size()))) return rc;
  if ((rc = m->d_mi64.alloc(sizeof(double) * m->G))) return rc;
  if ((rc = m->d_mi32.alloc(sizeof(float) * m->G))) return rc;
  SALVUS_CUDA(cudaMemcpyAsync(m->d_conn.ptr, m->conn.data(), sizeof(int32_t) * EP,
                              cudaMemcpyHostToDevice, m->stream));
  SALVUS_CUDA(cudaMemcpyAsync(m->d_inc_off.ptr, m->inc_off.data(), sizeof(int32_t) * (m->G + 1),
                              cudaMemcpyHostToDevice, m->stream));
  SALVUS_CUDA(cudaMemcpyAsync(m->d_inc_idx.ptr, m->inc_idx.data(), sizeof(int32_t) * EP,
                              cudaMemcpyHostToDevice, m->stream));
  SALVUS_CUDA(cudaMemcpyAsync(m->d_vtx.ptr, m->vtx.data(), sizeof(double) * m->vtx.size(),
                              cudaMemcpyHostToDevice, m->stream));
  SALVUS_CUDA(cudaMemcpyAsync(m->d_par.ptr, m->par.data(), sizeof(double) * m->par.size(),
                              cudaMemcpyHostToDevice, m->stream));
  if (m->physics == SALVUS_COUPLED2D) {
    const size_t nc = (size_t)m->n_cpl;
    std::vector<float> c32(m->cpl_coef.begin(), m->cpl_coef.end());
    if ((rc = m->d_elist.alloc(sizeof(int32_t) * m->E)) ||
        (rc = m->d_cls_k.alloc(sizeof(int32_t) * m->E)) ||
        (rc = m->d_cpl_pts.alloc(sizeof(int32_t) * 2 * nc)) ||
        (rc = m->d_cpl32.alloc(sizeof(float) * 2 * nc)) ||
        (rc = m->d_cpl64.alloc(sizeof(double) * 2 * nc)))
      return rc;
    SALVUS_CUDA(cudaMemcpyAsync(m->d_elist.ptr, m->elist.data(), sizeof(int32_t) * m->E,
                                cudaMemcpyHostToDevice, m->stream));
    SALVUS_CUDA(cudaMemcpyAsync(m->d_cls_k.ptr, m->cls_k.data(), sizeof(int32_t) * m->E,
                                cudaMemcpyHostToDevice, m->stream));
    if (nc) {
      SALVUS_CUDA(cudaMemcpyAsync(m->d_cpl_pts.ptr, m->cpl_pts.data(), sizeof(int32_t) * 2 * nc,
                                  cudaMemcpyHostToDevice, m->stream));
      SALVUS_CUDA(cudaMemcpyAsync(m->d_cpl32.ptr, c32.data(), sizeof(float) * 2 * nc,
                                  cudaMemcpyHostToDevice, m->stream));
      SALVUS_CUDA(cudaMemcpyAsync(m->d_cpl64.ptr, m->cpl_coef.data(), sizeof(double) * 2 * nc,
                                  cudaMemcpyHostToDevice, m->stream));
    }
    SALVUS_CUDA(cudaStreamSynchronize(m->stream));
  }
  DeviceBuffer mass_local;
  if ((rc = mass_local.alloc(sizeof(double) * EP))) return rc;
  if (m->affine) {
    // parallelepiped elastic hexahedra: material planes + per-element invJ
    const int nm = m->ti ? 5 : 2;
    if ((rc = m->d_rec32.alloc(sizeof(float) * (size_t)nm * EP)) ||
        (rc = m->d_jac32.alloc(sizeof(float) * 9 * (size_t)m->E)))
      return rc;
    GllTable gll{};
    for (int i = 0; i < m->n; ++i) {
      gll.xi[i] = m->basis.xi[i];
      gll.w[i] = m->basis.w[i];
    }
    affine_hex_records_kernel<<<blocks_for(EP, 128), 128, 0, m->stream>>>(
        m->E, m->n, m->P, m->ti, m->d_vtx.as<double>(), m->d_par.as<double>(), gll,
        m->d_rec32.as<float>(), m->d_jac32.as<float>(), mass_local.as<double>());
    g_launches++;
    if ((rc = check_launch("affine records"))) return rc;
  } else if ((rc = build_records<float, true>(m, m->d_rec32, mass_local))) {
    return rc;
  }
  // the node list of the fused steps (interior_free_nodes, at creation)
  if (m->n_gnodes > 0) {
    if ((rc = m->d_gnodes.alloc(sizeof(int32_t) * (size_t)m->n_gnodes))) return rc;
    SALVUS_CUDA(cudaMemcpyAsync(m->d_gnodes.ptr, m->gnodes.data(), sizeof(int32_t) * m->gnodes.size(),
                                cudaMemcpyHostToDevice, m->stream));
    SALVUS_CUDA(cudaStreamSynchronize(m->stream));
  }
  if (!m->fp32_only && (rc = build_records<double, false>(m, m->d_rec64, mass_local))) return rc;
  mass_gather_kernel<<<blocks_for(m->G, 256), 256, 0, m->stream>>>(
      m->G, m->d_inc_off.as<int32_t>(), m->d_inc_idx.as<int32_t>(), mass_local.as<double>(),
      m->d_mi64.as<double>(), m->d_mi32.as<float>());
  g_launches++;
  if ((rc = check_launch("mass"))) return rc;
  m->mi.resize(m->G);
  SALVUS_CUDA(cudaMemcpyAsync(m->mi.data(), m->d_mi64.ptr, sizeof(double) * m->G,
                              cudaMemcpyDeviceToHost, m->stream));
  SALVUS_CUDA(cudaStreamSynchronize(m->stream));
  return SALVUS_OK;
}

// ---------------------------------------------------------------------------
// problem helpers
template <typename real>
static real *F(const DeviceBuffer &b) { return b.as<real>(); }

static int upload_sources(salvus_problem *p) {
  if (!p->src_dirty) return SALVUS_OK;
  const salvus_mesh *m = p->mesh;
  const size_t ns = p->srcs.size();
  int rc;
  if (ns) {
    // batched problems group sources by shot (attach order kept within a shot)
    std::vector<size_t> order(ns);
    for (size_t s = 0; s < ns; ++s) order[s] = s;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
      return p->srcs[a].desc.shot < p->srcs[b].desc.shot;
    });
    std::vector<int64_t> el(ns);
    std::vector<double> par(3 * ns), w(ns * m->P * p->c);
    std::vector<int32_t> shot_off(p->shots_pad + 1, 0);
    for (size_t k = 0; k < ns; ++k) {
      const auto &src = p->srcs[order[k]];
      el[k] = src.elem;
      par[3 * k] = src.desc.center_freq;
      par[3 * k + 1] = src.desc.time_delay;
      par[3 * k + 2] = src.desc.amplitude;
      std::memcpy(&w[k * m->P * p->c], src.wts.data(), sizeof(double) * m->P * p->c);
      shot_off[src.desc.shot + 1]++;
    }
    for (int s = 0; s < p->shots_pad; ++s) shot_off[s + 1] += shot_off[s];
    if ((rc = p->d_shot_off.alloc(sizeof(int32_t) * shot_off.size()))) return rc;
    SALVUS_CUDA(cudaMemcpyAsync(p->d_shot_off.ptr, shot_off.data(), sizeof(int32_t) * shot_off.size(),
                                cudaMemcpyHostToDevice, p->stream));
    if ((rc = p->d_src_elem.alloc(sizeof(int64_t) * ns))) return rc;
    if ((rc = p->d_src_par.alloc(sizeof(double) * par.size()))) return rc;
    if ((rc = p->d_src_wts.alloc(sizeof(double) * w.size()))) return rc;
    SALVUS_CUDA(cudaMemcpyAsync(p->d_src_elem.ptr, el.data(), sizeof(int64_t) * ns,
                                cudaMemcpyHostToDevice, p->stream));
    SALVUS_CUDA(cudaMemcpyAsync(p->d_src_par.ptr, par.data(), sizeof(double) * par.size(),
                                cudaMemcpyHostToDevice, p->stream));
    SALVUS_CUDA(cudaMemcpyAsync(p->d_src_wts.ptr, w.data(), sizeof(double) * w.size(),
                                cudaMemcpyHostToDevice, p->stream));
    // distinct source elements, first appearance order (fused hexahedron step)
    std::vector<int64_t> ue;
    for (int64_t x : el)
      if (std::find(ue.begin(), ue.end(), x) == ue.end()) ue.push_back(x);
    if ((rc = p->d_src_uelem.alloc(sizeof(int64_t) * ue.size()))) return rc;
    SALVUS_CUDA(cudaMemcpyAsync(p->d_src_uelem.ptr, ue.data(), sizeof(int64_t) * ue.size(),
                                cudaMemcpyHostToDevice, p->stream));
    p->n_src_uelem = (int)ue.size();
    SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  } else {
    p->n_src_uelem = 0;
  }
  p->src_dirty = false;
  return SALVUS_OK;
}

static int upload_receivers(salvus_problem *p) {
  if (!p->rec_dirty) return SALVUS_OK;
  const salvus_mesh *m = p->mesh;
  const size_t nr = p->recs.size();
  int rc;
  std::vector<int64_t> el(nr ? nr : 1, 0);
  std::vector<double> l(nr ? nr * m->P : 1, 0.0);
  for (size_t r = 0; r < nr; ++r) {
    el[r] = p->recs[r].elem;
    std::memcpy(&l[r * m->P], p->recs[r].l.data(), sizeof(double) * m->P);
  }
  if ((rc = p->d_rec_elem.alloc(sizeof(int64_t) * el.size()))) return rc;
  if ((rc = p->d_rec_l.alloc(sizeof(double) * l.size()))) return rc;
  size_t sz = sizeof(double) * (size_t)(nr ? nr : 1) * p->c * p->seis_cap * p->shots_pad;
  if ((rc = p->d_seis.alloc(sz))) return rc;
  SALVUS_CUDA(cudaMemsetAsync(p->d_seis.ptr, 0, sz, p->stream));
  SALVUS_CUDA(cudaMemcpyAsync(p->d_rec_elem.ptr, el.data(), sizeof(int64_t) * el.size(),
                              cudaMemcpyHostToDevice, p->stream));
  SALVUS_CUDA(cudaMemcpyAsync(p->d_rec_l.ptr, l.data(), sizeof(double) * l.size(),
                              cudaMemcpyHostToDevice, p->stream));
  SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  p->rec_dirty = false;
  return SALVUS_OK;
}

static void drop_graph(salvus_problem *p) {
  if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
  p->graph_exec = nullptr;
  p->graph_steps = 0;
  if (p->tail_exec) cudaGraphExecDestroy(p->tail_exec);
  p->tail_exec = nullptr;
  p->tail_steps = 0;
}

// fluid-solid coupling integrals (meshes of fluid and solid quadrilaterals)
template <typename real>
static int launch_coupling(salvus_problem *p) {
  const salvus_mesh *m = p->mesh;
  if (m->physics != SALVUS_COUPLED2D || m->n_cpl == 0) return SALVUS_OK;
  const real *coef = sizeof(real) == 4 ? (const real *)m->d_cpl32.ptr : (const real *)m->d_cpl64.ptr;
  coupling_kernel<real><<<blocks_for(m->n_cpl, 256), 256, 0, p->stream>>>(
      m->n_cpl_fluid, m->n_cpl, m->d_cpl_pts.as<int32_t>(), coef, F<real>(p->d_v), F<real>(p->d_r));
  g_launches++;
  return check_launch("coupling");
}

template <typename real, int C>
static int launch_dirichlet(salvus_problem *p) {
  if (p->n_dir_pts == 0) return SALVUS_OK;
  dirichlet_zero_kernel<real, C><<<blocks_for(p->n_dir_pts, 256), 256, 0, p->stream>>>(
      p->n_dir_pts, p->d_dir_pts.as<int32_t>(), F<real>(p->d_r));
  g_launches++;
  return check_launch("dirichlet");
}

template <typename real, int C>
static int launch_sources(salvus_problem *p) {
  if (p->srcs.empty()) return SALVUS_OK;
  ProfScope ps(p, K_SRC);
  source_kernel<real, C><<<1, 256, 0, p->stream>>>(
      (int)p->srcs.size(), p->mesh->P, p->d_src_elem.as<int64_t>(), p->d_src_par.as<double>(),
      p->d_src_wts.as<double>(), p->d_step.as<int64_t>(), p->dt, F<real>(p->d_r));
  g_launches++;
  return check_launch("source");
}

// Receivers of step n read u after its update and advance the device step
// counter; step n + 1's stiffness launch only reads u.  In the steps a
// graph run captures (rec_overlap) they therefore run on a second stream,
// forked after the node update, and step n + 1 joins them after its
// stiffness launch, before its sources (which read the step counter) and
// its node update (which writes u); the captured sequence ends joined, so
// every later operation on the problem's stream is ordered after them.
// Host-launched and profiled steps keep them on the problem's stream.
static int join_receivers(salvus_problem *p) {
  if (!p->rec_pending) return SALVUS_OK;
  p->rec_pending = false;
  SALVUS_CUDA(cudaStreamWaitEvent(p->stream, p->ev_recorded, 0));
  return SALVUS_OK;
}

template <typename real, int C>
static int launch_receivers(salvus_problem *p) {
  ProfScope ps(p, K_REC);
  cudaStream_t st = p->stream;
  const bool fork = p->rec_overlap && !p->profiling && p->rec_stream;
  if (fork) {
    SALVUS_CUDA(cudaEventRecord(p->ev_updated, p->stream));
    SALVUS_CUDA(cudaStreamWaitEvent(p->rec_stream, p->ev_updated, 0));
    st = p->rec_stream;
  }
  const int nr = (int)p->recs.size();
  if (nr > 0) {
    receiver_kernel<real, C><<<nr, kRecThreads, 0, st>>>(
        p->mesh->P, p->d_rec_elem.as<int64_t>(), p->d_rec_l.as<double>(),
        p->mesh->d_conn.as<int32_t>(), F<real>(p->d_u), p->d_seis.as<double>(), p->seis_cap,
        p->d_step.as<int64_t>());
    g_launches++;
  }
  advance_step_kernel<<<1, 1, 0, st>>>(p->d_step.as<int64_t>());
  g_launches++;
  if (fork) {
    SALVUS_CUDA(cudaEventRecord(p->ev_recorded, p->rec_stream));
    p->rec_pending = true;
  }
  return check_launch("receivers");
}

template <typename real>
static const real *records(const salvus_problem *p) {
  return sizeof(real) == 4 ? (const real *)p->mesh->d_rec32.ptr : (const real *)p->mesh->d_rec64.ptr;
}
template <typename real>
static const real *inv_mass(const salvus_problem *p) {
  return sizeof(real) == 4 ? (const real *)p->mesh->d_mi32.ptr : (const real *)p->mesh->d_mi64.ptr;
}

// The fused FP32 step of parallelepiped elastic hexahedra advances the
// element-interior nodes inside the stiffness kernel and gathers the rest
// (kernels_hex_affine.cuh).  Measured on the 64^3 order-4 workload it is
// slower than the plain sequence on the same records (the interior update
// costs the stiffness kernel more than the shorter gather saves), so the
// hexahedron autotuner (tune_hex) picks between the two per problem;
// SALVUS_HEX_STEP=fused / plain forces the form (read at every step).  It is
// admissible for problems without Dirichlet points and with at most
// kFuseMaxSources sources (each interior column scans their elements).
constexpr int kFuseMaxSources = 16;
static bool hex_fusion_admissible(const salvus_problem *p) {
  const salvus_mesh *m = p->mesh;
  return m->affine && m->n_gnodes > 0 && p->prec == SALVUS_FP32 && p->shots == 1 &&
         p->n_dir_pts == 0 && (int)p->srcs.size() <= kFuseMaxSources;
}
static bool hex_interior_fusion(const salvus_problem *p) {
  if (!hex_fusion_admissible(p)) return false;
  const char *s = std::getenv("SALVUS_HEX_STEP");
  if (s && std::strcmp(s, "fused") == 0) return true;
  if (s && std::strcmp(s, "plain") == 0) return false;
  return p->hex_form == 1;
}

template <bool TI>
static int launch_fused_interior(salvus_problem *p, const HexInteriorUpdate &iu) {
  const salvus_mesh *m = p->mesh;
  const float *mat = m->d_rec32.as<float>();
  float *u = F<float>(p->d_u), *r = F<float>(p->d_r);
  switch (m->order) {
    case 2: return launch_elastic_affine<2, TI, true>(m, mat, u, r, p->stream, iu);
    case 3: return launch_elastic_affine<3, TI, true>(m, mat, u, r, p->stream, iu);
    case 4: return launch_elastic_affine<4, TI, true>(m, mat, u, r, p->stream, iu);
    case 5: return launch_elastic_affine<5, TI, true>(m, mat, u, r, p->stream, iu);
    case 6: return launch_elastic_affine<6, TI, true>(m, mat, u, r, p->stream, iu);
  }
  return fail(SALVUS_E_UNSUPPORTED, "fused hexahedron step: order %d", m->order);
}

static int step_fused_hex_interior(salvus_problem *p) {
  const salvus_mesh *m = p->mesh;
  int rc;
  // this stiffness launch writes u (interior nodes): the previous step's
  // receivers, which read u, finish first
  if ((rc = join_receivers(p))) return rc;
  {
    ProfScope ps(p, K_STIFF);
    HexInteriorUpdate iu{};
    iu.mi = m->d_mi32.as<float>();
    iu.v = F<float>(p->d_v);
    iu.ap = F<float>(p->d_ap);
    iu.dt = (float)p->dt;
    iu.nsrc_elem = p->n_src_uelem;
    iu.src_elem = p->d_src_uelem.as<int64_t>();
    if ((rc = m->ti ? launch_fused_interior<true>(p, iu) : launch_fused_interior<false>(p, iu)))
      return rc;
  }
  // sources, then the source elements' interior nodes
  if (!p->srcs.empty()) {
    ProfScope ps(p, K_SRC);
    auto go = [&](auto nt) {
      constexpr int N = decltype(nt)::value;
      source_fused_hex_kernel<N><<<1, 256, 0, p->stream>>>(
          (int)p->srcs.size(), m->P, p->d_src_elem.as<int64_t>(), p->d_src_par.as<double>(),
          p->d_src_wts.as<double>(), p->d_step.as<int64_t>(), p->dt, F<float>(p->d_r),
          p->n_src_uelem, p->d_src_uelem.as<int64_t>(), m->d_conn.as<int32_t>(),
          m->d_mi32.as<float>(), F<float>(p->d_u), F<float>(p->d_v), F<float>(p->d_ap),
          (float)p->dt);
    };
    switch (m->order) {
      case 2: go(std::integral_constant<int, 2>{}); break;
      case 3: go(std::integral_constant<int, 3>{}); break;
      case 4: go(std::integral_constant<int, 4>{}); break;
      case 5: go(std::integral_constant<int, 5>{}); break;
      case 6: go(std::integral_constant<int, 6>{}); break;
      default: return fail(SALVUS_E_UNSUPPORTED, "fused hexahedron step: order %d", m->order);
    }
    g_launches++;
    if ((rc = check_launch("source (fused step)"))) return rc;
  }
  {
    ProfScope ps(p, K_UPDATE);
    gather_list_kernel<float, 3, 0><<<blocks_for(m->n_gnodes, 256), 256, 0, p->stream>>>(
        m->n_gnodes, m->d_gnodes.as<int32_t>(), m->d_inc_off.as<int32_t>(),
        m->d_inc_idx.as<int32_t>(), F<float>(p->d_r), m->d_mi32.as<float>(), F<float>(p->d_u),
        F<float>(p->d_v), F<float>(p->d_ap), F<float>(p->d_a), (float)p->dt);
    g_launches++;
    if ((rc = check_launch("gather update (shared nodes)"))) return rc;
  }
  return launch_receivers<float, 3>(p);
}

template <typename real, int C>
static int step_fused_t(salvus_problem *p) {
  const salvus_mesh *m = p->mesh;
  int rc;
  if constexpr (std::is_same<real, float>::value && C == 3) {
    if (hex_interior_fusion(p)) return step_fused_hex_interior(p);
  }
  {
    ProfScope ps(p, K_STIFF);
    if ((rc = launch_stiffness<real>(m, records<real>(p), F<real>(p->d_u), F<real>(p->d_r), p->stream,
                                       p->d_err.as<int>(), p->wait_limit, p->hold_waits)))
      return rc;
  }
  if ((rc = join_receivers(p))) return rc;  // the previous step's receivers
  if ((rc = launch_dirichlet<real, C>(p))) return rc;
  if ((rc = launch_coupling<real>(p))) return rc;
  if ((rc = launch_sources<real, C>(p))) return rc;
  {
    ProfScope ps(p, K_UPDATE);
    // 128-thread CTAs: measured against 64 / 256 / 512 on the benchmark
    // meshes, 1 % (hexahedra) to 5 % (tetrahedra) faster than 256
    constexpr int kGatherThreads = 128;
    gather_kernel<real, C, 0><<<blocks_for(m->G, kGatherThreads), kGatherThreads, 0, p->stream>>>(
        m->G, m->d_inc_off.as<int32_t>(), m->d_inc_idx.as<int32_t>(), F<real>(p->d_r),
        inv_mass<real>(p), F<real>(p->d_u), F<real>(p->d_v), F<real>(p->d_ap), F<real>(p->d_a),
        (real)p->dt);
    g_launches++;
    if ((rc = check_launch("gather update"))) return rc;
  }
  return launch_receivers<real, C>(p);
}

// ---------------------------------------------------------------------------
// shot-batched step (FP32 acoustic quads)
struct BatchCfg {
  int sc, epc, npt;  // shot lanes, elements / node groups per CTA, nodes per thread
};
static const BatchCfg kStiffCfg[] = {{32, 1, 1}, {32, 2, 1}, {32, 4, 1}, {64, 1, 1},
                                     {64, 2, 1}, {128, 1, 1}, {128, 2, 1}, {256, 1, 1}};
static const BatchCfg kGatherCfg[] = {{32, 4, 1},  {32, 8, 1}, {64, 2, 1}, {64, 4, 1},
                                      {128, 1, 1}, {128, 2, 1}, {256, 1, 1}, {32, 4, 2},
                                      {64, 2, 2},  {128, 1, 2}, {128, 1, 4}, {256, 1, 2}};
constexpr int kNumStiffCfg = sizeof(kStiffCfg) / sizeof(kStiffCfg[0]);
constexpr int kNumGatherCfg = sizeof(kGatherCfg) / sizeof(kGatherCfg[0]);

// Fused batched step (kernels_batch.cuh, kFuse): interior nodes advanced in
// the stiffness kernel, edge nodes by the node-list gather.  Used when the
// mesh has interior nodes (order >= 2); SALVUS_BATCH_STEP=unfused selects
// the plain sequence (read at every step).
static bool batch_fusion(const salvus_problem *p) {
  if (p->mesh->n_gnodes <= 0) return false;
  const char *s = std::getenv("SALVUS_BATCH_STEP");
  return !(s && std::strcmp(s, "unfused") == 0);
}

template <int N, int SC, int EPC>
static void launch_qb(const salvus_problem *p, cudaStream_t st, bool fuse) {
  const salvus_mesh *m = p->mesh;
  dim3 grid((unsigned)((m->E + EPC - 1) / EPC), (unsigned)(p->shots_pad / SC));
  BatchInterior bi{};
  if (fuse) {
    bi.mi = m->d_mi32.as<float>();
    bi.w = F<float>(p->d_v);
    bi.dt = (float)p->dt;
    bi.shot_off = p->srcs.empty() ? nullptr : p->d_shot_off.as<int32_t>();
    bi.src_elem = p->d_src_elem.as<int64_t>();
    quad_acoustic_batched_kernel<N, SC, EPC, true><<<grid, SC * EPC, 0, st>>>(
        m->E, p->shots_pad, m->d_rec32.as<float>(), F<float>(p->d_u), F<float>(p->d_r),
        dmatrix<float>(m->basis), bi);
  } else {
    quad_acoustic_batched_kernel<N, SC, EPC, false><<<grid, SC * EPC, 0, st>>>(
        m->E, p->shots_pad, m->d_rec32.as<float>(), F<float>(p->d_u), F<float>(p->d_r),
        dmatrix<float>(m->basis), bi);
  }
}

template <int N>
static int launch_qb_cfg(const salvus_problem *p, int cfg, cudaStream_t st, bool fuse) {
  switch (cfg) {
    case 0: launch_qb<N, 32, 1>(p, st, fuse); break;
    case 1: launch_qb<N, 32, 2>(p, st, fuse); break;
    case 2: launch_qb<N, 32, 4>(p, st, fuse); break;
    case 3: launch_qb<N, 64, 1>(p, st, fuse); break;
    case 4: launch_qb<N, 64, 2>(p, st, fuse); break;
    case 5: launch_qb<N, 128, 1>(p, st, fuse); break;
    case 6: launch_qb<N, 128, 2>(p, st, fuse); break;
    case 7: launch_qb<N, 256, 1>(p, st, fuse); break;
    default: return fail(SALVUS_E_INVALID, "bad batch config %d", cfg);
  }
  g_launches++;
  return check_launch("batched stiffness");
}

static int batched_stiffness(const salvus_problem *p, int cfg, cudaStream_t st, bool fuse) {
  switch (p->mesh->order) {
    case 1: return launch_qb_cfg<1>(p, cfg, st, false);  // no interior nodes
    case 2: return launch_qb_cfg<2>(p, cfg, st, fuse);
    case 3: return launch_qb_cfg<3>(p, cfg, st, fuse);
    case 4: return launch_qb_cfg<4>(p, cfg, st, fuse);
    case 5: return launch_qb_cfg<5>(p, cfg, st, fuse);
    case 6: return launch_qb_cfg<6>(p, cfg, st, fuse);
  }
  return fail(SALVUS_E_UNSUPPORTED, "batched quads support orders 1..6");
}

template <int SC, int NPB, int NPT = 1>
static void launch_bg(const salvus_problem *p, cudaStream_t st, bool fuse) {
  const salvus_mesh *m = p->mesh;
  const int64_t n = fuse ? m->n_gnodes : m->G;
  dim3 grid((unsigned)((n + NPB * NPT - 1) / (NPB * NPT)), (unsigned)(p->shots_pad / SC));
  batched_gather_update_kernel<SC, NPB, NPT><<<grid, SC * NPB, 0, st>>>(
      n, p->shots_pad, m->d_inc_off.as<int32_t>(), m->d_inc_idx.as<int32_t>(),
      F<float>(p->d_r), m->d_mi32.as<float>(), F<float>(p->d_u), F<float>(p->d_v), (float)p->dt,
      fuse ? m->d_gnodes.as<int32_t>() : nullptr);
}

static int batched_gather(const salvus_problem *p, int cfg, cudaStream_t st, bool fuse) {
  switch (cfg) {
    case 0: launch_bg<32, 4>(p, st, fuse); break;
    case 1: launch_bg<32, 8>(p, st, fuse); break;
    case 2: launch_bg<64, 2>(p, st, fuse); break;
    case 3: launch_bg<64, 4>(p, st, fuse); break;
    case 4: launch_bg<128, 1>(p, st, fuse); break;
    case 5: launch_bg<128, 2>(p, st, fuse); break;
    case 6: launch_bg<256, 1>(p, st, fuse); break;
    case 7: launch_bg<32, 4, 2>(p, st, fuse); break;
    case 8: launch_bg<64, 2, 2>(p, st, fuse); break;
    case 9: launch_bg<128, 1, 2>(p, st, fuse); break;
    case 10: launch_bg<128, 1, 4>(p, st, fuse); break;
    case 11: launch_bg<256, 1, 2>(p, st, fuse); break;
    default: return fail(SALVUS_E_INVALID, "bad gather config %d", cfg);
  }
  g_launches++;
  return check_launch("batched gather");
}

// Times every admissible configuration of the batched stiffness and gather
// kernels on this problem and keeps the fastest.  The stiffness timing writes
// only the residual scratch; the gather timing runs on copies of u and w, so
// the problem's state is untouched.  Results are cached per (order, padded
// shots, elements, device) for the process.
static int autotune(salvus_problem *p) {
  if (p->tune_stiff >= 0 && p->tune_gather >= 0) return SALVUS_OK;
  struct Key {
    int order, shots;
    int64_t E;
    int dev;
  };
  static std::mutex cache_mu;
  static std::vector<std::pair<Key, std::pair<int, int>>> cache;
  {
    std::lock_guard<std::mutex> lk(cache_mu);
    for (auto &c : cache)
      if (c.first.order == p->mesh->order && c.first.shots == p->shots_pad &&
          c.first.E == p->mesh->E && c.first.dev == p->mesh->device) {
        p->tune_stiff = c.second.first;
        p->tune_gather = c.second.second;
        return SALVUS_OK;
      }
  }
  const char *env = std::getenv("SALVUS_BATCH_CONFIG");  // "stiff,gather" fixes the choice
  if (env) {
    int a = -1, b = -1;
    if (std::sscanf(env, "%d,%d", &a, &b) == 2 && a >= 0 && a < kNumStiffCfg && b >= 0 &&
        b < kNumGatherCfg && p->shots_pad % kStiffCfg[a].sc == 0 && p->shots_pad % kGatherCfg[b].sc == 0) {
      p->tune_stiff = a;
      p->tune_gather = b;
      return SALVUS_OK;
    }
  }
  cudaEvent_t e0, e1;
  SALVUS_CUDA(cudaEventCreate(&e0));
  SALVUS_CUDA(cudaEventCreate(&e1));
  int rc = SALVUS_OK;
  auto time_it = [&](auto &&fn) -> float {
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      cudaEventRecord(e0, p->stream);
      if ((rc = fn())) return 1e30f;
      cudaEventRecord(e1, p->stream);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      best = std::min(best, ms);
    }
    return best;
  };
  // both kernels are timed on zeroed scratch copies of u and w (the fused
  // stiffness kernel also advances interior nodes), so the problem's state
  // is untouched
  const bool fuse = batch_fusion(p);
  const size_t nf = (size_t)p->mesh->G * p->shots_pad * sizeof(float);
  DeviceBuffer su, sw;
  float bs = 1e30f;
  int cs = -1;
  if (rc == SALVUS_OK && ((rc = su.alloc(nf)) == SALVUS_OK) && ((rc = sw.alloc(nf)) == SALVUS_OK)) {
    std::swap(p->d_u.ptr, su.ptr);
    std::swap(p->d_v.ptr, sw.ptr);
    cudaMemsetAsync(p->d_u.ptr, 0, nf, p->stream);
    cudaMemsetAsync(p->d_v.ptr, 0, nf, p->stream);
    for (int c = 0; c < kNumStiffCfg && rc == SALVUS_OK; ++c) {
      if (p->shots_pad % kStiffCfg[c].sc) continue;
      float t = time_it([&] { return batched_stiffness(p, c, p->stream, fuse); });
      if (t < bs) { bs = t; cs = c; }
    }
    float bg = 1e30f;
    int cg = -1;
    for (int c = 0; c < kNumGatherCfg && rc == SALVUS_OK; ++c) {
      if (p->shots_pad % kGatherCfg[c].sc) continue;
      float t = time_it([&] { return batched_gather(p, c, p->stream, fuse); });
      if (t < bg) { bg = t; cg = c; }
    }
    std::swap(p->d_u.ptr, su.ptr);
    std::swap(p->d_v.ptr, sw.ptr);
    p->tune_gather = cg;
  }
  cudaStreamSynchronize(p->stream);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (cs < 0 || p->tune_gather < 0) return fail(SALVUS_E_INVALID, "no admissible batch configuration");
  p->tune_stiff = cs;
  std::lock_guard<std::mutex> lk(cache_mu);
  cache.push_back({{p->mesh->order, p->shots_pad, p->mesh->E, p->mesh->device},
                   {p->tune_stiff, p->tune_gather}});
  return SALVUS_OK;
}

static int step_batched(salvus_problem *p) {
  const salvus_mesh *m = p->mesh;
  int rc;
  {
    ProfScope ps(p, K_STIFF);
    if ((rc = batched_stiffness(p, p->tune_stiff, p->stream, batch_fusion(p)))) return rc;
  }
  if (!p->srcs.empty()) {
    ProfScope ps(p, K_SRC);
    const int threads = 256, total = p->shots_pad * m->P;
    // fused step: the source elements' interior nodes are finished here
    const bool fuse = batch_fusion(p) && m->order >= 2;
    batched_source_kernel<<<(total + threads - 1) / threads, threads, 0, p->stream>>>(
        p->shots_pad, m->P, p->d_shot_off.as<int32_t>(), p->d_src_elem.as<int64_t>(),
        p->d_src_par.as<double>(), p->d_src_wts.as<double>(), p->d_step.as<int64_t>(), p->dt,
        F<float>(p->d_r), fuse ? m->n : 0, m->d_conn.as<int32_t>(), m->d_mi32.as<float>(),
        F<float>(p->d_u), F<float>(p->d_v), (float)p->dt);
    g_launches++;
    if ((rc = check_launch("batched sources"))) return rc;
  }
  {
    ProfScope ps(p, K_UPDATE);
    if ((rc = batched_gather(p, p->tune_gather, p->stream, batch_fusion(p)))) return rc;
  }
  ProfScope ps(p, K_REC);
  if (!p->recs.empty()) {
    const int threads = p->shots_pad < 256 ? p->shots_pad : 256;
    batched_receiver_kernel<<<(unsigned)p->recs.size(), threads, 0, p->stream>>>(
        p->shots_pad, (int)p->recs.size(), m->P, p->d_rec_elem.as<int64_t>(),
        p->d_rec_l.as<double>(), m->d_conn.as<int32_t>(), F<float>(p->d_u),
        p->d_seis.as<double>(), p->seis_cap, p->d_step.as<int64_t>());
    g_launches++;
  }
  advance_step_kernel<<<1, 1, 0, p->stream>>>(p->d_step.as<int64_t>());
  g_launches++;
  return check_launch("batched receivers");
}

static int step_fused(salvus_problem *p) {
  if (p->shots > 1) return step_batched(p);
  return by_components(p->c, [&](auto cc) {
    constexpr int C = decltype(cc)::value;
    return p->prec == SALVUS_FP32 ? step_fused_t<float, C>(p) : step_fused_t<double, C>(p);
  });
}

template <typename real, int C>
static int assemble_t(salvus_problem *p) {
  const salvus_mesh *m = p->mesh;
  int rc;
  {
    ProfScope ps(p, K_STIFF);
    if ((rc = launch_stiffness<real>(m, records<real>(p), F<real>(p->d_u), F<real>(p->d_r), p->stream,
                                       p->d_err.as<int>(), p->wait_limit, p->hold_waits)))
      return rc;
  }
  if ((rc = launch_dirichlet<real, C>(p))) return rc;
  if ((rc = launch_coupling<real>(p))) return rc;
  if ((rc = launch_sources<real, C>(p))) return rc;
  ProfScope ps(p, K_GATHER);
  gather_kernel<real, C, 1><<<blocks_for(m->G, 256), 256, 0, p->stream>>>(
      m->G, m->d_inc_off.as<int32_t>(), m->d_inc_idx.as<int32_t>(), F<real>(p->d_r), nullptr,
      nullptr, nullptr, nullptr, F<real>(p->d_a), (real)0);
  g_launches++;
  return check_launch("gather");
}

template <typename real, int C>
static int minv_t(salvus_problem *p) {
  ProfScope ps(p, K_MINV);
  const int64_t N = p->mesh->G * C;
  inverse_mass_kernel<real, C><<<blocks_for(N, 256), 256, 0, p->stream>>>(
      p->mesh->G, inv_mass<real>(p), F<real>(p->d_a));
  g_launches++;
  return check_launch("inverse mass");
}

template <typename real, int C>
static int newmark_t(salvus_problem *p) {
  int rc;
  {
    ProfScope ps(p, K_NEWMARK);
    const int64_t N = p->mesh->G * C;
    newmark_kernel<real><<<blocks_for(N, 256), 256, 0, p->stream>>>(
        N, F<real>(p->d_a), F<real>(p->d_u), F<real>(p->d_v), F<real>(p->d_ap), (real)p->dt);
    g_launches++;
    if ((rc = check_launch("newmark"))) return rc;
  }
  return launch_receivers<real, C>(p);
}

// True when the FP32 stiffness launch of this mesh runs a kernel whose
// bounded waits report a timeout through the error word (tensor-core
// simplices); mirrors launch_stiffness.
bool stiffness_reports_errors(const salvus_mesh *m, int precision) {
  if (precision != SALVUS_FP32) return false;
  if (m->shape == SALVUS_TET) return m->tet_kernel == 0;
  if (m->shape == SALVUS_TRI) return m->tri_kernel == 0;
  return false;
}

// a = -K u for caller-owned device buffers, with the element-local residual
// in caller-provided scratch and timeouts of bounded device waits recorded in
// the caller-provided device word `err` (used by
// salvus_apply_stiffness_noalloc).
template <typename real>
static int apply_stiffness_into_t(const salvus_mesh *m, const real *rec, const real *u, real *a,
                                  real *scratch, int *err, cudaStream_t st) {
  int rc = launch_stiffness<real>(m, rec, u, scratch, st, err);
  if (rc) return rc;
  return by_components(m->c, [&](auto cc) {
    gather_kernel<real, decltype(cc)::value, 1><<<blocks_for(m->G, 256), 256, 0, st>>>(
        m->G, m->d_inc_off.as<int32_t>(), m->d_inc_idx.as<int32_t>(), scratch, nullptr, nullptr,
        nullptr, nullptr, a, (real)0);
    g_launches++;
    return check_launch("allocation-free gather");
  });
}

int apply_stiffness_into(const salvus_mesh *m, int precision, const void *u, void *a,
                         void *scratch, int *err, cudaStream_t st) {
  if (precision == SALVUS_FP32)
    return apply_stiffness_into_t<float>(m, m->d_rec32.as<float>(), (const float *)u, (float *)a,
                                         (float *)scratch, err, st);
  if (!m->d_rec64.ptr)
    return fail(SALVUS_E_STATE, "mesh holds no FP64 records (created with SALVUS_MESH_FP32_ONLY)");
  return apply_stiffness_into_t<double>(m, m->d_rec64.as<double>(), (const double *)u,
                                        (double *)a, (double *)scratch, err, st);
}

// Reads the device status word: set by kernels whose bounded waits ran out
// (the wait's code) or by the finite check (kNonFiniteCode).
int status_error(const salvus_problem *p, int h) {
  if (h == kNonFiniteCode)
    return fail(SALVUS_E_NONFINITE,
                "the wavefield became non-finite (NaN / Inf) by step %lld: the time step is "
                "unstable or an input field is not finite",
                (long long)p->step);
  if (h) return fail(SALVUS_E_TIMEOUT, "a bounded device wait gave up (code %d); results invalid", h);
  return SALVUS_OK;
}

static int device_status(salvus_problem *p) {
  int h = 0;
  SALVUS_CUDA(cudaMemcpyAsync(&h, p->d_err.ptr, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  return status_error(p, h);
}

int enqueue_seis_copy(salvus_problem *p, double *ring, int *status) {
  if (!p || !ring || !status) return fail(SALVUS_E_INVALID, "null argument");
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  const int64_t rows = (int64_t)p->shots * p->recs.size() * p->c;
  if (rows > 0 && p->d_seis.ptr)
    SALVUS_CUDA(cudaMemcpyAsync(ring, p->d_seis.ptr, sizeof(double) * rows * p->seis_cap,
                                cudaMemcpyDeviceToHost, p->stream));
  SALVUS_CUDA(cudaMemcpyAsync(status, p->d_err.ptr, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  return SALVUS_OK;
}

void seis_ring_shape(const salvus_problem *p, int64_t *rows, int64_t *capacity) {
  if (rows) *rows = (int64_t)p->shots * p->recs.size() * p->c;
  if (capacity) *capacity = p->seis_cap;
}

// Finite check of u (all shots) into the status word; part of every 32-step
// chunk (kFiniteEvery) of salvus_run and of the single-step entry points.
constexpr int kFiniteEvery = 32;
static int launch_finite_check(salvus_problem *p) {
  const int64_t n = p->mesh->G * p->c * p->shots_pad;
  const int64_t want = (n + 255) / 256, cap = (int64_t)p->mesh->sm_count * 8;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min(want, cap));
  if (p->prec == SALVUS_FP32)
    finite_check_kernel<float><<<grid, 256, 0, p->stream>>>(n, F<float>(p->d_u), p->d_err.as<int>());
  else
    finite_check_kernel<double><<<grid, 256, 0, p->stream>>>(n, F<double>(p->d_u), p->d_err.as<int>());
  g_launches++;
  return check_launch("finite check");
}

// Hexahedron autotuner (FP32 elastic meshes of parallelepipeds, one shot):
// times the plain step (stiffness, node gather/update) and, where the fused
// interior form is admissible, that form, each with CTAs of 128 / (N+1)^2
// elements and with twice as many, on zeroed scratch copies of u, v, a_ and
// a, and keeps the fastest.  All of them give bitwise the same wavefield
// (the same arithmetic per element and per node, in the same order), so the
// choice changes only the time.  Results are cached per (order, elements,
// nodes, anisotropy, admissible forms, device) for the process; the CTA
// width belongs to the mesh, the form to the problem.
// SALVUS_HEX_CONFIG="form,wide" fixes both; SALVUS_HEX_STEP still forces
// the form.  Without room for the scratch fields the defaults (plain, 128 /
// (N+1)^2) are kept.
static int tune_hex(salvus_problem *p) {
  if (p->hex_form >= 0) return SALVUS_OK;
  salvus_mesh *m = p->mesh;
  if (!(m->shape == SALVUS_HEX && m->affine && m->physics == SALVUS_ELASTIC3D &&
        p->prec == SALVUS_FP32 && p->shots == 1 && !m->host_only)) {
    p->hex_form = 0;
    return SALVUS_OK;
  }
  const bool fusable = hex_fusion_admissible(p) && m->order >= 2 && m->order <= 6;
  struct Key {
    int order;
    int64_t E, G;
    bool ti, fusable;
    int dev;
  };
  if (const char *env = std::getenv("SALVUS_HEX_CONFIG")) {
    int a = -1, b = -1;
    if (std::sscanf(env, "%d,%d", &a, &b) == 2 && (a == 0 || (a == 1 && fusable)) &&
        (b == 0 || b == 1)) {
      p->hex_form = a;
      m->hex_wide = b;
      return SALVUS_OK;
    }
  }
  // problems are prepared on several threads (the job server)
  static std::mutex cache_mu;
  static std::vector<std::pair<Key, std::pair<int, int>>> cache;
  {
    std::lock_guard<std::mutex> lk(cache_mu);
    for (auto &c : cache)
      if (c.first.order == m->order && c.first.E == m->E && c.first.G == m->G &&
          c.first.ti == m->ti && c.first.fusable == fusable && c.first.dev == m->device) {
        p->hex_form = c.second.first;
        m->hex_wide = c.second.second;
        return SALVUS_OK;
      }
  }
  p->hex_form = 0;
  const size_t nf = (size_t)m->G * 3 * sizeof(float);
  DeviceBuffer su, sv, sap, sa;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b < 4 * nf + (size_t(1) << 30) ||
      su.alloc(nf) || sv.alloc(nf) || sap.alloc(nf) || sa.alloc(nf)) {
    cudaGetLastError();
    return SALVUS_OK;
  }
  SALVUS_CUDA(cudaMemsetAsync(su.ptr, 0, nf, p->stream));
  SALVUS_CUDA(cudaMemsetAsync(sv.ptr, 0, nf, p->stream));
  SALVUS_CUDA(cudaMemsetAsync(sap.ptr, 0, nf, p->stream));
  SALVUS_CUDA(cudaMemsetAsync(sa.ptr, 0, nf, p->stream));
  std::swap(p->d_u.ptr, su.ptr);
  std::swap(p->d_v.ptr, sv.ptr);
  std::swap(p->d_ap.ptr, sap.ptr);
  std::swap(p->d_a.ptr, sa.ptr);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = SALVUS_OK;
  // one step of either form without sources and receivers (the same in both)
  auto sequence = [&](int form) -> int {
    int r;
    if (form == 0) {
      if ((r = launch_stiffness<float>(m, records<float>(p), F<float>(p->d_u), F<float>(p->d_r),
                                       p->stream, p->d_err.as<int>(), p->wait_limit, 0)))
        return r;
      gather_kernel<float, 3, 0><<<blocks_for(m->G, 256), 256, 0, p->stream>>>(
          m->G, m->d_inc_off.as<int32_t>(), m->d_inc_idx.as<int32_t>(), F<float>(p->d_r),
          m->d_mi32.as<float>(), F<float>(p->d_u), F<float>(p->d_v), F<float>(p->d_ap),
          F<float>(p->d_a), (float)p->dt);
    } else {
      HexInteriorUpdate iu{};
      iu.mi = m->d_mi32.as<float>();
      iu.v = F<float>(p->d_v);
      iu.ap = F<float>(p->d_ap);
      iu.dt = (float)p->dt;
      if ((r = m->ti ? launch_fused_interior<true>(p, iu) : launch_fused_interior<false>(p, iu)))
        return r;
      gather_list_kernel<float, 3, 0><<<blocks_for(m->n_gnodes, 256), 256, 0, p->stream>>>(
          m->n_gnodes, m->d_gnodes.as<int32_t>(), m->d_inc_off.as<int32_t>(),
          m->d_inc_idx.as<int32_t>(), F<float>(p->d_r), m->d_mi32.as<float>(), F<float>(p->d_u),
          F<float>(p->d_v), F<float>(p->d_ap), F<float>(p->d_a), (float)p->dt);
    }
    g_launches++;
    return check_launch("hexahedron autotuner");
  };
  float best = 1e30f;
  int bf = 0, bw = 0;
  for (int w = 0; w < 2 && rc == SALVUS_OK; ++w) {
    m->hex_wide = w;
    for (int f = 0; f < (fusable ? 2 : 1) && rc == SALVUS_OK; ++f) {
      if ((rc = sequence(f))) break;  // first launch (attributes, caches)
      float t = 1e30f;
      for (int rep = 0; rep < 3 && rc == SALVUS_OK; ++rep) {
        cudaEventRecord(e0, p->stream);
        for (int k = 0; k < 4 && rc == SALVUS_OK; ++k) rc = sequence(f);
        cudaEventRecord(e1, p->stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        t = std::min(t, ms);
      }
      if (rc == SALVUS_OK && t < best) {
        best = t;
        bf = f;
        bw = w;
      }
    }
  }
  cudaStreamSynchronize(p->stream);
  std::swap(p->d_u.ptr, su.ptr);
  std::swap(p->d_v.ptr, sv.ptr);
  std::swap(p->d_ap.ptr, sap.ptr);
  std::swap(p->d_a.ptr, sa.ptr);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  m->hex_wide = bw;
  if (rc) return rc;
  p->hex_form = bf;
  std::lock_guard<std::mutex> lk(cache_mu);
  cache.push_back({{m->order, m->E, m->G, m->ti, fusable, m->device}, {bf, bw}});
  return SALVUS_OK;
}

static int ready(salvus_problem *p) {
  if (!p) return fail(SALVUS_E_INVALID, "null problem");
  if (!p->dt_set) return fail(SALVUS_E_STATE, "time step not set (salvus_problem_set_dt)");
  int rc;
  if ((rc = upload_sources(p))) return rc;
  if ((rc = upload_receivers(p))) return rc;
  if (p->shots > 1 && (rc = autotune(p))) return rc;
  if ((rc = tune_hex(p))) return rc;
  return SALVUS_OK;
}

// ---------------------------------------------------------------------------
// problem groups: FP32 single-shot problems of one element class advance with
// one launch per stage (kernels_group.cuh)
template <int N>
static int group_stiffness_t(const salvus_mesh *m0, const GroupSlot *slots, const int32_t *owner,
                             int64_t blocks, cudaStream_t st) {
  if (m0->shape == SALVUS_QUAD) {
    group_quad_acoustic_stiffness<N><<<(unsigned)blocks, QuadColShape<N, quad_col_epb<N>()>::THREADS,
                                        0, st>>>(slots, owner, dmatrix<float>(m0->basis));
  } else if constexpr (N <= kMaxHexOrder) {
    constexpr int n2 = (N + 1) * (N + 1), EPB = 128 / n2 > 0 ? 128 / n2 : 1;
    using T = ElasticV2Shape<N, EPB, false>;
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(group_hex_elastic_stiffness<N, EPB>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
      attr = true;
    }
    group_hex_elastic_stiffness<N, EPB><<<(unsigned)blocks, T::THREADS, T::SMEM, st>>>(
        slots, owner, dmatrix<float>(m0->basis));
  }
  g_launches++;
  return check_launch("group stiffness");
}

static int group_stiffness(const salvus_mesh *m0, const GroupSlot *slots, const int32_t *owner,
                           int64_t blocks, cudaStream_t st) {
  switch (m0->order) {
    case 1: return group_stiffness_t<1>(m0, slots, owner, blocks, st);
    case 2: return group_stiffness_t<2>(m0, slots, owner, blocks, st);
    case 3: return group_stiffness_t<3>(m0, slots, owner, blocks, st);
    case 4: return group_stiffness_t<4>(m0, slots, owner, blocks, st);
    case 5: return group_stiffness_t<5>(m0, slots, owner, blocks, st);
    case 6: return group_stiffness_t<6>(m0, slots, owner, blocks, st);
    case 7: return group_stiffness_t<7>(m0, slots, owner, blocks, st);
    case 8: return group_stiffness_t<8>(m0, slots, owner, blocks, st);
    case 9: return group_stiffness_t<9>(m0, slots, owner, blocks, st);
    case 10: return group_stiffness_t<10>(m0, slots, owner, blocks, st);
  }
  return fail(SALVUS_E_UNSUPPORTED, "no grouped stiffness for order %d", m0->order);
}

// stiffness CTAs per member (the single-problem kernel's element groups)
static int64_t group_stiff_blocks(const salvus_mesh *m) {
  const int n2 = m->n * m->n;
  if (m->shape == SALVUS_QUAD) {
    const int epb = 128 / m->n > 0 ? 128 / m->n : 1;  // quad_col_epb<N>()
    return (m->E + epb - 1) / epb;
  }
  const int epb = 128 / n2 > 0 ? 128 / n2 : 1;  // v2 with 128-thread CTAs
  return (m->E + epb - 1) / epb;
}

}  // namespace salvus

struct salvus_group {
  std::vector<salvus_problem *> members;
  const salvus_mesh *m0 = nullptr;
  int c = 1;
  bool stages = true;  // one launch per stage; SALVUS_GROUP_STEP=persistent: one queue launch per step
  bool partitioned = false;  // SALVUS_GROUP_STEP=partitioned: one cooperative launch per step
  std::vector<salvus::GroupPart> parts;
  salvus::DeviceBuffer d_parts, d_bars;
  int coop_slots = 0;  // co-resident CTAs of the partitioned kernel
  std::vector<salvus::GroupSlot> slots;
  salvus::DeviceBuffer d_slots;
  // per-stage CTA -> member tables of the per-stage launches, one after the
  // other: stiffness (n_stiff), gather (n_gather), receivers (n_rec)
  std::vector<int32_t> owner;
  salvus::DeviceBuffer d_owner;
  int64_t n_stiff = 0, n_gather = 0, n_rec = 0;
  // persistent single-launch step: work-item queue
  std::vector<salvus::GroupCounts> counts;
  std::vector<salvus::GroupWork> work;
  int64_t total = 0;
  int grid = 0;
  salvus::DeviceBuffer d_counts, d_work, d_done, d_sync;
  long long wait_limit = salvus::kDefaultWaitLimit;  // bound of the device waits, SM cycles
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<cudaEvent_t> member_ev;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  int64_t sig[3] = {-1, -1, -1};
};

namespace salvus {

static int group_upload(salvus::DeviceBuffer &b, const void *src, size_t bytes, cudaStream_t st) {
  if (b.bytes < bytes) {
    int rc = b.alloc(bytes);
    if (rc) return rc;
  }
  SALVUS_CUDA(cudaMemcpyAsync(b.ptr, src, bytes, cudaMemcpyHostToDevice, st));
  return SALVUS_OK;
}

static int group_partitioned(salvus_group *g, bool launch);

static int group_fill(salvus_group *g) {
  int64_t bs = 0, bg = 0, br = 0;
  g->slots.resize(g->members.size());
  for (size_t k = 0; k < g->members.size(); ++k) {
    salvus_problem *p = g->members[k];
    const salvus_mesh *m = p->mesh;
    int rc = ready(p);
    if (rc) return rc;
    GroupSlot &s = g->slots[k];
    s.rec = m->d_rec32.as<float>();
    s.jac = m->affine ? m->d_jac32.as<float>() : nullptr;
    s.conn = m->d_conn.as<int32_t>();
    s.inc_off = m->d_inc_off.as<int32_t>();
    s.inc_idx = m->d_inc_idx.as<int32_t>();
    s.mi = m->d_mi32.as<float>();
    s.E = m->E;
    s.G = m->G;
    s.u = p->d_u.as<float>();
    s.v = p->d_v.as<float>();
    s.ap = p->d_ap.as<float>();
    s.a = p->d_a.as<float>();
    s.r = p->d_r.as<float>();
    s.dt = (float)p->dt;
    s.dtd = p->dt;
    s.step = p->d_step.as<int64_t>();
    s.nsrc = (int)p->srcs.size();
    s.nrec = (int)p->recs.size();
    s.src_elem = p->d_src_elem.as<int64_t>();
    s.src_par = p->d_src_par.as<double>();
    s.src_wts = p->d_src_wts.as<double>();
    s.rec_elem = p->d_rec_elem.as<int64_t>();
    s.rec_l = p->d_rec_l.as<double>();
    s.seis = p->d_seis.as<double>();
    s.cap = p->seis_cap;
    s.b_stiff = bs;
    s.b_gather = bg;
    s.b_rec = br;
    bs += group_stiff_blocks(m);
    bg += (m->G + 255) / 256;
    br += s.nrec;
  }
  g->n_stiff = bs;
  g->n_gather = bg;
  g->n_rec = br;
  int rc = group_upload(g->d_slots, g->slots.data(), sizeof(GroupSlot) * g->slots.size(), g->stream);
  if (rc) return rc;
  g->owner.resize((size_t)(bs + bg + br));
  {
    int32_t *o = g->owner.data();
    for (size_t k = 0; k < g->members.size(); ++k) {
      const GroupSlot &sk = g->slots[k];
      const salvus_mesh *mk = g->members[k]->mesh;
      std::fill(o + sk.b_stiff, o + sk.b_stiff + group_stiff_blocks(mk), (int32_t)k);
      std::fill(o + bs + sk.b_gather, o + bs + sk.b_gather + (mk->G + 255) / 256, (int32_t)k);
      std::fill(o + bs + bg + sk.b_rec, o + bs + bg + sk.b_rec + sk.nrec, (int32_t)k);
    }
  }
  if ((rc = group_upload(g->d_owner, g->owner.data(), sizeof(int32_t) * g->owner.size(), g->stream)))
    return rc;
  // work-item queue of the persistent step: every member's stiffness items
  // (kStiffPer element groups each), then per member source (1), gather items
  // (kGatherPer CTA-wide node tiles each), receivers (1 each), advance (1)
  constexpr int kStiffPer = 2, kGatherPer = 8;
  const int J = (int)g->members.size();
  const int tile = 128;  // CTA width of the persistent kernel
  g->counts.assign(J, GroupCounts{0, 0, 0});
  g->work.clear();
  auto add = [&](int type, int j, int64_t tiles, int per) -> int32_t {
    int32_t items = 0;
    for (int64_t f = 0; f < tiles; f += per, ++items)
      g->work.push_back(GroupWork{type, j, (int)f, (int)std::min<int64_t>(per, tiles - f)});
    return items;
  };
  for (int j = 0; j < J; ++j)
    g->counts[j].stiff = add(GI_STIFF, j, group_stiff_blocks(g->members[j]->mesh), kStiffPer);
  for (int j = 0; j < J; ++j) {
    add(GI_SRC, j, 1, 1);
    g->counts[j].gather = add(GI_GATHER, j, (g->members[j]->mesh->G + tile - 1) / tile, kGatherPer);
    g->counts[j].rec = add(GI_REC, j, (int64_t)g->members[j]->recs.size(), 1);
    add(GI_ADV, j, 1, 1);
  }
  g->total = (int64_t)g->work.size();
  if ((rc = group_upload(g->d_counts, g->counts.data(), sizeof(GroupCounts) * J, g->stream))) return rc;
  if ((rc = group_upload(g->d_work, g->work.data(), sizeof(GroupWork) * g->work.size(), g->stream)))
    return rc;
  if (g->d_done.bytes < sizeof(int32_t) * 4 * J) {
    if ((rc = g->d_done.alloc(sizeof(int32_t) * 4 * J))) return rc;
    SALVUS_CUDA(cudaMemsetAsync(g->d_done.ptr, 0, sizeof(int32_t) * 4 * J, g->stream));
  }
  if (!g->d_sync.ptr) {
    if ((rc = g->d_sync.alloc(sizeof(GroupSync)))) return rc;
    SALVUS_CUDA(cudaMemsetAsync(g->d_sync.ptr, 0, sizeof(GroupSync), g->stream));
  }
  // the partitioned step's CTA ranges and counters (allocated here, before any capture)
  if (g->partitioned) return group_partitioned(g, false);
  return SALVUS_OK;
}

template <int N, bool kHex, int C>
static int group_persistent_t(salvus_group *g) {
  constexpr int threads = 128;
  size_t smem = 0;
  if constexpr (kHex) {
    constexpr int n2 = (N + 1) * (N + 1), EPB = 128 / n2 > 0 ? 128 / n2 : 1;
    smem = ElasticV2Shape<N, EPB, false>::SMEM;
  }
  auto kern = group_persistent_step<N, kHex, C>;
  if (g->grid == 0) {
    if (smem) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    SALVUS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    g->grid = (per_sm > 0 ? per_sm : 1) * g->m0->sm_count;
  }
  const int grid = (int)std::min<int64_t>(g->grid, g->total);
  kern<<<grid, threads, smem, g->stream>>>(
      g->d_slots.as<GroupSlot>(), g->d_counts.as<GroupCounts>(), (int)g->members.size(),
      g->d_work.as<GroupWork>(), g->total, g->d_done.as<int32_t>(), g->d_sync.as<GroupSync>(),
      dmatrix<float>(g->m0->basis), g->m0->P, g->wait_limit);
  g_launches++;
  return check_launch("group persistent step");
}

static int group_persistent(salvus_group *g) {
  const salvus_mesh *m = g->m0;
  if (m->shape == SALVUS_HEX) {
    switch (m->order) {
      case 1: return group_persistent_t<1, true, 3>(g);
      case 2: return group_persistent_t<2, true, 3>(g);
      case 3: return group_persistent_t<3, true, 3>(g);
      case 4: return group_persistent_t<4, true, 3>(g);
      case 5: return group_persistent_t<5, true, 3>(g);
      case 6: return group_persistent_t<6, true, 3>(g);
    }
  } else {
    switch (m->order) {
      case 1: return group_persistent_t<1, false, 1>(g);
      case 2: return group_persistent_t<2, false, 1>(g);
      case 3: return group_persistent_t<3, false, 1>(g);
      case 4: return group_persistent_t<4, false, 1>(g);
      case 5: return group_persistent_t<5, false, 1>(g);
      case 6: return group_persistent_t<6, false, 1>(g);
      case 7: return group_persistent_t<7, false, 1>(g);
      case 8: return group_persistent_t<8, false, 1>(g);
      case 9: return group_persistent_t<9, false, 1>(g);
      case 10: return group_persistent_t<10, false, 1>(g);
    }
  }
  return fail(SALVUS_E_UNSUPPORTED, "no grouped step for order %d", m->order);
}

// launch=false: size the member CTA ranges (once) and allocate their counters;
// launch=true: one cooperative launch of the step
template <int N, bool kHex, int C>
static int group_partitioned_t(salvus_group *g, bool launch) {
  constexpr int threads = 128;
  size_t smem = 0;
  if constexpr (kHex) {
    constexpr int n2 = (N + 1) * (N + 1), EPB = 128 / n2 > 0 ? 128 / n2 : 1;
    smem = ElasticV2Shape<N, EPB, false>::SMEM;
  }
  auto kern = group_partitioned_step<N, kHex, C>;
  const int J = (int)g->members.size();
  if (!launch) {
    if (g->coop_slots == 0) {
      if (smem) SALVUS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      int per_sm = 0;
      SALVUS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
      g->coop_slots = (per_sm > 0 ? per_sm : 1) * g->m0->sm_count;
    }
    if (g->parts.size() == (size_t)J) return SALVUS_OK;
    // CTAs per member in proportion to its work (element points + nodes), at least one
    if (J > g->coop_slots)
      return fail(SALVUS_E_UNSUPPORTED, "%d members exceed the %d co-resident CTAs", J, g->coop_slots);
    const int tile = 128;
    std::vector<double> w(J);
    double wsum = 0;
    for (int j = 0; j < J; ++j) {
      const salvus_mesh *m = g->members[j]->mesh;
      w[j] = (double)m->E * m->P + (double)m->G;
      wsum += w[j];
    }
    std::vector<GroupPart> parts(J);
    const int spare = g->coop_slots - J;
    int first = 0;
    for (int j = 0; j < J; ++j) {
      const salvus_mesh *m = g->members[j]->mesh;
      GroupPart &pt = parts[j];
      pt.cta_first = first;
      pt.cta_count = 1 + (int)std::floor((double)spare * w[j] / wsum);
      pt.n_stiff = (int32_t)group_stiff_blocks(m);
      pt.n_gather = (int32_t)((m->G + tile - 1) / tile);
      first += pt.cta_count;
    }
    int rc = group_upload(g->d_parts, parts.data(), sizeof(GroupPart) * J, g->stream);
    if (rc) return rc;
    if ((rc = g->d_bars.alloc(sizeof(GroupBar) * J))) return rc;
    SALVUS_CUDA(cudaMemsetAsync(g->d_bars.ptr, 0, sizeof(GroupBar) * J, g->stream));
    g->parts = std::move(parts);
    return SALVUS_OK;
  }
  if (g->parts.size() != (size_t)J) return fail(SALVUS_E_INVALID, "partitioned group not set up");
  const int grid = g->parts.back().cta_first + g->parts.back().cta_count;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = g->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  SALVUS_CUDA(cudaLaunchKernelEx(&cfg, kern, (const GroupSlot *)g->d_slots.as<GroupSlot>(),
                                 (const GroupPart *)g->d_parts.as<GroupPart>(), J,
                                 g->d_bars.as<GroupBar>(), g->d_sync.as<GroupSync>(),
                                 dmatrix<float>(g->m0->basis), g->m0->P,
                                 (long long)g->wait_limit));
  g_launches++;
  return check_launch("group partitioned step");
}

static int group_partitioned(salvus_group *g, bool launch) {
  const salvus_mesh *m = g->m0;
  if (m->shape == SALVUS_HEX) {
    switch (m->order) {
      case 1: return group_partitioned_t<1, true, 3>(g, launch);
      case 2: return group_partitioned_t<2, true, 3>(g, launch);
      case 3: return group_partitioned_t<3, true, 3>(g, launch);
      case 4: return group_partitioned_t<4, true, 3>(g, launch);
      case 5: return group_partitioned_t<5, true, 3>(g, launch);
      case 6: return group_partitioned_t<6, true, 3>(g, launch);
    }
  } else {
    switch (m->order) {
      case 1: return group_partitioned_t<1, false, 1>(g, launch);
      case 2: return group_partitioned_t<2, false, 1>(g, launch);
      case 3: return group_partitioned_t<3, false, 1>(g, launch);
      case 4: return group_partitioned_t<4, false, 1>(g, launch);
      case 5: return group_partitioned_t<5, false, 1>(g, launch);
      case 6: return group_partitioned_t<6, false, 1>(g, launch);
      case 7: return group_partitioned_t<7, false, 1>(g, launch);
      case 8: return group_partitioned_t<8, false, 1>(g, launch);
      case 9: return group_partitioned_t<9, false, 1>(g, launch);
      case 10: return group_partitioned_t<10, false, 1>(g, launch);
    }
  }
  return fail(SALVUS_E_UNSUPPORTED, "no grouped step for order %d", m->order);
}

static int group_step(salvus_group *g) {
  if (g->partitioned) return group_partitioned(g, true);
  if (!g->stages) return group_persistent(g);
  const int J = (int)g->members.size();
  const int P = g->m0->P;
  const GroupSlot *slots = g->d_slots.as<GroupSlot>();
  int rc;
  const int32_t *own = g->d_owner.as<int32_t>();
  if ((rc = group_stiffness(g->m0, slots, own, g->n_stiff, g->stream))) return rc;
  if (g->c == 1) group_source<1><<<J, 256, 0, g->stream>>>(slots, P);
  else group_source<3><<<J, 256, 0, g->stream>>>(slots, P);
  if (g->c == 1) group_gather_update<1><<<(unsigned)g->n_gather, 256, 0, g->stream>>>(slots, own + g->n_stiff);
  else group_gather_update<3><<<(unsigned)g->n_gather, 256, 0, g->stream>>>(slots, own + g->n_stiff);
  if (g->n_rec > 0) {
    const int32_t *own_rec = own + g->n_stiff + g->n_gather;
    if (g->c == 1) group_receivers<1><<<(unsigned)g->n_rec, kRecThreads, 0, g->stream>>>(slots, own_rec, P);
    else group_receivers<3><<<(unsigned)g->n_rec, kRecThreads, 0, g->stream>>>(slots, own_rec, P);
  }
  group_advance<<<1, 256, 0, g->stream>>>(slots, J);
  g_launches += g->n_rec > 0 ? 4 : 3;
  return check_launch("group step");
}

}  // namespace salvus

using namespace salvus;

// ===========================================================================
extern "C" {

const char *salvus_last_error(void) { return salvus::last_error(); }

const char *salvus_version(void) {
  return "salvus_b200 0.1 (sm_100a; FP32/FP64 tensor-product SEM; deterministic gather assembly)";
}

int64_t salvus_launch_count(void) { return g_launches.load(); }

int salvus_element_tables(int32_t shape, int32_t order, int32_t *n_points, double *points,
                          double *weights, double *dphi) {
  Basis b;
  int rc = make_basis(shape, order, &b);
  if (rc) return rc;
  const int P = b.P, dim = b.dim;
  if (n_points) *n_points = P;
  std::vector<double> phi(P), dp((size_t)P * 3);
  for (int q = 0; q < P; ++q) {
    double ref[3];
    point_ref(b, q, ref);
    if (points)
      for (int a = 0; a < dim; ++a) points[(size_t)q * dim + a] = ref[a];
    if (weights) weights[q] = point_weight(b, q);
    if (dphi) {
      if (b.simplex) {
        for (int k = 0; k < dim; ++k)
          for (int i = 0; i < P; ++i) dphi[((size_t)k * P + i) * P + q] = b.SD[((size_t)k * P + i) * P + q];
      } else {
        basis_at(b, ref, phi.data(), dp.data());
        for (int k = 0; k < dim; ++k)
          for (int i = 0; i < P; ++i) dphi[((size_t)k * P + i) * P + q] = dp[(size_t)i * 3 + k];
      }
    }
  }
  return SALVUS_OK;
}

int salvus_mesh_create(const salvus_mesh_desc *d, int device, salvus_mesh **out) {
  if (!d || !out) return fail(SALVUS_E_INVALID, "null argument");
  *out = nullptr;
  if (d->shape < SALVUS_QUAD || d->shape > SALVUS_TET)
    return fail(SALVUS_E_UNSUPPORTED, "unknown element shape %d", d->shape);
  if (d->physics == SALVUS_ELASTIC3D && d->shape != SALVUS_HEX && d->shape != SALVUS_TET)
    return fail(SALVUS_E_UNSUPPORTED, "elastic 3-D physics needs hexahedra or tetrahedra");
  if ((d->physics == SALVUS_ELASTIC2D || d->physics == SALVUS_COUPLED2D) && d->shape != SALVUS_QUAD)
    return fail(SALVUS_E_UNSUPPORTED, "elastic 2-D and coupled physics need quadrilaterals");
  if (d->physics < SALVUS_ACOUSTIC || d->physics > SALVUS_COUPLED2D)
    return fail(SALVUS_E_INVALID, "unknown physics %d", d->physics);
  if (d->n_elements <= 0 || d->n_vertices <= 0 || !d->vertices || !d->cells || !d->params)
    return fail(SALVUS_E_INVALID, "empty mesh");
  std::unique_ptr<salvus_mesh> m(new salvus_mesh());
  m->device = device;
  m->fp32_only = (d->reserved & SALVUS_MESH_FP32_ONLY) != 0;
  {
    // FP32 tetrahedra: tensor cores by default; SALVUS_TET_KERNEL=cuda selects
    // the CUDA-core kernel (read when the mesh is created)
    const char *s = std::getenv("SALVUS_TET_KERNEL");
    m->tet_kernel = (s && std::strcmp(s, "cuda") == 0) ? 1 : 0;
    // triangles: CUDA cores with the derivative table in constant memory by
    // default; SALVUS_TRI_KERNEL=tc selects the tensor-core kernel (FP32),
    // =shared the shared-memory-table kernel (read when the mesh is created)
    const char *t = std::getenv("SALVUS_TRI_KERNEL");
    m->tri_kernel = (t && std::strcmp(t, "tc") == 0) ? 0 : (t && std::strcmp(t, "shared") == 0) ? 2 : 1;
  }
  m->shape = d->shape;
  m->order = d->order;
  m->physics = d->physics;
  int rc = make_basis(d->shape, d->order, &m->basis);
  if (rc) return rc;
  m->dim = m->basis.dim;
  m->nv = m->basis.nv;
  m->n = m->basis.n;
  m->P = m->basis.P;
  m->c = physics_components(d->physics);
  m->npar = physics_params(d->physics, d->reserved);
  m->E = d->n_elements;
  m->vtx.resize((size_t)(m->E * m->nv * m->dim));
  for (int64_t e = 0; e < m->E; ++e)
    for (int k = 0; k < m->nv; ++k) {
      int64_t vi = d->cells[e * m->nv + k];
      if (vi < 0 || vi >= d->n_vertices)
        return fail(SALVUS_E_INVALID, "element %lld references vertex %lld out of range",
                    (long long)e, (long long)vi);
      for (int a = 0; a < m->dim; ++a)
        m->vtx[(size_t)((e * m->nv + k) * m->dim + a)] = d->vertices[vi * m->dim + a];
    }
  for (int64_t e = 0; e < m->E; ++e) {
    // right-hand rule check (QuadP1::checkHull / HexP1::checkHull): detJ > 0
    // at every corner (simplices: the constant detJ)
    const double *v = m->vtx.data() + e * m->nv * m->dim;
    const int ncheck = is_simplex(m->shape) ? 1 : (m->dim == 2 ? 4 : 8);
    for (int q = 0; q < ncheck; ++q) {
      double ref[3] = {0, 0, 0};
      if (!is_simplex(m->shape))
        for (int a = 0; a < m->dim; ++a) ref[a] = ((q >> a) & 1) ? 1.0 : -1.0;
      double det;
      p1_jacobian(m->shape, v, ref, &det, nullptr);
      if (!(det > 0))
        return fail(SALVUS_E_INVALID, "element %lld is inverted or degenerate (detJ <= 0)",
                    (long long)e);
    }
  }
  const size_t npar_total = (size_t)m->npar * m->E * m->nv;
  m->par.assign(d->params, d->params + npar_total);
  for (size_t i = 0; i < npar_total; ++i)
    if (!std::isfinite(m->par[i])) return fail(SALVUS_E_INVALID, "non-finite material parameter");
  if (m->npar == 6) {
    // RHO VPV VPH VSV VSH ETA (Elastic3D.cpp:33-54).  An isotropic model
    // (VPH = VPV, VSH = VSV, ETA = 1 everywhere) keeps the two-constant
    // records and kernels; anything else gets the five-constant ones.
    const size_t K = (size_t)m->E * m->nv;
    const double *pr = m->par.data();
    bool iso = true;
    for (size_t i = 0; i < K && iso; ++i)
      iso = pr[2 * K + i] == pr[K + i] && pr[4 * K + i] == pr[3 * K + i] && pr[5 * K + i] == 1.0;
    if (iso) {
      std::vector<double> p3(3 * K);
      std::copy(pr, pr + K, p3.begin());                    // RHO
      std::copy(pr + K, pr + 2 * K, p3.begin() + K);        // VP = VPV
      std::copy(pr + 3 * K, pr + 4 * K, p3.begin() + 2 * K);  // VS = VSV
      m->par.swap(p3);
      m->npar = 3;
    } else {
      m->ti = true;
      m->tet_kernel = 1;  // tetrahedra: the CUDA-core kernel has the five-constant stress
    }
  }
  if (m->shape == SALVUS_HEX && m->physics == SALVUS_ELASTIC3D &&
      !(d->reserved & SALVUS_MESH_PER_POINT_GEOMETRY)) {
    // every element a parallelepiped: the inverse Jacobian at the eight
    // corners equals the one at the centre (to 1e-12 relative)
    bool affine = true;
    for (int64_t e = 0; e < m->E && affine; ++e) {
      const double *v = m->vtx.data() + e * 24;
      double c0[3] = {0, 0, 0}, det0, J0[9];
      p1_jacobian(m->shape, v, c0, &det0, J0);
      double scale = 0;
      for (int a = 0; a < 9; ++a) scale = std::max(scale, std::fabs(J0[a]));
      for (int q = 0; q < 8 && affine; ++q) {
        double ref[3], det, J[9];
        for (int a = 0; a < 3; ++a) ref[a] = ((q >> a) & 1) ? 1.0 : -1.0;
        p1_jacobian(m->shape, v, ref, &det, J);
        for (int a = 0; a < 9; ++a)
          if (std::fabs(J[a] - J0[a]) > 1e-12 * scale) affine = false;
      }
    }
    m->affine = affine;
  }
  if ((rc = flatten_mesh(m.get(), d->cells, d->n_vertices))) return rc;
  if (m->physics == SALVUS_COUPLED2D && (rc = setup_coupled(m.get(), d->cells))) return rc;
  interior_free_nodes(m.get());
  if (device >= 0) {
    if ((rc = mesh_setup_device(m.get()))) return rc;
  } else {
    m->host_only = true;  // numbering and coordinates only; no GPU residency
  }
  *out = m.release();
  return SALVUS_OK;
}

int salvus_mesh_destroy(salvus_mesh *m) {
  if (!m) return SALVUS_OK;
  if (m->host_only) {
    delete m;
    return SALVUS_OK;
  }
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaStream_t s = m->stream;
  delete m;
  if (s) cudaStreamDestroy(s);
  return SALVUS_OK;
}

int salvus_mesh_info(const salvus_mesh *m, int64_t *G, int32_t *c, int32_t *P) {
  if (!m) return fail(SALVUS_E_INVALID, "null mesh");
  if (G) *G = m->G;
  if (c) *c = m->c;
  if (P) *P = m->P;
  return SALVUS_OK;
}

int salvus_mesh_layout(const salvus_mesh *m, int32_t *per_element_jacobian,
                       int64_t *gathered_nodes) {
  if (!m) return fail(SALVUS_E_INVALID, "null mesh");
  if (per_element_jacobian) *per_element_jacobian = m->affine ? 1 : 0;
  if (gathered_nodes) *gathered_nodes = m->n_gnodes > 0 ? m->n_gnodes : m->G;
  return SALVUS_OK;
}

int salvus_mesh_node_coords(const salvus_mesh *m, double *xyz) {
  if (!m || !xyz) return fail(SALVUS_E_INVALID, "null argument");
  std::memcpy(xyz, m->xyz.data(), sizeof(double) * m->xyz.size());
  return SALVUS_OK;
}

int salvus_mesh_connectivity(const salvus_mesh *m, int64_t *conn) {
  if (!m || !conn) return fail(SALVUS_E_INVALID, "null argument");
  for (size_t i = 0; i < m->conn.size(); ++i) conn[i] = m->conn[i];
  return SALVUS_OK;
}

int salvus_mesh_locate_point(const salvus_mesh *m, const double *xyz, int64_t *elem, double *ref) {
  if (!m || !xyz || !elem || !ref) return fail(SALVUS_E_INVALID, "null argument");
  double x[3] = {xyz[0], xyz[1], m->dim == 3 ? xyz[2] : 0.0}, r[3] = {0, 0, 0};
  int rc = locate_point(m, x, elem, r);
  if (rc) return rc;
  for (int a = 0; a < m->dim; ++a) ref[a] = r[a];
  return SALVUS_OK;
}

int salvus_mesh_inverse_mass(const salvus_mesh *m, double *mi) {
  if (!m || !mi) return fail(SALVUS_E_INVALID, "null argument");
  if (m->host_only) return fail(SALVUS_E_STATE, "host-only mesh has no mass matrix");
  std::memcpy(mi, m->mi.data(), sizeof(double) * m->G);
  return SALVUS_OK;
}

int salvus_mesh_max_eigenvalue(salvus_mesh *m, int32_t iters, uint64_t seed, double *lam_out) {
  if (!m || !lam_out) return fail(SALVUS_E_INVALID, "null argument");
  if (m->host_only) return fail(SALVUS_E_STATE, "host-only mesh");
  if (m->fp32_only) return fail(SALVUS_E_STATE, "the eigenvalue estimate needs the FP64 records");
  SALVUS_CUDA(cudaSetDevice(m->device));
  const int64_t N = m->G * m->c;
  DeviceBuffer x, y, r, mass, part;
  int rc;
  if ((rc = x.alloc(8 * N)) || (rc = y.alloc(8 * N)) || (rc = r.alloc(8 * m->E * m->P * m->c)) ||
      (rc = mass.alloc(8 * m->G)) || (rc = part.alloc(8 * 1024)))
    return rc;
  std::vector<double> h(N), mh(m->G);
  std::mt19937_64 rng(seed ? seed : 1);
  std::uniform_real_distribution<double> U(-0.5, 0.5);
  for (auto &v : h) v = U(rng);
  for (int64_t g = 0; g < m->G; ++g) mh[g] = 1.0 / m->mi[g];
  SALVUS_CUDA(cudaMemcpyAsync(x.ptr, h.data(), 8 * N, cudaMemcpyHostToDevice, m->stream));
  SALVUS_CUDA(cudaMemcpyAsync(mass.ptr, mh.data(), 8 * m->G, cudaMemcpyHostToDevice, m->stream));
  const int nb = 512;
  std::vector<double> hp(nb);
  auto dot = [&](const double *a, const double *b, double &out) -> int {
    dot_kernel<double><<<nb, 256, 0, m->stream>>>(N, m->c, a, b, mass.as<double>(), part.as<double>());
    g_launches++;
    SALVUS_CUDA(cudaMemcpyAsync(hp.data(), part.ptr, 8 * nb, cudaMemcpyDeviceToHost, m->stream));
    SALVUS_CUDA(cudaStreamSynchronize(m->stream));
    double s = 0;
    for (int i = 0; i < nb; ++i) s += hp[i];
    out = s;
    return SALVUS_OK;
  };
  double lam = 0;
  for (int it = 0; it < iters; ++it) {
    if ((rc = launch_stiffness<double>(m, m->d_rec64.as<double>(), x.as<double>(), r.as<double>(),
                                       m->stream)))
      return rc;
    // y = -gather(r) = K x ; then M^-1
    by_components(m->c, [&](auto cc) {
      constexpr int C = decltype(cc)::value;
      gather_kernel<double, C, 1><<<blocks_for(m->G, 256), 256, 0, m->stream>>>(
          m->G, m->d_inc_off.as<int32_t>(), m->d_inc_idx.as<int32_t>(), r.as<double>(), nullptr,
          nullptr, nullptr, nullptr, y.as<double>(), 0.0);
      inverse_mass_kernel<double, C><<<blocks_for(N, 256), 256, 0, m->stream>>>(
          m->G, m->d_mi64.as<double>(), y.as<double>());
      return SALVUS_OK;
    });
    g_launches += 2;
    scale_kernel<double><<<blocks_for(N, 256), 256, 0, m->stream>>>(N, y.as<double>(), -1.0);
    g_launches++;
    double xy, xx, yy;
    if ((rc = dot(x.as<double>(), y.as<double>(), xy)) || (rc = dot(x.as<double>(), x.as<double>(), xx)) ||
        (rc = dot(y.as<double>(), y.as<double>(), yy)))
      return rc;
    lam = xy / xx;
    std::swap(x.ptr, y.ptr);
    scale_kernel<double><<<blocks_for(N, 256), 256, 0, m->stream>>>(N, x.as<double>(),
                                                                     1.0 / std::sqrt(yy));
    g_launches++;
  }
  SALVUS_CUDA(cudaStreamSynchronize(m->stream));
  *lam_out = lam;
  return SALVUS_OK;
}

int salvus_problem_create(salvus_mesh *m, int32_t precision, int32_t n_shots, salvus_problem **out) {
  if (!m || !out) return fail(SALVUS_E_INVALID, "null argument");
  *out = nullptr;
  if (m->host_only) return fail(SALVUS_E_STATE, "mesh was created host-only (device < 0)");
  if (precision != SALVUS_FP32 && precision != SALVUS_FP64)
    return fail(SALVUS_E_INVALID, "unknown precision %d", precision);
  if (n_shots < 1) return fail(SALVUS_E_INVALID, "n_shots must be >= 1");
  if (precision == SALVUS_FP64 && m->fp32_only)
    return fail(SALVUS_E_STATE, "mesh was created with SALVUS_MESH_FP32_ONLY");
  if (n_shots > 1 && (precision != SALVUS_FP32 || m->shape != SALVUS_QUAD ||
                      m->physics != SALVUS_ACOUSTIC || m->order > 6))
    return fail(SALVUS_E_UNSUPPORTED,
                "shot batching is built for FP32 acoustic quads of order 1..6 (got shape %d, "
                "order %d, precision %d)", m->shape, m->order, precision);
  SALVUS_CUDA(cudaSetDevice(m->device));
  std::unique_ptr<salvus_problem> p(new salvus_problem());
  p->mesh = m;
  p->device = m->device;
  p->prec = precision;
  p->shots = n_shots;
  p->shots_pad = n_shots == 1 ? 1 : (n_shots + 31) / 32 * 32;
  p->c = m->c;
  p->rsize = precision == SALVUS_FP32 ? 4 : 8;
  SALVUS_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  const size_t nf = (size_t)m->G * p->c * p->rsize * p->shots_pad;
  const size_t na = n_shots == 1 ? nf : 16;  // batched problems keep no a / a_ fields
  int rc;
  if ((rc = p->d_u.alloc(nf)) || (rc = p->d_v.alloc(nf)) || (rc = p->d_a.alloc(na)) ||
      (rc = p->d_ap.alloc(na)) ||
      (rc = p->d_r.alloc((size_t)m->E * m->P * p->c * p->rsize * p->shots_pad)) ||
      (rc = p->d_step.alloc(sizeof(int64_t))) || (rc = p->d_err.alloc(sizeof(int))))
    return rc;
  SALVUS_CUDA(cudaMemsetAsync(p->d_err.ptr, 0, sizeof(int), p->stream));
  SALVUS_CUDA(cudaMemsetAsync(p->d_u.ptr, 0, nf, p->stream));
  SALVUS_CUDA(cudaMemsetAsync(p->d_v.ptr, 0, nf, p->stream));
  SALVUS_CUDA(cudaMemsetAsync(p->d_a.ptr, 0, na, p->stream));
  SALVUS_CUDA(cudaMemsetAsync(p->d_ap.ptr, 0, na, p->stream));
  SALVUS_CUDA(cudaMemsetAsync(p->d_step.ptr, 0, sizeof(int64_t), p->stream));
  SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  p->prof_ms.assign(K_NKINDS, 0.0);
  p->prof_n.assign(K_NKINDS, 0);
  *out = p.release();
  return SALVUS_OK;
}

int salvus_problem_destroy(salvus_problem *p) {
  if (!p) return SALVUS_OK;
  // the problem's own device: its mesh may already be gone
  cudaSetDevice(p->device);
  cudaStreamSynchronize(p->stream);
  drop_graph(p);
  for (auto &e : p->events) {
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  for (int b = 0; b < 2; ++b) {
    if (p->h_pin[b]) cudaFreeHost(p->h_pin[b]);
    if (p->pin_ev[b]) cudaEventDestroy(p->pin_ev[b]);
  }
  if (p->rec_stream) {
    cudaStreamSynchronize(p->rec_stream);
    cudaStreamDestroy(p->rec_stream);
    cudaEventDestroy(p->ev_updated);
    cudaEventDestroy(p->ev_recorded);
  }
  cudaStream_t s = p->stream;
  delete p;
  if (s) cudaStreamDestroy(s);
  return SALVUS_OK;
}

int salvus_problem_set_dt(salvus_problem *p, double dt) {
  if (!p) return fail(SALVUS_E_INVALID, "null problem");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(SALVUS_E_INVALID, "dt must be positive");
  if (p->dt != dt) drop_graph(p);
  p->dt = dt;
  p->dt_set = true;
  return SALVUS_OK;
}

int salvus_problem_add_source(salvus_problem *p, const salvus_source *s) {
  if (!p || !s) return fail(SALVUS_E_INVALID, "null argument");
  const salvus_mesh *m = p->mesh;
  if (s->shot < 0 || s->shot >= p->shots)
    return fail(SALVUS_E_INVALID, "shot index %d out of range", s->shot);
  if (s->kind == SALVUS_SOURCE_MOMENT_TENSOR && m->physics == SALVUS_ACOUSTIC)
    return fail(SALVUS_E_INVALID, "moment-tensor sources need elastic physics");
  if (s->kind != SALVUS_SOURCE_FORCE && s->kind != SALVUS_SOURCE_MOMENT_TENSOR)
    return fail(SALVUS_E_INVALID, "unknown source kind %d", s->kind);
  salvus_problem::Src src;
  src.desc = *s;
  int rc = locate_point(m, s->location, &src.elem, src.ref);
  if (rc) return rc;
  const int P = m->P, c = p->c;
  // components the owning element pushes: all, or on meshes of fluid and
  // solid elements u (fluid) / ux, uy (solid)
  int k0 = 0, k1 = c;
  if (m->physics == SALVUS_COUPLED2D) {
    const bool fl = m->par[(size_t)src.elem * 4] == 1.0;
    k0 = fl ? 0 : 1;
    k1 = fl ? 1 : 3;
    if (fl && s->kind == SALVUS_SOURCE_MOMENT_TENSOR)
      return fail(SALVUS_E_INVALID, "moment-tensor source inside a fluid element");
  }
  // delta-function coefficients phi_q(x_s) / (w_q detJ_q), times w_q detJ_q
  // by applyTestAndIntegrate (Scalar.cpp:87): phi_q(x_s) per unit force
  std::vector<double> phi(P), dphi((size_t)P * 3);
  basis_at(m->basis, src.ref, phi.data(), dphi.data());
  src.wts.assign((size_t)P * c, 0.0);
  if (s->kind == SALVUS_SOURCE_FORCE) {
    for (int q = 0; q < P; ++q)
      for (int a = k0; a < k1; ++a) src.wts[(size_t)q * c + a] = phi[q] * s->comp[a];
  } else {
    // 3-D comp = [Mxx Myy Mzz Myz Mxz Mxy]; 2-D comp = [Mxx Myy Mxy]
    const int d = m->dim;
    double det, iJ[9];
    p1_jacobian(m->shape, m->vtx.data() + src.elem * m->nv * d, src.ref, &det, iJ);
    double M[3][3] = {{s->comp[0], s->comp[5], s->comp[4]},
                      {s->comp[5], s->comp[1], s->comp[3]},
                      {s->comp[4], s->comp[3], s->comp[2]}};
    if (d == 2) {
      M[0][0] = s->comp[0];
      M[1][1] = s->comp[1];
      M[0][1] = M[1][0] = s->comp[2];
    }
    for (int q = 0; q < P; ++q) {
      const double *gref = &dphi[(size_t)q * 3];
      double gx[3] = {0, 0, 0};
      for (int a = 0; a < d; ++a)
        for (int k = 0; k < d; ++k) gx[a] += iJ[a * d + k] * gref[k];
      for (int a = 0; a < d; ++a) {
        double f = 0;
        for (int k = 0; k < d; ++k) f += M[a][k] * gx[k];
        src.wts[(size_t)q * c + k0 + a] = f;
      }
    }
  }
  p->srcs.push_back(std::move(src));
  p->src_dirty = true;
  drop_graph(p);
  return SALVUS_OK;
}

int salvus_problem_add_receiver(salvus_problem *p, const double *xyz) {
  if (!p || !xyz) return fail(SALVUS_E_INVALID, "null argument");
  const salvus_mesh *m = p->mesh;
  salvus_problem::Rec r;
  for (int a = 0; a < 3; ++a) r.xyz[a] = a < m->dim ? xyz[a] : 0.0;
  int rc = locate_point(m, r.xyz, &r.elem, r.ref);
  if (rc) return rc;
  r.l.resize(m->P);
  basis_at(m->basis, r.ref, r.l.data(), nullptr);
  p->recs.push_back(std::move(r));
  p->rec_dirty = true;
  drop_graph(p);
  return SALVUS_OK;
}

int salvus_problem_set_seismogram_capacity(salvus_problem *p, int64_t steps) {
  if (!p || steps <= 0) return fail(SALVUS_E_INVALID, "bad capacity");
  p->seis_cap = steps;
  p->rec_dirty = true;
  drop_graph(p);
  return SALVUS_OK;
}

// Host <-> device copies of whole fields through two pinned bounce chunks:
// the host copy into (out of) one chunk overlaps the DMA of the other, which
// runs at pinned-memory speed instead of the staged pageable path.  Small
// copies go directly.
static constexpr size_t kPinChunk = size_t(32) << 20;
// Host work on one chunk, split over the host threads (one thread's memcpy
// or conversion is slower than the DMA it feeds): fn(lo, hi) on [0, n).
static int host_threads() {
  static const int n = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
  return n;
}
// Persistent host workers for those copies: a field of the 64^3 workload
// is 13 chunks, and creating and joining a fresh set of threads for every
// chunk cost about as much as the conversion itself.  One parallel job runs
// at a time (callers serialise on run_mu); the calling thread takes part 0.
// The pool is created on first use and never destroyed (its threads are
// detached and end with the process); a process forked after that has no
// workers, so it runs the parts itself.
extern "C++" {
class HostPool {
 public:
  static HostPool &get() {
    static HostPool *pool = new HostPool(host_threads());
    return *pool;
  }
  int threads() const { return T_; }
  void run(size_t n, size_t part, const std::function<void(size_t, size_t)> &fn) {
    if (getpid() != pid_ || T_ == 1) {
      for (size_t lo = 0; lo < n; lo += part) fn(lo, std::min(n, lo + part));
      return;
    }
    std::lock_guard<std::mutex> rl(run_mu_);
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      n_ = n;
      part_ = part;
      remaining_ = T_ - 1;
      ++gen_;
    }
    cv_work_.notify_all();
    fn(0, std::min(part, n));
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [&] { return remaining_ == 0; });
    fn_ = nullptr;
  }

 private:
  explicit HostPool(int T) : T_(T), pid_(getpid()) {
    for (int t = 1; t < T_; ++t) std::thread([this, t] { loop(t); }).detach();
  }
  void loop(int t) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(size_t, size_t)> *fn;
      size_t lo, hi;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_work_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        fn = fn_;
        lo = std::min(n_, (size_t)t * part_);
        hi = std::min(n_, lo + part_);
      }
      if (lo < hi) (*fn)(lo, hi);
      std::lock_guard<std::mutex> lk(mu_);
      if (--remaining_ == 0) cv_done_.notify_one();
    }
  }
  const int T_;
  const pid_t pid_;
  std::mutex run_mu_, mu_;
  std::condition_variable cv_work_, cv_done_;
  const std::function<void(size_t, size_t)> *fn_ = nullptr;
  size_t n_ = 0, part_ = 0;
  uint64_t gen_ = 0;
  int remaining_ = 0;
};

template <typename Fn>
static void par_range(size_t n, Fn fn) {
  HostPool &pool = HostPool::get();
  const int T = pool.threads();
  const size_t part = ((n + T - 1) / T + 63) & ~size_t(63);
  const std::function<void(size_t, size_t)> f = fn;
  pool.run(n, part, f);
}
}  // extern "C++"
static void par_memcpy(void *dst, const void *src, size_t n) {
  par_range(n, [=](size_t lo, size_t hi) {
    std::memcpy((char *)dst + lo, (const char *)src + lo, hi - lo);
  });
}
// FP64 -> FP32 with round-to-nearest-even, the rounding of the device's
// conversion (cvt.rn.f32.f64), so both give the same bits.
static void par_convert(float *dst, const double *src, size_t n) {
  par_range(n, [=](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) dst[i] = (float)src[i];
  });
}
static int pin_ready(salvus_problem *p) {
  for (int b = 0; b < 2; ++b) {
    if (!p->h_pin[b]) SALVUS_CUDA(cudaMallocHost(&p->h_pin[b], kPinChunk));
    if (!p->pin_ev[b]) SALVUS_CUDA(cudaEventCreateWithFlags(&p->pin_ev[b], cudaEventDisableTiming));
  }
  return SALVUS_OK;
}
static int copy_h2d(salvus_problem *p, void *dst, const void *src, size_t bytes) {
  if (bytes < 2 * kPinChunk) {
    SALVUS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, p->stream));
    return SALVUS_OK;
  }
  int rc = pin_ready(p);
  if (rc) return rc;
  size_t off = 0;
  for (int k = 0; off < bytes; ++k) {
    const int b = k & 1;
    const size_t n = std::min(kPinChunk, bytes - off);
    if (k >= 2) SALVUS_CUDA(cudaEventSynchronize(p->pin_ev[b]));  // chunk free again
    par_memcpy(p->h_pin[b], (const char *)src + off, n);
    SALVUS_CUDA(cudaMemcpyAsync((char *)dst + off, p->h_pin[b], n, cudaMemcpyHostToDevice, p->stream));
    SALVUS_CUDA(cudaEventRecord(p->pin_ev[b], p->stream));
    off += n;
  }
  return SALVUS_OK;
}
// FP64 host array -> FP32 device field: the host threads convert each chunk
// into a pinned buffer while the previous chunk's DMA runs (half the bytes
// of an FP64 transfer cross PCIe).
static int copy_h2d_f32(salvus_problem *p, float *dst, const double *src, size_t n) {
  int rc = pin_ready(p);
  if (rc) return rc;
  const size_t per = kPinChunk / sizeof(float);
  size_t off = 0;
  for (int k = 0; off < n; ++k) {
    const int b = k & 1;
    const size_t m = std::min(per, n - off);
    if (k >= 2) SALVUS_CUDA(cudaEventSynchronize(p->pin_ev[b]));  // chunk free again
    par_convert(static_cast<float *>(p->h_pin[b]), src + off, m);
    SALVUS_CUDA(cudaMemcpyAsync(dst + off, p->h_pin[b], m * sizeof(float), cudaMemcpyHostToDevice,
                                p->stream));
    SALVUS_CUDA(cudaEventRecord(p->pin_ev[b], p->stream));
    off += m;
  }
  return SALVUS_OK;
}
static int copy_d2h(salvus_problem *p, void *dst, const void *src, size_t bytes) {
  if (bytes < 2 * kPinChunk) {
    SALVUS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, p->stream));
    return SALVUS_OK;
  }
  int rc = pin_ready(p);
  if (rc) return rc;
  const size_t nchunks = (bytes + kPinChunk - 1) / kPinChunk;
  auto issue = [&](size_t k) -> int {
    const size_t off = k * kPinChunk, n = std::min(kPinChunk, bytes - off);
    SALVUS_CUDA(cudaMemcpyAsync(p->h_pin[k & 1], (const char *)src + off, n, cudaMemcpyDeviceToHost,
                                p->stream));
    SALVUS_CUDA(cudaEventRecord(p->pin_ev[k & 1], p->stream));
    return SALVUS_OK;
  };
  if ((rc = issue(0))) return rc;
  for (size_t k = 0; k < nchunks; ++k) {
    // chunk (k + 1) & 1 was drained to the host in the previous iteration
    if (k + 1 < nchunks && (rc = issue(k + 1))) return rc;
    SALVUS_CUDA(cudaEventSynchronize(p->pin_ev[k & 1]));
    const size_t off = k * kPinChunk, n = std::min(kPinChunk, bytes - off);
    par_memcpy((char *)dst + off, p->h_pin[k & 1], n);
  }
  return SALVUS_OK;
}

static salvus::DeviceBuffer *field_buffer(salvus_problem *p, int32_t f) {
  switch (f) {
    case SALVUS_FIELD_U: return &p->d_u;
    case SALVUS_FIELD_V: return &p->d_v;
    case SALVUS_FIELD_A: return &p->d_a;
    case SALVUS_FIELD_A_PREV: return &p->d_ap;
  }
  return nullptr;
}

// One shot's column of a shot-batched field (u, or the half-step velocity w
// for SALVUS_FIELD_V; with a_ = 0 at the start, w = v there).
static int batched_field(salvus_problem *p, int32_t f, int32_t shot, double *vals, bool set) {
  if (f != SALVUS_FIELD_U && f != SALVUS_FIELD_V)
    return fail(SALVUS_E_UNSUPPORTED, "batched problems hold u and the half-step velocity only");
  if (shot < 0 || shot >= p->shots) return fail(SALVUS_E_INVALID, "shot %d out of range", shot);
  DeviceBuffer *b = f == SALVUS_FIELD_U ? &p->d_u : &p->d_v;
  const int64_t G = p->mesh->G;
  int rc;
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  if (p->d_stage.bytes < (size_t)(8 * G) && (rc = p->d_stage.alloc(8 * G))) return rc;
  if (set) {
    SALVUS_CUDA(cudaMemcpyAsync(p->d_stage.ptr, vals, 8 * G, cudaMemcpyHostToDevice, p->stream));
    shot_scatter_kernel<<<blocks_for(G, 256), 256, 0, p->stream>>>(G, p->shots_pad, shot,
                                                                   p->d_stage.as<double>(), b->as<float>());
  } else {
    shot_gather_kernel<<<blocks_for(G, 256), 256, 0, p->stream>>>(G, p->shots_pad, shot, b->as<float>(),
                                                                  p->d_stage.as<double>());
    SALVUS_CUDA(cudaMemcpyAsync(vals, p->d_stage.ptr, 8 * G, cudaMemcpyDeviceToHost, p->stream));
  }
  g_launches++;
  if ((rc = check_launch("shot field copy"))) return rc;
  SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  return SALVUS_OK;
}

int salvus_problem_set_field(salvus_problem *p, int32_t f, int32_t shot, const double *vals) {
  if (!p || !vals) return fail(SALVUS_E_INVALID, "null argument");
  if (p->shots > 1) return batched_field(p, f, shot, const_cast<double *>(vals), true);
  DeviceBuffer *b = field_buffer(p, f);
  if (!b || shot != 0) return fail(SALVUS_E_INVALID, "bad field %d / shot %d", f, shot);
  const size_t N = (size_t)p->mesh->G * p->c;
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  if (p->prec == SALVUS_FP64) {
    int rc = copy_h2d(p, b->ptr, vals, 8 * N);
    if (rc) return rc;
  } else {
    // FP64 host array -> FP32 on the host threads -> FP32 field
    int rc = copy_h2d_f32(p, b->as<float>(), vals, N);
    if (rc) return rc;
  }
  SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  return SALVUS_OK;
}

int salvus_problem_get_field(salvus_problem *p, int32_t f, int32_t shot, double *vals) {
  if (!p || !vals) return fail(SALVUS_E_INVALID, "null argument");
  if (p->shots > 1) return batched_field(p, f, shot, vals, false);
  DeviceBuffer *b = field_buffer(p, f);
  if (!b || shot != 0) return fail(SALVUS_E_INVALID, "bad field %d / shot %d", f, shot);
  const size_t N = (size_t)p->mesh->G * p->c;
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  if (p->prec == SALVUS_FP64) {
    int rc = copy_d2h(p, vals, b->ptr, 8 * N);
    if (rc) return rc;
  } else {
    int rc;
    if (p->d_stage.bytes < 8 * N && (rc = p->d_stage.alloc(8 * N))) return rc;
    convert_kernel<float, double><<<blocks_for((int64_t)N, 256), 256, 0, p->stream>>>(
        (int64_t)N, b->as<float>(), p->d_stage.as<double>());
    g_launches++;
    if ((rc = check_launch("convert"))) return rc;
    if ((rc = copy_d2h(p, vals, p->d_stage.ptr, 8 * N))) return rc;
  }
  SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  return device_status(p);
}

static int single_shot_only(salvus_problem *p) {
  if (p && p->shots > 1)
    return fail(SALVUS_E_UNSUPPORTED,
                "the three-call form is single-shot; batched problems use salvus_step / salvus_run");
  return SALVUS_OK;
}

int salvus_assemble(salvus_problem *p) {
  int rc = single_shot_only(p);
  if (rc) return rc;
  rc = ready(p);
  if (rc) return rc;
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  return by_components(p->c, [&](auto cc) {
    constexpr int C = decltype(cc)::value;
    return p->prec == SALVUS_FP32 ? assemble_t<float, C>(p) : assemble_t<double, C>(p);
  });
}

int salvus_apply_inverse_mass(salvus_problem *p) {
  int rc = single_shot_only(p);
  if (rc) return rc;
  rc = ready(p);
  if (rc) return rc;
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  return by_components(p->c, [&](auto cc) {
    constexpr int C = decltype(cc)::value;
    return p->prec == SALVUS_FP32 ? minv_t<float, C>(p) : minv_t<double, C>(p);
  });
}

int salvus_take_time_step(salvus_problem *p) {
  int rc = single_shot_only(p);
  if (rc) return rc;
  rc = ready(p);
  if (rc) return rc;
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  rc = by_components(p->c, [&](auto cc) {
    constexpr int C = decltype(cc)::value;
    return p->prec == SALVUS_FP32 ? newmark_t<float, C>(p) : newmark_t<double, C>(p);
  });
  if (rc == SALVUS_OK) p->step++;
  if (rc == SALVUS_OK && p->step % kFiniteEvery == 0) rc = launch_finite_check(p);
  return rc;
}

int salvus_step(salvus_problem *p) {
  int rc = ready(p);
  if (rc) return rc;
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  rc = step_fused(p);
  if (rc == SALVUS_OK) p->step++;
  if (rc == SALVUS_OK && p->step % kFiniteEvery == 0) rc = launch_finite_check(p);
  return rc;
}

int salvus_problem_set_wait_limit(salvus_problem *p, int64_t cycles) {
  if (!p) return fail(SALVUS_E_INVALID, "null problem");
  p->wait_limit = cycles > 0 ? (long long)cycles : salvus::kDefaultWaitLimit;
  drop_graph(p);  // captured launches hold the old bound
  return SALVUS_OK;
}

int salvus_problem_hold_device_waits(salvus_problem *p, int32_t enable) {
  if (!p) return fail(SALVUS_E_INVALID, "null problem");
  p->hold_waits = enable ? 1 : 0;
  drop_graph(p);  // captured launches hold the old setting
  return SALVUS_OK;
}

int salvus_problem_status(salvus_problem *p, int32_t clear) {
  if (!p) return fail(SALVUS_E_INVALID, "null problem");
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  const int rc = device_status(p);
  if (clear) {
    SALVUS_CUDA(cudaMemsetAsync(p->d_err.ptr, 0, sizeof(int), p->stream));
    SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  }
  return rc;
}

// Time loops replay CUDA graphs of captured fused steps: a run of n steps
// replays the 32-step graph n / 32 times and a graph of the remainder (the
// last remainder length is kept) when it is at least 8 steps, else launches
// those steps from the host.  Each graph ends with a finite check of u (the
// 32-step graph at every 32nd step, as host-launched runs do; a remainder
// graph at its end).
constexpr int kGraphChunk = 32, kGraphMin = 8;

static int capture_steps(salvus_problem *p, int steps, cudaGraphExec_t *exec, int64_t *launches) {
  const bool prof = p->profiling;
  p->profiling = false;
  // receivers forked onto the second stream in the captured steps only (in
  // host-launched steps the extra event calls would cost more host time
  // than the overlap saves on small meshes)
  p->rec_overlap = p->shots == 1 && p->rec_stream;
  cudaGraph_t graph;
  SALVUS_CUDA(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
  int crc = SALVUS_OK;
  const int64_t l0 = g_launches.load();
  for (int s = 0; s < steps && crc == SALVUS_OK; ++s) crc = step_fused(p);
  if (crc == SALVUS_OK) crc = launch_finite_check(p);
  // the captured sequence ends joined (a forked stream must rejoin the
  // capture), so every replay is self-contained
  const int jrc = join_receivers(p);
  if (crc == SALVUS_OK) crc = jrc;
  p->rec_overlap = false;
  cudaError_t ce = cudaStreamEndCapture(p->stream, &graph);
  // captured launches run only when the graph is replayed: count them there
  *launches = g_launches.load() - l0;
  g_launches -= *launches;
  p->profiling = prof;
  if (crc) {
    if (ce == cudaSuccess) cudaGraphDestroy(graph);
    return crc;
  }
  if (ce != cudaSuccess) return fail(SALVUS_E_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
  ce = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) return fail(SALVUS_E_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ce));
  return SALVUS_OK;
}

// the graphs a graph run of n_steps replays, captured if missing
static int prepare_graphs(salvus_problem *p, int64_t n_steps) {
  int rc;
  if (n_steps >= kGraphChunk && !p->graph_exec) {
    if ((rc = capture_steps(p, kGraphChunk, &p->graph_exec, &p->graph_launches))) return rc;
    p->graph_steps = kGraphChunk;
  }
  const int rem = (int)(n_steps % kGraphChunk);
  if (rem >= kGraphMin && p->tail_steps != rem) {
    if (p->tail_exec) cudaGraphExecDestroy(p->tail_exec);
    p->tail_exec = nullptr;
    p->tail_steps = 0;
    if ((rc = capture_steps(p, rem, &p->tail_exec, &p->tail_launches))) return rc;
    p->tail_steps = rem;
  }
  return SALVUS_OK;
}

static int rec_stream_ready(salvus_problem *p) {
  if (p->shots == 1 && !p->rec_stream) {  // created outside any graph capture
    SALVUS_CUDA(cudaStreamCreateWithFlags(&p->rec_stream, cudaStreamNonBlocking));
    SALVUS_CUDA(cudaEventCreateWithFlags(&p->ev_updated, cudaEventDisableTiming));
    SALVUS_CUDA(cudaEventCreateWithFlags(&p->ev_recorded, cudaEventDisableTiming));
  }
  return SALVUS_OK;
}

static int run_steps(salvus_problem *p, int64_t n_steps, int32_t mode);
int salvus_run(salvus_problem *p, int64_t n_steps, int32_t mode) {
  int rc = ready(p);
  if (rc) return rc;
  if (n_steps < 0) return fail(SALVUS_E_INVALID, "negative step count");
  if (mode != SALVUS_RUN_PLAIN && mode != SALVUS_RUN_GRAPH)
    return fail(SALVUS_E_INVALID, "unknown run mode %d", mode);
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  if ((rc = rec_stream_ready(p))) return rc;
  return run_steps(p, n_steps, mode);
}

int salvus_problem_prepare_run(salvus_problem *p, int64_t n_steps) {
  int rc = ready(p);
  if (rc) return rc;
  if (n_steps < 0) return fail(SALVUS_E_INVALID, "negative step count");
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  if ((rc = rec_stream_ready(p))) return rc;
  return prepare_graphs(p, n_steps);
}

static int plain_steps(salvus_problem *p, int64_t n) {
  int rc;
  for (int64_t s = 0; s < n; ++s) {
    if ((rc = step_fused(p))) return rc;
    p->step++;
    if (p->step % kFiniteEvery == 0 && (rc = launch_finite_check(p))) return rc;
  }
  return SALVUS_OK;
}

static int run_steps(salvus_problem *p, int64_t n_steps, int32_t mode) {
  if (mode == SALVUS_RUN_PLAIN || n_steps < kGraphMin) return plain_steps(p, n_steps);
  int rc = prepare_graphs(p, n_steps);
  if (rc) return rc;
  int64_t done = 0;
  while (n_steps - done >= p->graph_steps && p->graph_exec) {
    ProfScope ps(p, K_GRAPH);
    SALVUS_CUDA(cudaGraphLaunch(p->graph_exec, p->stream));
    g_launches += p->graph_launches;
    done += p->graph_steps;
    p->step += p->graph_steps;
  }
  if (p->tail_exec && n_steps - done == p->tail_steps) {
    ProfScope ps(p, K_GRAPH);
    SALVUS_CUDA(cudaGraphLaunch(p->tail_exec, p->stream));
    g_launches += p->tail_launches;
    done += p->tail_steps;
    p->step += p->tail_steps;
  }
  return plain_steps(p, n_steps - done);
}

// Energy of the current state: -K u into a scratch field (stiffness and
// Dirichlet zeroing, then the gather), then the compensated FP64 sums.
extern "C++" {
template <typename real, int C>
static int energy_t(salvus_problem *p, double *kinetic, double *strain) {
  const salvus_mesh *m = p->mesh;
  const size_t N = (size_t)m->G * C;
  int rc;
  if (p->d_escr.bytes < N * sizeof(real) && (rc = p->d_escr.alloc(N * sizeof(real)))) return rc;
  constexpr int kBlocks = 1024;
  if (p->d_epart.bytes < 2 * kBlocks * sizeof(double) &&
      (rc = p->d_epart.alloc(2 * kBlocks * sizeof(double))))
    return rc;
  if ((rc = launch_stiffness<real>(m, records<real>(p), F<real>(p->d_u), F<real>(p->d_r), p->stream,
                                   p->d_err.as<int>(), p->wait_limit, p->hold_waits)))
    return rc;
  if ((rc = launch_dirichlet<real, C>(p))) return rc;
  gather_kernel<real, C, 1><<<blocks_for(m->G, 256), 256, 0, p->stream>>>(
      m->G, m->d_inc_off.as<int32_t>(), m->d_inc_idx.as<int32_t>(), F<real>(p->d_r), nullptr,
      nullptr, nullptr, nullptr, p->d_escr.as<real>(), (real)0);
  g_launches++;
  if ((rc = check_launch("energy gather"))) return rc;
  energy_kernel<real, C><<<kBlocks, 256, 0, p->stream>>>(
      m->G, F<real>(p->d_u), F<real>(p->d_v), p->d_escr.as<real>(), m->d_mi64.as<double>(),
      p->d_epart.as<double>());
  g_launches++;
  if ((rc = check_launch("energy"))) return rc;
  std::vector<double> h(2 * kBlocks);
  SALVUS_CUDA(cudaMemcpyAsync(h.data(), p->d_epart.ptr, sizeof(double) * h.size(),
                              cudaMemcpyDeviceToHost, p->stream));
  SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  // Kahan over the block partials, in block order
  double sk = 0, ck = 0, ss = 0, cs = 0;
  for (int b = 0; b < kBlocks; ++b) {
    const double yk = h[2 * b] - ck, tk = sk + yk;
    ck = (tk - sk) - yk;
    sk = tk;
    const double ys = h[2 * b + 1] - cs, ts = ss + ys;
    cs = (ts - ss) - ys;
    ss = ts;
  }
  if (kinetic) *kinetic = sk;
  if (strain) *strain = ss;
  return device_status(p);
}
}  // extern "C++"

int salvus_problem_energy(salvus_problem *p, double *kinetic, double *strain) {
  if (!p) return fail(SALVUS_E_INVALID, "null problem");
  if (p->shots > 1)
    return fail(SALVUS_E_UNSUPPORTED, "energy is computed for single-shot problems");
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  return by_components(p->c, [&](auto cc) {
    constexpr int C = decltype(cc)::value;
    return p->prec == SALVUS_FP32 ? energy_t<float, C>(p, kinetic, strain)
                                  : energy_t<double, C>(p, kinetic, strain);
  });
}

int salvus_synchronize(salvus_problem *p) {
  if (!p) return fail(SALVUS_E_INVALID, "null problem");
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  return device_status(p);
}

int64_t salvus_problem_step_index(const salvus_problem *p) { return p ? p->step : -1; }

int salvus_problem_autotune(salvus_problem *p, int32_t *stiff_shot_lanes, int32_t *stiff_elements,
                            int32_t *gather_shot_lanes, int32_t *gather_nodes) {
  int rc = ready(p);
  if (rc) return rc;
  if (p->shots == 1) {
    if (stiff_shot_lanes) *stiff_shot_lanes = 1;
    if (stiff_elements) *stiff_elements = 0;
    if (gather_shot_lanes) *gather_shot_lanes = 1;
    if (gather_nodes) *gather_nodes = 256;
    return SALVUS_OK;
  }
  if (stiff_shot_lanes) *stiff_shot_lanes = kStiffCfg[p->tune_stiff].sc;
  if (stiff_elements) *stiff_elements = kStiffCfg[p->tune_stiff].epc;
  if (gather_shot_lanes) *gather_shot_lanes = kGatherCfg[p->tune_gather].sc;
  if (gather_nodes) *gather_nodes = kGatherCfg[p->tune_gather].epc * kGatherCfg[p->tune_gather].npt;
  return SALVUS_OK;
}

int salvus_problem_step_config(salvus_problem *p, int32_t *form, int32_t *elements_per_cta) {
  int rc = ready(p);
  if (rc) return rc;
  const salvus_mesh *m = p->mesh;
  int32_t f = SALVUS_STEP_PLAIN, epc = 0;
  if (p->shots > 1) {
    f = batch_fusion(p) && m->order >= 2 ? SALVUS_STEP_FUSED_INTERIOR : SALVUS_STEP_PLAIN;
    epc = kStiffCfg[p->tune_stiff].epc;
  } else if (m->shape == SALVUS_HEX && m->affine && p->prec == SALVUS_FP32 &&
             m->physics == SALVUS_ELASTIC3D) {
    f = hex_interior_fusion(p) ? SALVUS_STEP_FUSED_INTERIOR : SALVUS_STEP_PLAIN;
    const int n2 = (m->order + 1) * (m->order + 1), e1 = 128 / n2 > 0 ? 128 / n2 : 1;
    epc = e1 * (m->hex_wide ? 2 : 1);
  }
  if (form) *form = f;
  if (elements_per_cta) *elements_per_cta = epc;
  return SALVUS_OK;
}

int salvus_problem_stream(const salvus_problem *p, void **stream) {
  if (!p || !stream) return fail(SALVUS_E_INVALID, "null argument");
  *stream = (void *)p->stream;
  return SALVUS_OK;
}

int salvus_problem_info(const salvus_problem *p, int32_t *shots, int32_t *nrec, int32_t *c) {
  if (!p) return fail(SALVUS_E_INVALID, "null problem");
  if (shots) *shots = p->shots;
  if (nrec) *nrec = (int32_t)p->recs.size();
  if (c) *c = p->c;
  return SALVUS_OK;
}

int salvus_get_seismograms(salvus_problem *p, int64_t first, int64_t count, double *out) {
  if (!p || !out) return fail(SALVUS_E_INVALID, "null argument");
  if (count < 0 || first < 0 || first + count > p->step || first < p->step - p->seis_cap)
    return fail(SALVUS_E_INVALID, "steps [%lld, %lld) not held (step %lld, capacity %lld)",
                (long long)first, (long long)(first + count), (long long)p->step,
                (long long)p->seis_cap);
  if (p->recs.empty() || count == 0) return SALVUS_OK;
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  const int64_t rows = (int64_t)p->shots * p->recs.size() * p->c;
  std::vector<double> ring((size_t)(rows * p->seis_cap));
  SALVUS_CUDA(cudaMemcpyAsync(ring.data(), p->d_seis.ptr, 8 * ring.size(), cudaMemcpyDeviceToHost,
                              p->stream));
  SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  if (int rc = device_status(p)) return rc;
  for (int64_t rr = 0; rr < rows; ++rr)
    for (int64_t s = 0; s < count; ++s)
      out[rr * count + s] = ring[(size_t)(rr * p->seis_cap + (first + s) % p->seis_cap)];
  return SALVUS_OK;
}

int salvus_profile_enable(salvus_problem *p, int32_t enable) {
  if (!p) return fail(SALVUS_E_INVALID, "null problem");
  p->profiling = enable != 0;
  return SALVUS_OK;
}

int salvus_profile_read(salvus_problem *p, int32_t max_entries, const char **names, double *ms,
                        int64_t *launches, int32_t *n_entries) {
  if (!p) return fail(SALVUS_E_INVALID, "null problem");
  SALVUS_CUDA(cudaSetDevice(p->mesh->device));
  SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  for (auto &e : p->events) {
    float t = 0.f;
    cudaEventElapsedTime(&t, e.a, e.b);
    p->prof_ms[e.kind] += t;
    p->prof_n[e.kind] += 1;
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  p->events.clear();
  int k = 0;
  for (int i = 0; i < K_NKINDS && k < max_entries; ++i) {
    if (!p->prof_n[i]) continue;
    if (names) names[k] = kKindNames[i];
    if (ms) ms[k] = p->prof_ms[i];
    if (launches) launches[k] = p->prof_n[i];
    ++k;
  }
  if (n_entries) *n_entries = k;
  std::fill(p->prof_ms.begin(), p->prof_ms.end(), 0.0);
  std::fill(p->prof_n.begin(), p->prof_n.end(), 0);
  return SALVUS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// problem groups
int salvus_group_create(salvus_problem *const *members, int32_t n, salvus_group **out) {
  if (!members || !out || n < 1) return fail(SALVUS_E_INVALID, "empty group");
  *out = nullptr;
  const salvus_mesh *m0 = members[0] ? members[0]->mesh : nullptr;
  if (!m0) return fail(SALVUS_E_INVALID, "null problem in group");
  const bool quad_ac = m0->shape == SALVUS_QUAD && m0->physics == SALVUS_ACOUSTIC;
  const bool hex_el = m0->shape == SALVUS_HEX && m0->physics == SALVUS_ELASTIC3D;
  if (!quad_ac && !hex_el)
    return fail(SALVUS_E_UNSUPPORTED, "groups are built for acoustic quads and elastic hexahedra");
  for (int32_t k = 0; k < n; ++k) {
    const salvus_problem *p = members[k];
    if (!p) return fail(SALVUS_E_INVALID, "null problem in group");
    const salvus_mesh *m = p->mesh;
    if (p->prec != SALVUS_FP32 || p->shots != 1)
      return fail(SALVUS_E_UNSUPPORTED, "group members must be FP32 single-shot problems");
    if (p->n_dir_pts > 0)
      return fail(SALVUS_E_UNSUPPORTED, "group members cannot carry Dirichlet boundaries");
    if (m->ti)
      return fail(SALVUS_E_UNSUPPORTED,
                  "group members must have isotropic material (transversely isotropic meshes "
                  "run as single problems)");
    if (m->shape != m0->shape || m->order != m0->order || m->physics != m0->physics ||
        m->device != m0->device)
      return fail(SALVUS_E_INVALID, "group members must share shape, order, physics and device");
    for (int32_t q = 0; q < k; ++q)
      if (members[q] == p) return fail(SALVUS_E_INVALID, "problem listed twice in a group");
  }
  std::unique_ptr<salvus_group> g(new salvus_group());
  g->members.assign(members, members + n);
  g->m0 = m0;
  g->device = m0->device;
  g->c = m0->physics == SALVUS_ELASTIC3D ? 3 : 1;
  {
    // measured: one launch per stage beats both single-launch forms (the
    // work-queue and the member-partitioned kernel, whose combined bodies
    // run the latency-bound gather at the occupancy of the heaviest body),
    // so it is the default
    const char *s = std::getenv("SALVUS_GROUP_STEP");
    g->partitioned = s && std::strcmp(s, "partitioned") == 0;
    g->stages = !(s && (std::strcmp(s, "persistent") == 0 || g->partitioned));
  }
  SALVUS_CUDA(cudaSetDevice(m0->device));
  SALVUS_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  SALVUS_CUDA(cudaEventCreateWithFlags(&g->ev, cudaEventDisableTiming));
  g->member_ev.resize(n, nullptr);
  for (auto &e : g->member_ev) SALVUS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  *out = g.release();
  return SALVUS_OK;
}

int salvus_group_run(salvus_group *g, int64_t n_steps) {
  if (!g) return fail(SALVUS_E_INVALID, "null group");
  if (n_steps < 0) return fail(SALVUS_E_INVALID, "negative step count");
  SALVUS_CUDA(cudaSetDevice(g->m0->device));
  // order the group after every member's pending work
  for (size_t k = 0; k < g->members.size(); ++k) {
    SALVUS_CUDA(cudaEventRecord(g->member_ev[k], g->members[k]->stream));
    SALVUS_CUDA(cudaStreamWaitEvent(g->stream, g->member_ev[k], 0));
  }
  int rc = group_fill(g);
  if (rc) return rc;
  const int chunk = 32;
  const int64_t sig[3] = {g->n_stiff, g->n_gather, g->n_rec};
  if (g->graph && (sig[0] != g->sig[0] || sig[1] != g->sig[1] || sig[2] != g->sig[2])) {
    cudaGraphExecDestroy(g->graph);
    g->graph = nullptr;
  }
  if (!g->graph && n_steps >= chunk) {
    cudaGraph_t graph;
    SALVUS_CUDA(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
    int crc = SALVUS_OK;
    for (int s = 0; s < chunk && crc == SALVUS_OK; ++s) crc = group_step(g);
    cudaError_t ce = cudaStreamEndCapture(g->stream, &graph);
    if (crc) return crc;
    if (ce != cudaSuccess) return fail(SALVUS_E_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&g->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return fail(SALVUS_E_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ce));
    g->graph_steps = chunk;
    for (int a = 0; a < 3; ++a) g->sig[a] = sig[a];
  }
  int64_t done = 0;
  while (g->graph && n_steps - done >= g->graph_steps) {
    SALVUS_CUDA(cudaGraphLaunch(g->graph, g->stream));
    g_launches += (int64_t)g->graph_steps * (g->stages ? (g->n_rec > 0 ? 5 : 4) : 1);
    done += g->graph_steps;
  }
  for (; done < n_steps; ++done)
    if ((rc = group_step(g))) return rc;
  for (auto *p : g->members) p->step += n_steps;
  // members' later work waits for the group; then each member's finite check
  // on its own stream
  SALVUS_CUDA(cudaEventRecord(g->ev, g->stream));
  for (auto *p : g->members) {
    SALVUS_CUDA(cudaStreamWaitEvent(p->stream, g->ev, 0));
    if (n_steps > 0 && (rc = launch_finite_check(p))) return rc;
  }
  return SALVUS_OK;
}

int salvus_group_set_wait_limit(salvus_group *g, int64_t cycles) {
  if (!g) return fail(SALVUS_E_INVALID, "null group");
  g->wait_limit = cycles > 0 ? (long long)cycles : salvus::kDefaultWaitLimit;
  if (g->graph) cudaGraphExecDestroy(g->graph);  // captured launches hold the old bound
  g->graph = nullptr;
  return SALVUS_OK;
}

int salvus_group_clear_status(salvus_group *g) {
  if (!g) return fail(SALVUS_E_INVALID, "null group");
  SALVUS_CUDA(cudaSetDevice(g->m0->device));
  SALVUS_CUDA(cudaStreamSynchronize(g->stream));
  if (g->d_sync.ptr) SALVUS_CUDA(cudaMemset(g->d_sync.ptr, 0, sizeof(GroupSync)));
  for (auto *p : g->members) {
    SALVUS_CUDA(cudaMemsetAsync(p->d_err.ptr, 0, sizeof(int), p->stream));
    SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  }
  return SALVUS_OK;
}

int salvus_group_synchronize(salvus_group *g) {
  if (!g) return fail(SALVUS_E_INVALID, "null group");
  SALVUS_CUDA(cudaSetDevice(g->m0->device));
  SALVUS_CUDA(cudaStreamSynchronize(g->stream));
  if (g->d_sync.ptr) {
    GroupSync s{};
    SALVUS_CUDA(cudaMemcpy(&s, g->d_sync.ptr, sizeof(s), cudaMemcpyDeviceToHost));
    if (s.err) return fail(SALVUS_E_TIMEOUT, "a bounded wait of the grouped step gave up; results invalid");
  }
  for (auto *p : g->members)
    if (int rc = device_status(p)) return rc;
  return SALVUS_OK;
}

cudaStream_t salvus_group_stream_internal(const salvus_group *g) { return g ? g->stream : nullptr; }

int salvus_group_destroy(salvus_group *g) {
  if (!g) return SALVUS_OK;
  // the group's own device: its members' meshes may already be gone
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  if (g->graph) cudaGraphExecDestroy(g->graph);
  for (auto e : g->member_ev)
    if (e) cudaEventDestroy(e);
  if (g->ev) cudaEventDestroy(g->ev);
  g->d_slots.release();
  g->d_counts.release();
  g->d_work.release();
  g->d_done.release();
  g->d_sync.release();
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
  return SALVUS_OK;
}

// ---------------------------------------------------------------------------
// homogeneous Dirichlet boundaries
int salvus_mesh_boundary_nodes(const salvus_mesh *m, int64_t *count, int64_t *nodes) {
  if (!m || !count) return fail(SALVUS_E_INVALID, "null argument");
  std::vector<int64_t> b;
  int rc = boundary_nodes(m, b);
  if (rc) return rc;
  if (nodes) std::memcpy(nodes, b.data(), sizeof(int64_t) * b.size());
  *count = (int64_t)b.size();
  return SALVUS_OK;
}

int salvus_problem_set_dirichlet(salvus_problem *p, int64_t n, const int64_t *nodes) {
  if (!p || (n > 0 && !nodes) || n < 0) return fail(SALVUS_E_INVALID, "bad arguments");
  const salvus_mesh *m = p->mesh;
  if (p->shots > 1)
    return fail(SALVUS_E_UNSUPPORTED, "Dirichlet boundaries are not built for shot-batched problems");
  std::vector<char> flag((size_t)m->G, 0);
  for (int64_t k = 0; k < n; ++k) {
    if (nodes[k] < 0 || nodes[k] >= m->G) return fail(SALVUS_E_INVALID, "node %lld out of range",
                                                      (long long)nodes[k]);
    flag[(size_t)nodes[k]] = 1;
  }
  // every element point on a flagged node, ascending (element, point)
  std::vector<int32_t> pts;
  for (int64_t i = 0; i < m->E * m->P; ++i)
    if (flag[(size_t)m->conn[(size_t)i]]) pts.push_back((int32_t)i);
  SALVUS_CUDA(cudaSetDevice(m->device));
  if (!pts.empty()) {
    int rc = p->d_dir_pts.alloc(sizeof(int32_t) * pts.size());
    if (rc) return rc;
    SALVUS_CUDA(cudaMemcpyAsync(p->d_dir_pts.ptr, pts.data(), sizeof(int32_t) * pts.size(),
                                cudaMemcpyHostToDevice, p->stream));
    SALVUS_CUDA(cudaStreamSynchronize(p->stream));
  }
  p->n_dir_pts = (int64_t)pts.size();
  drop_graph(p);
  return SALVUS_OK;
}
