// kernels_stiffness.cuh -- per-element stiffness action r_e = -K_e u_e for
// tensor-product GLL elements, written to an element-local residual
// r[E][P][c] that the node-gather update assembles in a fixed order (so the
// result is bitwise deterministic without atomics or colouring passes).
//
// Reference arithmetic restated:
//   acoustic  Scalar::computeStiffnessTerm (Scalar.cpp:58-71): gradient
//             (TensorQuad.cpp:177-210, Hexahedra.cpp:580-632), stress vp^2 grad
//             (Scalar.cpp:42-55), gradient-test integral
//             (TensorQuad.cpp:351-397, Hexahedra.cpp:689-754);
//   elastic   Elastic3D::computeStiffnessTerm (Elastic3D.cpp:70-103) with
//             Voigt strains and c_ij stress (Elastic3D.cpp:106-118).
// The geometric factors are precomputed once (records, kernels_setup.cuh) so
// the per-step kernel streams them instead of rebuilding the Jacobian at every
// GLL point as the reference does (Hexahedra.cpp:600,702).
#pragma once

#include <cstdint>

#include "kernels_material.cuh"

namespace salvus {

template <typename real>
struct DMatrix {
  real d[kMaxN * kMaxN];  // d[i*n + j] = l_j'(xi_i)
};

__host__ __device__ constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

// ---------------------------------------------------------------------------
// Acoustic (quad and hex): one thread per element point, EPB elements per CTA.
template <int DIM, int N>
struct AcousticShape {
  static constexpr int n = N + 1;
  static constexpr int P = ipow(n, DIM);
  static constexpr int EPB = (256 / P) > 0 ? (256 / P) : 1;
  static constexpr int THREADS = ((EPB * P + 31) / 32) * 32;
  static constexpr int NG = DIM == 2 ? 3 : 6;
};

// rk: record index of the point, ce: its connectivity index (equal unless the
// element comes from a list with class-compact records)
template <int DIM>
__device__ __forceinline__ void load_acoustic_rec(const float *__restrict__ rec,
                                                  const int32_t *__restrict__, int64_t rk,
                                                  int64_t, float *g, int32_t *node) {
  if (DIM == 2) {
    float4 a = __ldg(reinterpret_cast<const float4 *>(rec) + rk);
    g[0] = a.x; g[1] = a.y; g[2] = a.z;
    *node = __float_as_int(a.w);
  } else {
    const float4 *q = reinterpret_cast<const float4 *>(rec) + 2 * rk;
    float4 a = __ldg(q), b = __ldg(q + 1);
    g[0] = a.x; g[1] = a.y; g[2] = a.z; g[3] = a.w; g[4] = b.x; g[5] = b.y;
    *node = __float_as_int(b.z);
  }
}

template <int DIM>
__device__ __forceinline__ void load_acoustic_rec(const double *__restrict__ rec,
                                                  const int32_t *__restrict__ conn, int64_t rk,
                                                  int64_t ce, double *g, int32_t *node) {
  constexpr int NG = DIM == 2 ? 3 : 6;
#pragma unroll
  for (int a = 0; a < NG; ++a) g[a] = rec[rk * NG + a];
  *node = conn[ce];
}

// bid: element-group index (the CTA index of a single-mesh launch; grouped
// multi-mesh launches pass the CTA's index within its mesh).
// C > 1: nodes carry C field components and this element class owns the
// first (meshes of fluid and solid elements); the residual's other
// components of the element's points are written as zero.  kList: the
// group's k-th element is mesh element elist[k], with record k.
template <int DIM, int N, typename real, int C = 1, bool kList = false>
__device__ __forceinline__ void acoustic_stiffness_body(int64_t bid, int64_t E,
                                                        const real *__restrict__ rec,
                                                        const int32_t *__restrict__ conn,
                                                        const real *__restrict__ u,
                                                        real *__restrict__ r,
                                                        const DMatrix<real> &Dm,
                                                        const int32_t *__restrict__ elist = nullptr) {
  using S = AcousticShape<DIM, N>;
  constexpr int n = S::n, P = S::P, EPB = S::EPB, n2 = n * n;
  __shared__ real sD[n * n];
  __shared__ real su[EPB][P];
  __shared__ real sF[EPB][DIM][P];
  const int t = threadIdx.x;
  const int le = t / P, p = t - le * P;
  if (t < n * n) sD[t] = Dm.d[t];
  const int64_t k_ = bid * EPB + le;
  const bool ok = le < EPB && k_ < E;
  int64_t e = k_;
  real g[S::NG];
  int32_t node = 0;
  if (ok) {
    if constexpr (kList) e = elist[k_];
    load_acoustic_rec<DIM>(rec, conn, k_ * P + p, e * P + p, g, &node);
    su[le][p] = u[(int64_t)node * C];
  }
  __syncthreads();
  const int i = p % n, j = (p / n) % n, k = DIM == 3 ? p / n2 : 0;
  if (ok) {
    real gr[3] = {0, 0, 0};
#pragma unroll
    for (int l = 0; l < n; ++l) {
      gr[0] += sD[i * n + l] * su[le][l + n * j + n2 * k];
      gr[1] += sD[j * n + l] * su[le][i + n * l + n2 * k];
      if (DIM == 3) gr[2] += sD[k * n + l] * su[le][i + n * j + n2 * l];
    }
    if (DIM == 2) {
      sF[le][0][p] = g[0] * gr[0] + g[1] * gr[1];
      sF[le][1][p] = g[1] * gr[0] + g[2] * gr[1];
    } else {
      // g = [G00 G01 G02 G11 G12 G22]
      sF[le][0][p] = g[0] * gr[0] + g[1] * gr[1] + g[2] * gr[2];
      sF[le][1][p] = g[1] * gr[0] + g[3] * gr[1] + g[4] * gr[2];
      if (DIM == 3) sF[le][DIM - 1][p] = g[2] * gr[0] + g[4] * gr[1] + g[5] * gr[2];
    }
  }
  __syncthreads();
  if (ok) {
    real out = 0;
#pragma unroll
    for (int l = 0; l < n; ++l) {
      out += sD[l * n + i] * sF[le][0][l + n * j + n2 * k];
      out += sD[l * n + j] * sF[le][1][i + n * l + n2 * k];
      if (DIM == 3) out += sD[l * n + k] * sF[le][DIM - 1][i + n * j + n2 * l];
    }
    r[(e * P + p) * C] = -out;
#pragma unroll
    for (int c = 1; c < C; ++c) r[(e * P + p) * C + c] = real(0);
  }
}

template <int DIM, int N, typename real>
__global__ void __launch_bounds__(AcousticShape<DIM, N>::THREADS)
acoustic_stiffness_kernel(int64_t E, const real *__restrict__ rec, const int32_t *__restrict__ conn,
                          const real *__restrict__ u, real *__restrict__ r, DMatrix<real> Dm) {
  acoustic_stiffness_body<DIM, N, real>(blockIdx.x, E, rec, conn, u, r, Dm);
}

// fluid elements of a mesh that also holds solid elements: nodes carry
// [u, ux, uy], the listed elements own u
template <int N, typename real>
__global__ void __launch_bounds__(AcousticShape<2, N>::THREADS)
acoustic_list_kernel(int64_t nE, const int32_t *__restrict__ elist, const real *__restrict__ rec,
                     const int32_t *__restrict__ conn, const real *__restrict__ u,
                     real *__restrict__ r, DMatrix<real> Dm) {
  acoustic_stiffness_body<2, N, real, 3, true>(blockIdx.x, nE, rec, conn, u, r, Dm, elist);
}

// ---------------------------------------------------------------------------
// Elastic hexahedra: one thread per (i, j) column of an element holding the
// n points along t in registers; r- and s-derivatives go through shared
// memory, t-derivatives stay in registers.
template <int N, typename real>
struct ElasticShape {
  static constexpr int n = N + 1, n2 = n * n, P = n2 * n;
  static constexpr int EPB = ((sizeof(real) == 4 ? 200 : 100) / n2) > 0
                                 ? ((sizeof(real) == 4 ? 200 : 100) / n2) : 1;
  static constexpr int THREADS = ((EPB * n2 + 31) / 32) * 32;
  // su[EPB][3][P] + sF[EPB][3][2][P]
  static constexpr size_t SMEM = sizeof(real) * (size_t)EPB * 9 * P;
};

// Records (kernels_setup.cuh): FP32 as float4 planes per element
// ([E][3|4][P]: invJ 0-3, invJ 4-7, (invJ 8, m0, m1, conn)[, (m2, m3, m4, 0)]),
// FP64 as [E][P][9 + kWords] (invJ, m); m = (lambda', mu') or, for
// transversely isotropic material, (A', C', F', L', N').
template <bool TI>
__device__ __forceinline__ void load_elastic_rec(const float *__restrict__ rec, int64_t e, int p,
                                                 int P, float *J, float *m) {
  constexpr int PL = TI ? 4 : 3;
  const float4 *q = reinterpret_cast<const float4 *>(rec) + e * PL * P + p;
  float4 a = __ldg(q), b = __ldg(q + P), c = __ldg(q + 2 * P);
  J[0] = a.x; J[1] = a.y; J[2] = a.z; J[3] = a.w;
  J[4] = b.x; J[5] = b.y; J[6] = b.z; J[7] = b.w;
  J[8] = c.x; m[0] = c.y; m[1] = c.z;
  if constexpr (TI) {
    float4 d = __ldg(q + 3 * P);
    m[2] = d.x; m[3] = d.y; m[4] = d.z;
  }
}
template <bool TI>
__device__ __forceinline__ void load_elastic_rec(const double *__restrict__ rec, int64_t e, int p,
                                                 int P, double *J, double *m) {
  constexpr int W = 9 + ElasticMat<TI>::kWords;
  const int64_t ep = e * P + p;
#pragma unroll
  for (int a = 0; a < 9; ++a) J[a] = rec[ep * W + a];
#pragma unroll
  for (int a = 0; a < ElasticMat<TI>::kWords; ++a) m[a] = rec[ep * W + 9 + a];
}

template <int N, typename real, bool TI = false>
__global__ void __launch_bounds__(ElasticShape<N, real>::THREADS)
elastic_hex_stiffness_kernel(int64_t E, const real *__restrict__ rec,
                             const int32_t *__restrict__ conn, const real *__restrict__ u,
                             real *__restrict__ r, DMatrix<real> Dm) {
  using S = ElasticShape<N, real>;
  constexpr int n = S::n, n2 = S::n2, P = S::P, EPB = S::EPB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  real *smem = reinterpret_cast<real *>(smem_raw);
  const int t = threadIdx.x;
  const int le = t / n2, ij = t - le * n2;
  const int i = ij % n, j = ij / n;
  const int64_t e = (int64_t)blockIdx.x * EPB + le;
  const bool ok = le < EPB && e < E;
  real *su = smem + (size_t)(ok ? le : 0) * 3 * P;             // [3][P]
  real *sF = smem + (size_t)EPB * 3 * P + (size_t)(ok ? le : 0) * 6 * P;  // [3][2][P]

  real Dri[n], Dsj[n], DTi[n], DTj[n];
#pragma unroll
  for (int l = 0; l < n; ++l) {
    Dri[l] = Dm.d[i * n + l];
    Dsj[l] = Dm.d[j * n + l];
    DTi[l] = Dm.d[l * n + i];
    DTj[l] = Dm.d[l * n + j];
  }
  real ux[n], uy[n], uz[n];
  if (ok) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
      const int32_t node = conn[e * P + p];
      ux[k] = u[3 * (int64_t)node + 0];
      uy[k] = u[3 * (int64_t)node + 1];
      uz[k] = u[3 * (int64_t)node + 2];
      su[0 * P + p] = ux[k];
      su[1 * P + p] = uy[k];
      su[2 * P + p] = uz[k];
    }
  }
  __syncthreads();
  real Ftx[n], Fty[n], Ftz[n];
  if (ok) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
      real J[9], mat[ElasticMat<TI>::kWords];
      load_elastic_rec<TI>(rec, e, p, P, J, mat);
      real d[3][3];  // d[c][b]: derivative of u_c along reference direction b
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const real *sc = su + c * P;
        real dr = 0, ds = 0, dt = 0;
#pragma unroll
        for (int l = 0; l < n; ++l) {
          dr += Dri[l] * sc[l + n * j + n2 * k];
          ds += Dsj[l] * sc[i + n * l + n2 * k];
        }
        const real *uc = c == 0 ? ux : (c == 1 ? uy : uz);
#pragma unroll
        for (int l = 0; l < n; ++l) dt += Dm.d[k * n + l] * uc[l];
        d[c][0] = dr; d[c][1] = ds; d[c][2] = dt;
      }
      // physical gradient g[c][a] = du_c/dx_a = sum_b invJ[a][b] d[c][b]
      real g[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a)
          g[c][a] = J[a * 3 + 0] * d[c][0] + J[a * 3 + 1] * d[c][1] + J[a * 3 + 2] * d[c][2];
      // Hooke with quadrature weight and detJ folded into the constants
      real sig[3][3];
      if constexpr (TI) stress_ti<real>(g, mat, sig);
      else stress_iso<real>(g, mat[0], mat[1], sig);
      // F_c[b] = sum_a invJ[a][b] sigma[c][a]
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        real F0 = J[0] * sig[c][0] + J[3] * sig[c][1] + J[6] * sig[c][2];
        real F1 = J[1] * sig[c][0] + J[4] * sig[c][1] + J[7] * sig[c][2];
        real F2 = J[2] * sig[c][0] + J[5] * sig[c][1] + J[8] * sig[c][2];
        sF[(c * 2 + 0) * P + p] = F0;
        sF[(c * 2 + 1) * P + p] = F1;
        if (c == 0) Ftx[k] = F2;
        else if (c == 1) Fty[k] = F2;
        else Ftz[k] = F2;
      }
    }
  }
  __syncthreads();
  if (ok) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const real *Fr = sF + (c * 2 + 0) * P, *Fs = sF + (c * 2 + 1) * P;
        const real *Ft = c == 0 ? Ftx : (c == 1 ? Fty : Ftz);
        real o = 0;
#pragma unroll
        for (int l = 0; l < n; ++l) {
          o += DTi[l] * Fr[l + n * j + n2 * k];
          o += DTj[l] * Fs[i + n * l + n2 * k];
          o += Dm.d[l * n + k] * Ft[l];
        }
        r[(e * P + p) * 3 + c] = -o;
      }
    }
  }
}

}  // namespace salvus
