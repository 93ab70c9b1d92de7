// kernels_hex_affine.cuh -- FP32 elastic hexahedra whose elements are all
// parallelepipeds (affine maps): the inverse Jacobian is one 3x3 matrix per
// element, so the per-point record shrinks to the folded material constants
// (plus the connectivity, read from the [E][P] map).
//
// Same arithmetic as the column-threaded kernel of kernels_hex_v2.cuh
// (Elastic3D.cpp:70-118 via Hexahedra.cpp:580-632 / 689-754) with J taken
// from the element instead of the point.  Global arrays:
//   jac  [E][9]    invJ (row-major [x_a][xi_b]) of each element
//   mat  [NM][E*P] material planes: lambda', mu' (isotropic) or A', C', F',
//                  L', N' (transversely isotropic), w detJ folded in
//   conn [E][P]    element point -> global node
//
// Fused step form (kFuse): the interior GLL points of an element (all three
// local indices in 1..N-1) are nodes that no other element touches, so the
// kernel finishes them itself -- the source terms of this element in attach
// order (source_body's arithmetic), the one-term assembly 0 + r (the node
// gather's first addition), the inverse mass and the Newmark update
// (newmark_point) -- and writes element-local residuals only for the points
// on the element's faces, which the node gather then assembles over the
// shared nodes alone.  Every operation and its order is the one of the
// unfused sequence (stiffness, sources, gather, update), so the two forms
// give bitwise the same wavefield.  In the fused form u is written for
// interior nodes during the launch, so u is read with coherent loads (the
// read-only path is for data no thread writes during the launch); each
// interior node is read and then written by the one thread that owns it.
#pragma once

#include <cstdint>

#include "kernels_hex_v2.cuh"
#include "kernels_material.cuh"
#include "kernels_step.cuh"

namespace salvus {

// Interior-node update of the fused step: Newmark state, inverse mass and the
// problem's sources (kernels_step.cuh source_body layout).
struct HexInteriorUpdate {
  const float *mi;
  float *v, *ap;
  float dt;
  double dtd;
  int nsrc;
  const int64_t *src_elem;
  const double *src_par;  // [nsrc][3] f0 t0 amp
  const double *src_wts;  // [nsrc][P][3]
  const int64_t *step;
};

template <int N, int EPB_, bool TI>
struct HexAffineShape {
  using V2 = ElasticV2Shape<N, EPB_, TI>;
  static constexpr int n = V2::n, n2 = V2::n2, P = V2::P, EPB = V2::EPB;
  static constexpr int THREADS = V2::THREADS;
  static constexpr int NM = ElasticMat<TI>::kWords;
  static constexpr int US = V2::US, FS = V2::FS;
  static constexpr size_t SMEM = V2::SMEM;
};

// One group of EPB elements (bid), all threads of the CTA (contains
// __syncthreads); also the body of the grouped hexahedron steps.
template <int N, int EPB_, bool TI, bool kFuse>
__device__ __forceinline__ void elastic_hex_affine_body(
    int64_t bid, int64_t E, const float *__restrict__ jac, const float *__restrict__ mat,
    const int32_t *__restrict__ conn, float *__restrict__ u, float *__restrict__ r,
    const DMatrix<float> &Dm, const HexInteriorUpdate &iu) {
  using S = HexAffineShape<N, EPB_, TI>;
  constexpr int n = S::n, n2 = S::n2, P = S::P, EPB = S::EPB, NM = S::NM;
  extern __shared__ __align__(16) float smem_af[];
  const int t = threadIdx.x;
  const int le = t / n2, ij = t - le * n2;
  const int i = ij % n, j = ij / n;
  const int64_t e = bid * EPB + le;
  const bool ok = le < EPB && e < E;
  float *su = smem_af + (size_t)(ok ? le : 0) * S::US;                      // [3][P]
  float *sF = smem_af + (size_t)EPB * S::US + (size_t)(ok ? le : 0) * S::FS;  // [3][2][P]

  float Dri[n], Dsj[n], DTi[n], DTj[n];
#pragma unroll
  for (int l = 0; l < n; ++l) {
    Dri[l] = Dm.d[i * n + l];
    Dsj[l] = Dm.d[j * n + l];
    DTi[l] = Dm.d[l * n + i];
    DTj[l] = Dm.d[l * n + j];
  }
  int32_t node[n];
  float ux[n], uy[n], uz[n];
  if (ok) {
#pragma unroll
    for (int k = 0; k < n; ++k) node[k] = __ldg(conn + e * P + ij + n2 * k);
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const float *up = u + 3 * (int64_t)node[k];
      if constexpr (kFuse) {
        ux[k] = up[0];
        uy[k] = up[1];
        uz[k] = up[2];
      } else {
        ux[k] = __ldg(up + 0);
        uy[k] = __ldg(up + 1);
        uz[k] = __ldg(up + 2);
      }
    }
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
      su[0 * P + p] = ux[k];
      su[1 * P + p] = uy[k];
      su[2 * P + p] = uz[k];
    }
  }
  float J[9];
#pragma unroll
  for (int a = 0; a < 9; ++a) J[a] = ok ? __ldg(jac + e * 9 + a) : 0.f;
  __syncthreads();
  float Ftx[n], Fty[n], Ftz[n];
  if (ok) {
    const int64_t P_E = (int64_t)P * E;
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
      float m[NM];
#pragma unroll
      for (int q = 0; q < NM; ++q) m[q] = __ldg(mat + q * P_E + e * P + p);
      float d[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float *sc = su + c * P;
        const float *uc = c == 0 ? ux : (c == 1 ? uy : uz);
        float dr = 0, ds = 0, dt = 0;
#pragma unroll
        for (int l = 0; l < n; ++l) {
          dr += Dri[l] * sc[l + n * j + n2 * k];
          ds += Dsj[l] * sc[i + n * l + n2 * k];
          dt += Dm.d[k * n + l] * uc[l];
        }
        d[c][0] = dr; d[c][1] = ds; d[c][2] = dt;
      }
      float g[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a)
          g[c][a] = J[a * 3 + 0] * d[c][0] + J[a * 3 + 1] * d[c][1] + J[a * 3 + 2] * d[c][2];
      float sig[3][3];
      if constexpr (TI) stress_ti<float>(g, m, sig);
      else stress_iso<float>(g, m[0], m[1], sig);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float F0 = J[0] * sig[c][0] + J[3] * sig[c][1] + J[6] * sig[c][2];
        const float F1 = J[1] * sig[c][0] + J[4] * sig[c][1] + J[7] * sig[c][2];
        const float F2 = J[2] * sig[c][0] + J[5] * sig[c][1] + J[8] * sig[c][2];
        sF[(c * 2 + 0) * P + p] = F0;
        sF[(c * 2 + 1) * P + p] = F1;
        if (c == 0) Ftx[k] = F2;
        else if (c == 1) Fty[k] = F2;
        else Ftz[k] = F2;
      }
    }
  }
  __syncthreads();
  if (!ok) return;
  // interior column: both in-plane indices strictly inside the element
  const bool icol = kFuse && i >= 1 && i <= n - 2 && j >= 1 && j <= n - 2;
  double t_now = 0;
  if (icol && iu.nsrc > 0) t_now = (double)(*iu.step) * iu.dtd;
#pragma unroll
  for (int k = 0; k < n; ++k) {
    const int p = ij + n2 * k;
    float o[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float *Fr = sF + (c * 2 + 0) * P, *Fs = sF + (c * 2 + 1) * P;
      const float *Ft = c == 0 ? Ftx : (c == 1 ? Fty : Ftz);
      float acc = 0;
#pragma unroll
      for (int l = 0; l < n; ++l) {
        acc += DTi[l] * Fr[l + n * j + n2 * k];
        acc += DTj[l] * Fs[i + n * l + n2 * k];
        acc += Dm.d[l * n + k] * Ft[l];
      }
      o[c] = -acc;
    }
    const bool interior = icol && k >= 1 && k <= n - 2;
    if (!interior) {
#pragma unroll
      for (int c = 0; c < 3; ++c) r[(e * P + p) * 3 + c] = o[c];
      continue;
    }
    if constexpr (kFuse) {
      // sources of this element in attach order (source_body)
      for (int s = 0; s < iu.nsrc; ++s) {
        if (iu.src_elem[s] != e) continue;
        const double stf = ricker_dev(t_now, iu.src_par[3 * s], iu.src_par[3 * s + 1],
                                      iu.src_par[3 * s + 2]);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          o[c] += (float)(iu.src_wts[((int64_t)s * P + p) * 3 + c] * stf);
      }
      // assembly (one incident point: 0 + r), inverse mass, Newmark
      const int64_t g = node[k];
      const float mm = iu.mi[g];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t x = g * 3 + c;
        float uo = c == 0 ? ux[k] : (c == 1 ? uy[k] : uz[k]);
        float vo = iu.v[x], apo = iu.ap[x];
        const float acc = add_rn(0.f, o[c]);
        newmark_point<float>(mul_rn(acc, mm), apo, vo, uo, iu.dt);
        u[x] = uo;
        iu.v[x] = vo;
        iu.ap[x] = apo;
      }
    }
  }
}

template <int N, int EPB_, bool TI, bool kFuse>
__global__ void __launch_bounds__(HexAffineShape<N, EPB_, TI>::THREADS)
elastic_hex_affine_kernel(int64_t E, const float *__restrict__ jac, const float *__restrict__ mat,
                          const int32_t *__restrict__ conn, float *__restrict__ u,
                          float *__restrict__ r, DMatrix<float> Dm, HexInteriorUpdate iu) {
  elastic_hex_affine_body<N, EPB_, TI, kFuse>(blockIdx.x, E, jac, mat, conn, u, r, Dm, iu);
}

}  // namespace salvus
