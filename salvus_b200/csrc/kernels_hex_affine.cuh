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
// kernel finishes them itself -- the one-term assembly 0 + r (the node
// gather's first addition), the inverse mass and the Newmark update
// (newmark_point) -- and writes element-local residuals only for the points
// on the element's faces, which the node gather then assembles over the
// shared nodes alone.  In the few elements that hold a source the interior
// residuals are written too; the source kernel adds the source terms in
// attach order and then finishes those nodes (source_interior_body).  Every operation and its order is the one of the
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

// Interior-node update of the fused step: Newmark state, inverse mass, and
// the elements that hold a source (their interior nodes are finished by the
// source kernel after the source terms are added: source_interior_body).
struct HexInteriorUpdate {
  const float *mi;
  float *v, *ap;
  float dt;
  int nsrc_elem;
  const int64_t *src_elem;  // distinct source elements
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
  // Elements holding a source keep the unfused form for their interior
  // points (residuals written; the source kernel adds the source terms and
  // finishes those nodes).  For the others, the interior operands (v, a_)
  // are loaded here, before the divergence, so that their latency overlaps
  // it (after the stores below the compiler could not reorder them: the
  // pointers may alias as far as it knows).
  bool fuse_here = icol;
  if constexpr (kFuse) {
    for (int s = 0; s < iu.nsrc_elem && fuse_here; ++s) fuse_here = __ldg(iu.src_elem + s) != e;
  }
  float vpre[n][3], apre[n][3];
  if constexpr (kFuse) {
    if (fuse_here) {
      const float *__restrict__ vv = iu.v;
      const float *__restrict__ aa = iu.ap;
#pragma unroll
      for (int k = 1; k < n - 1; ++k) {
        const int64_t g = node[k];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          vpre[k][c] = vv[g * 3 + c];
          apre[k][c] = aa[g * 3 + c];
        }
      }
    }
  }
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
    const bool interior = fuse_here && k >= 1 && k <= n - 2;
    if (!interior) {
#pragma unroll
      for (int c = 0; c < 3; ++c) r[(e * P + p) * 3 + c] = o[c];
      continue;
    }
    if constexpr (kFuse) {
      // assembly (one incident point: 0 + r), inverse mass, Newmark
      const int64_t g = node[k];
      const float mm = __ldg(iu.mi + g);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t x = g * 3 + c;
        float uo = c == 0 ? ux[k] : (c == 1 ? uy[k] : uz[k]);
        float vo = vpre[k][c], apo = apre[k][c];
        const float acc = add_rn(0.f, o[c]);
        newmark_point<float>(mul_rn(acc, mm), apo, vo, uo, iu.dt);
        u[x] = uo;
        iu.v[x] = vo;
        iu.ap[x] = apo;
      }
    }
  }
}

// Source kernel of the fused step (one CTA): the source terms in attach
// order into the element-local residual (source_body), then the interior
// nodes of the distinct source elements -- which the fused stiffness kernel
// left to it -- with the one-term assembly 0 + r, the inverse mass and the
// Newmark update: the arithmetic of the node gather, so the result is the
// unfused sequence's.
template <int N>
__global__ void source_fused_hex_kernel(int nsrc, int P, const int64_t *__restrict__ elem,
                                       const double *__restrict__ par,
                                       const double *__restrict__ wts,
                                       const int64_t *__restrict__ step, double dtd,
                                       float *__restrict__ r, int nse,
                                       const int64_t *__restrict__ src_elems,
                                       const int32_t *__restrict__ conn,
                                       const float *__restrict__ mi, float *__restrict__ u,
                                       float *__restrict__ v, float *__restrict__ ap, float dt) {
  source_body<float, 3>(nsrc, P, elem, par, wts, step, dtd, r);  // ends with __syncthreads
  constexpr int n = N + 1, m = N - 1, NI = m * m * m;
  for (int t = threadIdx.x; t < nse * NI * 3; t += blockDim.x) {
    const int se = t / (NI * 3), rem = t - se * NI * 3, q = rem / 3, c = rem - q * 3;
    const int i = 1 + q % m, j = 1 + (q / m) % m, k = 1 + q / (m * m);
    const int64_t e = src_elems[se];
    const int pt = i + n * j + n * n * k;
    const int64_t g = conn[e * P + pt], x = g * 3 + c;
    float uo = u[x], vo = v[x], apo = ap[x];
    newmark_point<float>(mul_rn(add_rn(0.f, r[(e * P + pt) * 3 + c]), mi[g]), apo, vo, uo, dt);
    u[x] = uo;
    v[x] = vo;
    ap[x] = apo;
  }
}

template <int N, int EPB_, bool TI>
__global__ void __launch_bounds__(HexAffineShape<N, EPB_, TI>::THREADS)
elastic_hex_affine_kernel(int64_t E, const float *__restrict__ jac, const float *__restrict__ mat,
                          const int32_t *__restrict__ conn, float *__restrict__ u,
                          float *__restrict__ r, DMatrix<float> Dm, HexInteriorUpdate iu) {
  elastic_hex_affine_body<N, EPB_, TI, false>(blockIdx.x, E, jac, mat, conn, u, r, Dm, iu);
}

// The fused form asks for 768 resident threads per SM (six 128-thread CTAs,
// a register cap): its interior-update registers would otherwise cost two
// CTAs per SM.
template <int THREADS>
constexpr int fuse_min_blocks() {
  return 768 / THREADS > 0 ? 768 / THREADS : 1;
}
template <int N, int EPB_, bool TI>
__global__ void __launch_bounds__(HexAffineShape<N, EPB_, TI>::THREADS,
                                  fuse_min_blocks<HexAffineShape<N, EPB_, TI>::THREADS>())
elastic_hex_affine_fused_kernel(int64_t E, const float *__restrict__ jac,
                                const float *__restrict__ mat, const int32_t *__restrict__ conn,
                                float *__restrict__ u, float *__restrict__ r, DMatrix<float> Dm,
                                HexInteriorUpdate iu) {
  elastic_hex_affine_body<N, EPB_, TI, true>(blockIdx.x, E, jac, mat, conn, u, r, Dm, iu);
}

}  // namespace salvus
