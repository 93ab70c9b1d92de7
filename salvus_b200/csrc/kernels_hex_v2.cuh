// kernels_hex_v2.cuh -- FP32 elastic hexahedron stiffness, column threads
// with 32-bit shared-memory planes.
//
// Same arithmetic as elastic_hex_stiffness_kernel (Elastic3D.cpp:70-118 via
// Hexahedra.cpp:580-632 / 689-754).  Differences that matter on B200:
//  * operands of the r- and s-contractions are read as 32-bit words, which
//    the shared-memory crossbar broadcasts to the n column threads of an
//    r- or s-line in one wavefront (128-bit reads cannot share a wavefront);
//  * each element's planes start at a word offset congruent to n^2 mod 32
//    (the element's thread count), so a warp whose 32 column threads
//    straddle two elements touches 32 distinct banks on every store;
//  * connectivity comes from word 11 of each 48-byte record, so no separate
//    connectivity stream is read; the record's last float4 (J8, lambda', mu',
//    conn) is fetched first to start the displacement gather early;
//  * records are three (transversely isotropic: four) float4 planes per
//    element ([E][3|4][P]), so the 32 lanes of a warp load 512 contiguous
//    bytes per instruction.
#pragma once

#include <cstdint>

#include "kernels_material.cuh"

namespace salvus {

// smallest w' >= w with w' = m (mod 32)
__host__ __device__ constexpr int pad_to_mod32(int w, int m) { return w + ((m - (w % 32)) + 32) % 32; }

template <int N, int EPB_, bool TI = false>
struct ElasticV2Shape {
  static constexpr int n = N + 1, n2 = n * n, P = n2 * n;
  static constexpr int EPB = EPB_;
  static constexpr int THREADS = ((EPB * n2 + 31) / 32) * 32;
  // float4 record planes per element: isotropic 3, transversely isotropic 4
  static constexpr int PLANES = TI ? 4 : 3;
  // padded per-element strides (words): u planes 3P, F planes 6P
  static constexpr int US = pad_to_mod32(3 * P, n2 % 32);
  static constexpr int FS = pad_to_mod32(6 * P, n2 % 32);
  static constexpr size_t SMEM = sizeof(float) * (size_t)EPB * (US + FS);
};

// Records ([E][PLANES][P] float4): plane 0 = invJ 0-3, plane 1 = invJ 4-7,
// plane 2 = (invJ 8, m0, m1, conn); TI adds plane 3 = (m2, m3, m4, 0), where
// m = (lambda', mu') for isotropic and (A', C', F', L', N') for transversely
// isotropic material (kernels_material.cuh).
template <int N, int EPB_, bool TI>
__device__ __forceinline__ void elastic_hex_v2_body(int64_t bid, int64_t E,
                                                    const float *__restrict__ rec,
                                                    const float *__restrict__ u,
                                                    float *__restrict__ r, const DMatrix<float> &Dm) {
  using S = ElasticV2Shape<N, EPB_, TI>;
  constexpr int n = S::n, n2 = S::n2, P = S::P, EPB = S::EPB;
  extern __shared__ __align__(16) float smem_v2[];
  const int t = threadIdx.x;
  const int le = t / n2, ij = t - le * n2;
  const int i = ij % n, j = ij / n;
  const int64_t e = bid * EPB + le;
  const bool ok = le < EPB && e < E;
  float *su = smem_v2 + (size_t)(ok ? le : 0) * S::US;                      // [3][P]
  float *sF = smem_v2 + (size_t)EPB * S::US + (size_t)(ok ? le : 0) * S::FS;  // [3][2][P]
  const float4 *rq = reinterpret_cast<const float4 *>(rec) + (e * S::PLANES) * P;

  float Dri[n], Dsj[n], DTi[n], DTj[n];
#pragma unroll
  for (int l = 0; l < n; ++l) {
    Dri[l] = Dm.d[i * n + l];
    Dsj[l] = Dm.d[j * n + l];
    DTi[l] = Dm.d[l * n + i];
    DTj[l] = Dm.d[l * n + j];
  }
  float ux[n], uy[n], uz[n];
  float4 rc[n];  // (J8, m0, m1, conn) per point of the column
  if (ok) {
#pragma unroll
    for (int k = 0; k < n; ++k) rc[k] = __ldg(rq + 2 * P + ij + n2 * k);
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int64_t node = __float_as_int(rc[k].w);
      ux[k] = __ldg(u + 3 * node + 0);
      uy[k] = __ldg(u + 3 * node + 1);
      uz[k] = __ldg(u + 3 * node + 2);
    }
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
      su[0 * P + p] = ux[k];
      su[1 * P + p] = uy[k];
      su[2 * P + p] = uz[k];
    }
  }
  __syncthreads();
  float Ftx[n], Fty[n], Ftz[n];
  if (ok) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
      const float4 ra = __ldg(rq + p);
      const float4 rb = __ldg(rq + P + p);
      const float J[9] = {ra.x, ra.y, ra.z, ra.w, rb.x, rb.y, rb.z, rb.w, rc[k].x};
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
      if constexpr (TI) {
        const float4 rt = __ldg(rq + 3 * P + p);
        const float m[5] = {rc[k].y, rc[k].z, rt.x, rt.y, rt.z};
        stress_ti<float>(g, m, sig);
      } else {
        stress_iso<float>(g, rc[k].y, rc[k].z, sig);
      }
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
  if (ok) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float *Fr = sF + (c * 2 + 0) * P, *Fs = sF + (c * 2 + 1) * P;
        const float *Ft = c == 0 ? Ftx : (c == 1 ? Fty : Ftz);
        float o = 0;
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

template <int N, int EPB_, bool TI>
__global__ void __launch_bounds__(ElasticV2Shape<N, EPB_, TI>::THREADS)
elastic_hex_stiffness_v2_kernel(int64_t E, const float *__restrict__ rec,
                                const float *__restrict__ u, float *__restrict__ r,
                                DMatrix<float> Dm) {
  elastic_hex_v2_body<N, EPB_, TI>(blockIdx.x, E, rec, u, r, Dm);
}

}  // namespace salvus
