// kernels_simplex.cuh -- P3 mass-lumped triangles (12 nodes) and tetrahedra
// (50 nodes): one-time FP64 geometry records and the per-step stiffness
// action r_e = -K_e u_e on CUDA cores (FP32 or FP64), written element-local
// like the tensor kernels so that the node-gather update assembles it in a
// fixed order.
//
// Reference arithmetic restated:
//   geometry   TriP1::inverseJacobian (TriP1.cpp:56-94),
//              TetP1::inverseJacobian (TetP1.cpp:91-150), material at the
//              nodes by ParAtIntPts (Triangle.cpp:408-428,
//              Tetrahedra.cpp:186-197) with the P1 vertex weights of
//              interpolateAtPoint (TriP1.cpp:96-109, TetP1.cpp:45-60);
//   mass       applyTestAndIntegrate (Triangle.cpp:349-355,
//              Tetrahedra.cpp:486-492): w_q detJ (x rho for elastic);
//   triangle   ScalarTri::computeStiffnessTerm (ScalarTri.cpp:12-17) applies
//              the dense K_e of Triangle::buildStiffnessMatrix
//              (Triangle.cpp:194-241), K_ij = detJ sum_q w_q vp_q^2
//              grad phi_i . grad phi_j (x_q); it is applied here in factored
//              form (reference gradient, metric, divergence) so the record
//              is 16 words per element instead of 144;
//   tetrahedron Scalar<Tetrahedra>: computeGradient (Tetrahedra.cpp:235-245)
//              times vp^2, then applyGradTestAndIntegrate (:248-274);
//   tet elastic (no reference element): Elastic3D::computeStiffnessTerm
//              (Elastic3D.cpp:70-118) with the tetrahedron's gradient and
//              gradient-test operators, isotropic lambda / mu.
//
// Records (one per element; affine geometry is constant over the element):
//   triangle acoustic     [G00 G01 G11 0 | s_0 .. s_11]            16 words
//   tetrahedron acoustic  [G00 G01 G02 G11 G12 G22 0 0 | s_0..s_49 | 0 x6]    64
//   tetrahedron elastic   [invJ (9) 0 x3 | lw_0..lw_49 | 0 0 | mw_0..mw_49 | 0 x6]
//                                                                            120
//   tetrahedron elastic, transversely isotropic
//                         [invJ (9) 0 x3 | A' 0 0 | C' 0 0 | F' 0 0 | L' 0 0 | N' | 0 x10]
//                                                                            280
// (padded so that every 8-node run of s / lw / mw starts on 16 bytes and an
// 8-node run that starts at node 48 stays inside the record)
// with G = detJ invJ^T invJ (invJ[x_a][xi_b] = d xi_b / d x_a), s_q = w_q vp_q^2,
// lw_q = w_q detJ lambda_q, mw_q = w_q detJ mu_q, and the transversely
// isotropic constants (kernels_material.cuh) times w_q detJ.
#pragma once

#include <cstdint>

#include "kernels_material.cuh"

namespace salvus {

struct SimplexTable {
  double x[50][3];  // node reference coordinates
  double w[50];     // nodal quadrature weights
};

constexpr int kTriRec = 16, kTetAcRec = 64, kTetElRec = 120, kTetTiRec = 280;
constexpr int kTetLambda = 12, kTetMu = 64;
// per-node material arrays of elastic tetrahedra start at kTetLambda +
// kTetMatStride * m (m = 0, 1 isotropic; m = 0..4 transversely isotropic)
constexpr int kTetMatStride = 52;

// One thread per element.
template <typename real>
__global__ void simplex_geometry_kernel(int64_t E, int shape, int physics, int P, int rw,
                                        const double *__restrict__ vtx,
                                        const double *__restrict__ par, SimplexTable tab,
                                        real *__restrict__ rec, double *__restrict__ mass_local,
                                        bool ti = false) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const bool tri = shape == 2;
  const int nv = tri ? 3 : 4, dim = tri ? 2 : 3;
  double v[12];
  for (int a = 0; a < nv * dim; ++a) v[a] = vtx[e * nv * dim + a];
  double det, iJ[9];
  if (tri) {
    const double J0 = 0.5 * (v[2] - v[0]), J1 = 0.5 * (v[3] - v[1]);
    const double J2 = 0.5 * (v[4] - v[0]), J3 = 0.5 * (v[5] - v[1]);
    det = J0 * J3 - J1 * J2;
    iJ[0] = J3 / det; iJ[1] = -J1 / det; iJ[2] = -J2 / det; iJ[3] = J0 / det;
  } else {
    double J[9];
    for (int m = 0; m < 3; ++m) {
      J[m] = v[6 + m] - v[m];
      J[3 + m] = v[3 + m] - v[m];
      J[6 + m] = v[9 + m] - v[m];
    }
    const double m00 = J[4] * J[8] - J[5] * J[7], m01 = J[5] * J[6] - J[3] * J[8],
                 m02 = J[3] * J[7] - J[4] * J[6];
    det = J[0] * m00 + J[1] * m01 + J[2] * m02;
    const double id = 1.0 / det;
    iJ[0] = m00 * id;
    iJ[1] = (J[2] * J[7] - J[1] * J[8]) * id;
    iJ[2] = (J[1] * J[5] - J[2] * J[4]) * id;
    iJ[3] = m01 * id;
    iJ[4] = (J[0] * J[8] - J[2] * J[6]) * id;
    iJ[5] = (J[2] * J[3] - J[0] * J[5]) * id;
    iJ[6] = m02 * id;
    iJ[7] = (J[1] * J[6] - J[0] * J[7]) * id;
    iJ[8] = (J[0] * J[4] - J[1] * J[3]) * id;
  }
  real *out = rec + e * rw;
  for (int a = 0; a < rw; ++a) out[a] = 0;
  const int npar = physics == 0 ? 1 : (ti ? 6 : 3);
  for (int q = 0; q < P; ++q) {
    const double r = tab.x[q][0], s = tab.x[q][1], t = tab.x[q][2];
    double lw[4];
    if (tri) {
      lw[0] = -0.5 * (r + s); lw[1] = 0.5 * (r + 1.0); lw[2] = 0.5 * (s + 1.0); lw[3] = 0;
    } else {
      lw[0] = 1.0 - r - s - t; lw[1] = s; lw[2] = r; lw[3] = t;
    }
    double pv[6];
    for (int k = 0; k < npar; ++k) {
      double acc = 0;
      for (int a = 0; a < nv; ++a) acc += lw[a] * par[((int64_t)k * E + e) * nv + a];
      pv[k] = acc;
    }
    const double wd = tab.w[q] * det;
    if (physics == 0) {
      out[(tri ? 4 : 8) + q] = (real)(tab.w[q] * pv[0] * pv[0]);
      mass_local[e * P + q] = wd;
    } else {
      double mc[5];
      const int nm = ti ? 5 : 2;
      if (ti) elastic_constants_ti(pv, mc);
      else elastic_constants_iso(pv[0], pv[1], pv[2], mc);
      for (int m = 0; m < nm; ++m) out[kTetLambda + kTetMatStride * m + q] = (real)(wd * mc[m]);
      mass_local[e * P + q] = wd * pv[0];
    }
  }
  if (physics == 0) {
    if (tri) {
      out[0] = (real)(det * (iJ[0] * iJ[0] + iJ[2] * iJ[2]));
      out[1] = (real)(det * (iJ[0] * iJ[1] + iJ[2] * iJ[3]));
      out[2] = (real)(det * (iJ[1] * iJ[1] + iJ[3] * iJ[3]));
    } else {
      int k = 0;
      for (int b = 0; b < 3; ++b)
        for (int c = b; c < 3; ++c)
          out[k++] = (real)(det * (iJ[b] * iJ[c] + iJ[3 + b] * iJ[3 + c] + iJ[6 + b] * iJ[6 + c]));
    }
  } else {
    for (int a = 0; a < 9; ++a) out[a] = (real)iJ[a];
  }
}

// ---------------------------------------------------------------------------
// Triangle, acoustic: one thread per element; the 2 x 12 x 12 derivative
// table sits in shared memory and every lane reads the same entry (broadcast).
template <typename real>
__global__ void __launch_bounds__(128)
tri_acoustic_kernel(int64_t E, const real *__restrict__ rec, const int32_t *__restrict__ conn,
                    const real *__restrict__ SD, const real *__restrict__ u, real *__restrict__ r) {
  constexpr int P = 12;
  __shared__ real sD[2 * P * P];
  for (int i = threadIdx.x; i < 2 * P * P; i += blockDim.x) sD[i] = SD[i];
  __syncthreads();
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const real *rc = rec + e * kTriRec;
  const real g00 = rc[0], g01 = rc[1], g11 = rc[2];
  real ue[P], acc[P];
#pragma unroll
  for (int j = 0; j < P; ++j) {
    ue[j] = u[conn[e * P + j]];
    acc[j] = 0;
  }
  // per quadrature node: reference gradient, metric and material, then its
  // contribution to every test function (keeps the live set at ~2P values)
#pragma unroll 2
  for (int q = 0; q < P; ++q) {
    real a0 = 0, a1 = 0;
#pragma unroll
    for (int j = 0; j < P; ++j) {
      a0 += sD[j * P + q] * ue[j];
      a1 += sD[P * P + j * P + q] * ue[j];
    }
    const real s = rc[4 + q];
    const real f0 = s * (g00 * a0 + g01 * a1);
    const real f1 = s * (g01 * a0 + g11 * a1);
#pragma unroll
    for (int i = 0; i < P; ++i) acc[i] += sD[i * P + q] * f0 + sD[P * P + i * P + q] * f1;
  }
#pragma unroll
  for (int i = 0; i < P; ++i) r[e * P + i] = -acc[i];
}

// The triangle's derivative table (2 x 12 x 12, the same for every mesh) in
// constant memory: with the loops fully unrolled every table entry is a
// compile-time constant-bank operand of its FMA, so the contractions issue
// no shared-memory loads at all (the shared-table kernel above is L1-bound).
__constant__ float c_tri_sd32[2 * 12 * 12];
__constant__ double c_tri_sd64[2 * 12 * 12];
template <typename real>
__device__ __forceinline__ real tri_sd(int i) {
  if constexpr (sizeof(real) == 4) return c_tri_sd32[i];
  else return c_tri_sd64[i];
}

// Same arithmetic and summation order as tri_acoustic_kernel.
template <typename real>
__global__ void __launch_bounds__(128)
tri_acoustic_const_kernel(int64_t E, const real *__restrict__ rec,
                          const int32_t *__restrict__ conn, const real *__restrict__ u,
                          real *__restrict__ r) {
  constexpr int P = 12;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  // the element's record, connectivity and residual as 16-byte words
  // (record 64 B, connectivity 48 B, residual 48 B per FP32 element)
  real rc[kTriRec];
  int32_t cn[P];
  if constexpr (sizeof(real) == 4) {
    const float4 *r4 = reinterpret_cast<const float4 *>(rec + e * kTriRec);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const float4 x = __ldg(r4 + v);
      rc[4 * v] = x.x; rc[4 * v + 1] = x.y; rc[4 * v + 2] = x.z; rc[4 * v + 3] = x.w;
    }
    const int4 *c4 = reinterpret_cast<const int4 *>(conn + e * P);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const int4 x = __ldg(c4 + v);
      cn[4 * v] = x.x; cn[4 * v + 1] = x.y; cn[4 * v + 2] = x.z; cn[4 * v + 3] = x.w;
    }
  } else {
#pragma unroll
    for (int a = 0; a < kTriRec; ++a) rc[a] = rec[e * kTriRec + a];
#pragma unroll
    for (int j = 0; j < P; ++j) cn[j] = conn[e * P + j];
  }
  const real g00 = rc[0], g01 = rc[1], g11 = rc[2];
  real ue[P], acc[P];
#pragma unroll
  for (int j = 0; j < P; ++j) {
    ue[j] = u[cn[j]];
    acc[j] = 0;
  }
#pragma unroll
  for (int q = 0; q < P; ++q) {
    real a0 = 0, a1 = 0;
#pragma unroll
    for (int j = 0; j < P; ++j) {
      a0 += tri_sd<real>(j * P + q) * ue[j];
      a1 += tri_sd<real>(P * P + j * P + q) * ue[j];
    }
    const real s = rc[4 + q];
    const real f0 = s * (g00 * a0 + g01 * a1);
    const real f1 = s * (g01 * a0 + g11 * a1);
#pragma unroll
    for (int i = 0; i < P; ++i)
      acc[i] += tri_sd<real>(i * P + q) * f0 + tri_sd<real>(P * P + i * P + q) * f1;
  }
  if constexpr (sizeof(real) == 4) {
    float4 *o4 = reinterpret_cast<float4 *>(r + e * P);
#pragma unroll
    for (int v = 0; v < 3; ++v)
      o4[v] = make_float4(-acc[4 * v], -acc[4 * v + 1], -acc[4 * v + 2], -acc[4 * v + 3]);
  } else {
#pragma unroll
    for (int i = 0; i < P; ++i) r[e * P + i] = -acc[i];
  }
}

// ---------------------------------------------------------------------------
// Tetrahedron (acoustic C = 1, elastic C = 3) on CUDA cores: one thread per
// element node, EPB elements per CTA.  The derivative table is held twice in
// shared memory, [k][j][q] for the gradient (lanes walk q) and [k][q][i] for
// the divergence (lanes walk i), so both contractions are bank-conflict-free.
template <typename real, int C, bool TI = false>
struct TetShape {
  static constexpr int P = 50;
  static constexpr int EPB = sizeof(real) == 4 ? 8 : 4;
  static constexpr int THREADS = EPB * P;
  static constexpr int RW = C == 1 ? kTetAcRec : (TI ? kTetTiRec : kTetElRec);
  static constexpr int NF = C == 1 ? 3 : 9;  // flux words per node
  static constexpr size_t SMEM =
      sizeof(real) * (size_t)(2 * 3 * P * P + EPB * P * C + EPB * P * NF + EPB * RW);
};

template <typename real, int C, bool TI = false>
__global__ void __launch_bounds__(TetShape<real, C, TI>::THREADS)
tet_stiffness_kernel(int64_t E, const real *__restrict__ rec, const int32_t *__restrict__ conn,
                     const real *__restrict__ SD, const real *__restrict__ u,
                     real *__restrict__ r) {
  using S = TetShape<real, C, TI>;
  constexpr int P = S::P, EPB = S::EPB, RW = S::RW, NF = S::NF, PP = P * P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  real *sD = reinterpret_cast<real *>(smem_raw);  // [3][j][q]
  real *sT = sD + 3 * PP;                         // [3][q][i]
  real *su = sT + 3 * PP;                         // [EPB][P][C]
  real *sF = su + EPB * P * C;                    // [EPB][P][NF]
  real *sR = sF + EPB * P * NF;                   // [EPB][RW]
  const int t = threadIdx.x;
  for (int x = t; x < 3 * PP; x += S::THREADS) {
    const int k = x / PP, rem = x - k * PP, j = rem / P, q = rem - j * P;
    const real d = SD[x];
    sD[x] = d;
    sT[k * PP + q * P + j] = d;
  }
  const int64_t e0 = (int64_t)blockIdx.x * EPB;
  const int nel = (int)((E - e0) < EPB ? (E - e0) : EPB);
  for (int x = t; x < nel * RW; x += S::THREADS) sR[x] = rec[e0 * RW + x];
  const int le = t / P, q = t - le * P;
  const bool ok = le < nel;
  const int64_t e = e0 + le;
  if (ok) {
    const int32_t node = conn[e * P + q];
#pragma unroll
    for (int c = 0; c < C; ++c) su[(le * P + q) * C + c] = u[(int64_t)node * C + c];
  }
  __syncthreads();
  if (ok) {
    // reference gradient of every component at node q
    real gr[C][3];
#pragma unroll
    for (int c = 0; c < C; ++c) gr[c][0] = gr[c][1] = gr[c][2] = 0;
    const real *ue = su + le * P * C;
#pragma unroll 5
    for (int j = 0; j < P; ++j) {
      const real d0 = sD[j * P + q], d1 = sD[PP + j * P + q], d2 = sD[2 * PP + j * P + q];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const real uj = ue[j * C + c];
        gr[c][0] += d0 * uj;
        gr[c][1] += d1 * uj;
        gr[c][2] += d2 * uj;
      }
    }
    const real *rc = sR + le * RW;
    real *F = sF + (le * P + q) * NF;
    if constexpr (C == 1) {
      const real s = rc[8 + q];
      F[0] = s * (rc[0] * gr[0][0] + rc[1] * gr[0][1] + rc[2] * gr[0][2]);
      F[1] = s * (rc[1] * gr[0][0] + rc[3] * gr[0][1] + rc[4] * gr[0][2]);
      F[2] = s * (rc[2] * gr[0][0] + rc[4] * gr[0][1] + rc[5] * gr[0][2]);
    } else {
      // physical gradient g[a][x] = sum_k invJ[x][k] gr[a][k]
      real g[3][3];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int x = 0; x < 3; ++x)
          g[a][x] = rc[x * 3 + 0] * gr[a][0] + rc[x * 3 + 1] * gr[a][1] + rc[x * 3 + 2] * gr[a][2];
      real sig[3][3];
      if constexpr (TI) {
        real mc[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) mc[m] = rc[kTetLambda + kTetMatStride * m + q];
        stress_ti<real>(g, mc, sig);
      } else {
        const real lw = rc[kTetLambda + q], mw = rc[kTetMu + q];
        const real tr = lw * (g[0][0] + g[1][1] + g[2][2]);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int x = 0; x < 3; ++x) sig[a][x] = mw * (g[a][x] + g[x][a]) + (a == x ? tr : real(0));
      }
      // reference flux F[a][k] = sum_x invJ[x][k] sigma[a][x]
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int k = 0; k < 3; ++k)
          F[a * 3 + k] = rc[0 * 3 + k] * sig[a][0] + rc[1 * 3 + k] * sig[a][1] + rc[2 * 3 + k] * sig[a][2];
    }
  }
  __syncthreads();
  if (ok) {
    const int i = q;
    real acc[C];
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] = 0;
    const real *Fe = sF + le * P * NF;
#pragma unroll 5
    for (int p = 0; p < P; ++p) {
      const real d0 = sT[p * P + i], d1 = sT[PP + p * P + i], d2 = sT[2 * PP + p * P + i];
#pragma unroll
      for (int c = 0; c < C; ++c)
        acc[c] += d0 * Fe[p * NF + c * 3 + 0] + d1 * Fe[p * NF + c * 3 + 1] +
                  d2 * Fe[p * NF + c * 3 + 2];
    }
#pragma unroll
    for (int c = 0; c < C; ++c) r[(e * P + i) * C + c] = -acc[c];
  }
}

}  // namespace salvus
