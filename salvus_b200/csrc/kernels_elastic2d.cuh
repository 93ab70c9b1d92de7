// kernels_elastic2d.cuh -- per-element stiffness action of 2-D elastic
// quadrilaterals (Elastic2D<TensorQuad<QuadP1>>), r_e = -K_e u_e, written to
// the element-local residual r[E][P][C] like every other element class.
//
// Reference arithmetic restated (Elastic2D.cpp:84-107): strain from two
// gradients (ux_x, ux_y, uy_x, uy_y; TensorQuad::computeGradient
// TensorQuad.cpp:177-210), stress (Elastic2D.cpp:62-78)
//   sxx = C11 ux_x + C13 uy_y,  syy = C13 ux_x + C33 uy_y,
//   sxy = C55 (ux_y + uy_x)
// (the reference's c13 / c23 coupling slots are never set and stay zero,
// Elastic2D.cpp:16-21,55-56), then two gradient-test integrals of (sxx, sxy)
// and (sxy, syy) (TensorQuad::applyGradTestAndIntegrate TensorQuad.cpp:351-397,
// in its per-quadrature-point form).
//
// One thread per element point, EPB elements per CTA; the two displacement
// components of the CTA's elements and the four reference-direction fluxes
// go through shared memory.  The body takes the node-field stride C and the
// first component OFF so that the same code serves meshes whose nodes carry
// further fields, and an optional element list (CTA k-th element -> mesh
// element) for meshes that mix element classes.
#pragma once

#include <cstdint>

namespace salvus {

// EPB_ = 0: as many elements as fit 256 threads
template <int N, int EPB_ = 0>
struct Elastic2DShape {
  static constexpr int n = N + 1;
  static constexpr int P = n * n;
  static constexpr int EPB = EPB_ > 0 ? EPB_ : ((256 / P) > 0 ? (256 / P) : 1);
  static constexpr int THREADS = ((EPB * P + 31) / 32) * 32;
};

// FP32 records: two float4 planes per element, [E][2][P] float4:
//   plane 0 = invJ (dxi/dx, deta/dx, dxi/dy, deta/dy)
//   plane 1 = (C11, C13, C33, C55) * w detJ
// so consecutive points of one plane are consecutive 16-byte words.
// FP64 records: [E][P][8] in the same word order.
__device__ __forceinline__ void load_elastic2d_rec(const float *__restrict__ rec, int64_t k, int p,
                                                   int P, float *J, float *c) {
  const float4 *q = reinterpret_cast<const float4 *>(rec) + k * 2 * P + p;
  const float4 a = __ldg(q), b = __ldg(q + P);
  J[0] = a.x; J[1] = a.y; J[2] = a.z; J[3] = a.w;
  c[0] = b.x; c[1] = b.y; c[2] = b.z; c[3] = b.w;
}
__device__ __forceinline__ void load_elastic2d_rec(const double *__restrict__ rec, int64_t k, int p,
                                                   int P, double *J, double *c) {
  const double *q = rec + (k * P + p) * 8;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    J[a] = q[a];
    c[a] = q[4 + a];
  }
}

// bid: element-group index.  nE elements are processed (the mesh's, or the
// list's length); record k of the group's k-th element, residual and
// connectivity of mesh element elist[k] (k itself without a list).
template <int N, typename real, int C, int OFF, int EPB_ = 0>
__device__ __forceinline__ void elastic2d_body(int64_t bid, int64_t nE,
                                               const int32_t *__restrict__ elist,
                                               const real *__restrict__ rec,
                                               const int32_t *__restrict__ conn,
                                               const real *__restrict__ u, real *__restrict__ r,
                                               const DMatrix<real> &Dm) {
  using S = Elastic2DShape<N, EPB_>;
  constexpr int n = S::n, P = S::P, EPB = S::EPB;
  __shared__ real sD[n * n];
  __shared__ real su[EPB][2][P];
  __shared__ real sF[EPB][4][P];
  const int t = threadIdx.x;
  const int le = t / P, p = t - le * P;
  if (t < n * n) sD[t] = Dm.d[t];
  const int64_t k = bid * EPB + le;
  const bool ok = le < EPB && k < nE;
  int64_t e = 0;
  real J[4], cw[4];
  if (ok) {
    e = elist ? (int64_t)elist[k] : k;
    load_elastic2d_rec(rec, k, p, P, J, cw);
    const int64_t node = conn[e * P + p];
    su[le][0][p] = u[node * C + OFF];
    su[le][1][p] = u[node * C + OFF + 1];
  }
  __syncthreads();
  const int i = p % n, j = p / n;
  if (ok) {
    real dxr = 0, dxs = 0, dyr = 0, dys = 0;
#pragma unroll
    for (int l = 0; l < n; ++l) {
      const real a = sD[i * n + l], b = sD[j * n + l];
      dxr += a * su[le][0][l + n * j];
      dxs += b * su[le][0][i + n * l];
      dyr += a * su[le][1][l + n * j];
      dys += b * su[le][1][i + n * l];
    }
    // physical gradients: d/dx_a = sum_k invJ[a][k] d/dxi_k
    const real uxx = J[0] * dxr + J[1] * dxs, uxy = J[2] * dxr + J[3] * dxs;
    const real uyx = J[0] * dyr + J[1] * dys, uyy = J[2] * dyr + J[3] * dys;
    const real sxx = cw[0] * uxx + cw[1] * uyy;
    const real syy = cw[1] * uxx + cw[2] * uyy;
    const real sxy = cw[3] * (uxy + uyx);
    // reference-direction fluxes F_k = sum_a invJ[a][k] sigma_a
    sF[le][0][p] = J[0] * sxx + J[2] * sxy;
    sF[le][1][p] = J[1] * sxx + J[3] * sxy;
    sF[le][2][p] = J[0] * sxy + J[2] * syy;
    sF[le][3][p] = J[1] * sxy + J[3] * syy;
  }
  __syncthreads();
  if (ok) {
    real ox = 0, oy = 0;
#pragma unroll
    for (int l = 0; l < n; ++l) {
      const real a = sD[l * n + i], b = sD[l * n + j];
      ox += a * sF[le][0][l + n * j] + b * sF[le][1][i + n * l];
      oy += a * sF[le][2][l + n * j] + b * sF[le][3][i + n * l];
    }
    r[(e * P + p) * C + OFF] = -ox;
    r[(e * P + p) * C + OFF + 1] = -oy;
    // components of other element classes (meshes of fluid and solid elements)
#pragma unroll
    for (int c = 0; c < C; ++c)
      if (c < OFF || c > OFF + 1) r[(e * P + p) * C + c] = real(0);
  }
}

template <int N, typename real, int C, int OFF, int EPB_ = 0>
__global__ void __launch_bounds__(Elastic2DShape<N, EPB_>::THREADS)
elastic2d_stiffness_kernel(int64_t nE, const int32_t *__restrict__ elist,
                           const real *__restrict__ rec, const int32_t *__restrict__ conn,
                           const real *__restrict__ u, real *__restrict__ r, DMatrix<real> Dm) {
  elastic2d_body<N, real, C, OFF, EPB_>(blockIdx.x, nE, elist, rec, conn, u, r, Dm);
}

}  // namespace salvus
