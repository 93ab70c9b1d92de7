// kernels_quad_col.cuh -- column-threaded stiffness kernels for
// quadrilaterals (acoustic Scalar and Elastic2D physics).
//
// One thread owns the n points of one i-column of an element (p = i + n j,
// j = 0..n-1): the eta-derivatives and the eta part of the divergence run
// along the thread's own column in registers with compile-time derivative
// entries, and only the xi direction goes through shared memory.  Per point
// that is 2n shared-memory loads instead of the 4n-8n of one thread per
// point, which is what limits the point-threaded kernels (their L1 / shared
// pipe runs at 80-90 % while DRAM runs at 35-45 %).  The records and the
// column's field values are loaded before the first barrier so that their
// latencies overlap.
//
// Arithmetic and summation order per point are those of the point-threaded
// bodies (kernels_stiffness.cuh, kernels_elastic2d.cuh); only the loop
// structure changes.
#pragma once

#include <cstdint>

namespace salvus {

// default elements per CTA: ~128-thread CTAs (one thread per column)
template <int N>
constexpr int quad_col_epb() {
  return 128 / (N + 1) > 0 ? 128 / (N + 1) : 1;
}

template <int N, int EPB_>
struct QuadColShape {
  static constexpr int n = N + 1;
  static constexpr int P = n * n;
  static constexpr int EPB = EPB_;
  static constexpr int THREADS = ((EPB * n + 31) / 32) * 32;
};

// Acoustic quads: r_e = -K_e u_e with G = w detJ vp^2 invJ^T invJ per point.
// C / kList as in acoustic_stiffness_body (fluid elements of fluid-solid
// meshes own component 0 of C and come from a list).
template <int N, int EPB, typename real, int C = 1, bool kList = false>
__device__ __forceinline__ void acoustic_quad_col_body(int64_t bid, int64_t nE,
                                                       const real *__restrict__ rec,
                                                       const int32_t *__restrict__ conn,
                                                       const real *__restrict__ u,
                                                       real *__restrict__ r,
                                                       const DMatrix<real> &Dm,
                                                       const int32_t *__restrict__ elist = nullptr) {
  using S = QuadColShape<N, EPB>;
  constexpr int n = S::n, P = S::P;
  __shared__ real sD[n * n];
  __shared__ real su[EPB][P];
  __shared__ real sF[EPB][P];
  const int t = threadIdx.x;
  const int le = t / n, i = t - le * n;
  const int64_t k = bid * EPB + le;
  const bool ok = le < EPB && k < nE;
  int64_t e = k;
  real g0[n], g1[n], g2[n], uu[n];
  if (t < n * n) sD[t] = Dm.d[t];
  if (ok) {
    if constexpr (kList) e = elist[k];
    int32_t node[n];
#pragma unroll
    for (int j = 0; j < n; ++j) {
      real g[3];
      load_acoustic_rec<2>(rec, conn, k * P + i + n * j, e * P + i + n * j, g, &node[j]);
      g0[j] = g[0];
      g1[j] = g[1];
      g2[j] = g[2];
    }
#pragma unroll
    for (int j = 0; j < n; ++j) {
      uu[j] = u[(int64_t)node[j] * C];
      su[le][i + n * j] = uu[j];
    }
  }
  __syncthreads();
  real Dri[n], DTi[n];
#pragma unroll
  for (int l = 0; l < n; ++l) {
    Dri[l] = sD[i * n + l];
    DTi[l] = sD[l * n + i];
  }
  real Fs[n];
  if (ok) {
#pragma unroll
    for (int j = 0; j < n; ++j) {
      real gr = 0, gs = 0;
#pragma unroll
      for (int l = 0; l < n; ++l) {
        gr += Dri[l] * su[le][l + n * j];
        gs += Dm.d[j * n + l] * uu[l];
      }
      sF[le][i + n * j] = g0[j] * gr + g1[j] * gs;
      Fs[j] = g1[j] * gr + g2[j] * gs;
    }
  }
  __syncthreads();
  if (ok) {
#pragma unroll
    for (int j = 0; j < n; ++j) {
      real out = 0;
#pragma unroll
      for (int l = 0; l < n; ++l) {
        out += DTi[l] * sF[le][l + n * j];
        out += Dm.d[l * n + j] * Fs[l];
      }
      const int64_t o = (e * P + i + n * j) * C;
      r[o] = -out;
#pragma unroll
      for (int c = 1; c < C; ++c) r[o + c] = real(0);
    }
  }
}

template <int N, int EPB, typename real>
__global__ void __launch_bounds__(QuadColShape<N, EPB>::THREADS)
acoustic_quad_col_kernel(int64_t E, const real *__restrict__ rec, const int32_t *__restrict__ conn,
                         const real *__restrict__ u, real *__restrict__ r, DMatrix<real> Dm) {
  acoustic_quad_col_body<N, EPB, real>(blockIdx.x, E, rec, conn, u, r, Dm);
}

template <int N, int EPB, typename real>
__global__ void __launch_bounds__(QuadColShape<N, EPB>::THREADS)
acoustic_quad_col_list_kernel(int64_t nE, const int32_t *__restrict__ elist,
                              const real *__restrict__ rec, const int32_t *__restrict__ conn,
                              const real *__restrict__ u, real *__restrict__ r, DMatrix<real> Dm) {
  acoustic_quad_col_body<N, EPB, real, 3, true>(blockIdx.x, nE, rec, conn, u, r, Dm, elist);
}

// Elastic2D quads (records and stress as in kernels_elastic2d.cuh).
template <int N, int EPB, typename real, int C, int OFF>
__device__ __forceinline__ void elastic2d_col_body(int64_t bid, int64_t nE,
                                                   const int32_t *__restrict__ elist,
                                                   const real *__restrict__ rec,
                                                   const int32_t *__restrict__ conn,
                                                   const real *__restrict__ u,
                                                   real *__restrict__ r,
                                                   const DMatrix<real> &Dm) {
  using S = QuadColShape<N, EPB>;
  constexpr int n = S::n, P = S::P;
  __shared__ real sD[n * n];
  __shared__ real su[EPB][2][P];
  __shared__ real sF[EPB][2][P];
  const int t = threadIdx.x;
  const int le = t / n, i = t - le * n;
  const int64_t k = bid * EPB + le;
  const bool ok = le < EPB && k < nE;
  int64_t e = k;
  real J[n][4], cw[n][4], ux[n], uy[n];
  if (t < n * n) sD[t] = Dm.d[t];
  if (ok) {
    if (elist) e = elist[k];
    int64_t node[n];
#pragma unroll
    for (int j = 0; j < n; ++j) {
      load_elastic2d_rec(rec, k, i + n * j, P, J[j], cw[j]);
      node[j] = conn[e * P + i + n * j];
    }
#pragma unroll
    for (int j = 0; j < n; ++j) {
      ux[j] = u[node[j] * C + OFF];
      uy[j] = u[node[j] * C + OFF + 1];
      su[le][0][i + n * j] = ux[j];
      su[le][1][i + n * j] = uy[j];
    }
  }
  __syncthreads();
  real Dri[n], DTi[n];
#pragma unroll
  for (int l = 0; l < n; ++l) {
    Dri[l] = sD[i * n + l];
    DTi[l] = sD[l * n + i];
  }
  real Fsx[n], Fsy[n];
  if (ok) {
#pragma unroll
    for (int j = 0; j < n; ++j) {
      real dxr = 0, dxs = 0, dyr = 0, dys = 0;
#pragma unroll
      for (int l = 0; l < n; ++l) {
        const real a = Dri[l], b = Dm.d[j * n + l];
        dxr += a * su[le][0][l + n * j];
        dxs += b * ux[l];
        dyr += a * su[le][1][l + n * j];
        dys += b * uy[l];
      }
      const real *Jj = J[j], *cj = cw[j];
      const real uxx = Jj[0] * dxr + Jj[1] * dxs, uxy = Jj[2] * dxr + Jj[3] * dxs;
      const real uyx = Jj[0] * dyr + Jj[1] * dys, uyy = Jj[2] * dyr + Jj[3] * dys;
      const real sxx = cj[0] * uxx + cj[1] * uyy;
      const real syy = cj[1] * uxx + cj[2] * uyy;
      const real sxy = cj[3] * (uxy + uyx);
      sF[le][0][i + n * j] = Jj[0] * sxx + Jj[2] * sxy;
      Fsx[j] = Jj[1] * sxx + Jj[3] * sxy;
      sF[le][1][i + n * j] = Jj[0] * sxy + Jj[2] * syy;
      Fsy[j] = Jj[1] * sxy + Jj[3] * syy;
    }
  }
  __syncthreads();
  if (ok) {
#pragma unroll
    for (int j = 0; j < n; ++j) {
      real ox = 0, oy = 0;
#pragma unroll
      for (int l = 0; l < n; ++l) {
        const real a = DTi[l], b = Dm.d[l * n + j];
        ox += a * sF[le][0][l + n * j] + b * Fsx[l];
        oy += a * sF[le][1][l + n * j] + b * Fsy[l];
      }
      const int64_t o = (e * P + i + n * j) * C;
      r[o + OFF] = -ox;
      r[o + OFF + 1] = -oy;
#pragma unroll
      for (int c = 0; c < C; ++c)
        if (c < OFF || c > OFF + 1) r[o + c] = real(0);
    }
  }
}

template <int N, int EPB, typename real, int C, int OFF>
__global__ void __launch_bounds__(QuadColShape<N, EPB>::THREADS)
elastic2d_col_kernel(int64_t nE, const int32_t *__restrict__ elist, const real *__restrict__ rec,
                     const int32_t *__restrict__ conn, const real *__restrict__ u,
                     real *__restrict__ r, DMatrix<real> Dm) {
  elastic2d_col_body<N, EPB, real, C, OFF>(blockIdx.x, nE, elist, rec, conn, u, r, Dm);
}

}  // namespace salvus
