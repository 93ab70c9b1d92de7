// kernels_step.cuh -- assembly by node gather, inverse mass, explicit
// Newmark update, Ricker source injection and receiver sampling.
//
// Reference arithmetic restated:
//   assembly        Problem::assembleIntoGlobalDof (Problem.cpp:143-214) with
//                   the scatter-add of addFieldOnElement (Problem.cpp:271-284),
//                   done here as a gather over each node's incident element
//                   points in ascending element order (deterministic);
//   inverse mass    Order2Newmark::applyInverseMassMatrix (Order2Newmark.cpp:68-83);
//   Newmark         Order2Newmark::takeTimeStep (Order2Newmark.cpp:85-114):
//                   v += dt/2 (a + a_), u += dt v + dt^2/2 a, a_ = a;
//   source          Scalar::computeSourceTerm (Scalar.cpp:79-88),
//                   Elastic3D::computeSourceTerm (Elastic3D.cpp:126-133),
//                   Ricker::fire (Ricker.cpp:27-33), evaluated at t_n = n dt;
//   receivers       Lagrange interpolation (TensorQuad.cpp:145-174,
//                   Hexahedra.cpp:494-532) of u at the receiver point,
//                   accumulated in FP64 with Kahan compensation.
#pragma once

#include <cstdint>

namespace salvus {

// mode 0: fused  a = mi * sum(r); Newmark update of (u, v, a_)
// mode 1: gather a = sum(r)
template <typename real, int C, int MODE>
__global__ void gather_kernel(int64_t G, const int32_t *__restrict__ off,
                              const int32_t *__restrict__ idx, const real *__restrict__ r,
                              const real *__restrict__ mi, real *__restrict__ u,
                              real *__restrict__ v, real *__restrict__ ap, real *__restrict__ a,
                              real dt) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  real acc[C];
#pragma unroll
  for (int c = 0; c < C; ++c) acc[c] = 0;
  const int32_t q0 = off[g], q1 = off[g + 1];
  for (int32_t q = q0; q < q1; ++q) {
    const int64_t ep = idx[q];
#pragma unroll
    for (int c = 0; c < C; ++c) acc[c] += r[ep * C + c];
  }
  if (MODE == 1) {
#pragma unroll
    for (int c = 0; c < C; ++c) a[g * C + c] = acc[c];
    return;
  }
  const real m = mi[g];
  const real acl = real(0.5) * dt, dsp = real(0.5) * dt * dt;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int64_t i = g * C + c;
    const real an = acc[c] * m;
    const real vn = acl * an + acl * ap[i] + v[i];
    u[i] = dt * vn + dsp * an + u[i];
    v[i] = vn;
    ap[i] = an;
  }
}

template <typename real, int C>
__global__ void inverse_mass_kernel(int64_t G, const real *__restrict__ mi, real *__restrict__ a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G * C) return;
  a[i] = a[i] * mi[i / C];
}

template <typename real>
__global__ void newmark_kernel(int64_t N, const real *__restrict__ a, real *__restrict__ u,
                               real *__restrict__ v, real *__restrict__ ap, real dt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const real acl = real(0.5) * dt, dsp = real(0.5) * dt * dt;
  const real an = a[i];
  const real vn = acl * an + acl * ap[i] + v[i];
  u[i] = dt * vn + dsp * an + u[i];
  v[i] = vn;
  ap[i] = an;
}

__device__ __forceinline__ double ricker_dev(double t, double f0, double t0, double amp) {
  const double pi = 3.14159265358979323846;
  const double factor = pi * pi * f0 * f0 * (t - t0) * (t - t0);
  return amp * ((1 - 2 * factor) * exp(-1 * factor));
}

// Sources in attach order, one CTA; adds w_{p,c} * stf(t_n) into the
// element-local residual of the source element.  src_par = [f0, t0, amp].
template <typename real, int C>
__global__ void source_kernel(int nsrc, int P, const int64_t *__restrict__ elem,
                              const double *__restrict__ par, const double *__restrict__ wts,
                              const int64_t *__restrict__ step, double dt, real *__restrict__ r) {
  const double t = (double)(*step) * dt;
  for (int s = 0; s < nsrc; ++s) {
    const double stf = ricker_dev(t, par[3 * s], par[3 * s + 1], par[3 * s + 2]);
    const int64_t base = elem[s] * P * C;
    for (int q = threadIdx.x; q < P * C; q += blockDim.x)
      r[base + q] += (real)(wts[(int64_t)s * P * C + q] * stf);
    __syncthreads();
  }
}

// Receivers (one CTA): seis[(rec*C + c)*cap + step % cap] = sum_p l_p u;
// then advances the device step counter.
template <typename real, int C>
__global__ void receiver_kernel(int nrec, int P, const int64_t *__restrict__ elem,
                                const double *__restrict__ lw, const int32_t *__restrict__ conn,
                                const real *__restrict__ u, double *__restrict__ seis, int64_t cap,
                                int64_t *__restrict__ step) {
  const int64_t n = *step;
  for (int q = threadIdx.x; q < nrec * C; q += blockDim.x) {
    const int rc = q / C, c = q - rc * C;
    const int64_t e = elem[rc];
    double s = 0.0, comp = 0.0;
    for (int p = 0; p < P; ++p) {
      const double y = lw[(int64_t)rc * P + p] * (double)u[(int64_t)conn[e * P + p] * C + c] - comp;
      const double tt = s + y;
      comp = (tt - s) - y;
      s = tt;
    }
    seis[(int64_t)q * cap + (n % cap)] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) *step = n + 1;
}

// Deterministic partial sums of x.y weighted by w (w may be null): one partial
// per CTA, summed on the host in block order.
template <typename real>
__global__ void dot_kernel(int64_t N, int C, const real *__restrict__ x, const real *__restrict__ y,
                           const double *__restrict__ w, double *__restrict__ partial) {
  __shared__ double sh[256];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (int64_t)gridDim.x * blockDim.x) {
    double wi = w ? w[i / C] : 1.0;
    s += (double)x[i] * (double)y[i] * wi;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

template <typename A, typename B>
__global__ void convert_kernel(int64_t N, const A *__restrict__ a, B *__restrict__ b) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) b[i] = (B)a[i];
}

template <typename real>
__global__ void scale_kernel(int64_t N, real *__restrict__ x, double s) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) x[i] = (real)((double)x[i] * s);
}

}  // namespace salvus
