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

// One Newmark update with explicitly rounded operations, so that the fused
// gather/update kernel and the three-call path (gather, inverse mass,
// Newmark) produce bitwise identical wavefields whatever the compiler's
// contraction choices.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

template <typename real>
__device__ __forceinline__ void newmark_point(real an, real &ap, real &v, real &u, real dt) {
  const real acl = mul_rn(real(0.5), dt), dsp = mul_rn(mul_rn(real(0.5), dt), dt);
  // v_{n} = dt/2 a + dt/2 a_ + v ; u = dt v + dt^2/2 a + u  (Order2Newmark.cpp:104-107)
  const real vn = add_rn(add_rn(mul_rn(acl, an), mul_rn(acl, ap)), v);
  u = add_rn(add_rn(mul_rn(dt, vn), mul_rn(dsp, an)), u);
  v = vn;
  ap = an;
}

// mode 0: fused  a = mi * sum(r); Newmark update of (u, v, a_)
// mode 1: gather a = sum(r)
// kInKernelR: r was written earlier in the same launch (fused group steps)
// and is read with coherent loads (ld.global.ca), not ld.global.nc.
template <typename real, int C, int MODE, bool kInKernelR = false>
__device__ __forceinline__ void gather_body(int64_t g, int64_t G, const int32_t *__restrict__ off,
                                            const int32_t *__restrict__ idx,
                                            const real *__restrict__ r,
                                            const real *__restrict__ mi, real *__restrict__ u,
                                            real *__restrict__ v, real *__restrict__ ap,
                                            real *__restrict__ a, real dt) {
  if (g >= G) return;
  // Newmark operands first: they do not depend on the gather, so their loads
  // overlap the dependent index -> residual chain below.
  real m = 0, uo[C], vo[C], apo[C];
  if (MODE == 0) {
    m = mi[g];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      uo[c] = u[g * C + c];
      vo[c] = v[g * C + c];
      apo[c] = ap[g * C + c];
    }
  }
  real acc[C];
#pragma unroll
  for (int c = 0; c < C; ++c) acc[c] = 0;
  const int32_t q0 = off[g], q1 = off[g + 1];
  const int cnt = q1 - q0;
  constexpr int kFast = 8;  // hexahedral / quadrilateral valence bound
  if (cnt <= kFast) {
    int32_t ep[kFast];
#pragma unroll
    for (int q = 0; q < kFast; ++q) ep[q] = q < cnt ? idx[q0 + q] : 0;
    real rv[kFast][C];
#pragma unroll
    for (int q = 0; q < kFast; ++q)
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const real *rp = r + (int64_t)ep[q] * C + c;
        rv[q][c] = q < cnt ? (kInKernelR ? __ldca(rp) : *rp) : real(0);
      }
    // ascending element order, as in the general loop
#pragma unroll
    for (int q = 0; q < kFast; ++q)
      if (q < cnt) {
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] += rv[q][c];
      }
  } else {
    // high-valence nodes (tetrahedron vertices: about two dozen incident
    // points): batches of kBatch independent loads, summed in the same
    // ascending order as one at a time
    constexpr int kBatch = 4;
    for (int32_t qb = q0; qb < q1; qb += kBatch) {
      const int nq = q1 - qb < kBatch ? q1 - qb : kBatch;
      int32_t ep[kBatch];
#pragma unroll
      for (int q = 0; q < kBatch; ++q) ep[q] = q < nq ? idx[qb + q] : 0;
      real rv[kBatch][C];
#pragma unroll
      for (int q = 0; q < kBatch; ++q)
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const real *rp = r + (int64_t)ep[q] * C + c;
          rv[q][c] = q < nq ? (kInKernelR ? __ldca(rp) : *rp) : real(0);
        }
#pragma unroll
      for (int q = 0; q < kBatch; ++q)
        if (q < nq) {
#pragma unroll
          for (int c = 0; c < C; ++c) acc[c] += rv[q][c];
        }
    }
  }
  if constexpr (MODE == 1) {
#pragma unroll
    for (int c = 0; c < C; ++c) a[g * C + c] = acc[c];
  } else {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const int64_t i = g * C + c;
      newmark_point<real>(mul_rn(acc[c], m), apo[c], vo[c], uo[c], dt);
      u[i] = uo[c];
      v[i] = vo[c];
      ap[i] = apo[c];
    }
  }
}

template <typename real, int C, int MODE>
__global__ void gather_kernel(int64_t G, const int32_t *__restrict__ off,
                              const int32_t *__restrict__ idx, const real *__restrict__ r,
                              const real *__restrict__ mi, real *__restrict__ u,
                              real *__restrict__ v, real *__restrict__ ap, real *__restrict__ a,
                              real dt) {
  gather_body<real, C, MODE>((int64_t)blockIdx.x * blockDim.x + threadIdx.x, G, off, idx, r, mi, u,
                             v, ap, a, dt);
}

// The gather / update over a list of nodes (the shared nodes of a fused
// hexahedron step, whose interior nodes the stiffness kernel advanced).
template <typename real, int C, int MODE>
__global__ void gather_list_kernel(int64_t n, const int32_t *__restrict__ nodes,
                                   const int32_t *__restrict__ off,
                                   const int32_t *__restrict__ idx, const real *__restrict__ r,
                                   const real *__restrict__ mi, real *__restrict__ u,
                                   real *__restrict__ v, real *__restrict__ ap,
                                   real *__restrict__ a, real dt) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  gather_body<real, C, MODE>(nodes[t], INT64_MAX, off, idx, r, mi, u, v, ap, a, dt);
}

// Blow-up detection: any NaN / Inf among n values sets the problem's device
// status word to kNonFiniteCode (unless a wait timeout code is already
// there).  Launched after every 32 steps on the displacement field: an
// unstable explicit step grows without bound and reaches Inf / NaN in u.
constexpr int kNonFiniteCode = 0x4e614e;  // distinct from the wait codes (1000-1099)
template <typename real>
__global__ void finite_check_kernel(int64_t n, const real *__restrict__ x, int *__restrict__ err) {
  bool bad = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    bad |= !isfinite(x[i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicCAS(err, 0, kNonFiniteCode);
}

// Homogeneous Dirichlet (HomogeneousDirichlet.cpp:65-73): zero the stiffness
// rows of the listed element-local points (before sources are added).
template <typename real, int C>
__global__ void dirichlet_zero_kernel(int64_t n, const int32_t *__restrict__ pts,
                                      real *__restrict__ r) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t ep = pts[i];
#pragma unroll
  for (int c = 0; c < C; ++c) r[ep * C + c] = real(0);
}

// Fluid-solid coupling surface integrals on meshes of fluid and solid quads
// (ElasticToAcoustic.cpp:26-41, AcousticToElastic2D.cpp:48-60), fields
// [u, ux, uy]: one thread per coupled element point with its coefficients
// summed over the element's coupled edges; the first n_fluid points belong to
// fluid elements (u += cx vx + cy vy), the rest to solid elements
// (ux += cx v, uy += cy v).  Runs after the stiffness (and Dirichlet zeroing)
// and before the sources, on the velocity field.
template <typename real>
__global__ void coupling_kernel(int64_t n_fluid, int64_t n, const int32_t *__restrict__ pts,
                                const real *__restrict__ coef, const real *__restrict__ v,
                                real *__restrict__ r) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t ep = pts[2 * i], g = pts[2 * i + 1];
  const real cx = coef[2 * i], cy = coef[2 * i + 1];
  if (i < n_fluid) {
    r[ep * 3] += cx * v[g * 3 + 1] + cy * v[g * 3 + 2];
  } else {
    const real vf = v[g * 3];
    r[ep * 3 + 1] += cx * vf;
    r[ep * 3 + 2] += cy * vf;
  }
}

template <typename real, int C>
__global__ void inverse_mass_kernel(int64_t G, const real *__restrict__ mi, real *__restrict__ a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G * C) return;
  a[i] = mul_rn(a[i], mi[i / C]);
}

template <typename real>
__global__ void newmark_kernel(int64_t N, const real *__restrict__ a, real *__restrict__ u,
                               real *__restrict__ v, real *__restrict__ ap, real dt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  real apv = ap[i], vv = v[i], uv = u[i];
  newmark_point<real>(a[i], apv, vv, uv, dt);
  u[i] = uv;
  v[i] = vv;
  ap[i] = apv;
}

__device__ __forceinline__ double ricker_dev(double t, double f0, double t0, double amp) {
  const double pi = 3.14159265358979323846;
  const double factor = pi * pi * f0 * f0 * (t - t0) * (t - t0);
  return amp * ((1 - 2 * factor) * exp(-1 * factor));
}

// Sources in attach order, one CTA; adds w_{p,c} * stf(t_n) into the
// element-local residual of the source element.  src_par = [f0, t0, amp].
template <typename real, int C>
__device__ __forceinline__ void source_body(int nsrc, int P, const int64_t *__restrict__ elem,
                                            const double *__restrict__ par,
                                            const double *__restrict__ wts,
                                            const int64_t *__restrict__ step, double dt,
                                            real *__restrict__ r) {
  const double t = (double)(*step) * dt;
  for (int s = 0; s < nsrc; ++s) {
    const double stf = ricker_dev(t, par[3 * s], par[3 * s + 1], par[3 * s + 2]);
    const int64_t base = elem[s] * P * C;
    for (int q = threadIdx.x; q < P * C; q += blockDim.x)
      r[base + q] += (real)(wts[(int64_t)s * P * C + q] * stf);
    __syncthreads();
  }
}

template <typename real, int C>
__global__ void source_kernel(int nsrc, int P, const int64_t *__restrict__ elem,
                              const double *__restrict__ par, const double *__restrict__ wts,
                              const int64_t *__restrict__ step, double dt, real *__restrict__ r) {
  source_body<real, C>(nsrc, P, elem, par, wts, step, dt, r);
}

// Receivers: one CTA per receiver, one thread per element point (strided);
// each thread keeps a Kahan-compensated FP64 partial per component, then a
// fixed-order tree combines the partials (deterministic).
// seis[(rec*C + c)*cap + step % cap] = sum_p l_p u_p.
// kInKernelU: u was written earlier in the same launch (fused group steps),
// so it is read with a coherent load (ld.global.ca, ordered by the waits'
// fences), never through the non-coherent read-only path (ld.global.nc),
// which is only defined for data that no thread writes during the launch.
constexpr int kRecThreads = 128;
template <typename real, int C, bool kInKernelU = false>
__device__ __forceinline__ void receiver_body(int rc, int P, const int64_t *__restrict__ elem,
                                              const double *__restrict__ lw,
                                              const int32_t *__restrict__ conn,
                                              const real *__restrict__ u,
                                              double *__restrict__ seis, int64_t cap,
                                              const int64_t *__restrict__ step) {
  __shared__ double part[C][kRecThreads];
  // CTAs wider than kRecThreads (grouped persistent steps) keep their extra
  // threads idle here but in every barrier
  const int t = threadIdx.x;
  const int64_t e = elem[rc];
  double s[C], comp[C];
#pragma unroll
  for (int c = 0; c < C; ++c) s[c] = comp[c] = 0.0;
  for (int p = t; p < P && t < kRecThreads; p += kRecThreads) {
    const double l = lw[(int64_t)rc * P + p];
    const int64_t node = conn[e * P + p];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const real uc = kInKernelU ? __ldca(u + node * C + c) : u[node * C + c];
      const double y = l * (double)uc - comp[c];
      const double tt = s[c] + y;
      comp[c] = (tt - s[c]) - y;
      s[c] = tt;
    }
  }
  if (t < kRecThreads)
#pragma unroll
    for (int c = 0; c < C; ++c) part[c][t] = s[c];
  __syncthreads();
  for (int o = kRecThreads / 2; o > 0; o >>= 1) {
    if (t < o)
#pragma unroll
      for (int c = 0; c < C; ++c) part[c][t] += part[c][t + o];
    __syncthreads();
  }
  if (t < C) seis[((int64_t)rc * C + t) * cap + (*step % cap)] = part[t][0];
}

template <typename real, int C>
__global__ void __launch_bounds__(kRecThreads)
receiver_kernel(int P, const int64_t *__restrict__ elem, const double *__restrict__ lw,
                const int32_t *__restrict__ conn, const real *__restrict__ u,
                double *__restrict__ seis, int64_t cap, const int64_t *__restrict__ step) {
  receiver_body<real, C>(blockIdx.x, P, elem, lw, conn, u, seis, cap, step);
}

// Advances the device step counter (one thread), after every kernel of the
// step that reads it.
__global__ void advance_step_kernel(int64_t *__restrict__ step) { *step += 1; }

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

// Energy 1/2 v^T M v and 1/2 u^T K u with FP64 compensated (Kahan) sums:
// each thread accumulates its grid-stride share of the nodes with a running
// compensation, the CTA adds the threads' sums in a fixed tree order, and
// partial[2 * block] / [2 * block + 1] (kinetic, strain) are summed on the
// host in block order -- the same bits on every run for a given grid.
// ku = -K u (the gathered stiffness action); M = 1 / mi per node, nodes
// without mass (mi = 0) carry none.
template <typename real, int C>
__global__ void __launch_bounds__(256)
energy_kernel(int64_t G, const real *__restrict__ u, const real *__restrict__ v,
              const real *__restrict__ ku, const double *__restrict__ mi,
              double *__restrict__ partial) {
  __shared__ double sk[256], ss[256];
  double ek = 0.0, ck = 0.0, es = 0.0, cs = 0.0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < G;
       g += (int64_t)gridDim.x * blockDim.x) {
    const double m = mi[g] != 0.0 ? 1.0 / mi[g] : 0.0;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const double vv = (double)v[g * C + c], uu = (double)u[g * C + c];
      const double yk = 0.5 * m * vv * vv - ck;
      const double tk = ek + yk;
      ck = (tk - ek) - yk;
      ek = tk;
      const double ys = -0.5 * uu * (double)ku[g * C + c] - cs;
      const double ts = es + ys;
      cs = (ts - es) - ys;
      es = ts;
    }
  }
  sk[threadIdx.x] = ek;
  ss[threadIdx.x] = es;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sk[threadIdx.x] += sk[threadIdx.x + o];
      ss[threadIdx.x] += ss[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sk[0];
    partial[2 * blockIdx.x + 1] = ss[0];
  }
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
