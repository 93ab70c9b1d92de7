// kernels_batch.cuh -- shot-batched kernels: S shots on one mesh advance
// together.  Fields are shot-interleaved, f[node][S] (S padded to a multiple
// of 32), so a warp's lanes are consecutive shots: every field load and store
// is coalesced and each geometry / connectivity word is read once for all
// shots of a CTA.
//
// The arithmetic per shot is the reference's (Scalar::computeStiffnessTerm,
// Scalar.cpp:58-71; Ricker::fire, Ricker.cpp:27-33); the time update uses the
// velocity-at-half-step form of the reference's Newmark scheme
// (Order2Newmark.cpp:99-108): with w = v + dt/2 a_ the pair
//   v += dt/2 (a + a_);  u += dt v + dt^2/2 a
// is exactly  w += dt a;  u += dt w  (one fewer field to stream).
#pragma once

#include <cstdint>

namespace salvus {

// Interior-node update of the fused batched step (kFuse): the points with
// both local indices in 1..N-1 are nodes of this element alone, so the
// stiffness thread of (element, shot) finishes them -- the one-term assembly
// 0 + r, the inverse mass and the half-step-velocity update
// (batched_gather_update_kernel's arithmetic) -- and writes residuals only
// for the element's edge points.  Where the shot has a source in the element
// the interior residuals are written too, and batched_source_kernel adds the
// source terms and then finishes those nodes.  Same operations in the same
// order as the unfused sequence, so both forms give bitwise the same
// wavefields.
struct BatchInterior {
  const float *mi;
  float *w;
  float dt;
  const int32_t *shot_off;  // sources of shot s: [shot_off[s], shot_off[s + 1])
  const int64_t *src_elem;
};

// half-step-velocity update of one node (one shot): w += dt a; u += dt w,
// with explicitly rounded operations so that every kernel applying it gives
// the same bits
__device__ __forceinline__ void half_step_update(float acc, float m, float dt, float &w, float &u) {
  w = __fmaf_rn(dt, __fmul_rn(acc, m), w);
  u = __fmaf_rn(dt, w, u);
}

// One thread = one shot of one quad element; the element's n^2 values of
// that shot live in registers, so the tensor-product contractions need no
// shared memory.  CTA = EPC elements x SC shots.
template <int N, int SC, int EPC, bool kFuse = false>
__global__ void __launch_bounds__(SC *EPC)
quad_acoustic_batched_kernel(int64_t E, int S, const float *__restrict__ rec,
                             float *__restrict__ u, float *__restrict__ r,
                             DMatrix<float> Dm, BatchInterior bi) {
  constexpr int n = N + 1, P = n * n;
  __shared__ float4 sg[EPC * P];  // G00 G01 G11 conn of the CTA's elements
  const int64_t e0 = (int64_t)blockIdx.x * EPC;
  for (int q = threadIdx.x; q < EPC * P; q += blockDim.x) {
    const int64_t ee = e0 + q / P;
    sg[q] = ee < E ? __ldg(reinterpret_cast<const float4 *>(rec) + e0 * P + q)
                   : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  const int ey = threadIdx.x / SC, lane = threadIdx.x - ey * SC;
  const int64_t e = e0 + ey;
  const int s = blockIdx.y * SC + lane;
  if (e >= E || s >= S) return;
  const float4 *g = sg + ey * P;
  float uu[P];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    // the fused form writes u of interior nodes during the launch: coherent loads
    const float *up = u + (int64_t)__float_as_int(g[p].w) * S + s;
    uu[p] = kFuse ? *up : __ldg(up);
  }
  // fused form: whether one of this shot's sources sits in this element (then
  // the unfused form for its interior points), and the interior nodes' w,
  // loaded before the arithmetic so that their latency overlaps it (w is
  // written below; the read-only inverse mass is read where it is used)
  bool fuse_here = kFuse;
  float wpre[P];
  if constexpr (kFuse) {
    if (bi.shot_off)
      for (int k = bi.shot_off[s]; k < bi.shot_off[s + 1] && fuse_here; ++k)
        fuse_here = __ldg(bi.src_elem + k) != e;
    if (fuse_here) {
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const int i = p % n, j = p / n;
        if (i < 1 || i > n - 2 || j < 1 || j > n - 2) continue;
        wpre[p] = bi.w[(int64_t)__float_as_int(g[p].w) * S + s];
      }
    }
  }
  float Fr[P], Fs[P];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const int i = p % n, j = p / n;
    float gr = 0.f, gs = 0.f;
#pragma unroll
    for (int l = 0; l < n; ++l) {
      gr += Dm.d[i * n + l] * uu[l + n * j];
      gs += Dm.d[j * n + l] * uu[i + n * l];
    }
    const float4 G = g[p];
    Fr[p] = G.x * gr + G.y * gs;
    Fs[p] = G.y * gr + G.z * gs;
  }
  float *out = r + (e * P) * S + s;
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const int i = p % n, j = p / n;
    float o = 0.f;
#pragma unroll
    for (int l = 0; l < n; ++l) {
      o += Dm.d[l * n + i] * Fr[l + n * j];
      o += Dm.d[l * n + j] * Fs[i + n * l];
    }
    if (!fuse_here || i < 1 || i > n - 2 || j < 1 || j > n - 2) {
      out[(int64_t)p * S] = -o;
      continue;
    }
    if constexpr (kFuse) {
      const int64_t x = (int64_t)__float_as_int(g[p].w) * S + s;
      float wv = wpre[p], uv = uu[p];
      half_step_update(__fadd_rn(0.f, -o), __ldg(bi.mi + __float_as_int(g[p].w)), bi.dt, wv, uv);
      bi.w[x] = wv;
      u[x] = uv;
    }
  }
}

// Ricker sources of every shot into the element-local residual.  Thread =
// (shot, point); a shot's sources are applied in attach order.  Fused step
// (n > 0, the element's points per line): afterwards the thread of an
// interior point finishes that node of each distinct source element of its
// shot -- the node the fused stiffness kernel left to it -- with the
// gather's arithmetic (one-term assembly 0 + r, inverse mass, update).
__global__ void batched_source_kernel(int S, int P, const int32_t *__restrict__ shot_off,
                                      const int64_t *__restrict__ elem,
                                      const double *__restrict__ par,
                                      const double *__restrict__ wts,
                                      const int64_t *__restrict__ step, double dt,
                                      float *__restrict__ r, int n = 0,
                                      const int32_t *__restrict__ conn = nullptr,
                                      const float *__restrict__ mi = nullptr,
                                      float *__restrict__ u = nullptr,
                                      float *__restrict__ w = nullptr, float dtf = 0.f) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= S * P) return;
  const int p = q % P, s = q / P;
  const double t = (double)(*step) * dt;
  for (int k = shot_off[s]; k < shot_off[s + 1]; ++k) {
    const double stf = ricker_dev(t, par[3 * k], par[3 * k + 1], par[3 * k + 2]);
    r[(elem[k] * P + p) * S + s] += (float)(wts[(int64_t)k * P + p] * stf);
  }
  if (n == 0) return;
  const int i = p % n, j = p / n;
  if (i < 1 || i > n - 2 || j < 1 || j > n - 2) return;
  for (int k = shot_off[s]; k < shot_off[s + 1]; ++k) {
    bool first = true;  // each distinct source element once
    for (int k2 = shot_off[s]; k2 < k && first; ++k2) first = elem[k2] != elem[k];
    if (!first) continue;
    const int64_t e = elem[k];
    const int32_t node = conn[e * P + p];
    const int64_t x = (int64_t)node * S + s;
    float wv = w[x], uv = u[x];
    half_step_update(__fadd_rn(0.f, r[(e * P + p) * S + s]), mi[node], dtf, wv, uv);
    w[x] = wv;
    u[x] = uv;
  }
}

// Node gather + inverse mass + half-step-velocity update, thread = (NPT
// consecutive nodes, shot).  CTA = NPB node groups x SC shots.  The NPT
// nodes' dependent load chains (offsets -> incidence -> residual) are issued
// side by side so that more bytes are in flight per thread; the per-node
// arithmetic and summation order do not depend on NPT.
// nodes != nullptr: thread slot t handles node nodes[t] (the edge nodes of
// the fused form), G is then the list's length.
template <int SC, int NPB, int NPT>
__global__ void __launch_bounds__(SC *NPB)
batched_gather_update_kernel(int64_t G, int S, const int32_t *__restrict__ off,
                             const int32_t *__restrict__ idx, const float *__restrict__ r,
                             const float *__restrict__ mi, float *__restrict__ u,
                             float *__restrict__ w, float dt,
                             const int32_t *__restrict__ nodes = nullptr) {
  const int ny = threadIdx.x / SC, lane = threadIdx.x - ny * SC;
  const int64_t g0 = ((int64_t)blockIdx.x * NPB + ny) * NPT;
  const int s = blockIdx.y * SC + lane;
  if (g0 >= G || s >= S) return;
  constexpr int kFast = 4;  // quadrilateral valence bound
  float uo[NPT], wo[NPT], m[NPT];
  int32_t q0[NPT], cnt[NPT];
  int64_t gk[NPT];
#pragma unroll
  for (int k = 0; k < NPT; ++k) {
    const bool live = g0 + k < G;
    const int64_t g = !live ? 0 : nodes ? (int64_t)__ldg(nodes + g0 + k) : g0 + k;
    gk[k] = g;
    const int64_t i = g * S + s;
    uo[k] = live ? u[i] : 0.f;
    wo[k] = live ? w[i] : 0.f;
    m[k] = live ? __ldg(mi + g) : 0.f;
    q0[k] = live ? __ldg(off + g) : 0;
    cnt[k] = live ? __ldg(off + g + 1) - q0[k] : 0;
  }
  // all incidence indices first, then all residual loads in flight at once
  int32_t ep[NPT][kFast];
#pragma unroll
  for (int k = 0; k < NPT; ++k)
#pragma unroll
    for (int q = 0; q < kFast; ++q) ep[k][q] = q < cnt[k] ? __ldg(idx + q0[k] + q) : 0;
  float rv[NPT][kFast];
#pragma unroll
  for (int k = 0; k < NPT; ++k)
#pragma unroll
    for (int q = 0; q < kFast; ++q)
      rv[k][q] = q < cnt[k] ? __ldg(r + (int64_t)ep[k][q] * S + s) : 0.f;
#pragma unroll
  for (int k = 0; k < NPT; ++k) {
    if (g0 + k >= G) break;
    const int64_t g = gk[k];
    // summed in ascending element order
    float acc = 0.f;
    if (cnt[k] <= kFast) {
#pragma unroll
      for (int q = 0; q < kFast; ++q)
        if (q < cnt[k]) acc += rv[k][q];
    } else {
      for (int32_t q = q0[k]; q < q0[k] + cnt[k]; ++q)
        acc += __ldg(r + (int64_t)__ldg(idx + q) * S + s);
    }
    float wn = wo[k], un = uo[k];
    half_step_update(acc, m[k], dt, wn, un);
    const int64_t i = g * S + s;
    w[i] = wn;
    u[i] = un;
  }
}

// Receivers of every shot: block = receiver, thread = shot; FP64 Kahan over
// the element points.  seis[(s * R + rec) * cap + step % cap].
__global__ void batched_receiver_kernel(int S, int R, int P, const int64_t *__restrict__ elem,
                                        const double *__restrict__ lw,
                                        const int32_t *__restrict__ conn,
                                        const float *__restrict__ u, double *__restrict__ seis,
                                        int64_t cap, const int64_t *__restrict__ step) {
  const int rc = blockIdx.x;
  const int64_t e = elem[rc];
  const int64_t slot = *step % cap;
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double acc = 0.0, comp = 0.0;
    for (int p = 0; p < P; ++p) {
      const double y = lw[(int64_t)rc * P + p] * (double)u[(int64_t)conn[e * P + p] * S + s] - comp;
      const double tt = acc + y;
      comp = (tt - acc) - y;
      acc = tt;
    }
    seis[((int64_t)s * R + rc) * cap + slot] = acc;
  }
}

// Column k of a shot-interleaved field <-> a contiguous FP64 array.
__global__ void shot_scatter_kernel(int64_t G, int S, int k, const double *__restrict__ src,
                                    float *__restrict__ f) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < G) f[g * S + k] = (float)src[g];
}
__global__ void shot_gather_kernel(int64_t G, int S, int k, const float *__restrict__ f,
                                   double *__restrict__ dst) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < G) dst[g] = (double)f[g * S + k];
}

}  // namespace salvus
