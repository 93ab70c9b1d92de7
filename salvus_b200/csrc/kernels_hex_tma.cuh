// kernels_hex_tma.cuh -- FP32 elastic hexahedron stiffness with the element
// records staged into shared memory by TMA bulk copies.
//
// Same arithmetic as elastic_hex_stiffness_kernel (Elastic3D.cpp:70-118 via
// Hexahedra.cpp:580-632 / 689-754): per (i, j) column thread, the n points
// along t live in registers; r- and s-direction operands come from shared
// memory, packed as float4 (x, y, z, pad) so one load serves all three
// components.  Shared memory per group of EPB elements:
//   srec [EPB][3][P] float4   48 B records (invJ 9, lambda', mu', conn) in
//                            the three-plane layout of the global records;
//                            after a point's record is consumed its slot
//                            holds (F_r xyz, -) and (F_s xyz, -)
//   su   [EPB][P]    float4   gathered u (x, y, z, pad); reused to stage the
//                            residual for coalesced 16-byte stores
//   bar  mbarrier(s)         completion of the bulk copies
// Two kernels: a one-group-per-CTA form, and a persistent form whose CTAs
// walk the element groups with two record buffers, so the next group's
// records stream in while the current group is computed.
// Every wait on a bulk copy is bounded: on timeout the CTA records an error
// in *err, lets the copy drain (bounded again) and returns.
#pragma once

#include <cstdint>

namespace salvus {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Orders this thread's earlier generic-proxy shared-memory writes before
// later async-proxy (bulk copy) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of *bar with an iteration limit; returns false on
// timeout.  Each try_wait suspends for a bounded, hardware-defined time.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

constexpr uint32_t kBulkWaitLimit = 1u << 20;

template <int N>
struct ElasticTmaShape {
  static constexpr int n = N + 1, n2 = n * n, P = n2 * n;
  // EPB * P * 3 must be a multiple of 4 so every group's residual block starts
  // on a 16-byte boundary (float4 stores); odd P needs EPB % 4 == 0.
  static constexpr int EPB0 = (200 / n2) > 0 ? (200 / n2) : 1;
  static constexpr int EPB = (P % 4 == 0) ? EPB0 : (EPB0 >= 4 ? EPB0 / 4 * 4 : 4);
  static constexpr int THREADS = ((EPB * n2 + 31) / 32) * 32;
  static constexpr size_t REC_BYTES = (size_t)P * 48;  // per element
  static constexpr size_t REC_GROUP = REC_BYTES * EPB;
  static constexpr size_t U_GROUP = (size_t)EPB * P * 16;
  static constexpr size_t SMEM = REC_GROUP + U_GROUP + 16;
  static constexpr size_t SMEM_PERSISTENT = 2 * REC_GROUP + U_GROUP + 32;
};

// Stiffness of one group of elements whose records are in erec_base (shared
// memory).  Called by all threads of the CTA; contains __syncthreads.
template <int N>
__device__ __forceinline__ void elastic_group(float4 *__restrict__ srec, float4 *__restrict__ su,
                                              int nvalid, int64_t e0,
                                              const float *__restrict__ u,
                                              float *__restrict__ r, const DMatrix<float> &Dm,
                                              const float *Dri, const float *Dsj,
                                              const float *DTi, const float *DTj) {
  using S = ElasticTmaShape<N>;
  constexpr int n = S::n, n2 = S::n2, P = S::P;
  const int t = threadIdx.x;
  const int le = t / n2, ij = t - le * n2;
  const int i = ij % n, j = ij / n;
  const bool ok = le < nvalid;
  float4 *erec = srec + (size_t)(ok ? le : 0) * P * 3;
  float4 *eu = su + (size_t)(ok ? le : 0) * P;
  float ux[n], uy[n], uz[n];
  if (ok) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
      const int node = __float_as_int(erec[2 * P + p].w);
      ux[k] = __ldg(u + 3 * (int64_t)node + 0);
      uy[k] = __ldg(u + 3 * (int64_t)node + 1);
      uz[k] = __ldg(u + 3 * (int64_t)node + 2);
    }
#pragma unroll
    for (int k = 0; k < n; ++k) eu[ij + n2 * k] = make_float4(ux[k], uy[k], uz[k], 0.f);
  }
  __syncthreads();
  float Ftx[n], Fty[n], Ftz[n];
  if (ok) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
      const float4 ra = erec[p], rb = erec[P + p], rc = erec[2 * P + p];
      const float J[9] = {ra.x, ra.y, ra.z, ra.w, rb.x, rb.y, rb.z, rb.w, rc.x};
      const float lam = rc.y, mu = rc.z;
      float d[3][3];
      {
        float rx = 0, ry = 0, rz = 0, sx = 0, sy = 0, sz = 0, tx = 0, ty = 0, tz = 0;
#pragma unroll
        for (int l = 0; l < n; ++l) {
          const float4 a = eu[l + n * j + n2 * k];
          const float4 b = eu[i + n * l + n2 * k];
          rx += Dri[l] * a.x; ry += Dri[l] * a.y; rz += Dri[l] * a.z;
          sx += Dsj[l] * b.x; sy += Dsj[l] * b.y; sz += Dsj[l] * b.z;
          const float dk = Dm.d[k * n + l];
          tx += dk * ux[l]; ty += dk * uy[l]; tz += dk * uz[l];
        }
        d[0][0] = rx; d[0][1] = sx; d[0][2] = tx;
        d[1][0] = ry; d[1][1] = sy; d[1][2] = ty;
        d[2][0] = rz; d[2][1] = sz; d[2][2] = tz;
      }
      float g[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a)
          g[c][a] = J[a * 3 + 0] * d[c][0] + J[a * 3 + 1] * d[c][1] + J[a * 3 + 2] * d[c][2];
      const float tr = g[0][0] + g[1][1] + g[2][2];
      const float sxx = lam * tr + 2 * mu * g[0][0];
      const float syy = lam * tr + 2 * mu * g[1][1];
      const float szz = lam * tr + 2 * mu * g[2][2];
      const float sxy = mu * (g[0][1] + g[1][0]);
      const float sxz = mu * (g[0][2] + g[2][0]);
      const float syz = mu * (g[1][2] + g[2][1]);
      const float sig[3][3] = {{sxx, sxy, sxz}, {sxy, syy, syz}, {sxz, syz, szz}};
      float F[3][3];  // F[c][b]
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int b = 0; b < 3; ++b)
          F[c][b] = J[0 * 3 + b] * sig[c][0] + J[1 * 3 + b] * sig[c][1] + J[2 * 3 + b] * sig[c][2];
      erec[p] = make_float4(F[0][0], F[1][0], F[2][0], 0.f);
      erec[P + p] = make_float4(F[0][1], F[1][1], F[2][1], 0.f);
      Ftx[k] = F[0][2]; Fty[k] = F[1][2]; Ftz[k] = F[2][2];
    }
  }
  __syncthreads();
  float *stage = reinterpret_cast<float *>(su);  // [EPB][P][3] residual
  if (ok) {
#pragma unroll
    for (int k = 0; k < n; ++k) {
      const int p = ij + n2 * k;
      float ox = 0, oy = 0, oz = 0;
#pragma unroll
      for (int l = 0; l < n; ++l) {
        const float4 a = erec[l + n * j + n2 * k];
        const float4 b = erec[P + i + n * l + n2 * k];
        const float dk = Dm.d[l * n + k];
        ox += DTi[l] * a.x + DTj[l] * b.x + dk * Ftx[l];
        oy += DTi[l] * a.y + DTj[l] * b.y + dk * Fty[l];
        oz += DTi[l] * a.z + DTj[l] * b.z + dk * Ftz[l];
      }
      float *o = stage + ((size_t)le * P + p) * 3;
      o[0] = -ox; o[1] = -oy; o[2] = -oz;
    }
  }
  __syncthreads();
  // coalesced 16-byte stores of the group's contiguous residual block
  const int nvec = nvalid * P * 3 / 4;
  const float4 *s4 = reinterpret_cast<const float4 *>(stage);
  float4 *g4 = reinterpret_cast<float4 *>(r + e0 * P * 3);
  for (int q = t; q < nvec; q += blockDim.x) g4[q] = s4[q];
  const int tail = nvalid * P * 3 - nvec * 4;
  if (t < tail) r[e0 * P * 3 + nvec * 4 + t] = stage[nvec * 4 + t];
  // Before the CTA reuses srec / su: order this thread's generic writes to
  // srec ahead of the next bulk copy into it, and let every thread finish
  // reading the staged residual.
  fence_proxy_async_smem();
  __syncthreads();
}

template <int N>
__device__ __forceinline__ void load_d_regs(const DMatrix<float> &Dm, float *Dri, float *Dsj,
                                            float *DTi, float *DTj) {
  constexpr int n = N + 1, n2 = n * n;
  const int ij = threadIdx.x % n2;
  const int i = ij % n, j = ij / n;
#pragma unroll
  for (int l = 0; l < n; ++l) {
    Dri[l] = Dm.d[i * n + l];
    Dsj[l] = Dm.d[j * n + l];
    DTi[l] = Dm.d[l * n + i];
    DTj[l] = Dm.d[l * n + j];
  }
}

template <int N>
__global__ void __launch_bounds__(ElasticTmaShape<N>::THREADS)
elastic_hex_stiffness_tma_kernel(int64_t E, const float *__restrict__ rec,
                                 const float *__restrict__ u, float *__restrict__ r,
                                 DMatrix<float> Dm, int *__restrict__ err) {
  using S = ElasticTmaShape<N>;
  constexpr int n = S::n, P = S::P, EPB = S::EPB;
  extern __shared__ __align__(128) unsigned char smem_tma[];
  float4 *srec = reinterpret_cast<float4 *>(smem_tma);  // [EPB][P][3]
  float4 *su = srec + (size_t)EPB * P * 3;              // [EPB][P]
  uint64_t *bar = reinterpret_cast<uint64_t *>(su + (size_t)EPB * P);

  const int t = threadIdx.x;
  const int64_t e0 = (int64_t)blockIdx.x * EPB;
  const int nvalid = (int)((E - e0) < EPB ? (E - e0) : EPB);
  if (t == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (t == 0) {
    const uint32_t bytes = (uint32_t)(nvalid * S::REC_BYTES);
    mbar_arrive_expect_tx(bar, bytes);
    bulk_copy_g2s(srec, rec + e0 * P * 12, bytes, bar);
  }
  float Dri[n], Dsj[n], DTi[n], DTj[n];
  load_d_regs<N>(Dm, Dri, Dsj, DTi, DTj);
  const bool arrived = mbar_wait_bounded(bar, 0, kBulkWaitLimit);
  if (__syncthreads_or(!arrived)) {
    if (t == 0) atomicExch(err, 1);
    mbar_wait_bounded(bar, 0, kBulkWaitLimit);  // let the copy drain
    return;
  }
  elastic_group<N>(srec, su, nvalid, e0, u, r, Dm, Dri, Dsj, DTi, DTj);
}

// Persistent form: CTA b handles groups b, b + gridDim.x, ...; records of
// the next group are bulk-copied into the other buffer while this group is
// computed.
template <int N>
__global__ void __launch_bounds__(ElasticTmaShape<N>::THREADS, 2)
elastic_hex_stiffness_tma_persistent(int64_t E, const float *__restrict__ rec,
                                     const float *__restrict__ u, float *__restrict__ r,
                                     DMatrix<float> Dm, int *__restrict__ err) {
  using S = ElasticTmaShape<N>;
  constexpr int n = S::n, P = S::P, EPB = S::EPB;
  extern __shared__ __align__(128) unsigned char smem_tma[];
  float4 *srec0 = reinterpret_cast<float4 *>(smem_tma);   // [2][EPB][P][3]
  float4 *su = srec0 + 2 * (size_t)EPB * P * 3;           // [EPB][P]
  uint64_t *bar = reinterpret_cast<uint64_t *>(su + (size_t)EPB * P);  // [2]
  const int64_t ngroups = (E + EPB - 1) / EPB;
  const int t = threadIdx.x;
  auto nvalid_of = [&](int64_t g) -> int {
    const int64_t rem = E - g * EPB;
    return (int)(rem < EPB ? rem : EPB);
  };
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int64_t g = blockIdx.x;
  if (t == 0 && g < ngroups) {
    const uint32_t bytes = (uint32_t)(nvalid_of(g) * S::REC_BYTES);
    mbar_arrive_expect_tx(&bar[0], bytes);
    bulk_copy_g2s(srec0, rec + g * EPB * P * 12, bytes, &bar[0]);
  }
  float Dri[n], Dsj[n], DTi[n], DTj[n];
  load_d_regs<N>(Dm, Dri, Dsj, DTi, DTj);
  for (int it = 0; g < ngroups; ++it, g += gridDim.x) {
    const int b = it & 1;
    float4 *cur = srec0 + (size_t)b * EPB * P * 3;
    const int64_t gn = g + gridDim.x;
    if (t == 0 && gn < ngroups) {
      // buffer b^1 was last read in the previous iteration, which every
      // thread finished (trailing __syncthreads of elastic_group)
      fence_proxy_async_smem();
      const uint32_t bytes = (uint32_t)(nvalid_of(gn) * S::REC_BYTES);
      mbar_arrive_expect_tx(&bar[b ^ 1], bytes);
      bulk_copy_g2s(srec0 + (size_t)(b ^ 1) * EPB * P * 3, rec + gn * EPB * P * 12, bytes,
                    &bar[b ^ 1]);
    }
    const bool arrived = mbar_wait_bounded(&bar[b], (uint32_t)((it >> 1) & 1), kBulkWaitLimit);
    if (__syncthreads_or(!arrived)) {
      if (t == 0) atomicExch(err, 1);
      // drain both buffers' copies before leaving
      mbar_wait_bounded(&bar[b], (uint32_t)((it >> 1) & 1), kBulkWaitLimit);
      if (gn < ngroups) mbar_wait_bounded(&bar[b ^ 1], (uint32_t)(((it + 1) >> 1) & 1), kBulkWaitLimit);
      return;
    }
    elastic_group<N>(cur, su, nvalid_of(g), g * EPB, u, r, Dm, Dri, Dsj, DTi, DTj);
  }
}

}  // namespace salvus
