// kernels_tri_tc.cuh -- FP32 P3 triangle stiffness (12 nodes, acoustic) with
// both dense contractions on the tensor cores (tcgen05, TF32 inputs, FP32
// accumulation in tensor memory) and the three-term split-precision
// correction of kernels_simplex_tc.cuh, so the result carries FP32-level
// accuracy.  Same arithmetic as tri_acoustic_kernel (ScalarTri /
// Triangle::buildStiffnessMatrix in factored form, Triangle.cpp:194-241):
//
//   GEMM 1  gradient:   D1[e][16 k + q] = sum_j u_e[j] dphi_j/dxi_k (x_q)
//           M = 128 elements, N = 32 (2 directions x 16, 12 used), K = 16 (12 used)
//   pointwise  F_e[k][q] = s_q (G_k0 g_0 + G_k1 g_1), written as the A operand
//   GEMM 2  divergence: D2[e][i] = sum_{k,q} F_e[k][q] dphi_i/dxi_k (x_q)
//           M = 128, N = 16 (12 used), K = 32 (2 x 16)
//
// B operands (host-built, K-major no-swizzle core-matrix order, TF32 hi and
// FP32 lo parts, 8 KB in all):
//   B1[16 k + q][j] = dphi_j/dxi_k (x_q)     32 x 16
//   B2[i][16 k + q] = dphi_i/dxi_k (x_q)     16 x 32
// Padding rows / columns are zero in the tables and in the A operands.
//
// A CTA = 4 worker warps (one element per thread, 128 per tile) and one
// issuer warp that owns 64 tensor-memory columns; several CTAs share an SM,
// so one CTA's gathers overlap another's MMAs, and within a CTA the next
// tile's loads are in flight while this tile's MMAs and pointwise stage run.
// Hand-offs go through mbarriers with bounded waits (a timeout sets *err and
// stops the CTA cleanly).
#pragma once

#include <cstdint>

#include "kernels_simplex_tc.cuh"

namespace salvus {

struct TriTcShape {
  static constexpr int P = 12;
  static constexpr int NE = 128;
  static constexpr int WORKERS = 128, THREADS = 160;
  static constexpr uint32_t B_BYTES = 32 * 16 * 4;     // each of B1, B2 per part
  static constexpr uint32_t A1_SBO = 4 * 128;          // K = 16 -> 4 core matrices
  static constexpr uint32_t A1_BYTES = 128 * 16 * 4;   // per part
  static constexpr uint32_t A2_SBO = 8 * 128;          // K = 32 -> 8 core matrices
  static constexpr uint32_t A2_BYTES = 128 * 32 * 4;   // per part
  static constexpr uint32_t B1_SBO = 4 * 128, B2_SBO = 8 * 128;
  static constexpr uint32_t OFF_B1 = 0;
  static constexpr uint32_t OFF_B2 = 2 * B_BYTES;
  static constexpr uint32_t TAB_BYTES = 4 * B_BYTES;  // 8192
  static constexpr uint32_t OFF_A1 = TAB_BYTES;
  static constexpr uint32_t OFF_A2 = OFF_A1 + 2 * A1_BYTES;
  static constexpr uint32_t OFF_BAR = OFF_A2 + 2 * A2_BYTES;
  static constexpr uint32_t SMEM = OFF_BAR + 128;
  static constexpr uint32_t TMEM_COLS = 64;
  static constexpr uint32_t D2_COL = 32;
};

__global__ void __launch_bounds__(160)
tri_tc_kernel(int64_t E, const float *__restrict__ rec, const int32_t *__restrict__ conn,
              const uint4 *__restrict__ table, const float *__restrict__ u, float *__restrict__ r,
              int *__restrict__ err, long long wait_limit, int hold) {
  using S = TriTcShape;
  constexpr int P = S::P, NE = S::NE;
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + S::OFF_BAR);
  // bar[0] A1 full (128) | bar[1] GEMM 1 done | bar[2] A2 full (128) |
  // bar[3] GEMM 2 done | bar[4] drain
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + S::OFF_BAR + 5 * 8);
  volatile int *flag = reinterpret_cast<volatile int *>(sm + S::OFF_BAR + 5 * 8 + 4);
  // a barrier nothing arrives on (hold != 0: the timeout-path test)
  uint64_t *never = reinterpret_cast<uint64_t *>(sm + S::OFF_BAR + 7 * 8);
  const uint32_t sbase = smem_addr(sm);

  for (int i = tid; i < (int)(S::TAB_BYTES / 16); i += S::THREADS)
    reinterpret_cast<uint4 *>(sm)[i] = table[i];
  if (tid == 0) {
    mbar_init(&bar[0], S::WORKERS);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], S::WORKERS);
    mbar_init(&bar[3], 1);
    mbar_init(&bar[4], 1);
    mbar_init(never, 1);
    *flag = 0;
    fence_mbar_init();
  }
  if (warp == 4) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tslot)),
                 "r"(S::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_proxy_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tslot;
  const int64_t ntiles = (E + NE - 1) / NE;

  if (warp == 4) {
    // ---------------- MMA issuer (whole warp loops, lane 0 issues) ----------------
    constexpr uint32_t I1 = tc::idesc_tf32(128, 32, false);
    constexpr uint32_t I2 = tc::idesc_tf32(128, 16, false);
    const uint32_t b1_hi = sbase + S::OFF_B1, b1_lo = b1_hi + S::B_BYTES;
    const uint32_t b2_hi = sbase + S::OFF_B2, b2_lo = b2_hi + S::B_BYTES;
    const uint32_t a1_hi = sbase + S::OFF_A1, a1_lo = a1_hi + S::A1_BYTES;
    const uint32_t a2_hi = sbase + S::OFF_A2, a2_lo = a2_hi + S::A2_BYTES;
    const bool leader = lane == 0;
    auto wwait = [&](uint64_t *b, uint32_t p, int code) {
      return __all_sync(0xffffffffu, tc::wait(b, p, flag, code, wait_limit) ? 1 : 0) != 0;
    };
    uint32_t it = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
      const uint32_t par = it & 1;
      if (!wwait(&bar[0], par, 1100)) break;
      tc::fence_after();
      if (leader) {
        for (int s = 0; s < 2; ++s) {
          const uint32_t ko = (uint32_t)s * 256u;
          const uint64_t ah = tc::desc(a1_hi + ko, 128, S::A1_SBO);
          const uint64_t al = tc::desc(a1_lo + ko, 128, S::A1_SBO);
          const uint64_t bh = tc::desc(b1_hi + ko, 128, S::B1_SBO);
          const uint64_t bl = tc::desc(b1_lo + ko, 128, S::B1_SBO);
          tc::mma_tf32(tmem, ah, bh, I1, s > 0);
          tc::mma_tf32(tmem, al, bh, I1, 1);
          tc::mma_tf32(tmem, ah, bl, I1, 1);
        }
        tc::commit(&bar[1]);
      }
      __syncwarp();
      if (!wwait(&bar[2], par, 1102)) break;
      tc::fence_after();
      if (leader) {
        for (int s = 0; s < 4; ++s) {
          const uint32_t ko = (uint32_t)s * 256u;
          const uint64_t ah = tc::desc(a2_hi + ko, 128, S::A2_SBO);
          const uint64_t al = tc::desc(a2_lo + ko, 128, S::A2_SBO);
          const uint64_t bh = tc::desc(b2_hi + ko, 128, S::B2_SBO);
          const uint64_t bl = tc::desc(b2_lo + ko, 128, S::B2_SBO);
          tc::mma_tf32(tmem + S::D2_COL, ah, bh, I2, s > 0);
          tc::mma_tf32(tmem + S::D2_COL, al, bh, I2, 1);
          tc::mma_tf32(tmem + S::D2_COL, ah, bl, I2, 1);
        }
        tc::commit(&bar[3]);
      }
      __syncwarp();
    }
    // drain every MMA issued by lane 0 before the memory is released
    if (leader) {
      tc::commit(&bar[4]);
      const long long t0 = clock64();
      while (!mbar_try_wait(&bar[4], 0) && clock64() - t0 < (1ll << 31)) {
      }
    }
    __syncwarp();
  } else {
    // ---------------- workers: thread = element row ----------------
    const int row = warp * 32 + lane;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    unsigned char *a1h = sm + S::OFF_A1, *a1l = a1h + S::A1_BYTES;
    unsigned char *a2h = sm + S::OFF_A2, *a2l = a2h + S::A2_BYTES;
    auto wwait = [&](uint64_t *b, uint32_t p, int code) {
      return __all_sync(0xffffffffu, tc::wait(b, p, flag, code, wait_limit) ? 1 : 0) != 0;
    };
    // The next tile's connectivity, record and u are loaded while this
    // tile's MMAs and pointwise stage run (software pipelining across tiles).
    float uv[16], rc[16];
    auto load_tile = [&](int64_t tile) {
      const int64_t e = tile * NE + row;
      if (tile < ntiles && e < E) {
        const int4 *c4 = reinterpret_cast<const int4 *>(conn + e * P);
        int cn[12];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
          const int4 x = __ldg(c4 + v);
          cn[4 * v] = x.x; cn[4 * v + 1] = x.y; cn[4 * v + 2] = x.z; cn[4 * v + 3] = x.w;
        }
        const float4 *r4 = reinterpret_cast<const float4 *>(rec + e * kTriRec);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const float4 x = __ldg(r4 + v);
          rc[4 * v] = x.x; rc[4 * v + 1] = x.y; rc[4 * v + 2] = x.z; rc[4 * v + 3] = x.w;
        }
#pragma unroll
        for (int j = 0; j < 12; ++j) uv[j] = __ldg(u + cn[j]);
      } else {
#pragma unroll
        for (int j = 0; j < 12; ++j) uv[j] = 0.f;
#pragma unroll
        for (int v = 0; v < 16; ++v) rc[v] = 0.f;
      }
#pragma unroll
      for (int j = 12; j < 16; ++j) uv[j] = 0.f;
    };
    load_tile(blockIdx.x);
    // hold: wait first on a barrier nothing arrives on, so that the wait runs
    // out after wait_limit cycles and the CTA takes its timeout path
    const bool held = hold && !wwait(never, 0u, 1099);
    uint32_t it = 0;
    for (int64_t tile = blockIdx.x; !held && tile < ntiles; tile += gridDim.x, ++it) {
      const uint32_t par = it & 1;
      const int64_t e = tile * NE + row;
      const bool ok = e < E;
      // A1 <- u (hi, lo)
#pragma unroll
      for (int jc = 0; jc < 4; ++jc) {
        float4 h, l;
        tc::split(uv[4 * jc + 0], h.x, l.x);
        tc::split(uv[4 * jc + 1], h.y, l.y);
        tc::split(uv[4 * jc + 2], h.z, l.z);
        tc::split(uv[4 * jc + 3], h.w, l.w);
        const uint32_t off = tc::kmajor_off(row, 4 * jc, S::A1_SBO);
        *reinterpret_cast<float4 *>(a1h + off) = h;
        *reinterpret_cast<float4 *>(a1l + off) = l;
      }
      tc::fence_before();
      fence_proxy_async_smem();
      tc::arrive(&bar[0]);
      // this tile's metric and weights, then the next tile's loads in flight
      float cur[16];
#pragma unroll
      for (int v = 0; v < 16; ++v) cur[v] = rc[v];
      load_tile(tile + gridDim.x);
      if (!wwait(&bar[1], par, 1001)) break;
      tc::fence_after();
      float g[2][16];
#pragma unroll
      for (int c8 = 0; c8 < 4; ++c8)
        tc::ld8(tmem + lane_base + (uint32_t)(8 * c8), &g[c8 >> 1][8 * (c8 & 1)]);
      tc::ld_wait();
      // fluxes F[k][q] = s_q (G_k0 g0 + G_k1 g1); padding nodes zero
      const float g00 = cur[0], g01 = cur[1], g11 = cur[2];
      float F[2][16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float s = q < 12 ? cur[4 + q] : 0.f;
        F[0][q] = s * (g00 * g[0][q] + g01 * g[1][q]);
        F[1][q] = s * (g01 * g[0][q] + g11 * g[1][q]);
      }
#pragma unroll
      for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int qc = 0; qc < 4; ++qc) {
          float4 h, l;
          tc::split(F[k][4 * qc + 0], h.x, l.x);
          tc::split(F[k][4 * qc + 1], h.y, l.y);
          tc::split(F[k][4 * qc + 2], h.z, l.z);
          tc::split(F[k][4 * qc + 3], h.w, l.w);
          const uint32_t off = tc::kmajor_off(row, 16 * k + 4 * qc, S::A2_SBO);
          *reinterpret_cast<float4 *>(a2h + off) = h;
          *reinterpret_cast<float4 *>(a2l + off) = l;
        }
      tc::fence_before();
      fence_proxy_async_smem();
      tc::arrive(&bar[2]);
      if (!wwait(&bar[3], par, 1003)) break;
      tc::fence_after();
      float out[16];
      tc::ld8(tmem + lane_base + S::D2_COL, out);
      tc::ld8(tmem + lane_base + S::D2_COL + 8u, out + 8);
      tc::ld_wait();
      if (ok) {
        float4 *o4 = reinterpret_cast<float4 *>(r + e * P);
#pragma unroll
        for (int v = 0; v < 3; ++v)
          o4[v] = make_float4(-out[4 * v], -out[4 * v + 1], -out[4 * v + 2], -out[4 * v + 3]);
      }
    }
  }
  tc::fence_before();
  __syncthreads();
  if (*flag && tid == 0 && err) atomicExch(err, *flag);
  if (warp == 4) {
    __syncwarp();
    tc::fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(S::TMEM_COLS)
                 : "memory");
  }
}

}  // namespace salvus
