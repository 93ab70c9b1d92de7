// kernels_group.cuh -- time steps for a group of independent FP32 problems
// (meshes of one element class, uneven sizes).  Every piece of work runs the
// same per-CTA body as the single-problem kernel, on its member's arrays, so
// each member's arithmetic -- and its result, bit for bit -- is the one it
// gets alone.
//
// Per step, per member, the single-problem order (abi.cu step_fused_t):
// stiffness, source, gather/update, receivers, step-counter advance.
//
// group_persistent_step: ONE launch per step for the whole group.  Resident
// CTAs take work items from a queue, all members' stiffness tiles first, then
// per member its source item, gather tiles, receiver items and advance item.
// An item waits (bounded) only for its own member's earlier items, which sit
// earlier in the queue and so were taken by running CTAs that never wait on
// later items: no deadlock, and no device-wide barrier between stages, so one
// member's gather overlaps another's stiffness.  The last CTA to finish resets
// the queue for the next launch.
//
// The per-stage kernels below (one launch per stage) are kept as the
// reference form of the same work.
#pragma once

#include <cstdint>

namespace salvus {

struct GroupSlot {
  // mesh (hexahedra: jac != nullptr for parallelepiped meshes, whose rec holds
  // the material planes of kernels_hex_affine.cuh)
  const float *rec, *jac;
  const int32_t *conn, *inc_off, *inc_idx;
  const float *mi;
  int64_t E, G;
  // problem
  float *u, *v, *ap, *a, *r;
  float dt;
  double dtd;
  int64_t *step;
  int nsrc, nrec;
  const int64_t *src_elem;
  const double *src_par, *src_wts;
  const int64_t *rec_elem;
  const double *rec_l;
  double *seis;
  int64_t cap;
  // first CTA of this member in each grouped launch
  int64_t b_stiff, b_gather, b_rec;
};

// Stiffness of element group bid of one member: the body its solo run uses
// (parallelepiped records or per-point records), so the result is the same.
template <int N, int EPB>
__device__ __forceinline__ void group_hex_body(const GroupSlot &m, int64_t bid,
                                               const DMatrix<float> &Dm) {
  if (m.jac) {
    const HexInteriorUpdate none{};
    elastic_hex_affine_body<N, EPB, false, false>(bid, m.E, m.jac, m.rec, m.conn, m.u, m.r, Dm,
                                                  none);
  } else {
    elastic_hex_v2_body<N, EPB, false>(bid, m.E, m.rec, m.u, m.r, Dm);
  }
}

// owner[b]: the member whose CTA range of this launch holds CTA b (a table
// per stage, filled on the host; one load instead of a search).

template <int N>
__global__ void __launch_bounds__(QuadColShape<N, quad_col_epb<N>()>::THREADS)
group_quad_acoustic_stiffness(const GroupSlot *__restrict__ slots,
                              const int32_t *__restrict__ owner, DMatrix<float> Dm) {
  const GroupSlot &m = slots[owner[blockIdx.x]];
  acoustic_quad_col_body<N, quad_col_epb<N>(), float>(blockIdx.x - m.b_stiff, m.E, m.rec, m.conn,
                                                       m.u, m.r, Dm);
}

template <int N, int EPB>
__global__ void __launch_bounds__(ElasticV2Shape<N, EPB, false>::THREADS)
group_hex_elastic_stiffness(const GroupSlot *__restrict__ slots,
                            const int32_t *__restrict__ owner, DMatrix<float> Dm) {
  const GroupSlot &m = slots[owner[blockIdx.x]];
  group_hex_body<N, EPB>(m, blockIdx.x - m.b_stiff, Dm);
}

// one CTA per member
template <int C>
__global__ void group_source(const GroupSlot *__restrict__ slots, int P) {
  const GroupSlot &m = slots[blockIdx.x];
  if (m.nsrc > 0) source_body<float, C>(m.nsrc, P, m.src_elem, m.src_par, m.src_wts, m.step, m.dtd, m.r);
}

template <int C>
__global__ void group_gather_update(const GroupSlot *__restrict__ slots,
                                    const int32_t *__restrict__ owner) {
  const GroupSlot &m = slots[owner[blockIdx.x]];
  const int64_t g = (blockIdx.x - m.b_gather) * (int64_t)blockDim.x + threadIdx.x;
  gather_body<float, C, 0>(g, m.G, m.inc_off, m.inc_idx, m.r, m.mi, m.u, m.v, m.ap, m.a, m.dt);
}

template <int C>
__global__ void __launch_bounds__(kRecThreads)
group_receivers(const GroupSlot *__restrict__ slots, const int32_t *__restrict__ owner, int P) {
  const GroupSlot &m = slots[owner[blockIdx.x]];
  receiver_body<float, C>((int)(blockIdx.x - m.b_rec), P, m.rec_elem, m.rec_l, m.conn, m.u, m.seis,
                          m.cap, m.step);
}

__global__ void group_advance(const GroupSlot *__restrict__ slots, int J) {
  for (int s = threadIdx.x; s < J; s += blockDim.x) *slots[s].step += 1;
}

// ---------------------------------------------------------------------------
// persistent single-launch step
enum GroupItem { GI_STIFF = 0, GI_SRC = 1, GI_GATHER = 2, GI_REC = 3, GI_ADV = 4 };

struct GroupCounts {  // work items per member and type
  int32_t stiff, gather, rec;
};

struct GroupSync {
  unsigned long long head;
  unsigned int finished;
  int err;
};

// spin (bounded: `limit` SM cycles, 2^31 -- about a second -- by default)
// until *c >= target; thread 0 only
__device__ __forceinline__ bool group_wait(const int32_t *c, int32_t target, GroupSync *sync,
                                           long long limit) {
  const long long t0 = clock64();
  while (*(volatile const int32_t *)c < target) {
    if (*(volatile int *)&sync->err) return false;
    if (clock64() - t0 > limit) {
      atomicExch(&sync->err, 1);
      return false;
    }
    __nanosleep(64);
  }
  __threadfence();
  return true;
}

// Work item: type, member, first tile, tile count (stiffness: element
// groups of the single-problem kernel; gather: CTA-wide node tiles).
struct GroupWork {
  int type, member, first, count;
};

template <int N, bool kHex, int C>
__global__ void __launch_bounds__(128)
group_persistent_step(const GroupSlot *__restrict__ slots, const GroupCounts *__restrict__ counts,
                      int J, const GroupWork *__restrict__ work, int64_t total,
                      int32_t *__restrict__ done /* [J][4] */, GroupSync *__restrict__ sync,
                      DMatrix<float> Dm, int P, long long wait_limit) {
  constexpr int n2 = (N + 1) * (N + 1);
  constexpr int EPB = kHex ? (128 / n2 > 0 ? 128 / n2 : 1) : 1;
  __shared__ long long s_item;
  __shared__ int s_ok;
  const int t = threadIdx.x;
  // thread 0 claims the next item while the CTA works on the current one
  long long next = 0;
  if (t == 0) next = (long long)atomicAdd(&sync->head, 1ull);
  for (;;) {
    __syncthreads();
    if (t == 0) {
      s_item = next;
      if (next < total) next = (long long)atomicAdd(&sync->head, 1ull);
    }
    __syncthreads();
    const long long item = s_item;
    if (item >= total) break;
    const GroupWork w = work[item];
    const GroupSlot &m = slots[w.member];
    const GroupCounts &cn = counts[w.member];
    int32_t *dj = done + 4 * w.member;
    // dependencies (thread 0 waits, the CTA follows)
    if (t == 0) {
      bool ok = true;
      if (w.type == GI_SRC) ok = group_wait(dj + GI_STIFF, cn.stiff, sync, wait_limit);
      else if (w.type == GI_GATHER) ok = group_wait(dj + GI_SRC, 1, sync, wait_limit);
      else if (w.type == GI_REC) ok = group_wait(dj + GI_GATHER, cn.gather, sync, wait_limit);
      else if (w.type == GI_ADV)
        ok = group_wait(dj + GI_GATHER, cn.gather, sync, wait_limit) && group_wait(dj + GI_REC, cn.rec, sync, wait_limit);
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) continue;  // a wait gave up: the error word is set, skip the work
    switch (w.type) {
      case GI_STIFF:
        for (int b = w.first; b < w.first + w.count; ++b) {
          if constexpr (kHex)
            group_hex_body<N, EPB>(m, b, Dm);
          else
            acoustic_quad_col_body<N, quad_col_epb<N>(), float>(b, m.E, m.rec, m.conn, m.u, m.r, Dm);
          __syncthreads();
        }
        break;
      case GI_SRC:
        if (m.nsrc > 0) source_body<float, C>(m.nsrc, P, m.src_elem, m.src_par, m.src_wts, m.step, m.dtd, m.r);
        break;
      case GI_GATHER:
        for (int b = w.first; b < w.first + w.count; ++b)
          gather_body<float, C, 0, true>((int64_t)b * blockDim.x + t, m.G, m.inc_off, m.inc_idx, m.r, m.mi,
                                   m.u, m.v, m.ap, m.a, m.dt);
        break;
      case GI_REC:
        receiver_body<float, C, true>(w.first, P, m.rec_elem, m.rec_l, m.conn, m.u, m.seis, m.cap, m.step);
        break;
      default:
        if (t == 0) *m.step += 1;
        break;
    }
    __syncthreads();
    if (t == 0 && w.type != GI_ADV) {
      __threadfence();
      atomicAdd(dj + w.type, 1);
    }
  }
  // the last CTA out resets the queue and the counters for the next launch
  __shared__ int s_last;
  if (t == 0) {
    __threadfence();
    s_last = atomicAdd(&sync->finished, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    for (int x = t; x < 4 * J; x += blockDim.x) done[x] = 0;
    __syncthreads();
    if (t == 0) {
      sync->head = 0ull;
      sync->finished = 0u;
      __threadfence();
    }
  }
}

// ---------------------------------------------------------------------------
// member-partitioned single-launch step
//
// group_partitioned_step: ONE cooperative launch per step.  Every member owns
// a contiguous range of co-resident CTAs (sized to its share of the group's
// work) and runs its whole step inside that range: stiffness tiles
// round-robin over its CTAs; the member's first CTA, once all of them are
// through the stiffness, adds the sources; after a flag every CTA takes its
// gather tiles; after all gathers the receivers are spread over the CTAs;
// the first CTA then advances the step.  A CTA only ever waits (bounded) for
// CTAs of its own member, so members never hold each other up, and the
// cooperative launch guarantees that all CTAs are resident.
struct GroupPart {
  int32_t cta_first, cta_count;  // the member's CTAs
  int32_t n_stiff, n_gather;     // element groups, 128-node gather tiles
};
struct GroupBar {  // per member; the member's last CTA out zeroes it
  int32_t stiff_done, src_done, gather_done, rec_done, out;
};

template <int N, bool kHex, int C>
__global__ void __launch_bounds__(128, kHex ? 5 : 10)
group_partitioned_step(const GroupSlot *__restrict__ slots, const GroupPart *__restrict__ parts,
                       int J, GroupBar *__restrict__ bars, GroupSync *__restrict__ sync,
                       DMatrix<float> Dm, int P, long long wait_limit) {
  constexpr int n2 = (N + 1) * (N + 1);
  constexpr int EPB = kHex ? (128 / n2 > 0 ? 128 / n2 : 1) : 1;
  __shared__ int s_ok;
  const int t = threadIdx.x;
  // member of this CTA (cta_first ascending)
  int lo = 0, hi = J - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (parts[mid].cta_first <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const GroupPart pt = parts[lo];
  const GroupSlot &m = slots[lo];
  GroupBar *gb = bars + lo;
  const int b = (int)blockIdx.x - pt.cta_first, nb = pt.cta_count;
  auto member_wait = [&](const int32_t *c, int32_t target) {
    if (t == 0) s_ok = group_wait(c, target, sync, wait_limit);
    __syncthreads();
    return s_ok != 0;
  };
  auto arrive = [&](int32_t *c) {
    __syncthreads();
    if (t == 0) {
      __threadfence();
      atomicAdd(c, 1);
    }
  };
  // stiffness
  for (int k = b; k < pt.n_stiff; k += nb) {
    if constexpr (kHex)
      group_hex_body<N, EPB>(m, k, Dm);
    else
      acoustic_quad_col_body<N, quad_col_epb<N>(), float>(k, m.E, m.rec, m.conn, m.u, m.r, Dm);
    __syncthreads();
  }
  arrive(&gb->stiff_done);
  bool ok = true;
  if (b == 0) {
    ok = member_wait(&gb->stiff_done, nb);
    if (ok && m.nsrc > 0)
      source_body<float, C>(m.nsrc, P, m.src_elem, m.src_par, m.src_wts, m.step, m.dtd, m.r);
    __syncthreads();
    if (t == 0) {
      __threadfence();
      atomicExch(&gb->src_done, 1);
    }
  }
  ok = ok && member_wait(&gb->src_done, 1);
  // gather and update
  if (ok)
    for (int k = b; k < pt.n_gather; k += nb)
      gather_body<float, C, 0, true>((int64_t)k * 128 + t, m.G, m.inc_off, m.inc_idx, m.r, m.mi,
                                     m.u, m.v, m.ap, m.a, m.dt);
  arrive(&gb->gather_done);
  ok = ok && member_wait(&gb->gather_done, nb);
  // receivers
  if (ok)
    for (int k = b; k < m.nrec; k += nb)
      receiver_body<float, C, true>(k, P, m.rec_elem, m.rec_l, m.conn, m.u, m.seis, m.cap, m.step);
  arrive(&gb->rec_done);
  if (b == 0) {
    ok = ok && member_wait(&gb->rec_done, nb);
    if (ok && t == 0) *m.step += 1;
  }
  // the member's last CTA out resets its counters for the next launch
  __syncthreads();
  if (t == 0) {
    __threadfence();
    if (atomicAdd(&gb->out, 1) == nb - 1) {
      gb->stiff_done = 0;
      gb->src_done = 0;
      gb->gather_done = 0;
      gb->rec_done = 0;
      gb->out = 0;
      __threadfence();
    }
  }
}

}  // namespace salvus
