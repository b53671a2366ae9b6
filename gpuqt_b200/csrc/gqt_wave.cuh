// The wavefront moment loop of the FP64 form: S Chebyshev steps in one persistent
// launch, so that all but the leading step read their vectors from L2.
//
// The sites are cut into C chunks of CS consecutive sites. A work item is one step s
// of one chunk: it needs step s - 1 done on the chunks its sites' neighbours lie in,
// and once it is done step s + 1 may overwrite the chunk's T_{s-1} (the recurrence
// writes T_s over T_{s-2} in place). Chunks are visited in a position order (the
// identity, or a fold 0, C-1, 1, C-2, ... that brings the chunks a periodic boundary
// joins next to each other) in which every item's dependencies lie within K
// positions.
//
// Items are handed out by one atomic ticket counter in the order of their level
// tau = q + j * Lg (q the position, j = s - s0 the step within the launch, Lg > K the
// lag between consecutive steps), lower steps first within a level. An item waits only
// for items of step s - 1 at positions q - K .. q + K, whose level is at most
// tau - (Lg - K) < tau, so their tickets are smaller: they were taken by blocks that
// are already running and that, by the same argument, finish. No block waits on a
// block that has not started, so the launch needs no co-residency guarantee. Every
// wait is bounded all the same: a wait that runs out sets an error flag the host
// reads and the block carries on.
//
// Per-site arithmetic is that of k_step (ExactArith, reference operation order), so
// every T_m is bit-identical to the step-by-step loop's. Vectors written during the
// launch are read through L2 only (ld.global.cg): a chunk's T buffer is rewritten
// every two steps, and L1 is not coherent across blocks. Each item leaves one
// compensated moment partial per warp in a slab row of its step; k_slab_combine then
// sums a step's 8 C partials in chunk order, so the moments do not depend on the
// schedule.
#pragma once

#include "gqt_kernels.cuh"

namespace gqt {

// The schedule of one wavefront launch (host-computed, see wave_plan).
struct WavePlan {
  int chunks;  // C
  int sites;   // CS: sites per chunk (a multiple of kBlock)
  int halo;    // K: positions an item depends on, either side
  int lag;     // Lg: levels between consecutive steps of one chunk
  int fold;    // 1: positions visit the chunks in folded order
};

// Counters of a wavefront loop (device memory, zero at the start of every launch:
// the last block to leave a launch resets them).
struct WaveCtl {
  unsigned ticket;
  unsigned exited;
  unsigned err;  // set when a bounded wait ran out
  unsigned pad;
};

constexpr int kWaveWarps = kBlock / 32;

__host__ __device__ __forceinline__ int wave_chunk(const WavePlan& p, int q)
{
  if (!p.fold)
    return q;
  return (q & 1) ? p.chunks - 1 - (q >> 1) : (q >> 1);
}

__host__ __device__ __forceinline__ unsigned wave_tickets(const WavePlan& p, int steps)
{
  return (unsigned)steps * (unsigned)(p.chunks + (steps - 1) * p.lag);
}

__device__ __forceinline__ int ld_acquire(const int* f)
{
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(f) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(int* f, int v)
{
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(f), "r"(v) : "memory");
}

// Wait until *f >= need, for a bounded time (2^22 polls, on the order of a second);
// on timeout flag the error. Once any wait has timed out, every wait of the loop
// returns at once: the launch then ends promptly with invalid moments, which the host
// reports, instead of spending the bound again on every item.
__device__ __forceinline__ void wave_wait(const int* f, int need, WaveCtl* ctl)
{
  const volatile unsigned* err = &ctl->err;
  for (int it = 0; it < (1 << 22); ++it) {
    if (ld_acquire(f) >= need)
      return;
    if ((it & 255) == 0 && *err)
      return;
    __nanosleep(128);
  }
  atomicOr(&ctl->err, 1u);
}

// The streamed inputs of one site: potential, T_{s-1}, T_{s-2} (through L2: this
// launch writes them) and left (never written by the loop).
struct WaveIn {
  double p;
  double2 x, y0, l;
};

template <int Z>
__device__ __forceinline__ void wave_fetch(const Op& op, int i, const double2* t0,
                                           const double2* t1, const double2* left,
                                           RowIdx<Z>& r, WaveIn& w)
{
  fetch_row<Z, true>(op, i, r);
  w.p = __ldg(op.pot + i);
  w.x = __ldcg(t1 + i);
  w.y0 = __ldcg(t0 + i);
  w.l = __ldg(left + i);
}

// Steps s0 .. s0 + steps - 1 of the moment loop (s0 >= 2) over the coded operator, one
// vector. Buffers: T_0 = R (read only), T_m = A for odd m, B for even m >= 2 (T_m is
// written over T_{m-2}); left is read only. done[q] holds the last step completed at
// position q; slab row j receives step s0 + j's partials, [chunk][warp][4] doubles.
template <int Z>
__global__ void __launch_bounds__(kBlock, step_min_blocks<Z>()) k_wave(
  Op op, WavePlan wp, int s0, int steps, const double2* __restrict__ R, double2* A, double2* B,
  const double2* __restrict__ left, int* done, WaveCtl* ctl, double* __restrict__ slab)
{
  const Tables tb = load_tables<true>(op);
  __shared__ unsigned s_ticket;
  const unsigned total = wave_tickets(wp, steps);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0)
      s_ticket = atomicAdd(&ctl->ticket, 1u);
    __syncthreads();
    const unsigned t = s_ticket;
    __syncthreads();
    if (t >= total)
      break;  // uniform: every thread read the same ticket
    const int tau = (int)(t / (unsigned)steps);
    const int j = (int)(t % (unsigned)steps);
    const int q = tau - j * wp.lag;
    if (q < 0 || q >= wp.chunks)
      continue;  // outside the wavefront's ramps
    const int s = s0 + j;
    // step s - 1 must be done on every position this chunk's rows reach
    for (int d = threadIdx.x; d <= 2 * wp.halo; d += kBlock) {
      const int qq = q - wp.halo + d;
      if (qq >= 0 && qq < wp.chunks)
        wave_wait(done + qq, s - 1, ctl);
    }
    __syncthreads();
    const double2* t1 = ((s - 1) & 1) ? A : B;
    const double2* t0 = (s == 2) ? R : (((s - 2) & 1) ? A : B);
    double2* out = (s & 1) ? A : B;
    const int c = wave_chunk(wp, q);
    const int first = c * wp.sites;
    const int last = (first + wp.sites < op.n) ? first + wp.sites : op.n;
    CSum re{0.0, 0.0}, im{0.0, 0.0};
    int i = first + (int)threadIdx.x;
    RowIdx<Z> cur;
    WaveIn wn;
    if (i < last)
      wave_fetch<Z>(op, i, t0, t1, left, cur, wn);
    for (; i < last; i += kBlock) {
      // k_step's pipelined body: the next site's row and streams are in flight while
      // this site's gathers are
      const WaveIn w = wn;
      RowIdx<Z> nxt = cur;
      if (i + kBlock < last)
        wave_fetch<Z>(op, i + kBlock, t0, t1, left, nxt, wn);
      double tr = ExactArith::mul(w.p, w.x.x);
      double ti = ExactArith::mul(w.p, w.x.y);
      int jn[Z];
      double2 h[Z], y[Z];
#pragma unroll
      for (int m = 0; m < Z; ++m) {
        jn[m] = i + tb.delta[cur.idx[m]];
        h[m] = tb.hop[cur.idx[m]];
      }
#pragma unroll
      for (int m = 0; m < Z; ++m)
        if (m < cur.cnt)
          y[m] = __ldcg(t1 + jn[m]);
#pragma unroll
      for (int m = 0; m < Z; ++m) {
        if (m < cur.cnt) {
          tr = ExactArith::add(tr, ExactArith::cre(h[m].x, h[m].y, y[m].x, y[m].y));
          ti = ExactArith::add(ti, ExactArith::cim(h[m].x, h[m].y, y[m].x, y[m].y));
        }
      }
      tr = ExactArith::two_x_minus(ExactArith::scale(tr, op), w.y0.x);
      ti = ExactArith::two_x_minus(ExactArith::scale(ti, op), w.y0.y);
      const double2 r = make_double2(tr, ti);
      __stcg(out + i, r);
      dot_term(re, im, r, w.l);
      cur = nxt;
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
      csum_merge(re, shfl_xor(re, off));
      csum_merge(im, shfl_xor(im, off));
    }
    if (lane == 0) {
      double* pp = slab + (((size_t)j * wp.chunks + c) * kWaveWarps + warp) * 4;
      pp[0] = re.s;
      pp[1] = re.c;
      pp[2] = im.s;
      pp[3] = im.c;
    }
    // this item's T_s and partials are visible before its position reports step s
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
      st_release(done + q, s);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&ctl->exited, 1u) == gridDim.x - 1) {
      ctl->ticket = 0u;  // every block has left: ready for the next launch
      ctl->exited = 0u;
    }
  }
}

// Start of a wavefront moment loop: steps 0 and 1 done everywhere, counters cleared,
// and the slab combine told the partials per row (counter[1], as the deferred steps do).
__global__ void __launch_bounds__(kBlock) k_wave_init(int* done, int chunks, WaveCtl* ctl,
                                                      unsigned* counter, unsigned per_row)
{
  for (int q = blockIdx.x * kBlock + threadIdx.x; q < chunks; q += gridDim.x * kBlock)
    done[q] = 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->ticket = 0u;
    ctl->exited = 0u;
    counter[1] = per_row;
  }
}

}  // namespace gqt
