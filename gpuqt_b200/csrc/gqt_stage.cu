// The staged Chebyshev step of the FP32 moment loops over the coded operator (sm_100a).
//
// The sites are cut into tiles of TS consecutive sites; block b takes tiles b, b + G,
// b + 2G, ... (G resident blocks), so the GPU sweeps one compact front of tiles and the
// rows a tile gathers were read by nearby tiles shortly before (L2 hits). A gather of
// site i reads T_{k-1} at i + d for the offset d of its code. The frequent offsets form
// a few windows: window w covers the offsets [lo_w, hi_w], so a tile starting at site t
// reads the rows [t + lo_w, t + TS + hi_w) of it. With the vectors interleaved per site
// ([site][vector]), each window is one contiguous byte range of T_{k-1}.
//
// One producer thread (a warp of its own) copies a tile's windows and its T_{k-2} rows
// into one of S shared-memory stages with bulk asynchronous copies (cp.async.bulk,
// completing on the stage's full mbarrier), up to S tiles ahead of the compute warps,
// which release a stage through its empty mbarrier. The compute threads read
// these operands from shared memory (one 16-byte load per row and thread,
// conflict-free); the codes, the potential and (GQT_FP32R, moment <left|T_k>) the left
// entries of the next tile are loaded one tile ahead into registers. Offsets outside the windows (the periodic wraps: a
// few rows per lattice line) are gathered from global memory.
//
// Per element the arithmetic is that of k_step_vec with FastArith (src/sigma.cu:33-61's
// recurrence, the operator in FP64, T_k rounded to FP32 once), so T_k is the unstaged
// step's bit for bit: entries past a row's length are the padding entries of the coded
// table (offset 0, hopping 0) and add an exact zero instead of being skipped. The
// moments are the same per-thread FP64 sums taken over the sites in another order.
//
// Every wait on an mbarrier is bounded; one that runs out sets *op.stage_err and ends
// the loop of the warp (or of the producer, which stops copying) that waited; the
// producer waits once more (bounded) for every copy it issued before the block exits.
#include "gqt_forms_impl.cuh"

#include <mutex>
#include <unordered_map>

namespace gqt {

namespace {

constexpr int kMaxStages = 4;
constexpr int kComputeWarps = kBlock / 32;
constexpr int kStageThreads = kBlock + 32;  // the compute warps and one producer warp
constexpr int kStageW = 4;  // vectors per thread: two 16-byte chunks of a row

// Byte layout of one stage for a launch (host-computed from the operator's windows).
struct StageLayout {
  int stages;
  int stage_bytes;
  int nw;
  int win_lo[kStageWin];    // window w holds rows [tile + win_lo, tile + win_lo + win_rows)
  int win_rows[kStageWin];
  int win_off[kStageWin];   // byte offset of window w in a stage
  int t0_off;               // T_{k-2} rows of the tile (kCheb), -1 otherwise
};

__device__ __forceinline__ uint32_t sm_addr(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sm_addr(b)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect(uint64_t* b, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_addr(b)),
               "r"(bytes)
               : "memory");
}

// One try: true once phase `parity` of b has completed; the thread may be suspended for
// up to about 1 microsecond (the suspend-time hint) while it has not.
__device__ __forceinline__ void mbar_arrive(uint64_t* b)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sm_addr(b)) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* b, unsigned parity)
{
  unsigned ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
    "selp.u32 %0, 1, 0, p;\n\t}"
    : "=r"(ok)
    : "r"(sm_addr(b)), "r"(parity), "r"(1000u)
    : "memory");
  return ok != 0;
}

// Wait for phase `parity` of b, for at most 2^20 tries (about a second): false when it
// did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity)
{
  for (int it = 0; it < (1 << 20); ++it)
    if (mbar_test(b, parity))
      return true;
  return false;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          uint64_t* b)
{
  asm volatile(
    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
      "r"(sm_addr(dst)),
    "l"(src), "r"(bytes), "r"(sm_addr(b))
    : "memory");
}

__device__ __forceinline__ void fence_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Result index of sum slot k of the threads with lane % (V / 4) == q, H = V / 4 chunks in
// half a row: vector 2 q + k for k < 2, 2 (q + H) + k - 2 otherwise; P = 2 for the pair
// sums ([2 v] <T_k|T_k>, [2 v + 1] <T_{k-1}|T_k> in slots 2k', 2k' + 1).
template <int H, int P>
struct StageSlots {
  __device__ __forceinline__ int operator()(int q, int k, int) const
  {
    const int kk = k / P;
    return P * (2 * q + (kk & 1) + (kk >> 1) * 2 * H) + k % P;
  }
};

// F32 = false: the GQT_FP32 form (operator and arithmetic in FP64, T_k rounded to FP32).
// F32 = true: the GQT_FP32R form (recurrence_f32 below).
// The GQT_FP32R form, a recurrence in FP32. The operator H / E_max (hoppings and
// potential multiplied by RN(1 / E_max) in FP64) is kept as two FP32 parts, hi =
// RN_fp32(a) and lo = RN_fp32(a - hi), so that it is not perturbed at FP32 precision (a
// fixed perturbation of H shifts the spectrum, and its error grows linearly with the
// moment index); (H / E_max) T_{k-1} is summed with FP32 fused multiply-adds, the hi
// products and the lo products in two accumulators (neighbours in ELL order), and T_k =
// 2 (hi + lo) - T_{k-2} is formed with one rounding of the hi part (cheb_part). The
// moments are summed in FP64 from the stored FP32 values (the product of two FP32
// values is exact in FP64).
__device__ __forceinline__ float2 split_f32(double a)
{
  const float hi = (float)a;
  return make_float2(hi, (float)(a - (double)hi));
}

// (hi.x, hi.y, lo.x, lo.y) of a hopping divided by E_max
__device__ __forceinline__ float4 scaled_hop(double2 h, const Op& op)
{
  const float2 x = split_f32(h.x * op.inv_emax), y = split_f32(h.y * op.inv_emax);
  return make_float4(x.x, y.x, x.y, y.y);
}

// One vector element of the FP32 recurrence: hi and lo accumulators of both parts.
struct AccF32 {
  float r, i, rl, il;
};

// acc = p x (p = (hi, lo) of the potential divided by E_max)
__device__ __forceinline__ AccF32 acc_start(float2 p, float2 x)
{
  return AccF32{p.x * x.x, p.x * x.y, p.y * x.x, p.y * x.y};
}

// acc += h y, complex
__device__ __forceinline__ void cmac_f32(AccF32& a, float4 h, float2 y)
{
  a.r = fmaf(h.x, y.x, a.r);
  a.r = fmaf(-h.y, y.y, a.r);
  a.i = fmaf(h.x, y.y, a.i);
  a.i = fmaf(h.y, y.x, a.i);
  a.rl = fmaf(h.z, y.x, a.rl);
  a.rl = fmaf(-h.w, y.y, a.rl);
  a.il = fmaf(h.z, y.y, a.il);
  a.il = fmaf(h.w, y.x, a.il);
}

// One part of T_k = 2 (hi + lo) - T_{k-2} with a single rounding of the hi sum: 2 hi -
// T_{k-2} is split exactly into s + e (Knuth's TwoSum; 2 hi is exact), then 2 lo and e
// are added to s. The lo accumulator is mostly below half an ulp of hi (each lo part
// of the operator is below half an ulp of its hi part), so RN(hi + lo) is mostly hi:
// rounding that sum first dropped the lo parts and applied H rounded to FP32, a fixed
// perturbation of H whose error grows with the moment index. Adding 2 lo after rounding 2 hi - T_{k-2} drops
// them wherever T_{k-2} sets the scale. In a model of the recurrence (graphene, 2000
// moments) those finishes gave 14x and 7x the moment error of this one. Explicit
// round-to-nearest intrinsics keep the compiler from fusing the sequence.
__device__ __forceinline__ float cheb_part(float hi, float lo, float y0)
{
  const float s = __fmaf_rn(2.0f, hi, -y0);
  const float a1 = __fadd_rn(s, y0);      // the part of s from 2 hi
  const float b1 = __fsub_rn(s, a1);      // the part of s from -T_{k-2}
  const float e = __fadd_rn(__fmaf_rn(2.0f, hi, -a1), __fsub_rn(-y0, b1));
  return __fadd_rn(s, __fmaf_rn(2.0f, lo, e));
}

// T_k = 2 acc - T_{k-2} (kCheb), or acc (kApply)
template <int MODE>
__device__ __forceinline__ float2 acc_finish(const AccF32& a, float2 y0)
{
  if constexpr (MODE == kCheb)
    return make_float2(cheb_part(a.r, a.rl, y0.x), cheb_part(a.i, a.il, y0.y));
  else
    return make_float2(a.r + a.rl, a.i + a.il);
}

// MULTI: one step of a realisation batch (op.stage_rtab: each model's windows; md: the
// models' tiles and the per-block, per-model sum slots that k_tile_reduce combines).
// Tiles never straddle two models (every model is padded to 1024 sites). A block's
// tiles come in increasing order, so the models it meets are consecutive runs: when the
// next tile is in another model, the compute warps reduce their sums over the block
// (a named barrier of the compute warps only) and write the block's slot of the model.
template <int V, int Z, int MODE, int DOT, bool F32, bool MULTI = false>
__global__ void __launch_bounds__(kStageThreads, 2)
  k_step_staged(Op op, StageLayout sl, const float2* t0, const float2* __restrict__ t1,
                float2* out, const float2* __restrict__ left, Dot dot, MultiDot md)
{
  using A = FastArith;
  constexpr int W = kStageW;
  constexpr int kTps = V / W;        // threads per site
  constexpr int TS = kBlock / kTps;  // sites per tile
  constexpr int RB = V * (int)sizeof(float2);
  static_assert(kBlock % kTps == 0 && 32 % kTps == 0, "a site's threads share a warp");
  extern __shared__ __align__(128) unsigned char stage_smem[];
  const int S = sl.stages;
  // per stage: full (the copies have landed) and empty (every compute warp has read it)
  uint64_t* full = reinterpret_cast<uint64_t*>(stage_smem + (size_t)S * sl.stage_bytes);
  uint64_t* empty = full + kMaxStages;
  double2* hop = reinterpret_cast<double2*>(empty + kMaxStages);
  // GQT_FP32R: the hoppings divided by E_max as FP32 (hi, lo) parts
  float4* hopf = reinterpret_cast<float4*>(hop + op.n_codes);
  // per code: byte offset in a stage of site 0's neighbour row (-1: gathered from global
  // memory), and the offset j - i. MULTI: the byte offsets per model and code (coff) and
  // the offsets j - i per code (cdelta) instead.
  int2* cinfo = reinterpret_cast<int2*>(hopf + op.n_codes);
  int* coff = reinterpret_cast<int*>(hopf + op.n_codes);
  // MULTI: md's fields as values (lambdas then capture no kernel parameter by address)
  const int R = MULTI ? md.n_real : 1;
  const int* const tile_first = md.tile_first;
  const long long tile_sites = md.tile_sites;
  double* const partials = md.partials;
  int* cdelta = coff + (size_t)R * op.n_codes;
  // MULTI: each model's window starts [R][kStageWin], then its window count [R]
  int* rlo = cdelta + op.n_codes;
  const int* rnw = rlo + R * kStageWin;
  __shared__ int abort_flag;  // MULTI: a wait ran out; the block computes no further

  for (int c = threadIdx.x; c < op.n_codes; c += blockDim.x) {
    hop[c] = op.code_hop[c];
    hopf[c] = scaled_hop(op.code_hop[c], op);
    if constexpr (!MULTI) {
      const int d = op.code_delta[c];
      int o = -1;
#pragma unroll
      for (int w = 0; w < kStageWin; ++w)
        if (w < sl.nw && o < 0 && d >= sl.win_lo[w] && d <= sl.win_lo[w] + sl.win_rows[w] - TS)
          o = sl.win_off[w] + (d - sl.win_lo[w]) * RB;
      cinfo[c] = make_int2(o, d);
    }
  }
  if constexpr (MULTI) {
    const int* tab = op.stage_rtab;
    for (int k = threadIdx.x; k < R * (kStageWin + 1); k += blockDim.x)
      rlo[k] = tab[k];
    for (int c = threadIdx.x; c < op.n_codes; c += blockDim.x)
      cdelta[c] = op.code_delta[c];
    const int* slot = tab + R * (kStageWin + 1);
    for (int k = threadIdx.x; k < R * op.n_codes; k += blockDim.x) {
      const int r = k / op.n_codes, d = op.code_delta[k % op.n_codes], w = slot[k];
      // the planner put d inside model r's window w, which its slot is wide enough for
      // (constant indices into sl: a runtime one would copy it to local memory)
      int o = -1;
#pragma unroll
      for (int q = 0; q < kStageWin; ++q)
        if (q == w && q < sl.nw)
          o = sl.win_off[q] + (d - tab[r * kStageWin + q]) * RB;
      coff[k] = o;
    }
  }
  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < S; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, kComputeWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_async_smem();
  }
  __syncthreads();

  const int n = op.n;
  const int G = (int)gridDim.x;
  const int ntiles = (n + TS - 1) / TS;
  const int mine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / G + 1 : 0;
  // the site's own row (offset 0, in window 0)
  const int xofs = sl.win_off[0] - sl.win_lo[0] * RB;
  // MULTI: the model of this block's tile j (tiles come in increasing order)
  int rp = 0;
  auto model_of = [&](int j, int& r) {
    const long long first = (long long)((int)blockIdx.x + j * G) * TS;
    while (r + 1 < R && first >= (long long)tile_first[r + 1] * tile_sites)
      ++r;
  };

  // Thread 0: the copies of this block's tile j into stage j % S.
  auto produce = [&](int j) {
    const int s = j % S;
    unsigned char* st = stage_smem + (size_t)s * sl.stage_bytes;
    const long long first = (long long)((int)blockIdx.x + j * G) * TS;
    const long long last = first + TS < n ? first + TS : n;
    int wlo[kStageWin];  // window starts (MULTI: the tile's model's)
    int nw = sl.nw;
#pragma unroll
    for (int w = 0; w < kStageWin; ++w)
      wlo[w] = sl.win_lo[w];
    if constexpr (MULTI) {
      model_of(j, rp);
      nw = rnw[rp] < sl.nw ? rnw[rp] : sl.nw;
#pragma unroll
      for (int w = 0; w < kStageWin; ++w)
        wlo[w] = rlo[rp * kStageWin + w];
    }
    // window w's rows clamped to the vector: [c0, c1)
    auto clamp = [&](int w, long long& c0, long long& c1) {
      const long long a = first + wlo[w], b = a + sl.win_rows[w];
      c0 = a > 0 ? a : 0;
      c1 = b < n ? b : n;
    };
    unsigned bytes = 0;
#pragma unroll
    for (int w = 0; w < kStageWin; ++w) {
      long long c0, c1;
      clamp(w, c0, c1);
      if (w < nw && c1 > c0)
        bytes += (unsigned)((c1 - c0) * RB);
    }
    const unsigned tile_bytes = (unsigned)((last - first) * RB);
    if constexpr (MODE == kCheb)
      bytes += tile_bytes;
    mbar_arrive_expect(full + s, bytes);
#pragma unroll
    for (int w = 0; w < kStageWin; ++w) {
      long long c0, c1;
      clamp(w, c0, c1);
      if (w < nw && c1 > c0)
        bulk_load(st + sl.win_off[w] + (c0 - (first + wlo[w])) * RB,
                  t1 + (size_t)c0 * V, (unsigned)((c1 - c0) * RB), full + s);
    }
    if constexpr (MODE == kCheb)
      bulk_load(st + sl.t0_off, t0 + (size_t)first * V, tile_bytes, full + s);
  };

  // This thread computes site l of every tile and the vectors of two 16-byte chunks of
  // a row, half a row apart: chunk q and q + V/4. On rows of 8 chunks (V = 16) odd
  // sites take them in the other order, so the 8 threads of a quarter warp (two sites)
  // read 8 distinct chunks: no shared-memory bank conflict. Slot k < 2 holds vector
  // 2 ca + k, slot k >= 2 vector 2 cb + k - 2.
  constexpr int kHalf = V / 4;
  const int l = (int)threadIdx.x / kTps;
  const int q = (int)threadIdx.x % kTps;
  const int sw = (V == 16) ? (l & 1) : 0;
  const int ca = q + sw * kHalf, cb = q + (1 - sw) * kHalf;
  auto widen4 = [&](const float4& a, const float4& b, double2 (&y)[W]) {
    y[0] = make_double2(a.x, a.y);
    y[1] = make_double2(a.z, a.w);
    y[2] = make_double2(b.x, b.y);
    y[3] = make_double2(b.z, b.w);
  };
  auto lds4 = [&](const unsigned char* row, double2 (&y)[W]) {
    widen4(*reinterpret_cast<const float4*>(row + ca * 16),
           *reinterpret_cast<const float4*>(row + cb * 16), y);
  };
  auto split4 = [&](const float4& a, const float4& b, float2 (&y)[W]) {
    y[0] = make_float2(a.x, a.y);
    y[1] = make_float2(a.z, a.w);
    y[2] = make_float2(b.x, b.y);
    y[3] = make_float2(b.z, b.w);
  };
  auto ldsf4 = [&](const unsigned char* row, float2 (&y)[W]) {
    split4(*reinterpret_cast<const float4*>(row + ca * 16),
           *reinterpret_cast<const float4*>(row + cb * 16), y);
  };
  constexpr int kSums = DOT == kDotPair ? 2 * W : W;
  CSum re[kSums], im[kSums];
#pragma unroll
  for (int k = 0; k < kSums; ++k)
    re[k] = im[k] = CSum{0.0, 0.0};

  // codes, potential and (moment <left|T_k>) this thread's left chunks of tile j's
  // site l, loaded one tile ahead into registers: left is read only by the moment, so
  // it takes no shared memory
  // (GQT_FP32R: the potential's FP32 parts pr, made once per operator; GQT_FP32: p)
  auto fetch = [&](int j, int (&c)[Z], double& p, float2& pr, float4& la, float4& lb) {
    const int i = ((int)blockIdx.x + j * G) * TS + l;
    if (i < n) {
#pragma unroll
      for (int m = 0; m < Z; ++m)
        c[m] = op.code[(size_t)m * n + i];
      if constexpr (F32)
        pr = op.pot_r[i];
      else
        p = op.pot[i];
      if constexpr (DOT == kDotLeft && F32) {
        const float4* row = reinterpret_cast<const float4*>(left + (size_t)i * V);
        la = __ldg(row + ca);
        lb = __ldg(row + cb);
      }
    }
  };
  int cc[Z] = {};
  double p = 0.0;
  float2 pr = {};
  float4 la = {}, lb = {};
  // Warps 0 .. kComputeWarps - 1 compute; thread kBlock (the next warp) issues the copies.
  // A compute warp waits for a stage's full barrier and, once its lanes have read the
  // stage, arrives on the stage's empty barrier; the producer refills a stage when all
  // compute warps have arrived. No barrier spans the block inside the loop, and a wait
  // that runs out ends the loop of that warp (uniformly: __any_sync) or of the producer.
  const bool compute = threadIdx.x < kBlock;
  if (threadIdx.x == kBlock) {
    int issued = 0;
    for (int jj = 0; jj < mine; ++jj) {
      const int s = jj % S;
      if (MULTI && *(volatile int*)&abort_flag)
        break;
      if (jj >= S && !mbar_wait(empty + s, (unsigned)(jj / S - 1) & 1u)) {
        atomicOr(op.stage_err, 1u);
        if constexpr (MULTI)
          *(volatile int*)&abort_flag = 1;
        break;
      }
      fence_async_smem();
      produce(jj);
      issued = jj + 1;
    }
    // every copy issued has landed before the block leaves
    for (int jj = issued > S ? issued - S : 0; jj < issued; ++jj)
      mbar_wait(full + jj % S, (unsigned)(jj / S) & 1u);
  }
  // MULTI: the block's sums of model rr, reduced over the compute warps (named barrier 1,
  // the producer warp takes no part), into the block's slot of that model; the sums
  // restart from zero.
  constexpr int kVS = DOT == kDotPair ? 2 * V : V;
  int rc = -1;           // MULTI: the model whose sums the threads hold
  unsigned touched = 0;  // MULTI: the models whose slot this block has written
  auto flush = [&](int rr) {
    if constexpr (MULTI) {
      __shared__ double msh[kComputeWarps][kVS][4];
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      constexpr int P = DOT == kDotPair ? 2 : 1;
      // Two slots at a time, in place (the sums restart from zero afterwards), in the
      // order of even sites (chunk q, then chunk q + V/4): odd sites hold the halves
      // swapped.
      auto put = [&](int k, CSum a, CSum b) {
#pragma unroll
        for (int off = 16; off >= kTps; off >>= 1) {
          csum_merge(a, shfl_xor(a, off));
          csum_merge(b, shfl_xor(b, off));
        }
        if (lane < kTps) {
          const int v = StageSlots<kHalf, P>{}(lane, k, kSums);
          msh[warp][v][0] = a.s;
          msh[warp][v][1] = a.c;
          msh[warp][v][2] = b.s;
          msh[warp][v][3] = b.c;
        }
      };
      constexpr int H = kSums / 2;
#pragma unroll
      for (int k = 0; k < H; ++k) {
        const CSum a0 = re[k], b0 = im[k], a1 = re[k + H], b1 = im[k + H];
        re[k] = im[k] = re[k + H] = im[k + H] = CSum{0.0, 0.0};
        put(k, sw ? a1 : a0, sw ? b1 : b0);
        put(k + H, sw ? a0 : a1, sw ? b0 : b1);
      }
      asm volatile("bar.sync 1, %0;" ::"n"(kBlock) : "memory");
      if (threadIdx.x < kVS) {
        const int v = threadIdx.x;
        CSum x{msh[0][v][0], msh[0][v][1]}, y{msh[0][v][2], msh[0][v][3]};
        for (int w = 1; w < kComputeWarps; ++w) {
          csum_merge(x, CSum{msh[w][v][0], msh[w][v][1]});
          csum_merge(y, CSum{msh[w][v][2], msh[w][v][3]});
        }
        double* dst = partials + (((size_t)blockIdx.x * R + rr) * kVS + v) * 4;
        dst[0] = x.s;
        dst[1] = x.c;
        dst[2] = y.s;
        dst[3] = y.c;
      }
      asm volatile("bar.sync 1, %0;" ::"n"(kBlock) : "memory");
      touched |= 1u << rr;
    }
  };
  if (compute && mine > 0) {
    fetch(0, cc, p, pr, la, lb);
    if constexpr (MULTI) {
      rc = 0;
      model_of(0, rc);
    }
  }
  for (int j = 0; compute && j < mine; ++j) {
    int cn[Z] = {};
    double pn = 0.0;
    float2 prn = {};
    float4 lan = {}, lbn = {};
    if (j + 1 < mine)
      fetch(j + 1, cn, pn, prn, lan, lbn);
    int cbase = 0;     // MULTI: the model's row of the code table
    int own = xofs;    // the site's own row in the stage
    if constexpr (MULTI) {
      cbase = rc * op.n_codes;
      own = sl.win_off[0] - rlo[rc * kStageWin] * RB;
    }
    const int s = j % S;
    bool skip = false;
    if constexpr (MULTI) {
      // After a wait ran out (in any warp) the block skips its remaining tiles but keeps
      // taking part in the flushes, so no named barrier waits for a warp that left.
      const bool stop = *(volatile int*)&abort_flag != 0;
      const bool late = !stop && !mbar_wait(full + s, (unsigned)(j / S) & 1u);
      if (__any_sync(0xffffffffu, late)) {
        if (late)
          atomicOr(op.stage_err, 1u);
        *(volatile int*)&abort_flag = 1;
      }
      skip = __any_sync(0xffffffffu, stop || late);
    } else {
      const bool late = !mbar_wait(full + s, (unsigned)(j / S) & 1u);
      if (__any_sync(0xffffffffu, late)) {
        if (late)
          atomicOr(op.stage_err, 1u);
        break;
      }
    }
    const unsigned char* st = stage_smem + (size_t)s * sl.stage_bytes + l * RB;
    const int i = ((int)blockIdx.x + j * G) * TS + l;
    if (!skip && F32 && i < n) {
      float2 x[W];
      ldsf4(st + own, x);
      const float2 pf = pr;
      AccF32 acc[W];
#pragma unroll
      for (int k = 0; k < W; ++k)
        acc[k] = acc_start(pf, x[k]);
#pragma unroll
      for (int m = 0; m < Z; ++m) {
        const int c = cc[m];
        const int2 ci = MULTI ? make_int2(coff[cbase + c], cdelta[c]) : cinfo[c];
        const float4 h = hopf[c];
        float2 y[W];
        if (ci.x >= 0) {
          ldsf4(st + ci.x, y);
        } else {
          const float4* row = reinterpret_cast<const float4*>(t1 + (size_t)(i + ci.y) * V);
          split4(__ldg(row + ca), __ldg(row + cb), y);
        }
#pragma unroll
        for (int k = 0; k < W; ++k)
          cmac_f32(acc[k], h, y[k]);
      }
      float2 y0[W] = {};
      if constexpr (MODE == kCheb)
        ldsf4(st + sl.t0_off, y0);
      float2 r[W];
#pragma unroll
      for (int k = 0; k < W; ++k)
        r[k] = acc_finish<MODE>(acc[k], y0[k]);
      float4* orow = reinterpret_cast<float4*>(out + (size_t)i * V);
      orow[ca] = make_float4(r[0].x, r[0].y, r[1].x, r[1].y);
      orow[cb] = make_float4(r[2].x, r[2].y, r[3].x, r[3].y);
      if constexpr (DOT == kDotLeft) {
        float2 lf[W];
        split4(la, lb, lf);
#pragma unroll
        for (int k = 0; k < W; ++k) {
          const double rx = r[k].x, ry = r[k].y, lx = lf[k].x, ly = lf[k].y;
          re[k].s = fma(rx, lx, fma(ry, ly, re[k].s));
          im[k].s = fma(ry, lx, fma(-rx, ly, im[k].s));
        }
      } else if constexpr (DOT == kDotPair) {
#pragma unroll
        for (int k = 0; k < W; ++k) {
          const double ox = r[k].x, oy = r[k].y, xx = x[k].x, xy = x[k].y;
          re[2 * k].s = fma(ox, ox, fma(oy, oy, re[2 * k].s));
          re[2 * k + 1].s = fma(ox, xx, fma(oy, xy, re[2 * k + 1].s));
          im[2 * k + 1].s = fma(oy, xx, fma(-ox, xy, im[2 * k + 1].s));
        }
      }
    }
    if (!skip && !F32 && i < n) {
      double2 x[W];
      lds4(st + own, x);
      double tr[W], ti[W];
#pragma unroll
      for (int k = 0; k < W; ++k) {
        tr[k] = A::mul(p, x[k].x);
        ti[k] = A::mul(p, x[k].y);
      }
#pragma unroll
      for (int m = 0; m < Z; ++m) {
        const int c = cc[m];
        const int2 ci = MULTI ? make_int2(coff[cbase + c], cdelta[c]) : cinfo[c];
        const double2 h = hop[c];
        double2 y[W];
        if (ci.x >= 0) {
          lds4(st + ci.x, y);
        } else {
          const float4* row = reinterpret_cast<const float4*>(t1 + (size_t)(i + ci.y) * V);
          widen4(__ldg(row + ca), __ldg(row + cb), y);
        }
#pragma unroll
        for (int k = 0; k < W; ++k) {
          tr[k] = A::add(tr[k], A::cre(h.x, h.y, y[k].x, y[k].y));
          ti[k] = A::add(ti[k], A::cim(h.x, h.y, y[k].x, y[k].y));
        }
      }
      double2 r[W];
      if constexpr (MODE == kCheb) {
        double2 y0[W];
        lds4(st + sl.t0_off, y0);
#pragma unroll
        for (int k = 0; k < W; ++k)
          r[k] = make_double2(A::two_x_minus(A::scale(tr[k], op), y0[k].x),
                              A::two_x_minus(A::scale(ti[k], op), y0[k].y));
      } else {
#pragma unroll
        for (int k = 0; k < W; ++k)
          r[k] = make_double2(A::scale(tr[k], op), A::scale(ti[k], op));
      }
      const float4 oa = make_float4(__double2float_rn(r[0].x), __double2float_rn(r[0].y),
                                    __double2float_rn(r[1].x), __double2float_rn(r[1].y));
      const float4 ob = make_float4(__double2float_rn(r[2].x), __double2float_rn(r[2].y),
                                    __double2float_rn(r[3].x), __double2float_rn(r[3].y));
      float4* orow = reinterpret_cast<float4*>(out + (size_t)i * V);
      orow[ca] = oa;
      orow[cb] = ob;
      if constexpr (DOT == kDotLeft) {
        // (the FP64-arithmetic variant loads left here: held a tile ahead it spilled)
        const float4* lrow = reinterpret_cast<const float4*>(left + (size_t)i * V);
        double2 lf[W];
        widen4(__ldg(lrow + ca), __ldg(lrow + cb), lf);
#pragma unroll
        for (int k = 0; k < W; ++k) {
          re[k].s = fma(r[k].x, lf[k].x, fma(r[k].y, lf[k].y, re[k].s));
          im[k].s = fma(r[k].y, lf[k].x, fma(-r[k].x, lf[k].y, im[k].s));
        }
      } else if constexpr (DOT == kDotPair) {
        // T_k and T_{k-1} as stored
        double2 o[W];
        widen4(oa, ob, o);
#pragma unroll
        for (int k = 0; k < W; ++k) {
          re[2 * k].s = fma(o[k].x, o[k].x, fma(o[k].y, o[k].y, re[2 * k].s));
          re[2 * k + 1].s = fma(o[k].x, x[k].x, fma(o[k].y, x[k].y, re[2 * k + 1].s));
          im[2 * k + 1].s = fma(o[k].y, x[k].x, fma(-o[k].x, x[k].y, im[2 * k + 1].s));
        }
      }
    }
    // this warp has read stage s
    __syncwarp();
    if (!skip && (threadIdx.x & 31) == 0)
      mbar_arrive(empty + s);
#pragma unroll
    for (int m = 0; m < Z; ++m)
      cc[m] = cn[m];
    p = pn;
    pr = prn;
    la = lan;
    lb = lbn;
    if constexpr (MULTI) {
      // The block's sums of model rc end with its last tile there. The next tile's model
      // follows from the tile index alone, so every compute thread flushes in step.
      int rn = rc;
      if (j + 1 < mine)
        model_of(j + 1, rn);
      if (j + 1 == mine || rn != rc)
        flush(rc);
      rc = rn;
    }
  }
  if constexpr (MULTI) {
    if (compute) {
      // slots of models this block never met hold zero sums
      double* slots = partials + (size_t)blockIdx.x * R * kVS * 4;
      for (int k = threadIdx.x; k < R * kVS * 4; k += kBlock)
        if (!((touched >> (k / (kVS * 4))) & 1u))
          slots[k] = 0.0;
    }
  } else {
    // Slots in the order of even sites (chunk q, then chunk q + V/4) on every thread.
    if (sw) {
#pragma unroll
      for (int k = 0; k < kSums / 2; ++k) {
        const CSum a = re[k], b = im[k];
        re[k] = re[k + kSums / 2];
        im[k] = im[k + kSums / 2];
        re[k + kSums / 2] = a;
        im[k + kSums / 2] = b;
      }
    }
    if constexpr (DOT == kDotLeft)
      dot_finish_w<V, W, StageSlots<kHalf, 1>, kComputeWarps>(re, im, dot, {});
    else if constexpr (DOT == kDotPair)
      dot_finish_w<2 * V, 2 * W, StageSlots<kHalf, 2>, kComputeWarps>(re, im, dot, {});
  }
}

// Stage layout for V vectors over the first nw windows: the windows, then T_{k-2} as
// the launch needs it; true when at least two stages of it fit. budget: the shared memory
// the stages may take (two blocks per SM).
bool stage_layout_nw(const Op& op, int V, int mode, int nw, int stages, StageLayout& sl,
                     int budget)
{
  const int TS = kBlock * kStageW / V, RB = V * (int)sizeof(float2);
  sl = StageLayout{};
  sl.nw = nw;
  int off = 0;
  for (int w = 0; w < sl.nw; ++w) {
    sl.win_lo[w] = op.stage_lo[w];
    sl.win_rows[w] = TS + op.stage_hi[w] - op.stage_lo[w];
    sl.win_off[w] = off;
    off += sl.win_rows[w] * RB;
  }
  sl.t0_off = -1;
  if (mode == kCheb) {
    sl.t0_off = off;
    off += TS * RB;
  }
  sl.stage_bytes = (off + 127) / 128 * 128;
  if (stages <= 1) {
    // as many stages as fit the budget, at most kMaxStages
    stages = budget / sl.stage_bytes;
    stages = stages > kMaxStages ? kMaxStages : stages;
  }
  // at most kMaxStages, and no more than fit 200 KB (a block's shared memory is at most
  // 227 KB, the moment sums and the code table take the rest)
  const int fit = (200 << 10) / sl.stage_bytes;
  stages = stages > fit ? fit : stages;
  sl.stages = stages > kMaxStages ? kMaxStages : stages;
  return sl.nw > 0 && sl.stages >= 2;
}

// The windows come most used first (after the one holding offset 0); when two stages of
// all of them do not fit, the last ones are left out (their entries gather from global
// memory) until two do.
bool stage_layout(const Op& op, int V, int mode, int dot, int stages, StageLayout& sl,
                  int budget = 104 << 10)
{
  (void)dot;  // left never takes shared memory: both moment modes share the layout
  for (int nw = op.stage_nw; nw >= 1; --nw)
    if (stage_layout_nw(op, V, mode, nw, stages, sl, budget))
      return true;
  return false;
}

// Dynamic shared memory of a launch beside its stages: the barriers, the hopping table in
// FP64 and FP32 parts and the code offsets (R > 1, a realisation batch of R models: per
// model and code, with the offsets j - i per code and each model's window starts).
size_t stage_table_bytes(const Op& op, int R)
{
  const size_t base = 2 * kMaxStages * sizeof(uint64_t) +
                      (size_t)op.n_codes * (sizeof(double2) + sizeof(float4));
  if (R <= 1)
    return base + (size_t)op.n_codes * sizeof(int2);
  return base + ((size_t)R * op.n_codes + op.n_codes + (size_t)R * (kStageWin + 1)) * sizeof(int);
}

// The stages' share of a realisation-batch launch: the one-model budget less what the
// batch adds, the per-model tables and the block reduction of a model's sums (static,
// kComputeWarps x the model's sums x 32 B). On the 8-model benchmark batch that leaves
// two stages. Three fit two blocks per SM too (112 KB each), but measured on B200 they
// ran the symmetric loop at 1.99e11 site-moments/s against 2.49e11 with two, and the
// direct loop at the same rate.
int multi_stage_budget(const Op& op, int R, int V, int dot)
{
  const int kVS = dot == kDotPair ? 2 * V : V;
  const int added = (int)stage_table_bytes(op, R) - (int)stage_table_bytes(op, 1);
  return (104 << 10) - added - kComputeWarps * kVS * 4 * (int)sizeof(double);
}

template <int V, int Z, int MODE, int DOT, bool F32, bool MULTI>
gqt_status launch_staged(const Op& op, const StageLayout& sl, const float2* t0,
                         const float2* t1, float2* out, const float2* left, const Dot& d,
                         MultiDot md)
{
  auto* kernel = k_step_staged<V, Z, MODE, DOT, F32, MULTI>;
  const int R = MULTI ? md.n_real : 1;
  const size_t smem = (size_t)sl.stages * sl.stage_bytes + stage_table_bytes(op, R);
  static std::mutex mu;
  static std::unordered_map<size_t, int> per_sm;  // blocks per SM by shared memory size
  static size_t attr = 0;                         // the kernel's shared memory limit set
  int bps;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (smem > attr) {
      GQT_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
      attr = smem;
    }
    auto it = per_sm.find(smem);
    if (it == per_sm.end()) {
      int b = 0;
      GQT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kStageThreads, smem));
      it = per_sm.emplace(smem, b > 0 ? b : 1).first;
    }
    bps = it->second;
  }
  const int TS = kBlock * kStageW / V;
  const int ntiles = (op.n + TS - 1) / TS;
  const int cap = device_info().sms * bps;
  const int grid = ntiles < cap ? ntiles : cap;
  if (MULTI) {
    if (grid > max_grid())
      return fail(GQT_ERR_STATE, "staged batch step: grid %d above the slot rows", grid);
    md.blocks = grid;
    if (md.blocks_out)
      *md.blocks_out = grid;
  }
  kernel<<<grid, kStageThreads, smem, stream()>>>(op, sl, t0, t1, out, left, d, md);
  count_launches(1);
  GQT_CUDA(cudaGetLastError());
  return GQT_OK;
}

template <int V, bool F32, bool MULTI = false>
gqt_status staged_v(const Op& op, int mode, int dot, const StageLayout& sl, const void* t0,
                    const void* t1, void* out, const void* left, const Dot& d,
                    const MultiDot& md = MultiDot{})
{
  const float2* a0 = (const float2*)t0;
  const float2* a1 = (const float2*)t1;
  float2* o = (float2*)out;
  const float2* lf = (const float2*)left;
  auto go = [&](auto zc) -> gqt_status {
    constexpr int Z = decltype(zc)::value;
    if (dot == kDotPair) {
      if constexpr (V <= 16) {
        if (mode == kApply)
          return launch_staged<V, Z, kApply, kDotPair, F32, MULTI>(op, sl, a0, a1, o, lf, d,
                                                                   md);
        return launch_staged<V, Z, kCheb, kDotPair, F32, MULTI>(op, sl, a0, a1, o, lf, d, md);
      } else {
        return fail(GQT_ERR_ARG, "symmetric moments: at most 16 vectors per launch");
      }
    }
    if (mode == kApply)
      return launch_staged<V, Z, kApply, kDotLeft, F32, MULTI>(op, sl, a0, a1, o, lf, d, md);
    return launch_staged<V, Z, kCheb, kDotLeft, F32, MULTI>(op, sl, a0, a1, o, lf, d, md);
  };
  switch (op.z) {
    case 3:
      return go(std::integral_constant<int, 3>{});
    case 4:
      return go(std::integral_constant<int, 4>{});
    default:
      return go(std::integral_constant<int, 6>{});
  }
}

}  // namespace

// Whether the staged step serves a step of this operator, vector count and mode, and
// its layout (the vectors' alignment aside). R > 1: a realisation batch of R models
// (the GQT_FP32R step only).
static bool stage_fits(const Op& op, int nvec, int mode, int dot, bool f32, StageLayout& sl,
                       int R = 1)
{
  if (op.stage_nw <= 0 || !op.code || !op.stage_err || (mode != kApply && mode != kCheb))
    return false;
  if ((op.stage_rtab != nullptr) != (R > 1) || (R > 1 && !f32))
    return false;
  // Automatic (0), from B200 measurements with 16 vectors on graphene 2,097,152 sites
  // (rows of 3), square 1024^2 (rows of 4) and cubic 256^3 (rows of 6): the GQT_FP32R
  // steps are always staged (their unstaged step ran 20-60 % slower); the GQT_FP32
  // steps on rows of 6 only (direct 11 %, pair 11 % faster there; on rows of 3 and 4
  // the unstaged steps, at 32 warps per SM, were as fast or 10-15 % faster).
  if (op.stage_stages < 0)
    return false;
  if (op.stage_stages == 0 && !f32 && op.z < 6)
    return false;
  if (nvec != 16 && nvec != 32)
    return false;
  if (dot != kDotLeft && dot != kDotPair)
    return false;
  if (dot == kDotPair && nvec > 16)
    return false;
  if (op.z != 3 && op.z != 4 && op.z != 6)
    return false;
  const int budget = R > 1 ? multi_stage_budget(op, R, nvec, dot) : (104 << 10);
  return budget > 0 && stage_layout(op, nvec, mode, dot, op.stage_stages, sl, budget);
}

bool stage_applies(const Op& op, int nvec, int mode, int dot, const void* t0, const void* t1,
                   const void* left, bool f32)
{
  // bulk copies start on 16-byte boundaries (rows are nvec * 8 >= 32 bytes)
  auto aligned = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
  if (!aligned(t1) || (mode == kCheb && !aligned(t0)) || (dot == kDotLeft && !aligned(left)))
    return false;
  StageLayout sl;
  return stage_fits(op, nvec, mode, dot, f32, sl);
}

int stage_plan(const Op& op, int nvec, int dot, bool f32, int* windows, int R)
{
  StageLayout sl;
  const bool on = stage_fits(op, nvec, kCheb, dot, f32, sl, R);
  if (windows)
    *windows = on ? sl.nw : 0;
  return on ? sl.stages : 0;
}

gqt_status stage_step(const Op& op, int nvec, int mode, int dot, const void* t0,
                      const void* t1, void* out, const void* left, const Dot& d, bool f32)
{
  StageLayout sl;
  if (!stage_layout(op, nvec, mode, dot, op.stage_stages, sl))
    return fail(GQT_ERR_STATE, "staged step: no stage layout for %d vectors", nvec);
  switch (nvec) {
    case 16:
      return f32 ? staged_v<16, true>(op, mode, dot, sl, t0, t1, out, left, d)
                 : staged_v<16, false>(op, mode, dot, sl, t0, t1, out, left, d);
    case 32:
      return f32 ? staged_v<32, true>(op, mode, dot, sl, t0, t1, out, left, d)
                 : staged_v<32, false>(op, mode, dot, sl, t0, t1, out, left, d);
    default:
      return fail(GQT_ERR_ARG, "staged step: unsupported vector count %d", nvec);
  }
}

// The GQT_FP32R step of a realisation batch (mode kApply or kCheb): the staged step with
// each model's windows, its sums per (block, model) in md's slots, combined by
// k_tile_reduce here unless md.defer (then by the caller, over a window of steps).
gqt_status stage_step_multi(const Op& op, int nvec, int mode, int dot, const void* t0,
                            const void* t1, void* out, const void* left, const MultiDot& md)
{
  auto aligned = [](const void* p) { return ((uintptr_t)p & 15u) == 0; };
  StageLayout sl;
  if (!aligned(t1) || !aligned(out) || (mode == kCheb && !aligned(t0)) ||
      (dot == kDotLeft && !aligned(left)) ||
      !stage_fits(op, nvec, mode, dot, true, sl, md.n_real))
    return fail(GQT_ERR_STATE,
                "the FP32R form runs a realisation batch through its staged step only "
                "(coded operator, rows of 3, 4 or 6, 16 or 32 vectors, 16 for symmetric "
                "sets, staging not off); %d vectors here", nvec);
  MultiDot m = md;
  int grid = 0;
  m.blocks_out = &grid;
  const Dot none{};
  gqt_status st = GQT_OK;
  if (nvec == 16)
    st = staged_v<16, true, true>(op, mode, dot, sl, t0, t1, out, left, none, m);
  else
    st = staged_v<32, true, true>(op, mode, dot, sl, t0, t1, out, left, none, m);
  if (st != GQT_OK)
    return st;
  if (md.blocks_out)
    *md.blocks_out = grid;
  if (md.defer)
    return GQT_OK;
  m.blocks = grid;
  return forms_fp32(nvec)->fmt[1].tile_reduce(m, dot == kDotPair, 1, 0);
}


// ------------------------------------------------------------------ the GQT_FP32R form
namespace {

// The potential divided by E_max as FP32 (hi, lo) parts, as the steps used to form it
// per element: split_f32(pot * RN(1 / E_max)).
__global__ void __launch_bounds__(kBlock) k_split_pot(const double* __restrict__ pot,
                                                      double inv_emax, float2* out, int n)
{
  for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock)
    out[i] = split_f32(pot[i] * inv_emax);
}

}  // namespace

gqt_status ensure_pot_r(const gqt_ham* h)
{
  if (h->pot_r)
    return GQT_OK;
  GQT_CUDA(cudaMalloc(&h->pot_r, (size_t)h->n * sizeof(float2)));
  const int grid = (h->n + kBlock - 1) / kBlock < max_grid() ? (h->n + kBlock - 1) / kBlock
                                                             : max_grid();
  k_split_pot<<<grid, kBlock, 0, stream()>>>(h->pot, 1.0 / h->energy_max, h->pot_r, h->n);
  count_launches(1);
  GQT_CUDA(cudaGetLastError());
  return GQT_OK;
}

namespace {

// The GQT_FP32R step without staging (the ELL arrays, operators without windows, vectors
// not on 16-byte boundaries): grid-stride items of one site and 4 consecutive vectors,
// with the staged step's arithmetic (entries past a row's length are skipped).
// three blocks per SM (85 registers) on rows of known length; two on rows of unknown
// length, which spilled at three
template <int Z>
constexpr int r_min_blocks()
{
  return Z > 0 ? 3 : 2;
}

template <int V, int Z, int MODE, int DOT, bool C>
__global__ void __launch_bounds__(kBlock, r_min_blocks<Z>()) k_step_r(Op op, const float2* t0,
                                                   const float2* __restrict__ t1, float2* out,
                                                   const float2* __restrict__ left, Dot dot)
{
  constexpr int W = 4;
  constexpr int kTps = V / W;
  const Tables tb = load_tables<C>(op);
  auto ld4 = [](const float2* p, float2 (&y)[W]) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    const float4 b = *reinterpret_cast<const float4*>(p + 2);
    y[0] = make_float2(a.x, a.y);
    y[1] = make_float2(a.z, a.w);
    y[2] = make_float2(b.x, b.y);
    y[3] = make_float2(b.z, b.w);
  };
  constexpr int kSums = DOT == kDotPair ? 2 * W : W;
  CSum re[kSums], im[kSums];
#pragma unroll
  for (int k = 0; k < kSums; ++k)
    re[k] = im[k] = CSum{0.0, 0.0};
  const size_t items = (size_t)op.n * kTps;
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < items;
       g += (size_t)gridDim.x * kBlock) {
    const int i = (int)(g / kTps);
    const size_t base = (size_t)i * V + (size_t)(g % kTps) * W;
    float2 x[W];
    ld4(t1 + base, x);
    const float2 pf = op.pot_r[i];
    AccF32 acc[W];
#pragma unroll
    for (int k = 0; k < W; ++k)
      acc[k] = acc_start(pf, x[k]);
    const int cnt = op.uniform ? (Z > 0 ? Z : op.z) : op.nn[i];
    for_entries<Z>(cnt, [&](int m) {
      int j, c;
      double2 h;
      ell_entry<C>(op, tb, (size_t)m * op.n + i, i, j, h, c);
      const float4 hf = scaled_hop(h, op);
      float2 y[W];
      ld4(t1 + (size_t)j * V + (base - (size_t)i * V), y);
#pragma unroll
      for (int k = 0; k < W; ++k)
        cmac_f32(acc[k], hf, y[k]);
    });
    float2 y0[W] = {};
    if constexpr (MODE == kCheb)
      ld4(t0 + base, y0);
    float2 r[W];
#pragma unroll
    for (int k = 0; k < W; ++k)
      r[k] = acc_finish<MODE>(acc[k], y0[k]);
    reinterpret_cast<float4*>(out + base)[0] = make_float4(r[0].x, r[0].y, r[1].x, r[1].y);
    reinterpret_cast<float4*>(out + base)[1] = make_float4(r[2].x, r[2].y, r[3].x, r[3].y);
    if constexpr (DOT == kDotLeft) {
      float2 lf[W];
      ld4(left + base, lf);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const double rx = r[k].x, ry = r[k].y, lx = lf[k].x, ly = lf[k].y;
        re[k].s = fma(rx, lx, fma(ry, ly, re[k].s));
        im[k].s = fma(ry, lx, fma(-rx, ly, im[k].s));
      }
    } else {
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const double ox = r[k].x, oy = r[k].y, xx = x[k].x, xy = x[k].y;
        re[2 * k].s = fma(ox, ox, fma(oy, oy, re[2 * k].s));
        re[2 * k + 1].s = fma(ox, xx, fma(oy, xy, re[2 * k + 1].s));
        im[2 * k + 1].s = fma(oy, xx, fma(-ox, xy, im[2 * k + 1].s));
      }
    }
  }
  if constexpr (DOT == kDotLeft)
    dot_finish_w<V, W>(re, im, dot);
  else
    dot_finish_w<2 * V, 2 * W>(re, im, dot);
}

template <int V, int DOT, bool C>
gqt_status run_r(const Op& op, int mode, const void* t0, const void* t1, void* out,
                 const void* left, const Dot& d)
{
  if (C && stage_applies(op, V, mode, DOT, t0, t1, left, true))
    return stage_step(op, V, mode, DOT, t0, t1, out, left, d, true);
  const float2* a0 = (const float2*)t0;
  const float2* a1 = (const float2*)t1;
  float2* o = (float2*)out;
  const float2* lf = (const float2*)left;
  const size_t items = (size_t)op.n * (V / 4);
  return with_z(op.z, [&](auto zc) -> gqt_status {
    constexpr int Z = decltype(zc)::value;
    if (mode == kApply)
      return launch_op(k_step_r<V, Z, kApply, DOT, C>, items, op, a0, a1, o, lf, d);
    return launch_op(k_step_r<V, Z, kCheb, DOT, C>, items, op, a0, a1, o, lf, d);
  });
}

template <int V, bool C>
gqt_status step_r(const Op& op, int mode, const void* t0, const void* t1, void* out,
                  const void* left, const Dot* dot)
{
  if (!dot)
    return fail(GQT_ERR_ARG, "the FP32R form runs moment loops only");
  return run_r<V, kDotLeft, C>(op, mode, t0, t1, out, left, *dot);
}

template <int V, bool C>
gqt_status step_pair_r(const Op& op, int mode, const void* t0, const void* t1, void* out,
                       const Dot& d)
{
  if constexpr (V > 16)
    return fail(GQT_ERR_ARG, "symmetric moments: at most 16 vectors per launch (got %d)", V);
  else
    return run_r<V, kDotPair, C>(op, mode, t0, t1, out, nullptr, d);
}

// A step of a realisation batch: moment 0 (<left|right> of the stored vectors, the same
// sums in every FP32 form) through the FP32 form's batch kernel, the others staged.
template <int V, bool C>
gqt_status step_multi_r(const Op& op, int mode, const void* t0, const void* t1, void* out,
                        const void* left, const MultiDot& md, int dot)
{
  if (mode == kDotOnly)
    return forms_fp32(V)->fmt[C ? 1 : 0].step_multi(op, mode, t0, t1, out, left, md, dot);
  if (!C)
    return fail(GQT_ERR_STATE, "the FP32R form runs a realisation batch on the coded "
                               "operator only");
  return stage_step_multi(op, V, mode, dot, t0, t1, out, left, md);
}

template <int V>
gqt_status tile_reduce_r(const MultiDot& md, bool pair, int rows, size_t row_stride)
{
  return forms_fp32(V)->fmt[1].tile_reduce(md, pair, rows, row_stride);
}

template <int V>
gqt_status dot_r(size_t total, const void* state, const void* left, const Dot& d)
{
  return launch(k_dot<float2, V>, total, total, (const float2*)state, (const float2*)left, d);
}

template <int V>
const FormOps* table_r()
{
  static const FormOps t = [] {
    FormOps f{};
    f.precision = GQT_FP32R;
    f.nvec = V;
    f.elem_bytes = sizeof(float2);
    f.fmt[0].step = step_r<V, false>;
    f.fmt[0].step_pair = step_pair_r<V, false>;
    f.fmt[0].step_multi = step_multi_r<V, false>;
    f.fmt[0].tile_reduce = tile_reduce_r<V>;
    f.fmt[1].step = step_r<V, true>;
    f.fmt[1].step_pair = step_pair_r<V, true>;
    f.fmt[1].step_multi = step_multi_r<V, true>;
    f.fmt[1].tile_reduce = tile_reduce_r<V>;
    f.dot = dot_r<V>;
    return f;
  }();
  return &t;
}

}  // namespace

const FormOps* forms_fp32r(int nvec)
{
  switch (nvec) {
    case 4:
      return table_r<4>();
    case 16:
      return table_r<16>();
    case 32:
      return table_r<32>();
    default:
      return nullptr;
  }
}

}  // namespace gqt
