// Device kernels of the LSQT hot path (sm_100a).
//
// Every kernel is HBM-bound ELL work: a site reads its row of the column-major ELL
// arrays (coalesced across a warp), gathers its neighbours' vector values (served
// mostly from L1/L2 because lattice neighbours are close in index) and streams its
// own vector entries. Vectors are interleaved complex ([site][vector] double2 or
// float2), so a gather is one 8- or 16-byte load and V vectors of one site share
// one ELL row read.
//
// Two arithmetic policies:
//   ExactArith  FP64 with every product, sum and the division by E_max rounded
//               separately (no FMA contraction), in the order of the reference's
//               CPU twins (src/hamiltonian.cu:188-221 etc.): per-site results are
//               bit-identical to the reference.
//   FastArith   FP64 with FMA for the FP32-storage form: inputs are widened to FP64,
//               the operator stays FP64, and only the stored vector is rounded.
//
// Moments <left|T_m> are fused into the step that produces T_m: each thread keeps
// compensated (TwoSum) FP64 partial sums, a block combines them with warp shuffles
// and shared memory, and the last block to finish (arrival counter) combines the
// block partials in fixed block order. The result does not depend on timing.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

namespace gqt {

constexpr int kBlock = 256;
// Windows of T_{k-1} rows the staged step (gqt_stage.cu) copies into shared memory per tile.
constexpr int kStageWin = 8;

struct Op {
  int n;
  int z;
  int uniform;
  const int* __restrict__ nn;
  const int* __restrict__ nl;
  const double2* __restrict__ hop;
  const double* __restrict__ pot;
  const float2* __restrict__ pot_r;  // the FP32R form's split potential (gqt_ham::pot_r)
  const double* __restrict__ xx;
  double emax;
  double inv_emax;  // RN(1 / emax)
  int lib_div;      // 1: emax outside [2^-100, 2^100], divide with __ddiv_rn
  int wpt;  // vectors per thread chosen for this launch (0: the form's default)
  // Coded operator (null code: read the ELL arrays above): entry e is row code[e] of
  // the table, giving j - i, the hopping and xx.
  const uint8_t* __restrict__ code;
  const int* __restrict__ code_delta;
  const double2* __restrict__ code_hop;
  const double* __restrict__ code_xx;
  int n_codes;
  uintptr_t xlo;  // FP32X storage: residual of the element at p is at xlo + p / 2
  // Staged step of the FP32 moment loops over the coded operator (0 windows: not
  // staged): window w covers the neighbour offsets j - i in [stage_lo[w], stage_hi[w]],
  // window 0 holds offset 0; a wait that runs out sets *stage_err.
  int stage_nw;
  int stage_stages;  // -1 off; 0 automatic; 1 as many stages as fit; 2..4 stages
  int stage_lo[kStageWin];
  int stage_hi[kStageWin];
  unsigned* stage_err;
  // Realisation batches (null for one model): gqt_ham::stage_rtab; the slots are then
  // stage_lo[w] = 0, stage_hi[w] = the slot's width.
  const int* __restrict__ stage_rtab;
};

struct Dot {
  double* partials;  // [gridDim.x][V][4]
  unsigned* counter; // [0] arrival counter, [1] grid of the deferred launches
  double2* mu;       // this moment's V results
  // 1: the block writes its partials and leaves; k_slab_combine combines them later
  // in the same order (block 0 records gridDim.x in counter[1]).
  int defer;
  uintptr_t xlo;  // FP32X storage of the vectors read (as Op::xlo)
};

// ------------------------------------------------------------------ operator entries
// The coded operator's table, staged in dynamic shared memory at kernel start
// (n_codes * 28 bytes, passed at launch as op_smem_bytes). Every kernel that reads the
// operator is compiled once per format: C = true reads the codes and the table, C =
// false the ELL arrays.
struct Tables {
  const int* delta;
  const double2* hop;
  const double* xx;
};

inline size_t op_smem_bytes(const Op& op) { return op.code ? (size_t)op.n_codes * 28 : 0; }

template <bool C>
__device__ __forceinline__ Tables load_tables(const Op& op)
{
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  if constexpr (!C)
    return Tables{nullptr, nullptr, nullptr};
  const int n = op.n_codes;
  double2* hop = reinterpret_cast<double2*>(dyn_smem);
  double* xx = reinterpret_cast<double*>(dyn_smem + (size_t)n * 16);
  int* delta = reinterpret_cast<int*>(dyn_smem + (size_t)n * 24);
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    hop[k] = op.code_hop[k];
    xx[k] = op.code_xx[k];
    delta[k] = op.code_delta[k];
  }
  __syncthreads();
  return Tables{delta, hop, xx};
}

// Programmatic dependent launch: a step launched with the programmatic-serialisation
// attribute may start while the previous kernel in its stream finishes. Before
// pdl_wait it touches only what no kernel writes (the operator and its table); after
// it, the previous grid has completed and its writes are visible. Each block calls
// pdl_trigger once its main loop is done, so the next step's blocks can be scheduled
// onto the SMs this grid frees while its last block combines the moment. Both are
// no-ops in a launch without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger()
{
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Entry e = m * n + i of row i: neighbour j, hopping h, and the table row c (coded
// form only) for ell_xx.
template <bool C>
__device__ __forceinline__ void ell_entry(const Op& op, const Tables& tb, size_t e, int i,
                                          int& j, double2& h, int& c)
{
  if constexpr (C) {
    c = op.code[e];
    j = i + tb.delta[c];
    h = tb.hop[c];
  } else {
    c = 0;
    j = op.nl[e];
    h = op.hop[e];
  }
}

template <bool C>
__device__ __forceinline__ double ell_xx(const Op& op, const Tables& tb, size_t e, int c)
{
  if constexpr (C)
    return tb.xx[c];
  else
    return op.xx[e];
}

// ------------------------------------------------------------------ arithmetic
struct ExactArith {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  // a / E_max correctly rounded, from fused multiply-adds (Markstein's theorem:
  // P. W. Markstein, IBM J. Res. Dev. 34(1), 1990; Muller et al., Handbook of
  // Floating-Point Arithmetic, FMA-based division). With y = RN(1/E) (op.inv_emax, an
  // IEEE division on the host) and q within one ulp of a/E, r = a - qE is exact and
  // RN(q + r y) = RN(a/E). q0 = RN(a y) is within 1.5 ulp; one correction makes it
  // faithful, the second rounds correctly. The exact remainders need |a| and E well
  // inside the normal range: zero, tiny, huge or non-finite a, and an E outside
  // [2^-100, 2^100] (op.lib_div), take the library division.
  static __device__ __forceinline__ double scale(double a, const Op& op)
  {
    const double m = fabs(a);
    if (!(m >= 0x1p-900 && m <= 0x1p900) || op.lib_div)
      return __ddiv_rn(a, op.emax);
    const double b = op.emax, y = op.inv_emax;
    double q = __dmul_rn(a, y);
    double r = __fma_rn(-q, b, a);
    q = __fma_rn(r, y, q);
    r = __fma_rn(-q, b, a);
    return __fma_rn(r, y, q);
  }
  // a*c - b*d and a*d + b*c, each product and sum rounded on its own
  static __device__ __forceinline__ double cre(double a, double b, double c, double d)
  {
    return __dsub_rn(__dmul_rn(a, c), __dmul_rn(b, d));
  }
  static __device__ __forceinline__ double cim(double a, double b, double c, double d)
  {
    return __dadd_rn(__dmul_rn(a, d), __dmul_rn(b, c));
  }
  static __device__ __forceinline__ double two_x_minus(double x, double y)
  {
    return __dsub_rn(__dmul_rn(2.0, x), y);
  }
};

struct FastArith {
  static __device__ __forceinline__ double mul(double a, double b) { return a * b; }
  static __device__ __forceinline__ double add(double a, double b) { return a + b; }
  static __device__ __forceinline__ double sub(double a, double b) { return a - b; }
  static __device__ __forceinline__ double scale(double a, const Op& op)
  {
    return a * op.inv_emax;
  }
  static __device__ __forceinline__ double cre(double a, double b, double c, double d)
  {
    return fma(a, c, -b * d);
  }
  static __device__ __forceinline__ double cim(double a, double b, double c, double d)
  {
    return fma(a, d, b * c);
  }
  static __device__ __forceinline__ double two_x_minus(double x, double y)
  {
    return fma(2.0, x, -y);
  }
};

// ------------------------------------------------------------------ storage
// Every load and store takes `xlo`, which only the FP32X form (below) reads.
__device__ __forceinline__ double2 ld(const double2* p, uintptr_t = 0) { return *p; }
__device__ __forceinline__ double2 ld(const float2* p, uintptr_t = 0)
{
  float2 f = *p;
  return make_double2((double)f.x, (double)f.y);
}
__device__ __forceinline__ void st(double2* p, double2 v, uintptr_t = 0) { *p = v; }
__device__ __forceinline__ void st(float2* p, double2 v, uintptr_t = 0)
{
  *p = make_float2(__double2float_rn(v.x), __double2float_rn(v.y));
}
// The value a store of v leaves in memory, widened back to FP64.
__device__ __forceinline__ double2 stored(const double2*, double2 v) { return v; }
__device__ __forceinline__ double2 stored(const float2*, double2 v)
{
  return make_double2((double)__double2float_rn(v.x), (double)__double2float_rn(v.y));
}

// FP32X storage (the moment recurrence of the GQT_FP32X form): an element v is kept as
// hi = RN_fp32(v) and lo = RN_bf16(v - hi), 12 bytes per complex element instead of
// FP64's 16, with about 32 significant bits. hi is an xf2 at address p; its residual,
// a bf16 pair, lies at xlo + p / 2: the vectors of a moment loop are carved from one
// workspace arena whose residual region is the FP32 region's image under that map, so
// the residuals of consecutive elements are consecutive 4-byte words and W elements'
// residuals are one 4W-byte load.
struct __align__(8) xf2 {
  float x, y;
};
__device__ __forceinline__ const __nv_bfloat162* xres(const xf2* p, uintptr_t xlo)
{
  return reinterpret_cast<const __nv_bfloat162*>(xlo + reinterpret_cast<uintptr_t>(p) / 2);
}
__device__ __forceinline__ __nv_bfloat162* xres(xf2* p, uintptr_t xlo)
{
  return reinterpret_cast<__nv_bfloat162*>(xlo + reinterpret_cast<uintptr_t>(p) / 2);
}
__device__ __forceinline__ double2 xjoin(float hx, float hy, __nv_bfloat162 l)
{
  const float2 lf = __bfloat1622float2(l);
  return make_double2((double)hx + (double)lf.x, (double)hy + (double)lf.y);
}
// hi and the rounded residual of v
__device__ __forceinline__ void xsplit(double2 v, float2& h, __nv_bfloat162& l)
{
  h = make_float2(__double2float_rn(v.x), __double2float_rn(v.y));
  l = __floats2bfloat162_rn(__double2float_rn(v.x - (double)h.x),
                            __double2float_rn(v.y - (double)h.y));
}
__device__ __forceinline__ double2 ld(const xf2* p, uintptr_t xlo)
{
  const xf2 h = *p;
  return xjoin(h.x, h.y, *xres(p, xlo));
}
__device__ __forceinline__ void st(xf2* p, double2 v, uintptr_t xlo)
{
  float2 h;
  __nv_bfloat162 l;
  xsplit(v, h, l);
  *reinterpret_cast<float2*>(p) = h;
  *xres(p, xlo) = l;
}
__device__ __forceinline__ double2 stored(const xf2*, double2 v)
{
  float2 h;
  __nv_bfloat162 l;
  xsplit(v, h, l);
  return xjoin(h.x, h.y, l);
}

// ------------------------------------------------------------------ compensated sums
struct CSum {
  double s, c;
};

__device__ __forceinline__ void csum_add(CSum& a, double x)
{
  double t = __dadd_rn(a.s, x);
  double z = __dsub_rn(t, a.s);
  double e = __dadd_rn(__dsub_rn(a.s, __dsub_rn(t, z)), __dsub_rn(x, z));
  a.s = t;
  a.c = __dadd_rn(a.c, e);
}

__device__ __forceinline__ void csum_merge(CSum& a, const CSum& b)
{
  double t = __dadd_rn(a.s, b.s);
  double z = __dsub_rn(t, a.s);
  double e = __dadd_rn(__dsub_rn(a.s, __dsub_rn(t, z)), __dsub_rn(b.s, z));
  a.s = t;
  a.c = __dadd_rn(__dadd_rn(a.c, b.c), e);
}

// <left|state> term of one element, in the reference's form (src/vector.cu:300-329):
// re = a*c + b*d, im = b*c - a*d with (a, b) = state and (c, d) = left.
__device__ __forceinline__ void dot_term(CSum& re, CSum& im, double2 s, double2 l)
{
  csum_add(re, __dadd_rn(__dmul_rn(s.x, l.x), __dmul_rn(s.y, l.y)));
  csum_add(im, __dsub_rn(__dmul_rn(s.y, l.x), __dmul_rn(s.x, l.y)));
}

// The real part of dot_term(re, im, s, s): the imaginary part b*a - a*b of a product
// of a value with itself is exactly zero, and adding zero leaves a compensated sum
// unchanged bit for bit, so the pair mode's <T_k|T_k> keeps only its real sum.
__device__ __forceinline__ void dot_term_self(CSum& re, double2 s)
{
  csum_add(re, __dadd_rn(__dmul_rn(s.x, s.x), __dmul_rn(s.y, s.y)));
}

__device__ __forceinline__ CSum shfl_xor(const CSum& a, int off)
{
  CSum b;
  b.s = __shfl_xor_sync(0xffffffffu, a.s, off);
  b.c = __shfl_xor_sync(0xffffffffu, a.c, off);
  return b;
}

// The grid stage of a moment: one block combines the partials of nblocks blocks
// ([block][V][4]) in fixed block order and writes mu[v] for v < V. Thread t sums
// blocks t/V, t/V + kBlock/V, ... of vector t % V; lanes and warps then merge in a
// fixed pattern, so the result depends only on nblocks and the partials. Must be
// reached by every thread of the block.
template <int V>
__device__ __forceinline__ void grid_combine(const double* partials, int nblocks, double2* mu,
                                             double (&sh)[kBlock / 32][V][4])
{
  constexpr int kWarps = kBlock / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int v = threadIdx.x % V;
  constexpr int kStride = kBlock / V;
  CSum r{0.0, 0.0}, i{0.0, 0.0};
  // threads past kBlock (a block with a producer warp) take no part
  int b = threadIdx.x < kBlock ? (int)threadIdx.x / V : nblocks;
  // Four blocks' partials are loaded before they are merged (in block order), so the
  // L2 round trips overlap.
  for (; b + 3 * kStride < nblocks; b += 4 * kStride) {
    double q[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double* p = partials + ((size_t)(b + u * kStride) * V + v) * 4;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        q[u][k] = __ldcg(p + k);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      csum_merge(r, CSum{q[u][0], q[u][1]});
      csum_merge(i, CSum{q[u][2], q[u][3]});
    }
  }
  for (; b < nblocks; b += kStride) {
    const double* p = partials + ((size_t)b * V + v) * 4;
    csum_merge(r, CSum{__ldcg(p + 0), __ldcg(p + 1)});
    csum_merge(i, CSum{__ldcg(p + 2), __ldcg(p + 3)});
  }
#pragma unroll
  for (int off = 16; off >= V; off >>= 1) {
    csum_merge(r, shfl_xor(r, off));
    csum_merge(i, shfl_xor(i, off));
  }
  __syncthreads();
  if (lane < V && warp < kWarps) {
    sh[warp][lane][0] = r.s;
    sh[warp][lane][1] = r.c;
    sh[warp][lane][2] = i.s;
    sh[warp][lane][3] = i.c;
  }
  __syncthreads();
  if (threadIdx.x < V) {
    CSum rr{sh[0][v][0], sh[0][v][1]}, ii{sh[0][v][2], sh[0][v][3]};
    for (int w = 1; w < kWarps; ++w) {
      csum_merge(rr, CSum{sh[w][v][0], sh[w][v][1]});
      csum_merge(ii, CSum{sh[w][v][2], sh[w][v][3]});
    }
    mu[v] = make_double2(__dadd_rn(rr.s, rr.c), __dadd_rn(ii.s, ii.c));
  }
}

// Vector of slot k of the threads with lane % (V / W) == q: the W consecutive vectors
// q W .. q W + W - 1.
struct ContigSlots {
  __device__ __forceinline__ int operator()(int q, int k, int w) const { return q * w + k; }
};

// Combine per-thread partials across the block, then across the grid (last block,
// fixed order, or k_slab_combine later when dot.defer is set), and write dot.mu[v] for
// v < V. Slot k of a thread holds the sums of vector map(q, k, W), q = lane % (V/W)
// (by default W consecutive vectors from q W). Must be reached by every thread of the
// block.
// Only the first NW warps hold sums (a block may have more warps, which take no part).
template <int V, int W, class Map = ContigSlots, int NW = kBlock / 32>
__device__ __forceinline__ void dot_finish_w(CSum (&re)[W], CSum (&im)[W], const Dot& dot,
                                             Map map = Map{})
{
  static_assert(V >= 1 && V <= 32 && (V & (V - 1)) == 0, "V must be a power of two <= 32");
  static_assert(W >= 1 && W <= V && V % W == 0, "W must divide V");
  constexpr int kTps = V / W;  // threads sharing one site
  constexpr int kWarps = NW;
  __shared__ double sh[kWarps][V][4];
  __shared__ unsigned is_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

#pragma unroll
  for (int off = 16; off >= kTps; off >>= 1) {
#pragma unroll
    for (int k = 0; k < W; ++k) {
      csum_merge(re[k], shfl_xor(re[k], off));
      csum_merge(im[k], shfl_xor(im[k], off));
    }
  }
  if (lane < kTps && warp < kWarps) {
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const int v = map(lane, k, W);
      sh[warp][v][0] = re[k].s;
      sh[warp][v][1] = re[k].c;
      sh[warp][v][2] = im[k].s;
      sh[warp][v][3] = im[k].c;
    }
  }
  __syncthreads();
  if (threadIdx.x < V) {
    const int v = threadIdx.x;
    CSum r{sh[0][v][0], sh[0][v][1]}, i{sh[0][v][2], sh[0][v][3]};
    for (int w = 1; w < kWarps; ++w) {
      csum_merge(r, CSum{sh[w][v][0], sh[w][v][1]});
      csum_merge(i, CSum{sh[w][v][2], sh[w][v][3]});
    }
    double* p = dot.partials + ((size_t)blockIdx.x * V + v) * 4;
    p[0] = r.s;
    p[1] = r.c;
    p[2] = i.s;
    p[3] = i.c;
    if (dot.defer) {
      if (blockIdx.x == 0 && v == 0)
        dot.counter[1] = gridDim.x;
    } else {
      __threadfence();
    }
  }
  if (dot.defer)
    return;  // uniform: a launch parameter
  __syncthreads();
  if (threadIdx.x == 0)
    is_last = (atomicAdd(dot.counter, 1u) == gridDim.x - 1) ? 1u : 0u;
  __syncthreads();
  if (!is_last)
    return;
  __threadfence();
  grid_combine<V>(dot.partials, (int)gridDim.x, dot.mu, sh);
  if (threadIdx.x == 0)
    *dot.counter = 0u;  // ready for the next launch on this stream
}

template <int V>
__device__ __forceinline__ void dot_finish(CSum re, CSum im, const Dot& dot)
{
  CSum r[1] = {re}, i[1] = {im};
  dot_finish_w<V, 1>(r, i, dot);
}

// ------------------------------------------------------------------ packed access
// W consecutive complex elements of one site, as wide loads: two float2 per float4,
// one double2 each. Offsets are multiples of W elements, so the loads are aligned.
template <int W>
__device__ __forceinline__ void ldw(const float2* p, double2 (&o)[W], uintptr_t = 0)
{
  if constexpr (W == 1) {
    o[0] = ld(p);
  } else {
#pragma unroll
    for (int k = 0; k < W / 2; ++k) {
      const float4 f = reinterpret_cast<const float4*>(p)[k];
      o[2 * k] = make_double2((double)f.x, (double)f.y);
      o[2 * k + 1] = make_double2((double)f.z, (double)f.w);
    }
  }
}

template <int W>
__device__ __forceinline__ void ldw(const double2* p, double2 (&o)[W], uintptr_t = 0)
{
#pragma unroll
  for (int k = 0; k < W; ++k)
    o[k] = p[k];
}

template <int W>
__device__ __forceinline__ void stw(float2* p, const double2 (&v)[W], uintptr_t = 0)
{
  if constexpr (W == 1) {
    st(p, v[0]);
  } else {
#pragma unroll
    for (int k = 0; k < W / 2; ++k)
      reinterpret_cast<float4*>(p)[k] =
        make_float4(__double2float_rn(v[2 * k].x), __double2float_rn(v[2 * k].y),
                    __double2float_rn(v[2 * k + 1].x), __double2float_rn(v[2 * k + 1].y));
  }
}

template <int W>
__device__ __forceinline__ void stw(double2* p, const double2 (&v)[W], uintptr_t = 0)
{
#pragma unroll
  for (int k = 0; k < W; ++k)
    p[k] = v[k];
}

// W consecutive FP32X elements: the hi parts as float4 loads, the residuals as one
// 4W-byte load (W = 1, 2 or 4; the offsets are multiples of W elements).
template <int W>
__device__ __forceinline__ void ldw_hi(const xf2* p, float2 (&h)[W])
{
  if constexpr (W == 1) {
    h[0] = *reinterpret_cast<const float2*>(p);
  } else {
#pragma unroll
    for (int k = 0; k < W / 2; ++k) {
      const float4 f = reinterpret_cast<const float4*>(p)[k];
      h[2 * k] = make_float2(f.x, f.y);
      h[2 * k + 1] = make_float2(f.z, f.w);
    }
  }
}

template <int W>
__device__ __forceinline__ void xres_ld(const xf2* p, uintptr_t xlo, __nv_bfloat162 (&l)[W])
{
  const __nv_bfloat162* r = xres(p, xlo);
  if constexpr (W == 4) {
    const uint4 u = *reinterpret_cast<const uint4*>(r);
    const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
      l[k] = *reinterpret_cast<const __nv_bfloat162*>(&w[k]);
  } else if constexpr (W == 2) {
    const uint2 u = *reinterpret_cast<const uint2*>(r);
    l[0] = *reinterpret_cast<const __nv_bfloat162*>(&u.x);
    l[1] = *reinterpret_cast<const __nv_bfloat162*>(&u.y);
  } else {
#pragma unroll
    for (int k = 0; k < W; ++k)
      l[k] = r[k];
  }
}

template <int W>
__device__ __forceinline__ void ldw(const xf2* p, double2 (&o)[W], uintptr_t xlo)
{
  float2 h[W];
  ldw_hi<W>(p, h);
  __nv_bfloat162 l[W];
  xres_ld<W>(p, xlo, l);
#pragma unroll
  for (int k = 0; k < W; ++k)
    o[k] = xjoin(h[k].x, h[k].y, l[k]);
}

template <int W>
__device__ __forceinline__ void stw(xf2* p, const double2 (&v)[W], uintptr_t xlo)
{
  float2 h[W];
  __nv_bfloat162 l[W];
#pragma unroll
  for (int k = 0; k < W; ++k)
    xsplit(v[k], h[k], l[k]);
  if constexpr (W == 1) {
    *reinterpret_cast<float2*>(p) = h[0];
  } else {
#pragma unroll
    for (int k = 0; k < W / 2; ++k)
      reinterpret_cast<float4*>(p)[k] = make_float4(h[2 * k].x, h[2 * k].y, h[2 * k + 1].x,
                                                    h[2 * k + 1].y);
  }
  __nv_bfloat162* r = xres(p, xlo);
  if constexpr (W == 4) {
    uint4 u;
    u.x = *reinterpret_cast<const unsigned*>(&l[0]);
    u.y = *reinterpret_cast<const unsigned*>(&l[1]);
    u.z = *reinterpret_cast<const unsigned*>(&l[2]);
    u.w = *reinterpret_cast<const unsigned*>(&l[3]);
    *reinterpret_cast<uint4*>(r) = u;
  } else if constexpr (W == 2) {
    uint2 u;
    u.x = *reinterpret_cast<const unsigned*>(&l[0]);
    u.y = *reinterpret_cast<const unsigned*>(&l[1]);
    *reinterpret_cast<uint2*>(r) = u;
  } else {
#pragma unroll
    for (int k = 0; k < W; ++k)
      r[k] = l[k];
  }
}

// W consecutive elements kept in their storage type (the same wide loads as ldw). A
// value a kernel needs twice, far apart, costs half the registers as float2 and is
// widened exactly at each use.
template <int W>
__device__ __forceinline__ void ldw_raw(const float2* p, float2 (&o)[W], uintptr_t = 0)
{
  if constexpr (W == 1) {
    o[0] = *p;
  } else {
#pragma unroll
    for (int k = 0; k < W / 2; ++k) {
      const float4 f = reinterpret_cast<const float4*>(p)[k];
      o[2 * k] = make_float2(f.x, f.y);
      o[2 * k + 1] = make_float2(f.z, f.w);
    }
  }
}

template <int W>
__device__ __forceinline__ void ldw_raw(const double2* p, double2 (&o)[W], uintptr_t = 0)
{
#pragma unroll
  for (int k = 0; k < W; ++k)
    o[k] = p[k];
}

// An FP32X element as stored: hi and its residual (12 bytes, three registers).
struct xraw {
  float2 h;
  __nv_bfloat162 l;
};
template <int W>
__device__ __forceinline__ void ldw_raw(const xf2* p, xraw (&o)[W], uintptr_t xlo)
{
  float2 h[W];
  ldw_hi<W>(p, h);
  __nv_bfloat162 l[W];
  xres_ld<W>(p, xlo, l);
#pragma unroll
  for (int k = 0; k < W; ++k)
    o[k] = xraw{h[k], l[k]};
}

// The register type ldw_raw fills for a storage type.
template <typename VT2>
struct Raw {
  using type = VT2;
};
template <>
struct Raw<xf2> {
  using type = xraw;
};

__device__ __forceinline__ double2 widen(double2 v) { return v; }
__device__ __forceinline__ double2 widen(float2 v)
{
  return make_double2((double)v.x, (double)v.y);
}
__device__ __forceinline__ double2 widen(const xraw& v) { return xjoin(v.h.x, v.h.y, v.l); }

// ------------------------------------------------------------------ the operator row
// f(m) for the entries m < cnt of a row, unrolled when the bound Z is known.
template <int Z, class F>
__device__ __forceinline__ void for_entries(int cnt, F&& f)
{
  if constexpr (Z > 0) {
#pragma unroll
    for (int m = 0; m < Z; ++m)
      if (m < cnt)
        f(m);
  } else {
    for (int m = 0; m < cnt; ++m)
      f(m);
  }
}

// acc += sum_m H_im x_{j_m} for one (site i, vector v), neighbours in ELL order.
// Z > 0: the row length bound is known at compile time and the loop is unrolled.
template <int V, int Z, class A, bool C, typename VT2>
__device__ __forceinline__ void hop_row(const Op& op, const Tables& tb, int i, int v,
                                        const VT2* __restrict__ x, double& tr, double& ti)
{
  const int cnt = op.uniform ? (Z > 0 ? Z : op.z) : op.nn[i];
  if constexpr (Z > 0) {
#pragma unroll
    for (int m = 0; m < Z; ++m) {
      if (m < cnt) {
        const size_t e = (size_t)m * op.n + i;
        int j, c;
        double2 h;
        ell_entry<C>(op, tb, e, i, j, h, c);
        const double2 y = ld(x + (size_t)j * V + v, op.xlo);
        tr = A::add(tr, A::cre(h.x, h.y, y.x, y.y));
        ti = A::add(ti, A::cim(h.x, h.y, y.x, y.y));
      }
    }
  } else {
    for (int m = 0; m < cnt; ++m) {
      const size_t e = (size_t)m * op.n + i;
      int j, c;
      double2 h;
      ell_entry<C>(op, tb, e, i, j, h, c);
      const double2 y = ld(x + (size_t)j * V + v, op.xlo);
      tr = A::add(tr, A::cre(h.x, h.y, y.x, y.y));
      ti = A::add(ti, A::cim(h.x, h.y, y.x, y.y));
    }
  }
}

enum StepMode { kApply = 0, kCheb = 1 };

// What a step fuses after writing T_k (the DOT template parameter): nothing; the moment
// <left|T_k>; or the pair <T_k|T_k>, <T_{k-1}|T_k> of a symmetric moment set (left =
// right = phi), from which T_j T_k = (T_{j+k} + T_{|j-k|}) / 2 gives mu_2k and
// mu_{2k-1} (k_pair_moments).
enum DotMode { kNoDot = 0, kDotLeft = 1, kDotPair = 2 };

// Grid-stride loop shape of each operator kernel, per format (C), storage type and
// row bound Z. The pipelined loop loads the next element's row (and, in k_step, its
// streamed inputs) one iteration ahead, so an iteration waits on one memory round
// trip instead of two; it costs registers, hence resident warps. Chosen from B200
// measurements (graphene 2,097,152 sites, square 1,048,576, cubic 16,777,216): the
// step gains 10-60 % from it in both formats (with its register budget fixed by
// step_min_blocks); the other coded kernels 10-50 % (the evolution term k_cheb2
// excepted); the other ELL kernels lose. GQT_PIPELINE = 0 or 1 at compile time
// forces one loop shape everywhere.
#ifndef GQT_PIPELINE
#define GQT_PIPELINE -1
#endif
enum PipeKernel { kPipeStep, kPipeStepVec, kPipeStepMulti, kPipeXop, kPipeCheb2, kPipeCheb2x };

template <int K, bool C, typename VT2, int Z>
__host__ __device__ constexpr bool pipelined()
{
  if constexpr (Z <= 0) {
    return false;  // the pipelined loops need the row bound at compile time
  } else if constexpr (GQT_PIPELINE >= 0) {
    return GQT_PIPELINE > 0;
  } else {
    switch (K) {
      case kPipeStep:
        return true;
      case kPipeStepVec:
      case kPipeStepMulti:
      case kPipeXop:
      case kPipeCheb2x:
        return C;
      default:
        return false;
    }
  }
}

// One site's row, fetched one grid-stride iteration ahead of its use: the row length
// and the table rows (coded form) or neighbour indices (ELL form) of its Z entries.
// Entries past the row length are in bounds (padding) and skipped through cnt.
template <int Z>
struct RowIdx {
  int cnt;
  int idx[Z];
};

template <int Z, bool C>
__device__ __forceinline__ void fetch_row(const Op& op, int i, RowIdx<Z>& r)
{
  r.cnt = op.uniform ? Z : op.nn[i];
#pragma unroll
  for (int m = 0; m < Z; ++m) {
    const size_t e = (size_t)m * op.n + i;
    if constexpr (C)
      r.idx[m] = op.code[e];
    else
      r.idx[m] = op.nl[e];
  }
}

// hop_row from a prefetched row: every gather is issued before the arithmetic, which
// keeps the reference's neighbour order.
template <int V, int Z, class A, bool C, typename VT2>
__device__ __forceinline__ void hop_row_pre(const Op& op, const Tables& tb, int i, int v,
                                            const RowIdx<Z>& r, const VT2* __restrict__ x,
                                            double& tr, double& ti)
{
  int j[Z];
  double2 h[Z], y[Z];
#pragma unroll
  for (int m = 0; m < Z; ++m) {
    if constexpr (C) {
      j[m] = i + tb.delta[r.idx[m]];
      h[m] = tb.hop[r.idx[m]];
    } else {
      j[m] = r.idx[m];
      h[m] = m < r.cnt ? op.hop[(size_t)m * op.n + i] : make_double2(0.0, 0.0);
    }
  }
#pragma unroll
  for (int m = 0; m < Z; ++m)
    if (m < r.cnt)
      y[m] = ld(x + (size_t)j[m] * V + v, op.xlo);
#pragma unroll
  for (int m = 0; m < Z; ++m) {
    if (m < r.cnt) {
      tr = A::add(tr, A::cre(h[m].x, h[m].y, y[m].x, y[m].y));
      ti = A::add(ti, A::cim(h[m].x, h[m].y, y[m].x, y[m].y));
    }
  }
}

// Neighbour j and hopping h of entry m of row i, from its prefetched index.
template <bool C>
__device__ __forceinline__ void row_entry(const Op& op, const Tables& tb, int i, int m,
                                          int idx, int& j, double2& h)
{
  if constexpr (C) {
    j = i + tb.delta[idx];
    h = tb.hop[idx];
  } else {
    j = idx;
    h = op.hop[(size_t)m * op.n + i];
  }
}

// acc[k] += sum_m H_im x_{j_m, v0 + k} for W consecutive vectors, from a prefetched row.
template <int V, int W, int Z, class A, bool C, typename VT2>
__device__ __forceinline__ void hop_row_w(const Op& op, const Tables& tb, int i, int v0,
                                          const RowIdx<Z>& r, const VT2* __restrict__ x,
                                          double (&tr)[W], double (&ti)[W])
{
#pragma unroll
  for (int m = 0; m < Z; ++m) {
    if (m < r.cnt) {
      int j;
      double2 h;
      row_entry<C>(op, tb, i, m, r.idx[m], j, h);
      double2 y[W];
      ldw<W>(x + (size_t)j * V + v0, y, op.xlo);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        tr[k] = A::add(tr[k], A::cre(h.x, h.y, y[k].x, y[k].y));
        ti[k] = A::add(ti[k], A::cim(h.x, h.y, y[k].x, y[k].y));
      }
    }
  }
}

// xx of entry m of row i, from its prefetched index.
template <bool C>
__device__ __forceinline__ double row_xx(const Op& op, const Tables& tb, int i, int m, int idx)
{
  if constexpr (C)
    return tb.xx[idx];
  else
    return op.xx[(size_t)m * op.n + i];
}

// Runs f(g, row) over this thread's grid-stride items g < total (site g / PER), with
// each item's row loaded one iteration ahead: an iteration then waits on one memory
// round trip (its gathers) instead of two (row, then gathers).
template <int Z, int PER, bool C, class F>
__device__ __forceinline__ void pipelined_rows(const Op& op, size_t total, F&& f)
{
  const size_t stride = (size_t)gridDim.x * kBlock;
  size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x;
  RowIdx<Z> cur;
  if (g < total)
    fetch_row<Z, C>(op, (int)(g / PER), cur);
  for (; g < total; g += stride) {
    RowIdx<Z> nxt = cur;
    if (g + stride < total)
      fetch_row<Z, C>(op, (int)((g + stride) / PER), nxt);
    f(g, cur);
    cur = nxt;
  }
}

// The ELL form's hoppings of one row, loaded one iteration ahead with its indices (the
// coded form keeps its hoppings in shared memory).
template <int Z>
struct RowHop {
  double2 h[Z];
};
template <>
struct RowHop<0> {};  // coded form: nothing travels

template <int Z>
__device__ __forceinline__ void fetch_hops(const Op& op, int i, RowHop<Z>& r)
{
  if constexpr (Z > 0) {
#pragma unroll
    for (int m = 0; m < Z; ++m)
      r.h[m] = op.hop[(size_t)m * op.n + i];
  }
}

// hop_row from a prefetched ELL row and its prefetched hoppings.
template <int V, int Z, class A, typename VT2>
__device__ __forceinline__ void hop_row_ahead(int v, const RowIdx<Z>& r, const RowHop<Z>& hr,
                                              const VT2* __restrict__ x, uintptr_t xlo,
                                              double& tr, double& ti)
{
  double2 y[Z];
#pragma unroll
  for (int m = 0; m < Z; ++m)
    if (m < r.cnt)
      y[m] = ld(x + (size_t)r.idx[m] * V + v, xlo);
#pragma unroll
  for (int m = 0; m < Z; ++m) {
    if (m < r.cnt) {
      tr = A::add(tr, A::cre(hr.h[m].x, hr.h[m].y, y[m].x, y[m].y));
      ti = A::add(ti, A::cim(hr.h[m].x, hr.h[m].y, y[m].x, y[m].y));
    }
  }
}

// The streamed inputs of one element: potential, T_{m-1}, T_{m-2} and left.
struct Streams {
  double p;
  double2 x, y0, l;
};

template <typename VT2, int V, int MODE, int DOT>
__device__ __forceinline__ void fetch_streams(const Op& op, size_t g, const VT2* t0,
                                              const VT2* __restrict__ t1,
                                              const VT2* __restrict__ left, Streams& s)
{
  s.p = op.pot[g / V];
  s.x = ld(t1 + g, op.xlo);
  s.y0 = make_double2(0.0, 0.0);
  s.l = s.y0;
  if constexpr (MODE == kCheb)
    s.y0 = ld(t0 + g, op.xlo);
  if constexpr (DOT == kDotLeft)
    s.l = ld(left + g, op.xlo);
}

// The fused moment terms of one element: o = T_k as stored, x = T_{k-1}, l = left.
template <int DOT>
__device__ __forceinline__ void step_dot(CSum (&re)[2], CSum (&im)[2], double2 o, double2 x,
                                         double2 l)
{
  if constexpr (DOT == kDotLeft) {
    dot_term(re[0], im[0], o, l);
  } else if constexpr (DOT == kDotPair) {
    dot_term_self(re[0], o);
    dot_term(re[1], im[1], o, x);
  }
}

// out = H t1 / E_max (kApply) or out = 2 H t1 / E_max - t0 (kCheb), optionally fused
// with the moment <left|out>. out may alias t0 (a site reads t0 before writing out).
// Follows gpu_apply_hamiltonian / gpu_kernel_polynomial (src/hamiltonian.cu:153-186,
// :886-925) with gpu_find_inner_product_1/2 (src/vector.cu:243-401) fused in.
//
// With a compile-time row bound (Z > 0) the grid-stride loop is software-pipelined:
// the next element's row indices are loaded while this element's gathers are in
// flight, so an iteration waits on one memory round trip (the gathers) instead of
// two (row, then gathers).
// Resident blocks per SM the step is compiled for (its register budget): 3 for rows of
// up to four entries, 2 for six (the pipelined row of six holds twice the indices).
// Measured on B200 against the compiler's own choice, which varied from 43 to 114
// registers between near-identical builds of the same loop. The pair mode on the ELL
// arrays (hoppings travelling with the prefetched row, two compensated products) takes
// 2: at 3 it spilled 50-180 bytes per thread.
// GQT_STEP_BLOCKS_ROWS6 (compile time, default 2) sets the budget for rows of six: at 3
// (80 registers, 80 bytes spilled) the FP64 step ran 13-21 % slower on B200 (cubic slab
// 32x256x256: 4.9e10 against 5.7e10 site-moments/s; cubic 256^3: 4.6e10 against 5.9e10).
#ifndef GQT_STEP_BLOCKS_ROWS6
#define GQT_STEP_BLOCKS_ROWS6 2
#endif
template <int Z, int DOT = kDotLeft, bool C = true>
constexpr int step_min_blocks()
{
  if constexpr (DOT == kDotPair && !C)
    return 2;
  return Z >= 6 ? GQT_STEP_BLOCKS_ROWS6 : 3;
}

template <typename VT2, int V, int Z, class A, int MODE, int DOT, bool C>
__global__ void __launch_bounds__(kBlock, step_min_blocks<Z, DOT, C>()) k_step(Op op, const VT2* t0,
                                                 const VT2* __restrict__ t1, VT2* out,
                                                 const VT2* __restrict__ left, Dot dot)
{
  static_assert(DOT != kDotPair || V == 1, "pair moments: one vector per thread");
  const Tables tb = load_tables<C>(op);
  const size_t total = (size_t)op.n * V;
  const size_t stride = (size_t)gridDim.x * kBlock;
  CSum re[2] = {{0.0, 0.0}, {0.0, 0.0}}, im[2] = {{0.0, 0.0}, {0.0, 0.0}};
  size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x;
  if constexpr (Z > 0 && pipelined<kPipeStep, C, VT2, Z>()) {
    RowIdx<Z> cur;
    constexpr bool kHops = !C;
    RowHop<(kHops ? Z : 0)> hc;  // ELL form: the row's hoppings travel with its indices
    Streams sc;
    if (g < total) {
      fetch_row<Z, C>(op, (int)(g / V), cur);
      if constexpr (kHops)
        fetch_hops<Z>(op, (int)(g / V), hc);
    }
    pdl_wait();
    if (g < total)
      fetch_streams<VT2, V, MODE, DOT>(op, g, t0, t1, left, sc);
    for (; g < total; g += stride) {
      const int i = (int)(g / V);
      const int v = (int)(g % V);
      const size_t gn = g + stride;
      const Streams s = sc;
      RowIdx<Z> nxt = cur;
      RowHop<(kHops ? Z : 0)> hn = hc;
      if (gn < total) {
        fetch_row<Z, C>(op, (int)(gn / V), nxt);
        if constexpr (kHops)
          fetch_hops<Z>(op, (int)(gn / V), hn);
        fetch_streams<VT2, V, MODE, DOT>(op, gn, t0, t1, left, sc);
      }
      double tr = A::mul(s.p, s.x.x);
      double ti = A::mul(s.p, s.x.y);
      if constexpr (kHops)
        hop_row_ahead<V, Z, A>(v, cur, hc, t1, op.xlo, tr, ti);
      else
        hop_row_pre<V, Z, A, C>(op, tb, i, v, cur, t1, tr, ti);
      tr = A::scale(tr, op);
      ti = A::scale(ti, op);
      if constexpr (MODE == kCheb) {
        tr = A::two_x_minus(tr, s.y0.x);
        ti = A::two_x_minus(ti, s.y0.y);
      }
      const double2 r = make_double2(tr, ti);
      st(out + g, r, op.xlo);
      step_dot<DOT>(re, im, stored(out, r), s.x, s.l);
      cur = nxt;
      hc = hn;
    }
  } else {
    pdl_wait();
    for (; g < total; g += stride) {
      const int i = (int)(g / V);
      const int v = (int)(g % V);
      const double p = op.pot[i];
      const double2 x = ld(t1 + g, op.xlo);
      double tr = A::mul(p, x.x);
      double ti = A::mul(p, x.y);
      hop_row<V, Z, A, C>(op, tb, i, v, t1, tr, ti);
      tr = A::scale(tr, op);
      ti = A::scale(ti, op);
      if constexpr (MODE == kCheb) {
        const double2 y0 = ld(t0 + g, op.xlo);
        tr = A::two_x_minus(tr, y0.x);
        ti = A::two_x_minus(ti, y0.y);
      }
      const double2 r = make_double2(tr, ti);
      st(out + g, r, op.xlo);
      if constexpr (DOT == kDotLeft)
        step_dot<DOT>(re, im, stored(out, r), x, ld(left + g, op.xlo));
      else
        step_dot<DOT>(re, im, stored(out, r), x, x);
    }
  }
  pdl_trigger();
  if constexpr (DOT == kDotLeft)
    dot_finish<V>(re[0], im[0], dot);
  else if constexpr (DOT == kDotPair)
    dot_finish_w<2, 2>(re, im, dot);
}

// <left|state> alone (moment 0).
template <typename VT2, int V>
__global__ void __launch_bounds__(kBlock) k_dot(size_t total, const VT2* __restrict__ state,
                                                const VT2* __restrict__ left, Dot dot)
{
  CSum re{0.0, 0.0}, im{0.0, 0.0};
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
       g += (size_t)gridDim.x * kBlock)
    dot_term(re, im, ld(state + g, dot.xlo), ld(left + g, dot.xlo));
  dot_finish<V>(re, im, dot);
}

// Batched step: each thread advances W consecutive vectors of one site, so a site's
// ELL row, potential and row length are read once per W vectors and every vector
// access is a wide load. Same arithmetic per element as k_step; with FastArith the
// moment uses the FP64 value of T_m before its FP32 rounding and plain FP64 per-thread
// sums (a few dozen terms each), merged with TwoSum across lanes, blocks and the grid.
// Register budgets of the batched steps, as blocks per SM, measured on B200 against the
// compiler's own choice: k_step_vec at 4 (64 registers: +9 % for 16 FP32 vectors on
// graphene, +7 % on cubic, +17 % for 32 vectors on the ELL arrays); k_step_multi at 3
// with the coded table, 4 on the ELL arrays.
// The streamed inputs of one k_step_vec item (W vectors of one site) in their storage
// type: potential, T_{k-1}, T_{k-2} (kCheb) and left (kDotLeft).
template <typename VT2, int W, int MODE, int DOT>
struct VecStreams {
  double p;
  typename Raw<VT2>::type x[W];
  typename Raw<VT2>::type y0[MODE == kCheb ? W : 1];
  typename Raw<VT2>::type l[DOT == kDotLeft ? W : 1];
};

template <int V, int W, int TPS, int MODE, int DOT, typename VT2>
__device__ __forceinline__ void fetch_vec_streams(const Op& op, size_t g, const VT2* t0,
                                                  const VT2* __restrict__ t1,
                                                  const VT2* __restrict__ left,
                                                  VecStreams<VT2, W, MODE, DOT>& s)
{
  const int i = (int)(g / TPS);
  const size_t base = (size_t)i * V + (size_t)(g % TPS) * W;
  s.p = op.pot[i];
  ldw_raw<W>(t1 + base, s.x, op.xlo);
  if constexpr (MODE == kCheb)
    ldw_raw<W>(t0 + base, s.y0, op.xlo);
  if constexpr (DOT == kDotLeft)
    ldw_raw<W>(left + base, s.l, op.xlo);
}

// Whether k_step_vec loads an item's streamed inputs one grid-stride iteration ahead
// (with its row), so that they are in flight during the previous item's gathers: the
// in-place store of T_k (over T_{k-2}) keeps the compiler from hoisting them itself.
// GQT_VEC_STREAMS = 0 or 1 at compile time forces it off or on.
#ifndef GQT_VEC_STREAMS
#define GQT_VEC_STREAMS 1
#endif
// Whether the direct steps load left before storing T_k (left is read-only, but the
// compiler cannot move its load above the store itself): 0 or 1 at compile time.
#ifndef GQT_LEFT_EARLY
#define GQT_LEFT_EARLY 0
#endif
template <typename VT2, int DOT>
__host__ __device__ constexpr bool vec_streams_ahead()
{
  // pair mode only (the direct step's 4-vector items spill holding a second set), and
  // not for FP32X (its residuals' registers spill at the look-ahead's budget)
  return GQT_VEC_STREAMS > 0 && DOT == kDotPair && !std::is_same<VT2, xf2>::value;
}

// The pair mode of a symmetric set keeps three sums per vector and T_{k-1} for the whole
// item. The FP32 form advances 4 vectors per thread there with its streamed inputs one
// item ahead: 2 blocks per SM (128 registers). The FP64 form, with the look-ahead,
// takes 3 blocks (2 on rows of unknown length: 12-24 bytes of spills at 3); the FP32X
// form, without it, 3 on rows of six and of unknown length (at 4 they spilled 16-140
// bytes per thread) and 4 otherwise.
constexpr int kVecMinBlocks = 4;
template <typename VT2, int Z, int DOT>
constexpr int vec_min_blocks()
{
  constexpr bool f64 = std::is_same<VT2, double2>::value;
  if constexpr (DOT != kDotPair)
    return kVecMinBlocks;
  else if constexpr (std::is_same<VT2, float2>::value)
    return 2;
  else if constexpr (Z <= 0)
    return f64 ? 2 : 3;
  else if constexpr (vec_streams_ahead<VT2, DOT>())
    return 3;  // FP64: the look-ahead's second set of streams
  else
    return Z >= 6 ? 3 : kVecMinBlocks;
}
template <bool C, int Z = 4, int DOT = kDotLeft>
constexpr int multi_min_blocks()
{
  return (C || (DOT == kDotPair && Z <= 0)) ? 3 : 4;
}

template <typename VT2, int V, int W, int Z, class A, int MODE, int DOT, bool C>
__global__ void __launch_bounds__(kBlock, vec_min_blocks<VT2, Z, DOT>()) k_step_vec(Op op, const VT2* t0,
                                                     const VT2* __restrict__ t1, VT2* out,
                                                     const VT2* __restrict__ left, Dot dot)
{
  const Tables tb = load_tables<C>(op);
  constexpr int kTps = V / W;
  constexpr bool kExact = std::is_same<A, ExactArith>::value;
  const size_t items = (size_t)op.n * kTps;
  // Pair moments keep two sums per vector: [2w] <T_k|T_k>, [2w + 1] <T_{k-1}|T_k>.
  constexpr int kSums = DOT == kDotPair ? 2 * W : W;
  CSum re[kSums], im[kSums];
#pragma unroll
  for (int k = 0; k < kSums; ++k)
    re[k] = im[k] = CSum{0.0, 0.0};
  // Pipelined as in k_step where the policy says so: the next item's row first, and
  // (kPreS) its streamed inputs too.
  constexpr bool kPre = Z > 0 && pipelined<kPipeStepVec, C, VT2, Z>();
  constexpr bool kPreS = kPre && vec_streams_ahead<VT2, DOT>();
  RowIdx<(Z > 0 ? Z : 1)> cur, nxt;
  VecStreams<VT2, W, MODE, DOT> sc;
  const size_t stride = (size_t)gridDim.x * kBlock;
  size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x;
  if constexpr (kPre) {
    if (g < items) {
      fetch_row<(Z > 0 ? Z : 1), C>(op, (int)(g / kTps), cur);
      if constexpr (kPreS)
        fetch_vec_streams<V, W, kTps, MODE, DOT>(op, g, t0, t1, left, sc);
    }
  }
  for (; g < items; g += stride) {
    VecStreams<VT2, W, MODE, DOT> s;
    if constexpr (kPreS)
      s = sc;
    if constexpr (kPre) {
      nxt = cur;
      if (g + stride < items) {
        fetch_row<(Z > 0 ? Z : 1), C>(op, (int)((g + stride) / kTps), nxt);
        if constexpr (kPreS)
          fetch_vec_streams<V, W, kTps, MODE, DOT>(op, g + stride, t0, t1, left, sc);
      }
    }
    const int i = (int)(g / kTps);
    const int v0 = (int)(g % kTps) * W;
    const size_t base = (size_t)i * V + v0;
    if constexpr (!kPreS) {
      // without the look-ahead T_{k-2} and left are loaded late, each right before use
      // (held across the gathers they cost 4-vector items 140-160 bytes of spills)
      s.p = op.pot[i];
      ldw_raw<W>(t1 + base, s.x, op.xlo);
    }
    const double p = s.p;
    const auto& x = s.x;  // T_{k-1} as stored; the pair mode reads it again
    double tr[W], ti[W];
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const double2 xk = widen(x[k]);
      tr[k] = A::mul(p, xk.x);
      ti[k] = A::mul(p, xk.y);
    }
    if constexpr (kPre) {
      hop_row_w<V, W, (Z > 0 ? Z : 1), A, C>(op, tb, i, v0, cur, t1, tr, ti);
    } else {
      const int cnt = op.uniform ? (Z > 0 ? Z : op.z) : op.nn[i];
      auto body = [&](int m) {
        const size_t e = (size_t)m * op.n + i;
        int j, c;
        double2 h;
        ell_entry<C>(op, tb, e, i, j, h, c);
        double2 y[W];
        ldw<W>(t1 + (size_t)j * V + v0, y, op.xlo);
#pragma unroll
        for (int k = 0; k < W; ++k) {
          tr[k] = A::add(tr[k], A::cre(h.x, h.y, y[k].x, y[k].y));
          ti[k] = A::add(ti[k], A::cim(h.x, h.y, y[k].x, y[k].y));
        }
      };
      if constexpr (Z > 0) {
#pragma unroll
        for (int m = 0; m < Z; ++m)
          if (m < cnt)
            body(m);
      } else {
        for (int m = 0; m < cnt; ++m)
          body(m);
      }
    }
    double2 r[W];
    if constexpr (DOT == kDotLeft && !kPreS && GQT_LEFT_EARLY)
      ldw_raw<W>(left + base, s.l, op.xlo);
    if constexpr (MODE == kCheb) {
      if constexpr (!kPreS)
        ldw_raw<W>(t0 + base, s.y0, op.xlo);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const double2 y0 = widen(s.y0[k]);
        r[k] = make_double2(A::two_x_minus(A::scale(tr[k], op), y0.x),
                            A::two_x_minus(A::scale(ti[k], op), y0.y));
      }
    } else {
#pragma unroll
      for (int k = 0; k < W; ++k)
        r[k] = make_double2(A::scale(tr[k], op), A::scale(ti[k], op));
    }
    stw<W>(out + base, r, op.xlo);
    if constexpr (DOT == kDotLeft) {
      if constexpr (!kPreS && !GQT_LEFT_EARLY)
        ldw_raw<W>(left + base, s.l, op.xlo);
      double2 l[W];
#pragma unroll
      for (int k = 0; k < W; ++k)
        l[k] = widen(s.l[k]);
#pragma unroll
      for (int k = 0; k < W; ++k) {
        if constexpr (kExact) {
          dot_term(re[k], im[k], stored(out, r[k]), l[k]);
        } else {
          re[k].s = fma(r[k].x, l[k].x, fma(r[k].y, l[k].y, re[k].s));
          im[k].s = fma(r[k].y, l[k].x, fma(-r[k].x, l[k].y, im[k].s));
        }
      }
    } else if constexpr (DOT == kDotPair) {
      // x holds T_{k-1} as stored; T_k as stored is stored(out, r).
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const double2 o = stored(out, r[k]);
        const double2 xk = widen(x[k]);
        if constexpr (kExact) {
          dot_term_self(re[2 * k], o);
          dot_term(re[2 * k + 1], im[2 * k + 1], o, xk);
        } else {
          re[2 * k].s = fma(o.x, o.x, fma(o.y, o.y, re[2 * k].s));
          re[2 * k + 1].s = fma(o.x, xk.x, fma(o.y, xk.y, re[2 * k + 1].s));
          im[2 * k + 1].s = fma(o.y, xk.x, fma(-o.x, xk.y, im[2 * k + 1].s));
        }
      }
    }
    if constexpr (kPre)
      cur = nxt;
  }
  if constexpr (DOT == kDotLeft)
    dot_finish_w<V, W>(re, im, dot);
  else if constexpr (DOT == kDotPair)
    dot_finish_w<2 * V, 2 * W>(re, im, dot);
}

// ------------------------------------------------------------------ realisation batches
// A batch is a block-diagonal operator of R independent models (disorder realisations
// of uneven lattice sizes), each padded to whole tiles of `tile_sites` sites and with
// its operator pre-divided by its own E_max. Moments are kept per realisation.
struct MultiDot {
  double* partials;        // [blocks][R][V][4]: each block's sums per realisation
  double2* mu;             // this moment's R * V results, [r][v]
  const int* tile_first;   // [R + 1]: realisation r owns tiles [tile_first[r], tile_first[r+1])
  int n_tiles;
  int tile_sites;
  int n_real;
  int blocks;              // grid of the step launch
  // Host side only: 1 = leave the partials for a later k_tile_reduce over a window of
  // steps (the launch writes the step's grid to *blocks_out).
  int defer;
  int* blocks_out;
};

enum { kDotOnly = 2 };

// Threads < V receive the block sum of vector threadIdx.x (W vectors per thread,
// v0 = (lane % (V/W)) * W). Every thread must call it; it synchronises twice.
template <int V, int W>
__device__ __forceinline__ void block_reduce_w(CSum (&re)[W], CSum (&im)[W], CSum& out_re,
                                               CSum& out_im, double (*sh)[V][4])
{
  constexpr int kTps = V / W;
  constexpr int kWarps = kBlock / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off >= kTps; off >>= 1) {
#pragma unroll
    for (int k = 0; k < W; ++k) {
      csum_merge(re[k], shfl_xor(re[k], off));
      csum_merge(im[k], shfl_xor(im[k], off));
    }
  }
  if (lane < kTps) {
#pragma unroll
    for (int k = 0; k < W; ++k) {
      sh[warp][lane * W + k][0] = re[k].s;
      sh[warp][lane * W + k][1] = re[k].c;
      sh[warp][lane * W + k][2] = im[k].s;
      sh[warp][lane * W + k][3] = im[k].c;
    }
  }
  __syncthreads();
  if (threadIdx.x < V) {
    const int v = threadIdx.x;
    out_re = CSum{sh[0][v][0], sh[0][v][1]};
    out_im = CSum{sh[0][v][2], sh[0][v][3]};
    for (int w = 1; w < kWarps; ++w) {
      csum_merge(out_re, CSum{sh[w][v][0], sh[w][v][1]});
      csum_merge(out_im, CSum{sh[w][v][2], sh[w][v][3]});
    }
  }
  __syncthreads();
}

// One Chebyshev step (or moment 0 / moment 1) over every realisation of a batch.
// Blocks take 256-site tiles grid-stride (tile t goes to block t % G), so the whole
// GPU sweeps one compact wavefront and the neighbour gathers stay in L2; one block
// round of 256 threads never straddles two realisations. A block's tiles come in
// increasing order, so each realisation it meets is one contiguous run: per-thread
// sums are reduced over the block when the run ends and written to the block's slot
// of that realisation; slots of realisations it never meets are zeroed.
// k_tile_reduce then sums the blocks per realisation in fixed order.
template <typename VT2, int V, int W, int Z, class A, int MODE, bool C, int DOT = kDotLeft>
__global__ void __launch_bounds__(kBlock, multi_min_blocks<C, Z, DOT>()) k_step_multi(Op op, const VT2* t0,
                                                       const VT2* __restrict__ t1, VT2* out,
                                                       const VT2* __restrict__ left, MultiDot md)
{
  const Tables tb = load_tables<C>(op);
  constexpr int kTps = V / W;
  constexpr int kWarps = kBlock / 32;
  constexpr bool kExact = std::is_same<A, ExactArith>::value;
  // Sums per realisation: V moments <left|out>, or for the pair mode of a symmetric set
  // 2V ([2v] <T_k|T_k>, [2v + 1] <T_{k-1}|T_k>); a thread holds kSums of them.
  static_assert(DOT == kDotLeft || (DOT == kDotPair && MODE != kDotOnly), "dot mode");
  constexpr int kVS = DOT == kDotPair ? 2 * V : V;
  constexpr int kSums = DOT == kDotPair ? 2 * W : W;
  __shared__ double sh[kWarps][kVS][4];
  const int R = md.n_real;
  const size_t items_per_tile = (size_t)md.tile_sites * kTps;
  double* slots = md.partials + (size_t)blockIdx.x * R * kVS * 4;
  int r = 0;
  unsigned touched = 0u;  // realisations this block has written (R <= 32)
  CSum re[kSums], im[kSums];
#pragma unroll
  for (int k = 0; k < kSums; ++k)
    re[k] = im[k] = CSum{0.0, 0.0};

  auto flush = [&](int rr) {
    CSum br{0.0, 0.0}, bi{0.0, 0.0};
    block_reduce_w<kVS, kSums>(re, im, br, bi, sh);
    if (threadIdx.x < kVS) {
      double* q = slots + ((size_t)rr * kVS + threadIdx.x) * 4;
      q[0] = br.s;
      q[1] = br.c;
      q[2] = bi.s;
      q[3] = bi.c;
    }
    touched |= 1u << rr;
#pragma unroll
    for (int k = 0; k < kSums; ++k)
      re[k] = im[k] = CSum{0.0, 0.0};
  };

  bool any = false;
  for (int t = blockIdx.x; t < md.n_tiles; t += gridDim.x) {
    if (t >= md.tile_first[r + 1]) {  // block-uniform: the next tile is in a later model
      if (any)
        flush(r);
      while (t >= md.tile_first[r + 1])
        ++r;
    }
    any = true;
    // Software-pipelined within the tile: the next item's row is loaded first, and in
    // pair mode (kPreS) its streamed inputs too, as in k_step_vec.
    constexpr bool kPre = Z > 0 && pipelined<kPipeStepMulti, C, VT2, Z>() && MODE != kDotOnly;
    // (rows of six spill with the look-ahead at this kernel's budget)
    constexpr bool kPreS = kPre && vec_streams_ahead<VT2, DOT>() && Z < 6;
    constexpr int kSM = MODE == kDotOnly ? kApply : MODE;  // VecStreams' mode
    RowIdx<(Z > 0 ? Z : 1)> cur, nxt;
    VecStreams<VT2, W, kSM, DOT> sc;
    if constexpr (kPre) {
      if (threadIdx.x < items_per_tile) {
        const size_t g0 = (size_t)t * items_per_tile + threadIdx.x;
        fetch_row<(Z > 0 ? Z : 1), C>(op, (int)(g0 / kTps), cur);
        if constexpr (kPreS)
          fetch_vec_streams<V, W, kTps, kSM, DOT>(op, g0, t0, t1, left, sc);
      }
    }
    for (size_t it = threadIdx.x; it < items_per_tile; it += kBlock) {
      const size_t g = (size_t)t * items_per_tile + it;
      VecStreams<VT2, W, kSM, DOT> s;
      if constexpr (kPreS)
        s = sc;
      if constexpr (kPre) {
        nxt = cur;
        if (it + kBlock < items_per_tile) {
          fetch_row<(Z > 0 ? Z : 1), C>(op, (int)((g + kBlock) / kTps), nxt);
          if constexpr (kPreS)
            fetch_vec_streams<V, W, kTps, kSM, DOT>(op, g + kBlock, t0, t1, left, sc);
        }
      }
      const int i = (int)(g / kTps);
      const int v0 = (int)(g % kTps) * W;
      const size_t base = (size_t)i * V + v0;
      double2 r2[W];
      double2 l[DOT == kDotLeft ? W : 1];
      if constexpr (!kPreS && MODE != kDotOnly) {
        s.p = op.pot[i];
        ldw_raw<W>(t1 + base, s.x);
      }
      const auto& x = s.x;  // T_{k-1} as stored (the pair mode's second product)
      if constexpr (MODE == kDotOnly) {
        ldw<W>(t1 + base, r2);
      } else {
        const double p = s.p;
        double tr[W], ti[W];
#pragma unroll
        for (int k = 0; k < W; ++k) {
          const double2 xk = widen(x[k]);
          tr[k] = A::mul(p, xk.x);
          ti[k] = A::mul(p, xk.y);
        }
        if constexpr (kPre) {
          hop_row_w<V, W, (Z > 0 ? Z : 1), A, C>(op, tb, i, v0, cur, t1, tr, ti);
        } else {
          const int cnt = op.uniform ? (Z > 0 ? Z : op.z) : op.nn[i];
          auto body = [&](int m) {
            const size_t e = (size_t)m * op.n + i;
            int j, c;
            double2 h;
            ell_entry<C>(op, tb, e, i, j, h, c);
            double2 y[W];
            ldw<W>(t1 + (size_t)j * V + v0, y);
#pragma unroll
            for (int k = 0; k < W; ++k) {
              tr[k] = A::add(tr[k], A::cre(h.x, h.y, y[k].x, y[k].y));
              ti[k] = A::add(ti[k], A::cim(h.x, h.y, y[k].x, y[k].y));
            }
          };
          if constexpr (Z > 0) {
#pragma unroll
            for (int m = 0; m < Z; ++m)
              if (m < cnt)
                body(m);
          } else {
            for (int m = 0; m < cnt; ++m)
              body(m);
          }
        }
        if constexpr (DOT == kDotLeft && GQT_LEFT_EARLY)
          ldw<W>(left + base, l);
        if constexpr (MODE == kCheb) {
          if constexpr (!kPreS)
            ldw_raw<W>(t0 + base, s.y0);
#pragma unroll
          for (int k = 0; k < W; ++k) {
            const double2 y0 = widen(s.y0[k]);
            r2[k] = make_double2(A::two_x_minus(A::scale(tr[k], op), y0.x),
                                 A::two_x_minus(A::scale(ti[k], op), y0.y));
          }
        } else {
#pragma unroll
          for (int k = 0; k < W; ++k)
            r2[k] = make_double2(A::scale(tr[k], op), A::scale(ti[k], op));
        }
        stw<W>(out + base, r2);
      }
      if constexpr (DOT == kDotLeft) {
        if constexpr (MODE == kDotOnly || !GQT_LEFT_EARLY)
          ldw<W>(left + base, l);
#pragma unroll
        for (int k = 0; k < W; ++k) {
          if constexpr (kExact) {
            dot_term(re[k], im[k], MODE == kDotOnly ? r2[k] : stored(out, r2[k]), l[k]);
          } else {
            re[k].s = fma(r2[k].x, l[k].x, fma(r2[k].y, l[k].y, re[k].s));
            im[k].s = fma(r2[k].y, l[k].x, fma(-r2[k].x, l[k].y, im[k].s));
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < W; ++k) {
          const double2 o = stored(out, r2[k]);
          const double2 xk = widen(x[k]);
          if constexpr (kExact) {
            dot_term_self(re[2 * k], o);
            dot_term(re[2 * k + 1], im[2 * k + 1], o, xk);
          } else {
            re[2 * k].s = fma(o.x, o.x, fma(o.y, o.y, re[2 * k].s));
            re[2 * k + 1].s = fma(o.x, xk.x, fma(o.y, xk.y, re[2 * k + 1].s));
            im[2 * k + 1].s = fma(o.y, xk.x, fma(-o.x, xk.y, im[2 * k + 1].s));
          }
        }
      }
      if constexpr (kPre)
        cur = nxt;
    }
  }
  if (any)
    flush(r);
  // Realisations this block never met get zero sums.
  for (int k = threadIdx.x; k < R * kVS * 4; k += kBlock) {
    const int rr = k / (kVS * 4);
    if (!((touched >> rr) & 1u))
      slots[k] = 0.0;
  }
}

// Per-realisation moments of batch steps: block (p, j) sums the slots of pair
// p = (r, v) of step j over the step's blocks in fixed order and writes
// mu[j * pairs + p]. Step j's slots start j * row_stride doubles into md.partials: one
// launch reduces one step (gridDim.y = 1) or a window of deferred steps, with the same
// sums in the same order either way.
template <int V>
__global__ void __launch_bounds__(kBlock) k_tile_reduce(MultiDot md, size_t row_stride)
{
  const int p = blockIdx.x;
  const int pairs = md.n_real * V;
  const double* row = md.partials + (size_t)blockIdx.y * row_stride;
  CSum re{0.0, 0.0}, im{0.0, 0.0};
  for (int b = threadIdx.x; b < md.blocks; b += kBlock) {
    const double* q = row + ((size_t)b * pairs + p) * 4;
    csum_merge(re, CSum{q[0], q[1]});
    csum_merge(im, CSum{q[2], q[3]});
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    csum_merge(re, shfl_xor(re, off));
    csum_merge(im, shfl_xor(im, off));
  }
  __shared__ double sh[kBlock / 32][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sh[warp][0] = re.s;
    sh[warp][1] = re.c;
    sh[warp][2] = im.s;
    sh[warp][3] = im.c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    CSum a{sh[0][0], sh[0][1]}, b{sh[0][2], sh[0][3]};
    for (int w = 1; w < kBlock / 32; ++w) {
      csum_merge(a, CSum{sh[w][0], sh[w][1]});
      csum_merge(b, CSum{sh[w][2], sh[w][3]});
    }
    md.mu[(size_t)blockIdx.y * pairs + p] =
      make_double2(__dadd_rn(a.s, a.c), __dadd_rn(b.s, b.c));
  }
}

// [X,H] in / E_max (src/hamiltonian.cu:240-271) or V in = -i sum H xx in
// (src/hamiltonian.cu:323-352).
template <typename VT2, int V, int Z, class A, bool CURRENT, bool C>
__global__ void __launch_bounds__(kBlock) k_xop(Op op, const VT2* __restrict__ in,
                                                VT2* __restrict__ out)
{
  const Tables tb = load_tables<C>(op);
  const size_t total = (size_t)op.n * V;
  auto term = [&](double& tr, double& ti, double2 h, double2 y, double x) {
    if constexpr (CURRENT) {
      tr = A::add(tr, A::mul(A::cre(h.x, h.y, y.x, y.y), x));
      ti = A::add(ti, A::mul(A::cim(h.x, h.y, y.x, y.y), x));
    } else {
      tr = A::sub(tr, A::mul(A::cre(h.x, h.y, y.x, y.y), x));
      ti = A::sub(ti, A::mul(A::cim(h.x, h.y, y.x, y.y), x));
    }
  };
  auto finish = [&](size_t g, double tr, double ti) {
    if constexpr (CURRENT) {
      st(out + g, make_double2(ti, -tr));
    } else {
      st(out + g, make_double2(A::scale(tr, op), A::scale(ti, op)));
    }
  };
  if constexpr (Z > 0 && pipelined<kPipeXop, C, VT2, Z>()) {
    pipelined_rows<Z, V, C>(op, total, [&](size_t g, const RowIdx<Z>& r) {
      const int i = (int)(g / V);
      const int v = (int)(g % V);
      double tr = 0.0, ti = 0.0;
#pragma unroll
      for (int m = 0; m < Z; ++m) {
        if (m < r.cnt) {
          int j;
          double2 h;
          row_entry<C>(op, tb, i, m, r.idx[m], j, h);
          term(tr, ti, h, ld(in + (size_t)j * V + v), row_xx<C>(op, tb, i, m, r.idx[m]));
        }
      }
      finish(g, tr, ti);
    });
  } else {
    for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
         g += (size_t)gridDim.x * kBlock) {
      const int i = (int)(g / V);
      const int v = (int)(g % V);
      const int cnt = op.uniform ? op.z : op.nn[i];
      double tr = 0.0, ti = 0.0;
      for_entries<Z>(cnt, [&](int m) {
        const size_t e = (size_t)m * op.n + i;
        int j, c;
        double2 h;
        ell_entry<C>(op, tb, e, i, j, h, c);
        term(tr, ti, h, ld(in + (size_t)j * V + v), ell_xx<C>(op, tb, e, c));
      });
      finish(g, tr, ti);
    }
  }
}

// ------------------------------------------------------------------ time evolution
// out accumulates in OT2 (the state itself in the FP64 form, an FP64 accumulator in
// the FP32 form); the Chebyshev vectors are VT2.

// gpu_chebyshev_01 (src/hamiltonian.cu:404-423); b1 already multiplied by direction.
template <typename VT2, typename OT2, class A>
__global__ void __launch_bounds__(kBlock) k_cheb01(size_t total, const VT2* __restrict__ s0,
                                                   const VT2* __restrict__ s1, OT2* out,
                                                   double b0, double b1)
{
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
       g += (size_t)gridDim.x * kBlock) {
    const double2 a = ld(s0 + g), b = ld(s1 + g);
    st(out + g, make_double2(A::add(A::mul(b0, a.x), A::mul(b1, b.y)),
                             A::sub(A::mul(b0, a.y), A::mul(b1, b.x))));
  }
}

// gpu_chebyshev_1x (src/hamiltonian.cu:619-633).
template <typename VT2, typename OT2, class A>
__global__ void __launch_bounds__(kBlock) k_cheb1x(size_t total, const VT2* __restrict__ s1x,
                                                   OT2* out, double b1)
{
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
       g += (size_t)gridDim.x * kBlock) {
    const double2 a = ld(s1x + g);
    st(out + g, make_double2(A::mul(b1, a.y), A::mul(-b1, a.x)));
  }
}

// The four accumulation labels of src/hamiltonian.cu:498-523 / :727-752.
template <class A>
__device__ __forceinline__ double2 accumulate(double2 o, double b, double tr, double ti,
                                              int label)
{
  switch (label) {
    case 1:
      return make_double2(A::add(o.x, A::mul(b, tr)), A::add(o.y, A::mul(b, ti)));
    case 2:
      return make_double2(A::sub(o.x, A::mul(b, tr)), A::sub(o.y, A::mul(b, ti)));
    case 3:
      return make_double2(A::add(o.x, A::mul(b, ti)), A::sub(o.y, A::mul(b, tr)));
    default:
      return make_double2(A::sub(o.x, A::mul(b, ti)), A::add(o.y, A::mul(b, tr)));
  }
}

// gpu_chebyshev_2 (src/hamiltonian.cu:465-529): s2 = 2 H s1 / E_max - s0 and
// out += (label) * bessel * s2. s2 may alias s0.
template <typename VT2, typename OT2, int V, int Z, class A, bool C>
__global__ void __launch_bounds__(kBlock) k_cheb2(Op op, const VT2* s0,
                                                  const VT2* __restrict__ s1, VT2* s2,
                                                  OT2* __restrict__ out, double bessel,
                                                  int label)
{
  const Tables tb = load_tables<C>(op);
  const size_t total = (size_t)op.n * V;
  auto item = [&](size_t g, auto&& row) {
    const int i = (int)(g / V);
    const int v = (int)(g % V);
    const double p = op.pot[i];
    const double2 x = ld(s1 + g);
    double tr = A::mul(p, x.x), ti = A::mul(p, x.y);
    row(i, v, tr, ti);
    tr = A::scale(tr, op);
    ti = A::scale(ti, op);
    const double2 y0 = ld(s0 + g);
    tr = A::two_x_minus(tr, y0.x);
    ti = A::two_x_minus(ti, y0.y);
    st(out + g, accumulate<A>(ld(out + g), bessel, tr, ti, label));
    st(s2 + g, make_double2(tr, ti));
  };
  if constexpr (Z > 0 && pipelined<kPipeCheb2, C, VT2, Z>()) {
    pipelined_rows<Z, V, C>(op, total, [&](size_t g, const RowIdx<Z>& r) {
      item(g, [&](int i, int v, double& tr, double& ti) {
        hop_row_pre<V, Z, A, C>(op, tb, i, v, r, s1, tr, ti);
      });
    });
  } else {
    for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
         g += (size_t)gridDim.x * kBlock)
      item(g, [&](int i, int v, double& tr, double& ti) {
        hop_row<V, Z, A, C>(op, tb, i, v, s1, tr, ti);
      });
  }
}

// gpu_chebyshev_2x (src/hamiltonian.cu:666-758): the coupled recurrences of T_m and
// [X, T_m], accumulating out += (label) * bessel * [X, T_m]. s2 may alias s0 and s2x
// may alias s0x.
template <typename VT2, typename OT2, int V, int Z, class A, bool C>
__global__ void __launch_bounds__(kBlock) k_cheb2x(Op op, const VT2* s0, const VT2* s0x,
                                                   const VT2* __restrict__ s1,
                                                   const VT2* __restrict__ s1x, VT2* s2,
                                                   VT2* s2x, OT2* __restrict__ out,
                                                   double bessel, int label)
{
  const Tables tb = load_tables<C>(op);
  const size_t total = (size_t)op.n * V;
  auto item = [&](size_t g, auto&& row) {
    const int i = (int)(g / V);
    const int v = (int)(g % V);
    const double p = op.pot[i];
    const double2 a1 = ld(s1 + g), a1x = ld(s1x + g);
    double tr = A::mul(p, a1.x), ti = A::mul(p, a1.y);
    double txr = A::mul(p, a1x.x), txi = A::mul(p, a1x.y);
    // One neighbour term of both recurrences, in the reference's order.
    auto term = [&](double2 h, double2 c, double2 cx, double x) {
      const double hre = A::cre(h.x, h.y, c.x, c.y);
      const double him = A::cim(h.x, h.y, c.x, c.y);
      tr = A::add(tr, hre);
      ti = A::add(ti, him);
      txr = A::add(txr, A::cre(h.x, h.y, cx.x, cx.y));
      txi = A::add(txi, A::cim(h.x, h.y, cx.x, cx.y));
      txr = A::sub(txr, A::mul(hre, x));
      txi = A::sub(txi, A::mul(him, x));
    };
    row(i, v, term);
    const double2 y0 = ld(s0 + g), y0x = ld(s0x + g);
    tr = A::two_x_minus(A::scale(tr, op), y0.x);
    ti = A::two_x_minus(A::scale(ti, op), y0.y);
    txr = A::two_x_minus(A::scale(txr, op), y0x.x);
    txi = A::two_x_minus(A::scale(txi, op), y0x.y);
    st(s2 + g, make_double2(tr, ti));
    st(s2x + g, make_double2(txr, txi));
    st(out + g, accumulate<A>(ld(out + g), bessel, txr, txi, label));
  };
  if constexpr (Z > 0 && pipelined<kPipeCheb2x, C, VT2, Z>()) {
    pipelined_rows<Z, V, C>(op, total, [&](size_t g, const RowIdx<Z>& r) {
      item(g, [&](int i, int v, auto&& term) {
#pragma unroll
        for (int m = 0; m < Z; ++m) {
          if (m < r.cnt) {
            int j;
            double2 h;
            row_entry<C>(op, tb, i, m, r.idx[m], j, h);
            term(h, ld(s1 + (size_t)j * V + v), ld(s1x + (size_t)j * V + v),
                 row_xx<C>(op, tb, i, m, r.idx[m]));
          }
        }
      });
    });
  } else {
    for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
         g += (size_t)gridDim.x * kBlock)
      item(g, [&](int i, int v, auto&& term) {
        const int cnt = op.uniform ? op.z : op.nn[i];
        for_entries<Z>(cnt, [&](int m) {
          const size_t e = (size_t)m * op.n + i;
          int j, c;
          double2 h;
          ell_entry<C>(op, tb, e, i, j, h, c);
          term(h, ld(s1 + (size_t)j * V + v), ld(s1x + (size_t)j * V + v), ell_xx<C>(op, tb, e, c));
        });
      });
  }
}

// ------------------------------------------------------------------ vector kernels
template <typename VT2>
__global__ void __launch_bounds__(kBlock) k_add(size_t total, VT2* __restrict__ dst,
                                                const VT2* __restrict__ src)
{
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
       g += (size_t)gridDim.x * kBlock) {
    const double2 a = ld(dst + g), b = ld(src + g);
    st(dst + g, make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y)));
  }
}

// gpu_apply_sz (src/vector.cu:160-172): even sites copied, odd sites negated.
template <typename VT2>
__global__ void __launch_bounds__(kBlock) k_apply_sz(size_t total, int nvec,
                                                     VT2* __restrict__ dst,
                                                     const VT2* __restrict__ src)
{
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
       g += (size_t)gridDim.x * kBlock) {
    const size_t i = g / (size_t)nvec;
    VT2 a = src[g];
    if (i & 1) {
      a.x = -a.x;
      a.y = -a.y;
    }
    dst[g] = a;
  }
}

// Host split arrays (vector-major) <-> device interleaved [site][vector].
template <typename VT2>
__global__ void __launch_bounds__(kBlock) k_interleave(int n, int nvec,
                                                       const double* __restrict__ re,
                                                       const double* __restrict__ im,
                                                       VT2* __restrict__ out)
{
  const size_t total = (size_t)n * nvec;
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
       g += (size_t)gridDim.x * kBlock) {
    const size_t i = g / (size_t)nvec, k = g % (size_t)nvec;
    st(out + g, make_double2(re[k * n + i], im[k * n + i]));
  }
}

template <typename VT2>
__global__ void __launch_bounds__(kBlock) k_deinterleave(int n, int nvec,
                                                         const VT2* __restrict__ in,
                                                         double* __restrict__ re,
                                                         double* __restrict__ im)
{
  const size_t total = (size_t)n * nvec;
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
       g += (size_t)gridDim.x * kBlock) {
    const size_t i = g / (size_t)nvec, k = g % (size_t)nvec;
    const double2 a = ld(in + g);
    re[k * n + i] = a.x;
    im[k * n + i] = a.y;
  }
}

// out[m] = sum_k in[m*segment + k], one block per segment (gpu_find_inner_product_2,
// src/vector.cu:347-401), compensated.
template <int UNUSED = 0>
__global__ void __launch_bounds__(kBlock) k_segment_sum(const double2* __restrict__ in,
                                                        int segment, double2* __restrict__ out)
{
  CSum re{0.0, 0.0}, im{0.0, 0.0};
  const double2* base = in + (size_t)blockIdx.x * segment;
  for (int k = threadIdx.x; k < segment; k += kBlock) {
    csum_add(re, base[k].x);
    csum_add(im, base[k].y);
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    csum_merge(re, shfl_xor(re, off));
    csum_merge(im, shfl_xor(im, off));
  }
  __shared__ double sh[kBlock / 32][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sh[warp][0] = re.s;
    sh[warp][1] = re.c;
    sh[warp][2] = im.s;
    sh[warp][3] = im.c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    CSum r{sh[0][0], sh[0][1]}, i{sh[0][2], sh[0][3]};
    for (int w = 1; w < kBlock / 32; ++w) {
      csum_merge(r, CSum{sh[w][0], sh[w][1]});
      csum_merge(i, CSum{sh[w][2], sh[w][3]});
    }
    out[blockIdx.x] = make_double2(__dadd_rn(r.s, r.c), __dadd_rn(i.s, i.c));
  }
}

// Grid stage of a window of deferred moments (Dot::defer): block b combines the
// partials of moment b (slab + b * stride, counter[1] blocks) into mu + b * V, in the
// order of the last-block stage of dot_finish_w, so a deferred moment is bit-identical
// to an immediate one.
template <int V>
__global__ void __launch_bounds__(kBlock) k_slab_combine(const double* __restrict__ slab,
                                                         size_t stride,
                                                         const unsigned* __restrict__ counter,
                                                         double2* mu)
{
  __shared__ double sh[kBlock / 32][V][4];
  grid_combine<V>(slab + (size_t)blockIdx.x * stride, (int)counter[1],
                  mu + (size_t)blockIdx.x * V, sh);
}

// Moments of a symmetric set from its pair products: slot k (1 <= k <= K) of `pairs`
// holds, per vector v, A_k = <T_k|T_k> at [k][2v] and B_k = <T_{k-1}|T_k> at
// [k][2v + 1]; slot 0 holds mu_0 = <phi|phi> at [0][v]. With T_j T_k = (T_{j+k} +
// T_{|j-k|}) / 2: mu_1 = B_1, mu_2k = 2 A_k - mu_0, mu_{2k-1} = 2 B_k - mu_1.
// Writes mu[m][v] for m < M (the layout of the direct moment loop).
template <typename T2>
__global__ void __launch_bounds__(kBlock) k_pair_moments(const T2* __restrict__ pairs, int M,
                                                         int V, T2* __restrict__ mu)
{
  const int t = blockIdx.x * kBlock + threadIdx.x;
  if (t >= M * V)
    return;
  const int m = t / V, v = t % V;
  const T2 mu0 = pairs[v];
  T2 r;
  if (m == 0) {
    r = mu0;
  } else if (m == 1) {
    r = pairs[(size_t)2 * V + 2 * v + 1];
  } else if ((m & 1) == 0) {
    const T2 a = pairs[(size_t)(m / 2) * 2 * V + 2 * v];
    r = make_double2(__dsub_rn(__dmul_rn(2.0, a.x), mu0.x), __dsub_rn(__dmul_rn(2.0, a.y), mu0.y));
  } else {
    const T2 mu1 = pairs[(size_t)2 * V + 2 * v + 1];
    const T2 b = pairs[(size_t)((m + 1) / 2) * 2 * V + 2 * v + 1];
    r = make_double2(__dsub_rn(__dmul_rn(2.0, b.x), mu1.x), __dsub_rn(__dmul_rn(2.0, b.y), mu1.y));
  }
  mu[t] = r;
}

// dst = src across storage forms (FP64 <-> FP32).
template <typename ST2, typename DT2>
__global__ void __launch_bounds__(kBlock) k_convert(size_t total, const ST2* __restrict__ src,
                                                    DT2* __restrict__ dst)
{
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
       g += (size_t)gridDim.x * kBlock)
    st(dst + g, ld(src + g));
}

// dst = src into FP32X storage (the FP32X moment loop's copies of its input vectors).
template <typename ST2>
__global__ void __launch_bounds__(kBlock) k_to_x(size_t total, const ST2* __restrict__ src,
                                                 xf2* __restrict__ dst, uintptr_t xlo)
{
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
       g += (size_t)gridDim.x * kBlock)
    st(dst + g, ld(src + g), xlo);
}

// FP64 accumulator -> FP32 state (end of an FP32-form evolution).
template <typename OT2>
__global__ void __launch_bounds__(kBlock) k_narrow(size_t total, const double2* __restrict__ in,
                                                   OT2* __restrict__ out)
{
  for (size_t g = (size_t)blockIdx.x * kBlock + threadIdx.x; g < total;
       g += (size_t)gridDim.x * kBlock)
    st(out + g, in[g]);
}

}  // namespace gqt
