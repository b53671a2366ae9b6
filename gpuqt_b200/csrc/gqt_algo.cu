// Operator and algorithm entry points of the C ABI: apply / commutator / current,
// the Chebyshev terms, the moment loop (find_moments_chebyshev), evolve, evolvex and
// the Jackson-damped Chebyshev summation. See include/gpuqt.h.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gqt_algo.h"
#include "gqt_forms.h"
#include "gqt_internal.h"
#include "gqt_wave.cuh"

namespace gqt {

Workspace::~Workspace()
{
  for (auto& kv : graphs)
    cudaGraphExecDestroy(kv.second);
  for (auto& kv : bufs)
    for (void* p : kv.second.v)
      cudaFree(p);
  cudaFree(acc);
  cudaFree(dot.partials);
  cudaFree(dot.counter);
  cudaFree(mu);
  cudaFreeHost(mu_host);
  cudaFree(pairs);
  cudaFree(xarena);
  cudaFree(wave_done);
  cudaFree(wave_ctl);
  if (ev_in)
    cudaEventDestroy(ev_in);
  if (ev_out)
    cudaEventDestroy(ev_out);
  if (capture_stream)
    cudaStreamDestroy(capture_stream);
}

Workspace* new_workspace() { return new Workspace(); }

gqt_status ws_vector(Workspace& ws, int precision, int nvec, size_t bytes, int i, void** out)
{
  auto& b = ws.bufs[{precision, nvec}];
  if (b.bytes != bytes) {
    cudaStreamSynchronize(stream());
    for (void* p : b.v)
      cudaFree(p);
    b.v.clear();
    b.bytes = bytes;
  }
  while ((int)b.v.size() <= i) {
    void* p = nullptr;
    GQT_CUDA(cudaMalloc(&p, bytes));
    b.v.push_back(p);
  }
  *out = b.v[i];
  return GQT_OK;
}

gqt_status ws_dot(Workspace& ws, size_t doubles, DotScratch** out)
{
  const size_t need = doubles > (size_t)max_grid() * 32 * 4 ? doubles : (size_t)max_grid() * 32 * 4;
  if ((size_t)ws.dot.blocks < need) {
    cudaStreamSynchronize(stream());
    // Graphs captured with the old buffer can never run again.
    for (auto& kv : ws.graphs)
      cudaGraphExecDestroy(kv.second);
    ws.graphs.clear();
    cudaFree(ws.dot.partials);
    ws.dot.partials = nullptr;
    ws.dot.blocks = 0;
    GQT_CUDA(cudaMalloc(&ws.dot.partials, need * sizeof(double)));
    ws.dot.blocks = (int)need;  // capacity in doubles
  }
  if (!ws.dot.counter) {
    GQT_CUDA(cudaMalloc(&ws.dot.counter, 2 * sizeof(unsigned)));
    GQT_CUDA(cudaMemset(ws.dot.counter, 0, 2 * sizeof(unsigned)));
  }
  *out = &ws.dot;
  return GQT_OK;
}

gqt_status ws_arena_x(Workspace& ws, size_t elems)
{
  // Slots start on 64-element boundaries, so every W-element access (W <= 4) of the
  // FP32 parts and of the residuals is aligned to its width.
  const size_t slot = (elems + 63) / 64 * 64;
  if (ws.xslot >= slot && ws.xarena)
    return GQT_OK;
  cudaStreamSynchronize(stream());
  // Graphs captured with the old arena can never run again.
  for (auto& kv : ws.graphs)
    cudaGraphExecDestroy(kv.second);
  ws.graphs.clear();
  cudaFree(ws.xarena);
  ws.xarena = nullptr;
  ws.xslot = 0;
  GQT_CUDA(cudaMalloc(&ws.xarena, (size_t)kXSlots * slot * 12));
  ws.xslot = slot;
  const uintptr_t base = reinterpret_cast<uintptr_t>(ws.xarena);  // 256-byte aligned
  const uintptr_t res = base + (uintptr_t)kXSlots * slot * 8;
  ws.xlo = res - base / 2;
  return GQT_OK;
}

// The slab of deferred block partials ([window][grid][results][4] doubles, after the
// immediate partials) stays within 32 MiB: 256 steps for one vector, 27 for 32, and
// 2-3 for realisation batches of hundreds of (realisation, vector) sums.
int defer_window(int results)
{
  const size_t per = (size_t)max_grid() * results * 4 * sizeof(double);
  const size_t w = ((size_t)32 << 20) / per;
  return (int)(w < 2 ? 2 : (w > 256 ? 256 : w));
}

namespace {

Op make_op(const gqt_ham* h, int nvec = 1)
{
  Op op{};
  if (h->use_codes) {
    op.code = h->code;
    op.code_delta = h->code_delta;
    op.code_hop = h->code_hop;
    op.code_xx = h->code_xx;
    op.n_codes = h->n_codes;
  }
  op.wpt = (nvec >= 0 && nvec <= 32) ? h->wpt[nvec] : 0;
  op.n = h->n;
  op.z = h->z;
  op.uniform = h->uniform;
  op.nn = h->nn;
  op.nl = h->nl;
  op.hop = h->hop;
  op.pot = h->pot;
  op.pot_r = h->pot_r;
  op.xx = h->xx;
  op.emax = h->energy_max;
  op.inv_emax = 1.0 / h->energy_max;
  op.lib_div = !(h->energy_max >= 0x1p-100 && h->energy_max <= 0x1p100);
  if (h->use_codes && h->n_real == 1 && h->stage_nw > 0 && h->stage_err) {
    op.stage_nw = h->stage_nw;
    op.stage_stages = h->stage_stages;
    for (int w = 0; w < h->stage_nw; ++w) {
      op.stage_lo[w] = h->stage_lo[w];
      op.stage_hi[w] = h->stage_hi[w];
    }
    op.stage_err = h->stage_err;
  } else if (h->use_codes && h->n_real > 1 && h->stage_rtab && h->stage_rnw > 0 &&
             h->stage_err) {
    // realisation batch: common slots, each model's windows in the device table
    op.stage_nw = h->stage_rnw;
    op.stage_stages = h->stage_stages;
    for (int w = 0; w < h->stage_rnw; ++w) {
      op.stage_lo[w] = 0;
      op.stage_hi[w] = h->stage_rwidth[w];
    }
    op.stage_err = h->stage_err;
    op.stage_rtab = h->stage_rtab;
  }
  return op;
}

gqt_status check_pair(const gqt_ham* h, const gqt_vec* a, const char* what)
{
  if (!h)
    return fail(GQT_ERR_ARG, "%s: null Hamiltonian", what);
  if (!a || !a->data)
    return fail(GQT_ERR_ARG, "%s: null vector", what);
  if (a->n != h->n)
    return fail(GQT_ERR_ARG, "%s: vector has %d sites, Hamiltonian %d", what, a->n, h->n);
  return GQT_OK;
}

gqt_status check_like(const gqt_vec* a, const gqt_vec* b, const char* what)
{
  if (!b || !b->data)
    return fail(GQT_ERR_ARG, "%s: null vector", what);
  if (a->n != b->n || a->nvec != b->nvec || a->precision != b->precision)
    return fail(GQT_ERR_ARG, "%s: vectors differ in size, count or precision", what);
  return GQT_OK;
}

const FormOps* ops_for(const gqt_vec* v, const char* what)
{
  const FormOps* f = form_ops(v->precision, v->nvec);
  if (!f)
    fail(GQT_ERR_ARG, "%s: unsupported vector form", what);
  return f;
}

gqt_status check_label(int label, const char* what)
{
  if (label < 1 || label > 4)
    return fail(GQT_ERR_ARG, "%s: label must be 1..4 (got %d)", what, label);
  return GQT_OK;
}

gqt_status need_fp64(const gqt_vec* v, const char* what)
{
  if (v->precision != GQT_FP64)
    return fail(GQT_ERR_ARG,
                "%s: single Chebyshev terms take FP64 vectors; use gqt_evolve/gqt_evolvex "
                "for the FP32 form",
                what);
  return GQT_OK;
}

// The label of term m of evolve (src/sigma.cu:136-145).
int evolve_label(int m, int direction)
{
  const int r = m % 4;
  if (r == 0)
    return 1;
  if (r == 2)
    return 2;
  if ((r == 1 && direction == 1) || (r == 3 && direction == -1))
    return 3;
  return 4;
}

// The label of term m of evolvex (src/sigma.cu:180-190).
int evolvex_label(int m, int direction)
{
  const int r = m % 4;
  if (r == 1)
    return 3;
  if (r == 3)
    return 4;
  if ((r == 0 && direction == 1) || (r == 2 && direction == -1))
    return 1;
  return 2;
}

// Moment launches whose grid stage is deferred (Dot::defer): the j-th step of a window
// writes its block partials to slab row j (rows start one immediate-partials stride into
// the scratch), and after `len` steps, or the last one, one k_slab_combine launch turns
// the window's rows into its moments. The outputs of consecutive moments are
// `results` double2 apart. A step then ends without the arrival counter and the
// last block's serial combination, which otherwise closes every launch.
struct Deferred {
  DotScratch* ds;
  int results;
  int len;
  size_t stride;  // doubles per row
  double2* first = nullptr;
  int used = 0;

  Deferred(DotScratch* d, int r)
      : ds(d), results(r), len(defer_window(r)), stride((size_t)max_grid() * r * 4)
  {
  }

  Dot next(double2* mu)
  {
    if (used == 0)
      first = mu;
    return Dot{ds->partials + (size_t)(1 + used++) * stride, ds->counter, mu, 1};
  }

  gqt_status flush(bool last)
  {
    if (used == 0 || (!last && used < len))
      return GQT_OK;
    const double* slab = ds->partials + stride;
    cudaStream_t s = stream();
    switch (results) {
      case 1:
        k_slab_combine<1><<<used, kBlock, 0, s>>>(slab, stride, ds->counter, first);
        break;
      case 2:
        k_slab_combine<2><<<used, kBlock, 0, s>>>(slab, stride, ds->counter, first);
        break;
      case 4:
        k_slab_combine<4><<<used, kBlock, 0, s>>>(slab, stride, ds->counter, first);
        break;
      case 8:
        k_slab_combine<8><<<used, kBlock, 0, s>>>(slab, stride, ds->counter, first);
        break;
      case 16:
        k_slab_combine<16><<<used, kBlock, 0, s>>>(slab, stride, ds->counter, first);
        break;
      case 32:
        k_slab_combine<32><<<used, kBlock, 0, s>>>(slab, stride, ds->counter, first);
        break;
      default:
        return fail(GQT_ERR_ARG, "deferred moments: %d sums per moment", results);
    }
    count_launches(1);
    GQT_CUDA(cudaGetLastError());
    used = 0;
    return GQT_OK;
  }
};

// The same deferral for realisation batches: the j-th kCheb step of a window writes its
// per-block slots to slab row j, and one k_tile_reduce launch over the window's rows
// turns them into moments (`results` = R x sums per realisation, consecutive moments
// `results` double2 apart). Rows are max_grid() x results x 4 doubles.
struct BatchDeferred {
  const FormOps* f;
  Op op;
  DotScratch* ds;
  int results;
  bool pair;
  int len;
  size_t stride;
  int blocks = 0;
  MultiDot first{};
  int used = 0;

  BatchDeferred(const FormOps* f_, const Op& op_, DotScratch* d, int r, bool p)
      : f(f_), op(op_), ds(d), results(r), pair(p), len(defer_window(r)),
        stride((size_t)max_grid() * r * 4)
  {
  }

  MultiDot next(const MultiDot& base, double2* mu)
  {
    MultiDot md = base;
    md.partials = ds->partials + (size_t)(1 + used) * stride;
    md.mu = mu;
    md.defer = 1;
    md.blocks_out = &blocks;
    if (used == 0)
      first = md;
    ++used;
    return md;
  }

  gqt_status flush(bool last)
  {
    if (used == 0 || (!last && used < len))
      return GQT_OK;
    MultiDot md = first;
    md.blocks = blocks;  // every kCheb step of the loop launches the same kernel
    GQT_TRY(f->tile_reduce(op, md, pair, used, stride));
    used = 0;
    return GQT_OK;
  }
};

// ------------------------------------------------------------------ wavefront loop

// Whether the wavefront loop applies to this moment loop (before planning).
bool wave_eligible(const gqt_ham* h, const gqt_vec* right, bool pair)
{
  return h->loop_window >= 2 && !pair && h->n_real == 1 && right->precision == GQT_FP64 &&
         right->nvec == 1 && h->use_codes && h->code &&
         (h->z == 3 || h->z == 4 || h->z == 6);
}

// The chunk plan of the coded operator (entries j = i + delta): for every chunk, the
// chunks its entries can reach, with each delta assumed at every site of the chunk
// (j is always a site, so a reach is clipped to [0, n)). The halo is the largest
// distance between a chunk and one it reaches, in positions of the identity order or
// of the folded one (0, C-1, 1, C-2, ...: a periodic boundary joins chunks 0 and C-1),
// whichever is smaller. Not applicable when the halo exceeds a quarter of the chunks.
gqt_status wave_plan(const gqt_ham* h)
{
  h->wave_halo = -2;
  const int n = h->n, cs = h->loop_chunk;
  const int C = (n + cs - 1) / cs;
  if (C < 16)
    return GQT_OK;
  std::vector<int> d(h->n_codes);
  GQT_CUDA(cudaMemcpy(d.data(), h->code_delta, d.size() * sizeof(int), cudaMemcpyDeviceToHost));
  std::sort(d.begin(), d.end());
  d.erase(std::unique(d.begin(), d.end()), d.end());
  int best = -1, best_fold = 0;
  std::vector<int> pos(C);
  for (int fold = 0; fold <= 1; ++fold) {
    WavePlan wp{C, cs, 0, 1, fold};
    for (int q = 0; q < C; ++q)
      pos[wave_chunk(wp, q)] = q;
    int K = 0;
    for (int c = 0; c < C; ++c) {
      const long long first = (long long)c * cs;
      const long long last = std::min<long long>(first + cs, n) - 1;
      for (int delta : d) {
        long long lo = first + delta, hi = last + delta;
        if (hi < 0 || lo > n - 1)
          continue;
        lo = std::max<long long>(lo, 0);
        hi = std::min<long long>(hi, n - 1);
        for (long long c2 = lo / cs; c2 <= hi / cs; ++c2)
          K = std::max(K, std::abs(pos[c2] - pos[c]));
      }
    }
    if (best < 0 || K < best) {
      best = K;
      best_fold = fold;
    }
  }
  if (best > C / 4)
    return GQT_OK;
  h->wave_chunks = C;
  h->wave_sites = cs;
  h->wave_halo = best;
  h->wave_fold = best_fold;
  return GQT_OK;
}

// Plan (once) and size the workspace of a wavefront loop; outside any capture.
gqt_status wave_prepare(const gqt_ham* h, Workspace& ws)
{
  if (h->wave_halo == -1)
    GQT_TRY(wave_plan(h));
  if (h->wave_halo < 0)
    return GQT_OK;
  if (ws.wave_done_n < h->wave_chunks) {
    cudaStreamSynchronize(stream());
    for (auto& kv : ws.graphs)
      cudaGraphExecDestroy(kv.second);
    ws.graphs.clear();
    cudaFree(ws.wave_done);
    ws.wave_done = nullptr;
    ws.wave_done_n = 0;
    GQT_CUDA(cudaMalloc(&ws.wave_done, (size_t)h->wave_chunks * sizeof(int)));
    ws.wave_done_n = h->wave_chunks;
  }
  if (!ws.wave_ctl) {
    GQT_CUDA(cudaMalloc(&ws.wave_ctl, 4 * sizeof(unsigned)));
    GQT_CUDA(cudaMemset(ws.wave_ctl, 0, 4 * sizeof(unsigned)));
  }
  return GQT_OK;
}

// Doubles of the dot scratch a wavefront loop of window S needs: the immediate
// partials, then S slab rows of chunks x warps partials.
size_t wave_scratch(const gqt_ham* h)
{
  return (size_t)max_grid() * 32 * 4 +
         (size_t)h->loop_window * h->wave_chunks * kWaveWarps * 4;
}

template <int Z>
gqt_status wave_windows(const gqt_ham* h, const Op& op, const gqt_vec* left,
                        const gqt_vec* right, int M, double2* mu, void* A, void* B,
                        DotScratch* ds, Workspace& ws)
{
  cudaStream_t s = stream();
  const int S = h->loop_window;
  const int G = grid_for((const void*)k_wave<Z>, (size_t)1 << 40);
  // lag: the halo plus about one round of the resident blocks' tickets, so an item's
  // dependencies were handed out a round earlier
  WavePlan wp{h->wave_chunks, h->wave_sites, h->wave_halo,
              h->wave_halo + (G + S - 1) / S + 2, h->wave_fold};
  WaveCtl* ctl = reinterpret_cast<WaveCtl*>(ws.wave_ctl);
  k_wave_init<<<(wp.chunks + kBlock - 1) / kBlock, kBlock, 0, s>>>(
    ws.wave_done, wp.chunks, ctl, ds->counter, (unsigned)(wp.chunks * kWaveWarps));
  count_launches(1);
  GQT_CUDA(cudaGetLastError());
  double* slab = ds->partials + (size_t)max_grid() * 32 * 4;
  const size_t row = (size_t)wp.chunks * kWaveWarps * 4;
  for (int s0 = 2; s0 < M; s0 += S) {
    const int steps = std::min(S, M - s0);
    k_wave<Z><<<G, kBlock, op_smem_bytes(op), s>>>(
      op, wp, s0, steps, (const double2*)right->data, (double2*)A, (double2*)B,
      (const double2*)left->data, ws.wave_done, ctl, slab);
    k_slab_combine<1><<<steps, kBlock, 0, s>>>(slab, row, ds->counter, mu + s0);
    count_launches(2);
    GQT_CUDA(cudaGetLastError());
  }
  return GQT_OK;
}

// The moment loop with steps 2 .. M-1 as wavefront windows (moments 0 and 1 as in the
// step loop).
gqt_status wave_launches(const gqt_ham* h, const FormOps* f, const gqt_vec* left,
                         const gqt_vec* right, int M, double2* mu, void* A, void* B,
                         DotScratch* ds)
{
  Op op = make_op(h, 1);
  Dot d{ds->partials, ds->counter, mu};
  GQT_TRY(f->dot((size_t)h->n, right->data, left->data, d));
  if (M < 2)
    return GQT_OK;
  d.mu = mu + 1;
  GQT_TRY(f->step(op, kApply, nullptr, right->data, A, left->data, &d));
  if (M < 3)
    return GQT_OK;
  Workspace& ws = *h->ws;
  switch (h->z) {
    case 3:
      return wave_windows<3>(h, op, left, right, M, mu, A, B, ds, ws);
    case 4:
      return wave_windows<4>(h, op, left, right, M, mu, A, B, ds, ws);
    default:
      return wave_windows<6>(h, op, left, right, M, mu, A, B, ds, ws);
  }
}

// The launch sequence of the moment loop (src/sigma.cu:33-61) on the current stream.
// Buffers: T_0 = right (read only), T_1 -> A, then T_m overwrites T_{m-2} in place.
gqt_status moment_launches(const gqt_ham* h, const FormOps* f, const gqt_vec* left,
                           const gqt_vec* right, int M, double2* mu, void* A, void* B,
                           DotScratch* ds)
{
  Op op = make_op(h, right->nvec);
  op.xlo = right->xlo;
  const int V = right->nvec;
  const size_t total = (size_t)h->n * V;
  if (h->n_real > 1) {
    // Realisation batch: the same sequence with per-realisation moments.
    const int RV = h->n_real * V;
    MultiDot md{ds->partials, mu, h->tile_first, h->n_tiles, h->tile_sites, h->n_real, 0};
    GQT_TRY(f->step_multi(op, kDotOnly, nullptr, right->data, nullptr, left->data, md));
    if (M < 2)
      return GQT_OK;
    md.mu = mu + RV;
    GQT_TRY(f->step_multi(op, kApply, nullptr, right->data, A, left->data, md));
    const void* prev = right->data;
    void* cur = A;
    BatchDeferred bd(f, op, ds, RV, false);
    for (int m = 2; m < M; ++m) {
      void* out = (prev == right->data) ? B : (void*)prev;
      GQT_TRY(f->step_multi(op, kCheb, prev, cur, out, left->data,
                            bd.next(md, mu + (size_t)m * RV)));
      GQT_TRY(bd.flush(m == M - 1));
      prev = cur;
      cur = out;
    }
    return GQT_OK;
  }
  if (wave_eligible(h, right, false) && h->wave_halo >= 0)
    return wave_launches(h, f, left, right, M, mu, A, B, ds);
  Dot d{ds->partials, ds->counter, mu, 0, right->xlo};
  GQT_TRY(f->dot(total, right->data, left->data, d));
  if (M < 2)
    return GQT_OK;
  d.mu = mu + V;
  GQT_TRY(f->step(op, kApply, nullptr, right->data, A, left->data, &d));
  const void* prev = right->data;  // T_{m-2}
  void* cur = A;                   // T_{m-1}
  Deferred df(ds, V);
  for (int m = 2; m < M; ++m) {
    void* out = (prev == right->data) ? B : (void*)prev;
    const Dot e = df.next(mu + (size_t)m * V);
    GQT_TRY(f->step(op, kCheb, prev, cur, out, left->data, &e));
    GQT_TRY(df.flush(m == M - 1));
    prev = cur;
    cur = out;
  }
  return GQT_OK;
}

// The symmetric moment set mu_m = <phi|T_m|phi>, m < M, from K = M / 2 steps: slot 0
// of `pairs` gets mu_0, slot k the pair <T_k|T_k>, <T_{k-1}|T_k> of step k, and
// k_pair_moments turns them into mu (layout [m][v]). The left stream of the direct
// loop is not read, and the recurrence runs half as many steps.
gqt_status moment_launches_pair(const gqt_ham* h, const FormOps* f, const gqt_vec* phi, int M,
                                double2* mu, double2* pairs, void* A, void* B, DotScratch* ds)
{
  Op op = make_op(h, phi->nvec);
  op.xlo = phi->xlo;
  const int V = phi->nvec;
  const size_t total = (size_t)h->n * V;
  if (h->n_real > 1) {
    // Realisation batch: slot 0 holds mu_0 per (realisation, vector), slot k the pairs
    // [r][2v + t]; k_pair_moments then runs over R * V flattened moments.
    const int RV = h->n_real * V;
    MultiDot md{ds->partials, pairs, h->tile_first, h->n_tiles, h->tile_sites, h->n_real, 0};
    GQT_TRY(f->step_multi(op, kDotOnly, nullptr, phi->data, nullptr, phi->data, md));
    const int K = M / 2;
    if (K >= 1) {
      md.mu = pairs + (size_t)2 * RV;
      GQT_TRY(f->step_multi(op, kApply, nullptr, phi->data, A, nullptr, md, kDotPair));
      const void* prev = phi->data;
      void* cur = A;
      BatchDeferred bd(f, op, ds, 2 * RV, true);
      for (int k = 2; k <= K; ++k) {
        void* out = (prev == phi->data) ? B : (void*)prev;
        GQT_TRY(f->step_multi(op, kCheb, prev, cur, out, nullptr,
                              bd.next(md, pairs + (size_t)k * 2 * RV), kDotPair));
        GQT_TRY(bd.flush(k == K));
        prev = cur;
        cur = out;
      }
    }
    const int n = M * RV;
    k_pair_moments<double2><<<(n + kBlock - 1) / kBlock, kBlock, 0, stream()>>>(pairs, M, RV, mu);
    count_launches(1);
    GQT_CUDA(cudaGetLastError());
    return GQT_OK;
  }
  Dot d{ds->partials, ds->counter, pairs, 0, phi->xlo};
  GQT_TRY(f->dot(total, phi->data, phi->data, d));
  const int K = M / 2;
  if (K >= 1) {
    d.mu = pairs + (size_t)2 * V;
    GQT_TRY(f->step_pair(op, kApply, nullptr, phi->data, A, d));
    const void* prev = phi->data;
    void* cur = A;
    Deferred df(ds, 2 * V);
    for (int k = 2; k <= K; ++k) {
      void* out = (prev == phi->data) ? B : (void*)prev;
      const Dot e = df.next(pairs + (size_t)k * 2 * V);
      GQT_TRY(f->step_pair(op, kCheb, prev, cur, out, e));
      GQT_TRY(df.flush(k == K));
      prev = cur;
      cur = out;
    }
  }
  const int n = M * V;
  k_pair_moments<double2><<<(n + kBlock - 1) / kBlock, kBlock, 0, stream()>>>(pairs, M, V, mu);
  count_launches(1);
  GQT_CUDA(cudaGetLastError());
  return GQT_OK;
}

}  // namespace

}  // namespace gqt

using namespace gqt;

// ------------------------------------------------------------------ operators
extern "C" gqt_status gqt_apply(const gqt_ham* h, const gqt_vec* in, gqt_vec* out)
{
  GQT_TRY(check_pair(h, in, "gqt_apply"));
  GQT_TRY(check_like(in, out, "gqt_apply"));
  if (in->data == out->data)
    return fail(GQT_ERR_ARG, "gqt_apply: input and output must differ");
  const FormOps* f = ops_for(in, "gqt_apply");
  if (!f)
    return GQT_ERR_ARG;
  return f->step(make_op(h, in->nvec), kApply, nullptr, in->data, out->data, nullptr, nullptr);
}

static gqt_status xop_entry(const gqt_ham* h, const gqt_vec* in, gqt_vec* out, bool current,
                            const char* what)
{
  GQT_TRY(check_pair(h, in, what));
  GQT_TRY(check_like(in, out, what));
  if (in->data == out->data)
    return fail(GQT_ERR_ARG, "%s: input and output must differ", what);
  if (!h->has_xx)
    return fail(GQT_ERR_STATE, "%s: the Hamiltonian was created without xx", what);
  if (h->n_real > 1)
    return fail(GQT_ERR_STATE, "%s: not defined on a realisation batch", what);
  const FormOps* f = ops_for(in, what);
  if (!f)
    return GQT_ERR_ARG;
  return f->xop(make_op(h), current, in->data, out->data);
}

extern "C" gqt_status gqt_apply_commutator(const gqt_ham* h, const gqt_vec* in, gqt_vec* out)
{
  return xop_entry(h, in, out, false, "gqt_apply_commutator");
}

extern "C" gqt_status gqt_apply_current(const gqt_ham* h, const gqt_vec* in, gqt_vec* out)
{
  return xop_entry(h, in, out, true, "gqt_apply_current");
}

extern "C" gqt_status gqt_kernel_polynomial(const gqt_ham* h, const gqt_vec* s0,
                                            const gqt_vec* s1, gqt_vec* s2)
{
  GQT_TRY(check_pair(h, s1, "gqt_kernel_polynomial"));
  GQT_TRY(check_like(s1, s0, "gqt_kernel_polynomial"));
  GQT_TRY(check_like(s1, s2, "gqt_kernel_polynomial"));
  if (s2->data == s1->data)
    return fail(GQT_ERR_ARG, "gqt_kernel_polynomial: s2 must not alias s1");
  const FormOps* f = ops_for(s1, "gqt_kernel_polynomial");
  if (!f)
    return GQT_ERR_ARG;
  return f->step(make_op(h, s1->nvec), kCheb, s0->data, s1->data, s2->data, nullptr, nullptr);
}

extern "C" gqt_status gqt_chebyshev_01(const gqt_ham* h, const gqt_vec* s0, const gqt_vec* s1,
                                       gqt_vec* out, double b0, double b1, int direction)
{
  GQT_TRY(check_pair(h, s0, "gqt_chebyshev_01"));
  GQT_TRY(check_like(s0, s1, "gqt_chebyshev_01"));
  GQT_TRY(check_like(s0, out, "gqt_chebyshev_01"));
  GQT_TRY(need_fp64(s0, "gqt_chebyshev_01"));
  const FormOps* f = ops_for(s0, "gqt_chebyshev_01");
  if (!f)
    return GQT_ERR_ARG;
  return f->cheb01((size_t)s0->n * s0->nvec, s0->data, s1->data, (double2*)out->data, b0,
                   b1 * direction);
}

extern "C" gqt_status gqt_chebyshev_2(const gqt_ham* h, const gqt_vec* s0, const gqt_vec* s1,
                                      gqt_vec* s2, gqt_vec* out, double bessel, int label)
{
  GQT_TRY(check_pair(h, s1, "gqt_chebyshev_2"));
  GQT_TRY(check_like(s1, s0, "gqt_chebyshev_2"));
  GQT_TRY(check_like(s1, s2, "gqt_chebyshev_2"));
  GQT_TRY(check_like(s1, out, "gqt_chebyshev_2"));
  GQT_TRY(need_fp64(s1, "gqt_chebyshev_2"));
  GQT_TRY(check_label(label, "gqt_chebyshev_2"));
  if (s2->data == s1->data || out->data == s1->data || out->data == s2->data)
    return fail(GQT_ERR_ARG, "gqt_chebyshev_2: s2/out must not alias s1 or each other");
  const FormOps* f = ops_for(s1, "gqt_chebyshev_2");
  if (!f)
    return GQT_ERR_ARG;
  return f->cheb2(make_op(h), s0->data, s1->data, s2->data, (double2*)out->data, bessel,
                  label);
}

extern "C" gqt_status gqt_chebyshev_1x(const gqt_ham* h, const gqt_vec* in, gqt_vec* out,
                                       double b1)
{
  GQT_TRY(check_pair(h, in, "gqt_chebyshev_1x"));
  GQT_TRY(check_like(in, out, "gqt_chebyshev_1x"));
  GQT_TRY(need_fp64(in, "gqt_chebyshev_1x"));
  const FormOps* f = ops_for(in, "gqt_chebyshev_1x");
  if (!f)
    return GQT_ERR_ARG;
  return f->cheb1x((size_t)in->n * in->nvec, in->data, (double2*)out->data, b1);
}

extern "C" gqt_status gqt_chebyshev_2x(const gqt_ham* h, const gqt_vec* s0, const gqt_vec* s0x,
                                       const gqt_vec* s1, const gqt_vec* s1x, gqt_vec* s2,
                                       gqt_vec* s2x, gqt_vec* out, double bessel, int label)
{
  const char* w = "gqt_chebyshev_2x";
  GQT_TRY(check_pair(h, s1, w));
  for (const gqt_vec* v : {s0, s0x, s1x, (const gqt_vec*)s2, (const gqt_vec*)s2x,
                           (const gqt_vec*)out})
    GQT_TRY(check_like(s1, v, w));
  GQT_TRY(need_fp64(s1, w));
  GQT_TRY(check_label(label, w));
  const void* gathered[2] = {s1->data, s1x->data};
  for (const void* g : gathered)
    if (s2->data == g || s2x->data == g || out->data == g)
      return fail(GQT_ERR_ARG, "%s: outputs must not alias s1 or s1x", w);
  const FormOps* f = ops_for(s1, w);
  if (!f)
    return GQT_ERR_ARG;
  return f->cheb2x(make_op(h), s0->data, s0x->data, s1->data, s1x->data, s2->data, s2x->data,
                   (double2*)out->data, bessel, label);
}

// ------------------------------------------------------------------ reductions
namespace {
thread_local std::map<int, DotScratch> t_dot;  // per device, for Hamiltonian-free dots
thread_local std::map<int, double2*> t_mu;
}  // namespace

extern "C" gqt_status gqt_inner_product(const gqt_vec* state, const gqt_vec* left, double* re,
                                        double* im)
{
  if (!state || !state->data)
    return fail(GQT_ERR_ARG, "gqt_inner_product: null vector");
  GQT_TRY(check_like(state, left, "gqt_inner_product"));
  if (!re || !im)
    return fail(GQT_ERR_ARG, "gqt_inner_product: null output");
  const FormOps* f = ops_for(state, "gqt_inner_product");
  if (!f)
    return GQT_ERR_ARG;
  int dev = 0;
  cudaGetDevice(&dev);
  DotScratch& ds = t_dot[dev];
  double2*& mu = t_mu[dev];
  if (!ds.partials) {
    GQT_CUDA(cudaMalloc(&ds.partials, (size_t)max_grid() * 32 * 4 * sizeof(double)));
    GQT_CUDA(cudaMalloc(&ds.counter, sizeof(unsigned)));
    GQT_CUDA(cudaMemset(ds.counter, 0, sizeof(unsigned)));
    GQT_CUDA(cudaMalloc(&mu, 32 * sizeof(double2)));
  }
  Dot d{ds.partials, ds.counter, mu};
  GQT_TRY(f->dot((size_t)state->n * state->nvec, state->data, left->data, d));
  std::vector<double2> h(state->nvec);
  GQT_CUDA(cudaMemcpyAsync(h.data(), mu, sizeof(double2) * state->nvec, cudaMemcpyDeviceToHost,
                           stream()));
  GQT_CUDA(cudaStreamSynchronize(stream()));
  for (int k = 0; k < state->nvec; ++k) {
    re[k] = h[k].x;
    im[k] = h[k].y;
  }
  return GQT_OK;
}

static DotScratch* thread_dot()
{
  int dev = 0;
  cudaGetDevice(&dev);
  DotScratch& ds = t_dot[dev];
  if (!ds.partials) {
    if (cudaMalloc(&ds.partials, (size_t)max_grid() * 32 * 4 * sizeof(double)) != cudaSuccess)
      return nullptr;
    if (cudaMalloc(&ds.counter, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(ds.counter, 0, sizeof(unsigned)) != cudaSuccess)
      return nullptr;
  }
  return &ds;
}

extern "C" gqt_status gqt_inner_product_into(const gqt_vec* state, const gqt_vec* left,
                                             gqt_vec* target, int index)
{
  const char* w = "gqt_inner_product_into";
  if (!state || !state->data || !target || !target->data)
    return fail(GQT_ERR_ARG, "%s: null vector", w);
  GQT_TRY(check_like(state, left, w));
  if (state->nvec != 1 || target->nvec != 1 || target->precision != GQT_FP64)
    return fail(GQT_ERR_ARG, "%s: needs single vectors and an FP64 target", w);
  if (index < 0 || index >= target->n)
    return fail(GQT_ERR_ARG, "%s: index %d outside the target (%d)", w, index, target->n);
  const FormOps* f = ops_for(state, w);
  if (!f)
    return GQT_ERR_ARG;
  DotScratch* ds = thread_dot();
  if (!ds)
    return fail(GQT_ERR_ALLOC, "%s: scratch allocation failed", w);
  Dot d{ds->partials, ds->counter, (double2*)target->data + index};
  return f->dot((size_t)state->n, state->data, left->data, d);
}

extern "C" gqt_status gqt_vec_segment_sum(const gqt_vec* in, int segment, int count,
                                          gqt_vec* out)
{
  const char* w = "gqt_vec_segment_sum";
  if (!in || !in->data || !out || !out->data)
    return fail(GQT_ERR_ARG, "%s: null vector", w);
  if (in->precision != GQT_FP64 || out->precision != GQT_FP64 || in->nvec != 1 ||
      out->nvec != 1)
    return fail(GQT_ERR_ARG, "%s: needs single FP64 vectors", w);
  if (segment <= 0 || count <= 0 || (size_t)segment * count > (size_t)in->n || count > out->n)
    return fail(GQT_ERR_ARG, "%s: segment %d x count %d does not fit", w, segment, count);
  k_segment_sum<0><<<count, kBlock, 0, stream()>>>((const double2*)in->data, segment,
                                                   (double2*)out->data);
  count_launches(1);
  GQT_CUDA(cudaGetLastError());
  return GQT_OK;
}

// ------------------------------------------------------------------ moments
static gqt_status moments_prepare(const gqt_ham* h, const gqt_vec* left, const gqt_vec* right,
                                  int M, const FormOps** f, void** A, void** B,
                                  DotScratch** ds)
{
  const char* w = "gqt_moments";
  GQT_TRY(check_pair(h, right, w));
  GQT_TRY(check_like(right, left, w));
  if (M < 1)
    return fail(GQT_ERR_ARG, "%s: number of moments must be > 0 (got %d)", w, M);
  *f = ops_for(right, w);
  if (!*f)
    return GQT_ERR_ARG;
  Workspace& ws = *h->ws;
  if (right->precision == GQT_FP32X) {
    // the recurrence's two buffers share the inputs' arena (one residual map)
    *A = ws_xslot(ws, 2);
    *B = ws_xslot(ws, 3);
  } else {
    const size_t bytes = right->bytes;
    GQT_TRY(ws_vector(ws, right->precision, right->nvec, bytes, 0, A));
    GQT_TRY(ws_vector(ws, right->precision, right->nvec, bytes, 1, B));
  }
  // Block partials: [grid][R][V][4] doubles for a batch, [grid][V][4] otherwise, followed
  // by the slab of a window of deferred moments.
  const int results = h->n_real * right->nvec;
  const size_t rows = 1 + (size_t)defer_window(results);
  GQT_TRY(ws_dot(ws, rows * max_grid() * results * 4, ds));
  return GQT_OK;
}

// The moment loop (direct, or the symmetric pair loop) as one CUDA graph launch.
static gqt_status moments_run(const gqt_ham* h, const gqt_vec* left, const gqt_vec* right,
                              int M, void* mu_dev, bool pair, const char* w)
{
  const FormOps* f;
  void *A, *B;
  DotScratch* ds;
  GQT_TRY(moments_prepare(h, left, right, M, &f, &A, &B, &ds));
  if (!mu_dev)
    return fail(GQT_ERR_ARG, "%s: null output", w);
  Workspace& ws = *h->ws;
  if (right->precision == GQT_FP32R)
    GQT_TRY(ensure_pot_r(h));  // before any capture: it allocates
  if (wave_eligible(h, right, pair)) {
    GQT_TRY(wave_prepare(h, ws));
    if (h->wave_halo >= 0)
      GQT_TRY(ws_dot(ws, wave_scratch(h), &ds));
  }
  cudaStream_t s = stream();
  if (pair) {
    if (!h->hermitian)
      return fail(GQT_ERR_STATE,
                  "%s: the operator is not Hermitian (the doubling identity needs H = H^+)", w);
    if (h->n_real == 1 && right->nvec > 16)
      return fail(GQT_ERR_ARG, "%s: at most 16 vectors (got %d)", w, right->nvec);
    // Pair sums: twice the block partials of the direct loop (and of its slab).
    const int results = 2 * h->n_real * right->nvec;
    const size_t rows = 1 + (size_t)defer_window(results);
    GQT_TRY(ws_dot(ws, rows * max_grid() * results * 4, &ds));
    const size_t need = (size_t)(M / 2 + 1) * 2 * h->n_real * right->nvec * sizeof(double2);
    if (ws.pairs_bytes < need) {
      cudaStreamSynchronize(s);
      cudaFree(ws.pairs);
      ws.pairs = nullptr;
      ws.pairs_bytes = 0;
      GQT_CUDA(cudaMalloc(&ws.pairs, need));
      ws.pairs_bytes = need;
      // Graphs captured with the old buffer can never run again.
      for (auto& kv : ws.graphs)
        cudaGraphExecDestroy(kv.second);
      ws.graphs.clear();
    }
  }

  // The n_moments launches are captured once per (left, right, M, output, form) and
  // replayed as one graph launch afterwards.
  Workspace::GraphKey key{left->data, right->data,      M, mu_dev,
                          right->precision, right->nvec, pair ? 1 : 0};
  auto it = ws.graphs.find(key);
  if (it == ws.graphs.end()) {
    if (!ws.capture_stream) {
      GQT_CUDA(cudaStreamCreateWithFlags(&ws.capture_stream, cudaStreamNonBlocking));
      GQT_CUDA(cudaEventCreateWithFlags(&ws.ev_in, cudaEventDisableTiming));
      GQT_CUDA(cudaEventCreateWithFlags(&ws.ev_out, cudaEventDisableTiming));
    }
    cudaStream_t saved = s;
    gqt_set_stream(ws.capture_stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(ws.capture_stream, cudaStreamCaptureModeThreadLocal);
    gqt_status st = GQT_OK;
    if (e == cudaSuccess) {
      const uint64_t before = gqt_launch_count();
      st = pair ? moment_launches_pair(h, f, right, M, (double2*)mu_dev, ws.pairs, A, B, ds)
                : moment_launches(h, f, left, right, M, (double2*)mu_dev, A, B, ds);
      // Captured launches run later, when the graph is launched.
      ws.graph_launches[key] = gqt_launch_count() - before;
      gqt_reset_launch_count();
      count_launches(before);
      e = cudaStreamEndCapture(ws.capture_stream, &g);
    }
    gqt_set_stream(saved);
    if (st != GQT_OK) {
      if (g)
        cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess)
      return cuda_fail(e, "stream capture of the moment loop", __FILE__, __LINE__);
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
      return cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__);
    it = ws.graphs.emplace(key, exec).first;
  }
  // The graph runs on the workspace's own stream, ordered after and before the
  // caller's stream by events (the legacy default stream cannot launch graphs
  // directly into a capture-compatible order).
  GQT_CUDA(cudaEventRecord(ws.ev_in, s));
  GQT_CUDA(cudaStreamWaitEvent(ws.capture_stream, ws.ev_in, 0));
  GQT_CUDA(cudaGraphLaunch(it->second, ws.capture_stream));
  count_launches(ws.graph_launches[key]);
  GQT_CUDA(cudaEventRecord(ws.ev_out, ws.capture_stream));
  GQT_CUDA(cudaStreamWaitEvent(s, ws.ev_out, 0));
  return GQT_OK;
}

extern "C" gqt_status gqt_moments_device(const gqt_ham* h, const gqt_vec* left,
                                         const gqt_vec* right, int M, void* mu_dev)
{
  return moments_run(h, left, right, M, mu_dev, false, "gqt_moments_device");
}

static gqt_status convert_data(int n, int nvec, int from, const void* src, int to, void* dst)
{
  const size_t total = (size_t)n * nvec;
  if (from == to) {
    const size_t elem = from == GQT_FP64 ? sizeof(double2) : sizeof(float2);
    if (src != dst)
      GQT_CUDA(cudaMemcpyAsync(dst, src, total * elem, cudaMemcpyDeviceToDevice, stream()));
    return GQT_OK;
  }
  const int grid = from == GQT_FP64 ? grid_for((const void*)k_convert<double2, float2>, total)
                                    : grid_for((const void*)k_convert<float2, double2>, total);
  if (from == GQT_FP64)
    k_convert<double2, float2><<<grid, kBlock, 0, stream()>>>(total, (const double2*)src,
                                                              (float2*)dst);
  else
    k_convert<float2, double2><<<grid, kBlock, 0, stream()>>>(total, (const float2*)src,
                                                              (double2*)dst);
  count_launches(1);
  GQT_CUDA(cudaGetLastError());
  return GQT_OK;
}

extern "C" gqt_status gqt_vec_convert(gqt_vec* dst, const gqt_vec* src)
{
  if (!dst || !src || !dst->data || !src->data)
    return fail(GQT_ERR_ARG, "gqt_vec_convert: null vector");
  if (dst->n != src->n || dst->nvec != src->nvec)
    return fail(GQT_ERR_ARG, "gqt_vec_convert: vectors differ in size or count");
  return convert_data(src->n, src->nvec, src->precision, src->data, dst->precision, dst->data);
}

// moments_run in another arithmetic form than the vectors' (converted copies).
static gqt_status moments_form_run(const gqt_ham* h, const gqt_vec* left, const gqt_vec* right,
                                   int M, int precision, void* mu_dev, bool pair,
                                   const char* w)
{
  if (!h || !left || !right || !left->data || !right->data)
    return fail(GQT_ERR_ARG, "%s: null argument", w);
  if (precision == right->precision && precision == left->precision)
    return moments_run(h, left, right, M, mu_dev, pair, w);
  if (!form_ops(precision, right->nvec))
    return fail(GQT_ERR_ARG, "%s: form %d has no %d-vector launch", w, precision, right->nvec);
  if (left->n != right->n || left->nvec != right->nvec)
    return fail(GQT_ERR_ARG, "%s: left and right differ in size or count", w);
  if (precision == GQT_FP32X) {
    // Copies of left and right in the FP32X arena (slots 1 and 0); the recurrence runs
    // in slots 2 and 3.
    if (h->n_real > 1)
      return fail(GQT_ERR_STATE, "%s: the FP32X form runs on one model, not a batch", w);
    if (right->precision == GQT_FP32X || left->precision == GQT_FP32X)
      return fail(GQT_ERR_ARG, "%s: FP32X vectors are internal to the moment loop", w);
    GQT_TRY(check_pair(h, right, w));
    Workspace& ws = *h->ws;
    const size_t elems = (size_t)right->n * right->nvec;
    GQT_TRY(ws_arena_x(ws, elems));
    const bool same = left->data == right->data;
    GQT_TRY(convert_to_x(elems, right->precision, right->data, ws_xslot(ws, 0), ws.xlo));
    if (!same)
      GQT_TRY(convert_to_x(elems, left->precision, left->data, ws_xslot(ws, 1), ws.xlo));
    gqt_vec R = *right, L = *left;
    R.precision = L.precision = GQT_FP32X;
    R.bytes = L.bytes = elems * 8;
    R.xlo = L.xlo = ws.xlo;
    R.data = ws_xslot(ws, 0);
    L.data = same ? R.data : ws_xslot(ws, 1);
    return moments_run(h, &L, &R, M, mu_dev, pair, w);
  }
  // GQT_FP32R stores its vectors as GQT_FP32 does: FP32 vectors run as they are.
  const int store = precision == GQT_FP32R ? GQT_FP32 : precision;
  if (precision == GQT_FP32R) {
    if (right->precision == GQT_FP32X || left->precision == GQT_FP32X ||
        right->precision == GQT_FP32R || left->precision == GQT_FP32R)
      return fail(GQT_ERR_ARG, "%s: the FP32R form reads FP32 or FP64 vectors", w);
    if (right->precision == GQT_FP32 && left->precision == GQT_FP32) {
      gqt_vec R = *right, L = *left;
      R.precision = L.precision = GQT_FP32R;
      return moments_run(h, &L, &R, M, mu_dev, pair, w);
    }
  }
  // The converted copies live in workspace slots 4 and 5 of the target form (slots
  // 0-3 are the recurrence and evolution temporaries).
  Workspace& ws = *h->ws;
  const size_t bytes = (size_t)right->n * right->nvec *
                       (store == GQT_FP64 ? sizeof(double2) : sizeof(float2));
  void *lc = nullptr, *rc = nullptr;
  GQT_TRY(ws_vector(ws, store, right->nvec, bytes, 5, &rc));
  GQT_TRY(ws_vector(ws, store, right->nvec, bytes, 4, &lc));
  GQT_TRY(convert_data(right->n, right->nvec, right->precision, right->data, store, rc));
  const bool same = left->data == right->data;
  if (!same)
    GQT_TRY(convert_data(left->n, left->nvec, left->precision, left->data, store, lc));
  gqt_vec R = *right, L = *left;
  R.precision = L.precision = precision;
  R.bytes = L.bytes = bytes;
  R.data = rc;
  L.data = same ? rc : lc;
  return moments_run(h, &L, &R, M, mu_dev, pair, w);
}

extern "C" gqt_status gqt_moments_device_form(const gqt_ham* h, const gqt_vec* left,
                                              const gqt_vec* right, int M, int precision,
                                              void* mu_dev)
{
  return moments_form_run(h, left, right, M, precision, mu_dev, false,
                          "gqt_moments_device_form");
}

extern "C" gqt_status gqt_moments_doubled_device(const gqt_ham* h, const gqt_vec* state, int M,
                                                 int precision, void* mu_dev)
{
  return moments_form_run(h, state, state, M, precision, mu_dev, true,
                          "gqt_moments_doubled_device");
}

extern "C" gqt_status gqt_moments(const gqt_ham* h, const gqt_vec* left, const gqt_vec* right,
                                  int M, double* mu_re, double* mu_im)
{
  if (!right)
    return fail(GQT_ERR_ARG, "gqt_moments: null vector");
  return gqt_moments_form(h, left, right, M, right->precision, mu_re, mu_im);
}

// A moment loop into the workspace's device buffer, then to host arrays [vector][m].
static gqt_status moments_host(const gqt_ham* h, const gqt_vec* left, const gqt_vec* right,
                               int M, int precision, bool pair, double* mu_re, double* mu_im,
                               const char* w)
{
  if (!mu_re || !mu_im)
    return fail(GQT_ERR_ARG, "%s: null output", w);
  if (!h)
    return fail(GQT_ERR_ARG, "%s: null Hamiltonian", w);
  if (!right)
    return fail(GQT_ERR_ARG, "%s: null vector", w);
  if (M < 1)
    return fail(GQT_ERR_ARG, "%s: number of moments must be > 0 (got %d)", w, M);
  Workspace& ws = *h->ws;
  const int V = right->nvec * h->n_real;  // results per moment: [r][vector]
  const size_t need = (size_t)M * V * sizeof(double2);
  if (ws.mu_bytes < need) {
    cudaStreamSynchronize(stream());
    cudaFree(ws.mu);
    ws.mu = nullptr;
    ws.mu_bytes = 0;
    GQT_CUDA(cudaMalloc(&ws.mu, need));
    ws.mu_bytes = need;
    // Graphs keyed on the old buffer can never match again; drop them.
    for (auto& kv : ws.graphs)
      cudaGraphExecDestroy(kv.second);
    ws.graphs.clear();
  }
  // The moments come back through a pinned buffer (a plain DMA), not the driver's
  // staging path for pageable memory.
  if (ws.mu_host_bytes < need) {
    cudaFreeHost(ws.mu_host);
    ws.mu_host = nullptr;
    ws.mu_host_bytes = 0;
    GQT_CUDA(cudaMallocHost(&ws.mu_host, need));
    ws.mu_host_bytes = need;
  }
  GQT_TRY(moments_form_run(h, left, right, M, precision, ws.mu, pair, w));
  const double2* host = ws.mu_host;
  GQT_CUDA(cudaMemcpyAsync(ws.mu_host, ws.mu, need, cudaMemcpyDeviceToHost, stream()));
  GQT_CUDA(cudaStreamSynchronize(stream()));
  if (ws.wave_ctl) {
    // a wavefront loop whose bounded wait ran out flagged it (never expected: every
    // wait is on an earlier ticket)
    unsigned err = 0;
    GQT_CUDA(cudaMemcpy(&err, ws.wave_ctl + 2, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (err) {
      GQT_CUDA(cudaMemset(ws.wave_ctl + 2, 0, sizeof(unsigned)));
      return fail(GQT_ERR_STATE, "%s: a wait of the wavefront loop timed out; moments invalid",
                  w);
    }
  }
  if (h->stage_err) {
    // a staged step whose bounded wait for its shared-memory copies ran out flagged it
    unsigned err = 0;
    GQT_CUDA(cudaMemcpy(&err, h->stage_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (err) {
      GQT_CUDA(cudaMemset(h->stage_err, 0, sizeof(unsigned)));
      return fail(GQT_ERR_STATE, "%s: a wait of the staged step timed out; moments invalid", w);
    }
  }
  for (int k = 0; k < V; ++k)
    for (int m = 0; m < M; ++m) {
      mu_re[(size_t)k * M + m] = host[(size_t)m * V + k].x;
      mu_im[(size_t)k * M + m] = host[(size_t)m * V + k].y;
    }
  return GQT_OK;
}

extern "C" gqt_status gqt_moments_form(const gqt_ham* h, const gqt_vec* left,
                                       const gqt_vec* right, int M, int precision,
                                       double* mu_re, double* mu_im)
{
  return moments_host(h, left, right, M, precision, false, mu_re, mu_im, "gqt_moments");
}

extern "C" gqt_status gqt_moments_doubled(const gqt_ham* h, const gqt_vec* state, int M,
                                          int precision, double* mu_re, double* mu_im)
{
  return moments_host(h, state, state, M, precision, true, mu_re, mu_im, "gqt_moments_doubled");
}

// ------------------------------------------------------------------ time evolution
static gqt_status evolve_common(const gqt_ham* h, int direction, double dt, gqt_vec* state,
                                bool commutator)
{
  const char* w = commutator ? "gqt_evolvex" : "gqt_evolve";
  GQT_TRY(check_pair(h, state, w));
  if (direction != 1 && direction != -1)
    return fail(GQT_ERR_ARG, "%s: direction must be +1 or -1 (got %d)", w, direction);
  if (commutator && !h->has_xx)
    return fail(GQT_ERR_STATE, "%s: the Hamiltonian was created without xx", w);
  if (h->n_real > 1)
    return fail(GQT_ERR_STATE, "%s: a realisation batch has one time scale per model", w);
  const FormOps* f = ops_for(state, w);
  if (!f)
    return GQT_ERR_ARG;
  Workspace& ws = *h->ws;
  const Op op = make_op(h);
  const size_t total = (size_t)state->n * state->nvec;
  const size_t bytes = state->bytes;
  void *s0, *s1, *s0x = nullptr, *s1x = nullptr;
  GQT_TRY(ws_vector(ws, state->precision, state->nvec, bytes, 0, &s0));
  GQT_TRY(ws_vector(ws, state->precision, state->nvec, bytes, 1, &s1));
  if (commutator) {
    GQT_TRY(ws_vector(ws, state->precision, state->nvec, bytes, 2, &s0x));
    GQT_TRY(ws_vector(ws, state->precision, state->nvec, bytes, 3, &s1x));
  }
  // The FP64 form accumulates straight into the state; the FP32 form into an FP64
  // accumulator that is rounded to the state once at the end.
  double2* out = (double2*)state->data;
  if (state->precision != GQT_FP64) {
    const size_t need = total * sizeof(double2);
    if (ws.acc_bytes < need) {
      cudaStreamSynchronize(stream());
      cudaFree(ws.acc);
      ws.acc = nullptr;
      ws.acc_bytes = 0;
      GQT_CUDA(cudaMalloc(&ws.acc, need));
      ws.acc_bytes = need;
    }
    out = ws.acc;
  }
  cudaStream_t s = stream();
  GQT_CUDA(cudaMemcpyAsync(s0, state->data, bytes, cudaMemcpyDeviceToDevice, s));
  GQT_TRY(f->step(op, kApply, nullptr, state->data, s1, nullptr, nullptr));
  if (!commutator) {
    const double b0 = j0(dt);
    const double b1 = 2.0 * j1(dt);
    GQT_TRY(f->cheb01(total, s0, s1, out, b0, b1 * direction));
    for (int m = 2; m < 1000000; ++m) {
      double bm = jn(m, dt);
      if (bm < 1.0e-15 && bm > -1.0e-15)
        break;
      bm *= 2.0;
      GQT_TRY(f->cheb2(op, s0, s1, s0, out, bm, evolve_label(m, direction)));
      std::swap(s0, s1);
    }
  } else {
    GQT_CUDA(cudaMemsetAsync(s0x, 0, bytes, s));
    GQT_TRY(f->xop(op, false, state->data, s1x));
    const double b1 = 2.0 * j1(dt);
    GQT_TRY(f->cheb1x(total, s1x, out, b1));
    for (int m = 2; m <= 1000000; ++m) {
      double bm = jn(m, dt);
      if (bm < 1.0e-15 && bm > -1.0e-15)
        break;
      bm *= 2.0;
      GQT_TRY(f->cheb2x(op, s0, s0x, s1, s1x, s0, s0x, out, bm, evolvex_label(m, direction)));
      std::swap(s0, s1);
      std::swap(s0x, s1x);
    }
  }
  if (state->precision != GQT_FP64) {
    const int grid = grid_for((const void*)k_narrow<float2>, total);
    k_narrow<float2><<<grid, kBlock, 0, s>>>(total, out, (float2*)state->data);
    count_launches(1);
    GQT_CUDA(cudaGetLastError());
  }
  return GQT_OK;
}

extern "C" gqt_status gqt_evolve(const gqt_ham* h, int direction, double dt_scaled,
                                 gqt_vec* state)
{
  return evolve_common(h, direction, dt_scaled, state, false);
}

extern "C" gqt_status gqt_evolvex(const gqt_ham* h, int direction, double dt_scaled,
                                  gqt_vec* state)
{
  return evolve_common(h, direction, dt_scaled, state, true);
}

// ------------------------------------------------------------------ summation (host)
extern "C" gqt_status gqt_chebyshev_summation(int M, double* mu_re, double* mu_im, int n_energy,
                                              const double* energy, double energy_max,
                                              double volume, double* out)
{
  if (M < 2)
    return fail(GQT_ERR_ARG, "gqt_chebyshev_summation: needs at least 2 moments (got %d)", M);
  if (!mu_re || !mu_im || (!energy && n_energy > 0) || (!out && n_energy > 0))
    return fail(GQT_ERR_ARG, "gqt_chebyshev_summation: null argument");
  const double PI = 3.141592653589793;
  // Jackson damping (src/sigma.cu:76-86).
  for (int k = 0; k < M; ++k) {
    const double factor = 1.0 / (M + 1);
    const double damping =
      (1 - k * factor) * std::cos(k * PI * factor) + std::sin(k * PI * factor) * factor /
                                                       std::tan(PI * factor);
    mu_re[k] *= damping;
    mu_im[k] *= damping;
  }
  // Chebyshev summation (src/sigma.cu:89-110).
  for (int e = 0; e < n_energy; ++e) {
    const double es = energy[e] / energy_max;
    double c0 = 1.0, c1 = es, c2;
    double temp = mu_re[1] * c1;
    for (int s2 = 2; s2 < M; ++s2) {
      c2 = 2.0 * es * c1 - c0;
      c0 = c1;
      c1 = c2;
      temp += mu_re[s2] * c2;
    }
    temp *= 2.0;
    temp += mu_re[0];
    temp *= 2.0 / (PI * volume);
    temp /= std::sqrt(1.0 - es * es);
    out[e] = temp / energy_max;
  }
  return GQT_OK;
}

// ------------------------------------------------------------------ loop selection
extern "C" gqt_status gqt_ham_set_loop(gqt_ham* h, int window, int chunk_sites)
{
  if (!h)
    return fail(GQT_ERR_ARG, "gqt_ham_set_loop: null handle");
  if (window != 0 && (window < 2 || window > 64))
    return fail(GQT_ERR_ARG, "gqt_ham_set_loop: window must be 0 or 2..64 (got %d)", window);
  if (chunk_sites == 0)
    chunk_sites = 1024;
  if (chunk_sites < kBlock || chunk_sites > (1 << 16) || chunk_sites % kBlock)
    return fail(GQT_ERR_ARG,
                "gqt_ham_set_loop: chunk_sites must be a multiple of %d up to 65536 (got %d)",
                kBlock, chunk_sites);
  if (chunk_sites != h->loop_chunk) {
    h->loop_chunk = chunk_sites;
    h->wave_halo = -1;  // plan again
  }
  if (h->ws) {
    // Graphs captured so far launch the other loop.
    cudaStreamSynchronize(stream());
    for (auto& kv : h->ws->graphs)
      cudaGraphExecDestroy(kv.second);
    h->ws->graphs.clear();
  }
  h->loop_window = window;
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_loop(const gqt_ham* h, int* window, int* chunks, int* halo)
{
  if (!h)
    return fail(GQT_ERR_ARG, "gqt_ham_loop: null handle");
  if (window)
    *window = h->loop_window;
  if (chunks)
    *chunks = h->wave_halo >= 0 ? h->wave_chunks : 0;
  if (halo)
    *halo = h->wave_halo;
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_set_staging(gqt_ham* h, int stages)
{
  if (!h)
    return fail(GQT_ERR_ARG, "gqt_ham_set_staging: null handle");
  if (stages < -1 || stages > 4)
    return fail(GQT_ERR_ARG, "gqt_ham_set_staging: stages must be -1..4 (got %d)", stages);
  if (h->ws) {
    // Graphs captured so far launch the other step.
    cudaStreamSynchronize(stream());
    for (auto& kv : h->ws->graphs)
      cudaGraphExecDestroy(kv.second);
    h->ws->graphs.clear();
  }
  h->stage_stages = stages;
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_staging(const gqt_ham* h, int* stages, int* windows,
                                      int* lo, int* hi)
{
  if (!h)
    return fail(GQT_ERR_ARG, "gqt_ham_staging: null handle");
  if (stages)
    *stages = h->stage_stages;
  if (windows)
    *windows = h->use_codes ? h->stage_nw : 0;
  for (int w = 0; w < h->stage_nw; ++w) {
    if (lo)
      lo[w] = h->stage_lo[w];
    if (hi)
      hi[w] = h->stage_hi[w];
  }
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_stage_plan(const gqt_ham* h, int nvec, int precision,
                                         int symmetric, int* stages, int* windows)
{
  if (!h || !stages)
    return fail(GQT_ERR_ARG, "gqt_ham_stage_plan: null argument");
  *stages = 0;
  if (windows)
    *windows = 0;
  if (precision != GQT_FP32 && precision != GQT_FP32R)
    return GQT_OK;
  const Op op = make_op(h, nvec);
  *stages = stage_plan(op, nvec, symmetric ? kDotPair : kDotLeft, precision == GQT_FP32R,
                       windows, h->n_real);
  return GQT_OK;
}

// ------------------------------------------------------------------ autotuner
extern "C" gqt_status gqt_autotune_nvec(const gqt_ham* h, int precision, int n_moments,
                                        const int* candidates, int n_candidates, int* best,
                                        double* rates)
{
  const char* w = "gqt_autotune_nvec";
  if (!h || !candidates || n_candidates < 1 || !best)
    return fail(GQT_ERR_ARG, "%s: null argument or no candidates", w);
  if (n_moments < 2)
    return fail(GQT_ERR_ARG, "%s: needs at least 2 probe moments", w);
  long long sites = 0;
  for (int r = 0; r < h->n_real; ++r)
    sites += h->real_n[r];
  cudaStream_t s = stream();
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  GQT_CUDA(cudaEventCreate(&e0));
  GQT_CUDA(cudaEventCreate(&e1));
  double best_rate = -1.0;
  gqt_status st = GQT_OK;
  Workspace& ws = *h->ws;
  bool changed = false;
  int best_tile = 0;
  for (int k = 0; k < n_candidates && st == GQT_OK; ++k) {
    const int V = candidates[k];
    double rate = 0.0;
    if (form_ops(precision, V)) {
      gqt_vec* x = nullptr;
      double2* mu = nullptr;
      // GQT_FP32R probes run on FP32 vectors (the form's storage)
      st = gqt_vec_create(h->n, V, precision == GQT_FP32R ? GQT_FP32 : precision, &x);
      if (st == GQT_OK) {
        const size_t bytes = (size_t)n_moments * h->n_real * V * sizeof(double2);
        cudaError_t ce = cudaMalloc(&mu, bytes);
        if (ce != cudaSuccess)
          st = cuda_fail(ce, "cudaMalloc(probe moments)", __FILE__, __LINE__);
      }
      // Shapes: vectors per thread 4 (the default) and 2, where the form has both; on a
      // realisation batch, each with every tile size.
      const int shapes[2] = {0, 2};
      const int n_shapes = (precision == GQT_FP32 && V >= 4) ? 2 : 1;
      // (the FP32R batch step hands out its own tiles: the batch tile does not apply)
      const int n_tiles = (h->n_real > 1 && precision != GQT_FP32R) ? kBatchTiles : 1;
      int best_w = 0, best_t = h->tile_sites;
      for (int q = 0; q < n_shapes * n_tiles && st == GQT_OK; ++q) {
        const int si = q / n_tiles;
        // the vectors-per-thread shape is the FP32 form's (FP32R leaves it as it is)
        if (precision != GQT_FP32R)
          h->wpt[V] = shapes[si];
        if (h->n_real > 1) {
          st = batch_set_tile(const_cast<gqt_ham*>(h), kBatchTileSizes[q % n_tiles]);
          if (st != GQT_OK)
            break;
        }
        // warm-up, graph capture
        st = gqt_moments_device_form(h, x, x, n_moments, precision, mu);
        float ms = 0.f;
        if (st == GQT_OK) {
          cudaEventRecord(e0, s);
          st = gqt_moments_device_form(h, x, x, n_moments, precision, mu);
          if (st == GQT_OK)
            st = gqt_moments_device_form(h, x, x, n_moments, precision, mu);
          cudaEventRecord(e1, s);
          cudaError_t ce = cudaEventSynchronize(e1);
          if (ce == cudaSuccess)
            ce = cudaEventElapsedTime(&ms, e0, e1);
          if (st == GQT_OK && ce != cudaSuccess)
            st = cuda_fail(ce, "autotune timing", __FILE__, __LINE__);
        }
        const double r = (st == GQT_OK && ms > 0.f)
                           ? 2.0 * (double)V * (double)sites * n_moments / (ms * 1e-3)
                           : 0.0;
        if (r > rate) {
          rate = r;
          best_w = shapes[si];
          best_t = h->tile_sites;
        }
        // The probe's graph was captured with this shape; drop it before the next.
        cudaStreamSynchronize(s);
        for (auto it = ws.graphs.begin(); it != ws.graphs.end();) {
          if (x && std::get<0>(it->first) == x->data) {
            cudaGraphExecDestroy(it->second);
            it = ws.graphs.erase(it);
          } else {
            ++it;
          }
        }
      }
      if (precision != GQT_FP32R) {
        if (h->wpt[V] != best_w || n_shapes > 1 || n_tiles > 1)
          changed = true;
        h->wpt[V] = best_w;
      }
      if (rate > best_rate)
        best_tile = best_t;
      cudaFree(mu);
      gqt_vec_destroy(x);
    }
    if (rates)
      rates[k] = rate;
    if (rate > best_rate) {
      best_rate = rate;
      *best = V;
    }
  }
  // A batch keeps the tile size of the fastest candidate.
  if (h->n_real > 1 && best_tile > 0 && st == GQT_OK)
    st = batch_set_tile(const_cast<gqt_ham*>(h), best_tile);
  if (changed) {
    // Graphs captured before the tuning launch the old shapes; recapture on next use.
    cudaStreamSynchronize(s);
    for (auto& kv : ws.graphs)
      cudaGraphExecDestroy(kv.second);
    ws.graphs.clear();
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != GQT_OK)
    return st;
  if (best_rate <= 0.0)
    return fail(GQT_ERR_ARG, "%s: no candidate is a supported vector count", w);
  return GQT_OK;
}
