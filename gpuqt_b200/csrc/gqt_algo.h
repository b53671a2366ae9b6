// Algorithm layer: per-Hamiltonian workspace (temporary vectors, moment reduction
// scratch, cached CUDA graphs of the moment loop).
#pragma once

#include <map>
#include <tuple>
#include <vector>

#include "gqt_internal.h"

namespace gqt {

struct Workspace {
  // Temporary vectors per (precision, nvec), allocated on first use and reused.
  struct Bufs {
    size_t bytes = 0;
    std::vector<void*> v;
  };
  std::map<std::pair<int, int>, Bufs> bufs;
  double2* acc = nullptr;  // FP64 accumulator of the FP32 form's evolution
  size_t acc_bytes = 0;
  DotScratch dot;          // block partials + arrival counter of fused moment launches
  double2* mu = nullptr;   // device moments for the host-returning entry points
  size_t mu_bytes = 0;
  double2* mu_host = nullptr;  // pinned copy of mu read by those entry points
  size_t mu_host_bytes = 0;
  cudaStream_t capture_stream = nullptr;  // used when the caller's stream is the legacy one
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  double2* pairs = nullptr;  // pair products of the symmetric moment loop
  size_t pairs_bytes = 0;
  // FP32X moment loops: one arena of kXSlots slots (right, left, T_a, T_b) of `xslot`
  // elements each, the FP32 parts of all slots first, then their BF16 residuals, so
  // that the residual of the element at p lies at xlo + p / 2.
  unsigned char* xarena = nullptr;
  size_t xslot = 0;
  uintptr_t xlo = 0;
  // Wavefront moment loop: the last step done per chunk position, and its counters
  // (ticket, exited, error, pad).
  int* wave_done = nullptr;
  int wave_done_n = 0;
  unsigned* wave_ctl = nullptr;
  // Instantiated moment loops: (left, right, n_moments, mu, precision, nvec, loop),
  // loop 0 the direct one, 1 the symmetric (pair) one.
  using GraphKey = std::tuple<const void*, const void*, int, void*, int, int, int>;
  std::map<GraphKey, cudaGraphExec_t> graphs;
  std::map<GraphKey, uint64_t> graph_launches;  // kernel launches one replay runs
  ~Workspace();
};

Workspace* new_workspace();

// The i-th temporary vector of a form (n * nvec elements of elem bytes).
gqt_status ws_vector(Workspace& ws, int precision, int nvec, size_t bytes, int i, void** out);
gqt_status ws_dot(Workspace& ws, size_t doubles, DotScratch** out);
// The FP32X arena for `elems` elements per slot; slot k's FP32 part is returned by
// ws_xslot(ws, k).
constexpr int kXSlots = 4;
gqt_status ws_arena_x(Workspace& ws, size_t elems);
inline void* ws_xslot(const Workspace& ws, int k) { return ws.xarena + (size_t)k * ws.xslot * 8; }
// Moments per window of deferred grid stages for `results` sums per moment.
int defer_window(int results);

}  // namespace gqt
