// Internal declarations shared by the library's translation units (not installed).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "gpuqt.h"

namespace gqt {

// Thread-local error message and stream (see gpuqt.h).
gqt_status fail(gqt_status code, const char* fmt, ...);
gqt_status cuda_fail(cudaError_t e, const char* what, const char* file, int line);
cudaStream_t stream();
void count_launches(uint64_t k);

// Device properties cached per device.
struct DeviceInfo {
  int sms = 0;
};
const DeviceInfo& device_info();

// One reduction lane set: per-block partials of one fused launch and the arrival
// counter of the last-block reduction. All launches on one stream share it, in order.
struct DotScratch {
  double* partials = nullptr;  // [blocks][nvec][4] (re_hi, re_lo, im_hi, im_lo)
  unsigned* counter = nullptr;
  int blocks = 0;
  int nvec = 0;
};

// Tile sizes (sites) the batch step can run with; models are padded to the largest.
constexpr int kBatchTiles = 3;
constexpr int kBatchTileSizes[kBatchTiles] = {256, 512, 1024};
// Select tile size `tile` (one of kBatchTileSizes) for a realisation batch.
gqt_status batch_set_tile(gqt_ham* h, int tile);

// Temporary vectors and graph cache reused by the algorithm entry points.
struct Workspace;

}  // namespace gqt

#define GQT_CUDA(call)                                                 \
  do {                                                                 \
    cudaError_t e_ = (call);                                           \
    if (e_ != cudaSuccess)                                             \
      return gqt::cuda_fail(e_, #call, __FILE__, __LINE__);            \
  } while (0)

#define GQT_TRY(expr)            \
  do {                           \
    gqt_status s_ = (expr);      \
    if (s_ != GQT_OK)            \
      return s_;                 \
  } while (0)

struct gqt_vec {
  int n = 0;
  int nvec = 0;
  int precision = GQT_FP64;
  void* data = nullptr;  // double2 or float2, [site][vector]
  size_t bytes = 0;
  int device = 0;
  // GQT_FP32X copies (workspace only): data holds the FP32 parts, the residual of the
  // element at p lies at xlo + p / 2
  uintptr_t xlo = 0;
};

struct gqt_ham {
  int n = 0;
  int z = 0;
  double energy_max = 1.0;
  int uniform = 0;  // every row has z entries: neighbor_number is not read
  int device = 0;
  int* nn = nullptr;        // [n], null when uniform
  int* nl = nullptr;        // [z*n] column-major
  double2* hop = nullptr;   // [z*n] column-major
  double* xx = nullptr;     // [z*n] column-major
  double* pot = nullptr;    // [n]
  // [n]: the FP32R form's (hi, lo) FP32 parts of pot * RN(1 / energy_max), made on that
  // form's first use with the kernels' own arithmetic (null until then)
  mutable float2* pot_r = nullptr;
  bool has_xx = false;
  // Coded operator (built when the (j - i, hopping, xx) entries of the ELL take at
  // most GQT_MAX_CODES distinct values, as lattice models do): one byte per entry and
  // a small table holding the same doubles, so results are unchanged.
  uint8_t* code = nullptr;      // [z*n] column-major
  int* code_delta = nullptr;    // [n_codes]: j - i
  double2* code_hop = nullptr;  // [n_codes]
  double* code_xx = nullptr;    // [n_codes]
  int n_codes = 0;
  int hermitian = 0;  // H = H^+ (checked at upload; the symmetric moment loop needs it)
  int use_codes = 0;            // kernels read the codes (default when they exist)
  // Realisation batch (gqt_ham_create_batch): n_real > 1 block-diagonal models, each
  // padded to whole tiles and pre-divided by its own E_max (energy_max is then 1).
  int n_real = 1;
  int tile_sites = 0;         // sites per tile of the batch step (the autotuner's choice)
  int n_tiles = 0;
  int* tile_first = nullptr;  // device, [n_real + 1]: first tile of each model
  // device, [kBatchTiles][n_real + 1]: tile_first for each tile size of kBatchTileSizes
  // (every model is padded to the largest, so each divides every model's offset)
  int* tile_first_all = nullptr;
  std::vector<int> real_offset, real_n;
  std::vector<double> real_emax;
  // Vectors per thread of the batched step for each vector count (0: the form's
  // default); set by the autotuner.
  mutable int wpt[33] = {};
  // Moment loop of the FP64 form: 0 one launch per step; S >= 2 the wavefront loop,
  // S steps per launch (gqt_ham_set_loop). Its plan, made on first use: chunks of
  // wave_sites sites, the halo in positions (-1 not planned yet, -2 not applicable)
  // and the position order (1: folded).
  int loop_window = 0;
  int loop_chunk = 1024;  // sites per chunk of the wavefront loop
  mutable int wave_chunks = 0, wave_sites = 0, wave_halo = -1, wave_fold = 0;
  // Staged step of the FP32 moment loops (coded operator, gqt_ham_set_staging): the
  // windows of frequent neighbour offsets [stage_lo[w], stage_hi[w]] (window 0 holds 0),
  // the setting (-1 off; 0 automatic, the default: the symmetric loop is staged; 1 as
  // many stages as fit; 2..4 that many) and the device flag a wait that ran out sets.
  int stage_nw = 0;
  int stage_lo[8] = {}, stage_hi[8] = {};
  int stage_stages = 0;
  unsigned* stage_err = nullptr;
  // Realisation batches: each model's own windows in stage_rnw common slots (slot w is
  // stage_rwidth[w] + 1 offsets wide, the widest of the models' w-th windows). Device
  // table: [n_real][8] window lo, [n_real] windows of the model, [n_real][n_codes] the
  // slot holding each code's offset for that model (-1: gathered from global memory).
  int stage_rnw = 0;
  int stage_rwidth[8] = {};
  int* stage_rtab = nullptr;
  std::unique_ptr<gqt::Workspace> ws;
  ~gqt_ham();
};
