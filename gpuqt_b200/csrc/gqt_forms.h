// Launch tables: one per arithmetic form (FP64 exact / FP32 storage) and vector-block
// width V. The algorithm layer (gqt_algo.cu) calls through these so each form's
// template instantiations live in their own translation unit.
#pragma once

#include <cuda_runtime.h>

#include "gqt_internal.h"
#include "gqt_kernels.cuh"

namespace gqt {

// The kernels that read the operator, for one format (ELL arrays or coded table).
struct OpFns {
  // out = H t1 (mode kApply) or 2 H t1 - t0 (kCheb); dot != nullptr fuses <left|out>.
  gqt_status (*step)(const Op& op, int mode, const void* t0, const void* t1, void* out,
                     const void* left, const Dot* dot);
  // The same step fusing the pair <T_k|T_k>, <T_{k-1}|T_k> (t1 = T_{k-1}) of a symmetric
  // moment set into dot->mu[0 .. 2 nvec); GQT_ERR_ARG for more than 16 vectors.
  gqt_status (*step_pair)(const Op& op, int mode, const void* t0, const void* t1, void* out,
                          const Dot& dot);
  // One step of a realisation batch (mode kDotOnly, kApply or kCheb) with moments per
  // realisation: <left|out> (dot kDotLeft), or the pair products of a symmetric set
  // (kDotPair: 2 nvec sums per realisation, [2v] <T_k|T_k>, [2v + 1] <T_{k-1}|T_k>).
  gqt_status (*step_multi)(const Op& op, int mode, const void* t0, const void* t1, void* out,
                           const void* left, const MultiDot& md, int dot);
  // The per-realisation moments of `rows` batch steps launched with md.defer set (pair:
  // the steps fused the pair products); step j's slots start j * row_stride doubles into
  // md.partials and its results go to md.mu + j * R * (pair ? 2 : 1) * nvec.
  gqt_status (*tile_reduce)(const MultiDot& md, bool pair, int rows, size_t row_stride);
  gqt_status (*xop)(const Op& op, bool current, const void* in, void* out);
  // Evolution terms; out is a double2 accumulator (the FP64 state itself, or the
  // FP32 form's FP64 accumulator).
  gqt_status (*cheb2)(const Op& op, const void* s0, const void* s1, void* s2, double2* out,
                      double bessel, int label);
  gqt_status (*cheb2x)(const Op& op, const void* s0, const void* s0x, const void* s1,
                       const void* s1x, void* s2, void* s2x, double2* out, double bessel,
                       int label);
};

struct FormOps {
  int precision;
  int nvec;
  size_t elem_bytes;  // bytes of one complex vector element
  OpFns fmt[2];       // [0]: ELL arrays, [1]: coded table
  gqt_status (*dot)(size_t total, const void* state, const void* left, const Dot& dot);
  gqt_status (*cheb01)(size_t total, const void* s0, const void* s1, double2* out, double b0,
                       double b1);
  gqt_status (*cheb1x)(size_t total, const void* s1x, double2* out, double b1);
  gqt_status (*add)(size_t total, void* dst, const void* src);
  gqt_status (*apply_sz)(size_t total, int nvec, void* dst, const void* src);
  gqt_status (*interleave)(int n, int nvec, const double* re, const double* im, void* out);
  gqt_status (*deinterleave)(int n, int nvec, const void* in, double* re, double* im);

  // The operator kernels of op's format.
  const OpFns& of(const Op& op) const { return fmt[op.code != nullptr ? 1 : 0]; }
  gqt_status step(const Op& op, int mode, const void* t0, const void* t1, void* out,
                  const void* left, const Dot* d) const
  {
    return of(op).step(op, mode, t0, t1, out, left, d);
  }
  gqt_status step_pair(const Op& op, int mode, const void* t0, const void* t1, void* out,
                       const Dot& d) const
  {
    return of(op).step_pair(op, mode, t0, t1, out, d);
  }
  gqt_status step_multi(const Op& op, int mode, const void* t0, const void* t1, void* out,
                        const void* left, const MultiDot& md, int dot = kDotLeft) const
  {
    return of(op).step_multi(op, mode, t0, t1, out, left, md, dot);
  }
  gqt_status tile_reduce(const Op& op, const MultiDot& md, bool pair, int rows,
                         size_t row_stride) const
  {
    return of(op).tile_reduce(md, pair, rows, row_stride);
  }
  gqt_status xop(const Op& op, bool current, const void* in, void* out) const
  {
    return of(op).xop(op, current, in, out);
  }
  gqt_status cheb2(const Op& op, const void* s0, const void* s1, void* s2, double2* out,
                   double bessel, int label) const
  {
    return of(op).cheb2(op, s0, s1, s2, out, bessel, label);
  }
  gqt_status cheb2x(const Op& op, const void* s0, const void* s0x, const void* s1,
                    const void* s1x, void* s2, void* s2x, double2* out, double bessel,
                    int label) const
  {
    return of(op).cheb2x(op, s0, s0x, s1, s1x, s2, s2x, out, bessel, label);
  }
};

const FormOps* forms_fp64(int nvec);
const FormOps* forms_fp32(int nvec);
// GQT_FP32X: moment loops only (dot, step, step_pair; nvec 1, 4, 16).
const FormOps* forms_fp32x(int nvec);
// GQT_FP32R (gqt_stage.cu): moment loops only (dot, step, step_pair; nvec 4, 16 and 32).
const FormOps* forms_fp32r(int nvec);
// src (GQT_FP64 or GQT_FP32 storage, `total` elements) into FP32X storage at dst.
gqt_status convert_to_x(size_t total, int from, const void* src, void* dst, uintptr_t xlo);
// The coded format's operator kernels (gqt_forms_fp64_coded.cu, gqt_forms_fp32_coded.cu).
OpFns op_fns_fp64_coded(int nvec);
OpFns op_fns_fp32_coded(int nvec);
inline const FormOps* form_ops(int precision, int nvec)
{
  if (precision == GQT_FP64)
    return forms_fp64(nvec);
  if (precision == GQT_FP32)
    return forms_fp32(nvec);
  if (precision == GQT_FP32X)
    return forms_fp32x(nvec);
  if (precision == GQT_FP32R)
    return forms_fp32r(nvec);
  return nullptr;
}

// The staged step of the FP32 moment loops over the coded operator (gqt_stage.cu): whether
// it serves this step (op has staging windows, nvec 16 or 32, rows of 3, 4 or 6, dot kDotLeft
// or kDotPair, 16-byte aligned vectors), and the step itself; f32 selects the GQT_FP32R
// arithmetic (the recurrence in FP32) instead of GQT_FP32's.
bool stage_applies(const Op& op, int nvec, int mode, int dot, const void* t0, const void* t1,
                   const void* left, bool f32 = false);
gqt_status stage_step(const Op& op, int nvec, int mode, int dot, const void* t0,
                      const void* t1, void* out, const void* left, const Dot& d,
                      bool f32 = false);
// The stages and windows (*windows) the staged Chebyshev step of a moment loop would use
// for nvec vectors (dot kDotLeft: direct, kDotPair: symmetric sets); 0 when it would not
// be staged.
int stage_plan(const Op& op, int nvec, int dot, bool f32, int* windows, int R = 1);
// The FP32R form's split potential of h (gqt_ham::pot_r), made on first use.
gqt_status ensure_pot_r(const gqt_ham* h);
// Grid size for a grid-stride kernel: enough blocks to cover `total` elements, capped
// at the number of blocks that are resident at once on all SMs.
int grid_for(const void* kernel, size_t total);
// Upper bound of grid_for over all kernels (sizes the dot partials).
int max_grid();

}  // namespace gqt
