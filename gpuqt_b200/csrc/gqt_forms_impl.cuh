// Template bodies of the launch tables; included by the gqt_forms_*.cu files only.
// OpImpl holds the kernels that read the operator, instantiated once per format
// (C: coded table, or the ELL arrays) in their own translation units; FormImpl holds
// the rest and assembles the table.
#pragma once

#include <type_traits>

#include "gqt_forms.h"

namespace gqt {

template <class F>
gqt_status with_z(int z, F&& f)
{
  switch (z) {
    case 3:
      return f(std::integral_constant<int, 3>{});
    case 4:
      return f(std::integral_constant<int, 4>{});
    case 6:
      return f(std::integral_constant<int, 6>{});
    default:
      return f(std::integral_constant<int, 0>{});
  }
}

template <typename K, typename... Args>
gqt_status launch(K* kernel, size_t total, Args... args)
{
  const int grid = grid_for((const void*)kernel, total);
  kernel<<<grid, kBlock, 0, stream()>>>(args...);
  count_launches(1);
  GQT_CUDA(cudaGetLastError());
  return GQT_OK;
}

// Kernels that read the operator take Op first; with a coded operator its table
// goes to dynamic shared memory.
template <typename K, typename... Args>
gqt_status launch_op(K* kernel, size_t total, const Op& op, Args... args)
{
  const int grid = grid_for((const void*)kernel, total);
  kernel<<<grid, kBlock, op_smem_bytes(op), stream()>>>(op, args...);
  count_launches(1);
  GQT_CUDA(cudaGetLastError());
  return GQT_OK;
}

// launch_op with programmatic stream serialisation: the kernel may start while the
// previous kernel in the stream finishes, and must call pdl_wait before it reads or
// writes anything a previous kernel produces (k_step does).
template <typename... KArgs, typename... Args>
gqt_status launch_op_pdl(void (*kernel)(Op, KArgs...), size_t total, const Op& op, Args... args)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid_for((const void*)kernel, total));
  cfg.blockDim = dim3(kBlock);
  cfg.dynamicSmemBytes = op_smem_bytes(op);
  cfg.stream = stream();
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  GQT_CUDA(cudaLaunchKernelEx(&cfg, kernel, op, args...));
  count_launches(1);
  return GQT_OK;
}

template <typename K, typename... Args>
gqt_status launch_smem(K* kernel, size_t total, size_t smem, Args... args)
{
  const int grid = grid_for((const void*)kernel, total);
  kernel<<<grid, kBlock, smem, stream()>>>(args...);
  count_launches(1);
  GQT_CUDA(cudaGetLastError());
  return GQT_OK;
}

// Storage types with FP32 elements (float2; xf2, FP32 with a BF16 residual).
template <typename VT2>
struct Fp32Like
    : std::integral_constant<bool, std::is_same<VT2, float2>::value ||
                                       std::is_same<VT2, xf2>::value> {
};

// Vectors a thread advances per step launch: 4 float2 (two 16-byte loads), 2 double2,
// or 2 FP32X elements (a 16-byte load and an 8-byte residual load; at 4 the residuals'
// registers spilled on rows of 4 and 6).
template <typename VT2, int V>
constexpr int vectors_per_thread()
{
  constexpr int w = std::is_same<VT2, float2>::value ? 4 : 2;
  return V < w ? V : w;
}

template <typename VT2, int V, class A, bool C>
struct OpImpl {
  // Default vectors per thread, and the alternative the autotuner may choose (two
  // vectors per thread: half the accumulator registers, twice the threads per site).
  static constexpr int W = vectors_per_thread<VT2, V>();
  static constexpr int W2 = (std::is_same<VT2, float2>::value && V >= 4) ? 2 : W;
  // Vectors a thread advances in the pair mode of a symmetric moment set. The pair mode
  // keeps three FP64 sums per vector and T_{k-1} until the end of an item. k_step_vec:
  // 4 float2 with 128 registers (2 blocks per SM; 13.6 % faster on B200 than 2 float2
  // at 85 registers), 2 FP32X elements, 1 double2. k_step_multi (80 registers): 2
  // FP32-element vectors, 1 double2.
  static constexpr int WP = std::is_same<VT2, float2>::value
                              ? (V < 4 ? V : 4)
                              : (std::is_same<VT2, xf2>::value ? (V < 2 ? V : 2) : 1);
  static constexpr int WPM = Fp32Like<VT2>::value ? (V < 2 ? V : 2) : 1;

  static gqt_status step(const Op& op, int mode, const void* t0, const void* t1, void* out,
                         const void* left, const Dot* dot)
  {
    const size_t total = (size_t)op.n * V;
    const VT2* a0 = (const VT2*)t0;
    const VT2* a1 = (const VT2*)t1;
    VT2* o = (VT2*)out;
    const VT2* l = (const VT2*)left;
    Dot d = dot ? *dot : Dot{nullptr, nullptr, nullptr};
    if constexpr (C && std::is_same<VT2, float2>::value) {
      if (dot && stage_applies(op, V, mode, kDotLeft, t0, t1, left))
        return stage_step(op, V, mode, kDotLeft, t0, t1, out, left, d);
    }
    return with_z(op.z, [&](auto zc) -> gqt_status {
      constexpr int Z = decltype(zc)::value;
      if constexpr (W > 1) {
        // several vectors per thread: one launch item per (site, W vectors)
        auto run = [&](auto wc) -> gqt_status {
          constexpr int WW = decltype(wc)::value;
          const size_t items = (size_t)op.n * (V / WW);
          if (mode == kApply) {
            if (dot)
              return launch_op(k_step_vec<VT2, V, WW, Z, A, kApply, true, C>, items, op, a0, a1, o, l,
                            d);
            return launch_op(k_step_vec<VT2, V, WW, Z, A, kApply, false, C>, items, op, a0, a1, o, l,
                          d);
          }
          if (dot)
            return launch_op(k_step_vec<VT2, V, WW, Z, A, kCheb, true, C>, items, op, a0, a1, o, l, d);
          return launch_op(k_step_vec<VT2, V, WW, Z, A, kCheb, false, C>, items, op, a0, a1, o, l, d);
        };
        if constexpr (W2 != W) {
          if (op.wpt == W2)
            return run(std::integral_constant<int, W2>{});
        }
        if constexpr (std::is_same<VT2, xf2>::value && Z == 3 && V >= 4) {
          // FP32X on rows of three: 4 vectors per thread fit the register budget there
          // (rows of 4 and 6 spill at 4, hence 2 elsewhere)
          return run(std::integral_constant<int, 4>{});
        }
        return run(std::integral_constant<int, W>{});
      }
      // Programmatic dependent launch for the FP64 step (+1-2 % there; the FP32 step
      // lost 7 % with it on B200).
      auto go = [&](auto* kernel) -> gqt_status {
        if constexpr (std::is_same<VT2, double2>::value)
          return launch_op_pdl(kernel, total, op, a0, a1, o, l, d);
        else
          return launch_op(kernel, total, op, a0, a1, o, l, d);
      };
      if (mode == kApply) {
        if (dot)
          return go(k_step<VT2, V, Z, A, kApply, true, C>);
        return go(k_step<VT2, V, Z, A, kApply, false, C>);
      }
      if (dot)
        return go(k_step<VT2, V, Z, A, kCheb, true, C>);
      return go(k_step<VT2, V, Z, A, kCheb, false, C>);
    });
  }

  static gqt_status step_pair(const Op& op, int mode, const void* t0, const void* t1, void* out,
                              const Dot& d)
  {
    if constexpr (V > 16) {
      return fail(GQT_ERR_ARG, "symmetric moments: at most 16 vectors per launch (got %d)", V);
    } else {
      const VT2* a0 = (const VT2*)t0;
      const VT2* a1 = (const VT2*)t1;
      VT2* o = (VT2*)out;
      if constexpr (C && std::is_same<VT2, float2>::value) {
        if (stage_applies(op, V, mode, kDotPair, t0, t1, nullptr))
          return stage_step(op, V, mode, kDotPair, t0, t1, out, nullptr, d);
      }
      return with_z(op.z, [&](auto zc) -> gqt_status {
        constexpr int Z = decltype(zc)::value;
        if constexpr (V > 1) {
          const size_t items = (size_t)op.n * (V / WP);
          if (mode == kApply)
            return launch_op(k_step_vec<VT2, V, WP, Z, A, kApply, kDotPair, C>, items, op, a0,
                             a1, o, (const VT2*)nullptr, d);
          return launch_op(k_step_vec<VT2, V, WP, Z, A, kCheb, kDotPair, C>, items, op, a0, a1,
                           o, (const VT2*)nullptr, d);
        } else {
          const size_t total = (size_t)op.n * V;
          if (mode == kApply)
            return launch_op(k_step<VT2, V, Z, A, kApply, kDotPair, C>, total, op, a0, a1, o,
                             (const VT2*)nullptr, d);
          return launch_op(k_step<VT2, V, Z, A, kCheb, kDotPair, C>, total, op, a0, a1, o,
                           (const VT2*)nullptr, d);
        }
      });
    }
  }

  static gqt_status step_multi(const Op& op, int mode, const void* t0, const void* t1,
                               void* out, const void* left, const MultiDot& md_in, int dot)
  {
    const VT2* a0 = (const VT2*)t0;
    const VT2* a1 = (const VT2*)t1;
    VT2* o = (VT2*)out;
    const VT2* l = (const VT2*)left;
    MultiDot md = md_in;
    const size_t items = (size_t)md.n_tiles * kBlock;
    GQT_TRY(with_z(op.z, [&](auto zc) -> gqt_status {
      constexpr int Z = decltype(zc)::value;
      auto go = [&](auto* kernel) -> gqt_status {
        md.blocks = grid_for((const void*)kernel, items);
        if (md.blocks_out)
          *md.blocks_out = md.blocks;
        kernel<<<md.blocks, kBlock, op_smem_bytes(op), stream()>>>(op, a0, a1, o, l, md);
        count_launches(1);
        GQT_CUDA(cudaGetLastError());
        return GQT_OK;
      };
      if (dot == kDotPair && mode != kDotOnly) {
        if (mode == kApply)
          return go(k_step_multi<VT2, V, WPM, Z, A, kApply, C, kDotPair>);
        return go(k_step_multi<VT2, V, WPM, Z, A, kCheb, C, kDotPair>);
      }
      auto pick = [&](auto wc) -> gqt_status {
        constexpr int WW = decltype(wc)::value;
        if (mode == kDotOnly)
          return go(k_step_multi<VT2, V, WW, Z, A, kDotOnly, C>);
        if (mode == kApply)
          return go(k_step_multi<VT2, V, WW, Z, A, kApply, C>);
        return go(k_step_multi<VT2, V, WW, Z, A, kCheb, C>);
      };
      if constexpr (W2 != W) {
        if (op.wpt == W2)
          return pick(std::integral_constant<int, W2>{});
      }
      return pick(std::integral_constant<int, W>{});
    }));
    if (md.defer)
      return GQT_OK;  // the caller reduces a window of steps at once (tile_reduce)
    return tile_reduce(md, dot == kDotPair && mode != kDotOnly, 1, 0);
  }

  // k_tile_reduce over `rows` steps whose slots lie row_stride doubles apart.
  static gqt_status tile_reduce(const MultiDot& md, bool pair, int rows, size_t row_stride)
  {
    if (pair)
      k_tile_reduce<2 * V><<<dim3(md.n_real * 2 * V, rows), kBlock, 0, stream()>>>(md,
                                                                                row_stride);
    else
      k_tile_reduce<V><<<dim3(md.n_real * V, rows), kBlock, 0, stream()>>>(md, row_stride);
    count_launches(1);
    GQT_CUDA(cudaGetLastError());
    return GQT_OK;
  }

  static gqt_status xop(const Op& op, bool current, const void* in, void* out)
  {
    const size_t total = (size_t)op.n * V;
    return with_z(op.z, [&](auto zc) -> gqt_status {
      constexpr int Z = decltype(zc)::value;
      if (current)
        return launch_op(k_xop<VT2, V, Z, A, true, C>, total, op, (const VT2*)in, (VT2*)out);
      return launch_op(k_xop<VT2, V, Z, A, false, C>, total, op, (const VT2*)in, (VT2*)out);
    });
  }

  static gqt_status cheb2(const Op& op, const void* s0, const void* s1, void* s2,
                          double2* out, double bessel, int label)
  {
    const size_t total = (size_t)op.n * V;
    return with_z(op.z, [&](auto zc) -> gqt_status {
      constexpr int Z = decltype(zc)::value;
      return launch_op(k_cheb2<VT2, double2, V, Z, A, C>, total, op, (const VT2*)s0,
                    (const VT2*)s1, (VT2*)s2, out, bessel, label);
    });
  }

  static gqt_status cheb2x(const Op& op, const void* s0, const void* s0x, const void* s1,
                           const void* s1x, void* s2, void* s2x, double2* out,
                           double bessel, int label)
  {
    const size_t total = (size_t)op.n * V;
    return with_z(op.z, [&](auto zc) -> gqt_status {
      constexpr int Z = decltype(zc)::value;
      return launch_op(k_cheb2x<VT2, double2, V, Z, A, C>, total, op, (const VT2*)s0,
                    (const VT2*)s0x, (const VT2*)s1, (const VT2*)s1x, (VT2*)s2, (VT2*)s2x,
                    out, bessel, label);
    });
  }

  static OpFns fns()
  {
    return OpFns{step, step_pair, step_multi, tile_reduce, xop, cheb2, cheb2x};
  }
};

template <typename VT2, int V, class A>
struct FormImpl {
  static gqt_status dot(size_t total, const void* state, const void* left, const Dot& d)
  {
    return launch(k_dot<VT2, V>, total, total, (const VT2*)state, (const VT2*)left, d);
  }

  static gqt_status cheb01(size_t total, const void* s0, const void* s1, double2* out,
                           double b0, double b1)
  {
    return launch(k_cheb01<VT2, double2, A>, total, total, (const VT2*)s0, (const VT2*)s1,
                  out, b0, b1);
  }

  static gqt_status cheb1x(size_t total, const void* s1x, double2* out, double b1)
  {
    return launch(k_cheb1x<VT2, double2, A>, total, total, (const VT2*)s1x, out, b1);
  }

  static gqt_status add(size_t total, void* dst, const void* src)
  {
    return launch(k_add<VT2>, total, total, (VT2*)dst, (const VT2*)src);
  }

  static gqt_status apply_sz(size_t total, int nvec, void* dst, const void* src)
  {
    return launch(k_apply_sz<VT2>, total, total, nvec, (VT2*)dst, (const VT2*)src);
  }

  static gqt_status interleave(int n, int nvec, const double* re, const double* im, void* out)
  {
    return launch(k_interleave<VT2>, (size_t)n * nvec, n, nvec, re, im, (VT2*)out);
  }

  static gqt_status deinterleave(int n, int nvec, const void* in, double* re, double* im)
  {
    return launch(k_deinterleave<VT2>, (size_t)n * nvec, n, nvec, (const VT2*)in, re, im);
  }

  // The table of this form: the ELL kernels from OpImpl<..., false> (this
  // translation unit) and the coded ones from their own unit.
  static const FormOps* table(int precision, OpFns coded)
  {
    static const FormOps t = [&] {
      FormOps f{};
      f.precision = precision;
      f.nvec = V;
      f.elem_bytes = sizeof(VT2);
      f.fmt[0] = OpImpl<VT2, V, A, false>::fns();
      f.fmt[1] = coded;
      f.dot = dot;
      f.cheb01 = cheb01;
      f.cheb1x = cheb1x;
      f.add = add;
      f.apply_sz = apply_sz;
      f.interleave = interleave;
      f.deinterleave = deinterleave;
      return f;
    }();
    return &t;
  }
};

}  // namespace gqt
