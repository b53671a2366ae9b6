// FP32X form (GQT_FP32X): the moment recurrence on vectors stored as FP32 plus a BF16
// residual (xf2 storage, 12 bytes per complex element), FP64 operator and FP64 sums.
// Only the moment loops use it (direct and symmetric sets, one model): its vectors
// are workspace copies carved from one arena, whose residual map (Op::xlo, Dot::xlo)
// the loop passes to every launch. Both operator formats are compiled here.
#include "gqt_forms_impl.cuh"

namespace gqt {

namespace {

template <int V>
gqt_status dot_x(size_t total, const void* state, const void* left, const Dot& d)
{
  return launch(k_dot<xf2, V>, total, total, (const xf2*)state, (const xf2*)left, d);
}

template <int V, bool C>
OpFns fns_x()
{
  OpFns f{};
  f.step = OpImpl<xf2, V, FastArith, C>::step;
  f.step_pair = OpImpl<xf2, V, FastArith, C>::step_pair;
  return f;
}

template <int V>
const FormOps* table_x()
{
  static const FormOps t = [] {
    FormOps f{};
    f.precision = GQT_FP32X;
    f.nvec = V;
    f.elem_bytes = 12;
    f.fmt[0] = fns_x<V, false>();
    f.fmt[1] = fns_x<V, true>();
    f.dot = dot_x<V>;
    return f;
  }();
  return &t;
}

}  // namespace

const FormOps* forms_fp32x(int nvec)
{
  switch (nvec) {
    case 1:
      return table_x<1>();
    case 4:
      return table_x<4>();
    case 16:
      return table_x<16>();
    default:
      return nullptr;
  }
}

gqt_status convert_to_x(size_t total, int from, const void* src, void* dst, uintptr_t xlo)
{
  if (from == GQT_FP64) {
    return launch(k_to_x<double2>, total, total, (const double2*)src, (xf2*)dst, xlo);
  }
  if (from == GQT_FP32) {
    return launch(k_to_x<float2>, total, total, (const float2*)src, (xf2*)dst, xlo);
  }
  return fail(GQT_ERR_ARG, "FP32X copy: source form %d", from);
}

}  // namespace gqt
