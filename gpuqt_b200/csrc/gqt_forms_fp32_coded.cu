// FP32-storage form, coded operator format: the kernels that read the operator, compiled for
// the one-byte codes and the shared-memory table (a unit of its own so both formats
// compile in parallel).
#include "gqt_forms_impl.cuh"

namespace gqt {

OpFns op_fns_fp32_coded(int nvec)
{
  switch (nvec) {
    case 1:
      return OpImpl<float2, 1, FastArith, true>::fns();
    case 4:
      return OpImpl<float2, 4, FastArith, true>::fns();
    case 8:
      return OpImpl<float2, 8, FastArith, true>::fns();
    case 16:
      return OpImpl<float2, 16, FastArith, true>::fns();
    case 32:
      return OpImpl<float2, 32, FastArith, true>::fns();
    default:
      return OpFns{};
  }
}

}  // namespace gqt
