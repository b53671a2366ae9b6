// FP32-storage form: interleaved float2 vectors, FP64 operator and FP64 sums.
#include "gqt_forms_impl.cuh"

namespace gqt {

const FormOps* forms_fp32(int nvec)
{
  switch (nvec) {
    case 1:
      return FormImpl<float2, 1, FastArith>::table(GQT_FP32, op_fns_fp32_coded(1));
    case 4:
      return FormImpl<float2, 4, FastArith>::table(GQT_FP32, op_fns_fp32_coded(4));
    case 8:
      return FormImpl<float2, 8, FastArith>::table(GQT_FP32, op_fns_fp32_coded(8));
    case 16:
      return FormImpl<float2, 16, FastArith>::table(GQT_FP32, op_fns_fp32_coded(16));
    case 32:
      return FormImpl<float2, 32, FastArith>::table(GQT_FP32, op_fns_fp32_coded(32));
    default:
      return nullptr;
  }
}

}  // namespace gqt
