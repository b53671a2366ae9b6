// FP64 form: interleaved double2 vectors, exact reference-order arithmetic.
#include "gqt_forms_impl.cuh"

namespace gqt {

const FormOps* forms_fp64(int nvec)
{
  switch (nvec) {
    case 1:
      return FormImpl<double2, 1, ExactArith>::table(GQT_FP64, op_fns_fp64_coded(1));
    case 4:
      return FormImpl<double2, 4, ExactArith>::table(GQT_FP64, op_fns_fp64_coded(4));
    case 16:
      return FormImpl<double2, 16, ExactArith>::table(GQT_FP64, op_fns_fp64_coded(16));
    default:
      return nullptr;
  }
}

}  // namespace gqt
