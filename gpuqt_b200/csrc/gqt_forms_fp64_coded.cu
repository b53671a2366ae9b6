// FP64 form, coded operator format: the kernels that read the operator, compiled for
// the one-byte codes and the shared-memory table (a unit of its own so both formats
// compile in parallel).
#include "gqt_forms_impl.cuh"

namespace gqt {

OpFns op_fns_fp64_coded(int nvec)
{
  switch (nvec) {
    case 1:
      return OpImpl<double2, 1, ExactArith, true>::fns();
    case 4:
      return OpImpl<double2, 4, ExactArith, true>::fns();
    case 16:
      return OpImpl<double2, 16, ExactArith, true>::fns();
    default:
      return OpFns{};
  }
}

}  // namespace gqt
