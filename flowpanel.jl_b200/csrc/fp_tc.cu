// FP32 trailing update C -= A B of the mixed-precision LU on the tcgen05
// tensor cores (3xTF32 split). Until the tensor-core kernel is enabled the
// SIMT FP32 kernel of fp_lu.cu performs the update.
#include "fp_internal.cuh"

namespace fpb {

bool tc_gemm_sub_f32(fp_ctx*, const float*, const float*, float*, int64_t, int64_t, int64_t, int) {
  return false;
}

}  // namespace fpb
