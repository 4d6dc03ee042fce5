// Tensor-core M2L (tcgen05) lives here.
#include "fmm_internal.cuh"

namespace fmm {

fmm_status m2lTensorCore(Plan& P, cudaStream_t st)
{
   (void)P; (void)st;
   return setError(FMM_E_INVALID, "tensor-core M2L is not built in this library");
}

}  // namespace fmm
