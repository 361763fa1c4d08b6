// idct_tc.cu -- tensor-core iDCT (FP16 hi+lo basis, FP32 accumulate).
#include "cj_internal.h"

struct CJPlaneArgs;
int cj_idct_tc_plane(const CJPlaneArgs&, cudaStream_t) { return UNSUPPORTED_ERROR; }
int cj_idct_tc_raw(const int16_t*, const int16_t*, float*, int64_t, cudaStream_t) {
  return UNSUPPORTED_ERROR;
}
