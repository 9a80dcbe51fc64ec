// dense_tc.cu -- tensor-core (tcgen05) forms of the dense Gauss sketch.
#include <cuda_runtime.h>

#include "internal.h"

namespace skema {

bool tc_available(const skema_ctx* c) {
  (void)c;
  return false;
}

void tc_dense_window(skema_ctx* c, Mat Aw, int64_t R0, int64_t wr, float* T) {
  (void)c, (void)Aw, (void)R0, (void)wr, (void)T;
  fail(SKEMA_EUNSUPPORTED, "tensor-core sketch not built");
}

}  // namespace skema
