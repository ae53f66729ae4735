// Plain engine placeholder (replaced by the whole-GPU single-query engine).
#include "engine_host.h"

namespace vine {

void PlainWorkspace::release() {
  cudaFree(vs);
  cudaFree(nearq);
  cudaFree(far[0]);
  cudaFree(far[1]);
  cudaFree(table);
  cudaFree(table_used);
  cudaFree(locks);
  cudaFree(pool);
  cudaFree(sinklist);
  cudaFree(ctl);
  cudaFreeHost(ctl_host);
  *this = PlainWorkspace();
}

int plain_run(vine_graph *, const Resolved &, int32_t, const int32_t *, const int32_t *,
              const float *, const DeviceOutputs &, cudaStream_t, Label **) {
  return fail(VINE_ERR_INVALID, "plain engine not available in this build");
}

}  // namespace vine
