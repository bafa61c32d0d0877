// v3dm_match_tc.cu -- tcgen05 matching kernel (placeholder until the kernel lands).
#include "v3dm_device.cuh"

namespace v3dm {
struct TcPlan {
  int device;
};
cudaError_t tc_plan_create(TcPlan** p, int device) {
  *p = new TcPlan{device};
  return cudaSuccess;
}
void tc_plan_destroy(TcPlan* p) { delete p; }
cudaError_t tc_plan_bind(TcPlan*, const uint8_t*, int, const uint8_t*, int) { return cudaErrorNotSupported; }
cudaError_t launch_match_tc(TcPlan*, const MatchArgs&, cudaStream_t, int*) { return cudaErrorNotSupported; }
}  // namespace v3dm
namespace v3dm {
int tc_segments(TcPlan*) { return 1; }
}
