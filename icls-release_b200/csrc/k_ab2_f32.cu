// k_ab2_f32.cu — the AB2 predictor of the FP32 form (ab2.cuh), compiled
// without -fmad=false: multiply-add contraction shortens the kernel's
// dependent arithmetic chains.
#include "ab2.cuh"

namespace icls {

void ab2_launch_f32(Ctx& c, const MomArgs& a, int o) { ab2_launch<float>(c, a, o); }

}  // namespace icls
