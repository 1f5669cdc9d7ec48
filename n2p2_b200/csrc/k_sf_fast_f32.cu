// FP32 instances of the symmetry-function passes (mixed precision form).
#include "sf_launch.cuh"

namespace n2p2b200 {

void launchSFValuesF32(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st,
                       int variant)
{
    valuesT<float>(m, gt, b, sms, st, variant);
}

void launchSFForcesF32(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st,
                       int variant)
{
    forcesT<float>(m, gt, b, sms, st, variant);
}

} // namespace n2p2b200
