// FP32 instances of the symmetry-function passes (mixed precision form).
#include "sf_launch.cuh"

namespace n2p2b200 {

void launchSFValuesF32(DevModel const& m, BatchView const& b, int sms, cudaStream_t st, int variant)
{
    valuesT<float>(m, b, sms, st, variant);
}

void launchSFForcesF32(DevModel const& m, BatchView const& b, int sms, cudaStream_t st, int variant)
{
    forcesT<float>(m, b, sms, st, variant);
}

} // namespace n2p2b200
