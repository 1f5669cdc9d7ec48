// FP64 instances of the symmetry-function passes, and the precision dispatch.
#include "sf_launch.cuh"

namespace n2p2b200 {

void launchSFValuesF64(DevModel const& m, BatchView const& b, int sms, cudaStream_t st, int variant)
{
    valuesT<double>(m, b, sms, st, variant);
}

void launchSFForcesF64(DevModel const& m, BatchView const& b, int sms, cudaStream_t st, int variant)
{
    forcesT<double>(m, b, sms, st, variant);
}

void launchSFValues(DevModel const& m, BatchView const& b, int precision, int sms, cudaStream_t st, int variant)
{
    if (precision == 0) launchSFValuesF64(m, b, sms, st, variant);
    else launchSFValuesF32(m, b, sms, st, variant);
}

void launchSFForces(DevModel const& m, BatchView const& b, int precision, int sms, cudaStream_t st, int variant)
{
    if (precision == 0) launchSFForcesF64(m, b, sms, st, variant);
    else launchSFForcesF32(m, b, sms, st, variant);
}

} // namespace n2p2b200
