// FP64 instances of the symmetry-function passes, and the precision dispatch.
#include "sf_launch.cuh"

namespace n2p2b200 {

namespace {

// Words of acceptance ballots the G pass records for atom i: two per 64
// candidates of every angular group (the candidate counts of roundPhases,
// from the numbers of neighbours of each element inside the group's cutoff
// when the stage is sorted by distance, else of all neighbours).
__global__ void kMaskWords(DevModel model, BatchView b)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        const int64_t off = b.nbrOffset[i], end = b.nbrOffset[i + 1];
        // per cutoff slot the neighbour counts of elements 0-3 and 4-7 in 16-bit fields: exact up to
        // 65535 entries per atom, far beyond the 1024 of the last stage tier (larger atoms are flagged
        // by the symmetry-function passes and write no masks)
        uint64_t lo[4] = {0, 0, 0, 0}, hi[4] = {0, 0, 0, 0};
        if (end <= b.nbrCapacity)
            for (int64_t q = off + lane; q < end; q += 32)
            {
                const int e = b.nbrElem[q];
                const double d = b.nbrD[q];
                const uint64_t one = 1ull << (16 * (e & 3));
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    if (c < model.numCutoffSlots && (!model.sortByDistance || d < model.cutoff[c].rc))
                    {
                        if (e < 4) lo[c] += one;
                        else hi[c] += one;
                    }
            }
        int cnt[4][kDevMaxElements];
#pragma unroll
        for (int c = 0; c < 4; ++c)
        {
            uint64_t l = lo[c], h = hi[c];
            for (int o = 16; o > 0; o >>= 1)
            {
                l += __shfl_xor_sync(kFullMask, l, o);
                h += __shfl_xor_sync(kFullMask, h, o);
            }
#pragma unroll
            for (int f = 0; f < 4; ++f)
            {
                cnt[c][f] = (int)((l >> (16 * f)) & 0xffff);
                cnt[c][f + 4] = (int)((h >> (16 * f)) & 0xffff);
            }
        }
        DevElement const& E = model.el[b.elem[i]];
        int words = 0;
        for (int g = 0; g < E.groupCount; ++g)
        {
            DevGroup const& G = model.groups[E.groupBegin + g];
            if (G.type == 2) continue;
            const int nA = cnt[G.cutoffSlot][G.e1], nB = cnt[G.cutoffSlot][G.e2];
            int64_t count;
            if (G.e1 == G.e2)
            {
                const int m = nA + (nA & 1);
                count = nA < 2 ? 0 : (int64_t)(m - 1) * (m / 2);
            }
            else count = (int64_t)nA * nB;
            words += 2 * (int)((count + 63) / 64);
        }
        if (lane == 0) b.maskWords[i] = words;
    }
}

} // namespace

void launchMaskOffsets(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    int blocks = (b.N + 7) / 8;
    if (blocks < 1) blocks = 1;
    if (blocks > sms * 16) blocks = sms * 16;
    kMaskWords<<<blocks, 256, 0, st>>>(m, b);
    launchExclusiveScan(b.N, b.maskWords, b.maskOffset, b.scanTmp, &b.status->maskWords, st);
}

void launchSFValuesF64(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st,
                       int variant)
{
    valuesT<double>(m, gt, b, sms, st, variant);
}

void launchSFForcesF64(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st,
                       int variant)
{
    forcesT<double>(m, gt, b, sms, st, variant);
}

void launchSFValues(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int precision, int sms,
                    cudaStream_t st, int variant)
{
    if (precision == 0) launchSFValuesF64(m, gt, b, sms, st, variant);
    else launchSFValuesF32(m, gt, b, sms, st, variant);
}

void launchSFForces(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int precision, int sms,
                    cudaStream_t st, int variant)
{
    if (precision == 0) launchSFForcesF64(m, gt, b, sms, st, variant);
    else launchSFForcesF32(m, gt, b, sms, st, variant);
}

} // namespace n2p2b200
