// External neighbour lists (the LAMMPS interface) on the device: the
// entries of every centre built from the MD code's own full neighbour lists
// (PairHDNNP::transferNeighborList + InterfaceLammps::addNeighbor,
// pair_hdnnp.cpp:274-290, InterfaceLammps.cpp:410-441), and the transposed
// lists (for every local or ghost atom the entries that name it) from which
// kGatherTargets sums the forces.
//
//   kExtEntries<0/1>   warp per centre: count, then write, the candidates of
//                      mapped types within the pair cutoff and the model's
//                      largest cutoff, in list order (ballot compaction)
//   kExtTargetCount    entries per target (integer atomics: exact)
//   kExtTargetFill     entries into their target's segment (any order) ...
//   kExtTargetSort     ... then each segment ordered by entry index (rank
//                      sort, warp per target): the gather order, and so the
//                      forces, do not depend on timing
//   kExtTargetCentre   target -> centre map
#include "kernels.hpp"
#include "kernels_common.cuh"

namespace n2p2b200 {

namespace {

constexpr int kExtMaxEntries = 1024;   // per centre: the last symmetry-function tier's stage

template <int PASS>
__global__ void __launch_bounds__(256) kExtEntries(ExtRawView r, BatchView b)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < b.N; c += warpsPerGrid)
    {
        const int i = r.centerIndex[c];
        const double xi = r.x[3 * (size_t)i], yi = r.x[3 * (size_t)i + 1], zi = r.x[3 * (size_t)i + 2];
        const int64_t p0 = r.candOffset[c], p1 = r.candOffset[c + 1];
        int64_t base = 0;
        if (PASS == 1) base = b.nbrOffset[c];
        int count = 0;
        for (int64_t q0 = p0; q0 < p1; q0 += 32)
        {
            const int64_t q = q0 + lane;
            bool ok = false;
            int j = 0, e = -1;
            double rx = 0.0, ry = 0.0, rz = 0.0, d = 0.0;
            if (q < p1)
            {
                j = r.cand[q];
                if (j < 0 || j >= r.numAll)
                {
                    atomicAdd(&b.status->badInput, 1);
                    j = i;   // in bounds; its type check below decides nothing: ok stays false
                }
                const int t = (j == i) ? 0 : r.type[j];
                e = (t >= 1 && t <= r.numTypes) ? r.typeElement[t] : -1;
                if (e >= 0)
                {
                    // the pair style's arithmetic, no contraction
                    const double dx = __dsub_rn(xi, r.x[3 * (size_t)j]);
                    const double dy = __dsub_rn(yi, r.x[3 * (size_t)j + 1]);
                    const double dz = __dsub_rn(zi, r.x[3 * (size_t)j + 2]);
                    const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                    if (d2 <= r.pairCut2)
                    {
                        // InterfaceLammps::addNeighbor's unit conversion
                        rx = __dmul_rn(dx, r.cflength);
                        ry = __dmul_rn(dy, r.cflength);
                        rz = __dmul_rn(dz, r.cflength);
                        d = __dmul_rn(__dsqrt_rn(d2), r.cflength);
                        if (r.normalize)
                        {
                            rx = __dmul_rn(rx, r.convLength);
                            ry = __dmul_rn(ry, r.convLength);
                            rz = __dmul_rn(rz, r.convLength);
                            d = __dmul_rn(d, r.convLength);
                        }
                        // every group needs d < r_c: entries beyond the largest cutoff add nothing
                        ok = d <= r.rcmax;
                    }
                }
                else if (j != i && (t < 1 || t > r.numTypes)) atomicAdd(&b.status->badInput, 1);
            }
            const unsigned m = __ballot_sync(kFullMask, ok);
            if (PASS == 1 && ok)
            {
                const int64_t at = base + count + __popc(m & ((1u << lane) - 1u));
                if (at < b.nbrCapacity)
                {
                    b.nbrJ[at] = j;
                    b.nbrElem[at] = (uint8_t)e;
                    b.nbrD[at] = d;
                    b.nbrDx[at] = rx;
                    b.nbrDy[at] = ry;
                    b.nbrDz[at] = rz;
                }
            }
            count += __popc(m);
        }
        if (PASS == 0 && lane == 0)
        {
            b.nbrCount[c] = count;
            if (count > kExtMaxEntries) atomicAdd(&b.status->badInput, 1);
        }
    }
}

__global__ void kExtTargetCount(BatchView b, int numTargets, int* __restrict__ tCount)
{
    const int64_t total = b.status->totalNeighbors < b.nbrCapacity ? b.status->totalNeighbors : b.nbrCapacity;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    {
        const int k = b.nbrJ[e];
        if (k >= 0 && k < numTargets) atomicAdd(&tCount[k], 1);
        else atomicAdd(&b.status->badInput, 1);
    }
}

__global__ void kExtTargetFill(BatchView b, int numTargets, const int64_t* __restrict__ tOffset,
                               int* __restrict__ tFill, int64_t* __restrict__ tEntryTmp)
{
    const int64_t total = b.status->totalNeighbors < b.nbrCapacity ? b.status->totalNeighbors : b.nbrCapacity;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    {
        const int k = b.nbrJ[e];
        if (k < 0 || k >= numTargets) continue;
        const int slot = atomicAdd(&tFill[k], 1);
        tEntryTmp[tOffset[k] + slot] = e;
    }
}

// Entry indices are unique: an entry's rank in its segment is the number of
// smaller ones.
__global__ void __launch_bounds__(256) kExtTargetSort(int numTargets, const int64_t* __restrict__ tOffset,
                                                      const int64_t* __restrict__ tEntryTmp,
                                                      int64_t* __restrict__ tEntry)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < numTargets; k += warpsPerGrid)
    {
        const int64_t s0 = tOffset[k], s1 = tOffset[k + 1];
        for (int64_t a = s0 + lane; a < s1; a += 32)
        {
            const int64_t v = tEntryTmp[a];
            int64_t rank = 0;
            for (int64_t q = s0; q < s1; ++q) rank += tEntryTmp[q] < v ? 1 : 0;
            tEntry[s0 + rank] = v;
        }
    }
}

__global__ void kExtTargetCentre(int numCenters, const int* __restrict__ centerIndex, int numTargets,
                                 int* __restrict__ targetCenter)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < numCenters; c += gridDim.x * blockDim.x)
    {
        const int k = centerIndex[c];
        if (k >= 0 && k < numTargets) targetCenter[k] = c;
    }
}

int blocksFor(int64_t n, int threads, int sms, int perSM)
{
    int64_t need = (n + threads - 1) / threads;
    int64_t cap = (int64_t)sms * perSM;
    return (int)(need < 1 ? 1 : (need < cap ? need : cap));
}

} // namespace

void launchExternalEntries(ExtRawView const& r, BatchView const& b, int64_t* scanTmp, int sms, cudaStream_t st)
{
    const int blocks = blocksFor((int64_t)b.N * 32, 256, sms, 16);
    kExtEntries<0><<<blocks, 256, 0, st>>>(r, b);
    launchExclusiveScan(b.N, b.nbrCount, b.nbrOffset, scanTmp, &b.status->totalNeighbors, st);
    kExtEntries<1><<<blocks, 256, 0, st>>>(r, b);
}

void launchExternalTranspose(BatchView const& b, int numTargets, const int* centerIndex, int* tCount, int* tFill,
                             int64_t* tOffset, int64_t* tEntryTmp, int64_t* tEntry, int* targetCenter,
                             int64_t* scanTmp, int sms, cudaStream_t st)
{
    cudaMemsetAsync(tCount, 0, sizeof(int) * (size_t)numTargets, st);
    cudaMemsetAsync(tFill, 0, sizeof(int) * (size_t)numTargets, st);
    cudaMemsetAsync(targetCenter, 0xff, sizeof(int) * (size_t)numTargets, st);   // -1
    const int eb = sms * 16;
    kExtTargetCount<<<eb, 256, 0, st>>>(b, numTargets, tCount);
    launchExclusiveScan(numTargets, tCount, tOffset, scanTmp, nullptr, st);
    kExtTargetFill<<<eb, 256, 0, st>>>(b, numTargets, tOffset, tFill, tEntryTmp);
    kExtTargetSort<<<blocksFor((int64_t)numTargets * 32, 256, sms, 16), 256, 0, st>>>(numTargets, tOffset, tEntryTmp,
                                                                                    tEntry);
    kExtTargetCentre<<<blocksFor(b.N, 256, sms, 8), 256, 0, st>>>(b.N, centerIndex, numTargets, targetCenter);
}

} // namespace n2p2b200
