// Neighbour list of one structure into caller-owned device buffers, without
// any device allocation.
//
// Why: some callers cannot call cudaMalloc at the point where they need a
// neighbour list -- a host code whose device memory is owned by its own pool
// allocator, or a step loop that must not pay cudaMalloc's implicit device
// synchronisation.  They pass
// the positions and the output arrays; the scratch memory the build needs
// (cell lists, per-atom counts, scan partials, a status word) lives in one
// file-scope __device__ array of fixed size that every GPU loading the
// library holds until the process exits.
//
// The arithmetic, the candidate search and the ordering are those of the
// batched neighbour build (k_neighbor.cu), so the results are bit-identical
// to the entries n2p2_batch_get_neighbors returns for the same structure.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "kernels_common.cuh"
#include "kernels.hpp"

namespace n2p2b200 {

// Limits of the allocation-free build (documented in include/n2p2_b200.h).
constexpr int kNaMaxAtoms = 8192;
constexpr int kNaMaxCells = 32768;
constexpr int kNaMaxNeighbors = 256;   // per atom (ordering happens in shared memory)

namespace {

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Scratch carve-up (bytes).
constexpr size_t kOffAtomCell = 0;
constexpr size_t kOffAtomSlot = kOffAtomCell + align256(sizeof(int) * kNaMaxAtoms);
constexpr size_t kOffCount = kOffAtomSlot + align256(sizeof(int) * kNaMaxAtoms);
constexpr size_t kOffCellAtoms = kOffCount + align256(sizeof(int) * kNaMaxAtoms);
constexpr size_t kOffCellCount = kOffCellAtoms + align256(sizeof(int) * kNaMaxAtoms);
constexpr size_t kOffCellStart = kOffCellCount + align256(sizeof(int) * kNaMaxCells);
constexpr size_t kOffCellStart64 = kOffCellStart + align256(sizeof(int) * kNaMaxCells);
constexpr size_t kOffTiles = kOffCellStart64 + align256(sizeof(int64_t) * (kNaMaxCells + 1));
constexpr size_t kOffStatus = kOffTiles + align256(sizeof(int64_t) * 64);
constexpr size_t kScratchBytes = kOffStatus + align256(sizeof(int) * 8);

} // namespace

// The shared scratch of the allocation-free entry point.  In host code the
// name is only a handle: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

namespace {

__device__ __forceinline__ int naFloorDiv(int a, int b)
{
    int q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
    return q;
}

__device__ __forceinline__ double naPair(double ri, double rj, double const* box, int c, int b0, int b1, int b2)
{
    double v = __dsub_rn(ri, rj);
    v = __dadd_rn(v, __dmul_rn(box[0 * 3 + c], (double)b0));
    v = __dadd_rn(v, __dmul_rn(box[1 * 3 + c], (double)b1));
    v = __dadd_rn(v, __dmul_rn(box[2 * 3 + c], (double)b2));
    return v;
}

__global__ void kNaAssign(int N, DevStructInfo s, const double* __restrict__ r, int* __restrict__ atomCell,
                          int* __restrict__ atomSlot, int* __restrict__ cellCount, int* __restrict__ status)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    {
        int c3[3] = {0, 0, 0};
        if (s.periodic)
        {
            for (int a = 0; a < 3; ++a)
            {
                double f = s.invbox[0 * 3 + a] * r[3 * i] + s.invbox[1 * 3 + a] * r[3 * i + 1] +
                           s.invbox[2 * 3 + a] * r[3 * i + 2];
                if (!(f > -1e-9 && f < 1.0 + 1e-9)) atomicOr(&status[0], 1);   // not inside the cell
                f -= floor(f);
                int c = (int)floor(f * s.nc[a]);
                c3[a] = min(max(c, 0), s.nc[a] - 1);
            }
        }
        const int cell = (c3[0] * s.nc[1] + c3[1]) * s.nc[2] + c3[2];
        atomCell[i] = cell;
        atomSlot[i] = atomicAdd(&cellCount[cell], 1);
    }
}

__global__ void kNaScatter(int N, const int* __restrict__ atomCell, const int* __restrict__ atomSlot,
                           const int64_t* __restrict__ cellStart64, int* __restrict__ cellAtoms)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        cellAtoms[(int)cellStart64[atomCell[i]] + atomSlot[i]] = i;
}

// PASS 0 counts; PASS 1 collects the atom's entries in shared memory, orders
// them by (j, image) and writes them to the caller's arrays.
template <int PASS>
__global__ void __launch_bounds__(128) kNaSearch(int N, double rc2, DevStructInfo s, const double* __restrict__ r,
                                                 const int* __restrict__ atomCell, const int64_t* __restrict__ cellStart,
                                                 const int* __restrict__ cellCount, const int* __restrict__ cellAtoms,
                                                 int* __restrict__ count, const int64_t* __restrict__ offsets,
                                                 int64_t capacity, int32_t* __restrict__ outIndex,
                                                 int32_t* __restrict__ outImage, double* __restrict__ outD,
                                                 double* __restrict__ outDr, int* __restrict__ status)
{
    __shared__ int64_t sKey[4][kNaMaxNeighbors];
    __shared__ double sD[4][kNaMaxNeighbors];
    __shared__ double sDr[4][kNaMaxNeighbors][3];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int K = (2 * s.pbc[0] + 1) * (2 * s.pbc[1] + 1) * (2 * s.pbc[2] + 1);
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const double xi = r[3 * i], yi = r[3 * i + 1], zi = r[3 * i + 2];
        const int local = atomCell[i];
        const int cz = local % s.nc[2];
        const int cy = (local / s.nc[2]) % s.nc[1];
        const int cx = local / (s.nc[2] * s.nc[1]);
        int n = 0;
        for (int ox = -s.stencil[0]; ox <= s.stencil[0]; ++ox)
        {
            const int qx = cx + ox, tx = naFloorDiv(qx, s.nc[0]), wx = qx - tx * s.nc[0], b0 = -tx;
            if (b0 < -s.pbc[0] || b0 > s.pbc[0]) continue;
            for (int oy = -s.stencil[1]; oy <= s.stencil[1]; ++oy)
            {
                const int qy = cy + oy, ty = naFloorDiv(qy, s.nc[1]), wy = qy - ty * s.nc[1], b1 = -ty;
                if (b1 < -s.pbc[1] || b1 > s.pbc[1]) continue;
                for (int oz = -s.stencil[2]; oz <= s.stencil[2]; ++oz)
                {
                    const int qz = cz + oz, tz = naFloorDiv(qz, s.nc[2]), wz = qz - tz * s.nc[2], b2 = -tz;
                    if (b2 < -s.pbc[2] || b2 > s.pbc[2]) continue;
                    const int cell = (wx * s.nc[1] + wy) * s.nc[2] + wz;
                    const int cnt = cellCount[cell];
                    const int start = (int)cellStart[cell];
                    for (int t0 = 0; t0 < cnt; t0 += 32)
                    {
                        const int t = t0 + lane;
                        bool hit = false;
                        double dx = 0, dy = 0, dz = 0, d2 = 0;
                        int j = -1;
                        if (t < cnt)
                        {
                            j = cellAtoms[start + t];
                            if (!(j == i && b0 == 0 && b1 == 0 && b2 == 0))
                            {
                                dx = naPair(xi, r[3 * j], s.box, 0, b0, b1, b2);
                                dy = naPair(yi, r[3 * j + 1], s.box, 1, b0, b1, b2);
                                dz = naPair(zi, r[3 * j + 2], s.box, 2, b0, b1, b2);
                                d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                                hit = (d2 <= rc2);
                            }
                        }
                        const unsigned m = __ballot_sync(kFullMask, hit);
                        if (PASS == 1 && hit)
                        {
                            const int pos = n + __popc(m & ((1u << lane) - 1u));
                            if (pos < kNaMaxNeighbors)
                            {
                                const int code = ((b0 + s.pbc[0]) * (2 * s.pbc[1] + 1) + (b1 + s.pbc[1])) *
                                                     (2 * s.pbc[2] + 1) +
                                                 (b2 + s.pbc[2]);
                                sKey[w][pos] = (int64_t)j * K + code;
                                sD[w][pos] = __dsqrt_rn(d2);
                                sDr[w][pos][0] = dx;
                                sDr[w][pos][1] = dy;
                                sDr[w][pos][2] = dz;
                            }
                        }
                        n += __popc(m);
                    }
                }
            }
        }
        if (PASS == 0)
        {
            if (lane == 0)
            {
                count[i] = n;
                if (n > kNaMaxNeighbors) atomicOr(&status[0], 2);
            }
            continue;
        }
        __syncwarp();
        const int64_t off = offsets[i];
        if (n <= kNaMaxNeighbors && off + n <= capacity)
        {
            for (int e = lane; e < n; e += 32)
            {
                const int64_t k = sKey[w][e];
                int rank = 0;
                for (int q = 0; q < n; ++q) rank += (sKey[w][q] < k) ? 1 : 0;
                const int64_t dst = off + rank;
                outIndex[dst] = (int32_t)(k / K);
                outImage[dst] = (int32_t)(k % K);
                outD[dst] = sD[w][e];
                outDr[3 * dst + 0] = sDr[w][e][0];
                outDr[3 * dst + 1] = sDr[w][e][1];
                outDr[3 * dst + 2] = sDr[w][e][2];
            }
        }
        else if (lane == 0)
        {
            atomicOr(&status[0], 4);
        }
        __syncwarp();
    }
}

struct DeviceScratch
{
    unsigned char* ptr = nullptr;
};

std::mutex g_naMutex;
DeviceScratch g_naScratch[64];

// Device address of the scratch array on the current device (looked up once
// per device and kept for the process's life, so it is stale after a
// cudaDeviceReset; the first call must not happen during stream capture).
unsigned char* scratchForCurrentDevice()
{
    int dev = 0;
    cudaCheck(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) throw std::runtime_error("ERROR: device index out of range.\n");
    std::lock_guard<std::mutex> lock(g_naMutex);
    if (!g_naScratch[dev].ptr)
    {
        void* p = nullptr;
        cudaCheck(cudaGetSymbolAddress(&p, g_noallocScratch), "cudaGetSymbolAddress");
        g_naScratch[dev].ptr = static_cast<unsigned char*>(p);
    }
    return g_naScratch[dev].ptr;
}

} // namespace

void neighborListNoAlloc(const double* positions, int64_t numAtoms, const double* box, double cutoff,
                         int64_t capacity, int64_t* offsets, int32_t* index, int32_t* image, double* d, double* dr,
                         int64_t* numEntries, cudaStream_t st)
{
    if (numAtoms <= 0 || numAtoms > kNaMaxAtoms)
        throw std::runtime_error("ERROR: the allocation-free neighbour list takes 1.." + std::to_string(kNaMaxAtoms) +
                                 " atoms.\n");
    if (!(cutoff > 0.0)) throw std::runtime_error("ERROR: cutoff must be positive.\n");
    const int N = (int)numAtoms;
    DevStructInfo s;
    std::memset(&s, 0, sizeof(s));
    s.numAtoms = N;
    if (box)
    {
        s.periodic = 1;
        std::memcpy(s.box, box, sizeof(s.box));
        inverseBoxOf(s.box, s.invbox);
        structureGeometry(s, cutoff);
    }
    else
    {
        s.nc[0] = s.nc[1] = s.nc[2] = 1;
    }
    const int64_t cells = (int64_t)s.nc[0] * s.nc[1] * s.nc[2];
    if (cells > kNaMaxCells) throw std::runtime_error("ERROR: the allocation-free neighbour list takes at most " +
                                                      std::to_string(kNaMaxCells) + " cells; the box is too large.\n");
    unsigned char* base = scratchForCurrentDevice();
    int* atomCell = reinterpret_cast<int*>(base + kOffAtomCell);
    int* atomSlot = reinterpret_cast<int*>(base + kOffAtomSlot);
    int* count = reinterpret_cast<int*>(base + kOffCount);
    int* cellAtoms = reinterpret_cast<int*>(base + kOffCellAtoms);
    int* cellCount = reinterpret_cast<int*>(base + kOffCellCount);
    int64_t* cellStart64 = reinterpret_cast<int64_t*>(base + kOffCellStart64);
    int64_t* tiles = reinterpret_cast<int64_t*>(base + kOffTiles);
    int* status = reinterpret_cast<int*>(base + kOffStatus);
    // The scratch keeps the previous call's contents: clear what must start at zero.
    cudaCheck(cudaMemsetAsync(cellCount, 0, sizeof(int) * cells, st), "memset");
    cudaCheck(cudaMemsetAsync(status, 0, sizeof(int) * 8, st), "memset");
    const int blocks = (N + 127) / 128;
    kNaAssign<<<blocks, 128, 0, st>>>(N, s, positions, atomCell, atomSlot, cellCount, status);
    launchExclusiveScan((int)cells, cellCount, cellStart64, tiles, nullptr, st);
    kNaScatter<<<blocks, 128, 0, st>>>(N, atomCell, atomSlot, cellStart64, cellAtoms);
    const int wblocks = (N + 3) / 4;
    const double rc2 = cutoff * cutoff;
    kNaSearch<0><<<wblocks, 128, 0, st>>>(N, rc2, s, positions, atomCell, cellStart64, cellCount, cellAtoms, count,
                                          nullptr, 0, nullptr, nullptr, nullptr, nullptr, status);
    launchExclusiveScan(N, count, offsets, tiles, nullptr, st);
    kNaSearch<1><<<wblocks, 128, 0, st>>>(N, rc2, s, positions, atomCell, cellStart64, cellCount, cellAtoms, count,
                                          offsets, capacity, index, image, d, dr, status);
    cudaCheck(cudaGetLastError(), "kernel launch");
    // Recorded into the caller's graph: no host copy and no wait (neither may be captured); the
    // count and the limit checks are read after a replay by neighborListNoAllocStatus.
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    cudaCheck(cudaStreamIsCapturing(st, &capture), "cudaStreamIsCapturing");
    if (capture != cudaStreamCaptureStatusNone)
    {
        if (numEntries) *numEntries = -1;
        return;
    }
    neighborListNoAllocStatus(numAtoms, offsets, capacity, numEntries, st);
}

void neighborListNoAllocStatus(int64_t numAtoms, const int64_t* offsets, int64_t capacity, int64_t* numEntries,
                               cudaStream_t st)
{
    if (numAtoms <= 0 || numAtoms > kNaMaxAtoms)
        throw std::runtime_error("ERROR: the allocation-free neighbour list takes 1.." + std::to_string(kNaMaxAtoms) +
                                 " atoms.\n");
    const int* status = reinterpret_cast<const int*>(scratchForCurrentDevice() + kOffStatus);
    int hostStatus = 0;
    int64_t total = 0;
    cudaCheck(cudaMemcpyAsync(&total, offsets + numAtoms, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "D2H");
    cudaCheck(cudaMemcpyAsync(&hostStatus, status, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
    cudaCheck(cudaStreamSynchronize(st), "synchronize");
    if (numEntries) *numEntries = total;
    if (hostStatus & 1) throw std::runtime_error("ERROR: atoms outside the cell (fold positions into the box first).\n");
    if (hostStatus & 2)
        throw std::runtime_error("ERROR: more than " + std::to_string(kNaMaxNeighbors) +
                                 " neighbours of one atom (allocation-free limit).\n");
    if (total > capacity) throw std::runtime_error("ERROR: output capacity too small: " + std::to_string(total) +
                                                   " entries needed.\n");
    if (hostStatus & 4) throw std::runtime_error("ERROR: neighbour output incomplete.\n");
}

} // namespace n2p2b200
