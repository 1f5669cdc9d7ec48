// Neighbour-list build on sm_100a: remap, cell binning, candidate search over
// a periodic cell stencil, per-atom ordering and the reverse-entry index.
//
// Result contract (Structure::calculateNeighborList, Structure.cpp:287-398):
// for every atom i the entries are all (j, image) with
//     dr = r_i - r_j + bc0*box0 + bc1*box1 + bc2*box2,   dr.dr <= rc^2,
// excluding (i, 0), ordered by j ascending then (bc0, bc1, bc2)
// lexicographically, with d = sqrt(dr.dr).  Every floating-point step uses
// explicit round-to-nearest intrinsics in the reference's evaluation order
// (Vec3D.h:294-361), so d and dr are bit-identical to the reference.
#include "kernels_common.cuh"
#include "kernels.hpp"

namespace n2p2b200 {

namespace {

__device__ __forceinline__ int floorDiv(int a, int b)
{
    int q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
    return q;
}

__device__ __forceinline__ int imageCode(int bc0, int bc1, int bc2, int const* p)
{
    return ((bc0 + p[0]) * (2 * p[1] + 1) + (bc1 + p[1])) * (2 * p[2] + 1) + (bc2 + p[2]);
}

__device__ __forceinline__ void imageFromCode(int code, int const* p, int& bc0, int& bc1, int& bc2)
{
    int n2 = 2 * p[2] + 1, n1 = 2 * p[1] + 1;
    bc2 = code % n2 - p[2];
    code /= n2;
    bc1 = code % n1 - p[1];
    code /= n1;
    bc0 = code - p[0];
}

// dr = r_i - r_j + bc0*b0 + bc1*b1 + bc2*b2, component c, no contraction.
__device__ __forceinline__ double pairComponent(double ri, double rj, double const* box, int c, int bc0, int bc1,
                                                int bc2)
{
    double v = __dsub_rn(ri, rj);
    v = __dadd_rn(v, __dmul_rn(box[0 * 3 + c], (double)bc0));
    v = __dadd_rn(v, __dmul_rn(box[1 * 3 + c], (double)bc1));
    v = __dadd_rn(v, __dmul_rn(box[2 * 3 + c], (double)bc2));
    return v;
}

__device__ __forceinline__ double norm2Exact(double x, double y, double z)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}

} // namespace

// Structure::remap (Structure.cpp:1224-1248) in physical units, then
// Atom::toNormalizedUnits' r *= convLength (Atom.cpp:78-85).
__global__ void kPreparePositions(int N, const int* __restrict__ atomStruct, const DevStructInfo* __restrict__ info,
                                  const double* __restrict__ rin, double* __restrict__ px, double* __restrict__ py,
                                  double* __restrict__ pz, int doRemap, int doNormalize, double convLength)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    {
        DevStructInfo const& s = info[atomStruct[i]];
        double r[3] = {rin[3 * i + 0], rin[3 * i + 1], rin[3 * i + 2]};
        if (doRemap && s.periodic)
        {
            double f[3];
            for (int c = 0; c < 3; ++c)
            {
                double t = __dmul_rn(s.invboxPhys[0 * 3 + c], r[0]);
                t = __dadd_rn(t, __dmul_rn(s.invboxPhys[1 * 3 + c], r[1]));
                t = __dadd_rn(t, __dmul_rn(s.invboxPhys[2 * 3 + c], r[2]));
                f[c] = t;
            }
            for (int c = 0; c < 3; ++c)
            {
                if (f[c] > 1.0) f[c] = __dsub_rn(f[c], (double)(int)f[c]);
                if (f[c] < 0.0) f[c] = __dadd_rn(f[c], __dsub_rn(1.0, (double)(int)f[c]));
                if (f[c] == 1.0) f[c] = 0.0;
            }
            for (int c = 0; c < 3; ++c)
            {
                double t = __dmul_rn(s.boxPhys[0 * 3 + c], f[0]);
                t = __dadd_rn(t, __dmul_rn(s.boxPhys[1 * 3 + c], f[1]));
                t = __dadd_rn(t, __dmul_rn(s.boxPhys[2 * 3 + c], f[2]));
                r[c] = t;
            }
        }
        if (doNormalize)
        {
            for (int c = 0; c < 3; ++c) r[c] = __dmul_rn(r[c], convLength);
        }
        px[i] = r[0];
        py[i] = r[1];
        pz[i] = r[2];
    }
}

// Cell of every atom: fractional coordinate f = r . invbox, cell = floor(f*nc).
__global__ void kAssignCells(int N, const int* __restrict__ atomStruct, const DevStructInfo* __restrict__ info,
                             const double* __restrict__ px, const double* __restrict__ py,
                             const double* __restrict__ pz, int* __restrict__ atomCell, int* __restrict__ atomSlot,
                             int* __restrict__ cellCount)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    {
        DevStructInfo const& s = info[atomStruct[i]];
        int c3[3] = {0, 0, 0};
        if (s.periodic)
        {
            double r[3] = {px[i], py[i], pz[i]};
            for (int a = 0; a < 3; ++a)
            {
                double f = s.invbox[0 * 3 + a] * r[0] + s.invbox[1 * 3 + a] * r[1] + s.invbox[2 * 3 + a] * r[2];
                f -= floor(f);  // positions outside the cell are folded for binning only
                int c = (int)floor(f * s.nc[a]);
                c3[a] = min(max(c, 0), s.nc[a] - 1);
            }
        }
        int cell = s.cellBegin + (c3[0] * s.nc[1] + c3[1]) * s.nc[2] + c3[2];
        atomCell[i] = cell;
        atomSlot[i] = atomicAdd(&cellCount[cell], 1);
    }
}

// Cell-ordered atom indices and positions (the position copy lets the search
// read a cell's candidates with contiguous loads).
__global__ void kScatterCells(int N, const int* __restrict__ atomCell, const int* __restrict__ atomSlot,
                              const int* __restrict__ cellStart, const double* __restrict__ px,
                              const double* __restrict__ py, const double* __restrict__ pz,
                              int* __restrict__ cellAtoms, double4* __restrict__ cellPos)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    {
        const int q = cellStart[atomCell[i]] + atomSlot[i];
        cellAtoms[q] = i;
        cellPos[q] = make_double4(px[i], py[i], pz[i], (double)i);
    }
}

// One warp per centre atom.  PASS 0 counts, PASS 1 writes the unordered
// candidates into the atom's segment of the scratch arrays; PASS 2 does both
// at once into a fixed-stride segment (i * scrStride, sized from an earlier
// evaluation's largest count), keeping the count for the scan and the sort,
// and drops entries beyond the stride.  After a PASS 2 the fill pass runs as
// well, guarded by the status (guardStride): it returns at once unless some
// atom outgrew the stride, and then writes the packed segments the sort reads
// instead, so every list is complete either way.  The stencil cells
// (with their periodic images) are tabulated in shared memory, kStencilChunk
// at a time, with an exclusive scan of their atom counts; the warp then walks
// the concatenated candidates 32 at a time (lane -> cell by binary search), so
// every lane tests a candidate whatever the cell occupancy.
constexpr int kStencilChunk = 128;
constexpr int kSearchWarps = 8;

struct StencilTable
{
    int start[kStencilChunk];
    int pre[kStencilChunk + 1];
    int code[kStencilChunk];      // (bc0 + 512) << 20 | (bc1 + 512) << 10 | (bc2 + 512)
};

template <int PASS>
__global__ void __launch_bounds__(kSearchWarps * 32) kNeighborSearch(
    int N, double rc2, const int* __restrict__ atomStruct, const DevStructInfo* __restrict__ info,
    const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
    const int* __restrict__ atomCell, const int* __restrict__ cellStart, const int* __restrict__ cellCountArr,
    const double4* __restrict__ cellPos, int* __restrict__ nbrCount, const int64_t* __restrict__ nbrOffset,
    int64_t capacity, int64_t* __restrict__ scrKey, double* __restrict__ scrD, double* __restrict__ scrDx,
    double* __restrict__ scrDy, double* __restrict__ scrDz, DevStatus* __restrict__ status, int64_t scrStride,
    int64_t guardStride)
{
    if (PASS == 1 && guardStride > 0 && status->maxNeighbors <= guardStride) return;   // the strided search fit
    __shared__ StencilTable tables[kSearchWarps];
    StencilTable& tab = tables[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warpsPerGrid)
    {
        DevStructInfo const& s = info[atomStruct[i]];
        const double xi = px[i], yi = py[i], zi = pz[i];
        const int local = atomCell[i] - s.cellBegin;
        const int cz = local % s.nc[2];
        const int cy = (local / s.nc[2]) % s.nc[1];
        const int cx = local / (s.nc[2] * s.nc[1]);
        const int K = (2 * s.pbc[0] + 1) * (2 * s.pbc[1] + 1) * (2 * s.pbc[2] + 1);
        const int nx = 2 * s.stencil[0] + 1, ny = 2 * s.stencil[1] + 1, nz = 2 * s.stencil[2] + 1;
        const int numStencil = nx * ny * nz;
        int count = 0;
        int64_t base = 0, limit = 0;
        if (PASS == 1)
        {
            base = nbrOffset[i];
            limit = nbrOffset[i + 1];
            if (limit > capacity) limit = capacity;   // overflow is flagged by the host check
        }
        else if (PASS == 2)
        {
            base = (int64_t)i * scrStride;
            limit = base + scrStride;
        }
        for (int c0 = 0; c0 < numStencil; c0 += kStencilChunk)
        {
            __syncwarp();
            int carry = 0;
            for (int k0 = 0; k0 < kStencilChunk; k0 += 32)
            {
                const int k = k0 + lane, o = c0 + k;
                int cnt = 0, start = 0, code = 0;
                if (o < numStencil)
                {
                    const int ox = o / (ny * nz) - s.stencil[0];
                    const int oy = (o / nz) % ny - s.stencil[1];
                    const int oz = o % nz - s.stencil[2];
                    const int qx = cx + ox, tx = floorDiv(qx, s.nc[0]), wx = qx - tx * s.nc[0];
                    const int qy = cy + oy, ty = floorDiv(qy, s.nc[1]), wy = qy - ty * s.nc[1];
                    const int qz = cz + oz, tz = floorDiv(qz, s.nc[2]), wz = qz - tz * s.nc[2];
                    const int bc0 = -tx, bc1 = -ty, bc2 = -tz;
                    if (bc0 >= -s.pbc[0] && bc0 <= s.pbc[0] && bc1 >= -s.pbc[1] && bc1 <= s.pbc[1] &&
                        bc2 >= -s.pbc[2] && bc2 <= s.pbc[2])
                    {
                        const int cell = s.cellBegin + (wx * s.nc[1] + wy) * s.nc[2] + wz;
                        cnt = cellCountArr[cell];
                        start = cellStart[cell];
                        code = ((bc0 + 512) << 20) | ((bc1 + 512) << 10) | (bc2 + 512);
                    }
                }
                int incl = cnt;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1)
                {
                    const int y = __shfl_up_sync(kFullMask, incl, d);
                    if (lane >= d) incl += y;
                }
                tab.start[k] = start;
                tab.code[k] = code;
                tab.pre[k] = carry + incl - cnt;
                carry += __shfl_sync(kFullMask, incl, 31);
            }
            if (lane == 0) tab.pre[kStencilChunk] = carry;
            __syncwarp();
            const int total = carry;
            for (int p0 = 0; p0 < total; p0 += 32)
            {
                const int p = p0 + lane;
                bool hit = false;
                double dx = 0, dy = 0, dz = 0, d2 = 0;
                int j = -1, bc0 = 0, bc1 = 0, bc2 = 0;
                if (p < total)
                {
                    int lo = 0, hi = kStencilChunk;   // pre[lo] <= p < pre[hi]
#pragma unroll
                    for (int it = 0; it < 7; ++it)
                    {
                        const int mid = (lo + hi) >> 1;
                        if (tab.pre[mid] <= p) lo = mid;
                        else hi = mid;
                    }
                    const int code = tab.code[lo];
                    bc0 = (code >> 20) - 512;
                    bc1 = ((code >> 10) & 1023) - 512;
                    bc2 = (code & 1023) - 512;
                    const double4 q = cellPos[tab.start[lo] + (p - tab.pre[lo])];
                    j = (int)q.w;
                    if (!(j == i && bc0 == 0 && bc1 == 0 && bc2 == 0))
                    {
                        dx = pairComponent(xi, q.x, s.box, 0, bc0, bc1, bc2);
                        dy = pairComponent(yi, q.y, s.box, 1, bc0, bc1, bc2);
                        dz = pairComponent(zi, q.z, s.box, 2, bc0, bc1, bc2);
                        d2 = norm2Exact(dx, dy, dz);
                        hit = (d2 <= rc2);
                    }
                }
                if constexpr (PASS == 0)
                {
                    count += hit ? 1 : 0;
                }
                else
                {
                    const unsigned m = __ballot_sync(kFullMask, hit);
                    const int pos = __popc(m & ((1u << lane) - 1u));
                    if (hit)
                    {
                        const int64_t e = base + count + pos;
                        if (e < limit)
                        {
                            scrKey[e] = (int64_t)(j - s.atomBegin) * K + imageCode(bc0, bc1, bc2, s.pbc);
                            scrD[e] = __dsqrt_rn(d2);
                            scrDx[e] = dx;
                            scrDy[e] = dy;
                            scrDz[e] = dz;
                        }
                    }
                    count += __popc(m);
                }
            }
        }
        if (PASS != 1)
        {
            if (PASS == 0) count = warpSumInt(count);   // PASS 2 counts warp-wide already
            if (lane == 0)
            {
                nbrCount[i] = count;
                atomicMax(&status->maxNeighbors, count);
            }
        }
    }
}

// Orders every atom's segment by key = (j - atomBegin) * K + imageCode, i.e.
// j ascending, then images in the reference loop order.  Rank sort: keys are
// unique within a segment, so an entry's rank is the number of smaller keys.
// Ranks of the lane's keys e = lane + 32 r (r < R) among the segment's n
// unique keys: one pass over the keys for all R of them.
template <int R>
__device__ __forceinline__ void rankKeys32(const int* keys, int n, int lane, int (&kk)[8], int (&rank)[8])
{
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        const int e = lane + 32 * r;
        kk[r] = e < n ? keys[e] : 0x7fffffff;
        rank[r] = 0;
    }
#pragma unroll 4
    for (int q = 0; q < n; ++q)
    {
        const int kq = keys[q];
#pragma unroll
        for (int r = 0; r < R; ++r) rank[r] += kq < kk[r] ? 1 : 0;
    }
}

// Four blocks per SM (at most 64 registers): the sort waits on global loads,
// and 32 resident warps hide more of that wait than the 24 that 80 registers allow.
__global__ void __launch_bounds__(256, 4) kNeighborSort(
    int N, const int* __restrict__ atomStruct, const DevStructInfo* __restrict__ info,
    const int64_t* __restrict__ nbrOffset, int64_t capacity, const int64_t* __restrict__ scrKey,
    const double* __restrict__ scrD, const double* __restrict__ scrDx, const double* __restrict__ scrDy,
    const double* __restrict__ scrDz, const int* __restrict__ elem, int* __restrict__ nbrJ,
    int* __restrict__ nbrCode, uint8_t* __restrict__ nbrElem, double* __restrict__ nbrD,
    double* __restrict__ nbrDx, double* __restrict__ nbrDy, double* __restrict__ nbrDz, int64_t scrStride,
    const DevStatus* __restrict__ status)
{
    // the strided segments, unless an atom outgrew the stride and the fill pass wrote packed ones
    const bool strided = scrStride > 0 && status->maxNeighbors <= scrStride;
    constexpr int kSmemKeys = 512;
    __shared__ int64_t skeys[8][kSmemKeys];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warpsPerGrid)
    {
        const int64_t off = nbrOffset[i];
        const int64_t end = nbrOffset[i + 1];
        if (end > capacity) continue;
        const int n = (int)(end - off);
        const int64_t src = strided ? (int64_t)i * scrStride : off;   // the atom's scratch segment
        DevStructInfo const& s = info[atomStruct[i]];
        const int K = (2 * s.pbc[0] + 1) * (2 * s.pbc[1] + 1) * (2 * s.pbc[2] + 1);
        if (n <= 256 && (int64_t)s.numAtoms * K < 0x7fffffff)
        {
            // keys as 32-bit integers, every lane's (up to eight) ranked in one pass
            int* k32 = reinterpret_cast<int*>(skeys[w]);
            for (int e = lane; e < n; e += 32) k32[e] = (int)scrKey[src + e];
            __syncwarp();
            int kk[8], rank[8];
            switch ((n + 31) >> 5)
            {
            case 0: break;
            case 1: rankKeys32<1>(k32, n, lane, kk, rank); break;
            case 2: rankKeys32<2>(k32, n, lane, kk, rank); break;
            case 3: rankKeys32<3>(k32, n, lane, kk, rank); break;
            case 4: rankKeys32<4>(k32, n, lane, kk, rank); break;
            case 5: rankKeys32<5>(k32, n, lane, kk, rank); break;
            case 6: rankKeys32<6>(k32, n, lane, kk, rank); break;
            case 7: rankKeys32<7>(k32, n, lane, kk, rank); break;
            default: rankKeys32<8>(k32, n, lane, kk, rank); break;
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
            {
                const int e = lane + 32 * r;
                if (e >= n) break;
                const int64_t dst = off + rank[r];
                const int j = kk[r] / K + s.atomBegin;
                nbrJ[dst] = j;
                nbrCode[dst] = kk[r] % K;
                nbrElem[dst] = (uint8_t)elem[j];
                nbrD[dst] = scrD[src + e];
                nbrDx[dst] = scrDx[src + e];
                nbrDy[dst] = scrDy[src + e];
                nbrDz[dst] = scrDz[src + e];
            }
            __syncwarp();
            continue;
        }
        const bool inSmem = n <= kSmemKeys;
        if (inSmem)
            for (int e = lane; e < n; e += 32) skeys[w][e] = scrKey[src + e];
        __syncwarp();
        const int64_t* keys = inSmem ? skeys[w] : scrKey + src;
        for (int e = lane; e < n; e += 32)
        {
            const int64_t k = keys[e];
            int rank = 0;
            for (int q = 0; q < n; ++q) rank += (keys[q] < k) ? 1 : 0;
            const int64_t dst = off + rank;
            const int j = (int)(k / K) + s.atomBegin;
            nbrJ[dst] = j;
            nbrCode[dst] = (int)(k % K);
            nbrElem[dst] = (uint8_t)elem[j];
            nbrD[dst] = scrD[src + e];
            nbrDx[dst] = scrDx[src + e];
            nbrDy[dst] = scrDy[src + e];
            nbrDz[dst] = scrDz[src + e];
        }
        __syncwarp();
    }
}

// rev[e] for entry e = (i -> j, bc): the entry (j -> i, -bc) in j's list.
// Pairs are exactly symmetric because the pair vector arithmetic is odd under
// exchange of i and j with negated images.
__global__ void kNeighborReverse(int N, const int* __restrict__ atomStruct, const DevStructInfo* __restrict__ info,
                                 const int64_t* __restrict__ nbrOffset, int64_t capacity,
                                 const int* __restrict__ nbrJ, const int* __restrict__ nbrCode,
                                 int64_t* __restrict__ rev, DevStatus* __restrict__ status)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warpsPerGrid)
    {
        if (nbrOffset[i + 1] > capacity) continue;   // overflow: the host re-runs with more room
        DevStructInfo const& s = info[atomStruct[i]];
        const int K = (2 * s.pbc[0] + 1) * (2 * s.pbc[1] + 1) * (2 * s.pbc[2] + 1);
        for (int64_t e = nbrOffset[i] + lane; e < nbrOffset[i + 1]; e += 32)
        {
            const int j = nbrJ[e];
            if (nbrOffset[j + 1] > capacity)
            {
                rev[e] = -1;
                continue;
            }
            int bc0, bc1, bc2;
            imageFromCode(nbrCode[e], s.pbc, bc0, bc1, bc2);
            const int64_t want = (int64_t)(i - s.atomBegin) * K + imageCode(-bc0, -bc1, -bc2, s.pbc);
            int64_t lo = nbrOffset[j], hi = nbrOffset[j + 1] - 1, found = -1;
            while (lo <= hi)
            {
                int64_t mid = (lo + hi) >> 1;
                int64_t k = (int64_t)(nbrJ[mid] - s.atomBegin) * K + nbrCode[mid];
                if (k == want)
                {
                    found = mid;
                    break;
                }
                if (k < want) lo = mid + 1;
                else hi = mid - 1;
            }
            rev[e] = found;
            if (found < 0) atomicAdd(&status->badInput, 1);
        }
    }
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan (three phases) of int counts into int64 offsets.
// ---------------------------------------------------------------------------

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) kScanTiles(int n, const int* __restrict__ in,
                                                           int64_t* __restrict__ out, int64_t* __restrict__ tileSums)
{
    __shared__ int64_t warpTot[kScanThreads / 32];
    const int tile = blockIdx.x;
    const int base = tile * kScanTile + threadIdx.x * kScanItems;
    int64_t v[kScanItems];
    int64_t run = 0;
    for (int k = 0; k < kScanItems; ++k)
    {
        int idx = base + k;
        int64_t x = idx < n ? (int64_t)in[idx] : 0;
        v[k] = run;
        run += x;
    }
    // inclusive scan of per-thread totals across the block
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t incl = run;
    for (int o = 1; o < 32; o <<= 1)
    {
        int64_t y = __shfl_up_sync(kFullMask, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warpTot[w] = incl;
    __syncthreads();
    if (w == 0)
    {
        int64_t t = lane < kScanThreads / 32 ? warpTot[lane] : 0;
        for (int o = 1; o < 32; o <<= 1)
        {
            int64_t y = __shfl_up_sync(kFullMask, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kScanThreads / 32) warpTot[lane] = t;
    }
    __syncthreads();
    int64_t prefix = (incl - run) + (w > 0 ? warpTot[w - 1] : 0);
    for (int k = 0; k < kScanItems; ++k)
    {
        int idx = base + k;
        if (idx < n) out[idx] = prefix + v[k];
    }
    if (threadIdx.x == kScanThreads - 1) tileSums[tile] = prefix + run;
}

// Single block: exclusive scan of the tile sums (in place); writes the grand
// total to out[n] and, if given, to *total.
__global__ void __launch_bounds__(1024) kScanTileSums(int numTiles, int64_t* __restrict__ tileSums, int n,
                                                      int64_t* __restrict__ out, int64_t* __restrict__ total)
{
    __shared__ int64_t warpTot[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int per = (numTiles + blockDim.x - 1) / blockDim.x;
    const int begin = threadIdx.x * per;
    int64_t run = 0;
    for (int k = 0; k < per; ++k)
        if (begin + k < numTiles) run += tileSums[begin + k];
    int64_t incl = run;
    for (int o = 1; o < 32; o <<= 1)
    {
        int64_t y = __shfl_up_sync(kFullMask, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warpTot[w] = incl;
    __syncthreads();
    if (w == 0)
    {
        int64_t t = warpTot[lane];
        for (int o = 1; o < 32; o <<= 1)
        {
            int64_t y = __shfl_up_sync(kFullMask, t, o);
            if (lane >= o) t += y;
        }
        warpTot[lane] = t;
    }
    __syncthreads();
    int64_t prefix = (incl - run) + (w > 0 ? warpTot[w - 1] : 0);
    for (int k = 0; k < per; ++k)
    {
        if (begin + k < numTiles)
        {
            int64_t x = tileSums[begin + k];
            tileSums[begin + k] = prefix;
            prefix += x;
        }
    }
    if (threadIdx.x == blockDim.x - 1)
    {
        out[n] = prefix;
        if (total) *total = prefix;
    }
}

__global__ void kScanAdd(int n, const int64_t* __restrict__ tileSums, int64_t* __restrict__ out)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x)
        out[idx] += tileSums[idx / kScanTile];
}

void launchExclusiveScan(int n, const int* in, int64_t* out, int64_t* tileSums, int64_t* total, cudaStream_t st)
{
    int tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles < 1) tiles = 1;
    kScanTiles<<<tiles, kScanThreads, 0, st>>>(n, in, out, tileSums);
    kScanTileSums<<<1, 1024, 0, st>>>(tiles, tileSums, n, out, total);
    kScanAdd<<<(n + 255) / 256 > 0 ? (n + 255) / 256 : 1, 256, 0, st>>>(n, tileSums, out);
}

int scanTileCount(int n) { return (n + kScanTile - 1) / kScanTile + 1; }

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------

__global__ void kCast64to32(int n, const int64_t* __restrict__ in, int* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (int)in[i];
}

void launchPreparePositions(BatchView const& b, const double* rin, int doRemap, int doNormalize, double convLength,
                            cudaStream_t st)
{
    int blocks = (b.N + 255) / 256;
    kPreparePositions<<<blocks > 0 ? blocks : 1, 256, 0, st>>>(b.N, b.atomStruct, b.info, rin, b.px, b.py, b.pz,
                                                               doRemap, doNormalize, convLength);
}

void launchNeighborBuild(BatchView const& b, double rc2, cudaStream_t st)
{
    const int N = b.N;
    const int blocks = (N + 255) / 256 > 0 ? (N + 255) / 256 : 1;
    cudaMemsetAsync(b.cellCount, 0, sizeof(int) * (size_t)b.numCells, st);
    kAssignCells<<<blocks, 256, 0, st>>>(N, b.atomStruct, b.info, b.px, b.py, b.pz, b.atomCell, b.atomSlot,
                                         b.cellCount);
    launchExclusiveScan(b.numCells, b.cellCount, b.cellStart64, b.scanTmp, nullptr, st);
    kCast64to32<<<(b.numCells + 255) / 256 > 0 ? (b.numCells + 255) / 256 : 1, 256, 0, st>>>(b.numCells,
                                                                                          b.cellStart64, b.cellStart);
    kScatterCells<<<blocks, 256, 0, st>>>(N, b.atomCell, b.atomSlot, b.cellStart, b.px, b.py, b.pz, b.cellAtoms,
                                          b.cellPos);
    const int warpBlocks = (N + kSearchWarps - 1) / kSearchWarps > 0 ? (N + kSearchWarps - 1) / kSearchWarps : 1;
    if (b.scrStride > 0)
    {
        kNeighborSearch<2><<<warpBlocks, kSearchWarps * 32, 0, st>>>(N, rc2, b.atomStruct, b.info, b.px, b.py, b.pz,
                                                       b.atomCell, b.cellStart, b.cellCount, b.cellPos, b.nbrCount,
                                                       nullptr, 0, b.scrKey, b.scrD, b.scrDx, b.scrDy, b.scrDz,
                                                       b.status, b.scrStride, 0);
        launchExclusiveScan(N, b.nbrCount, b.nbrOffset, b.scanTmp, &b.status->totalNeighbors, st);
        kNeighborSearch<1><<<warpBlocks, kSearchWarps * 32, 0, st>>>(N, rc2, b.atomStruct, b.info, b.px, b.py, b.pz,
                                                       b.atomCell, b.cellStart, b.cellCount, b.cellPos, nullptr,
                                                       b.nbrOffset,
                                                       b.nbrCapacity, b.scrKey, b.scrD, b.scrDx, b.scrDy, b.scrDz,
                                                       b.status, 0, b.scrStride);
    }
    else
    {
        kNeighborSearch<0><<<warpBlocks, kSearchWarps * 32, 0, st>>>(N, rc2, b.atomStruct, b.info, b.px, b.py, b.pz,
                                                       b.atomCell, b.cellStart, b.cellCount, b.cellPos, b.nbrCount,
                                                       nullptr, 0,
                                                       nullptr, nullptr, nullptr, nullptr, nullptr, b.status, 0, 0);
        launchExclusiveScan(N, b.nbrCount, b.nbrOffset, b.scanTmp, &b.status->totalNeighbors, st);
        kNeighborSearch<1><<<warpBlocks, kSearchWarps * 32, 0, st>>>(N, rc2, b.atomStruct, b.info, b.px, b.py, b.pz,
                                                       b.atomCell, b.cellStart, b.cellCount, b.cellPos, nullptr,
                                                       b.nbrOffset,
                                                       b.nbrCapacity, b.scrKey, b.scrD, b.scrDx, b.scrDy, b.scrDz,
                                                       b.status, 0, 0);
    }
    kNeighborSort<<<warpBlocks, 256, 0, st>>>(N, b.atomStruct, b.info, b.nbrOffset, b.nbrCapacity, b.scrKey, b.scrD,
                                              b.scrDx, b.scrDy, b.scrDz, b.elem, b.nbrJ, b.nbrCode, b.nbrElem,
                                              b.nbrD, b.nbrDx, b.nbrDy, b.nbrDz, b.scrStride, b.status);
    kNeighborReverse<<<warpBlocks, 256, 0, st>>>(N, b.atomStruct, b.info, b.nbrOffset, b.nbrCapacity, b.nbrJ,
                                                 b.nbrCode, b.rev, b.status);
}

} // namespace n2p2b200
