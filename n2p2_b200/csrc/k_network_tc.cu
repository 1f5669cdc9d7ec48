// Atomic networks of the mixed-precision form on the 5th-generation tensor
// cores (tcgen05): per element, tiles of 128 atoms run the forward pass
// (NeuralNetwork::propagate, NeuralNetwork.cpp:386-394) and dE/dG
// (NeuralNetwork::calculateDEdG, NeuralNetwork.cpp:396-442) as four
// matrix products with FP32 accumulators in tensor memory:
//     Z1 = X W1^T,  Z2 = H1 W2^T,  D1 = (w3 . f2'(Z2)) W2,  dE/dG = (D1 . f1'(Z1)) W1.
// Operands are split into two bfloat16 halves (x = hi + lo, hi = bf16(x),
// lo = bf16(x - hi), 16 significant bits together) and every product is
// accumulated from all four partial products -- plain bfloat16 (8 bits)
// would put the atomic energies off by ~1e-3 relative, far beyond the
// 1 meV/atom budget; three partial products (no lo.lo) leave ~6e-6.  Biases, activations and the output layer run in FP32
// on the CUDA cores; G is read and E, dE/dG are written in FP64.
//
// Shared-memory operands use the K-major layout without swizzle that the
// tensor core reads through a matrix descriptor: 16-byte chunks of 8
// consecutive K elements, chunk (row r, k-chunk c) of an R-row matrix at
// byte (c R + r) 16, so 8-row core matrices are 128 contiguous bytes (stride
// between 8-row groups SBO = 128 B) and the two K chunks of one 16-wide MMA
// step are R 16 bytes apart (LBO).
//
// One thread (thread 0) issues the MMAs of a phase and commits them to an
// mbarrier; all threads wait on it with a bounded spin (a timeout is
// reported in DevStatus and the kernel winds down, freeing tensor memory).
#include "kernels_common.cuh"
#include "kernels.hpp"
#include "host_model.hpp"

#include <cuda_bf16.h>

namespace n2p2b200 {

namespace {

constexpr int kTile = 128;            // atoms per tile = MMA M = threads per CTA
constexpr int kMaxDim = 64;           // padded widths (inputs, hidden layers)
constexpr int kTmemCols = 256;        // four accumulators of <= 64 columns

struct TcDims
{
    int K0, H1, H2;                   // true widths
    int K0p, H1p, H2p;                // padded to 16
    int act1, act2;                   // hidden activations
};

// Shared memory of one CTA (dynamic, 1024-byte aligned pieces).
struct TcSmem
{
    // A operands: 128 rows x <= 64 columns, hi and lo planes
    alignas(1024) __nv_bfloat16 x[2][kTile * kMaxDim];
    alignas(1024) __nv_bfloat16 h1[2][kTile * kMaxDim];
    alignas(1024) __nv_bfloat16 d2[2][kTile * kMaxDim];
    alignas(1024) __nv_bfloat16 d1[2][kTile * kMaxDim];
    // B operands (rows = output columns of the product)
    alignas(1024) __nv_bfloat16 w1[2][kMaxDim * kMaxDim];    // [H1p][K0p]
    alignas(1024) __nv_bfloat16 w2[2][kMaxDim * kMaxDim];    // [H2p][H1p]
    alignas(1024) __nv_bfloat16 w2t[2][kMaxDim * kMaxDim];   // [H1p][H2p]
    alignas(1024) __nv_bfloat16 w1t[2][kMaxDim * kMaxDim];   // [K0p][H1p]
    float b1[kMaxDim], b2[kMaxDim], w3[kMaxDim];
    float b3;
    alignas(8) unsigned long long mbar;
    uint32_t tmemBase;
};

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Element (r, k) of an R-row K-major chunked matrix.
__device__ __forceinline__ int chunkIndex(int r, int k, int R) { return ((k >> 3) * R + r) * 8 + (k & 7); }

// Matrix descriptor: start address, LBO (between the K chunks), SBO (between
// 8-row groups), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t matDesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N.
__device__ __forceinline__ uint32_t instrDesc(int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t dTmem, uint64_t a, uint64_t b, uint32_t idesc, int accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(dTmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// D[128 x N] (+)= A[128 x K] B[N x K]^T with split operands: 4 products per
// 16-wide K step.  A and B are chunked matrices with 128 and N rows.
__device__ __forceinline__ void splitProduct(uint32_t dTmem, const __nv_bfloat16 (*A)[kTile * kMaxDim],
                                             const __nv_bfloat16 (*B)[kMaxDim * kMaxDim], int N, int K)
{
    const uint32_t idesc = instrDesc(N);
    const uint32_t aHi = smemAddr(A[0]), aLo = smemAddr(A[1]);
    const uint32_t bHi = smemAddr(B[0]), bLo = smemAddr(B[1]);
    int acc = 0;
    for (int s = 0; s < K / 16; ++s)
    {
        const uint32_t aOff = (uint32_t)(2 * s * kTile) * 16u, bOff = (uint32_t)(2 * s * N) * 16u;
        const uint64_t ah = matDesc(aHi + aOff, kTile * 16, 128), al = matDesc(aLo + aOff, kTile * 16, 128);
        const uint64_t bh = matDesc(bHi + bOff, (uint32_t)N * 16, 128), bl = matDesc(bLo + bOff, (uint32_t)N * 16, 128);
        mma(dTmem, ah, bh, idesc, acc);
        acc = 1;
        mma(dTmem, ah, bl, idesc, 1);
        mma(dTmem, al, bh, idesc, 1);
        mma(dTmem, al, bl, idesc, 1);
    }
}

__device__ __forceinline__ void commitTo(unsigned long long* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddr(bar))
                 : "memory");
}

// Bounded wait for the mbarrier phase with the given parity; false on timeout.
__device__ __forceinline__ bool waitPhase(unsigned long long* bar, uint32_t parity)
{
    const uint32_t a = smemAddr(bar);
    for (int it = 0; it < (1 << 20); ++it)
    {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive accumulator columns of this thread's row.
__device__ __forceinline__ void tmemLoad16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// Row `row` of an A operand: values v[0..n) (zeros up to np), split.
__device__ __forceinline__ void storeSplitRow(__nv_bfloat16 (*P)[kTile * kMaxDim], int row, const float* v, int np)
{
    for (int c = 0; c < np / 8; ++c)
    {
        __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            const float x = v[c * 8 + q];
            hi[q] = __float2bfloat16_rn(x);
            lo[q] = __float2bfloat16_rn(x - __bfloat162float(hi[q]));
        }
        *reinterpret_cast<uint4*>(&P[0][(c * kTile + row) * 8]) = *reinterpret_cast<uint4*>(hi);
        *reinterpret_cast<uint4*>(&P[1][(c * kTile + row) * 8]) = *reinterpret_cast<uint4*>(lo);
    }
}

__device__ __forceinline__ void activation(int af, float z, float& f, float& d)
{
    switch (af)
    {
    case AF_IDENTITY: f = z; d = 1.f; return;
    case AF_TANH:
    {
        const float t = tanhf(z);
        f = t;
        d = 1.f - t * t;
        return;
    }
    case AF_LOGISTIC:
        if (z > 35.f) { f = 1.f; d = 0.f; }
        else if (z < -35.f) { f = 0.f; d = 0.f; }
        else
        {
            const float t = 1.f / (1.f + expf(-z));
            f = t;
            d = t * (1.f - t);
        }
        return;
    case AF_SOFTPLUS:
        if (z > 35.f) { f = z; d = 1.f; }
        else if (z < -35.f) { f = 0.f; d = 0.f; }
        else
        {
            const float t = expf(z);
            f = log1pf(t);
            d = t / (1.f + t);
        }
        return;
    }
    f = 0.f;
    d = 0.f;
}

__device__ void loadWeights(TcSmem& S, DevModel const& m, DevElement const& E, TcDims const& d)
{
    const double* W1 = m.weights + E.wOffset[1];
    const double* B1 = m.weights + E.bOffset[1];
    const double* W2 = m.weights + E.wOffset[2];
    const double* B2 = m.weights + E.bOffset[2];
    const double* W3 = m.weights + E.wOffset[3];
    const double* B3 = m.weights + E.bOffset[3];
    auto put = [](__nv_bfloat16 (*P)[kMaxDim * kMaxDim], int idx, float x) {
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        P[0][idx] = h;
        P[1][idx] = __float2bfloat16_rn(x - __bfloat162float(h));
    };
    for (int t = threadIdx.x; t < kMaxDim * kMaxDim; t += blockDim.x)
    {
        const int r = t / kMaxDim, k = t % kMaxDim;
        if (r < d.H1p && k < d.K0p)   // W1 [H1p][K0p] and W1^T [K0p][H1p]
        {
            const float w = (r < d.H1 && k < d.K0) ? (float)W1[(size_t)r * d.K0 + k] : 0.f;
            put(S.w1, chunkIndex(r, k, d.H1p), w);
            put(S.w1t, chunkIndex(k, r, d.K0p), w);
        }
        if (r < d.H2p && k < d.H1p)   // W2 [H2p][H1p] and W2^T [H1p][H2p]
        {
            const float w = (r < d.H2 && k < d.H1) ? (float)W2[(size_t)r * d.H1 + k] : 0.f;
            put(S.w2, chunkIndex(r, k, d.H2p), w);
            put(S.w2t, chunkIndex(k, r, d.H1p), w);
        }
    }
    for (int t = threadIdx.x; t < kMaxDim; t += blockDim.x)
    {
        S.b1[t] = t < d.H1 ? (float)B1[t] : 0.f;
        S.b2[t] = t < d.H2 ? (float)B2[t] : 0.f;
        S.w3[t] = t < d.H2 ? (float)W3[t] : 0.f;
    }
    if (threadIdx.x == 0) S.b3 = (float)B3[0];
}

__device__ __forceinline__ TcDims dimsOf(DevElement const& E)
{
    TcDims d;
    d.K0 = E.neurons[0];
    d.H1 = E.neurons[1];
    d.H2 = E.neurons[2];
    d.K0p = (d.K0 + 15) & ~15;
    d.H1p = (d.H1 + 15) & ~15;
    d.H2p = (d.H2 + 15) & ~15;
    d.act1 = E.activation[1];
    d.act2 = E.activation[2];
    return d;
}

} // namespace

// One CTA per SM, 128 threads; tile t of the element-sorted atom list.
__global__ void __launch_bounds__(kTile, 1) kNetworkTC(DevModel model, BatchView b, int derivatives)
{
    extern __shared__ __align__(1024) unsigned char smemRaw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x;
    const int warp = tid >> 5;

    if (tid == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(&S.mbar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(&S.tmemBase)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    const uint32_t tmem = S.tmemBase;
    const uint32_t dZ1 = tmem, dZ2 = tmem + 64, dD1 = tmem + 128, dG = tmem + 192;
    const uint32_t laneBase = (uint32_t)(warp * 32) << 16;   // this warp's 32 accumulator rows

    // tiles of every element, in element order
    int tilesOf[kDevMaxElements + 1];
    tilesOf[0] = 0;
    for (int e = 0; e < model.numElements; ++e)
        tilesOf[e + 1] = tilesOf[e] + (b.elemBegin[e + 1] - b.elemBegin[e] + kTile - 1) / kTile;
    const int numTiles = tilesOf[model.numElements];

    uint32_t phase = 0;
    int loaded = -1;
    bool failed = false;
    for (int tile = blockIdx.x; tile < numTiles; tile += gridDim.x)
    {
        int e = 0;
        while (tile >= tilesOf[e + 1]) ++e;
        DevElement const& E = model.el[e];
        const TcDims d = dimsOf(E);
        if (e != loaded)
        {
            __syncthreads();
            loadWeights(S, model, E, d);
            loaded = e;
        }
        const int slot = b.elemBegin[e] + (tile - tilesOf[e]) * kTile + tid;
        const bool valid = slot < b.elemBegin[e + 1];
        const int atom = valid ? b.elemAtoms[slot] : -1;

        // X row (G of this atom, FP64 -> split bf16)
        {
            float v[kMaxDim];
            const double* g = valid ? b.G + (size_t)atom * b.gStride : nullptr;
            for (int k = 0; k < d.K0p; ++k) v[k] = (valid && k < d.K0) ? (float)g[k] : 0.f;
            storeSplitRow(S.x, tid, v, d.K0p);
        }
        fenceProxyAsync();
        fenceBeforeSync();
        __syncthreads();
        fenceAfterSync();

        // Z1 = X W1^T
        if (tid == 0)
        {
            splitProduct(dZ1, S.x, S.w1, d.H1p, d.K0p);
            commitTo(&S.mbar);
        }
        failed = __syncthreads_or(waitPhase(&S.mbar, phase) ? 0 : 1) != 0;
        phase ^= 1u;
        if (failed) break;
        fenceAfterSync();
        float s1[kMaxDim];
        {
            float v[kMaxDim];
            for (int c = 0; c < d.H1p / 16; ++c) tmemLoad16(dZ1 + laneBase + c * 16, v + c * 16);
            for (int j = 0; j < d.H1p; ++j)
            {
                float f, df;
                activation(d.act1, v[j] + S.b1[j], f, df);
                v[j] = j < d.H1 ? f : 0.f;
                s1[j] = j < d.H1 ? df : 0.f;
            }
            storeSplitRow(S.h1, tid, v, d.H1p);
        }
        fenceProxyAsync();
        fenceBeforeSync();
        __syncthreads();
        fenceAfterSync();

        // Z2 = H1 W2^T
        if (tid == 0)
        {
            splitProduct(dZ2, S.h1, S.w2, d.H2p, d.H1p);
            commitTo(&S.mbar);
        }
        failed = __syncthreads_or(waitPhase(&S.mbar, phase) ? 0 : 1) != 0;
        phase ^= 1u;
        if (failed) break;
        fenceAfterSync();
        {
            float v[kMaxDim];
            for (int c = 0; c < d.H2p / 16; ++c) tmemLoad16(dZ2 + laneBase + c * 16, v + c * 16);
            float energy = S.b3;
            for (int j = 0; j < d.H2p; ++j)
            {
                float f, df;
                activation(d.act2, v[j] + S.b2[j], f, df);
                if (j < d.H2) energy += S.w3[j] * f;
                v[j] = j < d.H2 ? S.w3[j] * df : 0.f;   // delta_2 = w3 . f2'(Z2)
            }
            if (valid) b.Eatom[atom] = (double)energy;
            storeSplitRow(S.d2, tid, v, d.H2p);
        }
        if (!derivatives) continue;
        fenceProxyAsync();
        fenceBeforeSync();
        __syncthreads();
        fenceAfterSync();

        // D1 = delta_2 W2 (B = W2^T), delta_1 = D1 . f1'(Z1)
        if (tid == 0)
        {
            splitProduct(dD1, S.d2, S.w2t, d.H1p, d.H2p);
            commitTo(&S.mbar);
        }
        failed = __syncthreads_or(waitPhase(&S.mbar, phase) ? 0 : 1) != 0;
        phase ^= 1u;
        if (failed) break;
        fenceAfterSync();
        {
            float v[kMaxDim];
            for (int c = 0; c < d.H1p / 16; ++c) tmemLoad16(dD1 + laneBase + c * 16, v + c * 16);
            for (int j = 0; j < d.H1p; ++j) v[j] *= s1[j];
            storeSplitRow(S.d1, tid, v, d.H1p);
        }
        fenceProxyAsync();
        fenceBeforeSync();
        __syncthreads();
        fenceAfterSync();

        // dE/dG = delta_1 W1 (B = W1^T)
        if (tid == 0)
        {
            splitProduct(dG, S.d1, S.w1t, d.K0p, d.H1p);
            commitTo(&S.mbar);
        }
        failed = __syncthreads_or(waitPhase(&S.mbar, phase) ? 0 : 1) != 0;
        phase ^= 1u;
        if (failed) break;
        fenceAfterSync();
        {
            float v[kMaxDim];
            for (int c = 0; c < d.K0p / 16; ++c) tmemLoad16(dG + laneBase + c * 16, v + c * 16);
            if (valid)
            {
                double* out = b.dEdG + (size_t)atom * b.gStride;
                for (int k = 0; k < d.K0; ++k) out[k] = (double)v[k];
            }
        }
        fenceBeforeSync();
        __syncthreads();   // accumulators and operands are reused by the next tile
        fenceAfterSync();
    }
    if (failed && tid == 0) atomicAdd(&b.status->tensorCoreTimeout, 1);
    fenceBeforeSync();
    __syncthreads();
    fenceAfterSync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

bool networkTCSupported(Model const& m)
{
    if (m.normalizeNeurons) return false;
    for (auto const& el : m.elements)
    {
        NetworkTopology const& t = el.topology;
        if (t.numLayers != 4) return false;
        if (t.neurons[0] > kMaxDim || t.neurons[1] > kMaxDim || t.neurons[2] > kMaxDim || t.neurons[3] != 1)
            return false;
        for (int l = 1; l <= 2; ++l)
        {
            const int af = t.activations[l];
            if (af != AF_IDENTITY && af != AF_TANH && af != AF_LOGISTIC && af != AF_SOFTPLUS) return false;
        }
        if (t.activations[3] != AF_IDENTITY) return false;
    }
    return true;
}

void launchNetworkTC(DevModel const& m, BatchView const& b, int derivatives, int sms, cudaStream_t st)
{
    const size_t smem = sizeof(TcSmem) + 1024;
    setDynamicSmemOnce(reinterpret_cast<const void*>(kNetworkTC), smem);
    int tiles = 0;
    for (int e = 0; e < m.numElements; ++e) tiles += (b.elemBegin[e + 1] - b.elemBegin[e] + kTile - 1) / kTile;
    const int grid = tiles < sms ? (tiles > 0 ? tiles : 1) : sms;
    kNetworkTC<<<grid, kTile, smem, st>>>(m, b, derivatives);
}

} // namespace n2p2b200
