// Instrumentation kernels (not on the evaluation path): algorithmic work
// counters of a batch and FP64/FP32 fused-multiply-add throughput probes used
// as the compute roofline of the symmetry-function kernels.
#include <cmath>
#include <stdexcept>

#include "kernels_common.cuh"
#include "kernels.hpp"

namespace n2p2b200 {

// counts[0] neighbour entries, [1] radial terms (pair x member),
// [2] radial pairs, [3] narrow triplets (unordered, accepted),
// [4] narrow triplet x member, [5] wide pairs (unordered, accepted),
// [6] wide pair x member, [7] symmetry-function values, [8] atoms,
// [9] derivative rows of all entries (sum over entries of the row count).
__global__ void kCountWork(DevModel model, BatchView b, unsigned long long* counts)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        const int64_t off = b.nbrOffset[i];
        const int64_t end = b.nbrOffset[i + 1];
        if (end > b.nbrCapacity) continue;
        const int n = (int)(end - off);
        DevElement const& E = model.el[b.elem[i]];
        unsigned long long c[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (lane == 0)
        {
            c[0] = n;
            c[7] = E.numSF;
            c[8] = 1;
        }
        for (int j = lane; j < n; j += 32) c[9] += E.rows[b.elem[b.nbrJ[off + j]]];
        for (int g = 0; g < E.groupCount; ++g)
        {
            DevGroup const G = model.groups[E.groupBegin + g];
            for (int j = lane; j < n; j += 32)
            {
                const int ej = b.elem[b.nbrJ[off + j]];
                const double rij = b.nbrD[off + j];
                if (G.type == 2)
                {
                    if (ej == G.e1 && rij < G.rc)
                    {
                        c[2] += 1;
                        c[1] += G.memberCount;
                    }
                    continue;
                }
                if (!((ej == G.e1 || ej == G.e2) && rij < G.rc)) continue;
                const int needK = (ej == G.e1) ? G.e2 : G.e1;
                for (int k = j + 1; k < n; ++k)
                {
                    if (b.elem[b.nbrJ[off + k]] != needK || !(b.nbrD[off + k] < G.rc)) continue;
                    if (G.type == 3)
                    {
                        const double dx = b.nbrDx[off + k] - b.nbrDx[off + j];
                        const double dy = b.nbrDy[off + k] - b.nbrDy[off + j];
                        const double dz = b.nbrDz[off + k] - b.nbrDz[off + j];
                        if (!(dx * dx + dy * dy + dz * dz < G.rc2)) continue;
                        c[3] += 1;
                        c[4] += G.memberCount;
                    }
                    else
                    {
                        c[5] += 1;
                        c[6] += G.memberCount;
                    }
                }
            }
        }
        for (int q = 0; q < 10; ++q)
        {
            unsigned long long v = c[q];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
            if (lane == 0 && v) atomicAdd(&counts[q], v);
        }
    }
}

void launchCountWork(DevModel const& m, BatchView const& b, unsigned long long* counts, int sms, cudaStream_t st)
{
    int blocks = (b.N + 7) / 8;
    if (blocks < 1) blocks = 1;
    if (blocks > sms * 16) blocks = sms * 16;
    kCountWork<<<blocks, 256, 0, st>>>(m, b, counts);
}

// Independent FMA chains per thread; `iters` x 8 chains x 2 flops per thread.
template <typename T>
__global__ void __launch_bounds__(256) kFmaProbe(int iters, T seed, T* out)
{
    T a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + T(threadIdx.x + k);
    const T m = T(0.999999), c = T(1e-7);
    for (int it = 0; it < iters; ++it)
    {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], m, c);
    }
    T s = T(0);
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == T(-12345.0)) out[threadIdx.x] = s;   // keeps the chains alive
}

double measureFmaPeak(int fp64, int sms)
{
    const int iters = 1 << 14;
    const int blocks = sms * 8;
    void* out = nullptr;
    cudaMalloc(&out, 4096);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep)
    {
        cudaEventRecord(e0);
        if (fp64) kFmaProbe<double><<<blocks, 256>>>(iters, 1.0, (double*)out);
        else kFmaProbe<float><<<blocks, 256>>>(iters, 1.0f, (float*)out);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * iters * (double)blocks * 256.0;
    return flops / (best * 1e-3) / 1e12;
}

// CutoffFunction::fdf (CutoffFunction.h:210-220) on the device, as the
// symmetry-function kernels evaluate it: FP64 (cutoffFdf, every pair's f_c)
// or the FP32 form of the mixed kernels' per-triplet f_c(r_jk) (cutoffFdfF32).
__global__ void kCutoffValues(DevCutoff c, int fp32, const double* __restrict__ r, int64_t n, double* __restrict__ f,
                              double* __restrict__ df)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    {
        if (fp32)
        {
            float a, b;
            cutoffFdfF32(c, (float)r[k], a, b);
            f[k] = a;
            df[k] = b;
        }
        else cutoffFdf(c, r[k], f[k], df[k]);
    }
}

void cutoffFunctionValues(int type, double rc, double alpha, int fp32, const double* r, int64_t n, double* f,
                          double* df)
{
    if (type < 0 || type > 8) throw std::invalid_argument("ERROR: unknown cutoff type.\n");
    if (alpha < 0.0 || alpha >= 1.0) throw std::invalid_argument("ERROR: 0 <= alpha < 1.0 is required.\n");
    if (n <= 0) return;
    DevCutoff c{};
    const double E = std::exp(1.0);
    c.type = type;
    c.rc = rc;
    c.rcinv = 1.0 / rc;
    c.alpha = alpha;
    c.rci = rc * alpha;
    c.iw = 1.0 / (c.rc - c.rci);
    c.tanhPre = std::pow((E + 1 / E) / (E - 1 / E), 3);
    c.rcF = (float)c.rc;
    c.rciF = (float)c.rci;
    c.iwF = (float)c.iw;
    double* d = nullptr;
    cudaCheck(cudaMalloc(&d, sizeof(double) * 3 * (size_t)n), "cudaMalloc");
    cudaCheck(cudaMemcpy(d, r, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice), "H2D");
    kCutoffValues<<<(int)std::min<int64_t>((n + 255) / 256, 1024), 256>>>(c, fp32, d, n, d + n, d + 2 * n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(f, d + n, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(df, d + 2 * n, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    cudaCheck(e, "cutoff values");
}

} // namespace n2p2b200
