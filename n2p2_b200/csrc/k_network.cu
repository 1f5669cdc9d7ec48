// Atomic neural networks (FP64 form), per-structure energy sums and the
// deterministic force gather.
//
// Network: NeuralNetwork::propagate / propagateLayer (NeuralNetwork.cpp:386-394,
// 761-896) for the activations of the reference, and dE/dG by reverse-mode
// accumulation, which equals NeuralNetwork::calculateDEdG
// (NeuralNetwork.cpp:396-442) including the normalize_nodes divisions.
#include <algorithm>

#include "kernels_common.cuh"

#include <math_constants.h>
#include "kernels.hpp"

namespace n2p2b200 {

namespace {

constexpr double kExpLimit = 35.0;   // EXP_LIMIT, NeuralNetwork.cpp:25

// Activation value and first derivative for one neuron.
__device__ __forceinline__ void activate(int af, double x, double& y, double& dy)
{
    switch (af)
    {
    case AF_IDENTITY: y = x; dy = 1.0; return;
    case AF_TANH:
    {
        double t = tanh(x);
        y = t;
        dy = 1.0 - t * t;
        return;
    }
    case AF_LOGISTIC:
        if (x > kExpLimit) { y = 1.0; dy = 0.0; }
        else if (x < -kExpLimit) { y = 0.0; dy = 0.0; }
        else
        {
            double t = 1.0 / (1.0 + exp(-x));
            y = t;
            dy = t * (1.0 - t);
        }
        return;
    case AF_SOFTPLUS:
        if (x > kExpLimit) { y = x; dy = 1.0; }
        else if (x < -kExpLimit) { y = 0.0; dy = 0.0; }
        else
        {
            double t = exp(x);
            y = log(1.0 + t);
            dy = 1.0 / (1.0 + 1.0 / t);
        }
        return;
    case AF_RELU:
        if (x > 0.0) { y = x; dy = 1.0; }
        else { y = 0.0; dy = 0.0; }
        return;
    case AF_GAUSSIAN:
    {
        double t = exp(-0.5 * x * x);
        y = t;
        dy = -x * t;
        return;
    }
    case AF_COS: y = cos(x); dy = -sin(x); return;
    case AF_REVLOGISTIC:
    {
        double t = 1.0 / (1.0 + exp(-x));
        y = 1.0 - t;
        dy = t * (t - 1.0);
        return;
    }
    case AF_EXP:
    {
        double t = exp(-x);
        y = t;
        dy = -t;
        return;
    }
    case AF_HARMONIC: y = x * x; dy = 2.0 * x; return;
    }
    y = 0.0;
    dy = 0.0;
}

constexpr int kNNWarps = 4;

struct NNWarpSmem
{
    double act[2][kMaxNeurons];   // hidden layers; a wider input layer is read from G directly
    double dfdx[kDevMaxLayers][kMaxNeurons];
    double g[2][kMaxNeurons];
};

} // namespace

// One warp per atom; lanes split the neurons of a layer.  Weights are read
// through the read-only cache (all warps of an element share them).
__global__ void __launch_bounds__(kNNWarps * 32) kNetworkFP64(DevModel model, BatchView b, int derivatives)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    NNWarpSmem* smAll = reinterpret_cast<NNWarpSmem*>(smemRaw);
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    NNWarpSmem& S = smAll[w];
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        const int ec = b.elem[i];
        DevElement const& E = model.el[ec];
        const int L = E.numLayers;
        const double* Gi = b.G + (size_t)i * b.gStride;
        __syncwarp();
        const bool staged = E.neurons[0] <= kMaxNeurons;
        if (staged)
            for (int k = lane; k < E.neurons[0]; k += 32) S.act[0][k] = Gi[k];
        __syncwarp();
        int cur = 0;
        for (int l = 1; l < L; ++l)
        {
            const int nin = E.neurons[l - 1], nout = E.neurons[l];
            const double* WT = model.weightsT + E.wOffset[l];   // lanes read consecutive output neurons
            const double* bias = model.weights + E.bOffset[l];
            const double* in = (l == 1 && !staged) ? Gi : S.act[cur];
            for (int k = lane; k < nout; k += 32)
            {
                double x = 0.0;
                for (int j = 0; j < nin; ++j) x += __ldg(&WT[(size_t)j * nout + k]) * in[j];
                x += __ldg(&bias[k]);
                if (model.normalizeNeurons) x /= nin;
                double y, dy;
                activate(E.activation[l], x, y, dy);
                S.act[cur ^ 1][k] = y;
                S.dfdx[l][k] = dy;
            }
            __syncwarp();
            cur ^= 1;
        }
        if (lane == 0) b.Eatom[i] = S.act[cur][0];
        if (!derivatives) continue;
        // Reverse pass: g_L = f'_L; g_{l-1} = f'_{l-1} * (W_l^T g_l) / n_{l-1}?; dEdG = W_1^T g_1 / n_0?
        __syncwarp();
        int gc = 0;
        if (lane == 0)
        {
            double g0 = S.dfdx[L - 1][0];
            if (model.normalizeNeurons) g0 /= E.neurons[L - 2];
            S.g[0][0] = g0;
        }
        __syncwarp();
        for (int l = L - 1; l >= 2; --l)
        {
            const int nin = E.neurons[l - 1], nout = E.neurons[l];
            const double* W = model.weights + E.wOffset[l];
            for (int j = lane; j < nin; j += 32)
            {
                double s = 0.0;
                for (int k = 0; k < nout; ++k) s += __ldg(&W[(size_t)k * nin + j]) * S.g[gc][k];
                s *= S.dfdx[l - 1][j];
                if (model.normalizeNeurons) s /= E.neurons[l - 2];
                S.g[gc ^ 1][j] = s;
            }
            __syncwarp();
            gc ^= 1;
        }
        {
            const int nin = E.neurons[0], nout = E.neurons[1];
            const double* W = model.weights + E.wOffset[1];
            double* out = b.dEdG + (size_t)i * b.gStride;
            for (int j = lane; j < nin; j += 32)
            {
                double s = 0.0;
                for (int k = 0; k < nout; ++k) s += __ldg(&W[(size_t)k * nin + j]) * S.g[gc][k];
                out[j] = s;
            }
        }
    }
}

namespace {

// ---------------------------------------------------------------------------
// Tiled FP64 networks: one block per tile of TILE (32, or 16 for wide networks) atoms of one element
// (element-grouped atom list).  Activations, derivatives and the reverse
// pass's vectors live in shared memory neuron-major ([neuron][atom], rows of
// netRow doubles); each thread computes a unit of kNetUnit atoms x one
// neuron, reading a weight once (through the read-only cache: every block of
// an element reads the same matrices) for kNetUnit fused multiply-adds.  Every sum
// runs over the reduction index in ascending order, as in propagateLayer.
constexpr int kNetThreads = 128;
constexpr int kNetUnit = 8;        // atoms per thread unit (independent sums)

// Row of a tile of TILE atoms: padded by four against bank conflicts (rows stay 32-byte aligned).
template <int TILE>
__host__ __device__ constexpr int netRow() { return TILE + 4; }

__host__ __device__ inline int netSmemDoubles(DevElement const& E, int row)
{
    int maxW = 0, sumD = 0;
    for (int l = 0; l < E.numLayers; ++l) maxW = E.neurons[l] > maxW ? E.neurons[l] : maxW;
    for (int l = 1; l < E.numLayers; ++l) sumD += E.neurons[l];
    return (2 * maxW + sumD + 2 * maxW) * row;   // activations, derivatives per layer, reverse vectors
}

// Sum over the reduction index r < n of w(r) x[r][a] for the unit's kNetUnit
// atoms (x rows ROW apart), in ascending r.
template <int ROW, typename WF>
__device__ __forceinline__ void netUnitSums(int n, WF w, const double* x, double (&v)[kNetUnit])
{
#pragma unroll
    for (int c = 0; c < kNetUnit; ++c) v[c] = 0.0;
#pragma unroll 4
    for (int r = 0; r < n; ++r)
    {
        const double wr = w(r);
#pragma unroll
        for (int c = 0; c < kNetUnit; c += 2)
        {
            const double2 p = *reinterpret_cast<const double2*>(x + r * ROW + c);
            v[c] += wr * p.x;
            v[c + 1] += wr * p.y;
        }
    }
}

// out[k][a] = act(sum_j W[k][j] in[j][a] + b[k]) (normalize: x / nin), with f' kept.
template <int TILE>
__device__ __forceinline__ void netForwardLayer(int af, int nin, int nout, const double* __restrict__ WT,
                                                const double* __restrict__ bias, int normalize, const double* in,
                                                double* out, double* df, int tid)
{
    for (int u = tid; u < (TILE / kNetUnit) * nout; u += kNetThreads)
    {
        const int k = u % nout, q = u / nout;
        double v[kNetUnit];
        netUnitSums<netRow<TILE>()>(nin, [&](int j) { return __ldg(&WT[(size_t)j * nout + k]); }, in + kNetUnit * q, v);
        const double bk = __ldg(&bias[k]);
#pragma unroll
        for (int c = 0; c < kNetUnit; ++c)
        {
            double x = v[c] + bk;
            if (normalize) x /= nin;
            double y, dy;
            activate(af, x, y, dy);
            out[k * netRow<TILE>() + kNetUnit * q + c] = y;
            df[k * netRow<TILE>() + kNetUnit * q + c] = dy;
        }
    }
}

// out[j][a] = scale[j][a] * sum_k W[k][j] g[k][a] (divided by div when > 0).
template <int TILE>
__device__ __forceinline__ void netBackwardLayer(int nin, int nout, const double* __restrict__ W, const double* g,
                                                 const double* scale, int div, double* out, int tid)
{
    for (int u = tid; u < (TILE / kNetUnit) * nin; u += kNetThreads)
    {
        const int j = u % nin, q = u / nin;
        double v[kNetUnit];
        netUnitSums<netRow<TILE>()>(nout, [&](int k) { return __ldg(&W[(size_t)k * nin + j]); }, g + kNetUnit * q, v);
#pragma unroll
        for (int c = 0; c < kNetUnit; ++c)
        {
            double x = v[c] * scale[j * netRow<TILE>() + kNetUnit * q + c];
            if (div > 0) x /= div;
            out[j * netRow<TILE>() + kNetUnit * q + c] = x;
        }
    }
}

template <int TILE>
__global__ void __launch_bounds__(kNetThreads, 3) kNetworkTiled(DevModel model, BatchView b, int derivatives)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    double* sm = reinterpret_cast<double*>(smemRaw);
    const int tid = threadIdx.x;
    // tiles of every element, in element order
    int tilesOf[kDevMaxElements + 1];
    tilesOf[0] = 0;
    for (int e = 0; e < model.numElements; ++e)
        tilesOf[e + 1] = tilesOf[e] + (b.elemBegin[e + 1] - b.elemBegin[e] + TILE - 1) / TILE;
    for (int tile = blockIdx.x; tile < tilesOf[model.numElements]; tile += gridDim.x)
    {
        int e = 0;
        while (tile >= tilesOf[e + 1]) ++e;
        DevElement const& E = model.el[e];
        const int L = E.numLayers;
        const int first = b.elemBegin[e] + (tile - tilesOf[e]) * TILE;
        const int count = min(TILE, b.elemBegin[e + 1] - first);
        int maxW = 0;
        for (int l = 0; l < L; ++l) maxW = max(maxW, E.neurons[l]);
        double* act[2] = {sm, sm + maxW * netRow<TILE>()};
        double* dfBase = sm + 2 * maxW * netRow<TILE>();
        double* gv[2];
        {
            int sumD = 0;
            for (int l = 1; l < L; ++l) sumD += E.neurons[l];
            gv[0] = dfBase + sumD * netRow<TILE>();
            gv[1] = gv[0] + maxW * netRow<TILE>();
        }
        __syncthreads();   // the previous tile's reads of the buffers are done (its output may sit in act[0])
        // the tile's G rows, neuron-major (atoms beyond the element's last: zeros)
        const int nin0 = E.neurons[0];
        for (int idx = tid; idx < TILE * nin0; idx += kNetThreads)
        {
            const int a = idx / nin0, j = idx - a * nin0;
            act[0][j * netRow<TILE>() + a] = a < count ? b.G[(size_t)b.elemAtoms[first + a] * b.gStride + j] : 0.0;
        }
        __syncthreads();
        int cur = 0;
        double* df = dfBase;
        double* dfOf[kDevMaxLayers];
        for (int l = 1; l < L; ++l)
        {
            dfOf[l] = df;
            netForwardLayer<TILE>(E.activation[l], E.neurons[l - 1], E.neurons[l], model.weightsT + E.wOffset[l],
                            model.weights + E.bOffset[l], model.normalizeNeurons, act[cur], act[cur ^ 1], df, tid);
            df += E.neurons[l] * netRow<TILE>();
            __syncthreads();
            cur ^= 1;
        }
        if (tid < count) b.Eatom[b.elemAtoms[first + tid]] = act[cur][tid];
        if (!derivatives) continue;
        // reverse pass: g = f'_L (/ n_{L-1}), g_{l-1} = f'_{l-1} (W_l^T g_l) (/ n_{l-2}), dE/dG = W_1^T g_1
        for (int a = tid; a < TILE; a += kNetThreads)
        {
            double g0 = dfOf[L - 1][a];
            if (model.normalizeNeurons) g0 /= E.neurons[L - 2];
            gv[0][a] = g0;
        }
        __syncthreads();
        int gc = 0;
        for (int l = L - 1; l >= 2; --l)
        {
            netBackwardLayer<TILE>(E.neurons[l - 1], E.neurons[l], model.weights + E.wOffset[l], gv[gc], dfOf[l - 1],
                             model.normalizeNeurons ? E.neurons[l - 2] : 0, gv[gc ^ 1], tid);
            __syncthreads();
            gc ^= 1;
        }
        // dE/dG into the atoms' rows (rows of atoms beyond the element are not written)
        const int nout1 = E.neurons[1];
        const double* W1 = model.weights + E.wOffset[1];
        for (int u = tid; u < (TILE / kNetUnit) * nin0; u += kNetThreads)
        {
            const int j = u % nin0, q = u / nin0;
            double v[kNetUnit];
            netUnitSums<netRow<TILE>()>(nout1, [&](int k) { return __ldg(&W1[(size_t)k * nin0 + j]); }, gv[gc] + kNetUnit * q, v);
#pragma unroll
            for (int c = 0; c < kNetUnit; ++c)
                if (kNetUnit * q + c < count)
                    b.dEdG[(size_t)b.elemAtoms[first + kNetUnit * q + c] * b.gStride + j] = v[c];
        }
        __syncthreads();
    }
}

} // namespace

// E_s = sum of atomic energies of structure s (Mode::calculateEnergy,
// Mode.cpp:1876-1901), one warp per structure, fixed summation order.
__global__ void kEnergySum(BatchView b)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < b.S; s += warpsPerGrid)
    {
        const int a0 = b.structAtomBegin[s], a1 = b.structAtomBegin[s + 1];
        double e = 0.0;
        for (int a = a0 + lane; a < a1; a += 32) e += b.Eatom[a];
        e = warpSum(e);
        if (lane == 0) b.Estruct[s] = e;
    }
}

// F_i = self force + sum over neighbours j != i of the force E_j puts on i
// (Mode::calculateForces 2G part, Mode.cpp:1922-1984): the force E_j puts on
// i is stored on the reverse entry (j -> i) of each entry (i -> j).  One warp
// per atom: lanes stride over the atom's entries (coalesced index loads) and
// the partial sums are combined by a fixed shuffle tree, so the result is the
// same on every run.
__global__ void kGatherForces(BatchView b)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        const int64_t off = b.nbrOffset[i];
        const int64_t end = b.nbrOffset[i + 1];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        if (end <= b.nbrCapacity)
            for (int64_t e = off + lane; e < end; e += 32)
            {
                const int64_t r = b.rev[e];
                if (r < 0 || b.nbrJ[e] == i) continue;
                fx += b.hx[r];
                fy += b.hy[r];
                fz += b.hz[r];
            }
        fx = warpSum(fx);
        fy = warpSum(fy);
        fz = warpSum(fz);
        if (lane == 0)
        {
            b.F[3 * (size_t)i + 0] = b.fSelf[3 * (size_t)i + 0] + fx;
            b.F[3 * (size_t)i + 1] = b.fSelf[3 * (size_t)i + 1] + fy;
            b.F[3 * (size_t)i + 2] = b.fSelf[3 * (size_t)i + 2] + fz;
        }
    }
}

// Forces on the atoms named by external neighbour lists (the LAMMPS
// interface's local and ghost atoms, InterfaceLammps::getForces,
// InterfaceLammps.cpp:679-740): F_k = sum, in entry order, of the force h
// that each entry's centre puts on k (the entries naming k, listed by the
// transposed lists tOffset/tEntry), plus the self force when k is a centre
// (targetCenter[k] >= 0).  One warp per target, lanes strided over its
// entries, fixed shuffle tree: the same result on every run, no atomics.
__global__ void kGatherTargets(BatchView b, int numTargets, const int64_t* __restrict__ tOffset,
                               const int64_t* __restrict__ tEntry, const int* __restrict__ targetCenter,
                               double* __restrict__ F)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < numTargets; k += warpsPerGrid)
    {
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int64_t t = tOffset[k] + lane; t < tOffset[k + 1]; t += 32)
        {
            const int64_t e = tEntry[t];
            fx += b.hx[e];
            fy += b.hy[e];
            fz += b.hz[e];
        }
        fx = warpSum(fx);
        fy = warpSum(fy);
        fz = warpSum(fz);
        if (lane == 0)
        {
            const int c = targetCenter[k];
            if (c >= 0)
            {
                fx += b.fSelf[3 * (size_t)c + 0];
                fy += b.fSelf[3 * (size_t)c + 1];
                fz += b.fSelf[3 * (size_t)c + 2];
            }
            F[3 * (size_t)k + 0] = fx;
            F[3 * (size_t)k + 1] = fy;
            F[3 * (size_t)k + 2] = fz;
        }
    }
}

void launchGatherTargets(BatchView const& b, int numTargets, const int64_t* tOffset, const int64_t* tEntry,
                         const int* targetCenter, double* F, int sms, cudaStream_t st)
{
    int blocks = (numTargets + 7) / 8;
    if (blocks < 1) blocks = 1;
    if (blocks > sms * 32) blocks = sms * 32;
    kGatherTargets<<<blocks, 256, 0, st>>>(b, numTargets, tOffset, tEntry, targetCenter, F);
}

// Extrapolation check of Element::updateSymmetryFunctionStatistics
// (Element.cpp:462-541): unscaled G outside [Gmin, Gmax] by more than
// 1000 machine epsilon counts one warning.  One thread per atom.
__global__ void kExtrapolationCheck(DevModel model, BatchView b)
{
    const double eps = 1000.0 * 2.220446049250313080847e-16;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < b.N; i += gridDim.x * blockDim.x)
    {
        DevElement const& E = model.el[b.elem[i]];
        const double* g = b.G + (size_t)i * b.gStride;
        int count = 0;
        for (int s = 0; s < E.numSF; ++s)
        {
            DevScaling const& sc = model.scaling[E.sfBegin + s];
            const double v = unscaleG(sc, g[s]);
            if (v + eps < sc.Gmin || v - eps > sc.Gmax) count++;
        }
        b.atomWarnings[i] = count;
        if (count) atomicAdd(&b.status->extrapolationWarnings, count);
    }
}

// Symmetry-function statistics of the batch (SymFncStatistics::addValue,
// SymFncStatistics.cpp:80-89, as nnp-scaling collects them): per element and
// function the minimum, maximum, sum and sum of squares of the unscaled G.
// Block (chunk, element) = up to kStatChunk of the element's atoms in atom
// order, thread = function; kSFStatisticsReduce adds the chunks in order, so
// the sums do not depend on timing.
constexpr int kStatChunk = 1024;

__global__ void kSFStatistics(DevModel model, BatchView b, int maxChunks, int maxSF, double* __restrict__ partial)
{
    const int e = blockIdx.y, chunk = blockIdx.x;
    const int a0 = b.elemBegin[e] + chunk * kStatChunk;
    const int a1 = min(a0 + kStatChunk, b.elemBegin[e + 1]);
    if (a0 >= a1) return;
    DevElement const& E = model.el[e];
    double* out = partial + ((size_t)e * maxChunks + chunk) * 4 * maxSF;
    for (int s = threadIdx.x; s < E.numSF; s += blockDim.x)
    {
        DevScaling const& sc = model.scaling[E.sfBegin + s];
        double mn = CUDART_INF, mx = -CUDART_INF, sum = 0.0, sum2 = 0.0;
        for (int k = a0; k < a1; ++k)
        {
            const double v = unscaleG(sc, b.G[(size_t)b.elemAtoms[k] * b.gStride + s]);
            sum = __dadd_rn(sum, v);
            sum2 = __dadd_rn(sum2, __dmul_rn(v, v));
            mn = fmin(mn, v);
            mx = fmax(mx, v);
        }
        out[s] = mn;
        out[maxSF + s] = mx;
        out[2 * maxSF + s] = sum;
        out[3 * maxSF + s] = sum2;
    }
}

__global__ void kSFStatisticsReduce(DevModel model, BatchView b, int maxChunks, int maxSF,
                                    const double* __restrict__ partial, double* __restrict__ result)
{
    const int e = blockIdx.x;
    DevElement const& E = model.el[e];
    const int chunks = (b.elemBegin[e + 1] - b.elemBegin[e] + kStatChunk - 1) / kStatChunk;
    for (int s = threadIdx.x; s < E.numSF; s += blockDim.x)
    {
        double mn = CUDART_INF, mx = -CUDART_INF, sum = 0.0, sum2 = 0.0;
        for (int c = 0; c < chunks; ++c)
        {
            const double* p = partial + ((size_t)e * maxChunks + c) * 4 * maxSF;
            mn = fmin(mn, p[s]);
            mx = fmax(mx, p[maxSF + s]);
            sum = __dadd_rn(sum, p[2 * maxSF + s]);
            sum2 = __dadd_rn(sum2, p[3 * maxSF + s]);
        }
        double* r = result + (size_t)e * 4 * maxSF;
        r[s] = mn;
        r[maxSF + s] = mx;
        r[2 * maxSF + s] = sum;
        r[3 * maxSF + s] = sum2;
    }
}

void launchSFStatistics(DevModel const& m, BatchView const& b, int numElements, int maxChunks, int maxSF,
                        double* partial, double* result, cudaStream_t st)
{
    kSFStatistics<<<dim3(maxChunks, numElements), 128, 0, st>>>(m, b, maxChunks, maxSF, partial);
    kSFStatisticsReduce<<<numElements, 128, 0, st>>>(m, b, maxChunks, maxSF, partial, result);
}

void launchExtrapolationCheck(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    int blocks = (b.N + 127) / 128;
    if (blocks < 1) blocks = 1;
    if (blocks > sms * 16) blocks = sms * 16;
    kExtrapolationCheck<<<blocks, 128, 0, st>>>(m, b);
}

void launchNetworkFP64(DevModel const& m, BatchView const& b, int derivatives, int sms, cudaStream_t st)
{
    // tiles of 32 atoms (16 for wide networks) while their shared memory leaves at least two blocks per SM
    int d32 = 0, d16 = 0, t32 = 0, t16 = 0;
    for (int e = 0; e < m.numElements; ++e)
    {
        d32 = std::max(d32, netSmemDoubles(m.el[e], netRow<32>()));
        d16 = std::max(d16, netSmemDoubles(m.el[e], netRow<16>()));
        t32 += (b.elemBegin[e + 1] - b.elemBegin[e] + 31) / 32;
        t16 += (b.elemBegin[e + 1] - b.elemBegin[e] + 15) / 16;
    }
    auto tiled = [&](auto kernel, size_t bytes, int tiles) {
        if (tiles == 0) return;
        setDynamicSmemOnce(reinterpret_cast<const void*>(kernel), bytes);
        const int perSM = std::max(1, std::min(4, (int)(233472 / (bytes + 1024))));
        kernel<<<std::min(tiles, sms * perSM), kNetThreads, bytes, st>>>(m, b, derivatives);
    };
    constexpr size_t kTileBudget = 110 * 1024;
    if ((size_t)d32 * sizeof(double) <= kTileBudget) return tiled(kNetworkTiled<32>, (size_t)d32 * sizeof(double), t32);
    if ((size_t)d16 * sizeof(double) <= kTileBudget) return tiled(kNetworkTiled<16>, (size_t)d16 * sizeof(double), t16);
    size_t smem = sizeof(NNWarpSmem) * kNNWarps;
    setDynamicSmemOnce(reinterpret_cast<const void*>(kNetworkFP64), smem);
    int blocks = (b.N + kNNWarps - 1) / kNNWarps;
    if (blocks < 1) blocks = 1;
    if (blocks > sms * 8) blocks = sms * 8;
    kNetworkFP64<<<blocks, kNNWarps * 32, smem, st>>>(m, b, derivatives);
}

void launchEnergySum(BatchView const& b, cudaStream_t st)
{
    int blocks = (b.S + 7) / 8;
    if (blocks < 1) blocks = 1;
    kEnergySum<<<blocks, 256, 0, st>>>(b);
}

void launchGatherForces(BatchView const& b, int sms, cudaStream_t st)
{
    int blocks = (b.N + 7) / 8;
    if (blocks < 1) blocks = 1;
    if (blocks > sms * 32) blocks = sms * 32;
    kGatherForces<<<blocks, 256, 0, st>>>(b);
}

} // namespace n2p2b200
