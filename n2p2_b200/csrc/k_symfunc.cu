// Symmetry-function kernels of the API form (G2 radial, G3 narrow angular,
// G9 wide angular) on sm_100a, one warp per centre atom with the atom's
// neighbour list staged in shared memory.  (The evaluation path's G and force
// kernels are in sf_fast.cuh, instantiated by k_sf_fast_f64.cu / k_sf_fast_f32.cu.)
//
//   kSFDerivatives G and dG/dr stored per neighbour row (the Atom::Neighbor::dGdr
//                  layout of Element::setupSymmetryFunctionMemory,
//                  Element.cpp:289-311) for callers that read dG/dr.
//   kContractStored the force contraction of stored dG/dr with dE/dG.
//   kCutoffValues  f_c and df_c of every neighbour entry.
//
// Reference formulas: SymGrpExpRad::calculate (SymGrpExpRad.cpp:144-239),
// SymGrpExpAngn::calculate (SymGrpExpAngn.cpp:156-403),
// SymGrpExpAngw::calculate (SymGrpExpAngw.cpp:156-376).
//
// Work split without atomics: lane l owns the neighbours j = l, l+32, ...
// and visits partners k on a circle, k = j+t mod n: the full circle
// accumulates the owner's dG/dr rows privately, the first half circle the G
// values (each unordered pair once).  All sums run in a fixed order, so
// results are bitwise reproducible.
#include "kernels_common.cuh"
#include "kernels.hpp"

namespace n2p2b200 {

namespace {

constexpr int kChunk = 16;    // members evaluated per sweep over the partners

// Neighbour staging area of one warp: FP64 or FP32 geometry + cutoff values.
template <typename T, int CAP>
struct NbrStage
{
    T x[CAP], y[CAP], z[CAP], d[CAP], fc[CAP], dfc[CAP];
    int e[CAP];
};

template <typename T>
__device__ __forceinline__ T texp(T v);
template <>
__device__ __forceinline__ double texp<double>(double v) { return exp(v); }
template <>
__device__ __forceinline__ float texp<float>(float v) { return __expf(v); }

template <typename T>
__device__ __forceinline__ T tsqrt(T v);
template <>
__device__ __forceinline__ double tsqrt<double>(double v) { return sqrt(v); }
template <>
__device__ __forceinline__ float tsqrt<float>(float v) { return sqrtf(v); }

template <typename T>
__device__ __forceinline__ T tpow(T b, T e);
template <>
__device__ __forceinline__ double tpow<double>(double b, double e) { return pow(b, e); }
template <>
__device__ __forceinline__ float tpow<float>(float b, float e) { return __powf(b, e); }

// Stage the neighbours of one atom.  Neighbour data are FP64 in HBM; the
// mixed form converts once here.  Cutoff values of the group's cutoff slot
// come from the per-entry table built in FP64.
template <typename T, int CAP>
__device__ __forceinline__ void stageNeighbors(NbrStage<T, CAP>& st, int64_t off, int n, BatchView const& b,
                                               int slot, int lane)
{
    const double* fcs = b.nbrFc + (size_t)slot * b.nbrCapacity;
    const double* dfcs = b.nbrDfc + (size_t)slot * b.nbrCapacity;
    __syncwarp();
    for (int m = lane; m < n; m += 32)
    {
        st.x[m] = (T)b.nbrDx[off + m];
        st.y[m] = (T)b.nbrDy[off + m];
        st.z[m] = (T)b.nbrDz[off + m];
        st.d[m] = (T)b.nbrD[off + m];
        st.fc[m] = (T)fcs[off + m];
        st.dfc[m] = (T)dfcs[off + m];
        st.e[m] = b.elem[b.nbrJ[off + m]];
    }
    __syncwarp();
}

// Atoms with at most CAP neighbours go to the standard variant; the rare
// atoms with more use the large-capacity variant (one warp per block).
template <int CAP, int LOWER>
__device__ __forceinline__ bool takesAtom(int n)
{
    return n <= CAP && n > LOWER;
}

__device__ __forceinline__ int halfRange(int j, int n)
{
    return (n - 1) / 2 + (((n & 1) == 0 && j < n / 2) ? 1 : 0);
}

} // namespace

// ---------------------------------------------------------------------------
// G and stored dG/dr (API form, FP64)
// ---------------------------------------------------------------------------
// Device dG/dr layout: [row][entry][xyz], rows counted in the centre
// element's table for the neighbour's element, so for a fixed row the
// entries of a warp are contiguous (coalesced stores and loads).
// Self derivatives: [atom][sf][xyz] with the G stride.
template <int CAP, int WARPS, int LOWER>
__global__ void __launch_bounds__(WARPS * 32) kSFDerivatives(DevModel model, BatchView b)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    NbrStage<double, CAP>* stage = reinterpret_cast<NbrStage<double, CAP>*>(smemRaw);
    using T = double;
    constexpr int kC = 8;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    // the warp's atoms i = warp + k warpsPerGrid, tested 32 at a time for the tier
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (int k0 = 0; warp + k0 * warpsPerGrid < b.N; k0 += 32)
    {
        const int mine = warp + (k0 + lane) * warpsPerGrid;
        bool inTier = false;
        if (mine < b.N && b.nbrOffset[mine + 1] <= b.nbrCapacity)
            inTier = takesAtom<CAP, LOWER>((int)(b.nbrOffset[mine + 1] - b.nbrOffset[mine]));
        unsigned todo = __ballot_sync(kFullMask, inTier);
        while (todo)
        {
            const int i = warp + (k0 + __ffs(todo) - 1) * warpsPerGrid;
            todo &= todo - 1;
            const int64_t off = b.nbrOffset[i];
            const int64_t end = b.nbrOffset[i + 1];
            if (end > b.nbrCapacity) continue;
            const int n = (int)(end - off);
            if (!takesAtom<CAP, LOWER>(n)) continue;
            NbrStage<double, CAP>& nb = stage[w];
            const int ec = b.elem[i];
            DevElement const& E = model.el[ec];
            for (int r = 0; r < model.maxRows; ++r)
                for (int j = lane; j < n; j += 32)
                {
                    double* p = b.dGdr + ((size_t)r * b.nbrCapacity + off + j) * 3;
                    p[0] = 0.0;
                    p[1] = 0.0;
                    p[2] = 0.0;
                }
            int stagedSlot = -1;
            for (int g = 0; g < E.groupCount; ++g)
            {
                DevGroup const G = model.groups[E.groupBegin + g];
                if (G.cutoffSlot != stagedSlot)
                {
                    stageNeighbors<double, CAP>(nb, off, n, b, G.cutoffSlot, lane);
                    stagedSlot = G.cutoffSlot;
                }
                const T rc = G.rc, rc2 = G.rc2;
                for (int m0 = 0; m0 < G.memberCount; m0 += kC)
                {
                    const int mc = min(kC, G.memberCount - m0);
                    const DevMember* mem = model.members + G.memberBegin + m0;
                    T acc[kC], selfx[kC], selfy[kC], selfz[kC];
    #pragma unroll
                    for (int q = 0; q < kC; ++q) acc[q] = selfx[q] = selfy[q] = selfz[q] = 0.0;
                    if (G.type == 2)
                    {
                        for (int j = lane; j < n; j += 32)
                        {
                            if (nb.e[j] != G.e1 || !(nb.d[j] < rc)) continue;
                            const T r = nb.d[j], fc = nb.fc[j], dfc = nb.dfc[j];
                            const T x = nb.x[j], y = nb.y[j], z = nb.z[j];
    #pragma unroll
                            for (int q = 0; q < kC; ++q)
                            {
                                if (q < mc)
                                {
                                    DevMember const& M = mem[q];
                                    const T pexp = exp(-M.eta * (r - M.rs) * (r - M.rs));
                                    acc[q] += pexp * fc;
                                    const T p1 = M.factorNorm * (dfc - 2.0 * M.eta * (r - M.rs) * fc) * pexp / r;
                                    selfx[q] += p1 * x;
                                    selfy[q] += p1 * y;
                                    selfz[q] += p1 * z;
                                    double* p = b.dGdr + ((size_t)M.rowE1 * b.nbrCapacity + off + j) * 3;
                                    p[0] -= p1 * x;
                                    p[1] -= p1 * y;
                                    p[2] -= p1 * z;
                                }
                            }
                        }
                    }
                    else
                    {
                        const bool narrow = (G.type == 3);
                        for (int j = lane; j < n; j += 32)
                        {
                            const int ej = nb.e[j];
                            const T rij = nb.d[j];
                            if (!((ej == G.e1 || ej == G.e2) && rij < rc)) continue;
                            const int needK = (ej == G.e1) ? G.e2 : G.e1;
                            const T x1 = nb.x[j], y1 = nb.y[j], z1 = nb.z[j], fcij = nb.fc[j], dfcij = nb.dfc[j];
                            const T r2ij = rij * rij;
                            const int Hg = halfRange(j, n);
                            T rowx[kC], rowy[kC], rowz[kC];
    #pragma unroll
                            for (int q = 0; q < kC; ++q) rowx[q] = rowy[q] = rowz[q] = 0.0;
                            for (int t = 1; t <= n - 1; ++t)
                            {
                                int k = j + t;
                                if (k >= n) k -= n;
                                if (nb.e[k] != needK || !(nb.d[k] < rc)) continue;
                                const T x2 = nb.x[k], y2 = nb.y[k], z2 = nb.z[k];
                                const T dx3 = x2 - x1, dy3 = y2 - y1, dz3 = z2 - z1;
                                const T rjk2 = dx3 * dx3 + dy3 * dy3 + dz3 * dz3;
                                if (narrow && !(rjk2 < rc2)) continue;
                                const T rik = nb.d[k], fcik = nb.fc[k];
                                T pfc, pr1, pr3 = 0.0, rjk = 0.0, r2sum;
                                if (narrow)
                                {
                                    rjk = sqrt(rjk2);
                                    double fcjk, dfcjk;
                                    cutoffFdf(model.cutoff[G.cutoffSlot], rjk, fcjk, dfcjk);
                                    pfc = fcij * fcik * fcjk;
                                    pr1 = fcik * fcjk * dfcij / rij;
                                    pr3 = fcij * fcik * dfcjk / rjk;
                                    r2sum = r2ij + rik * rik + rjk * rjk;
                                }
                                else
                                {
                                    pfc = fcij * fcik;
                                    pr1 = fcik * dfcij / rij;
                                    r2sum = r2ij + rik * rik;
                                }
                                const T rinv = 1.0 / rij / rik;
                                const T cost = (x1 * x2 + y1 * y2 + z1 * z2) * rinv;
                                const bool countG = (t <= Hg);
                                T vexp = 0.0, rijs = 0.0, rjks = 0.0;
    #pragma unroll
                                for (int q = 0; q < kC; ++q)
                                {
                                    if (q < mc)
                                    {
                                        DevMember const& M = mem[q];
                                        if (M.calcExp || q == 0)
                                        {
                                            if (M.rs > 0.0)
                                            {
                                                rijs = rij - M.rs;
                                                const T riks = rik - M.rs;
                                                rjks = rjk - M.rs;
                                                vexp = exp(-M.eta * (narrow ? (rijs * rijs + riks * riks + rjks * rjks)
                                                                            : (rijs * rijs + riks * riks)));
                                            }
                                            else vexp = exp(-M.eta * r2sum);
                                        }
                                        const T plambda = 1.0 + M.lambda * cost;
                                        T fg = vexp;
                                        if (plambda <= 0.0) fg = 0.0;
                                        else
                                        {
                                            if (M.useIntPow) fg *= powInt<T>(plambda, M.zetaInt - 1);
                                            else fg *= pow(plambda, M.zeta - 1.0);
                                        }
                                        if (countG) acc[q] += fg * plambda * pfc;
                                        fg *= M.factorNorm;
                                        const T pfczl = pfc * M.zetaLambda;
                                        const T p2etapl = plambda * M.factorDeriv;
                                        T p1, p3;
                                        if (M.rs > 0.0)
                                        {
                                            p1 = fg * (pfczl * (rinv - cost / r2ij - p2etapl * rijs / rij) + pr1 * plambda);
                                            p3 = narrow ? fg * (pfczl * (rinv + p2etapl * rjks / rjk) - pr3 * plambda)
                                                        : fg * pfczl * rinv;
                                        }
                                        else
                                        {
                                            p1 = fg * (pfczl * (rinv - cost / r2ij - p2etapl) + pr1 * plambda);
                                            p3 = narrow ? fg * (pfczl * (rinv + p2etapl) - pr3 * plambda)
                                                        : fg * pfczl * rinv;
                                        }
                                        selfx[q] += p1 * x1;
                                        selfy[q] += p1 * y1;
                                        selfz[q] += p1 * z1;
                                        rowx[q] -= p1 * x1 + p3 * dx3;
                                        rowy[q] -= p1 * y1 + p3 * dy3;
                                        rowz[q] -= p1 * z1 + p3 * dz3;
                                    }
                                }
                            }
    #pragma unroll
                            for (int q = 0; q < kC; ++q)
                            {
                                if (q < mc)
                                {
                                    const int row = (ej == G.e1) ? mem[q].rowE1 : mem[q].rowE2;
                                    double* p = b.dGdr + ((size_t)row * b.nbrCapacity + off + j) * 3;
                                    p[0] += rowx[q];
                                    p[1] += rowy[q];
                                    p[2] += rowz[q];
                                }
                            }
                        }
                    }
    #pragma unroll
                    for (int q = 0; q < kC; ++q)
                    {
                        if (q < mc)
                        {
                            double s = warpSum(acc[q]);
                            const double sx = warpSum(selfx[q]), sy = warpSum(selfy[q]), sz = warpSum(selfz[q]);
                            if (lane == q)
                            {
                                DevMember const& M = mem[q];
                                if (G.type != 2) s *= M.gNorm;
                                b.G[(size_t)i * b.gStride + M.sf] = scaleG(model.scaling[E.sfBegin + M.sf], s);
                                double* p = b.dGdrSelf + ((size_t)i * b.gStride + M.sf) * 3;
                                p[0] = sx;
                                p[1] = sy;
                                p[2] = sz;
                            }
                        }
                    }
                }
            }
        }
    }

}

// Per-entry contraction of stored dG/dr with dE/dG:
//   h_e = -sum_r dEdG[table(r)] dGdr[r][e]   (Atom::calculatePairForceShort, Atom.cpp:381-401)
//   self = -sum_s dEdG[s] dGdr_self[s]       (Atom::calculateSelfForceShort, Atom.cpp:371-379)
// summed sequentially in the reference's row order.
__global__ void __launch_bounds__(256) kContractStored(DevModel model, BatchView b)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        const int64_t off = b.nbrOffset[i];
        const int64_t end = b.nbrOffset[i + 1];
        if (end > b.nbrCapacity) continue;
        const int ec = b.elem[i];
        DevElement const& E = model.el[ec];
        const double* w = b.dEdG + (size_t)i * b.gStride;
        for (int64_t e = off + lane; e < end; e += 32)
        {
            const int en = b.elem[b.nbrJ[e]];
            const int rows = E.rows[en];
            const int* table = model.rowTable + E.tableBegin[en];
            double fx = 0.0, fy = 0.0, fz = 0.0;
            for (int r = 0; r < rows; ++r)
            {
                const double c = w[table[r]];
                const double* p = b.dGdr + ((size_t)r * b.nbrCapacity + e) * 3;
                fx -= c * p[0];
                fy -= c * p[1];
                fz -= c * p[2];
            }
            b.hx[e] = fx;
            b.hy[e] = fy;
            b.hz[e] = fz;
        }
        if (lane == 0)
        {
            double fx = 0.0, fy = 0.0, fz = 0.0;
            for (int s = 0; s < E.numSF; ++s)
            {
                const double* p = b.dGdrSelf + ((size_t)i * b.gStride + s) * 3;
                fx -= w[s] * p[0];
                fy -= w[s] * p[1];
                fz -= w[s] * p[2];
            }
            b.fSelf[3 * (size_t)i + 0] = fx;
            b.fSelf[3 * (size_t)i + 1] = fy;
            b.fSelf[3 * (size_t)i + 2] = fz;
        }
    }
}

// f_c / df_c of every neighbour entry for each distinct cutoff (FP64).
__global__ void kCutoffValues(DevModel model, BatchView b)
{
    const int64_t total = b.status->totalNeighbors < b.nbrCapacity ? b.status->totalNeighbors : b.nbrCapacity;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    {
        const double r = b.nbrD[e];
        for (int s = 0; s < model.numCutoffSlots; ++s)
        {
            double fc, dfc;
            cutoffFdf(model.cutoff[s], r, fc, dfc);
            b.nbrFc[(size_t)s * b.nbrCapacity + e] = fc;
            b.nbrDfc[(size_t)s * b.nbrCapacity + e] = dfc;
        }
    }
}

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------
namespace {

constexpr int kStdCap = 256, kStdWarps = 4;
constexpr int kBigCap = 2048, kBigWarps = 1;

int warpGrid(int N, int warpsPerBlock, int sms, int perSM)
{
    int blocksNeeded = (N + warpsPerBlock - 1) / warpsPerBlock;
    int cap = sms * perSM;
    return blocksNeeded < cap ? (blocksNeeded > 0 ? blocksNeeded : 1) : cap;
}

// Opt in to more than 48 KB of dynamic shared memory.  The attribute is set
// before the first launch of each instantiation (outside graph capture: the
// first evaluation of a batch always launches directly).
template <typename K>
void setSmem(K kernel, size_t bytes)
{
    setDynamicSmemOnce(reinterpret_cast<const void*>(kernel), bytes);
}

} // namespace

void launchCutoffValues(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    kCutoffValues<<<sms * 16, 256, 0, st>>>(m, b);
}

void launchSFDerivatives(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    size_t s1 = sizeof(NbrStage<double, kStdCap>) * kStdWarps;
    size_t s2 = sizeof(NbrStage<double, kBigCap>) * kBigWarps;
    setSmem(kSFDerivatives<kStdCap, kStdWarps, -1>, s1);
    setSmem(kSFDerivatives<kBigCap, kBigWarps, kStdCap>, s2);
    kSFDerivatives<kStdCap, kStdWarps, -1><<<warpGrid(b.N, kStdWarps, sms, 16), kStdWarps * 32, s1, st>>>(m, b);
    kSFDerivatives<kBigCap, kBigWarps, kStdCap><<<sms, kBigWarps * 32, s2, st>>>(m, b);
}

void launchContractStored(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    int blocks = (b.N + 7) / 8;
    if (blocks < 1) blocks = 1;
    if (blocks > sms * 32) blocks = sms * 32;
    kContractStored<<<blocks, 256, 0, st>>>(m, b);
}

} // namespace n2p2b200
