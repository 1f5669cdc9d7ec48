// Symmetry-function kernels (G2 radial, G3 narrow angular, G9 wide angular)
// on sm_100a, one warp per centre atom with the atom's neighbour list staged
// in shared memory.
//
//   kSFValues      G only (the input of the atomic networks).
//   kSFForces      the force pass of the adjoint schedule: with dE/dG known it
//                  evaluates, for every neighbour entry (i -> j), the force that
//                  E_i puts on j, and the self force on i, without storing dG/dr.
//   kSFDerivatives G and dG/dr stored per neighbour row (the Atom::Neighbor::dGdr
//                  layout of Element::setupSymmetryFunctionMemory,
//                  Element.cpp:289-311) for callers that read dG/dr.
//
// Reference formulas: SymGrpExpRad::calculate (SymGrpExpRad.cpp:144-239),
// SymGrpExpAngn::calculate (SymGrpExpAngn.cpp:156-403),
// SymGrpExpAngw::calculate (SymGrpExpAngw.cpp:156-376).
//
// Work split without atomics: lane l owns the neighbours j = l, l+32, ...
// Angular terms: the owner of j visits partners k on a circle, k = j+t mod n.
// For G the half circle is enough (each unordered pair once); the force pass
// visits the full circle so every owner accumulates its own j-row, and the
// self term, privately.  All sums run in a fixed order, so results are
// bitwise reproducible.
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
// G values
// ---------------------------------------------------------------------------
template <typename T, int CAP, int WARPS, int LOWER>
__global__ void __launch_bounds__(WARPS * 32) kSFValues(DevModel model, BatchView b)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    NbrStage<T, CAP>* stage = reinterpret_cast<NbrStage<T, CAP>*>(smemRaw);
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        const int64_t off = b.nbrOffset[i];
        const int64_t end = b.nbrOffset[i + 1];
        if (end > b.nbrCapacity) continue;
        const int n = (int)(end - off);
        if (LOWER >= 0 && n > CAP)
        {
            if (lane == 0) atomicAdd(&b.status->badInput, 1);
            continue;
        }
        if (!takesAtom<CAP, LOWER>(n)) continue;
        NbrStage<T, CAP>& nb = stage[w];
        const int ec = b.elem[i];
        DevElement const& E = model.el[ec];
        int stagedSlot = -1;
        for (int g = 0; g < E.groupCount; ++g)
        {
            DevGroup const G = model.groups[E.groupBegin + g];
            if (G.cutoffSlot != stagedSlot)
            {
                stageNeighbors<T, CAP>(nb, off, n, b, G.cutoffSlot, lane);
                stagedSlot = G.cutoffSlot;
            }
            const T rc = (T)G.rc;
            const T rc2 = (T)G.rc2;
            for (int m0 = 0; m0 < G.memberCount; m0 += kChunk)
            {
                const int mc = min(kChunk, G.memberCount - m0);
                const DevMember* mem = model.members + G.memberBegin + m0;
                T acc[kChunk];
#pragma unroll
                for (int q = 0; q < kChunk; ++q) acc[q] = T(0);
                if (G.type == 2)
                {
                    for (int j = lane; j < n; j += 32)
                    {
                        if (nb.e[j] != G.e1 || !(nb.d[j] < rc)) continue;
                        const T r = nb.d[j], fc = nb.fc[j];
#pragma unroll
                        for (int q = 0; q < kChunk; ++q)
                        {
                            if (q < mc)
                            {
                                const T eta = (T)__ldg(&mem[q].eta), rs = (T)__ldg(&mem[q].rs);
                                acc[q] += texp<T>(-eta * (r - rs) * (r - rs)) * fc;
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
                        const T x1 = nb.x[j], y1 = nb.y[j], z1 = nb.z[j], fcij = nb.fc[j];
                        const T r2ij = rij * rij;
                        const int H = halfRange(j, n);
                        for (int t0 = 1; t0 <= H; t0 += 32)
                        {
                            const int tm = min(32, H - t0 + 1);
                            unsigned mask = 0;
                            for (int bb = 0; bb < tm; ++bb)
                            {
                                int k = j + t0 + bb;
                                if (k >= n) k -= n;
                                bool ok = nb.e[k] == needK && nb.d[k] < rc;
                                if (ok && narrow)
                                {
                                    const T dx = nb.x[k] - x1, dy = nb.y[k] - y1, dz = nb.z[k] - z1;
                                    ok = (dx * dx + dy * dy + dz * dz) < rc2;
                                }
                                mask |= (ok ? 1u : 0u) << bb;
                            }
                            while (mask)
                            {
                                const int bb = __ffs(mask) - 1;
                                mask &= mask - 1;
                                int k = j + t0 + bb;
                                if (k >= n) k -= n;
                                const T x2 = nb.x[k], y2 = nb.y[k], z2 = nb.z[k];
                                const T rik = nb.d[k];
                                T pfc = fcij * nb.fc[k];
                                T r2sum = r2ij + rik * rik;
                                T rjk = T(0);
                                if (narrow)
                                {
                                    const T dx3 = x2 - x1, dy3 = y2 - y1, dz3 = z2 - z1;
                                    rjk = tsqrt<T>(dx3 * dx3 + dy3 * dy3 + dz3 * dz3);
                                    double fjk, dfjk;
                                    cutoffFdf(model.cutoff[G.cutoffSlot], (double)rjk, fjk, dfjk);
                                    pfc *= (T)fjk;
                                    r2sum += rjk * rjk;
                                }
                                const T rinv = T(1) / rij / rik;
                                const T cost = (x1 * x2 + y1 * y2 + z1 * z2) * rinv;
                                T vexp = T(0);
#pragma unroll
                                for (int q = 0; q < kChunk; ++q)
                                {
                                    if (q < mc)
                                    {
                                        const DevMember* M = mem + q;
                                        if (__ldg(&M->calcExp) || q == 0)
                                        {
                                            const T eta = (T)__ldg(&M->eta), rs = (T)__ldg(&M->rs);
                                            if (rs > T(0))
                                            {
                                                const T a = rij - rs, c = rik - rs, e3 = rjk - rs;
                                                vexp = texp<T>(-eta * (narrow ? (a * a + c * c + e3 * e3)
                                                                              : (a * a + c * c)));
                                            }
                                            else vexp = texp<T>(-eta * r2sum);
                                        }
                                        const T plambda = T(1) + (T)__ldg(&M->lambda) * cost;
                                        T fg = vexp;
                                        if (plambda <= T(0)) fg = T(0);
                                        else
                                        {
                                            if (__ldg(&M->useIntPow)) fg *= powInt<T>(plambda, __ldg(&M->zetaInt) - 1);
                                            else fg *= tpow<T>(plambda, (T)__ldg(&M->zeta) - T(1));
                                        }
                                        acc[q] += fg * plambda * pfc;
                                    }
                                }
                            }
                        }
                    }
                }
                // Warp tree sums in a fixed order; then scaling in FP64.
#pragma unroll
                for (int q = 0; q < kChunk; ++q)
                {
                    if (q < mc)
                    {
                        double s = warpSum((double)acc[q]);
                        if (lane == q)
                        {
                            DevMember const& M = mem[q];
                            if (G.type != 2) s *= M.gNorm;
                            b.G[(size_t)i * b.gStride + M.sf] = scaleG(model.scaling[E.sfBegin + M.sf], s);
                        }
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Force pass (adjoint schedule)
// ---------------------------------------------------------------------------
// With w_s = dE_i/dG_s and a_s = w_s * factorNorm_s * fg_s (the weighted
// angular term of member s), the reference's per-member derivative
// prefactors p1, p3 (SymGrpExpAngn.cpp:305-337) contract to
//   P1 = pfc ((1/(rij rik) - cos/rij^2) T1 - Uij) + pr1 T3
//   P3 = pfc (1/(rij rik) T1 + Ujk) - pr3 T3
// with T1 = sum a zeta lambda, T3 = sum a plambda,
//      Uij = sum a zeta lambda plambda factorDeriv (rij - rs)/rij (Ujk alike),
// and the force that E_i puts on neighbour j is P1 dr_ij + P3 dr_jk summed
// over its partners k; the self force on i is -sum P1 dr_ij.
template <typename T, int CAP>
struct ForceSmem
{
    NbrStage<T, CAP> nb;
    double h[3][CAP];
    double w[kMaxSFPerElement];
};

template <typename T, int CAP, int WARPS, int LOWER>
__global__ void __launch_bounds__(WARPS * 32) kSFForces(DevModel model, BatchView b)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    ForceSmem<T, CAP>* sm = reinterpret_cast<ForceSmem<T, CAP>*>(smemRaw);
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        const int64_t off = b.nbrOffset[i];
        const int64_t end = b.nbrOffset[i + 1];
        if (end > b.nbrCapacity) continue;
        const int n = (int)(end - off);
        if (!takesAtom<CAP, LOWER>(n)) continue;
        ForceSmem<T, CAP>& S = sm[w];
        NbrStage<T, CAP>& nb = S.nb;
        const int ec = b.elem[i];
        DevElement const& E = model.el[ec];
        __syncwarp();
        for (int s = lane; s < E.numSF; s += 32) S.w[s] = b.dEdG[(size_t)i * b.gStride + s];
        for (int j = lane; j < n; j += 32) S.h[0][j] = S.h[1][j] = S.h[2][j] = 0.0;
        __syncwarp();
        double sfx = 0.0, sfy = 0.0, sfz = 0.0;
        int stagedSlot = -1;
        for (int g = 0; g < E.groupCount; ++g)
        {
            DevGroup const G = model.groups[E.groupBegin + g];
            if (G.cutoffSlot != stagedSlot)
            {
                stageNeighbors<T, CAP>(nb, off, n, b, G.cutoffSlot, lane);
                stagedSlot = G.cutoffSlot;
            }
            const T rc = (T)G.rc;
            const T rc2 = (T)G.rc2;
            const DevMember* mem = model.members + G.memberBegin;
            const int M = G.memberCount;
            if (G.type == 2)
            {
                for (int j = lane; j < n; j += 32)
                {
                    if (nb.e[j] != G.e1 || !(nb.d[j] < rc)) continue;
                    const T r = nb.d[j], fc = nb.fc[j], dfc = nb.dfc[j];
                    T P = T(0);
                    for (int q = 0; q < M; ++q)
                    {
                        const T eta = (T)__ldg(&mem[q].eta), rs = (T)__ldg(&mem[q].rs);
                        const T pexp = texp<T>(-eta * (r - rs) * (r - rs));
                        const T p1 = (T)__ldg(&mem[q].factorNorm) * (dfc - T(2) * eta * (r - rs) * fc) * pexp / r;
                        P += (T)S.w[__ldg(&mem[q].sf)] * p1;
                    }
                    const double Pd = (double)P;
                    const double ddx = (double)nb.x[j] * Pd, ddy = (double)nb.y[j] * Pd, ddz = (double)nb.z[j] * Pd;
                    S.h[0][j] += ddx;
                    S.h[1][j] += ddy;
                    S.h[2][j] += ddz;
                    sfx -= ddx;
                    sfy -= ddy;
                    sfz -= ddz;
                }
                continue;
            }
            const bool narrow = (G.type == 3);
            for (int j = lane; j < n; j += 32)
            {
                const int ej = nb.e[j];
                const T rij = nb.d[j];
                if (!((ej == G.e1 || ej == G.e2) && rij < rc)) continue;
                const int needK = (ej == G.e1) ? G.e2 : G.e1;
                const T x1 = nb.x[j], y1 = nb.y[j], z1 = nb.z[j], fcij = nb.fc[j], dfcij = nb.dfc[j];
                const T r2ij = rij * rij;
                T ax = T(0), ay = T(0), az = T(0);
                T sx = T(0), sy = T(0), sz = T(0);
                const int H = n - 1;
                for (int t0 = 1; t0 <= H; t0 += 32)
                {
                    const int tm = min(32, H - t0 + 1);
                    unsigned mask = 0;
                    for (int bb = 0; bb < tm; ++bb)
                    {
                        int k = j + t0 + bb;
                        if (k >= n) k -= n;
                        bool ok = nb.e[k] == needK && nb.d[k] < rc;
                        if (ok && narrow)
                        {
                            const T dx = nb.x[k] - x1, dy = nb.y[k] - y1, dz = nb.z[k] - z1;
                            ok = (dx * dx + dy * dy + dz * dz) < rc2;
                        }
                        mask |= (ok ? 1u : 0u) << bb;
                    }
                    while (mask)
                    {
                        const int bb = __ffs(mask) - 1;
                        mask &= mask - 1;
                        int k = j + t0 + bb;
                        if (k >= n) k -= n;
                        const T x2 = nb.x[k], y2 = nb.y[k], z2 = nb.z[k];
                        const T rik = nb.d[k], fcik = nb.fc[k];
                        const T dx3 = x2 - x1, dy3 = y2 - y1, dz3 = z2 - z1;
                        T pfc, pr1, pr3 = T(0), rjk = T(0), r2sum;
                        const T rinv = T(1) / rij / rik;
                        const T cost = (x1 * x2 + y1 * y2 + z1 * z2) * rinv;
                        if (narrow)
                        {
                            rjk = tsqrt<T>(dx3 * dx3 + dy3 * dy3 + dz3 * dz3);
                            double fjk, dfjk;
                            cutoffFdf(model.cutoff[G.cutoffSlot], (double)rjk, fjk, dfjk);
                            const T fcjk = (T)fjk, dfcjk = (T)dfjk;
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
                        T T1 = T(0), T3 = T(0), Uij = T(0), Ujk = T(0);
                        T vexp = T(0), rijs = T(0), rjks = T(0);
                        for (int q = 0; q < M; ++q)
                        {
                            const DevMember* Mq = mem + q;
                            const T rs = (T)__ldg(&Mq->rs);
                            if (__ldg(&Mq->calcExp) || q == 0)
                            {
                                const T eta = (T)__ldg(&Mq->eta);
                                if (rs > T(0))
                                {
                                    rijs = rij - rs;
                                    const T riks = rik - rs;
                                    rjks = rjk - rs;
                                    vexp = texp<T>(-eta * (narrow ? (rijs * rijs + riks * riks + rjks * rjks)
                                                                  : (rijs * rijs + riks * riks)));
                                }
                                else vexp = texp<T>(-eta * r2sum);
                            }
                            const T plambda = T(1) + (T)__ldg(&Mq->lambda) * cost;
                            if (plambda <= T(0)) continue;
                            T fg = vexp;
                            if (__ldg(&Mq->useIntPow)) fg *= powInt<T>(plambda, __ldg(&Mq->zetaInt) - 1);
                            else fg *= tpow<T>(plambda, (T)__ldg(&Mq->zeta) - T(1));
                            const T a = (T)S.w[__ldg(&Mq->sf)] * (T)__ldg(&Mq->factorNorm) * fg;
                            const T zl = (T)__ldg(&Mq->zetaLambda);
                            const T azq = a * zl * plambda * (T)__ldg(&Mq->factorDeriv);
                            T1 += a * zl;
                            T3 += a * plambda;
                            if (rs > T(0))
                            {
                                Uij += azq * rijs / rij;
                                if (narrow) Ujk += azq * rjks / rjk;
                            }
                            else
                            {
                                Uij += azq;
                                Ujk += azq;
                            }
                        }
                        const T P1 = pfc * ((rinv - cost / r2ij) * T1 - Uij) + pr1 * T3;
                        const T P3 = narrow ? (pfc * (rinv * T1 + Ujk) - pr3 * T3) : (pfc * rinv * T1);
                        ax += P1 * x1 + P3 * dx3;
                        ay += P1 * y1 + P3 * dy3;
                        az += P1 * z1 + P3 * dz3;
                        sx -= P1 * x1;
                        sy -= P1 * y1;
                        sz -= P1 * z1;
                    }
                }
                S.h[0][j] += (double)ax;
                S.h[1][j] += (double)ay;
                S.h[2][j] += (double)az;
                sfx += (double)sx;
                sfy += (double)sy;
                sfz += (double)sz;
            }
        }
        __syncwarp();
        for (int j = lane; j < n; j += 32)
        {
            b.hx[off + j] = S.h[0][j];
            b.hy[off + j] = S.h[1][j];
            b.hz[off + j] = S.h[2][j];
        }
        sfx = warpSum(sfx);
        sfy = warpSum(sfy);
        sfz = warpSum(sfz);
        if (lane == 0)
        {
            b.fSelf[3 * (size_t)i + 0] = sfx;
            b.fSelf[3 * (size_t)i + 1] = sfy;
            b.fSelf[3 * (size_t)i + 2] = sfz;
        }
    }
}

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
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
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

template <typename T>
static void sfValuesT(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    size_t s1 = sizeof(NbrStage<T, kStdCap>) * kStdWarps;
    size_t s2 = sizeof(NbrStage<T, kBigCap>) * kBigWarps;
    setSmem(kSFValues<T, kStdCap, kStdWarps, -1>, s1);
    setSmem(kSFValues<T, kBigCap, kBigWarps, kStdCap>, s2);
    kSFValues<T, kStdCap, kStdWarps, -1><<<warpGrid(b.N, kStdWarps, sms, 16), kStdWarps * 32, s1, st>>>(m, b);
    kSFValues<T, kBigCap, kBigWarps, kStdCap><<<sms, kBigWarps * 32, s2, st>>>(m, b);
}

template <typename T>
static void sfForcesT(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    size_t s1 = sizeof(ForceSmem<T, kStdCap>) * kStdWarps;
    size_t s2 = sizeof(ForceSmem<T, kBigCap>) * kBigWarps;
    setSmem(kSFForces<T, kStdCap, kStdWarps, -1>, s1);
    setSmem(kSFForces<T, kBigCap, kBigWarps, kStdCap>, s2);
    kSFForces<T, kStdCap, kStdWarps, -1><<<warpGrid(b.N, kStdWarps, sms, 16), kStdWarps * 32, s1, st>>>(m, b);
    kSFForces<T, kBigCap, kBigWarps, kStdCap><<<sms, kBigWarps * 32, s2, st>>>(m, b);
}

void launchSFValues(DevModel const& m, BatchView const& b, int precision, int sms, cudaStream_t st)
{
    if (precision == 0) sfValuesT<double>(m, b, sms, st);
    else sfValuesT<float>(m, b, sms, st);
}

void launchSFForces(DevModel const& m, BatchView const& b, int precision, int sms, cudaStream_t st)
{
    if (precision == 0) sfForcesT<double>(m, b, sms, st);
    else sfForcesT<float>(m, b, sms, st);
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
