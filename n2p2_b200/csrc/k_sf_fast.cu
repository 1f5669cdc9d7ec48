// Symmetry-function kernels of the evaluation path (G values and the adjoint
// force pass), one warp per centre atom.
//
// Formulas: SymGrpExpRad::calculate (SymGrpExpRad.cpp:144-239),
// SymGrpExpAngn::calculate (SymGrpExpAngn.cpp:156-403),
// SymGrpExpAngw::calculate (SymGrpExpAngw.cpp:156-376).
//
// Layout and schedule:
//  * The atom's neighbours are staged in shared memory sorted by element
//    (stable), so the partners of a group form contiguous blocks and no
//    element test is left in the triplet loops.  Per neighbour the stage holds
//    dr, r, 1/r, f_c, df_c/r and, per group, the Gaussian factors
//    exp(-eta_b r^2) of the group's bases.
//  * Gaussians: exp(-eta (rij^2 + rik^2 + rjk^2)) = E_b(rij) E_b(rik) exp(-eta_b rjk^2)
//    raised to an integer power when eta = k eta_b (plan built on the host),
//    so a triplet costs one exponential per base instead of one per eta.
//  * Work split without atomics: lane l owns the block members l, l+32, ...
//    For G each unordered pair is visited once (half circle within a block,
//    or owner block x partner block); the force pass visits ordered pairs so
//    every owner accumulates its own neighbour row and the self term in
//    registers.  Candidate partners are compacted 32 at a time into a
//    bitmask before the arithmetic, so lanes idle only at chunk ends.
//  * All sums run in a fixed order: results are bitwise reproducible.
#include "kernels_common.cuh"
#include "kernels.hpp"

namespace n2p2b200 {

namespace {

constexpr int kChunkF = 16;   // members per sweep in the G pass

template <typename T>
__device__ __forceinline__ T fexp(T v);
template <>
__device__ __forceinline__ double fexp<double>(double v) { return exp(v); }
template <>
__device__ __forceinline__ float fexp<float>(float v) { return __expf(v); }

template <typename T>
__device__ __forceinline__ T frsqrt(T v);
template <>
__device__ __forceinline__ double frsqrt<double>(double v) { return rsqrt(v); }
template <>
__device__ __forceinline__ float frsqrt<float>(float v) { return rsqrtf(v); }

template <typename T>
__device__ __forceinline__ T fpow(T b, T e);
template <>
__device__ __forceinline__ double fpow<double>(double b, double e) { return pow(b, e); }
template <>
__device__ __forceinline__ float fpow<float>(float b, float e) { return __powf(b, e); }

template <typename T, int CAP>
struct Stage
{
    T x[CAP], y[CAP], z[CAP], r[CAP], rinv[CAP], fc[CAP], dfcr[CAP];
    T E[kMaxStagedBases][CAP];
    short perm[CAP];                       // staged slot -> position in the atom's list
    int blockBegin[kDevMaxElements + 1];
};

// Per-group member parameters (shared by all lanes).
template <typename T>
struct Members
{
    T cw[kMaxMembers];       // force pass: dE/dG * factorNorm
    T zl[kMaxMembers], fd[kMaxMembers], lambda[kMaxMembers], zeta[kMaxMembers], eta[kMaxMembers],
        rs[kMaxMembers];
    int zint[kMaxMembers], base[kMaxMembers], pw[kMaxMembers], flags[kMaxMembers];  // 1 intPow, 2 calcExp
};

constexpr int kQueue = 64;   // accepted (owner, partner) pairs waiting for a full warp

template <typename T, int CAP>
struct ValuesSmem
{
    Stage<T, CAP> st;
    Members<T> mb;
    int queue[kQueue];
};

template <typename T, int CAP>
struct ForcesSmem
{
    Stage<T, CAP> st;
    Members<T> mb;
    double h[3][CAP];
    int queue[kQueue];
};

// Candidate pairs of one angular group, enumerated owner-major in phases:
//   kind 0  circular: owner a in [0, nO), partner (a + 1 + t) mod nO, t < D
//   kind 1  half-extra: owner a < nO / 2, partner a + nO / 2 (even nO, G pass)
//   kind 2  rectangular: owner a in [0, nO), partner t in [0, D) of another block
struct Phase
{
    int kind, O0, nO, P0, D, count;
};

// Lane-private decoding of candidate p = p0 + lane, advanced by 32 per step
// without integer division in the loop.
struct Cursor
{
    int a, t;
    __device__ __forceinline__ void init(Phase const& ph, int lane)
    {
        if (ph.kind == 1 || ph.D <= 0)
        {
            a = lane;
            t = 0;
        }
        else
        {
            a = lane / ph.D;
            t = lane - a * ph.D;
        }
    }
    __device__ __forceinline__ void advance(Phase const& ph)
    {
        if (ph.kind == 1)
        {
            a += 32;
            return;
        }
        t += 32;
        while (t >= ph.D)
        {
            t -= ph.D;
            ++a;
        }
    }
    __device__ __forceinline__ void slots(Phase const& ph, int& so, int& sp) const
    {
        so = ph.O0 + a;
        if (ph.kind == 0)
        {
            int b = a + 1 + t;
            if (b >= ph.nO) b -= ph.nO;
            sp = ph.O0 + b;
        }
        else if (ph.kind == 1) sp = ph.O0 + a + ph.nO / 2;
        else sp = ph.P0 + t;
    }
};

// Test the next 32 candidates of a phase and append the accepted ones, in
// candidate order, to the warp's queue (qn entries from q[0]).
template <typename T, int CAP>
__device__ __forceinline__ void enqueueCandidates(Stage<T, CAP> const& S, Phase const& ph, Cursor& cur, int p0,
                                                  T rc, T rc2, bool narrow, int* queue, int& qn, int lane)
{
    const int p = p0 + lane;
    bool ok = false;
    int so = 0, sp = 0;
    if (p < ph.count)
    {
        cur.slots(ph, so, sp);
        ok = S.r[so] < rc && S.r[sp] < rc;
        if (ok && narrow)
        {
            const T dx = S.x[sp] - S.x[so], dy = S.y[sp] - S.y[so], dz = S.z[sp] - S.z[so];
            ok = (dx * dx + dy * dy + dz * dz) < rc2;
        }
    }
    const unsigned m = __ballot_sync(kFullMask, ok);
    if (ok) queue[qn + __popc(m & ((1u << lane) - 1u))] = (so << 16) | sp;
    qn += __popc(m);
    cur.advance(ph);
    __syncwarp();
}

// Drop the first `used` queue entries, keep the rest in order.
__device__ __forceinline__ void shiftQueue(int* queue, int& qn, int used, int lane)
{
    const int rest = qn - used;
    int v = (lane < rest) ? queue[used + lane] : 0;
    __syncwarp();
    if (lane < rest) queue[lane] = v;
    qn = rest;
    __syncwarp();
}

// Phases of a group: G pass (each unordered pair once) or force pass
// (ordered pairs, owner-major, both directions of a cross-element group).
__device__ __forceinline__ int groupPhases(int A0, int nA, int B0, int nB, bool same, bool ordered, Phase* ph)
{
    int n = 0;
    if (same)
    {
        if (nA < 2) return 0;
        if (ordered)
        {
            ph[n++] = Phase{0, A0, nA, A0, nA - 1, nA * (nA - 1)};
        }
        else
        {
            const int hb = (nA - 1) / 2;
            if (hb > 0) ph[n++] = Phase{0, A0, nA, A0, hb, nA * hb};
            if ((nA & 1) == 0) ph[n++] = Phase{1, A0, nA, A0, 0, nA / 2};
        }
    }
    else
    {
        if (nA == 0 || nB == 0) return 0;
        ph[n++] = Phase{2, A0, nA, B0, nB, nA * nB};
        if (ordered) ph[n++] = Phase{2, B0, nB, A0, nA, nA * nB};
    }
    return n;
}

// Neighbours of one atom into the stage, sorted by element (stable).
template <typename T, int CAP>
__device__ void stageGeometry(Stage<T, CAP>& S, int64_t off, int n, int numElements, BatchView const& b, int lane)
{
    __syncwarp();
    int base = 0;
    for (int e = 0; e < numElements; ++e)
    {
        if (lane == 0) S.blockBegin[e] = base;
        for (int m0 = 0; m0 < n; m0 += 32)
        {
            const int m = m0 + lane;
            const bool mine = (m < n) && (b.elem[b.nbrJ[off + m]] == e);
            const unsigned bal = __ballot_sync(kFullMask, mine);
            if (mine) S.perm[base + __popc(bal & ((1u << lane) - 1u))] = (short)m;
            base += __popc(bal);
        }
    }
    if (lane == 0) S.blockBegin[numElements] = base;
    __syncwarp();
    for (int s = lane; s < n; s += 32)
    {
        const int64_t e = off + S.perm[s];
        const double r = b.nbrD[e];
        S.x[s] = (T)b.nbrDx[e];
        S.y[s] = (T)b.nbrDy[e];
        S.z[s] = (T)b.nbrDz[e];
        S.r[s] = (T)r;
        S.rinv[s] = (T)(1.0 / r);
    }
    __syncwarp();
}

// f_c and df_c/r of the cutoff slot (values computed in FP64 per entry).
template <typename T, int CAP>
__device__ void stageCutoff(Stage<T, CAP>& S, int64_t off, int n, int slot, BatchView const& b, int lane)
{
    __syncwarp();
    const double* fc = b.nbrFc + (size_t)slot * b.nbrCapacity + off;
    const double* dfc = b.nbrDfc + (size_t)slot * b.nbrCapacity + off;
    for (int s = lane; s < n; s += 32)
    {
        const int m = S.perm[s];
        S.fc[s] = (T)fc[m];
        S.dfcr[s] = (T)(dfc[m] / b.nbrD[off + m]);
    }
    __syncwarp();
}

// Gaussian factors exp(-eta_b r^2) of the group's staged bases for the slots
// of the group's element blocks.
template <typename T, int CAP>
__device__ void stageFactors(Stage<T, CAP>& S, DevGroup const& G, int lane)
{
    __syncwarp();
    for (int pass = 0; pass < 2; ++pass)
    {
        const int e = pass == 0 ? G.e1 : G.e2;
        if (pass == 1 && G.e2 == G.e1) break;
        for (int s = S.blockBegin[e] + lane; s < S.blockBegin[e + 1]; s += 32)
        {
            const T r = S.r[s];
            for (int q = 0; q < G.numBases && q < kMaxStagedBases; ++q) S.E[q][s] = fexp<T>(-(T)G.baseEta[q] * r * r);
        }
    }
    __syncwarp();
}

template <typename T>
__device__ void stageMembers(Members<T>& mb, DevModel const& model, DevGroup const& G, const double* dEdG, int lane)
{
    __syncwarp();
    for (int q = lane; q < G.memberCount; q += 32)
    {
        DevMember const& M = model.members[G.memberBegin + q];
        mb.cw[q] = dEdG ? (T)(dEdG[M.sf] * M.factorNorm) : T(0);
        mb.zl[q] = (T)M.zetaLambda;
        mb.fd[q] = (T)M.factorDeriv;
        mb.lambda[q] = (T)M.lambda;
        mb.zeta[q] = (T)M.zeta;
        mb.eta[q] = (T)M.eta;
        mb.rs[q] = (T)M.rs;
        mb.zint[q] = M.zetaInt;
        mb.base[q] = M.expBase;
        mb.pw[q] = M.expPow;
        mb.flags[q] = (M.useIntPow ? 1 : 0) | (M.calcExp ? 2 : 0);
    }
    __syncwarp();
}

__device__ __forceinline__ int halfRange(int j, int n)
{
    return (n - 1) / 2 + (((n & 1) == 0 && j < n / 2) ? 1 : 0);
}

template <typename T>
__device__ __forceinline__ T angularPow(T pl, Members<T> const& mb, int q)
{
    return (mb.flags[q] & 1) ? powInt<T>(pl, mb.zint[q] - 1) : fpow<T>(pl, mb.zeta[q] - T(1));
}

} // namespace

// ---------------------------------------------------------------------------
// G values
// ---------------------------------------------------------------------------
template <typename T, int CAP, int WARPS, int LOWER>
__global__ void __launch_bounds__(WARPS * 32) kSFValuesF(DevModel model, BatchView b)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    ValuesSmem<T, CAP>& SM = reinterpret_cast<ValuesSmem<T, CAP>*>(smemRaw)[threadIdx.x >> 5];
    Stage<T, CAP>& S = SM.st;
    Members<T>& mb = SM.mb;
    const int lane = threadIdx.x & 31;
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
        if (!(n <= CAP && n > LOWER)) continue;
        const int ec = b.elem[i];
        DevElement const& E = model.el[ec];
        stageGeometry<T, CAP>(S, off, n, model.numElements, b, lane);
        int slot = -1;
        for (int g = 0; g < E.groupCount; ++g)
        {
            DevGroup const G = model.groups[E.groupBegin + g];
            if (G.cutoffSlot != slot)
            {
                stageCutoff<T, CAP>(S, off, n, G.cutoffSlot, b, lane);
                slot = G.cutoffSlot;
            }
            stageMembers<T>(mb, model, G, nullptr, lane);
            if (G.type != 2 && G.fast) stageFactors<T, CAP>(S, G, lane);
            const T rc = (T)G.rc, rc2 = (T)G.rc2;
            const DevMember* mem = model.members + G.memberBegin;
            for (int m0 = 0; m0 < G.memberCount; m0 += kChunkF)
            {
                const int mc = min(kChunkF, G.memberCount - m0);
                T acc[kChunkF];
#pragma unroll
                for (int q = 0; q < kChunkF; ++q) acc[q] = T(0);
                if (G.type == 2)
                {
                    for (int s = S.blockBegin[G.e1] + lane; s < S.blockBegin[G.e1 + 1]; s += 32)
                    {
                        const T r = S.r[s];
                        if (!(r < rc)) continue;
                        const T fc = S.fc[s];
                        T eb[kMaxBases];
#pragma unroll
                        for (int q = 0; q < kMaxBases; ++q)
                            eb[q] = (G.fast && q < G.numBases) ? fexp<T>(-(T)G.baseEta[q] * r * r) : T(0);
#pragma unroll
                        for (int q = 0; q < kChunkF; ++q)
                        {
                            if (q < mc)
                            {
                                const int qq = m0 + q;
                                T v;
                                if (G.fast)
                                {
                                    const int bq = mb.base[qq];
                                    T e0 = eb[0];
#pragma unroll
                                    for (int t = 1; t < kMaxBases; ++t)
                                        if (bq == t) e0 = eb[t];
                                    v = powInt<T>(e0, mb.pw[qq]);
                                }
                                else v = fexp<T>(-mb.eta[qq] * (r - mb.rs[qq]) * (r - mb.rs[qq]));
                                acc[q] += v * fc;
                            }
                        }
                    }
                }
                else
                {
                    const bool narrow = (G.type == 3);
                    const bool same = (G.e1 == G.e2);
                    const int A0 = S.blockBegin[G.e1], nA = S.blockBegin[G.e1 + 1] - A0;
                    const int B0 = S.blockBegin[G.e2], nB = S.blockBegin[G.e2 + 1] - B0;
                    for (int a = lane; a < nA; a += 32)
                    {
                        const int sa = A0 + a;
                        const T r1 = S.r[sa];
                        if (!(r1 < rc)) continue;
                        const T x1 = S.x[sa], y1 = S.y[sa], z1 = S.z[sa], ri1 = S.rinv[sa], fc1 = S.fc[sa];
                        T e1b[kMaxStagedBases];
#pragma unroll
                        for (int q = 0; q < kMaxStagedBases; ++q) e1b[q] = G.fast ? S.E[q][sa] : T(0);
                        const int cnt = same ? halfRange(a, nA) : nB;
                        for (int t0 = 0; t0 < cnt; t0 += 32)
                        {
                            const int tm = min(32, cnt - t0);
                            unsigned mask = 0;
                            for (int bb = 0; bb < tm; ++bb)
                            {
                                int p = same ? a + 1 + t0 + bb : t0 + bb;
                                if (same && p >= nA) p -= nA;
                                const int sb = (same ? A0 : B0) + p;
                                bool ok = S.r[sb] < rc;
                                if (ok && narrow)
                                {
                                    const T dx = S.x[sb] - x1, dy = S.y[sb] - y1, dz = S.z[sb] - z1;
                                    ok = (dx * dx + dy * dy + dz * dz) < rc2;
                                }
                                mask |= (ok ? 1u : 0u) << bb;
                            }
                            while (mask)
                            {
                                const int bb = __ffs(mask) - 1;
                                mask &= mask - 1;
                                int p = same ? a + 1 + t0 + bb : t0 + bb;
                                if (same && p >= nA) p -= nA;
                                const int sb = (same ? A0 : B0) + p;
                                const T x2 = S.x[sb], y2 = S.y[sb], z2 = S.z[sb];
                                const T cost = (x1 * x2 + y1 * y2 + z1 * z2) * (ri1 * S.rinv[sb]);
                                T pfc = fc1 * S.fc[sb];
                                T bv[kMaxStagedBases];
                                T rjk = T(0), rjk2 = T(0);
                                if (narrow)
                                {
                                    const T dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
                                    rjk2 = dx * dx + dy * dy + dz * dz;
                                    rjk = rjk2 * frsqrt<T>(rjk2);
                                    double fjk, dfjk;
                                    cutoffFdf(model.cutoff[G.cutoffSlot], (double)rjk, fjk, dfjk);
                                    pfc *= (T)fjk;
                                }
                                if (G.fast)
                                {
#pragma unroll
                                    for (int q = 0; q < kMaxStagedBases; ++q)
                                        bv[q] = (q < G.numBases)
                                                    ? e1b[q] * S.E[q][sb] *
                                                          (narrow ? fexp<T>(-(T)G.baseEta[q] * rjk2) : T(1))
                                                    : T(0);
                                }
                                const T r2 = S.r[sb];
                                T vexp = T(0);
#pragma unroll
                                for (int q = 0; q < kChunkF; ++q)
                                {
                                    if (q < mc)
                                    {
                                        const int qq = m0 + q;
                                        if ((mb.flags[qq] & 2) || q == 0)
                                        {
                                            if (G.fast)
                                                vexp = powInt<T>(mb.base[qq] == 0 ? bv[0] : bv[kMaxStagedBases - 1],
                                                                 mb.pw[qq]);
                                            else
                                            {
                                                const T u = r1 - mb.rs[qq], v2 = r2 - mb.rs[qq], w3 = rjk - mb.rs[qq];
                                                vexp = fexp<T>(-mb.eta[qq] *
                                                               (u * u + v2 * v2 + (narrow ? w3 * w3 : T(0))));
                                            }
                                        }
                                        const T pl = T(1) + mb.lambda[qq] * cost;
                                        if (pl > T(0)) acc[q] += vexp * angularPow<T>(pl, mb, qq) * pl * pfc;
                                    }
                                }
                            }
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < kChunkF; ++q)
                {
                    if (q < mc)
                    {
                        double s = warpSum((double)acc[q]);
                        if (lane == q)
                        {
                            DevMember const& M = mem[m0 + q];
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
// With a_s = dE/dG_s * factorNorm_s * fg_s, the reference's derivative
// prefactors p1, p3 (SymGrpExpAngn.cpp:305-337) contract, for the ordered
// pair (owner j, partner k), to
//   P1 = pfc ((1/(rij rik) - cos/rij^2) T1 - Uij) + pr1 T3
//   P3 = pfc (1/(rij rik) T1 + Ujk) - pr3 T3          (narrow)
//   P3 = pfc /(rij rik) T1                            (wide)
// T1 = sum a zeta lambda, T3 = sum a plambda,
// Uij = sum a zeta lambda plambda factorDeriv (rij - rs)/rij  (Ujk alike).
// The force E_i puts on j gains P1 dr_ij + P3 dr_jk; the self force on i
// loses P1 dr_ij.
template <typename T, int CAP, int WARPS, int LOWER>
__global__ void __launch_bounds__(WARPS * 32) kSFForcesF(DevModel model, BatchView b)
{
    extern __shared__ __align__(16) unsigned char smemRaw[];
    ForcesSmem<T, CAP>& SM = reinterpret_cast<ForcesSmem<T, CAP>*>(smemRaw)[threadIdx.x >> 5];
    Stage<T, CAP>& S = SM.st;
    Members<T>& mb = SM.mb;
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        const int64_t off = b.nbrOffset[i];
        const int64_t end = b.nbrOffset[i + 1];
        if (end > b.nbrCapacity) continue;
        const int n = (int)(end - off);
        if (!(n <= CAP && n > LOWER)) continue;
        const int ec = b.elem[i];
        DevElement const& E = model.el[ec];
        const double* dEdG = b.dEdG + (size_t)i * b.gStride;
        stageGeometry<T, CAP>(S, off, n, model.numElements, b, lane);
        for (int s = lane; s < n; s += 32) SM.h[0][s] = SM.h[1][s] = SM.h[2][s] = 0.0;
        double sfx = 0.0, sfy = 0.0, sfz = 0.0;
        int slot = -1;
        for (int g = 0; g < E.groupCount; ++g)
        {
            DevGroup const G = model.groups[E.groupBegin + g];
            if (G.cutoffSlot != slot)
            {
                stageCutoff<T, CAP>(S, off, n, G.cutoffSlot, b, lane);
                slot = G.cutoffSlot;
            }
            stageMembers<T>(mb, model, G, dEdG, lane);
            const int M = G.memberCount;
            const T rc = (T)G.rc, rc2 = (T)G.rc2;
            if (G.type == 2)
            {
                for (int s = S.blockBegin[G.e1] + lane; s < S.blockBegin[G.e1 + 1]; s += 32)
                {
                    const T r = S.r[s];
                    if (!(r < rc)) continue;
                    const T fc = S.fc[s], dfc = S.dfcr[s] * r, ri = S.rinv[s];
                    T eb[kMaxBases];
#pragma unroll
                    for (int q = 0; q < kMaxBases; ++q)
                        eb[q] = (G.fast && q < G.numBases) ? fexp<T>(-(T)G.baseEta[q] * r * r) : T(0);
                    T P = T(0);
                    for (int q = 0; q < M; ++q)
                    {
                        T v;
                        if (G.fast)
                        {
                            const int bq = mb.base[q];
                            T e0 = eb[0];
#pragma unroll
                            for (int t = 1; t < kMaxBases; ++t)
                                if (bq == t) e0 = eb[t];
                            v = powInt<T>(e0, mb.pw[q]);
                        }
                        else v = fexp<T>(-mb.eta[q] * (r - mb.rs[q]) * (r - mb.rs[q]));
                        P += mb.cw[q] * (dfc - T(2) * mb.eta[q] * (r - mb.rs[q]) * fc) * v * ri;
                    }
                    const double Pd = (double)P;
                    const double ddx = (double)S.x[s] * Pd, ddy = (double)S.y[s] * Pd, ddz = (double)S.z[s] * Pd;
                    SM.h[0][s] += ddx;
                    SM.h[1][s] += ddy;
                    SM.h[2][s] += ddz;
                    sfx -= ddx;
                    sfy -= ddy;
                    sfz -= ddz;
                }
                continue;
            }
            if (G.fast) stageFactors<T, CAP>(S, G, lane);
            const bool narrow = (G.type == 3);
            const bool same = (G.e1 == G.e2);
            for (int sweep = 0; sweep < (same ? 1 : 2); ++sweep)
            {
                const int eo = sweep == 0 ? G.e1 : G.e2;   // owners
                const int ep = sweep == 0 ? G.e2 : G.e1;   // partners
                const int O0 = S.blockBegin[eo], nO = S.blockBegin[eo + 1] - O0;
                const int P0 = S.blockBegin[ep], nP = S.blockBegin[ep + 1] - P0;
                for (int a = lane; a < nO; a += 32)
                {
                    const int sa = O0 + a;
                    const T r1 = S.r[sa];
                    if (!(r1 < rc)) continue;
                    const T x1 = S.x[sa], y1 = S.y[sa], z1 = S.z[sa], ri1 = S.rinv[sa], fc1 = S.fc[sa];
                    const T dfcr1 = S.dfcr[sa];
                    T e1b[kMaxStagedBases];
#pragma unroll
                    for (int q = 0; q < kMaxStagedBases; ++q) e1b[q] = G.fast ? S.E[q][sa] : T(0);
                    T ax = T(0), ay = T(0), az = T(0), px = T(0), py = T(0), pz = T(0);
                    const int cnt = same ? nO - 1 : nP;
                    for (int t0 = 0; t0 < cnt; t0 += 32)
                    {
                        const int tm = min(32, cnt - t0);
                        unsigned mask = 0;
                        for (int bb = 0; bb < tm; ++bb)
                        {
                            int p = same ? a + 1 + t0 + bb : t0 + bb;
                            if (same && p >= nO) p -= nO;
                            const int sb = P0 + p;
                            bool ok = S.r[sb] < rc;
                            if (ok && narrow)
                            {
                                const T dx = S.x[sb] - x1, dy = S.y[sb] - y1, dz = S.z[sb] - z1;
                                ok = (dx * dx + dy * dy + dz * dz) < rc2;
                            }
                            mask |= (ok ? 1u : 0u) << bb;
                        }
                        while (mask)
                        {
                            const int bb = __ffs(mask) - 1;
                            mask &= mask - 1;
                            int p = same ? a + 1 + t0 + bb : t0 + bb;
                            if (same && p >= nO) p -= nO;
                            const int sb = P0 + p;
                            const T x2 = S.x[sb], y2 = S.y[sb], z2 = S.z[sb];
                            const T ri2 = S.rinv[sb], fc2 = S.fc[sb];
                            const T dx3 = x2 - x1, dy3 = y2 - y1, dz3 = z2 - z1;
                            const T rinv = ri1 * ri2;
                            const T cost = (x1 * x2 + y1 * y2 + z1 * z2) * rinv;
                            T pfc, pr1, pr3 = T(0), rjk = T(0), rijk = T(0), rjk2 = T(0);
                            if (narrow)
                            {
                                rjk2 = dx3 * dx3 + dy3 * dy3 + dz3 * dz3;
                                rijk = frsqrt<T>(rjk2);
                                rjk = rjk2 * rijk;
                                double fjk, dfjk;
                                cutoffFdf(model.cutoff[G.cutoffSlot], (double)rjk, fjk, dfjk);
                                const T fcjk = (T)fjk, dfcjk = (T)dfjk;
                                pfc = fc1 * fc2 * fcjk;
                                pr1 = fc2 * fcjk * dfcr1;
                                pr3 = fc1 * fc2 * dfcjk * rijk;
                            }
                            else
                            {
                                pfc = fc1 * fc2;
                                pr1 = fc2 * dfcr1;
                            }
                            T bv[kMaxStagedBases];
                            if (G.fast)
                            {
#pragma unroll
                                for (int q = 0; q < kMaxStagedBases; ++q)
                                    bv[q] = (q < G.numBases)
                                                ? e1b[q] * S.E[q][sb] * (narrow ? fexp<T>(-(T)G.baseEta[q] * rjk2) : T(1))
                                                : T(0);
                            }
                            const T r2 = S.r[sb];
                            T T1 = T(0), T3 = T(0), Uij = T(0), Ujk = T(0), vexp = T(0);
                            for (int q = 0; q < M; ++q)
                            {
                                if ((mb.flags[q] & 2) || q == 0)
                                {
                                    if (G.fast)
                                        vexp = powInt<T>(mb.base[q] == 0 ? bv[0] : bv[kMaxStagedBases - 1], mb.pw[q]);
                                    else
                                    {
                                        const T u = r1 - mb.rs[q], v2 = r2 - mb.rs[q], w3 = rjk - mb.rs[q];
                                        vexp = fexp<T>(-mb.eta[q] * (u * u + v2 * v2 + (narrow ? w3 * w3 : T(0))));
                                    }
                                }
                                const T pl = T(1) + mb.lambda[q] * cost;
                                if (!(pl > T(0))) continue;
                                const T a = mb.cw[q] * vexp * angularPow<T>(pl, mb, q);
                                const T azl = a * mb.zl[q];
                                const T azq = azl * pl * mb.fd[q];
                                T1 += azl;
                                T3 += a * pl;
                                if (mb.rs[q] > T(0))
                                {
                                    Uij += azq * (r1 - mb.rs[q]) * ri1;
                                    if (narrow) Ujk += azq * (rjk - mb.rs[q]) * rijk;
                                }
                                else
                                {
                                    Uij += azq;
                                    Ujk += azq;
                                }
                            }
                            const T P1 = pfc * ((rinv - cost * ri1 * ri1) * T1 - Uij) + pr1 * T3;
                            const T P3 = narrow ? (pfc * (rinv * T1 + Ujk) - pr3 * T3) : (pfc * rinv * T1);
                            ax += P1 * x1 + P3 * dx3;
                            ay += P1 * y1 + P3 * dy3;
                            az += P1 * z1 + P3 * dz3;
                            px += P1 * x1;
                            py += P1 * y1;
                            pz += P1 * z1;
                        }
                    }
                    SM.h[0][sa] += (double)ax;
                    SM.h[1][sa] += (double)ay;
                    SM.h[2][sa] += (double)az;
                    sfx -= (double)px;
                    sfy -= (double)py;
                    sfz -= (double)pz;
                }
                __syncwarp();
            }
        }
        __syncwarp();
        for (int s = lane; s < n; s += 32)
        {
            const int64_t e = off + S.perm[s];
            b.hx[e] = SM.h[0][s];
            b.hy[e] = SM.h[1][s];
            b.hz[e] = SM.h[2][s];
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
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------
namespace {

constexpr int kStdCapF = 160, kStdWarpsF = 4;
constexpr int kBigCapF = 1024, kBigWarpsF = 1;

int gridFor(int N, int warpsPerBlock, int sms, int perSM)
{
    int need = (N + warpsPerBlock - 1) / warpsPerBlock;
    int cap = sms * perSM;
    return need < cap ? (need > 0 ? need : 1) : cap;
}

template <typename T>
void valuesT(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    const size_t s1 = sizeof(ValuesSmem<T, kStdCapF>) * kStdWarpsF;
    const size_t s2 = sizeof(ValuesSmem<T, kBigCapF>) * kBigWarpsF;
    auto k1 = kSFValuesF<T, kStdCapF, kStdWarpsF, -1>;
    auto k2 = kSFValuesF<T, kBigCapF, kBigWarpsF, kStdCapF>;
    setDynamicSmemOnce(reinterpret_cast<const void*>(k1), s1);
    setDynamicSmemOnce(reinterpret_cast<const void*>(k2), s2);
    k1<<<gridFor(b.N, kStdWarpsF, sms, 32), kStdWarpsF * 32, s1, st>>>(m, b);
    k2<<<sms, kBigWarpsF * 32, s2, st>>>(m, b);
}

template <typename T>
void forcesT(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    const size_t s1 = sizeof(ForcesSmem<T, kStdCapF>) * kStdWarpsF;
    const size_t s2 = sizeof(ForcesSmem<T, kBigCapF>) * kBigWarpsF;
    auto k1 = kSFForcesF<T, kStdCapF, kStdWarpsF, -1>;
    auto k2 = kSFForcesF<T, kBigCapF, kBigWarpsF, kStdCapF>;
    setDynamicSmemOnce(reinterpret_cast<const void*>(k1), s1);
    setDynamicSmemOnce(reinterpret_cast<const void*>(k2), s2);
    k1<<<gridFor(b.N, kStdWarpsF, sms, 32), kStdWarpsF * 32, s1, st>>>(m, b);
    k2<<<sms, kBigWarpsF * 32, s2, st>>>(m, b);
}

} // namespace

void launchSFValues(DevModel const& m, BatchView const& b, int precision, int sms, cudaStream_t st)
{
    if (precision == 0) valuesT<double>(m, b, sms, st);
    else valuesT<float>(m, b, sms, st);
}

void launchSFForces(DevModel const& m, BatchView const& b, int precision, int sms, cudaStream_t st)
{
    if (precision == 0) forcesT<double>(m, b, sms, st);
    else forcesT<float>(m, b, sms, st);
}

} // namespace n2p2b200
