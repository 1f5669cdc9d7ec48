// Symmetry-function kernels of the evaluation path (G values and the adjoint
// force pass), one warp per centre atom; included by one translation unit per
// precision (k_sf_fast_f64.cu, k_sf_fast_f32.cu).
//
// Formulas: SymGrpExpRad::calculate (SymGrpExpRad.cpp:144-239),
// SymGrpExpAngn::calculate (SymGrpExpAngn.cpp:156-403),
// SymGrpExpAngw::calculate (SymGrpExpAngw.cpp:156-376).
//
// Layout and schedule:
//  * The atom's neighbours are staged in shared memory sorted by element
//    (stable), so the partners of a group form contiguous blocks and no
//    element test is left in the triplet loops.  Per neighbour the stage holds
//    dr, r, 1/r, f_c, (df_c/r in the force pass) and, per group, the Gaussian
//    factors exp(-eta_b r^2) of the group's bases.
//  * Gaussians: exp(-eta (rij^2 + rik^2 + rjk^2)) = E_b(rij) E_b(rik) exp(-eta_b rjk^2)
//    raised to an integer power when eta = k eta_b (plan built on the host),
//    so a triplet costs one exponential per base instead of one per eta.
//  * Work split: each group's candidate (j, k) pairs are tested 64 at a time
//    and the accepted ones appended to a ring queue in shared memory, which
//    is consumed 32 triplets at a time, so lanes idle only in a group's last
//    partial batch.  The G pass enumerates owner-major; the force pass
//    evaluates each unordered pair once, enumerated in rounds of matchings,
//    and adds a round's contributions to distinct slots (no atomics).
//  * Tiers: an atom with n neighbours runs in the first kernel instance whose
//    stage holds n (tier bounds are launch arguments); the last tier flags
//    atoms beyond its stage.
//  * All sums run in a fixed order: results are bitwise reproducible.
#pragma once

#include "kernels_common.cuh"
#include "kernels.hpp"
#include "pair_rounds.cuh"

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

// 16-byte aligned: stageGeometry reuses the first arrays as FP64 scratch in
// the FP32 form, and every warp's block of the dynamic shared memory starts
// at a multiple of the struct's size.
template <typename T, int CAP, bool DF, int NB>
struct alignas(16) Stage
{
    T x[CAP], y[CAP], z[CAP], r[CAP], rinv[CAP], fc[CAP];
    T dfcr[DF ? CAP : 1];                  // (df_c/dr)/r, force pass only
    T E[NB][CAP];                          // Gaussian factors of the group's staged bases
    short perm[CAP];                       // staged slot -> position in the atom's list
    int blockBegin[kDevMaxElements + 1];
    int nBelow[4][kDevMaxElements];        // per cutoff slot and element: block entries with r < r_c
};

// Group gi of the model: the specialised kernels (FAST) read it from the
// group table argument (warp-uniform constant-bank loads), the generic ones
// copy it from the model's device array.
template <int FAST>
__device__ __forceinline__ DevGroup const& groupOf(DevGroupTable const& gt, DevModel const& model, int gi, DevGroup& scratch)
{
    if constexpr (FAST != 0) return gt.g[gi];
    else
    {
        scratch = model.groups[gi];
        return scratch;
    }
}

// A group's base widths and lambda values in the pass's precision (the
// FP32 copies are the FP64 values rounded once on the host).
template <typename T>
__device__ __forceinline__ T groupBaseEta(DevGroup const& G, int q)
{
    if constexpr (sizeof(T) == 4) return G.baseEtaF[q];
    else return G.baseEta[q];
}

template <typename T>
__device__ __forceinline__ T groupLambda(DevGroup const& G, int ls)
{
    if constexpr (sizeof(T) == 4) return G.lambdaValF[ls];
    else return G.lambdaVal[ls];
}

// Force-pass coefficients of one member-grid combination (eta, lambda,
// zeta): with w = dE/dG * factorNorm, c[0] = w zeta lambda, c[1] = w zeta
// lambda factorDeriv, c[2] = w (all 0 for an absent combination); one
// 16-byte aligned record read with vector loads.
template <typename T>
struct alignas(16) GridCoef
{
    T c[4];
};

// Per-group member parameters (shared by all lanes).
// COMPACT (model-specialised kernels): only what planned radial groups and
// member grids read.
// GPASS (model-specialised G pass): only the radial plan (base, pw); the
// arrays of the force pass and of unplanned members shrink to one entry, so
// the stage of a warp stays small enough for six blocks of four warps.
template <typename T, bool COMPACT, bool GPASS = false>
struct Members
{
    static constexpr bool kLean = COMPACT && GPASS;
    static constexpr int kM = kMaxMembers, kC = COMPACT ? 1 : kMaxMembers, kF = kLean ? 1 : kMaxMembers;
    T cw[kF];                // force pass: dE/dG * factorNorm
    T eta[kF], rs[kF];
    int base[kM], pw[kM];
    T zl[kC], fd[kC], lambda[kC], zeta[kC];
    int zint[kC], flags[kC];  // flags: 1 intPow, 2 calcExp
    GridCoef<T> gc[kLean ? 1 : 16];   // member grid: force-pass coefficients per (eta, lambda, zeta) combination
};

constexpr int kQueue = 128;  // ring of accepted (owner, partner) pairs waiting for a full warp (< 32 + 64)

template <typename T, int CAP, int FAST>
struct ValuesSmem
{
    Stage<T, CAP, false, FAST ? 1 : kMaxStagedBases> st;
    Members<T, FAST != 0, true> mb;
    int queue[kQueue];
};

// h: per staged neighbour, the force the centre's energy puts on it, summed
// over the atom's triplets in the pass's precision (FP32 in the mixed form,
// whose final per-atom accumulation, kGatherForces, is FP64).
template <typename T, int CAP, int FAST>
struct ForcesSmem
{
    Stage<T, CAP, true, FAST ? 1 : kMaxStagedBases> st;
    Members<T, FAST != 0> mb;
    T h[3][CAP];
    int queue[kQueue];
};

// Queue entries: round << 20 | owner slot << 10 | partner slot (slots < 1024).
__device__ __forceinline__ int entryOwner(int e) { return (e >> 10) & 1023; }
__device__ __forceinline__ int entryPartner(int e) { return e & 1023; }
__device__ __forceinline__ int entryRound(int e) { return e >> 20; }

// Test the next 64 candidates of a phase (two independent halves for
// latency hiding) and append the accepted ones, in candidate order, to the
// warp's ring queue (qn entries from q[qh]).
template <typename T, int CAP, bool DF, int NB>
__device__ __forceinline__ bool testCandidate(Stage<T, CAP, DF, NB> const& S, Phase const& ph, Cursor const& cur, int p,
                                              T rc, T rc2, bool narrow, int& entry)
{
    int so = 0, sp = 0;
    bool ok = false;
    // Both slots are inside the group's cutoff by construction: with the
    // stage sorted by distance the enumerated neighbours are the prefix with
    // r < r_c, otherwise every group's cutoff is the list's and an entry at
    // r = r_c exactly has f_c = df_c = 0, i.e. contributes exact zeros.
    if (p < ph.count && cur.slots(ph, so, sp))
    {
        ok = true;
        if (narrow)
        {
            const T dx = S.x[sp] - S.x[so], dy = S.y[sp] - S.y[so], dz = S.z[sp] - S.z[so];
            ok = (dx * dx + dy * dy + dz * dz) < rc2;
        }
    }
    entry = (cur.round(ph) << 20) | (so << 10) | sp;
    return ok;
}

template <typename T, int CAP, bool DF, int NB>
__device__ __forceinline__ void enqueueCandidates(Stage<T, CAP, DF, NB> const& S, Phase const& ph, Cursor& cur, int p0,
                                                  T rc, T rc2, bool narrow, int* queue, int qh, int& qn, int lane,
                                                  uint32_t* maskOut, const uint32_t* maskIn, int& mwi)
{
    Cursor c2 = cur;
    c2.advance(ph);
    int e1, e2;
    unsigned m1, m2;
    if (maskIn)
    {
        // acceptance recorded by the G pass for these 64 candidates
        m1 = __ldg(maskIn + mwi);
        m2 = __ldg(maskIn + mwi + 1);
        int so, sp;
        cur.slots(ph, so, sp);
        e1 = (cur.round(ph) << 20) | (so << 10) | sp;
        c2.slots(ph, so, sp);
        e2 = (c2.round(ph) << 20) | (so << 10) | sp;
    }
    else
    {
        const bool ok1 = testCandidate<T, CAP>(S, ph, cur, p0 + lane, rc, rc2, narrow, e1);
        const bool ok2 = testCandidate<T, CAP>(S, ph, c2, p0 + 32 + lane, rc, rc2, narrow, e2);
        m1 = __ballot_sync(kFullMask, ok1);
        m2 = __ballot_sync(kFullMask, ok2);
        if (maskOut && lane == 0)
        {
            maskOut[mwi] = m1;
            maskOut[mwi + 1] = m2;
        }
    }
    mwi += 2;
    const bool ok1 = (m1 >> lane) & 1u, ok2 = (m2 >> lane) & 1u;
    const unsigned below = (1u << lane) - 1u;
    if (ok1) queue[(qh + qn + __popc(m1 & below)) & (kQueue - 1)] = e1;
    if (ok2) queue[(qh + qn + __popc(m1) + __popc(m2 & below)) & (kQueue - 1)] = e2;
    qn += __popc(m1) + __popc(m2);
    cur = c2;
    cur.advance(ph);
    __syncwarp();
}

// Neighbours of one atom into the stage, sorted by element (stable) and, when
// the model has angular groups with a smaller cutoff than the list's, by
// distance within each element block, so that the neighbours inside a
// group's cutoff are a prefix of the block (nBelow).
template <typename T, int CAP, bool DF, int NB>
__device__ void stageGeometry(Stage<T, CAP, DF, NB>& S, int64_t off, int n, DevModel const& model, BatchView const& b,
                              int lane)
{
    const int numElements = model.numElements;
    __syncwarp();
    // neighbour elements of this lane's entries, all loads issued together
    constexpr int kChunks = (CAP + 31) / 32;
    int elemOf[kChunks];
#pragma unroll
    for (int c = 0; c < kChunks; ++c)
    {
        const int m = c * 32 + lane;
        elemOf[c] = m < n ? (int)b.nbrElem[off + m] : -1;
    }
    int base = 0;
    for (int e = 0; e < numElements; ++e)
    {
        if (lane == 0) S.blockBegin[e] = base;
#pragma unroll
        for (int c = 0; c < kChunks; ++c)
        {
            if (c * 32 >= n) break;
            const bool mine = elemOf[c] == e;
            const unsigned bal = __ballot_sync(kFullMask, mine);
            if (mine) S.perm[base + __popc(bal & ((1u << lane) - 1u))] = (short)(c * 32 + lane);
            base += __popc(bal);
        }
    }
    if (lane == 0) S.blockBegin[numElements] = base;
    __syncwarp();
    if (model.sortByDistance)
    {
        // FP64 distances and a scratch permutation in arrays filled below
        double* rd = sizeof(T) == 8 ? reinterpret_cast<double*>(S.r) : reinterpret_cast<double*>(S.x);
        short* tmp = sizeof(T) == 8 ? reinterpret_cast<short*>(S.x) : reinterpret_cast<short*>(S.z);
        for (int s = lane; s < n; s += 32) rd[s] = b.nbrD[off + S.perm[s]];
        __syncwarp();
        for (int s = lane; s < n; s += 32)
        {
            int e = 0;
            while (s >= S.blockBegin[e + 1]) ++e;
            const int b0 = S.blockBegin[e], b1 = S.blockBegin[e + 1];
            const double rs = rd[s];
            int rank = b0;
            for (int t = b0; t < b1; ++t)
            {
                const double rt = rd[t];
                rank += (rt < rs || (rt == rs && t < s)) ? 1 : 0;
            }
            tmp[rank] = S.perm[s];
        }
        __syncwarp();
        for (int c = 0; c < model.numCutoffSlots; ++c)
            for (int e = 0; e < numElements; ++e)
            {
                int cnt = 0;
                for (int s = S.blockBegin[e] + lane; s < S.blockBegin[e + 1]; s += 32)
                    cnt += rd[s] < model.cutoff[c].rc ? 1 : 0;
                cnt = warpSumInt(cnt);
                if (lane == 0) S.nBelow[c][e] = cnt;
            }
        __syncwarp();
        for (int s = lane; s < n; s += 32) S.perm[s] = tmp[s];
    }
    else if (lane < kDevMaxElements)
    {
        for (int c = 0; c < 4; ++c) S.nBelow[c][lane] = lane < numElements ? S.blockBegin[lane + 1] - S.blockBegin[lane] : 0;
    }
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
template <typename T, int CAP, bool DF, int NB>
__device__ void stageCutoff(Stage<T, CAP, DF, NB>& S, int64_t off, int n, int slot, BatchView const& b, int lane)
{
    __syncwarp();
    const double* fc = b.nbrFc + (size_t)slot * b.nbrCapacity + off;
    const double* dfc = b.nbrDfc + (size_t)slot * b.nbrCapacity + off;
    for (int s = lane; s < n; s += 32)
    {
        const int m = S.perm[s];
        S.fc[s] = (T)fc[m];
        if constexpr (DF) S.dfcr[s] = (T)(dfc[m] / b.nbrD[off + m]);
    }
    __syncwarp();
}

// Gaussian factors exp(-eta_b r^2) of the group's staged bases for the slots
// of the group's element blocks.
template <typename T, int CAP, bool DF, int NB>
__device__ void stageFactors(Stage<T, CAP, DF, NB>& S, DevGroup const& G, int lane)
{
    __syncwarp();
    for (int pass = 0; pass < 2; ++pass)
    {
        const int e = pass == 0 ? G.e1 : G.e2;
        if (pass == 1 && G.e2 == G.e1) break;
        for (int s = S.blockBegin[e] + lane; s < S.blockBegin[e + 1]; s += 32)
        {
            const T r = S.r[s];
            for (int q = 0; q < G.numBases && q < NB; ++q) S.E[q][s] = fexp<T>(-groupBaseEta<T>(G, q) * r * r);
        }
    }
    __syncwarp();
}

template <typename T, bool COMPACT, bool GPASS>
__device__ void stageMembers(Members<T, COMPACT, GPASS>& mb, DevModel const& model, DevGroup const& G, const double* dEdG,
                             int lane)
{
    constexpr bool lean = Members<T, COMPACT, GPASS>::kLean;
    __syncwarp();
    for (int q = lane; q < G.memberCount; q += 32)
    {
        DevMember const& M = model.members[G.memberBegin + q];
        if constexpr (!lean)
        {
            mb.cw[q] = dEdG ? (T)(dEdG[M.sf] * M.factorNorm) : T(0);
            mb.eta[q] = (T)M.eta;
            mb.rs[q] = (T)M.rs;
        }
        mb.base[q] = M.expBase;
        mb.pw[q] = M.expPow;
        if constexpr (!COMPACT)
        {
            mb.zl[q] = (T)M.zetaLambda;
            mb.fd[q] = (T)M.factorDeriv;
            mb.lambda[q] = (T)M.lambda;
            mb.zeta[q] = (T)M.zeta;
            mb.zint[q] = M.zetaInt;
            mb.flags[q] = (M.useIntPow ? 1 : 0) | (M.calcExp ? 2 : 0);
        }
    }
    if constexpr (!lean)
    {
        if (G.grid && dEdG && lane < 16)
        {
            const int q = G.comboMember[lane];
            GridCoef<T> cf{};
            if (q >= 0)
            {
                DevMember const& M = model.members[G.memberBegin + q];
                const double w = dEdG[M.sf] * M.factorNorm;
                cf.c[0] = (T)(w * M.zetaLambda);
                cf.c[1] = (T)(w * M.zetaLambda * M.factorDeriv);
                cf.c[2] = (T)w;
            }
            mb.gc[lane] = cf;
        }
    }
    __syncwarp();
}

// Rare paths kept out of line so the hot loops stay small: real-valued zeta
// and Gaussians with a shift r_s (which cannot use the factorised bases).
template <typename T>
__device__ __noinline__ T powReal(T b, T e)
{
    return fpow<T>(b, e);
}

template <typename T>
__device__ __noinline__ T gaussShifted(T eta, T rs, T r1, T r2, T r3, int narrow)
{
    const T u = r1 - rs, v = r2 - rs, w = r3 - rs;
    return fexp<T>(-eta * (u * u + v * v + (narrow ? w * w : T(0))));
}

template <typename T, bool COMPACT, bool GPASS>
__device__ __forceinline__ T angularPow(T pl, Members<T, COMPACT, GPASS> const& mb, int q)
{
    return (mb.flags[q] & 1) ? powInt<T>(pl, mb.zint[q] - 1) : powReal<T>(pl, mb.zeta[q] - T(1));
}

// Geometry of one triplet (owner j = slot so, partner k = slot sp).
template <typename T>
struct Triplet
{
    T x1, y1, z1, r1, ri1, fc1, dfcr1;
    T x2, y2, z2, r2, ri2, fc2;
    T dx3, dy3, dz3, rjk, rijk, rjk2;
    T rinv, cost, fcjk, dfcjk;
};

// Slot geometry of a triplet (everything but the j-k cutoff).
template <typename T, int CAP, bool DF, int NB>
__device__ __forceinline__ void tripletGeometry(Stage<T, CAP, DF, NB> const& S, int so, int sp, Triplet<T>& t)
{
    t.x1 = S.x[so];
    t.y1 = S.y[so];
    t.z1 = S.z[so];
    t.r1 = S.r[so];
    t.ri1 = S.rinv[so];
    t.fc1 = S.fc[so];
    if constexpr (DF) t.dfcr1 = S.dfcr[so];
    else t.dfcr1 = T(0);
    t.x2 = S.x[sp];
    t.y2 = S.y[sp];
    t.z2 = S.z[sp];
    t.r2 = S.r[sp];
    t.ri2 = S.rinv[sp];
    t.fc2 = S.fc[sp];
    t.dx3 = t.x2 - t.x1;
    t.dy3 = t.y2 - t.y1;
    t.dz3 = t.z2 - t.z1;
    t.rinv = t.ri1 * t.ri2;
    t.cost = (t.x1 * t.x2 + t.y1 * t.y2 + t.z1 * t.z2) * t.rinv;
    t.rjk2 = t.dx3 * t.dx3 + t.dy3 * t.dy3 + t.dz3 * t.dz3;
    t.rjk = T(0);
    t.rijk = T(0);
    t.fcjk = T(1);
    t.dfcjk = T(0);
}

// Cutoff types with a kernel instance of their own (CUT template argument);
// every other type runs the instance with the run-time dispatch.
constexpr int kCutAny = 0, kCutPoly2 = 6;

// The poly2 instances of the model-specialised kernels also take the integer
// powers of their member grids as compile-time bounded: at most 2 binary
// digits with two zeta slots (zeta <= 4, eta multiples <= 3), 4 with four
// slots (zeta <= 16, multiples <= 15).  Models beyond that run the kCutAny
// instances (run-time bounds).
template <int FAST, int CUT>
__host__ __device__ constexpr int sfPowBits()
{
    return CUT == kCutPoly2 ? (FAST == 2 ? 2 : 4) : 0;
}

// r_jk and its cutoff (narrow groups): FP64 in the FP64 form; in the FP32
// form the cancellation-free factored polynomials (cutoffFdfF32).
template <typename T, int CUT = kCutAny>
__device__ __forceinline__ void tripletJK(DevCutoff const& cut, Triplet<T>& t)
{
    t.rijk = frsqrt<T>(t.rjk2);
    t.rjk = t.rjk2 * t.rijk;
    if constexpr (CUT == kCutPoly2) cutoffPoly2(cut, t.rjk, t.fcjk, t.dfcjk);
    else if constexpr (sizeof(T) == 4) cutoffFdfF32(cut, t.rjk, t.fcjk, t.dfcjk);
    else cutoffFdf(cut, t.rjk, t.fcjk, t.dfcjk);
}

template <typename T, int CAP, bool DF, int NB>
__device__ __forceinline__ void loadTriplet(Stage<T, CAP, DF, NB> const& S, DevCutoff const& cut, bool narrow, int so, int sp,
                                            Triplet<T>& t)
{
    tripletGeometry<T, CAP>(S, so, sp, t);
    if (narrow) tripletJK<T>(cut, t);
}

// ILP triplets per lane at once (model-specialised kernels): entries
// lane + 32 u, u < ILP, of the queue window [qh, qh + take); a lane past
// the window repeats the window's first entry (in bounds, finite) and its
// ok[u] is false.  Each step is written for all u together so independent
// chains could interleave; the kernels run ILP = 1: two triplets per lane
// measured 1.5x slower on B200 (the extra live registers cut residency
// from 16 to 12 warps per SM and spilled in the force pass).
template <int CUT, typename T, int CAP, bool DF, int NB, int ILP>
__device__ __forceinline__ void loadTriplets(Stage<T, CAP, DF, NB> const& S, DevCutoff const& cut, bool narrow,
                                             const int* queue, int qh, int take, int lane, Triplet<T> (&t)[ILP],
                                             int (&so)[ILP], int (&sp)[ILP], bool (&ok)[ILP])
{
#pragma unroll
    for (int u = 0; u < ILP; ++u)
    {
        const int idx = lane + 32 * u;
        ok[u] = idx < take;
        const int e = queue[(qh + (ok[u] ? idx : 0)) & (kQueue - 1)];
        so[u] = entryOwner(e);
        sp[u] = entryPartner(e);
        tripletGeometry<T, CAP>(S, so[u], sp[u], t[u]);
    }
    if (narrow)
    {
#pragma unroll
        for (int u = 0; u < ILP; ++u) tripletJK<T, CUT>(cut, t[u]);
    }
}

// Gaussian bases of a triplet: E_b(rij) E_b(rik) exp(-eta_b rjk^2)
// (bv has kMaxStagedBases entries; bases beyond the stage's NB are 0).
template <typename T, int CAP, bool DF, int NB>
__device__ __forceinline__ void tripletBases(Stage<T, CAP, DF, NB> const& S, DevGroup const& G, bool narrow, int so, int sp,
                                             T rjk2, T* bv)
{
#pragma unroll
    for (int q = 0; q < kMaxStagedBases; ++q)
    {
        if (q < NB)
            bv[q] = (q < G.numBases) ? S.E[q][so] * S.E[q][sp] * (narrow ? fexp<T>(-groupBaseEta<T>(G, q) * rjk2) : T(1))
                                     : T(0);
        else
            bv[q] = T(0);
    }
}

// x^e for a warp-uniform 0 <= e < 32, in pow_int's multiplication order
// (result = 1, times x^(2^k) for each set bit k in increasing k;
// utility.cpp:292-316).  FP64: square-and-multiply over the set bits only
// (uniform branches, no lane diverges); FP32: a branch-free ladder over all
// five bits, cheaper where multiplies cost less than branches.
template <typename T>
__device__ __forceinline__ T powUniform(T x, int e)
{
    if constexpr (sizeof(T) == 8)
    {
        T r = T(1);
#pragma unroll 1
        while (e)
        {
            if (e & 1) r *= x;
            e >>= 1;
            if (e) x *= x;
        }
        return r;
    }
    else
    {
        const T p2 = x * x, p4 = p2 * p2, p8 = p4 * p4, p16 = p8 * p8;
        T r = (e & 1) ? x : T(1);
        r = (e & 2) ? r * p2 : r;
        r = (e & 4) ? r * p4 : r;
        r = (e & 8) ? r * p8 : r;
        r = (e & 16) ? r * p16 : r;
        return r;
    }
}

// The squares x^(2^k), k < bits, that pow_int forms (p[0] = x,
// p[k] = p[k-1]^2; utility.cpp:292-316), shared by the exponents of one
// base.  BITS > 0: a compile-time bound on the binary digits of every
// exponent (exactly BITS - 1 squarings); BITS = 0: the warp-uniform run-time
// `bits` (<= 5; FP32 then forms every square, FP64 selects).
template <typename T, int BITS>
__device__ __forceinline__ void powSquares(T x, int bits, T (&p)[5])
{
    p[0] = x;
#pragma unroll
    for (int k = 1; k < 5; ++k)
    {
        if constexpr (BITS > 0)
        {
            if (k < BITS) p[k] = p[k - 1] * p[k - 1];
        }
        else if constexpr (sizeof(T) == 4) p[k] = p[k - 1] * p[k - 1];
        else p[k] = (k < bits) ? p[k - 1] * p[k - 1] : T(1);
    }
}

// x^e from its squares in pow_int's multiplication order (1 times the
// square of each set bit of e, in increasing bit order), e < 2^bits and
// warp-uniform: the same rounding as powUniform with the squares formed once.
template <typename T, int BITS>
__device__ __forceinline__ T powFromSquares(T const (&p)[5], int e, int bits)
{
    T r = (e & 1) ? p[0] : T(1);
#pragma unroll
    for (int k = 1; k < 5; ++k)
    {
        if constexpr (BITS > 0)
        {
            if (k < BITS && ((e >> k) & 1)) r *= p[k];
        }
        else if constexpr (sizeof(T) == 4) r = ((e >> k) & 1) ? r * p[k] : r;
        else if (k < bits && ((e >> k) & 1)) r *= p[k];
    }
    return r;
}

// The two eta slots' Gaussians of a triplet, E_slot = base^etaPow (one
// set of squares when both slots use the same staged base).
template <typename T, int BITS>
__device__ __forceinline__ void gridEtas(T const* bv, DevGroup const& G, T (&vS)[2])
{
    T p[5];
    powSquares<T, BITS>(G.etaBase[0] == 0 ? bv[0] : bv[1], G.etaBits, p);
    vS[0] = powFromSquares<T, BITS>(p, G.etaPow[0], G.etaBits);
    if (G.etaBase[1] != G.etaBase[0]) powSquares<T, BITS>(G.etaBase[1] == 0 ? bv[0] : bv[1], G.etaBits, p);
    vS[1] = powFromSquares<T, BITS>(p, G.etaPow[1], G.etaBits);
}

// Member grid, G pass: acc[(eta * 2 + lambda) * STRIDE + zeta] += E_eta * pl^zeta * pfc
// (pl = 1 + lambda cos; terms with pl <= 0 vanish, SymGrpExpAngn.cpp:295).
template <typename T, int NZ, int STRIDE, int BITS = 0>
__device__ __forceinline__ void gridValues(T const* bv, DevGroup const& G, T cost, T pfc, T* acc)
{
    T vS[2];
    gridEtas<T, BITS>(bv, G, vS);
#pragma unroll
    for (int ls = 0; ls < 2; ++ls)
    {
        const T pl = T(1) + groupLambda<T>(G, ls) * cost;
        const T w = pl > T(0) ? pl * pfc : T(0);
        T q[5];
        if constexpr (NZ <= 2) powSquares<T, BITS>(pl, G.zetaBits, q);
#pragma unroll
        for (int zs = 0; zs < NZ; ++zs)
        {
            // four zeta slots: the squares per slot (fewer live registers)
            const T pz =
                (NZ <= 2 ? powFromSquares<T, BITS>(q, G.zetaM1[zs], G.zetaBits) : powUniform<T>(pl, G.zetaM1[zs])) * w;
#pragma unroll
            for (int es = 0; es < 2; ++es) acc[(es * 2 + ls) * STRIDE + zs] += vS[es] * pz;
        }
    }
}

// Member grid, force pass: the dE/dG-weighted member sums of one triplet,
// accumulated onto T1, T2, T3: with a = E_eta pl^(zeta - 1) per combination,
// T1 = sum c[0] a, T2 = Uij = Uik = Ujk (rs = 0) = pl sum c[1] a and
// T3 = pl sum c[2] a (terms with pl <= 0 vanish).
template <typename T, int NZ, bool COMPACT, int BITS = 0>
__device__ __forceinline__ void gridForces(T const* bv, DevGroup const& G, Members<T, COMPACT> const& mb, T cost, T& T1, T& T2,
                                           T& T3)
{
    T vS[2];
    gridEtas<T, BITS>(bv, G, vS);
#pragma unroll
    for (int ls = 0; ls < 2; ++ls)
    {
        const T pl = T(1) + groupLambda<T>(G, ls) * cost;
        const bool valid = pl > T(0);
        T q[5];
        if constexpr (NZ <= 2) powSquares<T, BITS>(pl, G.zetaBits, q);
        T S1 = T(0), S2 = T(0), S3 = T(0);
#pragma unroll
        for (int zs = 0; zs < NZ; ++zs)
        {
            const T pz1 =
                valid ? (NZ <= 2 ? powFromSquares<T, BITS>(q, G.zetaM1[zs], G.zetaBits) : powUniform<T>(pl, G.zetaM1[zs]))
                      : T(0);
#pragma unroll
            for (int es = 0; es < 2; ++es)
            {
                const GridCoef<T> cf = mb.gc[(es * 2 + ls) * 4 + zs];
                const T a = vS[es] * pz1;
                S1 += cf.c[0] * a;
                S2 += cf.c[1] * a;
                S3 += cf.c[2] * a;
            }
        }
        T1 += S1;
        T2 += S2 * pl;
        T3 += S3 * pl;
    }
}

// gridValues of U triplets (pfc = 0 for a triplet that is not to count:
// it then adds zeros).
template <typename T, int NZ, int STRIDE, int U, int BITS>
__device__ __forceinline__ void gridValuesN(T const (&bv)[U][kMaxStagedBases], DevGroup const& G, T const (&cost)[U],
                                            T const (&pfc)[U], T* acc)
{
#pragma unroll
    for (int u = 0; u < U; ++u) gridValues<T, NZ, STRIDE, BITS>(bv[u], G, cost[u], pfc[u], acc);
}

// gridForces of U triplets.
template <typename T, int NZ, bool COMPACT, int U, int BITS>
__device__ __forceinline__ void gridForcesN(T const (&bv)[U][kMaxStagedBases], DevGroup const& G,
                                            Members<T, COMPACT> const& mb, T const (&cost)[U], T (&T1)[U], T (&T2)[U],
                                            T (&T3)[U])
{
#pragma unroll
    for (int u = 0; u < U; ++u)
    {
        T1[u] = T2[u] = T3[u] = T(0);
        gridForces<T, NZ, COMPACT, BITS>(bv[u], G, mb, cost[u], T1[u], T2[u], T3[u]);
    }
}

} // namespace

// Whether atom i belongs to a kernel tier of stage capacity cap: its list
// fits the buffers and has lower < n <= cap entries (or, for the last tier
// with flagOverflow, more than cap, which that tier reports).
__device__ __forceinline__ bool atomInTier(BatchView const& b, int i, int lower, int cap, bool flagOverflow)
{
    if (i >= b.N) return false;
    const int64_t off = b.nbrOffset[i], end = b.nbrOffset[i + 1];
    if (end > b.nbrCapacity) return false;
    const int n = (int)(end - off);
    return (n <= cap && n > lower) || (flagOverflow && n > cap);
}

// ---------------------------------------------------------------------------
// G values
// ---------------------------------------------------------------------------
// Blocks per SM the register allocation must allow (measured on the water
// workloads): the specialised G pass with the poly2 cutoff fits 6 four-warp
// blocks (<= 80 registers; its lean member stage leaves room in shared
// memory; FP64 with four zeta slots 5), the FP32 force pass with two zeta
// slots 5; every other four-warp instance 4, the larger stages 1.
template <typename T, int WARPS, int FAST, int CUT, bool FORCES>
constexpr int sfMinBlocks()
{
    if (WARPS != 4 || FAST == 0 || CUT != 6) return WARPS != 4 ? 1 : 4;
    if (!FORCES) return (sizeof(T) == 8 && FAST == 4) ? 5 : 6;
    return (sizeof(T) == 4 && FAST == 2) ? 5 : 4;
}

template <typename T, int CAP, int WARPS, int FAST, int CUT>
__global__ void __launch_bounds__(WARPS * 32, (sfMinBlocks<T, WARPS, FAST, CUT, false>()))
    kSFValuesF(DevModel model, BatchView b, int lower, int flagOverflow, DevGroupTable gt)
{
    constexpr int ILP = 1;            // triplets per lane and step (see loadTriplets)
    constexpr int kStep = 32 * ILP;   // triplets per warp step
    extern __shared__ __align__(16) unsigned char smemRaw[];
    ValuesSmem<T, CAP, FAST>& SM = reinterpret_cast<ValuesSmem<T, CAP, FAST>*>(smemRaw)[threadIdx.x >> 5];
    auto& S = SM.st;
    auto& mb = SM.mb;
    const int lane = threadIdx.x & 31;
    // Accumulators per sweep: the member grid of the model (FAST = its zeta
    // slots) or a chunk of members.
    constexpr int ACC = FAST ? 4 * FAST : kChunkF;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    // the warp's atoms i = warp + k warpsPerGrid, tested 32 at a time (one load per lane instead of a
    // dependent load per atom: the upper tiers take few atoms)
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (int k0 = 0; warp + k0 * warpsPerGrid < b.N; k0 += 32)
    {
        const int mine = warp + (k0 + (threadIdx.x & 31)) * warpsPerGrid;
        unsigned todo = __ballot_sync(kFullMask, atomInTier(b, mine, lower, CAP, flagOverflow != 0));
        while (todo)
        {
            const int i = warp + (k0 + __ffs(todo) - 1) * warpsPerGrid;
            todo &= todo - 1;
            const int64_t off = b.nbrOffset[i];
            const int64_t end = b.nbrOffset[i + 1];
            if (end > b.nbrCapacity) continue;
            const int n = (int)(end - off);
            if (flagOverflow && n > CAP)
            {
                if (lane == 0) atomicAdd(&b.status->badInput, 1);
                continue;
            }
            if (!(n <= CAP && n > lower)) continue;
            const int ec = b.elem[i];
            DevElement const& E = model.el[ec];
            uint32_t* maskOut =
                (b.candMask && b.maskOffset[i + 1] <= b.maskCapacity) ? b.candMask + b.maskOffset[i] : nullptr;
            int mwi = 0;
            stageGeometry<T, CAP>(S, off, n, model, b, lane);
            int slot = -1;
            for (int g = 0; g < E.groupCount; ++g)
            {
                DevGroup scratch;
                DevGroup const& G = groupOf<FAST>(gt, model, E.groupBegin + g, scratch);
                const bool fastG = FAST || G.fast;
                if (G.cutoffSlot != slot)
                {
                    stageCutoff<T, CAP>(S, off, n, G.cutoffSlot, b, lane);
                    slot = G.cutoffSlot;
                }
                stageMembers(mb, model, G, nullptr, lane);
                if (G.type != 2 && fastG) stageFactors<T, CAP>(S, G, lane);
                const T rc = (T)G.rc, rc2 = (T)G.rc2;
                const DevMember* mem = model.members + G.memberBegin;
                const bool narrow = (G.type == 3);
                const bool grid = (G.type != 2) && (FAST || G.grid);
                const int mwiGroup = mwi;
                for (int m0 = 0; m0 < G.memberCount; m0 += (grid ? G.memberCount : ACC))
                {
                    mwi = mwiGroup;   // every member chunk enumerates the same candidates; the first records them
                    const int mc = min(ACC, G.memberCount - m0);
                    T acc[ACC];
    #pragma unroll
                    for (int q = 0; q < ACC; ++q) acc[q] = T(0);
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
                                eb[q] = (fastG && q < G.numBases) ? fexp<T>(-groupBaseEta<T>(G, q) * r * r) : T(0);
    #pragma unroll
                            for (int q = 0; q < ACC; ++q)
                            {
                                if (q < mc)
                                {
                                    const int qq = m0 + q;
                                    T v;
                                    if (fastG)
                                    {
                                        const int bq = mb.base[qq];
                                        T e0 = eb[0];
    #pragma unroll
                                        for (int t = 1; t < kMaxBases; ++t)
                                            if (bq == t) e0 = eb[t];
                                        v = powUniform<T>(e0, mb.pw[qq]);
                                    }
                                    else v = gaussShifted<T>(mb.eta[qq], mb.rs[qq], r, mb.rs[qq], mb.rs[qq], 0);
                                    acc[q] += v * fc;
                                }
                            }
                        }
                    }
                    else
                    {
                        const bool same = (G.e1 == G.e2);
                        const int A0 = S.blockBegin[G.e1], nA = S.nBelow[G.cutoffSlot][G.e1];
                        const int B0 = S.blockBegin[G.e2], nB = S.nBelow[G.cutoffSlot][G.e2];
                        Phase ph[2];
                        const int nph = roundPhases(A0, nA, B0, nB, same, ph);
                        int qn = 0, qh = 0;
                        for (int k = 0; k <= nph; ++k)
                        {
                            const bool drain = (k == nph);
                            Cursor cur;
                            int cnt = 0;
                            if (!drain)
                            {
                                cur.init(ph[k], lane);
                                cnt = ph[k].count;
                            }
                            int p0 = 0;
                            while (true)
                            {
                                if (qn < kStep && p0 < cnt)   // queue stays below kStep + 64 entries
                                {
                                    enqueueCandidates<T, CAP>(S, ph[k], cur, p0, rc, rc2, narrow, SM.queue, qh, qn, lane,
                                                              m0 == 0 ? maskOut : nullptr, nullptr, mwi);
                                    p0 += 64;
                                }
                                if (qn >= kStep || (drain && qn > 0))
                                {
                                    const int take = min(kStep, qn);
                                    if constexpr (FAST > 0)
                                    {
                                        Triplet<T> t[ILP];
                                        int so[ILP], sp[ILP];
                                        bool ok[ILP];
                                        loadTriplets<CUT, T, CAP>(S, model.cutoff[G.cutoffSlot], narrow, SM.queue, qh, take, lane,
                                                             t, so, sp, ok);
                                        T bv[ILP][kMaxStagedBases], cost[ILP], pfc[ILP];
    #pragma unroll
                                        for (int u = 0; u < ILP; ++u)
                                        {
                                            tripletBases<T, CAP>(S, G, narrow, so[u], sp[u], t[u].rjk2, bv[u]);
                                            cost[u] = t[u].cost;
                                            pfc[u] = ok[u] ? t[u].fc1 * t[u].fc2 * t[u].fcjk : T(0);
                                        }
                                        gridValuesN<T, FAST, FAST, ILP, sfPowBits<FAST, CUT>()>(bv, G, cost, pfc, acc);
                                    }
                                    else if (lane < take)
                                    {
                                        const int e = SM.queue[(qh + lane) & (kQueue - 1)];
                                        const int so = entryOwner(e), sp = entryPartner(e);
                                        Triplet<T> t;
                                        loadTriplet<T, CAP>(S, model.cutoff[G.cutoffSlot], narrow, so, sp, t);
                                        const T pfc = t.fc1 * t.fc2 * t.fcjk;
                                        T bv[kMaxStagedBases];
                                        if (fastG) tripletBases<T, CAP>(S, G, narrow, so, sp, t.rjk2, bv);
                                        T vexp = T(0);
                                        if (grid)
                                        {
                                            if (G.gridNZ <= 2) gridValues<T, 2, 4>(bv, G, t.cost, pfc, acc);
                                            else gridValues<T, 4, 4>(bv, G, t.cost, pfc, acc);
                                        }
                                        else
                                        {
    #pragma unroll
                                            for (int q = 0; q < ACC; ++q)
                                            {
                                                if (q < mc)
                                                {
                                                    const int qq = m0 + q;
                                                    if ((mb.flags[qq] & 2) || q == 0)
                                                        vexp = fastG ? powUniform<T>(mb.base[qq] == 0 ? bv[0] : bv[1], mb.pw[qq])
                                                                     : gaussShifted<T>(mb.eta[qq], mb.rs[qq], t.r1, t.r2,
                                                                                       t.rjk, narrow ? 1 : 0);
                                                    const T pl = T(1) + mb.lambda[qq] * t.cost;
                                                    if (pl > T(0)) acc[q] += vexp * angularPow<T>(pl, mb, qq) * pl * pfc;
                                                }
                                            }
                                        }
                                    }
                                    qh = (qh + take) & (kQueue - 1);
                                    qn -= take;
                                    __syncwarp();
                                }
                                else if (p0 >= cnt) break;
                            }
                        }
                    }
    #pragma unroll
                    for (int q = 0; q < ACC; ++q)
                    {
                        const int c = FAST ? (q / (FAST ? FAST : 1)) * 4 + q % (FAST ? FAST : 1) : q;
                        const int qq = grid ? (int)G.comboMember[c] : (q < mc ? m0 + q : -1);
                        if (qq >= 0)
                        {
                            double sum = warpSum((double)acc[q]);
                            if (lane == (q & 31))
                            {
                                DevMember const& M = mem[qq];
                                if (G.type != 2) sum *= M.gNorm;
                                b.G[(size_t)i * b.gStride + M.sf] = scaleG(model.scaling[E.sfBegin + M.sf], sum);
                            }
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
// prefactors p1, p2, p3 (SymGrpExpAngn.cpp:305-337) contract, for the
// unordered pair (j, k), to
//   P1 = pfc ((1/(rij rik) - cos/rij^2) T1 - Uij) + pr1 T3
//   P2 = pfc ((1/(rij rik) - cos/rik^2) T1 - Uik) + pr2 T3
//   P3 = pfc (1/(rij rik) T1 + Ujk) - pr3 T3          (narrow)
//   P3 = pfc /(rij rik) T1                            (wide)
// T1 = sum a zeta lambda, T3 = sum a plambda,
// Uij = sum a zeta lambda plambda factorDeriv (rij - rs)/rij  (Uik, Ujk alike).
// The force E_i puts on j gains P1 dr_ij + P3 dr_jk, on k P2 dr_ik - P3 dr_jk;
// the self force on i loses P1 dr_ij + P2 dr_ik.  Each pair is evaluated once.
// Pairs are enumerated in rounds of matchings, so the lanes of one round add
// their two contributions to distinct slots; rounds add one after another in
// a fixed order (deterministic, no atomics).

// One warp step of the force pass over the queue window [qh, qh + take),
// ILP triplets per lane (model-specialised kernels): lane l evaluates
// entries l + 32 u.  The self-force sums and the scatter into h keep the
// one-triplet-per-lane order (entry l before l + 32, and the window's
// halves scattered one after the other).
template <typename T, int CAP, int FAST, int CUT, int ILP>
__device__ __forceinline__ void forcesStepN(Stage<T, CAP, true, 1> const& S, Members<T, true> const& mb, DevGroup const& G,
                                            DevCutoff const& cut, bool narrow, const int* queue, int qh, int take,
                                            int lane, T (&h)[3][CAP], T& sfx, T& sfy, T& sfz)
{
    Triplet<T> t[ILP];
    int so[ILP], sp[ILP];
    bool ok[ILP];
    loadTriplets<CUT, T, CAP>(S, cut, narrow, queue, qh, take, lane, t, so, sp, ok);
    T bv[ILP][kMaxStagedBases], cost[ILP];
#pragma unroll
    for (int u = 0; u < ILP; ++u)
    {
        tripletBases<T, CAP>(S, G, narrow, so[u], sp[u], t[u].rjk2, bv[u]);
        cost[u] = t[u].cost;
    }
    T T1[ILP], T2[ILP], T3[ILP];
    gridForcesN<T, FAST, true, ILP, sfPowBits<FAST, CUT>()>(bv, G, mb, cost, T1, T2, T3);
    T o[ILP][3], q[ILP][3];
#pragma unroll
    for (int u = 0; u < ILP; ++u)
    {
        Triplet<T> const& x = t[u];
        const T dfcr2 = S.dfcr[sp[u]];
        const T pfc = x.fc1 * x.fc2 * x.fcjk;
        const T pr1 = x.fc2 * x.fcjk * x.dfcr1;
        const T pr2 = x.fc1 * x.fcjk * dfcr2;
        const T pr3 = narrow ? x.fc1 * x.fc2 * x.dfcjk * x.rijk : T(0);
        const T P1 = pfc * ((x.rinv - x.cost * x.ri1 * x.ri1) * T1[u] - T2[u]) + pr1 * T3[u];
        const T P2 = pfc * ((x.rinv - x.cost * x.ri2 * x.ri2) * T1[u] - T2[u]) + pr2 * T3[u];
        const T P3 = narrow ? (pfc * (x.rinv * T1[u] + T2[u]) - pr3 * T3[u]) : (pfc * x.rinv * T1[u]);
        o[u][0] = P1 * x.x1 + P3 * x.dx3;
        o[u][1] = P1 * x.y1 + P3 * x.dy3;
        o[u][2] = P1 * x.z1 + P3 * x.dz3;
        q[u][0] = P2 * x.x2 - P3 * x.dx3;
        q[u][1] = P2 * x.y2 - P3 * x.dy3;
        q[u][2] = P2 * x.z2 - P3 * x.dz3;
        if (ok[u])
        {
            sfx -= P1 * x.x1 + P2 * x.x2;
            sfy -= P1 * x.y1 + P2 * x.y2;
            sfz -= P1 * x.z1 + P2 * x.z2;
        }
    }
#pragma unroll
    for (int u = 0; u < ILP; ++u)
    {
        // one conflict-free add per round present in this half of the window
        const int idx = lane + 32 * u;
        const bool mine = idx < take;
        const int rnd = mine ? entryRound(queue[(qh + idx) & (kQueue - 1)]) : -1;
        const int prevRnd = __shfl_up_sync(kFullMask, rnd, 1);
        const unsigned heads = __ballot_sync(kFullMask, mine && (lane == 0 || prevRnd != rnd));
        const int mySub = __popc(heads & ((2u << lane) - 1u)) - 1;
        const int nSub = __popc(heads);
        for (int r = 0; r < nSub; ++r)
        {
            if (mine && mySub == r)
            {
                h[0][so[u]] += o[u][0];
                h[1][so[u]] += o[u][1];
                h[2][so[u]] += o[u][2];
                h[0][sp[u]] += q[u][0];
                h[1][sp[u]] += q[u][1];
                h[2][sp[u]] += q[u][2];
            }
            __syncwarp();
        }
    }
}

template <typename T, int CAP, int WARPS, int FAST, int CUT>
__global__ void __launch_bounds__(WARPS * 32, (sfMinBlocks<T, WARPS, FAST, CUT, true>()))
    kSFForcesF(DevModel model, BatchView b, int lower, DevGroupTable gt)
{
    constexpr int ILP = 1;            // triplets per lane and step (see loadTriplets)
    constexpr int kStep = 32 * ILP;   // triplets per warp step
    extern __shared__ __align__(16) unsigned char smemRaw[];
    ForcesSmem<T, CAP, FAST>& SM = reinterpret_cast<ForcesSmem<T, CAP, FAST>*>(smemRaw)[threadIdx.x >> 5];
    auto& S = SM.st;
    auto& mb = SM.mb;
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    // the warp's atoms i = warp + k warpsPerGrid, tested 32 at a time (one load per lane instead of a
    // dependent load per atom: the upper tiers take few atoms)
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (int k0 = 0; warp + k0 * warpsPerGrid < b.N; k0 += 32)
    {
        const int mine = warp + (k0 + (threadIdx.x & 31)) * warpsPerGrid;
        unsigned todo = __ballot_sync(kFullMask, atomInTier(b, mine, lower, CAP, false));
        while (todo)
        {
            const int i = warp + (k0 + __ffs(todo) - 1) * warpsPerGrid;
            todo &= todo - 1;
            const int64_t off = b.nbrOffset[i];
            const int64_t end = b.nbrOffset[i + 1];
            if (end > b.nbrCapacity) continue;
            const int n = (int)(end - off);
            if (!(n <= CAP && n > lower)) continue;
            const int ec = b.elem[i];
            DevElement const& E = model.el[ec];
            const double* dEdG = b.dEdG + (size_t)i * b.gStride;
            const uint32_t* maskIn =
                (b.candMask && b.maskOffset[i + 1] <= b.maskCapacity) ? b.candMask + b.maskOffset[i] : nullptr;
            int mwi = 0;
            stageGeometry<T, CAP>(S, off, n, model, b, lane);
            for (int s = lane; s < n; s += 32) SM.h[0][s] = SM.h[1][s] = SM.h[2][s] = T(0);
            // self force: the FP64 form sums every term into gs*; the FP32 form
            // sums a group's terms in FP32 and adds each group's total to sf* in FP64
            double sfx = 0.0, sfy = 0.0, sfz = 0.0;
            T gsx = T(0), gsy = T(0), gsz = T(0);
            int slot = -1;
            for (int g = 0; g < E.groupCount; ++g)
            {
                if constexpr (sizeof(T) == 4)
                {
                    sfx += (double)gsx;
                    sfy += (double)gsy;
                    sfz += (double)gsz;
                    gsx = gsy = gsz = T(0);
                }
                DevGroup scratch;
                DevGroup const& G = groupOf<FAST>(gt, model, E.groupBegin + g, scratch);
                const bool fastG = FAST || G.fast;
                if (G.cutoffSlot != slot)
                {
                    stageCutoff<T, CAP>(S, off, n, G.cutoffSlot, b, lane);
                    slot = G.cutoffSlot;
                }
                stageMembers(mb, model, G, dEdG, lane);
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
                            eb[q] = (fastG && q < G.numBases) ? fexp<T>(-groupBaseEta<T>(G, q) * r * r) : T(0);
                        T P = T(0);
                        for (int q = 0; q < M; ++q)
                        {
                            T v;
                            if (fastG)
                            {
                                const int bq = mb.base[q];
                                T e0 = eb[0];
    #pragma unroll
                                for (int t = 1; t < kMaxBases; ++t)
                                    if (bq == t) e0 = eb[t];
                                v = powUniform<T>(e0, mb.pw[q]);
                            }
                            else v = gaussShifted<T>(mb.eta[q], mb.rs[q], r, mb.rs[q], mb.rs[q], 0);
                            P += mb.cw[q] * (dfc - T(2) * mb.eta[q] * (r - mb.rs[q]) * fc) * v * ri;
                        }
                        const T ddx = S.x[s] * P, ddy = S.y[s] * P, ddz = S.z[s] * P;
                        SM.h[0][s] += ddx;
                        SM.h[1][s] += ddy;
                        SM.h[2][s] += ddz;
                        gsx -= ddx;
                        gsy -= ddy;
                        gsz -= ddz;
                    }
                    __syncwarp();
                    continue;
                }
                if (fastG) stageFactors<T, CAP>(S, G, lane);
                const bool narrow = (G.type == 3);
                const bool same = (G.e1 == G.e2);
                const int A0 = S.blockBegin[G.e1], nA = S.nBelow[G.cutoffSlot][G.e1];
                const int B0 = S.blockBegin[G.e2], nB = S.nBelow[G.cutoffSlot][G.e2];
                Phase ph[2];
                const int nph = roundPhases(A0, nA, B0, nB, same, ph);
                int qn = 0, qh = 0;
                for (int k = 0; k <= nph; ++k)
                {
                    const bool drain = (k == nph);
                    Cursor cur;
                    int cnt = 0;
                    if (!drain)
                    {
                        cur.init(ph[k], lane);
                        cnt = ph[k].count;
                    }
                    int p0 = 0;
                    while (true)
                    {
                        if (qn < kStep && p0 < cnt)   // queue stays below kStep + 64 entries
                        {
                            enqueueCandidates<T, CAP>(S, ph[k], cur, p0, rc, rc2, narrow, SM.queue, qh, qn, lane,
                                                      nullptr, maskIn, mwi);
                            p0 += 64;
                        }
                        if constexpr (FAST > 0)
                        {
                            if (qn >= kStep || (drain && qn > 0))
                            {
                                const int take = min(kStep, qn);
                                forcesStepN<T, CAP, FAST, CUT, ILP>(S, mb, G, model.cutoff[G.cutoffSlot], narrow, SM.queue, qh,
                                                              take, lane, SM.h, gsx, gsy, gsz);
                                qh = (qh + take) & (kQueue - 1);
                                qn -= take;
                                __syncwarp();
                            }
                            else if (p0 >= cnt) break;
                            continue;
                        }
                        if (qn >= 32 || (drain && qn > 0))
                        {
                            const int take = min(32, qn);
                            int keyO = 0, keyP = 0;
                            T ox = T(0), oy = T(0), oz = T(0), px = T(0), py = T(0), pz = T(0);
                            if (lane < take)
                            {
                                const int e = SM.queue[(qh + lane) & (kQueue - 1)];
                                const int so = entryOwner(e), sp = entryPartner(e);
                                keyO = so;
                                keyP = sp;
                                Triplet<T> t;
                                loadTriplet<T, CAP>(S, model.cutoff[G.cutoffSlot], narrow, so, sp, t);
                                const T dfcr2 = S.dfcr[sp];
                                const T pfc = t.fc1 * t.fc2 * t.fcjk;
                                const T pr1 = t.fc2 * t.fcjk * t.dfcr1;
                                const T pr2 = t.fc1 * t.fcjk * dfcr2;
                                const T pr3 = narrow ? t.fc1 * t.fc2 * t.dfcjk * t.rijk : T(0);
                                T bv[kMaxStagedBases];
                                if (fastG) tripletBases<T, CAP>(S, G, narrow, so, sp, t.rjk2, bv);
                                T T1 = T(0), T3 = T(0), Uij = T(0), Uik = T(0), Ujk = T(0), vexp = T(0);
                                if (G.grid)
                                {
                                    T T2 = T(0);
                                    if (G.gridNZ <= 2) gridForces<T, 2>(bv, G, mb, t.cost, T1, T2, T3);
                                    else gridForces<T, 4>(bv, G, mb, t.cost, T1, T2, T3);
                                    Uij = T2;
                                    Uik = T2;
                                    Ujk = T2;
                                }
                                else
                                {
                                for (int q = 0; q < M; ++q)
                                {
                                    if ((mb.flags[q] & 2) || q == 0)
                                        vexp = fastG ? powUniform<T>(mb.base[q] == 0 ? bv[0] : bv[1], mb.pw[q])
                                                      : gaussShifted<T>(mb.eta[q], mb.rs[q], t.r1, t.r2, t.rjk,
                                                                        narrow ? 1 : 0);
                                    const T pl = T(1) + mb.lambda[q] * t.cost;
                                    if (!(pl > T(0))) continue;
                                    const T a = mb.cw[q] * vexp * angularPow<T>(pl, mb, q);
                                    const T azl = a * mb.zl[q];
                                    const T azq = azl * pl * mb.fd[q];
                                    T1 += azl;
                                    T3 += a * pl;
                                    if (mb.rs[q] > T(0))
                                    {
                                        Uij += azq * (t.r1 - mb.rs[q]) * t.ri1;
                                        Uik += azq * (t.r2 - mb.rs[q]) * t.ri2;
                                        if (narrow) Ujk += azq * (t.rjk - mb.rs[q]) * t.rijk;
                                    }
                                    else
                                    {
                                        Uij += azq;
                                        Uik += azq;
                                        Ujk += azq;
                                    }
                                }
                                }
                                // both ends of the unordered pair (j, k): P1 for j, P2 (= P1 with j, k
                                // exchanged) for k; P3 is symmetric and enters with opposite signs.
                                const T P1 = pfc * ((t.rinv - t.cost * t.ri1 * t.ri1) * T1 - Uij) + pr1 * T3;
                                const T P2 = pfc * ((t.rinv - t.cost * t.ri2 * t.ri2) * T1 - Uik) + pr2 * T3;
                                const T P3 = narrow ? (pfc * (t.rinv * T1 + Ujk) - pr3 * T3) : (pfc * t.rinv * T1);
                                ox = P1 * t.x1 + P3 * t.dx3;
                                oy = P1 * t.y1 + P3 * t.dy3;
                                oz = P1 * t.z1 + P3 * t.dz3;
                                px = P2 * t.x2 - P3 * t.dx3;
                                py = P2 * t.y2 - P3 * t.dy3;
                                pz = P2 * t.z2 - P3 * t.dz3;
                                gsx -= P1 * t.x1 + P2 * t.x2;
                                gsy -= P1 * t.y1 + P2 * t.y2;
                                gsz -= P1 * t.z1 + P2 * t.z2;
                            }
                            // One conflict-free add per round present in the batch: inside a
                            // round no slot occurs twice.
                            const int rnd = lane < take ? entryRound(SM.queue[(qh + lane) & (kQueue - 1)]) : -1;
                            const int prevRnd = __shfl_up_sync(kFullMask, rnd, 1);
                            const unsigned heads = __ballot_sync(kFullMask, lane < take && (lane == 0 || prevRnd != rnd));
                            const int mySub = __popc(heads & ((2u << lane) - 1u)) - 1;
                            const int nSub = __popc(heads);
                            for (int r = 0; r < nSub; ++r)
                            {
                                if (lane < take && mySub == r)
                                {
                                    SM.h[0][keyO] += ox;
                                    SM.h[1][keyO] += oy;
                                    SM.h[2][keyO] += oz;
                                    SM.h[0][keyP] += px;
                                    SM.h[1][keyP] += py;
                                    SM.h[2][keyP] += pz;
                                }
                                __syncwarp();
                            }
                            qh = (qh + take) & (kQueue - 1);
                            qn -= take;
                            __syncwarp();
                        }
                        else if (p0 >= cnt) break;
                    }
                }
            }
            __syncwarp();
            for (int s = lane; s < n; s += 32)
            {
                const int64_t e = off + S.perm[s];
                b.hx[e] = (double)SM.h[0][s];
                b.hy[e] = (double)SM.h[1][s];
                b.hz[e] = (double)SM.h[2][s];
            }
            if constexpr (sizeof(T) == 4)
            {
                sfx += (double)gsx;
                sfy += (double)gsy;
                sfz += (double)gsz;
            }
            else
            {
                sfx = gsx;
                sfy = gsy;
                sfz = gsz;
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

}

} // namespace n2p2b200
