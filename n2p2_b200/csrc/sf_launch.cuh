// Launch sequence of the symmetry-function passes for one precision: the
// tiers of stage capacity, the first tier's shape chosen by the autotuner
// (engine.cu, Batch::autotune) among kSFShapeCount variants.
#pragma once

#include "sf_fast.cuh"

namespace n2p2b200 {

namespace {

constexpr int kMidCap = 384, kMidWarps = 2;     // second tier: atoms with up to 384 neighbours
constexpr int kBigCap = 1024, kBigWarps = 1;    // last tier (flags larger atoms)
constexpr int kGenericCap = 160, kGenericWarps = 4;

int gridFor(int N, int warpsPerBlock, int sms, int perSM)
{
    int need = (N + warpsPerBlock - 1) / warpsPerBlock;
    int cap = sms * perSM;
    return need < cap ? (need > 0 ? need : 1) : cap;
}

template <typename T, int CAP, int WARPS, int FAST, int CUT = kCutAny>
void valuesTier(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st, int lower,
                int flag, int perSM)
{
    static_assert(sizeof(ValuesSmem<T, CAP, FAST>) % 16 == 0, "per-warp blocks must stay 16-byte aligned");
    const size_t smem = sizeof(ValuesSmem<T, CAP, FAST>) * WARPS;
    auto k = kSFValuesF<T, CAP, WARPS, FAST, CUT>;
    setDynamicSmemOnce(reinterpret_cast<const void*>(k), smem);
    k<<<gridFor(b.N, WARPS, sms, perSM), WARPS * 32, smem, st>>>(m, b, lower, flag, gt);
}

template <typename T, int CAP, int WARPS, int FAST, int CUT = kCutAny>
void forcesTier(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st, int lower,
                int perSM)
{
    static_assert(sizeof(ForcesSmem<T, CAP, FAST>) % 16 == 0, "per-warp blocks must stay 16-byte aligned");
    const size_t smem = sizeof(ForcesSmem<T, CAP, FAST>) * WARPS;
    auto k = kSFForcesF<T, CAP, WARPS, FAST, CUT>;
    setDynamicSmemOnce(reinterpret_cast<const void*>(k), smem);
    k<<<gridFor(b.N, WARPS, sms, perSM), WARPS * 32, smem, st>>>(m, b, lower, gt);
}

// First-tier shapes (stage capacity, warps per block) of the specialised
// kernels; variant v of kSFShapes.
template <typename T, int FAST, int CUT>
void valuesFast(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st, int variant)
{
    int cap0 = 0;
    switch (variant)
    {
    case 0: valuesTier<T, 128, 4, FAST, CUT>(m, gt, b, sms, st, -1, 0, 32); cap0 = 128; break;
    case 1: valuesTier<T, 160, 4, FAST, CUT>(m, gt, b, sms, st, -1, 0, 32); cap0 = 160; break;
    default: valuesTier<T, 192, 2, FAST, CUT>(m, gt, b, sms, st, -1, 0, 64); cap0 = 192; break;
    }
    valuesTier<T, kMidCap, kMidWarps, FAST, CUT>(m, gt, b, sms, st, cap0, 0, 4);
    valuesTier<T, kBigCap, kBigWarps, FAST, CUT>(m, gt, b, sms, st, kMidCap, 1, 2);
}

template <typename T, int FAST, int CUT>
void forcesFast(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st, int variant)
{
    int cap0 = 0;
    switch (variant)
    {
    case 0: forcesTier<T, 128, 4, FAST, CUT>(m, gt, b, sms, st, -1, 32); cap0 = 128; break;
    case 1: forcesTier<T, 160, 4, FAST, CUT>(m, gt, b, sms, st, -1, 32); cap0 = 160; break;
    default: forcesTier<T, 192, 2, FAST, CUT>(m, gt, b, sms, st, -1, 64); cap0 = 192; break;
    }
    forcesTier<T, kMidCap, kMidWarps, FAST, CUT>(m, gt, b, sms, st, cap0, 4);
    forcesTier<T, kBigCap, kBigWarps, FAST, CUT>(m, gt, b, sms, st, kMidCap, 2);
}

// The cutoff type has an instance of its own (every cutoff slot of a model
// shares the model's type).
inline bool poly2Cutoff(DevModel const& m)
{
    return m.cutoff[0].type == kCutPoly2;
}

// The poly2 instance of `fast` zeta slots also requires the model's integer
// powers within its compile-time bound (sfPowBits).
inline bool poly2Instance(DevModel const& m, int fast)
{
    return poly2Cutoff(m) && m.powBits <= (fast == 2 ? sfPowBits<2, kCutPoly2>() : sfPowBits<4, kCutPoly2>());
}

template <typename T>
void valuesT(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st, int variant)
{
    if (m.allFast == 2 && poly2Instance(m, 2)) valuesFast<T, 2, kCutPoly2>(m, gt, b, sms, st, variant);
    else if (m.allFast == 4 && poly2Instance(m, 4)) valuesFast<T, 4, kCutPoly2>(m, gt, b, sms, st, variant);
    else if (m.allFast == 2) valuesFast<T, 2, kCutAny>(m, gt, b, sms, st, variant);
    else if (m.allFast == 4) valuesFast<T, 4, kCutAny>(m, gt, b, sms, st, variant);
    else
    {
        valuesTier<T, kGenericCap, kGenericWarps, 0>(m, gt, b, sms, st, -1, 0, 32);
        valuesTier<T, kBigCap, kBigWarps, 0>(m, gt, b, sms, st, kGenericCap, 1, 2);
    }
}

template <typename T>
void forcesT(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st, int variant)
{
    if (m.allFast == 2 && poly2Instance(m, 2)) forcesFast<T, 2, kCutPoly2>(m, gt, b, sms, st, variant);
    else if (m.allFast == 4 && poly2Instance(m, 4)) forcesFast<T, 4, kCutPoly2>(m, gt, b, sms, st, variant);
    else if (m.allFast == 2) forcesFast<T, 2, kCutAny>(m, gt, b, sms, st, variant);
    else if (m.allFast == 4) forcesFast<T, 4, kCutAny>(m, gt, b, sms, st, variant);
    else
    {
        forcesTier<T, kGenericCap, kGenericWarps, 0>(m, gt, b, sms, st, -1, 32);
        forcesTier<T, kBigCap, kBigWarps, 0>(m, gt, b, sms, st, kGenericCap, 2);
    }
}

} // namespace

} // namespace n2p2b200
