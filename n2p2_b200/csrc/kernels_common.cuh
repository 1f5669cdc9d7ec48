// Device helpers shared by the sm_100a kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_model.hpp"

namespace n2p2b200 {

constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ double warpSum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
    return v;
}

__device__ __forceinline__ float warpSum(float v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
    return v;
}

__device__ __forceinline__ int warpSumInt(int v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
    return v;
}

__device__ __forceinline__ int warpMaxInt(int v)
{
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(kFullMask, v, o));
    return v;
}

// Exponentiation by squaring with the multiplication order of the reference's
// pow_int (utility.cpp:292-316), so integer zeta gives the same rounding.
template <typename T>
__device__ __forceinline__ T powInt(T x, int n)
{
    unsigned m;
    if (n < 0)
    {
        x = T(1) / x;
        m = (unsigned)(-n);
    }
    else m = (unsigned)n;
    T result = T(1);
    do
    {
        if (m & 1u) result *= x;
        m >>= 1;
        x *= x;
    } while (m);
    return result;
}

// Cutoff function value and derivative, CutoffFunction::fdf
// (CutoffFunction.h:210-220) with the per-type bodies of CutoffFunction.cpp
// and CoreFunction.h:239-318.  Always evaluated in FP64.
// Core functions of x in [0, 1) (CoreFunction::fdf*, CoreFunction.h:189-319):
// exp (type 4) and the polynomials poly1..poly4 (types 5-8).
__device__ __forceinline__ void coreFdf(int type, double x, double& fx, double& dfx)
{
    const double kE = 2.718281828459045235360287471352662498;
    if (type == 4)
    {
        double t = 1.0 / (x * x - 1.0);
        double e = exp(t);
        fx = kE * e;
        dfx = -2.0 * kE * x * t * t * e;
    }
    else if (type == 5)
    {
        fx = (2.0 * x - 3.0) * x * x + 1.0;
        dfx = x * (6.0 * x - 6.0);
    }
    else if (type == 6)
    {
        double x2 = x * x;
        fx = ((15.0 - 6.0 * x) * x - 10.0) * x * x2 + 1.0;
        dfx = x2 * ((60.0 - 30.0 * x) * x - 30.0);
    }
    else if (type == 7)
    {
        double x2 = x * x;
        fx = (x * (x * (20.0 * x - 70.0) + 84.0) - 35.0) * x2 * x2 + 1.0;
        dfx = x2 * x * (x * (x * (140.0 * x - 420.0) + 420.0) - 140.0);
    }
    else
    {
        double x4 = x * x;
        x4 *= x4;
        fx = (x * (x * ((315.0 - 70.0 * x) * x - 540.0) + 420.0) - 126.0) * x * x4 + 1.0;
        dfx = x4 * (x * (x * ((2520.0 - 630.0 * x) * x - 3780.0) + 2520.0) - 630.0);
    }
}

__device__ __forceinline__ void cutoffFdf(DevCutoff const& c, double r, double& fc, double& dfc)
{
    if (r >= c.rc)
    {
        fc = 0.0;
        dfc = 0.0;
        return;
    }
    const double kPi = 3.141592653589793238462643383279502884;
    switch (c.type)
    {
    case 0:  // hard
        fc = 1.0;
        dfc = 0.0;
        return;
    case 1:  // cos
    {
        if (r < c.rci)
        {
            fc = 1.0;
            dfc = 0.0;
            return;
        }
        double x = (r - c.rci) * c.iw;
        double t = cos(kPi * x);
        fc = 0.5 * (t + 1.0);
        dfc = -0.5 * c.iw * kPi * sqrt(1.0 - t * t);
        return;
    }
    case 2:  // tanhU
    case 3:  // tanh (normalised to f(0)=1)
    {
        double t = tanh(1.0 - r * c.rcinv);
        double t2 = t * t;
        double pre = (c.type == 3) ? c.tanhPre : 1.0;
        fc = pre * t * t2;
        dfc = 3.0 * pre * t2 * (t2 - 1.0) * c.rcinv;
        return;
    }
    default:  // core functions: exp, poly1..poly4
    {
        if (r < c.rci)
        {
            fc = 1.0;
            dfc = 0.0;
            return;
        }
        double x = (r - c.rci) * c.iw;
        double fx, dfx;
        coreFdf(c.type, x, fx, dfx);
        fc = fx;
        dfc = dfx * c.iw;
        return;
    }
    }
}

// The cutoff function in FP32 (the mixed form's per-triplet f_c(r_jk); the
// per-pair f_c(r_ij) values come from cutoffFdf in FP64).  The polynomial
// cores (types 5-8, poly1..poly4) are 1 - S_n(x) for the smoothstep
// polynomials S_n, which factor as
//   1 - S_n(x) = u^(n+1) sum_{k=0..n} C(n+k, k) x^k,   u = 1 - x,
//   d/dx      = -(2n+1)!/(n!)^2 x^n u^n,
// (poly2: u^3 (1 + 3x + 6x^2) = ((15 - 6x)x - 10)x^3 + 1 and -30 x^2 u^2).
// With u = (r_c - r) iw computed directly there is no cancellation as
// r -> r_c, so FP32 keeps the relative accuracy near the cutoff that the
// expanded form only has in FP64.  Types without such a form (cos, tanh,
// exp) use cutoffFdf.
__device__ __forceinline__ void cutoffFdfF32(DevCutoff const& c, float r, float& fc, float& dfc)
{
    if (c.type >= 5 && c.type <= 8)
    {
        if (r >= c.rcF)
        {
            fc = 0.0f;
            dfc = 0.0f;
            return;
        }
        if (r < c.rciF)
        {
            fc = 1.0f;
            dfc = 0.0f;
            return;
        }
        const float x = (r - c.rciF) * c.iwF, u = (c.rcF - r) * c.iwF;
        const float xu = x * u, u2 = u * u;
        float p, d;
        switch (c.type)
        {
        case 5: p = u2 * (1.0f + 2.0f * x); d = -6.0f * xu; break;
        case 6: p = u2 * u * ((6.0f * x + 3.0f) * x + 1.0f); d = -30.0f * xu * xu; break;
        case 7: p = u2 * u2 * (((20.0f * x + 10.0f) * x + 4.0f) * x + 1.0f); d = -140.0f * xu * xu * xu; break;
        default:
            p = u2 * u2 * u * ((((70.0f * x + 35.0f) * x + 15.0f) * x + 5.0f) * x + 1.0f);
            d = -630.0f * (xu * xu) * (xu * xu);
            break;
        }
        fc = p;
        dfc = d * c.iwF;
        return;
    }
    if (c.type == 0)
    {
        fc = r < c.rcF ? 1.0f : 0.0f;
        dfc = 0.0f;
        return;
    }
    double f, df;
    cutoffFdf(c, (double)r, f, df);
    fc = (float)f;
    dfc = (float)df;
}

// The poly2 cutoff (type 6) without the type dispatch, for kernels
// instantiated per cutoff type: FP64 with the arithmetic of cutoffFdf, FP32
// with that of cutoffFdfF32; the values below r_ci (1, 0) and from r_c on
// (0, 0) are chosen by selects instead of branches.
__device__ __forceinline__ void cutoffPoly2(DevCutoff const& c, double r, double& fc, double& dfc)
{
    const double x = (r - c.rci) * c.iw;
    const double x2 = x * x;
    const double fx = ((15.0 - 6.0 * x) * x - 10.0) * x * x2 + 1.0;
    const double dfx = x2 * ((60.0 - 30.0 * x) * x - 30.0);
    const bool in = r < c.rc, inner = r < c.rci;
    fc = in ? (inner ? 1.0 : fx) : 0.0;
    dfc = (in && !inner) ? dfx * c.iw : 0.0;
}

__device__ __forceinline__ void cutoffPoly2(DevCutoff const& c, float r, float& fc, float& dfc)
{
    const float x = (r - c.rciF) * c.iwF, u = (c.rcF - r) * c.iwF;
    const float xu = x * u, u2 = u * u;
    const float p = u2 * u * ((6.0f * x + 3.0f) * x + 1.0f);
    const float d = -30.0f * xu * xu;
    const bool in = r < c.rcF, inner = r < c.rciF;
    fc = in ? (inner ? 1.0f : p) : 0.0f;
    dfc = (in && !inner) ? d * c.iwF : 0.0f;
}

// SymFnc::scale (SymFnc.cpp:169-195)
__device__ __forceinline__ double scaleG(DevScaling const& s, double v)
{
    switch (s.type)
    {
    case 0: return v;
    case 1: return s.Smin + s.scalingFactor * (v - s.Gmin);
    case 2: return v - s.Gmean;
    case 3:
    case 4: return s.Smin + s.scalingFactor * (v - s.Gmean);
    }
    return 0.0;
}

// SymFnc::unscale (SymFnc.cpp:197-223)
__device__ __forceinline__ double unscaleG(DevScaling const& s, double v)
{
    switch (s.type)
    {
    case 0: return v;
    case 1: return (v - s.Smin) / s.scalingFactor + s.Gmin;
    case 2: return v + s.Gmean;
    case 3:
    case 4: return (v - s.Smin) / s.scalingFactor + s.Gmean;
    }
    return 0.0;
}

} // namespace n2p2b200
