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
