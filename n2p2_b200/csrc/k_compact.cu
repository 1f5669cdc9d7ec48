// Compact symmetry functions on sm_100a: radial type 20 (SymGrpCompRad,
// SymGrpCompRad.cpp:130-245) and angular wide type 22 (SymGrpCompAngw,
// SymGrpCompAngw.cpp:134-366), values and the force pass.
//
// One warp per atom, neighbour data read from the entry arrays.  The G pass
// sums every member over the neighbours (radial) or the unordered pairs
// (j < k, angular) lane by lane and combines the lanes by a fixed shuffle
// tree.  The force pass gives every lane its own neighbours: for entry j it
// adds the force E_i puts on j over all partners k (each pair is evaluated
// from both ends, with the roles of j and k exchanged) and its half of the
// self force; it runs after the Gaussian force pass and adds to that pass's
// per-entry forces h and self forces.  No atomics; the same result on every
// run.
#include "kernels.hpp"
#include "kernels_common.cuh"

namespace n2p2b200 {

namespace {

constexpr int kCompactChunk = 8;   // members accumulated together in the G pass

// CompactFunction::fdf (CompactFunction.h:160-166) with the asymmetric core
// of CoreFunction::fdf (CoreFunction.h:189-202).  Only the radial functions
// take the asymmetric core ("p2a"): the angular function gets the core type
// alone (SymFncBaseComp::setCompactFunction, SymFncBaseCompAng.cpp:108).
__device__ __forceinline__ void compactFdf(int core, int asym, double center, double scale, double a, double& f,
                                           double& df)
{
    const double u = (a - center) * scale;
    const double x = fabs(u);
    double fx, dfx;
    if (asym)
    {
        coreFdf(core, (2.0 - x) * x, fx, dfx);
        dfx *= 2.0 - 2.0 * x;
    }
    else coreFdf(core, x, fx, dfx);
    f = fx;
    df = dfx * copysign(scale, u);
}

__device__ __forceinline__ bool pairElements(DevCompactGroup const& G, int ej, int ek)
{
    return (G.e1 == ej && G.e2 == ek) || (G.e2 == ej && G.e1 == ek);
}

// Angle of the pair (j, k) seen from the centre; false when cos is +-1 (the
// reference skips those pairs: the compact angular functions vanish there).
struct PairGeom
{
    double cost, acost, dacost, rinvij, rinvik, rinvijik, phiijik0, phiikij0;
    double dr30, dr31, dr32;
};

__device__ __forceinline__ bool pairGeometry(double rij, double rik, double x1, double y1, double z1, double x2,
                                             double y2, double z2, bool derivatives, PairGeom& p)
{
    p.dr30 = x2 - x1;
    p.dr31 = y2 - y1;
    p.dr32 = z2 - z1;
    p.rinvijik = 1.0 / (rij * rik);
    p.cost = (x1 * x2 + y1 * y2 + z1 * z2) * p.rinvijik;
    if (p.cost <= -1.0 || p.cost >= 1.0) return false;
    p.acost = acos(p.cost);
    p.rinvij = p.rinvijik * rik;
    p.rinvik = p.rinvijik * rij;
    p.phiijik0 = p.rinvij * (p.rinvik - p.rinvij * p.cost);
    p.phiikij0 = p.rinvik * (p.rinvij - p.rinvik * p.cost);
    p.dacost = derivatives ? -1.0 / sqrt(1.0 - p.cost * p.cost) : 0.0;
    return true;
}

__global__ void __launch_bounds__(128) kCompactValues(DevModel model, BatchView b)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        DevElement const& E = model.el[b.elem[i]];
        if (E.compactCount == 0) continue;
        const int64_t off = b.nbrOffset[i];
        const int64_t end = b.nbrOffset[i + 1];
        if (end > b.nbrCapacity) continue;
        const int n = (int)(end - off);
        for (int g = 0; g < E.compactCount; ++g)
        {
            DevCompactGroup const G = model.compactGroups[E.compactBegin + g];
            const DevCompactMember* mem = model.compactMembers + G.memberBegin;
            for (int m0 = 0; m0 < G.memberCount; m0 += kCompactChunk)
            {
                const int mc = min(kCompactChunk, G.memberCount - m0);
                double acc[kCompactChunk];
#pragma unroll
                for (int q = 0; q < kCompactChunk; ++q) acc[q] = 0.0;
                if (G.type == 20)
                {
                    for (int s = lane; s < n; s += 32)
                    {
                        const int64_t e = off + s;
                        if (b.nbrElem[e] != G.e1) continue;
                        const double d = b.nbrD[e];
#pragma unroll
                        for (int q = 0; q < kCompactChunk; ++q)
                        {
                            if (q >= mc) break;
                            DevCompactMember const& M = mem[m0 + q];
                            if (d > M.rl && d < M.rc)
                            {
                                double f, df;
                                compactFdf(M.core, M.asym, M.rCenter, M.rScale, d, f, df);
                                acc[q] += f;
                            }
                        }
                    }
                }
                else
                {
                    for (int sj = lane; sj < n - 1; sj += 32)
                    {
                        const int64_t ej = off + sj;
                        const int elj = b.nbrElem[ej];
                        const double rij = b.nbrD[ej];
                        if (!((G.e1 == elj || G.e2 == elj) && rij < G.rmax && rij > G.rmin)) continue;
                        const double x1 = b.nbrDx[ej], y1 = b.nbrDy[ej], z1 = b.nbrDz[ej];
                        double radij[kCompactChunk];
#pragma unroll
                        for (int q = 0; q < kCompactChunk; ++q)
                        {
                            radij[q] = 0.0;
                            if (q < mc)
                            {
                                DevCompactMember const& M = mem[m0 + q];
                                if (rij > M.rl && rij < M.rc)
                                {
                                    double df;
                                    compactFdf(M.core, M.asym, M.rCenter, M.rScale, rij, radij[q], df);
                                }
                            }
                        }
                        for (int sk = sj + 1; sk < n; ++sk)
                        {
                            const int64_t ek = off + sk;
                            if (!pairElements(G, elj, b.nbrElem[ek])) continue;
                            const double rik = b.nbrD[ek];
                            if (!(rik < G.rmax && rik > G.rmin)) continue;
                            PairGeom p;
                            if (!pairGeometry(rij, rik, x1, y1, z1, b.nbrDx[ek], b.nbrDy[ek], b.nbrDz[ek], false, p))
                                continue;
#pragma unroll
                            for (int q = 0; q < kCompactChunk; ++q)
                            {
                                if (q >= mc) break;
                                DevCompactMember const& M = mem[m0 + q];
                                if (radij[q] == 0.0 || rik <= M.rl || rik >= M.rc || p.acost <= M.aLeft ||
                                    p.acost >= M.aRight)
                                    continue;
                                double radik, dradik, ang, dang;
                                compactFdf(M.core, M.asym, M.rCenter, M.rScale, rik, radik, dradik);
                                compactFdf(M.core, 0, M.aCenter, M.aScale, p.acost, ang, dang);
                                acc[q] += radij[q] * radik * ang;
                            }
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < kCompactChunk; ++q)
                {
                    const double sum = warpSum(acc[q]);
                    if (q < mc && lane == 0)
                    {
                        const int sf = mem[m0 + q].sf;
                        b.G[(size_t)i * b.gStride + sf] = scaleG(model.scaling[E.sfBegin + sf], sum);
                    }
                }
            }
        }
    }
}

__global__ void __launch_bounds__(128) kCompactForces(DevModel model, BatchView b)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        DevElement const& E = model.el[b.elem[i]];
        if (E.compactCount == 0) continue;
        const int64_t off = b.nbrOffset[i];
        const int64_t end = b.nbrOffset[i + 1];
        if (end > b.nbrCapacity) continue;
        const int n = (int)(end - off);
        const double* dEdG = b.dEdG + (size_t)i * b.gStride;
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int sj = lane; sj < n; sj += 32)
        {
            const int64_t ej = off + sj;
            const int elj = b.nbrElem[ej];
            const double rij = b.nbrD[ej];
            const double x1 = b.nbrDx[ej], y1 = b.nbrDy[ej], z1 = b.nbrDz[ej];
            double hx = 0.0, hy = 0.0, hz = 0.0;   // force E_i puts on j
            for (int g = 0; g < E.compactCount; ++g)
            {
                DevCompactGroup const G = model.compactGroups[E.compactBegin + g];
                const DevCompactMember* mem = model.compactMembers + G.memberBegin;
                if (G.type == 20)
                {
                    if (elj != G.e1) continue;
                    for (int q = 0; q < G.memberCount; ++q)
                    {
                        DevCompactMember const& M = mem[q];
                        if (!(rij > M.rl && rij < M.rc)) continue;
                        double f, df;
                        compactFdf(M.core, M.asym, M.rCenter, M.rScale, rij, f, df);
                        // p1 = scalingFactor drad / rij (SymFncCompRad.cpp:183-190)
                        const double c = dEdG[M.sf] * (model.scaling[E.sfBegin + M.sf].scalingFactor * df / rij);
                        hx += c * x1;
                        hy += c * y1;
                        hz += c * z1;
                        sx -= c * x1;
                        sy -= c * y1;
                        sz -= c * z1;
                    }
                    continue;
                }
                if (!((G.e1 == elj || G.e2 == elj) && rij < G.rmax && rij > G.rmin)) continue;
                for (int sk = 0; sk < n; ++sk)
                {
                    if (sk == sj) continue;
                    const int64_t ek = off + sk;
                    if (!pairElements(G, elj, b.nbrElem[ek])) continue;
                    const double rik = b.nbrD[ek];
                    if (!(rik < G.rmax && rik > G.rmin)) continue;
                    PairGeom p;
                    if (!pairGeometry(rij, rik, x1, y1, z1, b.nbrDx[ek], b.nbrDy[ek], b.nbrDz[ek], true, p)) continue;
                    for (int q = 0; q < G.memberCount; ++q)
                    {
                        DevCompactMember const& M = mem[q];
                        if (!(rij > M.rl && rij < M.rc)) continue;   // radij == 0
                        if (rik <= M.rl || rik >= M.rc || p.acost <= M.aLeft || p.acost >= M.aRight) continue;
                        double radij, dradij, radik, dradik, ang, dang;
                        compactFdf(M.core, M.asym, M.rCenter, M.rScale, rij, radij, dradij);
                        if (radij == 0.0) continue;
                        compactFdf(M.core, M.asym, M.rCenter, M.rScale, rik, radik, dradik);
                        compactFdf(M.core, 0, M.aCenter, M.aScale, p.acost, ang, dang);
                        // SymGrpCompAngw.cpp:265-299, with j in the role of the first neighbour
                        const double sf = model.scaling[E.sfBegin + M.sf].scalingFactor;
                        double rad = radij * radik;
                        dang *= p.dacost;
                        const double phiijik = p.phiijik0 * dang;
                        const double psiijik = p.rinvijik * dang;
                        const double chiij = p.rinvij * radik * dradij;
                        double p1, p3;
                        if (dang != 0.0 && rad != 0.0)
                        {
                            rad *= sf;
                            ang *= sf;
                            p1 = rad * phiijik + ang * chiij;
                            p3 = rad * psiijik;
                        }
                        else if (ang != 0.0)
                        {
                            ang *= sf;
                            p1 = ang * chiij;
                            p3 = 0.0;
                        }
                        else continue;
                        // j: -dE/dr_j = dE/dG (p1 dr_ij + p3 dr_jk); the centre's share: -dE/dG p1 dr_ij
                        const double a = dEdG[M.sf];
                        hx += a * (p1 * x1 + p3 * p.dr30);
                        hy += a * (p1 * y1 + p3 * p.dr31);
                        hz += a * (p1 * z1 + p3 * p.dr32);
                        sx -= a * p1 * x1;
                        sy -= a * p1 * y1;
                        sz -= a * p1 * z1;
                    }
                }
            }
            if (hx != 0.0 || hy != 0.0 || hz != 0.0)
            {
                b.hx[ej] += hx;
                b.hy[ej] += hy;
                b.hz[ej] += hz;
            }
        }
        sx = warpSum(sx);
        sy = warpSum(sy);
        sz = warpSum(sz);
        if (lane == 0)
        {
            b.fSelf[3 * (size_t)i + 0] += sx;
            b.fSelf[3 * (size_t)i + 1] += sy;
            b.fSelf[3 * (size_t)i + 2] += sz;
        }
    }
}

} // namespace

void launchCompactValues(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    int blocks = (b.N + 3) / 4;
    if (blocks < 1) blocks = 1;
    if (blocks > sms * 16) blocks = sms * 16;
    kCompactValues<<<blocks, 128, 0, st>>>(m, b);
}

void launchCompactForces(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    int blocks = (b.N + 3) / 4;
    if (blocks < 1) blocks = 1;
    if (blocks > sms * 16) blocks = sms * 16;
    kCompactForces<<<blocks, 128, 0, st>>>(m, b);
}

} // namespace n2p2b200
