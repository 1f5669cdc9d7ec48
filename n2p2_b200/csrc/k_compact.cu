// Compact symmetry functions on sm_100a, values and the force pass, for all
// six compact types:
//   20 radial                   SymGrpCompRad.cpp:130-245
//   21 angular narrow           SymGrpCompAngn.cpp:146-410
//   22 angular wide             SymGrpCompAngw.cpp:134-366
//   23 radial weighted          SymGrpCompRadWeighted.cpp:122-205
//   24 angular narrow weighted  SymGrpCompAngnWeighted.cpp:135-393
//   25 angular wide weighted    SymGrpCompAngwWeighted.cpp:120-351
// The weighted types take every neighbour, weighted by its atomic number
// (the product of both for an angle); the narrow types also need the j-k
// distance inside the radial window and multiply by its radial function.
//
// One warp per atom, neighbour data read from the entry arrays.  The G pass
// sums every member over the neighbours (radial) or the unordered pairs
// (j < k, angular) lane by lane and combines the lanes by a fixed shuffle
// tree.  The force pass gives every lane its own neighbours: for entry j it
// adds the force E_i puts on j over all partners k (each pair is evaluated
// from both ends, with j in the role of the first neighbour) and its half of
// the self force; it runs after the Gaussian force pass and adds to that
// pass's per-entry forces h and self forces.  No atomics; the same result on
// every run.
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

__device__ __forceinline__ void radialFdf(DevCompactMember const& M, double r, double& f, double& df)
{
    compactFdf(M.core, M.asym, M.rCenter, M.rScale, r, f, df);
}

// Radial part of a neighbour for a member: 0 outside (rl, rc)
// (SymGrpCompAngn.cpp:175-197).
__device__ __forceinline__ double windowRadial(DevCompactMember const& M, double r, double& df)
{
    double f = 0.0;
    df = 0.0;
    if (r > M.rl && r < M.rc) radialFdf(M, r, f, df);
    return f;
}

// Angle of the pair (j, k) seen from the centre; false when cos is +-1 (the
// reference skips those pairs: the compact angular functions vanish there).
struct PairGeom
{
    double cost, acost, dacost, rinvij, rinvik, rinvijik, phiijik0, phiikij0;
    double dr30, dr31, dr32;
    double rjk, rinvjk;   // narrow types only
};

// The j-k distance test of the narrow groups (SymGrpCompAngn.cpp:218-226):
// false when it is outside the group's window.
__device__ __forceinline__ bool pairDistance(DevCompactGroup const& G, double x1, double y1, double z1, double x2,
                                             double y2, double z2, PairGeom& p)
{
    const double a = x2 - x1, b = y2 - y1, c = z2 - z1;
    const double r2 = a * a + b * b + c * c;
    if (r2 >= G.rmax * G.rmax || r2 <= G.rmin * G.rmin) return false;
    p.rjk = sqrt(r2);
    p.rinvjk = 1.0 / p.rjk;
    return true;
}

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

// Member break conditions of the angular groups (SymGrpCompAngn.cpp:263-272,
// SymGrpCompAngw.cpp:230-236): radFirst is the first neighbour's radial part
// (0 outside its window), rSecond the second neighbour's distance.
__device__ __forceinline__ bool memberSkipped(DevCompactMember const& M, bool narrow, double radFirst, double rSecond,
                                              PairGeom const& p)
{
    return radFirst == 0.0 || rSecond <= M.rl || rSecond >= M.rc ||
           (narrow && (p.rjk <= M.rl || p.rjk >= M.rc)) || p.acost <= M.aLeft || p.acost >= M.aRight;
}

// The narrow groups compute the j-k radial part only for the first member of
// a run of equal radial boundaries, or after a skipped member, and otherwise
// carry the last value forward (calculateComp, SymGrpCompAngn.cpp:253-296).
struct JkCarry
{
    double rad = 0.0, drad = 0.0;
    bool skip = false;
};

__device__ __forceinline__ void carryStep(DevCompactMember const& M, double rjk, JkCarry& c)
{
    if (M.calcComp || c.skip)
    {
        radialFdf(M, rjk, c.rad, c.drad);
        c.skip = false;
    }
}

// The carry entering member m0 of a pair, replayed from the last member
// before it that recomputes (member 0 always does).
__device__ __forceinline__ JkCarry carryBefore(const DevCompactMember* mem, int m0, double rFirst, double rSecond,
                                               PairGeom const& p)
{
    JkCarry c;
    if (m0 == 0 || mem[m0].calcComp) return c;
    int s = m0 - 1;
    while (s > 0 && !mem[s].calcComp) --s;
    for (int l = s; l < m0; ++l)
    {
        DevCompactMember const& M = mem[l];
        double df;
        if (memberSkipped(M, true, windowRadial(M, rFirst, df), rSecond, p))
        {
            c.skip = true;
            continue;
        }
        carryStep(M, p.rjk, c);
    }
    return c;
}

// G pass of one chunk of radial members (types 20, 23) over the lane's
// neighbours.
template <bool WEIGHTED>
__device__ __forceinline__ void radialChunk(DevModel const& model, BatchView const& b, DevCompactGroup const& G,
                                            const DevCompactMember* mem, int mc, int64_t off, int n, int lane,
                                            double (&acc)[kCompactChunk])
{
    for (int s = lane; s < n; s += 32)
    {
        const int64_t e = off + s;
        const int el = b.nbrElem[e];
        const double d = b.nbrD[e];
        if (!(WEIGHTED || el == G.e1) || !(d < G.rmax && d > G.rmin)) continue;
#pragma unroll
        for (int q = 0; q < kCompactChunk; ++q)
        {
            DevCompactMember const& M = mem[q];
            if (q < mc && d > M.rl && d < M.rc)
            {
                double f, df;
                radialFdf(M, d, f, df);
                acc[q] += WEIGHTED ? model.atomicNumber[el] * f : f;
            }
        }
    }
}

// G pass of one chunk of angular members (types 21, 22, 24, 25) over the
// lane's unordered neighbour pairs (j < k).
template <bool NARROW, bool WEIGHTED>
__device__ __forceinline__ void angularChunk(DevModel const& model, BatchView const& b, DevCompactGroup const& G,
                                             const DevCompactMember* mem, int m0, int mc, int64_t off, int n,
                                             int lane, double (&acc)[kCompactChunk])
{
    const DevCompactMember* cm = mem + m0;
    for (int sj = lane; sj < n - 1; sj += 32)
    {
        const int64_t ej = off + sj;
        const int elj = b.nbrElem[ej];
        const double rij = b.nbrD[ej];
        if (!((WEIGHTED || G.e1 == elj || G.e2 == elj) && rij < G.rmax && rij > G.rmin)) continue;
        const double x1 = b.nbrDx[ej], y1 = b.nbrDy[ej], z1 = b.nbrDz[ej];
        double radij[kCompactChunk];
#pragma unroll
        for (int q = 0; q < kCompactChunk; ++q)
        {
            double df;
            radij[q] = q < mc ? windowRadial(cm[q], rij, df) : 0.0;
        }
        for (int sk = sj + 1; sk < n; ++sk)
        {
            const int64_t ek = off + sk;
            const int elk = b.nbrElem[ek];
            if (!(WEIGHTED || (G.e1 == elj && G.e2 == elk) || (G.e2 == elj && G.e1 == elk))) continue;
            const double rik = b.nbrD[ek];
            if (!(rik < G.rmax && rik > G.rmin)) continue;
            const double x2 = b.nbrDx[ek], y2 = b.nbrDy[ek], z2 = b.nbrDz[ek];
            PairGeom p;
            if (NARROW && !pairDistance(G, x1, y1, z1, x2, y2, z2, p)) continue;
            if (!pairGeometry(rij, rik, x1, y1, z1, x2, y2, z2, false, p)) continue;
            double z = 1.0;
            if (WEIGHTED) z = model.atomicNumber[elj] * model.atomicNumber[elk];
            JkCarry carry;
            if (NARROW) carry = carryBefore(mem, m0, rij, rik, p);
#pragma unroll
            for (int q = 0; q < kCompactChunk; ++q)
            {
                if (q < mc)
                {
                    DevCompactMember const& M = cm[q];
                    if (memberSkipped(M, NARROW, radij[q], rik, p))
                    {
                        carry.skip = true;
                    }
                    else
                    {
                        double radik, dradik, ang, dang;
                        radialFdf(M, rik, radik, dradik);
                        if (NARROW) carryStep(M, p.rjk, carry);
                        compactFdf(M.core, 0, M.aCenter, M.aScale, p.acost, ang, dang);
                        if (WEIGHTED) ang *= z;
                        const double rad = NARROW ? radij[q] * radik * carry.rad : radij[q] * radik;
                        acc[q] += rad * ang;
                    }
                }
            }
        }
    }
}

// One launch per compact type present: every warp walks its atoms' groups of
// type TYPE only, so each type's kernel holds only its own state.
template <int TYPE>
__global__ void __launch_bounds__(128, 2) kCompactValues(DevModel model, BatchView b)
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
            if (G.type != TYPE) continue;
            const DevCompactMember* mem = model.compactMembers + G.memberBegin;
            for (int m0 = 0; m0 < G.memberCount; m0 += kCompactChunk)
            {
                const int mc = min(kCompactChunk, G.memberCount - m0);
                double acc[kCompactChunk];
#pragma unroll
                for (int q = 0; q < kCompactChunk; ++q) acc[q] = 0.0;
                if (TYPE == 20 || TYPE == 23)
                    radialChunk<TYPE == 23>(model, b, G, mem + m0, mc, off, n, lane, acc);
                else
                    angularChunk<TYPE == 21 || TYPE == 24, TYPE >= 24>(model, b, G, mem, m0, mc, off, n, lane, acc);
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

struct ForceAcc
{
    double hx = 0.0, hy = 0.0, hz = 0.0;   // force E_i puts on the lane's neighbour j
    double sx = 0.0, sy = 0.0, sz = 0.0;   // the lane's share of the self force
};

// Force pass of a radial group (types 20, 23) for neighbour j: p1 =
// scalingFactor drad / rij (SymGrpCompRad.cpp:176), times the atomic number
// for the weighted type (SymGrpCompRadWeighted.cpp:163).
template <bool WEIGHTED>
__device__ __forceinline__ void radialForces(DevModel const& model, DevElement const& E, DevCompactGroup const& G,
                                             const DevCompactMember* mem, const double* dEdG, int elj, double rij,
                                             double x1, double y1, double z1, ForceAcc& a)
{
    if (!(WEIGHTED || elj == G.e1) || !(rij < G.rmax && rij > G.rmin)) return;
    for (int q = 0; q < G.memberCount; ++q)
    {
        DevCompactMember const& M = mem[q];
        if (!(rij > M.rl && rij < M.rc)) continue;
        double f, df;
        radialFdf(M, rij, f, df);
        const double sfac = model.scaling[E.sfBegin + M.sf].scalingFactor;
        const double c = dEdG[M.sf] * (df * ((WEIGHTED ? model.atomicNumber[elj] * sfac : sfac) / rij));
        a.hx += c * x1;
        a.hy += c * y1;
        a.hz += c * z1;
        a.sx -= c * x1;
        a.sy -= c * y1;
        a.sz -= c * z1;
    }
}

// Force pass of an angular group (types 21, 22, 24, 25) for neighbour j over
// all partners k, with j in the role of the first neighbour
// (SymGrpCompAngn.cpp:298-338, SymGrpCompAngw.cpp:265-299).
template <bool NARROW, bool WEIGHTED>
__device__ __forceinline__ void angularForces(DevModel const& model, BatchView const& b, DevElement const& E,
                                              DevCompactGroup const& G, const DevCompactMember* mem,
                                              const double* dEdG, int64_t off, int n, int sj, int elj, double rij,
                                              double x1, double y1, double z1, ForceAcc& a)
{
    if (!((WEIGHTED || G.e1 == elj || G.e2 == elj) && rij < G.rmax && rij > G.rmin)) return;
    for (int sk = 0; sk < n; ++sk)
    {
        if (sk == sj) continue;
        const int64_t ek = off + sk;
        const int elk = b.nbrElem[ek];
        if (!(WEIGHTED || (G.e1 == elj && G.e2 == elk) || (G.e2 == elj && G.e1 == elk))) continue;
        const double rik = b.nbrD[ek];
        if (!(rik < G.rmax && rik > G.rmin)) continue;
        const double x2 = b.nbrDx[ek], y2 = b.nbrDy[ek], z2 = b.nbrDz[ek];
        PairGeom p;
        if (NARROW && !pairDistance(G, x1, y1, z1, x2, y2, z2, p)) continue;
        if (!pairGeometry(rij, rik, x1, y1, z1, x2, y2, z2, true, p)) continue;
        double z = 1.0;
        if (WEIGHTED) z = model.atomicNumber[elj] * model.atomicNumber[elk];
        // the reference visits the pair with the lower neighbour index first: its break test
        // reads that neighbour's radial value
        const bool ownFirst = sj < sk;
        JkCarry carry;
        for (int q = 0; q < G.memberCount; ++q)
        {
            DevCompactMember const& M = mem[q];
            // windows first; then the first neighbour's radial value must not vanish
            if (!(rij > M.rl && rij < M.rc) || !(rik > M.rl && rik < M.rc) ||
                (NARROW && (p.rjk <= M.rl || p.rjk >= M.rc)) || p.acost <= M.aLeft || p.acost >= M.aRight)
            {
                carry.skip = true;
                continue;
            }
            double radij, dradij, radik, dradik;
            radialFdf(M, rij, radij, dradij);
            radialFdf(M, rik, radik, dradik);
            if ((ownFirst ? radij : radik) == 0.0)
            {
                carry.skip = true;
                continue;
            }
            if (NARROW) carryStep(M, p.rjk, carry);
            double ang, dang;
            compactFdf(M.core, 0, M.aCenter, M.aScale, p.acost, ang, dang);
            if (WEIGHTED) ang *= z;
            const double sfac = model.scaling[E.sfBegin + M.sf].scalingFactor;
            double rad = NARROW ? radij * radik * carry.rad : radij * radik;
            dang *= p.dacost;
            const double phiijik = p.phiijik0 * dang;
            const double psiijik = p.rinvijik * dang;
            const double chiij = NARROW ? p.rinvij * dradij * radik * carry.rad : p.rinvij * radik * dradij;
            const double chijk = NARROW ? -p.rinvjk * radij * radik * carry.drad : 0.0;
            double p1, p3;
            if (dang != 0.0 && rad != 0.0)
            {
                rad *= sfac * z;
                ang *= sfac;
                p1 = rad * phiijik + ang * chiij;
                p3 = NARROW ? rad * psiijik + ang * chijk : rad * psiijik;
            }
            else if (ang != 0.0)
            {
                ang *= sfac;
                p1 = ang * chiij;
                p3 = NARROW ? ang * chijk : 0.0;
            }
            else continue;
            // j: -dE/dr_j = dE/dG (p1 dr_ij + p3 dr_jk); the centre's share: -dE/dG p1 dr_ij
            const double w = dEdG[M.sf];
            a.hx += w * (p1 * x1 + p3 * p.dr30);
            a.hy += w * (p1 * y1 + p3 * p.dr31);
            a.hz += w * (p1 * z1 + p3 * p.dr32);
            a.sx -= w * p1 * x1;
            a.sy -= w * p1 * y1;
            a.sz -= w * p1 * z1;
        }
    }
}

// One launch per compact type present, in type order after the Gaussian
// force pass; each adds its share to the per-entry and self forces.
template <int TYPE>
__global__ void __launch_bounds__(128, 2) kCompactForces(DevModel model, BatchView b)
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
        ForceAcc a;
        for (int sj = lane; sj < n; sj += 32)
        {
            const int64_t ej = off + sj;
            const int elj = b.nbrElem[ej];
            const double rij = b.nbrD[ej];
            const double x1 = b.nbrDx[ej], y1 = b.nbrDy[ej], z1 = b.nbrDz[ej];
            a.hx = a.hy = a.hz = 0.0;
            for (int g = 0; g < E.compactCount; ++g)
            {
                DevCompactGroup const G = model.compactGroups[E.compactBegin + g];
                if (G.type != TYPE) continue;
                const DevCompactMember* mem = model.compactMembers + G.memberBegin;
                if (TYPE == 20 || TYPE == 23)
                    radialForces<TYPE == 23>(model, E, G, mem, dEdG, elj, rij, x1, y1, z1, a);
                else
                    angularForces<TYPE == 21 || TYPE == 24, TYPE >= 24>(model, b, E, G, mem, dEdG, off, n, sj, elj,
                                                                        rij, x1, y1, z1, a);
            }
            if (a.hx != 0.0 || a.hy != 0.0 || a.hz != 0.0)
            {
                b.hx[ej] += a.hx;
                b.hy[ej] += a.hy;
                b.hz[ej] += a.hz;
            }
        }
        const double sx = warpSum(a.sx);
        const double sy = warpSum(a.sy);
        const double sz = warpSum(a.sz);
        if (lane == 0 && (sx != 0.0 || sy != 0.0 || sz != 0.0))
        {
            b.fSelf[3 * (size_t)i + 0] += sx;
            b.fSelf[3 * (size_t)i + 1] += sy;
            b.fSelf[3 * (size_t)i + 2] += sz;
        }
    }
}

} // namespace

namespace {

int compactBlocks(BatchView const& b, int sms)
{
    int blocks = (b.N + 3) / 4;
    if (blocks < 1) blocks = 1;
    if (blocks > sms * 16) blocks = sms * 16;
    return blocks;
}

} // namespace

void launchCompactValues(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    const int blocks = compactBlocks(b, sms);
    if (m.compactTypes & (1 << 0)) kCompactValues<20><<<blocks, 128, 0, st>>>(m, b);
    if (m.compactTypes & (1 << 1)) kCompactValues<21><<<blocks, 128, 0, st>>>(m, b);
    if (m.compactTypes & (1 << 2)) kCompactValues<22><<<blocks, 128, 0, st>>>(m, b);
    if (m.compactTypes & (1 << 3)) kCompactValues<23><<<blocks, 128, 0, st>>>(m, b);
    if (m.compactTypes & (1 << 4)) kCompactValues<24><<<blocks, 128, 0, st>>>(m, b);
    if (m.compactTypes & (1 << 5)) kCompactValues<25><<<blocks, 128, 0, st>>>(m, b);
}

void launchCompactForces(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    const int blocks = compactBlocks(b, sms);
    if (m.compactTypes & (1 << 0)) kCompactForces<20><<<blocks, 128, 0, st>>>(m, b);
    if (m.compactTypes & (1 << 1)) kCompactForces<21><<<blocks, 128, 0, st>>>(m, b);
    if (m.compactTypes & (1 << 2)) kCompactForces<22><<<blocks, 128, 0, st>>>(m, b);
    if (m.compactTypes & (1 << 3)) kCompactForces<23><<<blocks, 128, 0, st>>>(m, b);
    if (m.compactTypes & (1 << 4)) kCompactForces<24><<<blocks, 128, 0, st>>>(m, b);
    if (m.compactTypes & (1 << 5)) kCompactForces<25><<<blocks, 128, 0, st>>>(m, b);
}

} // namespace n2p2b200
