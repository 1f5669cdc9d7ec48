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
// Two kernel families, one launch per type present, after the Gaussian
// passes (adding to their G, per-entry forces h and self forces):
//  * staged angular kernels (kCompactWide*, below): one block per atom with
//    at most kWideCap neighbours, the members factored into a grid of
//    distinct radial x angular parts;
//  * direct kernels (kCompactValues / kCompactForces): the radial types and
//    the atoms with more neighbours.  One warp per atom over the entry
//    arrays; the G pass sums every member over the neighbours (radial) or
//    the unordered pairs (j < k, angular) lane by lane and combines the
//    lanes by a fixed shuffle tree; the force pass gives every lane its own
//    entries j and adds the force E_i puts on j over all partners k (each
//    pair evaluated from both ends, with j in the role of the first
//    neighbour) and its half of the self force.
// No atomics; the same result on every run.
#include <algorithm>

#include "kernels.hpp"
#include "kernels_common.cuh"
#include "pair_rounds.cuh"

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
__global__ void __launch_bounds__(128, 2) kCompactValues(DevModel model, BatchView b, int minNeighbors)
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
        if (n <= minNeighbors) continue;   // staged by the wide-angular kernels
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
__global__ void __launch_bounds__(128, 2) kCompactForces(DevModel model, BatchView b, int minNeighbors)
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
        if (n <= minNeighbors) continue;   // staged by the wide-angular kernels
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

// ---------------------------------------------------------------------------
// Wide angular types (22, 25) on staged neighbours, one block per atom.
//
// The members of an angular group factor into a grid: a member's term for a
// pair (j, k) is f_r(r_ij) f_r(r_ik) f_a(theta_ijk), with f_r one of the
// group's nR distinct radial parts and f_a one of its nA distinct angular
// parts (DevCompactFn).  A part is 0, with derivative 0, outside its open
// window, which is what the reference's window skips amount to
// (SymGrpCompAngw.cpp:230-236, SymGrpCompAngwWeighted.cpp:211-218); the one
// skip that is not a window test, the first neighbour's radial value being
// exactly 0, zeroes that neighbour's radial derivative in the force pass.
//   G pass: S[r][a] = sum over pairs of f_r(r_ij) f_r(r_ik) f_a(theta)
//           (times Z_j Z_k for type 25); each member reads its cell.
//   force:  W[r][a] = sum of dE/dG scalingFactor over the cell's members; per
//           pair U_r = sum_a W[r][a] f_a, V_r = sum_a W[r][a] f_a',
//           B_j = sum_r f_r'(r_ij) f_r(r_ik) U_r (B_k likewise), and
//           C = dtheta/dcos sum_r f_r(r_ij) f_r(r_ik) V_r; with d = r_i - r_j
//           the force on j is h_j = (B_j / r_ij - C cos / r_ij^2) d_j +
//           C / (r_ij r_ik) d_k (and j <-> k), and the centre's is -sum_j h_j.
// The atom's neighbours are staged sorted by element (stable), so a group's
// pairs are the rounds of matchings of one element block (tournament) or of
// two blocks (diagonals); the radial parts of the group's neighbours are
// staged per group.  Each warp takes batches of 32 consecutive pairs.  In
// the G pass a batch is a k = 32 slice of the product S = P^T A, P the
// pairs' radial products f_r f_r (32 x nR) and A their angular parts
// (32 x nA), run on the FP64 tensor cores (mma m8n8k4, FP64 accumulation)
// from a per-warp shared tile; the force pass adds a batch round by round to
// the warp's own force array, so no slot is written twice at once.  Every
// sum runs in a fixed order.
constexpr int kWideRows = kCompactStageRows;   // radial parts per chunk
constexpr int kWideCols = kCompactStageCols;   // angular parts per chunk
constexpr int kWideCap = 256;   // staged neighbours; atoms with more run the direct kernels
constexpr int kWideWarps = 4;
constexpr int kCellStride = 8;  // G pass cell sums: row r, column a at r * 8 + a
constexpr int kTileStride = 36; // per-warp tile: 32 pairs per row, padded against bank conflicts

// G-pass tile rows: the grid's, and for the narrow types one more per impure
// member (kWideRows + kCompactImpure = 16, the two 8-row halves of the mma).
template <bool NARROW>
__host__ __device__ constexpr int tileRows() { return NARROW ? 16 : kWideRows; }
template <bool NARROW>
__host__ __device__ constexpr int tileDoubles() { return (tileRows<NARROW>() + kWideCols) * kTileStride; }
template <bool NARROW>
__host__ __device__ constexpr int cellCount() { return tileRows<NARROW>() * kCellStride; }
static_assert(kWideRows + kCompactImpure <= 16, "impure rows beyond the mma halves");
static_assert(kWideCols <= kCellStride && kWideCols <= 8, "angular parts beyond the mma's 8 columns");

// Value and derivative of a radial part at r (0 outside the open window):
// CompactFunction::fdf with the part's core and asymmetry.
__device__ __forceinline__ void compactPartFdf(DevCompactFn const& f, double x, double& v, double& dv)
{
    v = 0.0;
    dv = 0.0;
    if (x > f.left && x < f.right) compactFdf(f.core, f.asym, f.center, f.scale, x, v, dv);
}

// The same for an angular part (symmetric core), the core fixed at compile
// time when ACORE != 0 (every angular part of the model has that core).
template <int ACORE>
__device__ __forceinline__ void angularPartFdf(DevCompactFn const& f, double x, double& v, double& dv)
{
    v = 0.0;
    dv = 0.0;
    if (x > f.left && x < f.right)
    {
        const double u = (x - f.center) * f.scale;
        double fx, dfx;
        coreFdf(ACORE != 0 ? ACORE : f.core, fabs(u), fx, dfx);
        v = fx;
        dv = dfx * copysign(f.scale, u);
    }
}

// D = A B + D for one 8 x 4 by 4 x 8 FP64 block (mma.sync m8n8k4): lane l
// holds A[l / 4][l % 4], B[l % 4][l / 4] and D[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void mmaF64(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// The block's shared memory: per staged slot the neighbour's d = r_i - r_j,
// r, 1/r, element and list position; the group chunk's parts and radial
// values (and derivatives); the G pass's per-warp tiles and cell sums, the
// force pass's per-warp force arrays and cell weights.
struct WideSmem
{
    double *x, *y, *z, *r, *rinv;   // [kWideCap]
    double *rad, *drad;             // [rows][kWideCap] radial values (and derivatives, force pass)
    double *h;                      // force pass: [warps][3][kWideCap]
    double *tile;                   // G pass: [warps][tile rows + kWideCols][kTileStride]
    double *cell;                   // G pass: [warps][tile rows * kCellStride] sums; force pass: W [kWideRows][kWideCols]
    double *walkW;                  // force pass: [kCompactWalk] weights of the replayed impure members
    DevCompactFn* fn;               // [kWideRows + kWideCols]: radial parts, then angular parts
    int* walk;                      // [kCompactWalk][4]: replayed members' rIdx, aIdx, calcComp, impure
    int* blockBegin;                // [kDevMaxElements + 1]
    short* perm;                    // [kWideCap] slot -> position in the atom's list
    unsigned char* el;              // [kWideCap]
};

__host__ __device__ inline size_t wideDoubles(int rows, int warps, bool forces, bool narrow)
{
    const size_t tile = narrow ? tileDoubles<true>() + cellCount<true>() : tileDoubles<false>() + cellCount<false>();
    return 5 * kWideCap + (size_t)rows * kWideCap * (forces ? 2 : 1) +
           (forces ? (size_t)warps * 3 * kWideCap + kWideRows * kWideCols + kCompactWalk : (size_t)warps * tile);
}

__host__ __device__ inline size_t wideSmemBytes(int rows, int warps, bool forces, bool narrow)
{
    return wideDoubles(rows, warps, forces, narrow) * sizeof(double) + (kWideRows + kWideCols) * sizeof(DevCompactFn) +
           (4 * kCompactWalk + kDevMaxElements + 1) * sizeof(int) + kWideCap * sizeof(short) + kWideCap;
}

__device__ __forceinline__ WideSmem wideCarve(char* base, int rows, int warps, bool forces, bool narrow)
{
    WideSmem S;
    double* d = reinterpret_cast<double*>(base);
    S.x = d;
    S.y = d + kWideCap;
    S.z = d + 2 * kWideCap;
    S.r = d + 3 * kWideCap;
    S.rinv = d + 4 * kWideCap;
    d += 5 * kWideCap;
    S.rad = d;
    d += rows * kWideCap;
    S.drad = S.h = S.tile = S.walkW = nullptr;
    if (forces)
    {
        S.drad = d;
        d += rows * kWideCap;
        S.h = d;
        d += warps * 3 * kWideCap;
        S.cell = d;
        d += kWideRows * kWideCols;
        S.walkW = d;
        d += kCompactWalk;
    }
    else
    {
        S.tile = d;
        d += warps * (narrow ? tileDoubles<true>() : tileDoubles<false>());
        S.cell = d;
        d += warps * (narrow ? cellCount<true>() : cellCount<false>());
    }
    S.fn = reinterpret_cast<DevCompactFn*>(d);
    S.walk = reinterpret_cast<int*>(S.fn + kWideRows + kWideCols);
    S.blockBegin = S.walk + 4 * kCompactWalk;
    S.perm = reinterpret_cast<short*>(S.blockBegin + kDevMaxElements + 1);
    S.el = reinterpret_cast<unsigned char*>(S.perm + kWideCap);
    return S;
}

// Stage the atom's n <= kWideCap neighbours sorted by element (stable).
__device__ void wideStage(WideSmem const& S, DevModel const& model, BatchView const& b, int64_t off, int n, int tid,
                          int threads)
{
    if (tid < 32)
    {
        const int lane = tid;
        const int ne = model.numElements;
        int count = 0;   // lane k < ne: entries of element k
        for (int c = 0; c < n; c += 32)
        {
            const int e = c + lane < n ? (int)b.nbrElem[off + c + lane] : -1;
            for (int k = 0; k < ne; ++k)
            {
                const int cnt = __popc(__ballot_sync(kFullMask, e == k));
                if (lane == k) count += cnt;
            }
        }
        int incl = count;
        for (int o = 1; o < 32; o <<= 1)
        {
            const int t = __shfl_up_sync(kFullMask, incl, o);
            if (lane >= o) incl += t;
        }
        int begin = incl - count;   // lane k <= ne: first slot of element k (lane ne: n)
        if (lane <= ne) S.blockBegin[lane] = begin;
        const unsigned below = (1u << lane) - 1u;
        for (int c = 0; c < n; c += 32)
        {
            const int e = c + lane < n ? (int)b.nbrElem[off + c + lane] : -1;
            for (int k = 0; k < ne; ++k)
            {
                const unsigned mask = __ballot_sync(kFullMask, e == k);
                const int bk = __shfl_sync(kFullMask, begin, k);
                if (e == k) S.perm[bk + __popc(mask & below)] = (short)(c + lane);
                if (lane == k) begin += __popc(mask);
            }
        }
    }
    __syncthreads();
    for (int s = tid; s < n; s += threads)
    {
        const int64_t e = off + S.perm[s];
        const double d = b.nbrD[e];
        S.x[s] = b.nbrDx[e];
        S.y[s] = b.nbrDy[e];
        S.z[s] = b.nbrDz[e];
        S.r[s] = d;
        S.rinv[s] = 1.0 / d;
        S.el[s] = b.nbrElem[e];
    }
    __syncthreads();
}

// A group's pairs: the neighbours of its element pair (all neighbours for the
// weighted type) as rounds of matchings; ns slots carry its radial values.
struct WidePairs
{
    Phase ph;
    int A0, nA, B0, nB, ns;
};

template <bool WEIGHTED>
__device__ __forceinline__ WidePairs widePairs(WideSmem const& S, DevCompactGroup const& G, int n)
{
    WidePairs P;
    bool same = true;
    if (WEIGHTED)
    {
        P.A0 = 0;
        P.nA = n;
        P.B0 = 0;
        P.nB = 0;
    }
    else
    {
        P.A0 = S.blockBegin[G.e1];
        P.nA = S.blockBegin[G.e1 + 1] - P.A0;
        P.B0 = S.blockBegin[G.e2];
        P.nB = S.blockBegin[G.e2 + 1] - P.B0;
        same = G.e1 == G.e2;
        if (same) P.nB = 0;
    }
    P.ns = P.nA + P.nB;
    P.ph = Phase{3, 0, 0, 0, 0, 0, 1};
    roundPhases(P.A0, P.nA, P.B0, P.nB, same, &P.ph);
    return P;
}

// Parts of the chunk (rows r0.., columns a0..), the radial values of the
// group's slots and, for a narrow group, its replayed members.
template <bool FORCES, bool NARROW>
__device__ __forceinline__ void wideStageChunk(WideSmem const& S, DevModel const& model, DevCompactGroup const& G,
                                               WidePairs const& P, const DevCompactMember* mem, const double* dEdG,
                                               DevElement const& E, int r0, int nRc, int a0, int nAc, int tid,
                                               int threads)
{
    if (tid < nRc) S.fn[tid] = model.compactFns[G.fnBegin + r0 + tid];
    else if (tid >= kWideRows && tid < kWideRows + nAc)
        S.fn[tid] = model.compactFns[G.fnBegin + G.nR + a0 + tid - kWideRows];
    if (NARROW && tid >= 32 && tid < 32 + G.walkEnd - G.walkBegin)
    {
        const int st = tid - 32;
        DevCompactMember const& M = mem[G.walkBegin + st];
        S.walk[4 * st] = M.rIdx;
        S.walk[4 * st + 1] = M.aIdx;
        S.walk[4 * st + 2] = M.calcComp;
        S.walk[4 * st + 3] = M.impure;
        if (FORCES)
            S.walkW[st] = M.impure >= 0 ? dEdG[M.sf] * model.scaling[E.sfBegin + M.sf].scalingFactor : 0.0;
    }
    __syncthreads();
    for (int k = tid; k < nRc * P.ns; k += threads)
    {
        const int rr = k / P.ns;
        const int j = k - rr * P.ns;
        const int s = j < P.nA ? P.A0 + j : P.B0 + (j - P.nA);
        double f, df;
        compactPartFdf(S.fn[rr], S.r[s], f, df);
        S.rad[rr * kWideCap + s] = f;
        if (FORCES) S.drad[rr * kWideCap + s] = df;
    }
}

// Skip tests of the narrow members for one pair (SymGrpCompAngn.cpp:263-272):
// bit r (r < 32) when the first neighbour's radial part r is not 0 and the
// second neighbour's distance and r_jk are inside its window; bit 32 + a when
// the angle is inside angular part a's window.
__device__ __forceinline__ unsigned long long walkMasks(WideSmem const& S, int u, int v, double rjk, double acost,
                                                       int nRc, int nAc)
{
    const bool firstU = S.perm[u] < S.perm[v];
    const int s1 = firstU ? u : v, s2 = firstU ? v : u;
    const double rsec = S.r[s2];
    unsigned mR = 0u, mA = 0u;
    for (int r = 0; r < nRc; ++r)
    {
        DevCompactFn const& f = S.fn[r];
        const double r1 = S.rad[r * kWideCap + s1];
        if (r1 != 0.0 && rsec > f.left && rsec < f.right && rjk > f.left && rjk < f.right)
            mR |= 1u << r;
    }
    for (int a = 0; a < nAc; ++a)
    {
        DevCompactFn const& f = S.fn[kWideRows + a];
        if (acost > f.left && acost < f.right) mA |= 1u << a;
    }
    return ((unsigned long long)mA << 32) | mR;
}

template <int TYPE>
__device__ __forceinline__ bool hasType(DevModel const& model, DevElement const& E)
{
    for (int g = 0; g < E.compactCount; ++g)
        if (model.compactGroups[E.compactBegin + g].type == TYPE) return true;
    return false;
}

template <int TYPE, int ACORE>
__global__ void __launch_bounds__(kWideWarps * 32, 4) kCompactWideValues(DevModel model, BatchView b, int rows)
{
    constexpr bool WEIGHTED = TYPE >= 24;
    constexpr bool NARROW = TYPE == 21 || TYPE == 24;
    constexpr int T = kWideWarps * 32;
    constexpr int TR = tileRows<NARROW>();
    extern __shared__ __align__(16) char smemRaw[];
    const WideSmem S = wideCarve(smemRaw, rows, kWideWarps, false, NARROW);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* PT = S.tile + warp * tileDoubles<NARROW>();   // this warp's tile: radial products, then angular parts
    double* AT = PT + TR * kTileStride;
    double* cw = S.cell + warp * cellCount<NARROW>();
    const int g4 = lane >> 2, t4 = lane & 3;              // mma fragment row / column of the lane
    for (int i = blockIdx.x; i < b.N; i += gridDim.x)
    {
        DevElement const& E = model.el[b.elem[i]];
        if (!hasType<TYPE>(model, E)) continue;
        const int64_t off = b.nbrOffset[i];
        const int64_t end = b.nbrOffset[i + 1];
        const int n = (int)(end - off);
        if (end > b.nbrCapacity || n > kWideCap) continue;
        wideStage(S, model, b, off, n, tid, T);
        for (int g = 0; g < E.compactCount; ++g)
        {
            DevCompactGroup const G = model.compactGroups[E.compactBegin + g];
            if (G.type != TYPE) continue;
            const WidePairs P = widePairs<WEIGHTED>(S, G, n);
            const DevCompactMember* mem = model.compactMembers + G.memberBegin;
            const int q = (32 * kWideWarps) / P.ph.minor, rem = 32 * kWideWarps - q * P.ph.minor;
            const int nImp = NARROW ? G.numImpure : 0;
            const int wl = NARROW ? G.walkEnd - G.walkBegin : 0;
            for (int r0 = 0; r0 < G.nR; r0 += kWideRows)
                for (int a0 = 0; a0 < G.nA; a0 += kWideCols)
                {
                    const int nRc = min(kWideRows, G.nR - r0), nAc = min(kWideCols, G.nA - a0);
                    wideStageChunk<false, NARROW>(S, model, G, P, mem, nullptr, E, r0, nRc, a0, nAc, tid, T);
                    __syncthreads();
                    // sums of tile rows 0-7 (c0x) and 8-15 (c1x), columns 2 t4 + {0, 1}
                    double c00 = 0.0, c01 = 0.0, c10 = 0.0, c11 = 0.0;
                    Cursor cur;
                    cur.init(P.ph, 32 * warp + lane);
                    for (int p0 = 32 * warp; p0 < P.ph.count; p0 += 32 * kWideWarps, cur.advance(P.ph, q, rem))
                    {
                        int u = 0, v = 0;
                        bool ok = p0 + lane < P.ph.count && cur.slots(P.ph, u, v);
                        double cost = 0.0, rjk = 0.0;
                        if (ok)
                        {
                            if (NARROW)
                            {
                                // the narrow groups' j-k distance window (SymGrpCompAngn.cpp:218-226)
                                const double ex = S.x[v] - S.x[u], ey = S.y[v] - S.y[u], ez = S.z[v] - S.z[u];
                                const double r2 = ex * ex + ey * ey + ez * ez;
                                ok = r2 < G.rmax * G.rmax && r2 > G.rmin * G.rmin;
                                rjk = sqrt(r2);
                            }
                            cost = (S.x[u] * S.x[v] + S.y[u] * S.y[v] + S.z[u] * S.z[v]) * (S.rinv[u] * S.rinv[v]);
                            ok = ok && cost > -1.0 && cost < 1.0;
                        }
                        // this pair's column of the tile (zeros for a bye, a pair out of range or cos = +-1)
                        for (int k = 0; k < nImp; ++k) PT[(kWideRows + k) * kTileStride + lane] = 0.0;
                        if (ok)
                        {
                            const double acost = acos(cost);
                            const double zw =
                                WEIGHTED ? model.atomicNumber[S.el[u]] * model.atomicNumber[S.el[v]] : 1.0;
                            for (int a = 0; a < nAc; ++a)
                            {
                                double f, df;
                                angularPartFdf<ACORE>(S.fn[kWideRows + a], acost, f, df);
                                AT[a * kTileStride + lane] = WEIGHTED ? f * zw : f;
                            }
                            for (int r = 0; r < nRc; ++r)
                            {
                                double pr = S.rad[r * kWideCap + u] * S.rad[r * kWideCap + v];
                                if (NARROW)
                                {
                                    double fq, dfq;
                                    compactPartFdf(S.fn[r], rjk, fq, dfq);
                                    pr *= fq;
                                }
                                PT[r * kTileStride + lane] = pr;
                            }
                            if (NARROW && wl > 0)
                            {
                                // replay the carried j-k radial part for the impure members (their own rows)
                                const unsigned long long mk = walkMasks(S, u, v, rjk, acost, nRc, nAc);
                                int src = -1;
                                bool cskip = false;
                                double qs = 0.0;
                                for (int st = 0; st < wl; ++st)
                                {
                                    const int R = S.walk[4 * st], A = S.walk[4 * st + 1];
                                    if (!((mk >> R) & 1ull) || !((mk >> (32 + A)) & 1ull))
                                    {
                                        cskip = true;
                                        continue;
                                    }
                                    if (S.walk[4 * st + 2] || cskip)
                                    {
                                        if (R != src)
                                        {
                                            double dq;
                                            compactPartFdf(S.fn[R], rjk, qs, dq);
                                            src = R;
                                        }
                                        cskip = false;
                                    }
                                    const int imp = S.walk[4 * st + 3];
                                    if (imp >= 0)
                                        PT[(kWideRows + imp) * kTileStride + lane] =
                                            S.rad[R * kWideCap + u] * S.rad[R * kWideCap + v] * qs;
                                }
                            }
                        }
                        else
                        {
                            for (int a = 0; a < nAc; ++a) AT[a * kTileStride + lane] = 0.0;
                            for (int r = 0; r < nRc; ++r) PT[r * kTileStride + lane] = 0.0;
                        }
                        __syncwarp();
                        // S += P^T A over the batch's 32 pairs, 4 per step; rows and columns beyond
                        // the chunk read zeros and their sums are never used
                        const bool row0 = g4 < nRc;
                        const bool row1 = g4 + 8 < nRc || (NARROW && g4 >= 2 && g4 - 2 < nImp);
                        const bool col = g4 < nAc;
#pragma unroll
                        for (int ks = 0; ks < 8; ++ks)
                        {
                            const int k = 4 * ks + t4;
                            const double a0f = row0 ? PT[g4 * kTileStride + k] : 0.0;
                            const double a1f = row1 ? PT[(g4 + 8) * kTileStride + k] : 0.0;
                            const double bf = col ? AT[g4 * kTileStride + k] : 0.0;
                            mmaF64(c00, c01, a0f, bf);
                            mmaF64(c10, c11, a1f, bf);
                        }
                        __syncwarp();
                    }
                    cw[g4 * kCellStride + 2 * t4] = c00;
                    cw[g4 * kCellStride + 2 * t4 + 1] = c01;
                    if (g4 + 8 < TR)
                    {
                        cw[(g4 + 8) * kCellStride + 2 * t4] = c10;
                        cw[(g4 + 8) * kCellStride + 2 * t4 + 1] = c11;
                    }
                    __syncthreads();
                    for (int mi = tid; mi < G.memberCount; mi += T)
                    {
                        DevCompactMember const& M = mem[mi];
                        const int rr = M.rIdx - r0, aa = M.aIdx - a0;
                        if (rr < 0 || rr >= nRc || aa < 0 || aa >= nAc) continue;
                        // impure members (narrow groups) have rows of their own after the grid's
                        const int c = ((NARROW && M.impure >= 0) ? kWideRows + M.impure : rr) * kCellStride + aa;
                        double sum = S.cell[c];
                        for (int w = 1; w < kWideWarps; ++w) sum += S.cell[w * cellCount<NARROW>() + c];
                        b.G[(size_t)i * b.gStride + M.sf] = scaleG(model.scaling[E.sfBegin + M.sf], sum);
                    }
                    __syncthreads();
                }
        }
    }
}

template <int TYPE, int ACORE, int COLS>
__global__ void __launch_bounds__(kWideWarps * 32, 3) kCompactWideForces(DevModel model, BatchView b, int rows)
{
    constexpr bool WEIGHTED = TYPE >= 24;
    constexpr bool NARROW = TYPE == 21 || TYPE == 24;
    constexpr int T = kWideWarps * 32;
    static_assert(COLS <= kWideCols, "angular parts per chunk");
    extern __shared__ __align__(16) char smemRaw[];
    const WideSmem S = wideCarve(smemRaw, rows, kWideWarps, true, NARROW);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* hw = S.h + warp * 3 * kWideCap;   // this warp's force array
    for (int k = tid; k < kWideWarps * 3 * kWideCap; k += T) S.h[k] = 0.0;
    for (int i = blockIdx.x; i < b.N; i += gridDim.x)
    {
        DevElement const& E = model.el[b.elem[i]];
        if (!hasType<TYPE>(model, E)) continue;
        const int64_t off = b.nbrOffset[i];
        const int64_t end = b.nbrOffset[i + 1];
        const int n = (int)(end - off);
        if (end > b.nbrCapacity || n > kWideCap) continue;
        const double* dEdG = b.dEdG + (size_t)i * b.gStride;
        wideStage(S, model, b, off, n, tid, T);
        for (int g = 0; g < E.compactCount; ++g)
        {
            DevCompactGroup const G = model.compactGroups[E.compactBegin + g];
            if (G.type != TYPE) continue;
            const WidePairs P = widePairs<WEIGHTED>(S, G, n);
            if (P.ph.count == 0) continue;
            const DevCompactMember* mem = model.compactMembers + G.memberBegin;
            const int q = (32 * kWideWarps) / P.ph.minor, rem = 32 * kWideWarps - q * P.ph.minor;
            const int wl = NARROW ? G.walkEnd - G.walkBegin : 0;
            for (int r0 = 0; r0 < G.nR; r0 += kWideRows)
                for (int a0 = 0; a0 < G.nA; a0 += COLS)
                {
                    const int nRc = min(kWideRows, G.nR - r0), nAc = min(COLS, G.nA - a0);
                    wideStageChunk<true, NARROW>(S, model, G, P, mem, dEdG, E, r0, nRc, a0, nAc, tid, T);
                    // cell weights of the grid's members (the impure ones are replayed per pair), summed
                    // in member order
                    if (tid < kWideRows * COLS)
                    {
                        double w = 0.0;
                        for (int mi = 0; mi < G.memberCount; ++mi)
                        {
                            DevCompactMember const& M = mem[mi];
                            const int rr = M.rIdx - r0, aa = M.aIdx - a0;
                            if (rr < 0 || rr >= nRc || aa < 0 || aa >= nAc || rr * COLS + aa != tid) continue;
                            if (NARROW && M.impure >= 0) continue;
                            w += dEdG[M.sf] * model.scaling[E.sfBegin + M.sf].scalingFactor;
                        }
                        S.cell[tid] = w;
                    }
                    __syncthreads();
                    Cursor cur;
                    cur.init(P.ph, 32 * warp + lane);
                    for (int p0 = 32 * warp; p0 < P.ph.count; p0 += 32 * kWideWarps, cur.advance(P.ph, q, rem))
                    {
                        int u = 0, v = 0;
                        bool ok = p0 + lane < P.ph.count && cur.slots(P.ph, u, v);
                        double cu = 0.0, cv = 0.0, gm = 0.0;
                        double rjk = 0.0;
                        if (ok && NARROW)
                        {
                            const double ex = S.x[v] - S.x[u], ey = S.y[v] - S.y[u], ez = S.z[v] - S.z[u];
                            const double r2 = ex * ex + ey * ey + ez * ez;
                            ok = r2 < G.rmax * G.rmax && r2 > G.rmin * G.rmin;
                            rjk = sqrt(r2);
                        }
                        if (ok)
                        {
                            const double riu = S.rinv[u], riv = S.rinv[v];
                            const double cost = (S.x[u] * S.x[v] + S.y[u] * S.y[v] + S.z[u] * S.z[v]) * (riu * riv);
                            ok = cost > -1.0 && cost < 1.0;
                            if (ok)
                            {
                                const double acost = acos(cost);
                                const double dacost = -1.0 / sqrt(1.0 - cost * cost);
                                double ang[COLS], dang[COLS];
#pragma unroll
                                for (int a = 0; a < COLS; ++a)
                                {
                                    ang[a] = 0.0;
                                    dang[a] = 0.0;
                                    if (a < nAc) angularPartFdf<ACORE>(S.fn[kWideRows + a], acost, ang[a], dang[a]);
                                }
                                // the reference's first neighbour of the pair is the lower list index
                                const bool firstU = S.perm[u] < S.perm[v];
                                double Bu = 0.0, Bv = 0.0, Bjk = 0.0, A = 0.0;
#pragma unroll
                                for (int r = 0; r < kWideRows; ++r)
                                {
                                    if (r < nRc)
                                    {
                                        const double ru = S.rad[r * kWideCap + u], rv = S.rad[r * kWideCap + v];
                                        double dru = S.drad[r * kWideCap + u], drv = S.drad[r * kWideCap + v];
                                        if (firstU ? ru == 0.0 : rv == 0.0)
                                        {
                                            if (firstU) dru = 0.0;
                                            else drv = 0.0;
                                        }
                                        double U = 0.0, V = 0.0;
#pragma unroll
                                        for (int a = 0; a < COLS; ++a)
                                        {
                                            const double w = S.cell[r * COLS + a];
                                            U += w * ang[a];
                                            V += w * dang[a];
                                        }
                                        if (NARROW)
                                        {
                                            double fq, dfq;
                                            compactPartFdf(S.fn[r], rjk, fq, dfq);
                                            Bu += dru * rv * fq * U;
                                            Bv += ru * drv * fq * U;
                                            Bjk += ru * rv * dfq * U;
                                            A += ru * rv * fq * V;
                                        }
                                        else
                                        {
                                            Bu += dru * rv * U;
                                            Bv += ru * drv * U;
                                            A += ru * rv * V;
                                        }
                                    }
                                }
                                if (NARROW && wl > 0)
                                {
                                    // the impure members with the carried j-k radial part
                                    const unsigned long long mk = walkMasks(S, u, v, rjk, acost, nRc, nAc);
                                    int src = -1;
                                    bool cskip = false;
                                    double qs = 0.0, dqs = 0.0;
                                    for (int st = 0; st < wl; ++st)
                                    {
                                        const int R = S.walk[4 * st], Ai = S.walk[4 * st + 1];
                                        if (!((mk >> R) & 1ull) || !((mk >> (32 + Ai)) & 1ull))
                                        {
                                            cskip = true;
                                            continue;
                                        }
                                        if (S.walk[4 * st + 2] || cskip)
                                        {
                                            if (R != src)
                                            {
                                                compactPartFdf(S.fn[R], rjk, qs, dqs);
                                                src = R;
                                            }
                                            cskip = false;
                                        }
                                        if (S.walk[4 * st + 3] < 0) continue;
                                        const double w = S.walkW[st];
                                        const double ru = S.rad[R * kWideCap + u], rv = S.rad[R * kWideCap + v];
                                        const double dru = S.drad[R * kWideCap + u], drv = S.drad[R * kWideCap + v];
                                        double fa, dfa;
                                        angularPartFdf<ACORE>(S.fn[kWideRows + Ai], acost, fa, dfa);
                                        Bu += w * (dru * rv * qs * fa);
                                        Bv += w * (ru * drv * qs * fa);
                                        Bjk += w * (ru * rv * dqs * fa);
                                        A += w * (ru * rv * qs * dfa);
                                    }
                                }
                                double C = A * dacost;
                                if (WEIGHTED)
                                {
                                    const double zw = model.atomicNumber[S.el[u]] * model.atomicNumber[S.el[v]];
                                    Bu *= zw;
                                    Bv *= zw;
                                    Bjk *= zw;
                                    C *= zw;
                                }
                                // with the j-k term (narrow): h_u -= B_jk / r_jk (d_v - d_u), h_v += the same
                                const double gjk = NARROW ? Bjk / rjk : 0.0;
                                cu = Bu * riu - C * cost * riu * riu + gjk;
                                cv = Bv * riv - C * cost * riv * riv + gjk;
                                gm = C * (riu * riv) - gjk;
                            }
                        }
                        // add the batch one round at a time: inside a round no slot occurs twice
                        const int rnd = cur.a;
                        const int last = min(31, P.ph.count - 1 - p0);
                        const int rLo = __shfl_sync(kFullMask, rnd, 0);
                        const int rHi = __shfl_sync(kFullMask, rnd, last);
                        for (int rr = rLo; rr <= rHi; ++rr)
                        {
                            if (ok && rnd == rr)
                            {
                                const double xu = S.x[u], yu = S.y[u], zu = S.z[u];
                                const double xv = S.x[v], yv = S.y[v], zv = S.z[v];
                                hw[u] += cu * xu + gm * xv;
                                hw[kWideCap + u] += cu * yu + gm * yv;
                                hw[2 * kWideCap + u] += cu * zu + gm * zv;
                                hw[v] += cv * xv + gm * xu;
                                hw[kWideCap + v] += cv * yv + gm * yu;
                                hw[2 * kWideCap + v] += cv * zv + gm * zu;
                            }
                            __syncwarp();
                        }
                    }
                    __syncthreads();
                }
        }
        // per-entry forces (warp arrays summed in order) and the centre's share
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int s = tid; s < n; s += T)
        {
            double f[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
            {
                f[c] = 0.0;
                for (int w = 0; w < kWideWarps; ++w)
                {
                    f[c] += S.h[(w * 3 + c) * kWideCap + s];
                    S.h[(w * 3 + c) * kWideCap + s] = 0.0;
                }
            }
            if (f[0] != 0.0 || f[1] != 0.0 || f[2] != 0.0)
            {
                const int64_t e = off + S.perm[s];
                b.hx[e] += f[0];
                b.hy[e] += f[1];
                b.hz[e] += f[2];
            }
            sx -= f[0];
            sy -= f[1];
            sz -= f[2];
        }
        sx = warpSum(sx);
        sy = warpSum(sy);
        sz = warpSum(sz);
        if (lane == 0)
        {
            S.cell[3 * warp + 0] = sx;
            S.cell[3 * warp + 1] = sy;
            S.cell[3 * warp + 2] = sz;
        }
        __syncthreads();
        if (tid == 0)
        {
            double t[3] = {0.0, 0.0, 0.0};
            for (int w = 0; w < kWideWarps; ++w)
                for (int c = 0; c < 3; ++c) t[c] += S.cell[3 * w + c];
            if (t[0] != 0.0 || t[1] != 0.0 || t[2] != 0.0)
                for (int c = 0; c < 3; ++c) b.fSelf[3 * (size_t)i + c] += t[c];
        }
        __syncthreads();
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

// One block per atom, at most perSM resident blocks per SM.
int wideBlocks(BatchView const& b, int sms, int perSM)
{
    return std::max(1, std::min(b.N, sms * perSM));
}

} // namespace

// The staged kernel of an angular type for the atoms with at most kWideCap
// neighbours, then the direct kernel for the rest (or the direct kernel
// alone for a narrow type the staged kernels do not fit).
template <bool FORCES, int TYPE>
int launchAngular(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    constexpr bool NARROW = TYPE == 21 || TYPE == 24;
    const int blocks = compactBlocks(b, sms);
    if (NARROW && !m.compactNarrowStaged)
    {
        if (FORCES) kCompactForces<TYPE><<<blocks, 128, 0, st>>>(m, b, -1);
        else kCompactValues<TYPE><<<blocks, 128, 0, st>>>(m, b, -1);
        return 1;
    }
    const int rows = std::max(1, std::min(m.compactRows, kWideRows));
    const size_t smem = wideSmemBytes(rows, kWideWarps, FORCES, NARROW);
    auto staged = [&](auto kernel, int perSM) {
        // resident blocks: the launch bound, or fewer when the stage is larger (228 KB of shared
        // memory per SM, 1 KB of it reserved per block)
        perSM = std::max(1, std::min(perSM, (int)(233472 / (smem + 1024))));
        setDynamicSmemOnce(reinterpret_cast<const void*>(kernel), smem);
        kernel<<<wideBlocks(b, sms, perSM), kWideWarps * 32, smem, st>>>(m, b, rows);
    };
    const bool poly2 = m.compactAngCore == kCorePoly2;
    if (FORCES)
    {
        // six angular parts per chunk where the model has no more (the SCAN and QM9 groups)
        if (m.compactCols <= 6)
        {
            if (poly2) staged(kCompactWideForces<TYPE, kCorePoly2, 6>, 3);
            else staged(kCompactWideForces<TYPE, 0, 6>, 3);
        }
        else if (poly2) staged(kCompactWideForces<TYPE, kCorePoly2, kWideCols>, 3);
        else staged(kCompactWideForces<TYPE, 0, kWideCols>, 3);
        kCompactForces<TYPE><<<blocks, 128, 0, st>>>(m, b, kWideCap);
    }
    else
    {
        if (poly2) staged(kCompactWideValues<TYPE, kCorePoly2>, NARROW ? 3 : 4);
        else staged(kCompactWideValues<TYPE, 0>, NARROW ? 3 : 4);
        kCompactValues<TYPE><<<blocks, 128, 0, st>>>(m, b, kWideCap);
    }
    return 2;
}

int launchCompactValues(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    const int blocks = compactBlocks(b, sms);
    int launches = 0;
    if (m.compactTypes & (1 << 0))
    {
        kCompactValues<20><<<blocks, 128, 0, st>>>(m, b, -1);
        ++launches;
    }
    if (m.compactTypes & (1 << 1)) launches += launchAngular<false, 21>(m, b, sms, st);
    if (m.compactTypes & (1 << 2)) launches += launchAngular<false, 22>(m, b, sms, st);
    if (m.compactTypes & (1 << 3))
    {
        kCompactValues<23><<<blocks, 128, 0, st>>>(m, b, -1);
        ++launches;
    }
    if (m.compactTypes & (1 << 4)) launches += launchAngular<false, 24>(m, b, sms, st);
    if (m.compactTypes & (1 << 5)) launches += launchAngular<false, 25>(m, b, sms, st);
    return launches;
}

int launchCompactForces(DevModel const& m, BatchView const& b, int sms, cudaStream_t st)
{
    const int blocks = compactBlocks(b, sms);
    int launches = 0;
    if (m.compactTypes & (1 << 0))
    {
        kCompactForces<20><<<blocks, 128, 0, st>>>(m, b, -1);
        ++launches;
    }
    if (m.compactTypes & (1 << 1)) launches += launchAngular<true, 21>(m, b, sms, st);
    if (m.compactTypes & (1 << 2)) launches += launchAngular<true, 22>(m, b, sms, st);
    if (m.compactTypes & (1 << 3))
    {
        kCompactForces<23><<<blocks, 128, 0, st>>>(m, b, -1);
        ++launches;
    }
    if (m.compactTypes & (1 << 4)) launches += launchAngular<true, 24>(m, b, sms, st);
    if (m.compactTypes & (1 << 5)) launches += launchAngular<true, 25>(m, b, sms, st);
    return launches;
}

} // namespace n2p2b200
