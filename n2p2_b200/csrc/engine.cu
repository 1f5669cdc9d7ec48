// Device-side engine; see engine.hpp.
#include "engine.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <unistd.h>

namespace n2p2b200 {

void cudaCheck(cudaError_t e, char const* what)
{
    if (e != cudaSuccess)
        throw std::runtime_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

void setDynamicSmemOnce(const void* kernel, size_t bytes)
{
    // per kernel and device the largest size set so far: a model that needs more raises it
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_pair(kernel, dev);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return;
    cudaCheck(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes),
              "cudaFuncSetAttribute");
    // Warp-per-atom kernels are limited by shared memory per SM: ask for the
    // largest carveout so as many blocks as the registers allow stay resident.
    cudaCheck(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100),
              "cudaFuncSetAttribute");
    done[key] = bytes;
}

// Size classes: 256-byte steps up to 64 KiB, then quarter steps between
// powers of two (at most 25 % slack).
static size_t poolBucket(size_t bytes)
{
    if (bytes <= 65536) return (bytes + 255) & ~(size_t)255;
    size_t p = 65536;
    while (p * 2 < bytes) p *= 2;
    const size_t q = p / 4;
    return ((bytes + q - 1) / q) * q;
}

DevicePool::~DevicePool() { trim(); }

void* DevicePool::get(size_t bytes)
{
    const size_t b = poolBucket(bytes);
    // the smallest cached block of at least the size class, up to twice it
    for (auto it = free_.lower_bound(b); it != free_.end() && it->first <= 2 * b; ++it)
        if (!it->second.empty())
        {
            void* p = it->second.back();
            it->second.pop_back();
            return p;
        }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        trim();
        cudaCheck(cudaMalloc(&p, b), "cudaMalloc");
    }
    size_[p] = b;
    return p;
}

void DevicePool::put(void* p)
{
    if (p) free_[size_.at(p)].push_back(p);
}

void DevicePool::trim()
{
    for (auto& kv : free_)
        for (void* p : kv.second)
        {
            cudaFree(p);
            size_.erase(p);
        }
    free_.clear();
}

namespace {

template <typename T>
T* devAlloc(DevicePool& pool, size_t count, std::vector<void*>& owned)
{
    if (count == 0) count = 1;
    void* p = pool.get(sizeof(T) * count);
    owned.push_back(p);
    return static_cast<T*>(p);
}

void freeAll(DevicePool& pool, std::vector<void*>& owned)
{
    for (void* p : owned) pool.put(p);
    owned.clear();
}

// Structure::calculateInverseBox (Structure.cpp:518-544), same operation order.
void inverseBox(double const* b, double* ib)
{
    auto B = [&](int k, int c) { return b[k * 3 + c]; };
    double invdet = B(0, 0) * B(1, 1) * B(2, 2) + B(1, 0) * B(2, 1) * B(0, 2) + B(2, 0) * B(0, 1) * B(1, 2) -
                    B(2, 0) * B(1, 1) * B(0, 2) - B(0, 0) * B(2, 1) * B(1, 2) - B(1, 0) * B(0, 1) * B(2, 2);
    invdet = 1.0 / invdet;
    ib[0] = B(1, 1) * B(2, 2) - B(2, 1) * B(1, 2);
    ib[1] = B(2, 1) * B(0, 2) - B(0, 1) * B(2, 2);
    ib[2] = B(0, 1) * B(1, 2) - B(1, 1) * B(0, 2);
    ib[3] = B(2, 0) * B(1, 2) - B(1, 0) * B(2, 2);
    ib[4] = B(0, 0) * B(2, 2) - B(2, 0) * B(0, 2);
    ib[5] = B(1, 0) * B(0, 2) - B(0, 0) * B(1, 2);
    ib[6] = B(1, 0) * B(2, 1) - B(2, 0) * B(1, 1);
    ib[7] = B(2, 0) * B(0, 1) - B(0, 0) * B(2, 1);
    ib[8] = B(0, 0) * B(1, 1) - B(1, 0) * B(0, 1);
    for (int k = 0; k < 9; ++k) ib[k] *= invdet;
}

void cross(double const* a, double const* v, double* w)
{
    w[0] = a[1] * v[2] - a[2] * v[1];
    w[1] = a[2] * v[0] - a[0] * v[2];
    w[2] = a[0] * v[1] - a[1] * v[0];
}

void normalize3(double* v)
{
    double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= n;
    v[1] /= n;
    v[2] /= n;
}

double dot3(double const* a, double const* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Structure::calculatePbcCopies (Structure.cpp:485-516) plus the plane
// spacings used for the cell grid.
void pbcCopies(double const* box, double rc, int* pbc, double* proj)
{
    double axb[3], axc[3], bxc[3];
    cross(box + 0, box + 3, axb);
    normalize3(axb);
    cross(box + 0, box + 6, axc);
    normalize3(axc);
    cross(box + 3, box + 6, bxc);
    normalize3(bxc);
    proj[0] = std::fabs(dot3(box + 0, bxc));
    proj[1] = std::fabs(dot3(box + 3, axc));
    proj[2] = std::fabs(dot3(box + 6, axb));
    for (int a = 0; a < 3; ++a)
    {
        pbc[a] = 0;
        while (pbc[a] * proj[a] <= rc) pbc[a]++;
    }
}

} // namespace

void inverseBoxOf(double const* box, double* invbox) { inverseBox(box, invbox); }

void structureGeometry(DevStructInfo& d, double rc)
{
    // periodic copies and plane spacings of the (normalised) box
    double proj[3];
    pbcCopies(d.box, rc, d.pbc, proj);
    for (int a = 0; a < 3; ++a)
        if (d.pbc[a] > 500)   // image offsets are packed in 10 bits by the search
            throw std::range_error("ERROR: box too small for the cutoff radius (more than 500 periodic copies).\n");
    const int n = d.numAtoms;
    int64_t cells = 1;
    for (int a = 0; a < 3; ++a)
    {
        // cell width >= rc/2 (plus a margin far above rounding), searched
        // ceil(rc / width) cells to each side
        double want = rc * 0.5 * (1.0 + 1e-6);
        int nc = (int)std::floor(proj[a] / want);
        nc = std::max(1, std::min(nc, 256));
        double w = proj[a] / nc;
        d.nc[a] = nc;
        d.stencil[a] = (int)std::ceil(rc / w + 1e-9);
        cells *= nc;
    }
    if (cells > 64 * (int64_t)n + 64)
    {
        // very sparse structure: coarser grid (search cost bounded by the atom count)
        for (int a = 0; a < 3; ++a)
        {
            int nc = std::max(1, (int)std::floor(proj[a] / (rc * (1.0 + 1e-6))));
            nc = std::min(nc, 64);
            d.nc[a] = nc;
            d.stencil[a] = (int)std::ceil(rc / (proj[a] / nc) + 1e-9);
        }
    }
}

// ---------------------------------------------------------------------------
// DeviceModel
// ---------------------------------------------------------------------------

DeviceModel::~DeviceModel() { release(); }

void DeviceModel::release()
{
    cudaFree(groups_);
    cudaFree(members_);
    cudaFree(scaling_);
    cudaFree(rowTable_);
    cudaFree(weights_);
    cudaFree(weightsT_);
    cudaFree(transIndex_);
    cudaFree(compactGroups_);
    cudaFree(compactMembers_);
    cudaFree(compactFns_);
    compactGroups_ = nullptr;
    compactMembers_ = nullptr;
    compactFns_ = nullptr;
    groups_ = nullptr;
    members_ = nullptr;
    scaling_ = nullptr;
    rowTable_ = nullptr;
    weights_ = nullptr;
    weightsT_ = nullptr;
    transIndex_ = nullptr;
}

void DeviceModel::upload(Model const& m)
{
    if (!m.setupDone) throw std::runtime_error("ERROR: setupGeneric() has not been called.\n");
    if (!m.scalingDone) throw std::runtime_error("ERROR: symmetry function scaling has not been set up.\n");
    release();
    networksSet = true;
    missingWeights.clear();
    DevModel v{};
    v.numElements = (int)m.elements.size();
    v.normalizeNeurons = m.normalizeNeurons ? 1 : 0;
    v.allFast = 2;
    v.maxCutoff = m.maxCutoffRadius;
    v.maxCutoff2 = m.maxCutoffRadius * m.maxCutoffRadius;

    std::vector<double> slotRc;
    std::vector<DevGroup> groups;
    std::vector<DevMember> members;
    std::vector<DevCompactGroup> compactGroups;
    std::vector<DevCompactMember> compactMembers;
    std::vector<DevCompactFn> compactFns;
    int compactRows = 0;
    int compactAngCore = -1;   // -1: no staged angular part seen yet
    int compactNarrowStaged = 1;
    int compactCols = 0;
    std::vector<DevScaling> scaling;
    std::vector<int> rowTable;
    std::vector<double> weights;
    int maxSF = 0, maxRows = 0;
    for (std::size_t e = 0; e < m.elements.size(); ++e)
    {
        ElementSetup const& el = m.elements[e];
        DevElement& de = v.el[e];
        de.numSF = (int)el.sf.size();
        if (de.numSF > kMaxSFPerElement) throw std::runtime_error("ERROR: too many symmetry functions per element.\n");
        maxSF = std::max(maxSF, de.numSF);
        de.sfBegin = (int)scaling.size();
        for (auto const& s : el.sf)
        {
            DevScaling sc{};
            sc.type = s.scalingType;
            sc.Smin = s.Smin;
            sc.Gmin = s.Gmin;
            sc.Gmax = s.Gmax;
            sc.Gmean = s.Gmean;
            sc.scalingFactor = s.scalingFactor;
            scaling.push_back(sc);
        }
        for (std::size_t en = 0; en < m.elements.size(); ++en)
        {
            de.rows[en] = (int)el.table[en].size();
            de.tableBegin[en] = (int)rowTable.size();
            for (int idx : el.table[en]) rowTable.push_back(idx);
            maxRows = std::max(maxRows, de.rows[en]);
        }
        de.groupBegin = (int)groups.size();
        de.groupCount = (int)el.groups.size();
        for (auto const& g : el.groups)
        {
            if ((int)g.members.size() > kMaxMembers) throw std::runtime_error("ERROR: symmetry function group too large.\n");
            DevGroup dg{};
            dg.type = g.type;
            dg.e1 = g.e1;
            dg.e2 = g.e2;
            dg.cutoffType = g.cutoffType;
            dg.rc = g.rc;
            dg.rc2 = g.rc * g.rc;
            auto it = std::find(slotRc.begin(), slotRc.end(), g.rc);
            if (it == slotRc.end())
            {
                if (slotRc.size() >= 4) throw std::runtime_error("ERROR: more than 4 distinct cutoff radii.\n");
                slotRc.push_back(g.rc);
                it = slotRc.end() - 1;
            }
            dg.cutoffSlot = (int)(it - slotRc.begin());
            dg.memberBegin = (int)members.size();
            dg.memberCount = (int)g.members.size();
            // Gaussian plan: exp(-eta r^2) of a member is an integer power
            // (<= 16) of an earlier base when eta/eta_base is integral, which
            // turns the per-triplet Gaussians into products of per-neighbour
            // factors and one exponential of r_jk^2 per base.
            std::vector<double> bases;
            std::vector<int> planBase(g.members.size(), -1), planPow(g.members.size(), 1);
            bool allRs0 = true;
            for (std::size_t q = 0; q < g.members.size(); ++q)
            {
                SymFunc const& s = el.sf[g.members[q]];
                if (s.rs != 0.0)
                {
                    allRs0 = false;
                    continue;
                }
                for (std::size_t b = 0; b < bases.size(); ++b)
                {
                    double ratio = s.eta / bases[b];
                    double k = std::round(ratio);
                    if (k >= 1.0 && k <= 16.0 && std::fabs(ratio - k) <= 1e-9 * ratio)
                    {
                        planBase[q] = (int)b;
                        planPow[q] = (int)k;
                        break;
                    }
                }
                if (planBase[q] < 0 && (int)bases.size() < kMaxBases)
                {
                    bases.push_back(s.eta);
                    planBase[q] = (int)bases.size() - 1;
                    planPow[q] = 1;
                }
            }
            dg.numBases = (int)bases.size();
            for (std::size_t b = 0; b < bases.size(); ++b) dg.baseEta[b] = bases[b];
            bool planned = true;
            for (int pb : planBase) planned = planned && pb >= 0;
            dg.fast = (allRs0 && planned && (g.type == 2 || dg.numBases <= kMaxStagedBases)) ? 1 : 0;
            // Member grid (angular groups): slots of distinct eta, lambda and
            // integer zeta; the kernels then evaluate each factor once per
            // triplet and combine them with fixed-index arithmetic.
            dg.grid = 0;
            for (int c = 0; c < 16; ++c) dg.comboMember[c] = -1;
            if (g.type != 2 && dg.fast && g.members.size() <= 16)
            {
                std::vector<double> etas, lams;
                std::vector<int> zetas;
                bool ok = true;
                for (std::size_t q = 0; q < g.members.size() && ok; ++q)
                {
                    SymFunc const& s = el.sf[g.members[q]];
                    if (!s.useIntegerPow || s.zetaInt < 1 || s.zetaInt > 32) ok = false;   // zeta-1 in 5 bits
                    if (std::find(etas.begin(), etas.end(), s.eta) == etas.end()) etas.push_back(s.eta);
                    if (std::find(lams.begin(), lams.end(), s.lambda) == lams.end()) lams.push_back(s.lambda);
                    if (std::find(zetas.begin(), zetas.end(), s.zetaInt) == zetas.end()) zetas.push_back(s.zetaInt);
                }
                ok = ok && etas.size() <= 2 && lams.size() <= 2 && zetas.size() <= 4;
                if (ok)
                {
                    for (std::size_t q = 0; q < g.members.size(); ++q)
                    {
                        SymFunc const& s = el.sf[g.members[q]];
                        int es = (int)(std::find(etas.begin(), etas.end(), s.eta) - etas.begin());
                        int ls = (int)(std::find(lams.begin(), lams.end(), s.lambda) - lams.begin());
                        int zs = (int)(std::find(zetas.begin(), zetas.end(), s.zetaInt) - zetas.begin());
                        int c = (es * 2 + ls) * 4 + zs;
                        if (dg.comboMember[c] >= 0) ok = false;   // duplicate function
                        dg.comboMember[c] = (signed char)q;
                        dg.etaBase[es] = planBase[q];
                        dg.etaPow[es] = planPow[q];
                    }
                    for (std::size_t k = 0; k < lams.size(); ++k) dg.lambdaVal[k] = lams[k];
                    for (std::size_t k = lams.size(); k < 2; ++k) dg.lambdaVal[k] = 0.0;
                    for (std::size_t k = 0; k < zetas.size(); ++k) dg.zetaM1[k] = zetas[k] - 1;
                    for (std::size_t k = zetas.size(); k < 4; ++k) dg.zetaM1[k] = 0;
                    for (std::size_t k = etas.size(); k < 2; ++k)
                    {
                        dg.etaBase[k] = 0;
                        dg.etaPow[k] = 1;
                    }
                    dg.gridNZ = (int)zetas.size();
                    auto digits = [](int v) {
                        int d = 0;
                        while (v > 0)
                        {
                            ++d;
                            v >>= 1;
                        }
                        return d;
                    };
                    dg.etaBits = digits(std::max(dg.etaPow[0], dg.etaPow[1]));
                    dg.zetaBits = 0;
                    for (int k = 0; k < dg.gridNZ; ++k) dg.zetaBits = std::max(dg.zetaBits, digits(dg.zetaM1[k]));
                }
                if (ok) dg.grid = 1;
                else for (int c = 0; c < 16; ++c) dg.comboMember[c] = -1;
            }
            for (std::size_t q = 0; q < g.members.size(); ++q)
            {
                SymFunc const& s = el.sf[g.members[q]];
                DevMember dm{};
                dm.eta = s.eta;
                dm.rs = s.rs;
                dm.lambda = s.lambda;
                dm.zeta = s.zeta;
                dm.sf = s.index;
                dm.zetaInt = s.zetaInt;
                dm.useIntPow = s.useIntegerPow ? 1 : 0;
                dm.calcExp = g.calculateExp[q] ? 1 : 0;
                dm.expBase = planBase[q];
                dm.expPow = planPow[q];
                dm.rowE1 = s.indexPerElement[s.e1];
                dm.rowE2 = (s.type == 2) ? dm.rowE1 : s.indexPerElement[s.e2];
                if (s.type == 2)
                {
                    dm.factorNorm = s.scalingFactor;
                    dm.gNorm = 1.0;
                }
                else
                {
                    dm.factorNorm = g.factorNorm[q];
                    dm.factorDeriv = g.factorDeriv[q];
                    dm.zetaLambda = s.zeta * s.lambda;
                    dm.gNorm = g.factorNorm[q] / s.scalingFactor;
                }
                members.push_back(dm);
            }
            if (!dg.fast || (dg.type != 2 && (!dg.grid || dg.numBases > 1))) v.allFast = 0;   // one staged base
            if (dg.grid) v.powBits = std::max(v.powBits, std::max(dg.etaBits, dg.zetaBits));
            if (dg.type != 2 && dg.rc < m.maxCutoffRadius) v.sortByDistance = 1;
            else if (dg.type != 2 && dg.gridNZ > 2 && v.allFast) v.allFast = 4;
            groups.push_back(dg);
        }
        // compact groups (SymGrpCompRad / SymGrpCompAngw members)
        de.compactBegin = (int)compactGroups.size();
        de.compactCount = (int)el.compactGroups.size();
        for (auto const& g : el.compactGroups)
        {
            DevCompactGroup cg{};
            cg.type = g.type;
            cg.e1 = g.e1;
            cg.e2 = g.e2;
            cg.memberBegin = (int)compactMembers.size();
            cg.memberCount = (int)g.members.size();
            // SymGrpBaseComp starts rmin and rmax at 0; addMember keeps rmin at 0 (min with 0 or
            // reset to 0) and raises rmax to the largest rc (SymGrpCompAngn.cpp:84-86)
            cg.rmin = 0.0;
            cg.rmax = 0.0;
            for (std::size_t mi = 0; mi < g.members.size(); ++mi)
            {
                SymFunc const& s = el.sf[g.members[mi]];
                DevCompactMember cm{};
                cm.sf = s.index;
                cm.core = s.core;
                cm.asym = s.asymmetric ? 1 : 0;
                cm.calcComp = g.calculateComp.at(mi);
                // CompactFunction::setLeftRight (CompactFunction.cpp:62-76)
                cm.rl = s.rl;
                cm.rc = s.rc;
                cm.rCenter = (s.rc + s.rl) / 2.0;
                cm.rScale = 1.0 / ((s.rc - s.rl) / 2.0);
                if (!s.radial())
                {
                    // SymFncBaseCompAng::setParameters: the angles in radians
                    const double pi = 3.14159265358979323846;
                    cm.aLeft = s.angleLeft * pi / 180.0;
                    cm.aRight = s.angleRight * pi / 180.0;
                    cm.aCenter = (cm.aRight + cm.aLeft) / 2.0;
                    cm.aScale = 1.0 / ((cm.aRight - cm.aLeft) / 2.0);
                }
                cg.rmax = std::max(cg.rmax, s.rc);
                compactMembers.push_back(cm);
            }
            if (g.type != 20 && g.type != 23)
            {
                // the members' distinct radial parts (core, asymmetry, window) and angular parts
                // (core, window): every member is one cell of this grid
                std::vector<DevCompactFn> rad, ang;
                auto find = [](std::vector<DevCompactFn>& list, DevCompactFn const& f) {
                    for (std::size_t k = 0; k < list.size(); ++k)
                        if (list[k].core == f.core && list[k].asym == f.asym && list[k].left == f.left &&
                            list[k].right == f.right)
                            return (int)k;
                    list.push_back(f);
                    return (int)list.size() - 1;
                };
                for (int mi = cg.memberBegin; mi < cg.memberBegin + cg.memberCount; ++mi)
                {
                    DevCompactMember& cm = compactMembers[mi];
                    cm.rIdx = find(rad, DevCompactFn{cm.rl, cm.rc, cm.rCenter, cm.rScale, cm.core, cm.asym});
                    cm.aIdx = find(ang, DevCompactFn{cm.aLeft, cm.aRight, cm.aCenter, cm.aScale, cm.core, 0});
                }
                cg.nR = (int)rad.size();
                cg.nA = (int)ang.size();
                cg.fnBegin = (int)compactFns.size();
                compactFns.insert(compactFns.end(), rad.begin(), rad.end());
                compactFns.insert(compactFns.end(), ang.begin(), ang.end());
                cg.walkBegin = cg.walkEnd = cg.numImpure = 0;
                bool staged = true;
                if (g.type == 21 || g.type == 24)
                {
                    // The reference carries the j-k radial part along a run of members that do not
                    // recompute it (calculateComp, SymGrpCompAngn.cpp:253-296): a member's value uses
                    // the radial part of the run's last recomputing member.  A member whose run since
                    // its last calculateComp member holds only its own radial part gets its own part
                    // whatever the pair's skips; the others ("impure") are replayed per pair.
                    int c0 = 0, numImpure = 0, wb = -1, we = 0;
                    for (int k = 0; k < cg.memberCount; ++k)
                    {
                        DevCompactMember& cm = compactMembers[cg.memberBegin + k];
                        if (cm.calcComp) c0 = k;
                        bool impure = false;
                        for (int j = c0; j < k; ++j)
                            if (compactMembers[cg.memberBegin + j].rIdx != cm.rIdx) impure = true;
                        cm.impure = impure ? numImpure++ : -1;
                        if (impure)
                        {
                            if (wb < 0) wb = c0;
                            we = k + 1;
                        }
                    }
                    cg.numImpure = numImpure;
                    if (numImpure > 0)
                    {
                        cg.walkBegin = wb;
                        cg.walkEnd = we;
                    }
                    staged = cg.nR <= kCompactStageRows && cg.nA <= kCompactStageCols &&
                             numImpure <= kCompactImpure && we - std::max(wb, 0) <= kCompactWalk;
                    if (!staged) compactNarrowStaged = 0;
                }
                else
                    for (int k = 0; k < cg.memberCount; ++k) compactMembers[cg.memberBegin + k].impure = -1;
                if (staged)
                {
                    compactRows = std::max(compactRows, cg.nR);
                    compactCols = std::max(compactCols, cg.nA);
                    for (auto const& f : ang)
                        compactAngCore = (compactAngCore == -1 || compactAngCore == f.core) ? f.core : 0;
                }
            }
            compactGroups.push_back(cg);
        }
        // network
        NetworkTopology const& t = el.topology;
        if (!el.hasWeights)   // symmetry functions alone still run (nnp-scaling); networks refuse to
        {
            networksSet = false;
            missingWeights = el.symbol;
        }
        if (t.numLayers > kDevMaxLayers) throw std::runtime_error("ERROR: too many network layers.\n");
        de.numLayers = t.numLayers;
        for (int l = 0; l < t.numLayers; ++l)
        {
            de.neurons[l] = t.neurons[l];
            de.activation[l] = t.activations[l];
            if (t.neurons[l] > kMaxNeurons && l > 0) throw std::runtime_error("ERROR: network layer too wide.\n");
        }
        for (int l = 1; l < t.numLayers; ++l)
        {
            de.wOffset[l] = (int)weights.size();
            if (el.hasWeights) weights.insert(weights.end(), el.W[l - 1].begin(), el.W[l - 1].end());
            else weights.insert(weights.end(), (size_t)t.neurons[l] * t.neurons[l - 1], 0.0);
            de.bOffset[l] = (int)weights.size();
            if (el.hasWeights) weights.insert(weights.end(), el.b[l - 1].begin(), el.b[l - 1].end());
            else weights.insert(weights.end(), (size_t)t.neurons[l], 0.0);
        }
    }
    v.maxSF = maxSF;
    v.maxRows = maxRows;
    v.numCutoffSlots = (int)slotRc.size();
    const double E = std::exp(1.0);
    for (std::size_t s = 0; s < slotRc.size(); ++s)
    {
        DevCutoff& c = v.cutoff[s];
        c.type = m.cutoffType;
        c.rc = slotRc[s];
        c.rcinv = 1.0 / slotRc[s];
        c.alpha = m.cutoffAlpha;
        c.rci = c.rc * c.alpha;
        c.iw = 1.0 / (c.rc - c.rci);
        c.tanhPre = std::pow((E + 1 / E) / (E - 1 / E), 3);
        c.rcF = (float)c.rc;
        c.rciF = (float)c.rci;
        c.iwF = (float)c.iw;
    }
    // transposed copy of every weight matrix (same offsets; biases copied):
    // element (k, j) of W_l [n_l x n_{l-1}] at j n_l + k, for reads that are
    // contiguous over output neurons
    std::vector<double> weightsT(weights);
    transIndexHost.resize(weights.size());
    for (size_t q = 0; q < weights.size(); ++q) transIndexHost[q] = (int)q;
    for (std::size_t e = 0; e < m.elements.size(); ++e)
    {
        DevElement const& de = v.el[e];
        for (int l = 1; l < de.numLayers; ++l)
        {
            const int nin = de.neurons[l - 1], nout = de.neurons[l];
            for (int k = 0; k < nout; ++k)
                for (int j = 0; j < nin; ++j)
                {
                    const int src = de.wOffset[l] + k * nin + j, dst = de.wOffset[l] + j * nout + k;
                    weightsT[dst] = weights[src];
                    transIndexHost[src] = dst;
                }
        }
    }
    auto up = [](void** dst, void const* src, size_t bytes) {
        cudaCheck(cudaMalloc(dst, bytes ? bytes : 16), "cudaMalloc(model)");
        if (bytes) cudaCheck(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy(model)");
    };
    for (auto& g : groups)
    {
        for (int b = 0; b < 4; ++b) g.baseEtaF[b] = (float)g.baseEta[b];
        for (int k = 0; k < 2; ++k) g.lambdaValF[k] = (float)g.lambdaVal[k];
    }
    up((void**)&groups_, groups.data(), groups.size() * sizeof(DevGroup));
    up((void**)&members_, members.data(), members.size() * sizeof(DevMember));
    up((void**)&scaling_, scaling.data(), scaling.size() * sizeof(DevScaling));
    up((void**)&rowTable_, rowTable.data(), rowTable.size() * sizeof(int));
    up((void**)&weights_, weights.data(), weights.size() * sizeof(double));
    up((void**)&weightsT_, weightsT.data(), weightsT.size() * sizeof(double));
    up((void**)&transIndex_, transIndexHost.data(), transIndexHost.size() * sizeof(int));
    up((void**)&compactGroups_, compactGroups.data(), compactGroups.size() * sizeof(DevCompactGroup));
    up((void**)&compactMembers_, compactMembers.data(), compactMembers.size() * sizeof(DevCompactMember));
    up((void**)&compactFns_, compactFns.data(), compactFns.size() * sizeof(DevCompactFn));
    v.numCompactGroups = (int)compactGroups.size();
    v.compactTypes = 0;
    for (auto const& cg : compactGroups) v.compactTypes |= 1 << (cg.type - 20);
    // ElementMap::atomicNumber of every element (the weights of the weighted compact functions)
    for (std::size_t e = 0; e < m.elements.size(); ++e) v.atomicNumber[e] = (double)m.elements[e].atomicNumber;
    v.compactGroups = compactGroups_;
    v.compactMembers = compactMembers_;
    v.compactFns = compactFns_;
    v.compactRows = compactRows;
    v.compactAngCore = std::max(compactAngCore, 0);
    v.compactNarrowStaged = compactNarrowStaged;
    v.compactCols = compactCols;
    v.groups = groups_;
    groupTable = DevGroupTable{};
    if (groups.size() <= (size_t)kParamGroups)
    {
        groupTable.count = (int)groups.size();
        std::copy(groups.begin(), groups.end(), groupTable.g);
    }
    else v.allFast = 0;   // the specialised kernels read the groups from their argument
    v.members = members_;
    v.scaling = scaling_;
    v.rowTable = rowTable_;
    v.weights = weights_;
    numWeights = weights.size();
    // FNV-1a over the evaluation plan (what the kernels' speed depends on)
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](const void* p, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        for (size_t k = 0; k < n; ++k) h = (h ^ c[k]) * 1099511628211ull;
    };
    mix(groups.data(), groups.size() * sizeof(DevGroup));
    mix(members.data(), members.size() * sizeof(DevMember));
    mix(compactGroups.data(), compactGroups.size() * sizeof(DevCompactGroup));
    mix(compactMembers.data(), compactMembers.size() * sizeof(DevCompactMember));
    mix(compactFns.data(), compactFns.size() * sizeof(DevCompactFn));
    mix(&v.numElements, sizeof(int));
    mix(&v.allFast, sizeof(int));
    mix(&v.sortByDistance, sizeof(int));
    mix(v.cutoff, sizeof(v.cutoff));
    fingerprint = h;
    tcNetwork = networkTCSupported(m);
    v.weightsT = weightsT_;
    view = v;
    this->maxSF = maxSF;
}

// ---------------------------------------------------------------------------
// Batch
// ---------------------------------------------------------------------------

Batch::Batch(Model const& model, DeviceModel const& dmodel, cudaStream_t stream, int sms)
    : model_(model), dmodel_(dmodel), stream_(stream), sms_(sms)
{
}

Batch::~Batch()
{
    releaseAll();
    pool_.trim();
}

void Batch::releaseGraph()
{
    if (graphExec_) cudaGraphExecDestroy(graphExec_);
    graphExec_ = nullptr;
    graphKey_ = -1;
}

void Batch::releaseAll()
{
    releaseGraph();
    freeAll(pool_, ownedMask_);
    maskBuf_ = nullptr;
    maskCap_ = 0;
    freeAll(pool_, ownedDGdr_);
    freeAll(pool_, ownedScr_);
    scrEntries_ = 0;
    nbrStride_ = strideWanted_ = 0;
    v_.scrStride = 0;
    freeAll(pool_, ownedNbr_);
    freeAll(pool_, owned_);
    dgdrAllocated_ = false;
}

void Batch::setStructures(std::vector<StructureInput> const& s, const int* elements, int remap)
{
    releaseAll();
    external_ = false;
    numTargets_ = 0;
    structs_ = s;
    S_ = (int)s.size();
    N_ = 0;
    structBegin_.assign(S_ + 1, 0);
    for (int k = 0; k < S_; ++k)
    {
        if (s[k].numAtoms <= 0) throw std::runtime_error("ERROR: structure without atoms.\n");
        structBegin_[k + 1] = structBegin_[k] + s[k].numAtoms;
    }
    N_ = structBegin_[S_];
    int ne = (int)model_.numElements();
    elemHost_.assign(elements, elements + N_);
    numAtomsPerElement_.assign((size_t)S_ * ne, 0);
    for (int k = 0; k < S_; ++k)
        for (int a = structBegin_[k]; a < structBegin_[k + 1]; ++a)
        {
            if (elemHost_[a] < 0 || elemHost_[a] >= ne) throw std::runtime_error("ERROR: element index out of range.\n");
            numAtomsPerElement_[(size_t)k * ne + elemHost_[a]]++;
        }
    remap_ = remap;

    // geometry per structure
    const double rc = model_.maxCutoffRadius;
    const double conv = model_.normalize ? model_.convLength : 1.0;
    std::vector<DevStructInfo> info(S_);
    int cellTotal = 0;
    int64_t capacity = 0;
    for (int k = 0; k < S_; ++k)
    {
        DevStructInfo& d = info[k];
        std::memset(&d, 0, sizeof(d));
        d.atomBegin = structBegin_[k];
        d.numAtoms = s[k].numAtoms;
        d.periodic = s[k].periodic;
        const int n = s[k].numAtoms;
        if (s[k].periodic)
        {
            std::memcpy(d.boxPhys, s[k].box, sizeof(d.boxPhys));
            inverseBox(d.boxPhys, d.invboxPhys);
            for (int q = 0; q < 9; ++q)
            {
                d.box[q] = model_.normalize ? d.boxPhys[q] * conv : d.boxPhys[q];
                d.invbox[q] = model_.normalize ? d.invboxPhys[q] / conv : d.invboxPhys[q];
            }
            structureGeometry(d, rc);
            const int64_t cells = (int64_t)d.nc[0] * d.nc[1] * d.nc[2];
            d.cellBegin = cellTotal;
            cellTotal += (int)cells;
            double vol = std::fabs(d.box[0] * (d.box[4] * d.box[8] - d.box[5] * d.box[7]) -
                                   d.box[1] * (d.box[3] * d.box[8] - d.box[5] * d.box[6]) +
                                   d.box[2] * (d.box[3] * d.box[7] - d.box[4] * d.box[6]));
            double expected = n / vol * 4.18879020478639 * rc * rc * rc;
            int64_t images = (int64_t)(2 * d.pbc[0] + 1) * (2 * d.pbc[1] + 1) * (2 * d.pbc[2] + 1);
            int64_t perAtom = std::min<int64_t>(images * n, (int64_t)std::ceil(expected * 1.4 + 32));
            capacity += perAtom * n;
        }
        else
        {
            d.nc[0] = d.nc[1] = d.nc[2] = 1;
            d.cellBegin = cellTotal;
            cellTotal += 1;
            capacity += (int64_t)n * (n - 1);
        }
    }

    allocateAtoms();
    uploadElementLists();
    v_.numCells = cellTotal;
    v_.cellCount = devAlloc<int>(pool_, cellTotal, owned_);
    v_.cellStart = devAlloc<int>(pool_, cellTotal, owned_);
    v_.cellStart64 = devAlloc<int64_t>(pool_, cellTotal + 1, owned_);
    v_.scanTmp = devAlloc<int64_t>(pool_, std::max(scanTileCount(cellTotal), scanTileCount(N_)) + 8, owned_);
    cudaCheck(cudaMemcpyAsync(infoDev_, info.data(), sizeof(DevStructInfo) * S_, cudaMemcpyHostToDevice, stream_),
              "upload structure info");
    std::vector<int> atomStruct(N_);
    for (int k = 0; k < S_; ++k)
        for (int a = structBegin_[k]; a < structBegin_[k + 1]; ++a) atomStruct[a] = k;
    cudaCheck(cudaMemcpyAsync(atomStructDev_, atomStruct.data(), sizeof(int) * N_, cudaMemcpyHostToDevice, stream_),
              "upload atom map");
    cudaCheck(cudaMemcpyAsync(elemDev_, elemHost_.data(), sizeof(int) * N_, cudaMemcpyHostToDevice, stream_),
              "upload elements");
    cudaCheck(cudaMemcpyAsync(structBeginDev_, structBegin_.data(), sizeof(int) * (S_ + 1), cudaMemcpyHostToDevice,
                              stream_),
              "upload offsets");
    cudaCheck(cudaStreamSynchronize(stream_), "setStructures");
    allocateNeighbors(std::max<int64_t>(capacity, 1));
    capacityVerified_ = false;
    pendingVerify_ = false;
    stage_ = StageState{};
    tuned_[0] = tuned_[1] = false;   // new workload: shapes come from the cache or are measured again
}

// Atoms grouped by element (the tensor-core networks run per element).
void Batch::uploadElementLists()
{
    const int ne = (int)model_.numElements();
    std::vector<int> order;
    order.reserve(N_);
    v_.elemBegin[0] = 0;
    for (int e = 0; e < ne; ++e)
    {
        for (int a = 0; a < N_; ++a)
            if (elemHost_[a] == e) order.push_back(a);
        v_.elemBegin[e + 1] = (int)order.size();
    }
    int* dev = devAlloc<int>(pool_, (size_t)std::max(N_, 1), owned_);
    if (N_ > 0)
        cudaCheck(cudaMemcpy(dev, order.data(), sizeof(int) * (size_t)N_, cudaMemcpyHostToDevice),
                  "upload element lists");
    v_.elemAtoms = dev;
}

// Shared part of both external forms: one system of `numCenters` atoms,
// its element lists and the buffers of the transposed lists.
void Batch::beginExternal(int numCenters, const int* elements, int numTargets, const int* centerTarget,
                          int64_t capacity)
{
    if (numCenters <= 0) throw std::runtime_error("ERROR: no local atoms.\n");
    const int ne = (int)model_.numElements();
    std::vector<char> seen((size_t)std::max(numTargets, 1), 0);
    for (int a = 0; a < numCenters; ++a)
    {
        const int k = centerTarget[a];
        if (k < 0 || k >= numTargets || seen[k])
            throw std::invalid_argument("ERROR: local atom indices must be distinct and below the atom count.\n");
        seen[k] = 1;
        if (elements[a] < 0 || elements[a] >= ne) throw std::runtime_error("ERROR: element index out of range.\n");
    }
    // Everything but the candidate-mask buffer is released: a caller that
    // sets new lists every step (an MD code) keeps masks of the last size.
    releaseGraph();
    freeAll(pool_, ownedDGdr_);
    freeAll(pool_, ownedScr_);
    scrEntries_ = 0;
    nbrStride_ = strideWanted_ = 0;
    v_.scrStride = 0;
    freeAll(pool_, ownedNbr_);
    freeAll(pool_, owned_);
    dgdrAllocated_ = false;
    external_ = true;
    S_ = 1;
    N_ = numCenters;
    structs_.assign(1, StructureInput{});
    structs_[0].numAtoms = N_;
    structBegin_ = {0, N_};
    elemHost_.assign(elements, elements + N_);
    numAtomsPerElement_.assign((size_t)ne, 0);
    for (int a = 0; a < N_; ++a) numAtomsPerElement_[elemHost_[a]]++;
    numTargets_ = numTargets;
    allocateAtoms();
    uploadElementLists();
    v_.numCells = 0;
    v_.scanTmp = devAlloc<int64_t>(pool_, scanTileCount(N_) + 8, owned_);   // entry offsets, candidate masks
    std::vector<DevStructInfo> info(1);
    std::memset(info.data(), 0, sizeof(DevStructInfo));
    info[0].numAtoms = N_;
    cudaCheck(cudaMemcpyAsync(infoDev_, info.data(), sizeof(DevStructInfo), cudaMemcpyHostToDevice, stream_),
              "upload structure info");
    cudaCheck(cudaMemsetAsync(atomStructDev_, 0, sizeof(int) * N_, stream_), "memset");
    cudaCheck(cudaMemcpyAsync(elemDev_, elemHost_.data(), sizeof(int) * N_, cudaMemcpyHostToDevice, stream_),
              "upload elements");
    cudaCheck(cudaMemcpyAsync(structBeginDev_, structBegin_.data(), sizeof(int) * 2, cudaMemcpyHostToDevice, stream_),
              "upload offsets");
    allocateNeighbors(std::max<int64_t>(capacity, 1));
    const size_t T = (size_t)std::max(numTargets, 1);
    tCount_ = devAlloc<int>(pool_, T, ownedNbr_);
    tFill_ = devAlloc<int>(pool_, T, ownedNbr_);
    tOffset_ = devAlloc<int64_t>(pool_, T + 1, ownedNbr_);
    tEntryTmp_ = devAlloc<int64_t>(pool_, (size_t)capacity_, ownedNbr_);
    tEntry_ = devAlloc<int64_t>(pool_, (size_t)capacity_, ownedNbr_);
    targetCenter_ = devAlloc<int>(pool_, T, ownedNbr_);
    centerIndex_ = devAlloc<int>(pool_, (size_t)N_, ownedNbr_);
    tScanTmp_ = devAlloc<int64_t>(pool_, scanTileCount((int)T) + 8, ownedNbr_);
    Ftarget_ = devAlloc<double>(pool_, 3 * T, ownedNbr_);
    entriesDev_ = devAlloc<int64_t>(pool_, 1, ownedNbr_);
    cudaCheck(cudaMemcpyAsync(centerIndex_, centerTarget, sizeof(int) * (size_t)N_, cudaMemcpyHostToDevice, stream_),
              "upload centre indices");
    cudaCheck(cudaMemsetAsync(Ftarget_, 0, sizeof(double) * 3 * T, stream_), "memset");
    capacityVerified_ = false;
    pendingVerify_ = false;
    stage_ = StageState{};
    tuned_[0] = tuned_[1] = false;
}

void Batch::setExternalNeighbors(int numCenters, const int* elements, int64_t numEntries, const int64_t* offsets,
                                 int numTargets, const int* target, const int* targetElement, const double* dr,
                                 const double* d, const int* centerTarget)
{
    if (numEntries < 0 || offsets[0] != 0 || offsets[numCenters] != numEntries)
        throw std::invalid_argument("ERROR: neighbour offsets do not match the entry count.\n");
    const int ne = (int)model_.numElements();
    const double rcmax = model_.maxCutoffRadius;
    for (int a = 0; a < numCenters; ++a)
    {
        if (offsets[a + 1] < offsets[a] || offsets[a + 1] - offsets[a] > 1024)
            throw std::runtime_error("ERROR: more than 1024 neighbours of one atom.\n");
        for (int64_t e = offsets[a]; e < offsets[a + 1]; ++e)
        {
            if (target[e] < 0 || target[e] >= numTargets)
                throw std::invalid_argument("ERROR: neighbour index out of range.\n");
            if (targetElement[e] < 0 || targetElement[e] >= ne)
                throw std::runtime_error("ERROR: element index out of range.\n");
            if (!(d[e] <= rcmax)) throw std::invalid_argument("ERROR: neighbour beyond the largest cutoff.\n");
        }
    }
    beginExternal(numCenters, elements, numTargets, centerTarget, std::max<int64_t>(numEntries, 1));
    extRaw_ = false;
    const size_t E = (size_t)numEntries;
    std::vector<uint8_t> el(std::max<size_t>(E, 1));
    std::vector<double> dx(std::max<size_t>(E, 1)), dy(dx.size()), dz(dx.size());
    for (size_t e = 0; e < E; ++e)
    {
        el[e] = (uint8_t)targetElement[e];
        dx[e] = dr[3 * e + 0];
        dy[e] = dr[3 * e + 1];
        dz[e] = dr[3 * e + 2];
    }
    auto up = [&](void* dst, const void* src, size_t bytes, char const* what) {
        if (bytes) cudaCheck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), what);
    };
    up(v_.nbrOffset, offsets, sizeof(int64_t) * ((size_t)N_ + 1), "upload offsets");
    up(v_.nbrJ, target, sizeof(int) * E, "upload neighbours");
    up(v_.nbrElem, el.data(), E, "upload neighbour elements");
    up(v_.nbrD, d, sizeof(double) * E, "upload distances");
    up(v_.nbrDx, dx.data(), sizeof(double) * E, "upload dr");
    up(v_.nbrDy, dy.data(), sizeof(double) * E, "upload dr");
    up(v_.nbrDz, dz.data(), sizeof(double) * E, "upload dr");
    up(entriesDev_, &numEntries, sizeof(int64_t), "upload entry count");
    cudaCheck(cudaStreamSynchronize(stream_), "setExternalNeighbors");   // host staging vectors go out of scope
}

void Batch::setExternalLists(ExternalLists const& l)
{
    if (l.numCenters <= 0) throw std::runtime_error("ERROR: no local atoms.\n");
    if (l.candOffset[0] != 0 || l.candOffset[l.numCenters] != l.numCand)
        throw std::invalid_argument("ERROR: candidate offsets do not match the candidate count.\n");
    for (int c = 0; c < l.numCenters; ++c)
        if (l.candOffset[c + 1] < l.candOffset[c]) throw std::invalid_argument("ERROR: decreasing candidate offsets.\n");
    if (l.numTypes < 0 || l.numAll <= 0) throw std::invalid_argument("ERROR: no atoms or types.\n");
    // entries are a subset of the candidates: the candidate count bounds them
    beginExternal(l.numCenters, l.centerElement, l.numAll, l.centerIndex, std::max<int64_t>(l.numCand, 1));
    extRaw_ = true;
    double* x = devAlloc<double>(pool_, 3 * (size_t)l.numAll, ownedNbr_);
    int* type = devAlloc<int>(pool_, (size_t)l.numAll, ownedNbr_);
    int* typeElement = devAlloc<int>(pool_, (size_t)l.numTypes + 1, ownedNbr_);
    int64_t* candOffset = devAlloc<int64_t>(pool_, (size_t)l.numCenters + 1, ownedNbr_);
    int* cand = devAlloc<int>(pool_, (size_t)std::max<int64_t>(l.numCand, 1), ownedNbr_);
    auto up = [&](void* dst, const void* src, size_t bytes, char const* what) {
        if (bytes) cudaCheck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_), what);
    };
    up(x, l.x, sizeof(double) * 3 * (size_t)l.numAll, "upload positions");
    up(type, l.type, sizeof(int) * (size_t)l.numAll, "upload types");
    up(typeElement, l.typeElement, sizeof(int) * ((size_t)l.numTypes + 1), "upload type map");
    up(candOffset, l.candOffset, sizeof(int64_t) * ((size_t)l.numCenters + 1), "upload candidate offsets");
    up(cand, l.cand, sizeof(int) * (size_t)l.numCand, "upload candidates");
    raw_ = ExtRawView{};
    raw_.x = x;
    raw_.type = type;
    raw_.typeElement = typeElement;
    raw_.numTypes = l.numTypes;
    raw_.numAll = l.numAll;
    raw_.centerIndex = centerIndex_;
    raw_.candOffset = candOffset;
    raw_.cand = cand;
    raw_.cflength = l.cflength;
    raw_.convLength = l.convLength;
    raw_.normalize = l.normalize ? 1 : 0;
    raw_.pairCut2 = l.pairCut2;
    raw_.rcmax = model_.maxCutoffRadius;
}

void Batch::targetForces(double* out)
{
    verify();
    if (!external_) throw std::runtime_error("ERROR: target forces need external neighbour lists.\n");
    cudaCheck(cudaMemcpyAsync(out, Ftarget_, sizeof(double) * 3 * (size_t)numTargets_, cudaMemcpyDeviceToHost, stream_),
              "F D2H");
    synchronize();
}

void Batch::allocateAtoms()
{
    const int N = N_;
    const int stride = dmodel_.maxSF;
    v_ = BatchView{};
    v_.N = N;
    v_.S = S_;
    v_.gStride = stride;
    infoDev_ = devAlloc<DevStructInfo>(pool_, S_, owned_);
    atomStructDev_ = devAlloc<int>(pool_, N, owned_);
    elemDev_ = devAlloc<int>(pool_, N, owned_);
    structBeginDev_ = devAlloc<int>(pool_, S_ + 1, owned_);
    rin_ = devAlloc<double>(pool_, 3 * (size_t)N, owned_);
    v_.info = infoDev_;
    v_.atomStruct = atomStructDev_;
    v_.elem = elemDev_;
    v_.structAtomBegin = structBeginDev_;
    v_.px = devAlloc<double>(pool_, N, owned_);
    v_.py = devAlloc<double>(pool_, N, owned_);
    v_.pz = devAlloc<double>(pool_, N, owned_);
    v_.atomCell = devAlloc<int>(pool_, N, owned_);
    v_.atomSlot = devAlloc<int>(pool_, N, owned_);
    v_.cellAtoms = devAlloc<int>(pool_, N, owned_);
    v_.cellPos = devAlloc<double4>(pool_, N, owned_);
    v_.nbrCount = devAlloc<int>(pool_, N, owned_);
    v_.nbrOffset = devAlloc<int64_t>(pool_, (size_t)N + 1, owned_);
    v_.G = devAlloc<double>(pool_, (size_t)N * stride, owned_);
    v_.dEdG = devAlloc<double>(pool_, (size_t)N * stride, owned_);
    v_.Eatom = devAlloc<double>(pool_, N, owned_);
    v_.Estruct = devAlloc<double>(pool_, S_, owned_);
    v_.fSelf = devAlloc<double>(pool_, 3 * (size_t)N, owned_);
    v_.F = devAlloc<double>(pool_, 3 * (size_t)N, owned_);
    v_.atomWarnings = devAlloc<int>(pool_, N, owned_);
    v_.maskWords = devAlloc<int>(pool_, N, owned_);
    v_.maskOffset = devAlloc<int64_t>(pool_, (size_t)N + 1, owned_);
    v_.status = devAlloc<DevStatus>(pool_, 1, owned_);
    // Pool blocks hold a previous user's data: clear what may be read before
    // the first evaluation writes it.
    cudaCheck(cudaMemsetAsync(v_.G, 0, sizeof(double) * (size_t)N * stride, stream_), "memset");
    cudaCheck(cudaMemsetAsync(v_.dEdG, 0, sizeof(double) * (size_t)N * stride, stream_), "memset");
    cudaCheck(cudaMemsetAsync(v_.status, 0, sizeof(DevStatus), stream_), "memset");
    cudaCheck(cudaMemsetAsync(v_.atomWarnings, 0, sizeof(int) * (size_t)N, stream_), "memset");
    cudaCheck(cudaMemsetAsync(v_.Estruct, 0, sizeof(double) * (size_t)S_, stream_), "memset");
    cudaCheck(cudaMemsetAsync(v_.F, 0, sizeof(double) * 3 * (size_t)N, stream_), "memset");
}

void Batch::allocateNeighbors(int64_t capacity)
{
    releaseGraph();
    freeAll(pool_, ownedDGdr_);
    dgdrAllocated_ = false;
    freeAll(pool_, ownedNbr_);
    const int slots = std::max(1, dmodel_.view.numCutoffSlots);
    capacity_ = capacity;
    v_.nbrCapacity = capacity;
    allocateScratch(std::max(capacity, (int64_t)N_ * nbrStride_));
    v_.nbrJ = devAlloc<int>(pool_, capacity, ownedNbr_);
    v_.nbrCode = devAlloc<int>(pool_, capacity, ownedNbr_);
    v_.nbrElem = devAlloc<uint8_t>(pool_, capacity, ownedNbr_);
    v_.nbrD = devAlloc<double>(pool_, capacity, ownedNbr_);
    v_.nbrDx = devAlloc<double>(pool_, capacity, ownedNbr_);
    v_.nbrDy = devAlloc<double>(pool_, capacity, ownedNbr_);
    v_.nbrDz = devAlloc<double>(pool_, capacity, ownedNbr_);
    v_.rev = devAlloc<int64_t>(pool_, capacity, ownedNbr_);
    v_.nbrFc = devAlloc<double>(pool_, (size_t)slots * capacity, ownedNbr_);
    v_.nbrDfc = devAlloc<double>(pool_, (size_t)slots * capacity, ownedNbr_);
    v_.hx = devAlloc<double>(pool_, capacity, ownedNbr_);
    v_.hy = devAlloc<double>(pool_, capacity, ownedNbr_);
    v_.hz = devAlloc<double>(pool_, capacity, ownedNbr_);
    v_.dGdr = nullptr;
    v_.dGdrSelf = nullptr;
}

// Unordered entries of the neighbour build: the packed entries (two passes)
// or N x stride (one pass).
void Batch::allocateScratch(int64_t entries)
{
    releaseGraph();
    freeAll(pool_, ownedScr_);
    scrEntries_ = entries;
    v_.scrKey = devAlloc<int64_t>(pool_, entries, ownedScr_);
    v_.scrD = devAlloc<double>(pool_, entries, ownedScr_);
    v_.scrDx = devAlloc<double>(pool_, entries, ownedScr_);
    v_.scrDy = devAlloc<double>(pool_, entries, ownedScr_);
    v_.scrDz = devAlloc<double>(pool_, entries, ownedScr_);
}

// Search stride for a largest neighbour count: 1/8 and 16 entries of room,
// a multiple of 8.
static int64_t strideFor(int64_t maxNeighbors)
{
    return (maxNeighbors + maxNeighbors / 8 + 16 + 7) / 8 * 8;
}

// Search mode of the neighbour build: 0 = count pass, scan, fill pass; > 0 =
// one pass into fixed-stride scratch (a recorded graph holds the mode).
void Batch::setStride(int64_t stride)
{
    if (stride == nbrStride_) return;
    releaseGraph();
    nbrStride_ = stride;
    v_.scrStride = stride;
    if (stride > 0 && (int64_t)N_ * stride > scrEntries_) allocateScratch((int64_t)N_ * stride);
}

void Batch::allocateDGdr()
{
    if (dgdrAllocated_) return;
    releaseGraph();
    const int rows = std::max(1, dmodel_.view.maxRows);
    v_.dGdr = devAlloc<double>(pool_, (size_t)rows * capacity_ * 3, ownedDGdr_);
    v_.dGdrSelf = devAlloc<double>(pool_, (size_t)N_ * v_.gStride * 3, ownedDGdr_);
    cudaCheck(cudaMemsetAsync(v_.dGdrSelf, 0, sizeof(double) * (size_t)N_ * v_.gStride * 3, stream_), "memset");
    dgdrAllocated_ = true;
}

void Batch::setPositionsHost(const double* r)
{
    if (external_) throw std::runtime_error("ERROR: external neighbour lists carry no positions.\n");
    verify();   // results of the previous positions stay complete until they are replaced
    stage_ = StageState{};
    cudaCheck(cudaMemcpyAsync(rin_, r, sizeof(double) * 3 * (size_t)N_, cudaMemcpyHostToDevice, stream_),
              "positions H2D");
}

void Batch::setPositionsDevice(const double* r)
{
    if (external_) throw std::runtime_error("ERROR: external neighbour lists carry no positions.\n");
    verify();
    stage_ = StageState{};
    cudaCheck(cudaMemcpyAsync(rin_, r, sizeof(double) * 3 * (size_t)N_, cudaMemcpyDeviceToDevice, stream_),
              "positions D2D");
}

// The kernel sequence of one evaluation (Mode::evaluateNNP, Mode.cpp:2029-2077).
void Batch::record(int flags, int precision, int checkExtrapolation, std::vector<Mark>* marks, int stages)
{
    DevModel const& m = dmodel_.view;
    const bool sfOnly = (flags & EVAL_SF_ONLY) != 0;
    const bool forces = (flags & EVAL_FORCES) != 0 && !sfOnly;
    const bool stored = (flags & EVAL_STORE_DGDR) != 0;
    const bool whole = stages == STAGE_ALL;   // an evaluation (not one of the separate stage calls)
    if (sfOnly) stages &= STAGE_NEIGHBORS | STAGE_SF;
    int launches = 0;
    auto mark = [&](char const* name) {
        if (!marks) return;
        Mark mk{name, nullptr};
        cudaCheck(cudaEventCreate(&mk.event), "cudaEventCreate");
        cudaCheck(cudaEventRecord(mk.event, stream_), "cudaEventRecord");
        marks->push_back(mk);
    };
    mark("start");
    if (stages & STAGE_NEIGHBORS)
    {
        cudaCheck(cudaMemsetAsync(v_.status, 0, sizeof(DevStatus), stream_), "status reset");
        if (external_)
        {
            if (extRaw_)
            {
                launchExternalEntries(raw_, v_, v_.scanTmp, sms_, stream_);
                launches += 5;
            }
            else   // the entry count the neighbour build would report (read by the cutoff stage)
                cudaCheck(cudaMemcpyAsync(&v_.status->totalNeighbors, entriesDev_, sizeof(int64_t),
                                          cudaMemcpyDeviceToDevice, stream_),
                          "entry count");
            launchExternalTranspose(v_, numTargets_, centerIndex_, tCount_, tFill_, tOffset_, tEntryTmp_, tEntry_,
                                    targetCenter_, tScanTmp_, sms_, stream_);
            launches += 7;
            mark("neighbor_list");
        }
        else
        {
            launchPreparePositions(v_, rin_, remap_, model_.normalize ? 1 : 0, model_.convLength, stream_);
            launches += 1;
            mark("prepare_positions");
            launchNeighborBuild(v_, model_.maxCutoffRadius * model_.maxCutoffRadius, stream_);
            launches += 3 + 3 + 1 + 1 + 1 + 3 + 1 + 1 + 1;
            mark("neighbor_list");
        }
        launchCutoffValues(m, v_, sms_, stream_);
        launches += 1;
        mark("cutoff_values");
    }
    if (stages & STAGE_SF)
    {
        if (!whole)   // a separate symmetry-function call counts its own warnings
            cudaCheck(cudaMemsetAsync(&v_.status->extrapolationWarnings, 0, sizeof(int), stream_), "status reset");
        // the G pass records its candidate acceptance for the force pass
        v_.candMask = nullptr;
        v_.maskCapacity = 0;
        if (forces && !stored)
        {
            launchMaskOffsets(m, v_, sms_, stream_);
            launches += 4;
            mark("candidate_masks");
            v_.candMask = maskBuf_;
            v_.maskCapacity = maskBuf_ ? maskCap_ : 0;
        }
        if (stored)
        {
            launchSFDerivatives(m, v_, sms_, stream_);
            launches += 2;
            mark("sf_derivatives");
        }
        else
        {
            launchSFValues(m, dmodel_.groupTable, v_, precision, sms_, stream_, sfShape_[0][precision]);
            launches += 2;
            if (m.numCompactGroups > 0) launches += launchCompactValues(m, v_, sms_, stream_);
            mark("sf_values");
        }
        if (checkExtrapolation)
        {
            launchExtrapolationCheck(m, v_, sms_, stream_);
            launches += 1;
            mark("extrapolation_check");
        }
    }
    if (stages & STAGE_NETWORKS)
    {
        if (precision == PREC_MIXED && dmodel_.tcNetwork) launchNetworkTC(m, v_, forces ? 1 : 0, sms_, stream_);
        else launchNetworkFP64(m, v_, forces ? 1 : 0, sms_, stream_);
        launches += 1;
        mark("network");
    }
    if (stages & STAGE_ENERGY)
    {
        launchEnergySum(v_, stream_);
        launches += 1;
        mark("energy_sum");
    }
    if (forces && (stages & STAGE_FORCES))
    {
        if (stored)
        {
            launchContractStored(m, v_, sms_, stream_);
            launches += 1;
            mark("contract_stored");
        }
        else
        {
            launchSFForces(m, dmodel_.groupTable, v_, precision, sms_, stream_, sfShape_[1][precision]);
            launches += 2;
            if (m.numCompactGroups > 0) launches += launchCompactForces(m, v_, sms_, stream_);
            mark("sf_forces");
        }
        if (external_) launchGatherTargets(v_, numTargets_, tOffset_, tEntry_, targetCenter_, Ftarget_, sms_, stream_);
        else launchGatherForces(v_, sms_, stream_);
        launches += 1;
        mark("gather_forces");
    }
    cudaCheck(cudaGetLastError(), "kernel launch");
    if (whole) launches_ = launches;
}

std::vector<std::pair<std::string, double>> Batch::profileStages(int flags, int precision, int checkExtrapolation)
{
    if (!capacityVerified_) evaluate(flags, precision, checkExtrapolation);
    std::vector<Mark> marks;
    record(flags, precision, checkExtrapolation, &marks);
    pendingVerify_ = true;
    synchronize();
    std::vector<std::pair<std::string, double>> out;
    for (size_t k = 1; k < marks.size(); ++k)
    {
        float ms = 0.f;
        cudaCheck(cudaEventElapsedTime(&ms, marks[k - 1].event, marks[k].event), "cudaEventElapsedTime");
        out.emplace_back(marks[k].name, (double)ms);
    }
    for (auto& mk : marks) cudaEventDestroy(mk.event);
    return out;
}

void Batch::countWork(int64_t* counts)
{
    verify();
    if (external_) throw std::runtime_error("ERROR: work counters need structures, not external neighbour lists.\n");
    if (dmodel_.view.numCompactGroups > 0)
        throw std::runtime_error("ERROR: work counters cover the Gaussian symmetry functions only.\n");
    unsigned long long* d = nullptr;
    cudaCheck(cudaMalloc(&d, sizeof(unsigned long long) * 10), "cudaMalloc");
    cudaCheck(cudaMemsetAsync(d, 0, sizeof(unsigned long long) * 10, stream_), "memset");
    launchCountWork(dmodel_.view, v_, d, sms_, stream_);
    unsigned long long h[10];
    cudaCheck(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, stream_), "D2H");
    synchronize();
    cudaFree(d);
    for (int k = 0; k < 10; ++k) counts[k] = (int64_t)h[k];
}

// ---------------------------------------------------------------------------
// Autotuning of the symmetry-function shapes
// ---------------------------------------------------------------------------

namespace {

std::string tuneCachePath()
{
    if (const char* p = std::getenv("N2P2_B200_TUNE_CACHE")) return p;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/n2p2_b200/autotune.json";
}

void makeParents(std::string const& path)
{
    for (size_t k = 1; k < path.size(); ++k)
        if (path[k] == '/') mkdir(path.substr(0, k).c_str(), 0755);
}

// The cache is a JSON object written one entry per line:
//   "key": {"values": v, "forces": f, "values_ms": [...], "forces_ms": [...]}
std::vector<std::pair<std::string, std::string>> readTuneCache(std::string const& path)
{
    std::vector<std::pair<std::string, std::string>> out;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line))
    {
        size_t a = line.find('"');
        if (a == std::string::npos) continue;
        size_t b = line.find('"', a + 1);
        size_t c = line.find('{', b == std::string::npos ? 0 : b);
        if (b == std::string::npos || c == std::string::npos) continue;
        size_t d = line.rfind('}');
        if (d == std::string::npos || d < c) continue;
        out.emplace_back(line.substr(a + 1, b - a - 1), line.substr(c, d - c + 1));
    }
    return out;
}

bool tuneField(std::string const& body, char const* name, int& v)
{
    std::string k = std::string("\"") + name + "\":";
    size_t p = body.find(k);
    if (p == std::string::npos) return false;
    v = std::atoi(body.c_str() + p + k.size());
    return true;
}

} // namespace

std::string Batch::tuneKey(int precision)
{
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp p{};
    cudaGetDeviceProperties(&p, dev);
    std::string gpu = p.name;
    for (char& c : gpu)
        if (c == '"' || c == ' ') c = '_';
    const DevStatus st = status();
    const double perAtom = N_ ? (double)st.totalNeighbors / N_ : 0.0;
    int nb = 0;
    while ((1 << (nb + 1)) <= N_) ++nb;
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s|sm%d|plan%016llx|p%d|n2^%d|nbr%d", gpu.c_str(), p.multiProcessorCount,
                  (unsigned long long)dmodel_.fingerprint, precision, nb, (int)std::lround(perAtom / 8.0) * 8);
    return buf;
}

void Batch::setShapes(int precision, int values, int forces)
{
    if (precision < 0 || precision > 1 || values < 0 || values >= kSFShapeCount || forces < 0 ||
        forces >= kSFShapeCount)
        throw std::invalid_argument("ERROR: shape variant out of range.\n");
    sfShape_[0][precision] = values;
    sfShape_[1][precision] = forces;
    tuned_[precision] = true;
    releaseGraph();
}

Batch::TuneResult Batch::autotune(int precision, int checkExtrapolation, bool useCache)
{
    if (!capacityVerified_) throw std::runtime_error("ERROR: evaluate the batch once before autotuning.\n");
    TuneResult r;
    const std::string key = tuneKey(precision);
    const std::string path = tuneCachePath();
    if (useCache)
    {
        for (auto const& e : readTuneCache(path))
        {
            int v = -1, f = -1;
            if (e.first == key && tuneField(e.second, "values", v) && tuneField(e.second, "forces", f) && v >= 0 &&
                v < kSFShapeCount && f >= 0 && f < kSFShapeCount)
            {
                r.values = v;
                r.forces = f;
                r.fromCache = true;
            }
        }
    }
    if (!r.fromCache)
    {
        // fill every pass input (neighbour data, dE/dG) once, then time the passes alone
        record(EVAL_FORCES, precision, checkExtrapolation);
        pendingVerify_ = true;
        DevModel const& m = dmodel_.view;
        cudaEvent_t e0, e1;
        cudaCheck(cudaEventCreate(&e0), "event");
        cudaCheck(cudaEventCreate(&e1), "event");
        for (int pass = 0; pass < 2; ++pass)
            for (int v = 0; v < kSFShapeCount; ++v)
            {
                auto launch = [&] {
                    if (pass == 0) launchSFValues(m, dmodel_.groupTable, v_, precision, sms_, stream_, v);
                    else launchSFForces(m, dmodel_.groupTable, v_, precision, sms_, stream_, v);
                };
                launch();
                double best = 1e300;
                for (int rep = 0; rep < 2; ++rep)
                {
                    cudaCheck(cudaEventRecord(e0, stream_), "event");
                    launch();
                    cudaCheck(cudaEventRecord(e1, stream_), "event");
                    cudaCheck(cudaEventSynchronize(e1), "event sync");
                    float ms = 0.f;
                    cudaCheck(cudaEventElapsedTime(&ms, e0, e1), "event time");
                    best = std::min(best, (double)ms);
                }
                (pass == 0 ? r.valuesMs : r.forcesMs)[v] = best;
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaCheck(cudaGetLastError(), "autotune");
        r.values = (int)(std::min_element(r.valuesMs, r.valuesMs + kSFShapeCount) - r.valuesMs);
        r.forces = (int)(std::min_element(r.forcesMs, r.forcesMs + kSFShapeCount) - r.forcesMs);
        // the passes ran with every shape; results are identical whichever ran last
        if (useCache)
        {
            auto entries = readTuneCache(path);
            std::ostringstream body;
            body << "{\"values\": " << r.values << ", \"forces\": " << r.forces << ", \"values_ms\": [";
            for (int v = 0; v < kSFShapeCount; ++v) body << (v ? ", " : "") << r.valuesMs[v];
            body << "], \"forces_ms\": [";
            for (int v = 0; v < kSFShapeCount; ++v) body << (v ? ", " : "") << r.forcesMs[v];
            body << "]}";
            bool replaced = false;
            for (auto& e : entries)
                if (e.first == key)
                {
                    e.second = body.str();
                    replaced = true;
                }
            if (!replaced) entries.emplace_back(key, body.str());
            makeParents(path);
            const std::string tmp = path + ".tmp." + std::to_string((long)getpid());
            {
                std::ofstream f(tmp);
                f << "{\n";
                for (size_t k = 0; k < entries.size(); ++k)
                    f << "  \"" << entries[k].first << "\": " << entries[k].second
                      << (k + 1 < entries.size() ? ",\n" : "\n");
                f << "}\n";
            }
            std::rename(tmp.c_str(), path.c_str());   // atomic replace; a failed write leaves no cache
        }
    }
    sfShape_[0][precision] = r.values;
    sfShape_[1][precision] = r.forces;
    tuned_[precision] = true;
    lastTune_[precision] = r;
    releaseGraph();
    return r;
}

void Batch::requireStructures()
{
    if (N_ == 0) throw std::runtime_error("ERROR: no structures set.\n");
}

void Batch::calculateNeighborList()
{
    requireStructures();
    verify();
    stage_ = StageState{};
    for (int attempt = 0;; ++attempt)
    {
        record(0, PREC_FP64, 0, nullptr, STAGE_NEIGHBORS);
        const DevStatus st = readStatus();
        if (st.totalNeighbors <= capacity_) break;
        if (attempt == 2) throw std::runtime_error("ERROR: neighbour capacity could not be established.\n");
        allocateNeighbors((int64_t)(st.totalNeighbors * 1.05) + 1024);
    }
    stage_.neighbors = true;
}

void Batch::calculateSymmetryFunctions(int derivatives, int precision, int checkExtrapolation)
{
    requireStructures();
    if (derivatives < 0 || derivatives > 2) throw std::invalid_argument("ERROR: derivatives must be 0, 1 or 2.\n");
    if (!stage_.neighbors) throw std::runtime_error("ERROR: neighbour list not calculated.\n");
    // Mode.cpp:1634-1635: skip the whole structure if the results exist
    if (stage_.sfDerivatives && (derivatives < 2 || stage_.sfStored)) return;
    if (stage_.sf && derivatives == 0) return;
    int flags = derivatives ? EVAL_FORCES : 0;
    if (derivatives == 2)
    {
        if (external_) throw std::runtime_error("ERROR: stored dG/dr is not available with external neighbour lists.\n");
        if (dmodel_.view.numCompactGroups > 0)
            throw std::runtime_error("ERROR: stored dG/dr is not available for compact symmetry functions.\n");
        if (precision != PREC_FP64) throw std::runtime_error("ERROR: stored dG/dr is FP64 only.\n");
        allocateDGdr();
        flags |= EVAL_STORE_DGDR;
    }
    record(flags, precision, checkExtrapolation, nullptr, STAGE_SF);
    stage_.sf = true;
    stage_.sfDerivatives = derivatives > 0;
    stage_.sfStored = derivatives == 2;
    stage_.sfPrecision = precision;
    stage_.networks = stage_.dEdG = stage_.energy = stage_.forces = false;
}

void Batch::calculateAtomicNeuralNetworks(int derivatives, int precision)
{
    requireStructures();
    if (!dmodel_.networksSet) throw std::runtime_error("ERROR: weights of element " + dmodel_.missingWeights + " not set.\n");
    if (!stage_.sf) throw std::runtime_error("ERROR: symmetry functions not calculated.\n");
    record(derivatives ? EVAL_FORCES : 0, precision, 0, nullptr, STAGE_NETWORKS);
    stage_.networks = true;
    stage_.dEdG = derivatives != 0;
    stage_.energy = stage_.forces = false;
}

void Batch::calculateEnergy()
{
    requireStructures();
    if (!stage_.networks) throw std::runtime_error("ERROR: atomic neural networks not calculated.\n");
    record(0, PREC_FP64, 0, nullptr, STAGE_ENERGY);
    stage_.energy = true;
}

void Batch::calculateForces()
{
    requireStructures();
    if (!stage_.sfDerivatives) throw std::runtime_error("ERROR: symmetry function derivatives not calculated.\n");
    if (!stage_.dEdG) throw std::runtime_error("ERROR: dE/dG not calculated (atomic networks without derivatives).\n");
    record(EVAL_FORCES | (stage_.sfStored ? EVAL_STORE_DGDR : 0), stage_.sfPrecision, 0, nullptr, STAGE_FORCES);
    stage_.forces = true;
}

void Batch::evaluate(int flags, int precision, int checkExtrapolation)
{
    if (N_ == 0) throw std::runtime_error("ERROR: no structures set.\n");
    if (!dmodel_.networksSet && !(flags & EVAL_SF_ONLY))
        throw std::runtime_error("ERROR: weights of element " + dmodel_.missingWeights + " not set.\n");
    if (flags & EVAL_STORE_DGDR)
    {
        if (external_) throw std::runtime_error("ERROR: stored dG/dr is not available with external neighbour lists.\n");
        if (dmodel_.view.numCompactGroups > 0)
            throw std::runtime_error("ERROR: stored dG/dr is not available for compact symmetry functions.\n");
        if (precision != PREC_FP64) throw std::runtime_error("ERROR: stored dG/dr is FP64 only.\n");
        allocateDGdr();
    }
    {
        const bool sfOnly = (flags & EVAL_SF_ONLY) != 0, f = (flags & EVAL_FORCES) && !sfOnly;
        stage_ = StageState{};
        stage_.neighbors = stage_.sf = true;
        stage_.sfDerivatives = f;
        stage_.sfStored = f && (flags & EVAL_STORE_DGDR);
        stage_.sfPrecision = precision;
        stage_.networks = stage_.energy = !sfOnly;
        stage_.dEdG = stage_.forces = f;
    }
    lastFlags_ = flags;
    lastPrecision_ = precision;
    lastCheck_ = checkExtrapolation;
    pendingVerify_ = false;
    if (!capacityVerified_)
    {
        setStride(0);   // the two-pass build finds the largest count
        for (int attempt = 0; attempt < 3; ++attempt)
        {
            record(flags, precision, checkExtrapolation);
            DevStatus st = readStatus();
            if (st.totalNeighbors <= capacity_) break;
            allocateNeighbors((int64_t)(st.totalNeighbors * 1.05) + 1024);
            if (flags & EVAL_STORE_DGDR) allocateDGdr();
        }
        DevStatus st = readStatus();
        if (st.totalNeighbors > capacity_) throw std::runtime_error("ERROR: neighbour capacity could not be established.\n");
        if ((flags & EVAL_FORCES) && st.maskWords > maskCap_)
        {
            // room for the candidate masks (atoms beyond it test their candidates again)
            releaseGraph();
            freeAll(pool_, ownedMask_);
            maskCap_ = st.maskWords + st.maskWords / 4 + 4096;
            maskBuf_ = devAlloc<uint32_t>(pool_, (size_t)maskCap_, ownedMask_);
        }
        // Later evaluations search once into a fixed stride of the largest count plus 1/8 and 16
        // (the count pass skipped), while N x stride stays within twice the packed entries; an
        // evaluation in which an atom outgrows the stride also runs the fill pass on the device.
        // (the scratch is allocated at the next evaluation: a batch evaluated once never needs it).
        strideWanted_ = 0;
        if (!external_ && st.maxNeighbors > 0)
        {
            const int64_t stride = strideFor(st.maxNeighbors);
            if ((int64_t)N_ * stride <= 2 * capacity_) strideWanted_ = stride;
        }
        capacityVerified_ = true;
        return;
    }
    setStride(strideWanted_);
    if (flags & EVAL_NO_GRAPH)
    {
        record(flags, precision, checkExtrapolation);
        pendingVerify_ = true;
        verify();
        return;
    }
    const int key = (flags & (EVAL_FORCES | EVAL_STORE_DGDR | EVAL_SF_ONLY)) | (precision << 4) |
                    ((checkExtrapolation ? 1 : 0) << 5);
    if (autotuneEnabled && !tuned_[precision] && !(flags & EVAL_STORE_DGDR)) autotune(precision, checkExtrapolation, true);
    if (graphExec_ == nullptr || graphKey_ != key)
    {
        releaseGraph();
        cudaGraph_t graph;
        cudaCheck(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed), "begin capture");
        try
        {
            record(flags, precision, checkExtrapolation);
        }
        catch (...)
        {
            cudaStreamEndCapture(stream_, &graph);
            throw;
        }
        cudaCheck(cudaStreamEndCapture(stream_, &graph), "end capture");
        cudaCheck(cudaGraphInstantiate(&graphExec_, graph, 0), "graph instantiate");
        cudaGraphDestroy(graph);
        graphKey_ = key;
    }
    cudaCheck(cudaGraphLaunch(graphExec_, stream_), "graph launch");
    pendingVerify_ = true;
}

void Batch::verify()
{
    if (!pendingVerify_) return;
    pendingVerify_ = false;
    const DevStatus st = readStatus();
    // An atom that outgrew the search stride made the evaluation run its fill pass as well (the
    // results are complete); later evaluations search into a wider stride, recorded anew.
    if (nbrStride_ > 0 && st.maxNeighbors > nbrStride_)
    {
        const int64_t stride = strideFor(st.maxNeighbors);
        strideWanted_ = (int64_t)N_ * stride <= 2 * capacity_ ? stride : 0;
    }
    if (st.totalNeighbors <= capacity_) return;
    // The lists outgrew the buffers sized at the first evaluation: size them
    // again and repeat the evaluation directly (the graph is recaptured at
    // the next call).
    ++overflowRecoveries_;
    capacityVerified_ = false;
    evaluate(lastFlags_, lastPrecision_, lastCheck_);
}

void Batch::synchronize() { cudaCheck(cudaStreamSynchronize(stream_), "synchronize"); }

DevStatus Batch::status()
{
    verify();
    return readStatus();
}

DevStatus Batch::readStatus()
{
    DevStatus st{};
    cudaCheck(cudaMemcpyAsync(&st, v_.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream_), "status D2H");
    synchronize();
    if (st.badInput) throw std::runtime_error("ERROR: invalid input detected on the device (atoms outside the cell, "
                                              "asymmetric neighbour pairs or more than 2048 neighbours).\n");
    if (st.tensorCoreTimeout) throw std::runtime_error("ERROR: a tensor-core network tile timed out waiting for its "
                                                       "matrix products.\n");
    return st;
}

int64_t Batch::numNeighborEntries()
{
    verify();
    int64_t total = 0;
    cudaCheck(cudaMemcpyAsync(&total, v_.nbrOffset + N_, sizeof(int64_t), cudaMemcpyDeviceToHost, stream_), "D2H");
    synchronize();
    return total;
}

void Batch::energies(double* out)
{
    verify();
    std::vector<double> e(S_);
    cudaCheck(cudaMemcpyAsync(e.data(), v_.Estruct, sizeof(double) * S_, cudaMemcpyDeviceToHost, stream_), "E D2H");
    synchronize();
    const int ne = (int)model_.numElements();
    for (int k = 0; k < S_; ++k)
    {
        double E = e[k];
        // Structure::toPhysicalUnits (Structure.cpp:1279-1306) and
        // Mode::addEnergyOffset (Mode.cpp:2079-2097)
        if (model_.normalize) E = E / model_.convEnergy + structs_[k].numAtoms * model_.meanEnergy;
        for (int q = 0; q < ne; ++q)
            E += numAtomsPerElement_[(size_t)k * ne + q] * model_.elements[q].atomicEnergyOffset;
        out[k] = E;
    }
}

void Batch::energiesToInternal(const double* phys, double* out) const
{
    const int ne = (int)model_.numElements();
    for (int k = 0; k < S_; ++k)
    {
        double E = phys[k];
        for (int q = 0; q < ne; ++q)
            E -= numAtomsPerElement_[(size_t)k * ne + q] * model_.elements[q].atomicEnergyOffset;
        if (model_.normalize) E = (E - structs_[k].numAtoms * model_.meanEnergy) * model_.convEnergy;
        out[k] = E;
    }
}

double Batch::forceToInternal() const
{
    return model_.normalize ? model_.convEnergy / model_.convLength : 1.0;
}

void Batch::forces(double* out)
{
    verify();
    cudaCheck(cudaMemcpyAsync(out, v_.F, sizeof(double) * 3 * (size_t)N_, cudaMemcpyDeviceToHost, stream_), "F D2H");
    synchronize();
    if (model_.normalize)
    {
        // Atom::toPhysicalUnits: f /= convEnergy / convLength (Atom.cpp:123-130)
        const double c = model_.convEnergy / model_.convLength;
        for (size_t q = 0; q < 3 * (size_t)N_; ++q) out[q] /= c;
    }
}

void Batch::copyNeighbors(int64_t* offsets, int* index, int* image, double* d, double* dr)
{
    verify();
    std::vector<int64_t> off(N_ + 1);
    cudaCheck(cudaMemcpy(off.data(), v_.nbrOffset, sizeof(int64_t) * (N_ + 1), cudaMemcpyDeviceToHost), "D2H");
    const int64_t M = off[N_];
    if (offsets) std::memcpy(offsets, off.data(), sizeof(int64_t) * (N_ + 1));
    if (index) cudaCheck(cudaMemcpy(index, v_.nbrJ, sizeof(int) * M, cudaMemcpyDeviceToHost), "D2H");
    if (image) cudaCheck(cudaMemcpy(image, v_.nbrCode, sizeof(int) * M, cudaMemcpyDeviceToHost), "D2H");
    if (d) cudaCheck(cudaMemcpy(d, v_.nbrD, sizeof(double) * M, cudaMemcpyDeviceToHost), "D2H");
    if (dr)
    {
        std::vector<double> x(M), y(M), z(M);
        cudaCheck(cudaMemcpy(x.data(), v_.nbrDx, sizeof(double) * M, cudaMemcpyDeviceToHost), "D2H");
        cudaCheck(cudaMemcpy(y.data(), v_.nbrDy, sizeof(double) * M, cudaMemcpyDeviceToHost), "D2H");
        cudaCheck(cudaMemcpy(z.data(), v_.nbrDz, sizeof(double) * M, cudaMemcpyDeviceToHost), "D2H");
        for (int64_t e = 0; e < M; ++e)
        {
            dr[3 * e + 0] = x[e];
            dr[3 * e + 1] = y[e];
            dr[3 * e + 2] = z[e];
        }
    }
}

namespace {
void packPerAtom(std::vector<double> const& src, int stride, std::vector<int> const& elem, Model const& m, double* out)
{
    size_t k = 0;
    for (size_t a = 0; a < elem.size(); ++a)
    {
        int ns = (int)m.elements[elem[a]].sf.size();
        for (int s = 0; s < ns; ++s) out[k++] = src[a * stride + s];
    }
}
} // namespace

void Batch::copyG(double* out)
{
    verify();
    std::vector<double> g((size_t)N_ * v_.gStride);
    cudaCheck(cudaMemcpy(g.data(), v_.G, sizeof(double) * g.size(), cudaMemcpyDeviceToHost), "D2H");
    packPerAtom(g, v_.gStride, elemHost_, model_, out);
}

void Batch::copyDEdG(double* out)
{
    verify();
    std::vector<double> g((size_t)N_ * v_.gStride);
    cudaCheck(cudaMemcpy(g.data(), v_.dEdG, sizeof(double) * g.size(), cudaMemcpyDeviceToHost), "D2H");
    packPerAtom(g, v_.gStride, elemHost_, model_, out);
}

void Batch::copyAtomicEnergies(double* out)
{
    verify();
    cudaCheck(cudaMemcpy(out, v_.Eatom, sizeof(double) * N_, cudaMemcpyDeviceToHost), "D2H");
}

void Batch::sfStatistics(int64_t* counts, double* stats)
{
    verify();
    const int ne = (int)model_.numElements();
    const int maxSF = std::max(dmodel_.maxSF, 1);
    int largest = 0;
    for (int e = 0; e < ne; ++e)
    {
        counts[e] = v_.elemBegin[e + 1] - v_.elemBegin[e];
        largest = std::max(largest, (int)counts[e]);
    }
    const int maxChunks = std::max(1, (largest + 1023) / 1024);
    std::vector<void*> tmp;
    double* partial = devAlloc<double>(pool_, (size_t)ne * maxChunks * 4 * maxSF, tmp);
    double* result = devAlloc<double>(pool_, (size_t)ne * 4 * maxSF, tmp);
    cudaCheck(cudaMemsetAsync(result, 0, sizeof(double) * (size_t)ne * 4 * maxSF, stream_), "memset");
    launchSFStatistics(dmodel_.view, v_, ne, maxChunks, maxSF, partial, result, stream_);
    cudaCheck(cudaGetLastError(), "statistics launch");
    cudaCheck(cudaMemcpyAsync(stats, result, sizeof(double) * (size_t)ne * 4 * maxSF, cudaMemcpyDeviceToHost, stream_),
              "statistics D2H");
    synchronize();
    freeAll(pool_, tmp);
}

void Batch::copyAtomWarnings(int* out)
{
    verify();
    cudaCheck(cudaMemcpy(out, v_.atomWarnings, sizeof(int) * N_, cudaMemcpyDeviceToHost), "D2H");
}

void Batch::copyPositions(double* out)
{
    verify();
    std::vector<double> x(N_), y(N_), z(N_);
    cudaCheck(cudaMemcpy(x.data(), v_.px, sizeof(double) * N_, cudaMemcpyDeviceToHost), "D2H");
    cudaCheck(cudaMemcpy(y.data(), v_.py, sizeof(double) * N_, cudaMemcpyDeviceToHost), "D2H");
    cudaCheck(cudaMemcpy(z.data(), v_.pz, sizeof(double) * N_, cudaMemcpyDeviceToHost), "D2H");
    for (int a = 0; a < N_; ++a)
    {
        out[3 * a + 0] = x[a];
        out[3 * a + 1] = y[a];
        out[3 * a + 2] = z[a];
    }
}

void Batch::copyDGdr(double* self, double* nbr)
{
    verify();
    if (!dgdrAllocated_) throw std::runtime_error("ERROR: dG/dr was not stored (evaluate with the store flag).\n");
    std::vector<int64_t> off(N_ + 1);
    cudaCheck(cudaMemcpy(off.data(), v_.nbrOffset, sizeof(int64_t) * (N_ + 1), cudaMemcpyDeviceToHost), "D2H");
    const int64_t M = off[N_];
    std::vector<int> J(M);
    cudaCheck(cudaMemcpy(J.data(), v_.nbrJ, sizeof(int) * M, cudaMemcpyDeviceToHost), "D2H");
    if (self)
    {
        std::vector<double> s((size_t)N_ * v_.gStride * 3);
        cudaCheck(cudaMemcpy(s.data(), v_.dGdrSelf, sizeof(double) * s.size(), cudaMemcpyDeviceToHost), "D2H");
        size_t k = 0;
        for (int a = 0; a < N_; ++a)
        {
            int ns = (int)model_.elements[elemHost_[a]].sf.size();
            for (int q = 0; q < ns * 3; ++q) self[k++] = s[(size_t)a * v_.gStride * 3 + q];
        }
    }
    if (nbr)
    {
        const int rowsMax = std::max(1, dmodel_.view.maxRows);
        std::vector<double> rowbuf((size_t)M * 3);
        size_t k = 0;
        // rows of entry e follow the centre element's table for the neighbour element
        std::vector<int> rowsOf(M);
        for (int a = 0; a < N_; ++a)
            for (int64_t e = off[a]; e < off[a + 1]; ++e)
                rowsOf[e] = (int)model_.elements[elemHost_[a]].table[elemHost_[J[e]]].size();
        std::vector<std::vector<double>> rows(rowsMax);
        for (int r = 0; r < rowsMax; ++r)
        {
            rows[r].resize((size_t)M * 3);
            cudaCheck(cudaMemcpy(rows[r].data(), v_.dGdr + (size_t)r * capacity_ * 3, sizeof(double) * M * 3,
                                 cudaMemcpyDeviceToHost),
                      "D2H");
        }
        for (int64_t e = 0; e < M; ++e)
            for (int r = 0; r < rowsOf[e]; ++r)
                for (int c = 0; c < 3; ++c) nbr[k++] = rows[r][(size_t)e * 3 + c];
    }
}

} // namespace n2p2b200
