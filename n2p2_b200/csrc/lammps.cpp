// LAMMPS interface, host side (see lammps.hpp).
#include "lammps.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <thread>
#include <vector>

namespace n2p2b200 {

namespace {

std::vector<std::string> splitOn(std::string const& s, char sep)
{
    std::vector<std::string> out;
    std::string cur;
    for (char c : s)
    {
        if (c == sep)
        {
            out.push_back(cur);
            cur.clear();
        }
        else cur += c;
    }
    out.push_back(cur);
    return out;
}

std::string format(char const* fmt, long long a, long long b)
{
    char buf[256];
    std::snprintf(buf, sizeof(buf), fmt, a, b);
    return buf;
}

constexpr int kNeighMask = 0x1FFFFFFF;   // LAMMPS NEIGHMASK: special-bond bits above it

} // namespace

void LammpsInterface::initialize(Model const& model, std::string const& emap, double cflength, double cfenergy,
                                 double lammpsCutoff, int lammpsNtypes, int myRank)
{
    if (!model.setupDone) throw std::runtime_error("ERROR: the model is not set up.\n");
    initialized_ = false;
    cflength_ = cflength;
    cfenergy_ = cfenergy;
    myRank_ = myRank;
    normalize_ = model.normalize;
    convLength_ = model.convLength;
    convEnergy_ = model.convEnergy;
    meanEnergy_ = model.meanEnergy;
    rcmax_ = model.maxCutoffRadius;
    offsets_.clear();
    for (auto const& e : model.elements) offsets_.push_back(e.atomicEnergyOffset);
    if (lammpsCutoff < maxCutoffRadius())
        throw std::runtime_error("ERROR: LAMMPS cutoff via pair_coeff keyword is smaller than maximum symmetry "
                                 "function cutoff.\n");
    typeToElement_.clear();
    const size_t ne = model.numElements();
    if (emap.empty())
    {
        if (ne != (size_t)lammpsNtypes)
            throw std::runtime_error(format("ERROR: No element mapping given and number of LAMMPS atom types (%lld) "
                                            "and NNP elements (%lld) does not match.\n",
                                            lammpsNtypes, (long long)ne));
        for (int t = 1; t <= lammpsNtypes; ++t) typeToElement_[t] = t - 1;
    }
    else
    {
        std::string compact;   // blanks and tabs removed
        for (char c : emap)
            if (c != ' ' && c != '\t') compact += c;
        std::vector<std::string> pairs = splitOn(compact, ',');
        if (ne < pairs.size())
            throw std::runtime_error(format("ERROR: Element mapping is inconsistent, NNP elements: %lld, emap "
                                            "elements: %lld.\n",
                                            (long long)ne, (long long)pairs.size()));
        for (auto const& p : pairs)
        {
            std::vector<std::string> ts = splitOn(p, ':');
            if (ts.size() != 2) throw std::runtime_error("ERROR: Invalid element mapping string: \"" + p + "\".\n");
            const int t = std::stoi(ts[0]);
            if (t > lammpsNtypes)
                throw std::runtime_error(format("ERROR: LAMMPS type \"%lld\" not present, there are only %lld types "
                                                "defined.\n",
                                                t, lammpsNtypes));
            typeToElement_[t] = model.elementMap.index(ts[1]);
        }
    }
    ignoreType_.assign((size_t)std::max(lammpsNtypes, 0) + 1, true);
    typeElement_.assign((size_t)std::max(lammpsNtypes, 0) + 1, -1);
    for (int t = 1; t <= lammpsNtypes; ++t)
    {
        auto it = typeToElement_.find(t);
        ignoreType_[t] = it == typeToElement_.end();
        if (!ignoreType_[t]) typeElement_[t] = it->second;
    }
    indexMap_.clear();
    center_.clear();
    dirty_ = true;
    initialized_ = true;
}

double LammpsInterface::maxCutoffRadius() const
{
    return normalize_ ? rcmax_ / convLength_ / cflength_ : rcmax_ / cflength_;
}

void LammpsInterface::setLocalAtoms(int numAtomsLocal, const int* atomType)
{
    if (!initialized_) throw std::runtime_error("ERROR: the LAMMPS interface is not initialized.\n");
    if (numAtomsLocal < 0) throw std::invalid_argument("ERROR: negative number of local atoms.\n");
    indexMap_.assign((size_t)numAtomsLocal, -1);
    center_.clear();
    centerElement_.clear();
    for (int i = 0; i < numAtomsLocal; ++i)
    {
        const int t = atomType[i];
        if (t < 1 || t >= (int)ignoreType_.size()) throw std::out_of_range("ERROR: LAMMPS atom type out of range.\n");
        if (ignoreType_[t]) continue;
        indexMap_[i] = (int)center_.size();
        center_.push_back(i);
        centerElement_.push_back(typeToElement_.at(t));
    }
    lists_ = LISTS_NONE;
    eCenter_.clear();
    eJ_.clear();
    eElem_.clear();
    eDr_.clear();
    eD_.clear();
    eOrdered_ = true;
    dirty_ = true;
    haveAtomic_ = false;
}

void LammpsInterface::addNeighbor(int i, int j, int type, double dx, double dy, double dz, double d2)
{
    if (i < 0 || i >= (int)indexMap_.size()) throw std::out_of_range("ERROR: local atom index out of range.\n");
    if (j < 0) throw std::out_of_range("ERROR: negative neighbour index.\n");
    if (type < 1 || type >= (int)ignoreType_.size()) throw std::out_of_range("ERROR: LAMMPS atom type out of range.\n");
    if (lists_ == LISTS_TRANSFERRED)
        throw std::runtime_error("ERROR: this step's lists were transferred in one call; addNeighbor does not "
                                 "extend them.\n");
    lists_ = LISTS_ADDED;
    if (ignoreType_[type] || indexMap_[i] < 0) return;
    // unit conversion in the order of InterfaceLammps::addNeighbor
    double rx = dx * cflength_, ry = dy * cflength_, rz = dz * cflength_;
    double d = std::sqrt(d2) * cflength_;
    if (normalize_)
    {
        rx *= convLength_;
        ry *= convLength_;
        rz *= convLength_;
        d *= convLength_;
    }
    // every symmetry-function group takes neighbours with d < r_c only: one
    // beyond the largest cutoff contributes nothing
    if (!(d <= rcmax_)) return;
    const int c = indexMap_[i];
    if (!eCenter_.empty() && c < eCenter_.back()) eOrdered_ = false;
    eCenter_.push_back(c);
    eJ_.push_back(j);
    eElem_.push_back(typeElement_[type]);
    eDr_.push_back(rx);
    eDr_.push_back(ry);
    eDr_.push_back(rz);
    eD_.push_back(d);
    dirty_ = true;
}

void* LammpsInterface::Pinned::ensure(size_t n)
{
    if (n > bytes)
    {
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        const size_t want = n + n / 4 + 4096;
        cudaCheck(cudaHostAlloc(&p, want, cudaHostAllocPortable), "cudaHostAlloc");
        bytes = want;
    }
    return p;
}

LammpsInterface::Pinned::~Pinned()
{
    if (p) cudaFreeHost(p);
}

LammpsInterface::~LammpsInterface() = default;

void LammpsInterface::transferNeighborList(int inum, const int* ilist, const int* numneigh,
                                           const int* const* firstneigh, const double* const* x, const int* type,
                                           double pairCutoff)
{
    if (!initialized_) throw std::runtime_error("ERROR: the LAMMPS interface is not initialized.\n");
    if (lists_ != LISTS_NONE)
        throw std::runtime_error("ERROR: this step already has neighbours (set the local atoms again first).\n");
    const int nLocal = (int)indexMap_.size();
    std::vector<char> listed((size_t)nLocal, 0);
    for (int ii = 0; ii < inum; ++ii)
    {
        const int i = ilist[ii];
        if (i < 0 || i >= nLocal) throw std::out_of_range("ERROR: local atom index out of range.\n");
        listed[i] = 1;
    }
    // candidates of every centre, in centre order, special-bond bits masked
    const int n = (int)center_.size();
    int64_t total = 0;
    for (int c = 0; c < n; ++c)
        if (listed[center_[c]]) total += numneigh[center_[c]];
    auto* off = static_cast<int64_t*>(candOffBuf_.ensure(sizeof(int64_t) * ((size_t)n + 1)));
    auto* cand = static_cast<int*>(candBuf_.ensure(sizeof(int) * (size_t)std::max<int64_t>(total, 1)));
    off[0] = 0;
    for (int c = 0; c < n; ++c) off[c + 1] = off[c] + (listed[center_[c]] ? numneigh[center_[c]] : 0);
    // the gather itself by host threads over ranges of centres (each writes its own segments)
    auto gather = [&](int c0, int c1) {
        int mx = 0;
        for (int c = c0; c < c1; ++c)
        {
            const int i = center_[c];
            mx = std::max(mx, i);
            if (!listed[i]) continue;
            const int* nb = firstneigh[i];
            int* out = cand + off[c];
            for (int q = 0; q < numneigh[i]; ++q)
            {
                const int j = nb[q] & kNeighMask;
                out[q] = j;
                mx = std::max(mx, j);
            }
        }
        return mx;
    };
    int maxIndex = 0;
    const int threads = total >= (1 << 20) ? (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency())) : 1;
    if (threads <= 1) maxIndex = gather(0, n);
    else
    {
        std::vector<int> mx((size_t)threads, 0);
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t)
        {
            const int c0 = (int)((int64_t)n * t / threads), c1 = (int)((int64_t)n * (t + 1) / threads);
            pool.emplace_back([&, t, c0, c1] { mx[(size_t)t] = gather(c0, c1); });
        }
        for (auto& th : pool) th.join();
        for (int v : mx) maxIndex = std::max(maxIndex, v);
    }
    numCand_ = off[n];
    numAll_ = maxIndex + 1;
    auto* xs = static_cast<double*>(xBuf_.ensure(sizeof(double) * 3 * (size_t)numAll_));
    auto* ts = static_cast<int*>(typeBuf_.ensure(sizeof(int) * (size_t)numAll_));
    for (int k = 0; k < numAll_; ++k)
    {
        xs[3 * (size_t)k + 0] = x[k][0];
        xs[3 * (size_t)k + 1] = x[k][1];
        xs[3 * (size_t)k + 2] = x[k][2];
        ts[k] = type[k];
    }
    pairCut2_ = pairCutoff * pairCutoff;
    lists_ = LISTS_TRANSFERRED;
    dirty_ = true;
}

void LammpsInterface::process(Batch& batch, int precision, bool checkExtrapolation)
{
    if (!initialized_) throw std::runtime_error("ERROR: the LAMMPS interface is not initialized.\n");
    haveAtomic_ = false;
    if (center_.empty())
    {
        energy_ = 0.0;
        return;
    }
    if (dirty_)
    {
        const int n = (int)center_.size();
        if (lists_ == LISTS_TRANSFERRED)
        {
            Batch::ExternalLists l;
            l.numCenters = n;
            l.centerElement = centerElement_.data();
            l.centerIndex = center_.data();
            l.candOffset = static_cast<const int64_t*>(candOffBuf_.p);
            l.cand = static_cast<const int*>(candBuf_.p);
            l.numCand = numCand_;
            l.numAll = numAll_;
            l.x = static_cast<const double*>(xBuf_.p);
            l.type = static_cast<const int*>(typeBuf_.p);
            l.typeElement = typeElement_.data();
            l.numTypes = (int)typeElement_.size() - 1;
            l.cflength = cflength_;
            l.convLength = convLength_;
            l.normalize = normalize_;
            l.pairCut2 = pairCut2_;
            batch.setExternalLists(l);
        }
        else
        {
            // addNeighbor entries (or none): centre-major CSR, call order within a centre
            const size_t E = eCenter_.size();
            std::vector<int64_t> offsets((size_t)n + 1, 0);
            for (size_t e = 0; e < E; ++e) offsets[(size_t)eCenter_[e] + 1]++;
            for (int c = 0; c < n; ++c) offsets[c + 1] += offsets[c];
            std::vector<int> target(std::max<size_t>(E, 1)), elem(std::max<size_t>(E, 1));
            std::vector<double> dr(3 * std::max<size_t>(E, 1)), d(std::max<size_t>(E, 1));
            std::vector<int64_t> fill(offsets.begin(), offsets.end() - 1);
            int numTargets = 0;
            for (int c = 0; c < n; ++c) numTargets = std::max(numTargets, center_[c] + 1);
            for (size_t e = 0; e < E; ++e)
            {
                const size_t at = eOrdered_ ? e : (size_t)fill[eCenter_[e]]++;
                target[at] = eJ_[e];
                elem[at] = eElem_[e];
                d[at] = eD_[e];
                dr[3 * at + 0] = eDr_[3 * e + 0];
                dr[3 * at + 1] = eDr_[3 * e + 1];
                dr[3 * at + 2] = eDr_[3 * e + 2];
                numTargets = std::max(numTargets, eJ_[e] + 1);
            }
            batch.setExternalNeighbors(n, centerElement_.data(), (int64_t)E, offsets.data(), numTargets,
                                       target.data(), elem.data(), dr.data(), d.data(), center_.data());
        }
        dirty_ = false;
    }
    batch.evaluate(EVAL_FORCES, precision, checkExtrapolation ? 1 : 0);
    double E = 0.0;
    batch.energies(&E);   // Structure::toPhysicalUnits and Mode::addEnergyOffset
    energy_ = E;
}

double LammpsInterface::atomicEnergy(Batch& batch, int index)
{
    if (index < 0 || index >= (int)center_.size()) throw std::out_of_range("ERROR: atom index out of range.\n");
    if (!haveAtomic_)
    {
        atomicEnergy_.resize(center_.size());
        batch.copyAtomicEnergies(atomicEnergy_.data());
        haveAtomic_ = true;
    }
    const double off = offsets_[centerElement_[index]];
    if (normalize_) return (atomicEnergy_[index] / convEnergy_ + meanEnergy_ + off) / cfenergy_;
    return (atomicEnergy_[index] + off) / cfenergy_;
}

void LammpsInterface::addForces(Batch& batch, double* const* atomF)
{
    if (center_.empty()) return;
    const int T = batch.numTargets();
    std::vector<double> F(3 * (size_t)T);
    batch.targetForces(F.data());
    const double cfforce = cflength_ / cfenergy_;
    const double convForce = normalize_ ? convLength_ / convEnergy_ : 1.0;
    for (int k = 0; k < T; ++k)
        for (int q = 0; q < 3; ++q) atomF[k][q] += F[3 * (size_t)k + q] * cfforce * convForce;
}

} // namespace n2p2b200
