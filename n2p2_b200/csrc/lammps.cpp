// LAMMPS interface, host side (see lammps.hpp).
#include "lammps.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <stdexcept>

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
    for (int t = 1; t <= lammpsNtypes; ++t) ignoreType_[t] = typeToElement_.find(t) == typeToElement_.end();
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
    const size_t n = center_.size();
    nbrJ_.assign(n, {});
    nbrElem_.assign(n, {});
    nbrDr_.assign(n, {});
    nbrD_.assign(n, {});
    dirty_ = true;
    haveAtomic_ = false;
}

void LammpsInterface::addNeighbor(int i, int j, int type, double dx, double dy, double dz, double d2)
{
    if (i < 0 || i >= (int)indexMap_.size()) throw std::out_of_range("ERROR: local atom index out of range.\n");
    if (j < 0) throw std::out_of_range("ERROR: negative neighbour index.\n");
    if (type < 1 || type >= (int)ignoreType_.size()) throw std::out_of_range("ERROR: LAMMPS atom type out of range.\n");
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
    nbrJ_[c].push_back(j);
    nbrElem_[c].push_back(typeToElement_.at(type));
    nbrDr_[c].push_back(rx);
    nbrDr_[c].push_back(ry);
    nbrDr_[c].push_back(rz);
    nbrD_[c].push_back(d);
    dirty_ = true;
}

void LammpsInterface::transferNeighborList(int inum, const int* ilist, const int* numneigh,
                                           const int* const* firstneigh, const double* const* x, const int* type,
                                           double pairCutoff)
{
    const double rc2 = pairCutoff * pairCutoff;
    for (int ii = 0; ii < inum; ++ii)
    {
        const int i = ilist[ii];
        for (int jj = 0; jj < numneigh[i]; ++jj)
        {
            const int j = firstneigh[i][jj] & kNeighMask;
            const double dx = x[i][0] - x[j][0];
            const double dy = x[i][1] - x[j][1];
            const double dz = x[i][2] - x[j][2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 <= rc2) addNeighbor(i, j, type[j], dx, dy, dz, d2);
        }
    }
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
        std::vector<int64_t> offsets((size_t)n + 1, 0);
        for (int c = 0; c < n; ++c) offsets[c + 1] = offsets[c] + (int64_t)nbrJ_[c].size();
        const size_t E = (size_t)offsets[n];
        std::vector<int> target(std::max<size_t>(E, 1)), elem(std::max<size_t>(E, 1));
        std::vector<double> dr(3 * std::max<size_t>(E, 1)), d(std::max<size_t>(E, 1));
        int numTargets = 0;
        for (int c = 0; c < n; ++c)
        {
            numTargets = std::max(numTargets, center_[c] + 1);
            size_t e0 = (size_t)offsets[c];
            for (size_t q = 0; q < nbrJ_[c].size(); ++q)
            {
                target[e0 + q] = nbrJ_[c][q];
                elem[e0 + q] = nbrElem_[c][q];
                d[e0 + q] = nbrD_[c][q];
                for (int k = 0; k < 3; ++k) dr[3 * (e0 + q) + k] = nbrDr_[c][3 * q + k];
                numTargets = std::max(numTargets, nbrJ_[c][q] + 1);
            }
        }
        batch.setExternalNeighbors(n, centerElement_.data(), (int64_t)E, offsets.data(), numTargets, target.data(),
                                   elem.data(), dr.data(), d.data(), center_.data());
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
