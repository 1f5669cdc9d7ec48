// Test-oracle harness around the REFERENCE n2p2 library (libnnp), compiled
// from the reference's own sources by oracle/Makefile into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY: tests/, the smoke check and bench.py's
// cpu_baseline / --impl reference leg load this library as the checker or as
// the timed CPU baseline.  The product never links it.
//
// The harness drives the reference exactly like Prediction::setup() /
// readStructureFromFile() / predict() (Prediction.cpp:36-78) and, between
// evaluateNNP (Mode.cpp:2029-2077) and the conversion back to physical units,
// snapshots the internal arrays (neighbour lists, G, dEdG, dGdr, atomic
// energies) so the GPU path can be compared item by item.
#include "Mode.h"
#include "Structure.h"
#include "Atom.h"
#include "Element.h"
#include "NeuralNetwork.h"
#include "utility.h"

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

using namespace std;
using namespace nnp;

namespace {

thread_local std::string g_err;

class RefMode : public Mode
{
public:
    // Same sequence as Prediction::setup() (Prediction.cpp:36-48); the
    // statistics flags are caller-chosen so timed runs can switch off the
    // stderr extrapolation warnings.
    void setupFromDir(string const& dir, bool writeExtrapolationWarnings)
    {
        log.writeToStdout = false;
        initialize();
        loadSettingsFile(dir + "/input.nn");
        setupGeneric(dir);
        setupSymmetryFunctionScaling(dir + "/scaling.data");
        map<string, string> formats{{"short", dir + "/weights.%03zu.data"},
                                    {"elec", dir + "/weightse.%03zu.data"}};
        setupNeuralNetworkWeights(formats);
        setupSymmetryFunctionStatistics(false, false,
                                        writeExtrapolationWarnings, false);
    }

    // Prediction::readStructureFromFile (Prediction.cpp:50-65) on a text block.
    void readStructure(Structure& s, string const& text)
    {
        s.reset();
        s.setElementMap(elementMap);
        vector<string> lines;
        istringstream in(text);
        string line;
        while (getline(in, line)) if (!line.empty()) lines.push_back(line);
        s.readFromLines(lines);
        removeEnergyOffset(s);
        if (normalize) s.toNormalizedUnits(meanEnergy, convEnergy, convLength, convCharge);
    }

    // Prediction::predict (Prediction.cpp:67-78) split around the snapshot.
    void finish(Structure& s)
    {
        if (normalize) s.toPhysicalUnits(meanEnergy, convEnergy, convLength, convCharge);
        addEnergyOffset(s, false);
        addEnergyOffset(s, true);
    }

    size_t numSF(size_t e) const { return elements.at(e).numSymmetryFunctions(); }
    size_t numRows(size_t ec, size_t en) const { return elements.at(ec).getSymmetryFunctionNumTable().at(en); }
    size_t nElem() const { return numElements; }
    double maxRc() const { return maxCutoffRadius; }
    // the per-structure work of nnp-scaling (nnp-scaling.cpp: neighbour list,
    // Mode::calculateSymmetryFunctionGroups without derivatives)
    void symmetryFunctionsOnly(Structure& s)
    {
        s.calculateNeighborList(maxCutoffRadius, false);
        calculateSymmetryFunctionGroups(s, false);
    }
    // Jacobian of one training observation with respect to every network
    // weight (elements in index order, each in its weight-file order), as
    // Training::update assembles it for 2G networks (Training.cpp:2582-2690)
    // from the reference's own NeuralNetwork::calculateDEdc (an energy: the
    // sum over the structure's atoms) and NeuralNetwork::calculateDFdc (force
    // component c of atom a: the sum over atoms of calculateDFdc with the
    // atom's dG/dx_{a,c}).  dG/dx_{a,c} is gathered as
    // Training::collectDGdxia does (Training.cpp:3590-3631, restated because
    // the training library is not built: the rows of the atom's neighbour
    // entries that name atom a, mapped through the element's symmetry
    // function table, plus the atom's own dG/dr when it is atom a).  Needs a
    // structure evaluated with forces (dG/dr stored).
    void jacobian(Structure& s, int property, size_t a, size_t c, vector<double>& out)
    {
        vector<size_t> offset(numElements + 1, 0);
        for (size_t e = 0; e < numElements; ++e)
            offset[e + 1] = offset[e] + (size_t)elements.at(e).neuralNetworks.at("short").getNumConnections();
        out.assign(offset[numElements], 0.0);
        vector<double> d;
        for (Atom& at : s.atoms)
        {
            NeuralNetwork& nn = elements.at(at.element).neuralNetworks.at("short");
            d.assign((size_t)nn.getNumConnections(), 0.0);
            for (size_t j = 0; j < at.G.size(); ++j) nn.setInput(j, at.G.at(j));
            nn.propagate();
            if (property == 0) nn.calculateDEdc(d.data());
            else
            {
                vector<double> dGdxia(at.numSymmetryFunctions, 0.0);
                vector<vector<size_t>> const& tableFull = elements.at(at.element).getSymmetryFunctionTable();
                for (size_t n = 0; n < at.numNeighbors; ++n)
                {
                    Atom::Neighbor const& nb = at.neighbors[n];
                    if (nb.index != a) continue;
                    vector<size_t> const& table = tableFull.at(nb.element);
                    for (size_t q = 0; q < nb.dGdr.size(); ++q) dGdxia[table.at(q)] += nb.dGdr[q][c];
                }
                if (at.index == a)
                    for (size_t q = 0; q < at.numSymmetryFunctions; ++q) dGdxia[q] += at.dGdr[q][c];
                bool any = false;
                for (double x : dGdxia) any = any || x != 0.0;
                if (!any) continue;   // an atom without atom a among its neighbours adds exact zeros
                nn.calculateDFdc(d.data(), dGdxia.data());
            }
            for (size_t q = 0; q < d.size(); ++q) out[offset[at.element] + q] += d[q];
        }
    }
};

struct Snapshot
{
    // internal (normalised) units, taken right after evaluateNNP
    vector<double>  r;          // 3N remapped positions
    vector<double>  box;        // 9
    vector<int64_t> nbrOffset;  // N+1
    vector<int64_t> nbrIndex;   // M
    vector<double>  nbrD;       // M
    vector<double>  nbrDr;      // 3M
    vector<int64_t> sfOffset;   // N+1 (in SF units)
    vector<double>  G;
    vector<double>  dEdG;
    vector<double>  dGdrSelf;   // 3 * sum(numSF)
    vector<int64_t> rowOffset;  // M+1 (in rows)
    vector<double>  dGdrNbr;    // 3 * total rows
    vector<double>  atomicEnergy;
    vector<double>  forcesInternal;
    double          energyInternal = 0.0;
    // physical units, after Prediction::predict's conversion
    double          energy = 0.0;
    vector<double>  forces;
};

struct Handle
{
    RefMode  mode;
    Snapshot snap;
    string   dir;
};

void takeSnapshot(Handle& h, Structure& s, bool useForces)
{
    Snapshot& o = h.snap;
    o = Snapshot();
    size_t N = s.atoms.size();
    for (int k = 0; k < 3; ++k)
        for (int c = 0; c < 3; ++c) o.box.push_back(s.box[k][c]);
    o.nbrOffset.push_back(0);
    o.sfOffset.push_back(0);
    o.rowOffset.push_back(0);
    for (size_t i = 0; i < N; ++i)
    {
        Atom const& a = s.atoms[i];
        for (int c = 0; c < 3; ++c) o.r.push_back(a.r[c]);
        for (size_t n = 0; n < a.numNeighbors; ++n)
        {
            Atom::Neighbor const& nb = a.neighbors[n];
            o.nbrIndex.push_back((int64_t)nb.index);
            o.nbrD.push_back(nb.d);
            for (int c = 0; c < 3; ++c) o.nbrDr.push_back(nb.dr[c]);
            size_t rows = useForces ? nb.dGdr.size() : 0;
            for (size_t q = 0; q < rows; ++q)
                for (int c = 0; c < 3; ++c) o.dGdrNbr.push_back(nb.dGdr[q][c]);
            o.rowOffset.push_back(o.rowOffset.back() + (int64_t)rows);
        }
        o.nbrOffset.push_back(o.nbrOffset.back() + (int64_t)a.numNeighbors);
        for (size_t q = 0; q < a.G.size(); ++q)
        {
            o.G.push_back(a.G[q]);
            o.dEdG.push_back(q < a.dEdG.size() ? a.dEdG[q] : 0.0);
            for (int c = 0; c < 3; ++c)
                o.dGdrSelf.push_back(useForces && q < a.dGdr.size() ? a.dGdr[q][c] : 0.0);
        }
        o.sfOffset.push_back(o.sfOffset.back() + (int64_t)a.G.size());
        o.atomicEnergy.push_back(a.energy);
        for (int c = 0; c < 3; ++c) o.forcesInternal.push_back(a.f[c]);
    }
    o.energyInternal = s.energy;
}

template <class T>
int64_t copyOut(vector<T> const& v, T* dst, int64_t cap)
{
    int64_t n = (int64_t)v.size();
    if (dst && cap >= n && n > 0) memcpy(dst, v.data(), sizeof(T) * n);
    return n;
}

} // namespace

extern "C" {

const char* nnpref_last_error() { return g_err.c_str(); }

void* nnpref_create(const char* dir, int writeExtrapolationWarnings)
{
    try
    {
        Handle* h = new Handle();
        h->dir = dir;
        h->mode.setupFromDir(dir, writeExtrapolationWarnings != 0);
        return h;
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return nullptr;
    }
}

void nnpref_destroy(void* p) { delete static_cast<Handle*>(p); }

int64_t nnpref_num_elements(void* p) { return (int64_t)static_cast<Handle*>(p)->mode.nElem(); }
int64_t nnpref_num_sf(void* p, int64_t e) { return (int64_t)static_cast<Handle*>(p)->mode.numSF((size_t)e); }
int64_t nnpref_num_rows(void* p, int64_t ec, int64_t en)
{
    return (int64_t)static_cast<Handle*>(p)->mode.numRows((size_t)ec, (size_t)en);
}
double nnpref_max_cutoff(void* p) { return static_cast<Handle*>(p)->mode.maxRc(); }

// Read one input.data block, run evaluateNNP, snapshot, convert back.
int nnpref_predict(void* p, const char* text, int useForces)
{
    Handle& h = *static_cast<Handle*>(p);
    try
    {
        Structure s;
        h.mode.readStructure(s, text);
        h.mode.evaluateNNP(s, useForces != 0);
        takeSnapshot(h, s, useForces != 0);
        h.mode.finish(s);
        h.snap.energy = s.energy;
        for (auto const& a : s.atoms)
            for (int c = 0; c < 3; ++c) h.snap.forces.push_back(a.f[c]);
        return 0;
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return 1;
    }
}

// Jacobian of a training observation (property 0: the structure's energy,
// 1: force component `component` of atom `atom`) at the model's weights, in
// internal units; returns its length (copies when out != NULL and cap
// suffices), -1 on failure.
int64_t nnpref_jacobian(void* p, const char* text, int property, int64_t atom, int component, double* out,
                        int64_t cap)
{
    Handle& h = *static_cast<Handle*>(p);
    try
    {
        Structure s;
        h.mode.readStructure(s, text);
        h.mode.evaluateNNP(s, true);
        vector<double> jac;
        h.mode.jacobian(s, property, (size_t)atom, (size_t)component, jac);
        return copyOut(jac, out, cap);
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return -1;
    }
}

// Gradient of a loss through one structure, sum_E aE dE/dw + sum_k u[k] dF_k/dw
// (k = 3 atom + component, F_k the force components), from the same
// reference Jacobians, the structure evaluated once; internal units.  Returns
// the weight count (copies when out != NULL and cap suffices), -1 on failure.
int64_t nnpref_loss_gradient(void* p, const char* text, double aE, const double* u, double* out, int64_t cap)
{
    Handle& h = *static_cast<Handle*>(p);
    try
    {
        Structure s;
        h.mode.readStructure(s, text);
        h.mode.evaluateNNP(s, true);
        vector<double> g, jac;
        h.mode.jacobian(s, 0, 0, 0, g);
        for (double& x : g) x *= aE;
        for (size_t a = 0; a < s.atoms.size(); ++a)
            for (size_t c = 0; c < 3; ++c)
            {
                const double w = u[3 * a + c];
                if (w == 0.0) continue;
                h.mode.jacobian(s, 1, a, c, jac);
                for (size_t q = 0; q < g.size(); ++q) g[q] += w * jac[q];
            }
        return copyOut(g, out, cap);
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return -1;
    }
}

double nnpref_energy(void* p) { return static_cast<Handle*>(p)->snap.energy; }
double nnpref_energy_internal(void* p) { return static_cast<Handle*>(p)->snap.energyInternal; }

// Getters: return the element count; copy when dst != NULL and cap suffices.
#define NNPREF_GETTER(name, field, T) \
    int64_t nnpref_##name(void* p, T* dst, int64_t cap) \
    { return copyOut(static_cast<Handle*>(p)->snap.field, dst, cap); }
NNPREF_GETTER(forces, forces, double)
NNPREF_GETTER(forces_internal, forcesInternal, double)
NNPREF_GETTER(positions, r, double)
NNPREF_GETTER(box, box, double)
NNPREF_GETTER(nbr_offset, nbrOffset, int64_t)
NNPREF_GETTER(nbr_index, nbrIndex, int64_t)
NNPREF_GETTER(nbr_d, nbrD, double)
NNPREF_GETTER(nbr_dr, nbrDr, double)
NNPREF_GETTER(sf_offset, sfOffset, int64_t)
NNPREF_GETTER(G, G, double)
NNPREF_GETTER(dEdG, dEdG, double)
NNPREF_GETTER(dGdr_self, dGdrSelf, double)
NNPREF_GETTER(row_offset, rowOffset, int64_t)
NNPREF_GETTER(dGdr_nbr, dGdrNbr, double)
NNPREF_GETTER(atomic_energy, atomicEnergy, double)
#undef NNPREF_GETTER

// Time Mode::evaluateNNP over a set of structures on `numThreads` host
// threads, structure-parallel, one Mode instance per thread (the reference's
// NN objects hold per-neuron state and are not shared between threads).
// Parsing and setup happen before the clock starts.  Returns wall seconds of
// the evaluation phase; energies (physical units) are written to `energies`.
static double timeBatch(const char* dir, int64_t numStructures, const char* const* texts, int64_t numThreads,
                        double* energies, bool sfOnly);

double nnpref_time_batch(const char* dir, int64_t numStructures, const char* const* texts,
                         int64_t numThreads, double* energies)
{
    return timeBatch(dir, numStructures, texts, numThreads, energies, false);
}

// The same for the symmetry functions alone (what nnp-scaling computes per
// structure); no energies.
double nnpref_time_sf_batch(const char* dir, int64_t numStructures, const char* const* texts, int64_t numThreads)
{
    return timeBatch(dir, numStructures, texts, numThreads, nullptr, true);
}

} // extern "C"

static double timeBatch(const char* dir, int64_t numStructures, const char* const* texts, int64_t numThreads,
                        double* energies, bool sfOnly)
{
    try
    {
        if (numThreads < 1) numThreads = 1;
        vector<Handle*> hs;
        vector<vector<Structure>> perThread(numThreads);
        vector<vector<int64_t>> ids(numThreads);
        for (int64_t t = 0; t < numThreads; ++t)
        {
            hs.push_back(new Handle());
            hs.back()->mode.setupFromDir(dir, false);
        }
        for (int64_t s = 0; s < numStructures; ++s)
        {
            int64_t t = s % numThreads;
            perThread[t].emplace_back();
            hs[t]->mode.readStructure(perThread[t].back(), texts[s]);
            ids[t].push_back(s);
        }
        auto t0 = chrono::steady_clock::now();
        vector<thread> pool;
        for (int64_t t = 0; t < numThreads; ++t)
        {
            pool.emplace_back([&, t]() {
                for (size_t k = 0; k < perThread[t].size(); ++k)
                {
                    Structure& st = perThread[t][k];
                    if (sfOnly) hs[t]->mode.symmetryFunctionsOnly(st);
                    else hs[t]->mode.evaluateNNP(st, true);
                }
            });
        }
        for (auto& th : pool) th.join();
        double sec = chrono::duration<double>(chrono::steady_clock::now() - t0).count();
        for (int64_t t = 0; t < numThreads; ++t)
        {
            for (size_t k = 0; k < perThread[t].size(); ++k)
            {
                Structure& st = perThread[t][k];
                if (!sfOnly) hs[t]->mode.finish(st);
                if (energies) energies[ids[t][k]] = st.energy;
            }
            delete hs[t];
        }
        return sec;
    }
    catch (std::exception const& e)
    {
        g_err = e.what();
        return -1.0;
    }
}


