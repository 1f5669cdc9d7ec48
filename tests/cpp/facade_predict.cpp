// Driver of the C++ Mode facade (include/n2p2_b200_mode.hpp) for the tests:
// a C++ caller written against the reference's nnp::Mode / nnp::Structure
// API, as nnp-predict is (Prediction::setup / predict, Prediction.cpp:36-78).
//
//   facade_predict errors <model dir>           set-up failures, no GPU
//   facade_predict predict <model dir>          evaluateNNP, then the stages
//                                               one by one; JSON on stdout
#include <cstdio>
#include <stdexcept>
#include <string>

#include "n2p2_b200_mode.hpp"

using n2p2b200::nnp::Mode;
using n2p2b200::nnp::Structure;

static void setup(Mode& m, std::string const& d)
{
    m.initialize();
    m.loadSettingsFile(d + "/input.nn");
    m.setupGeneric();
    m.setupSymmetryFunctionScaling(d + "/scaling.data");
    m.setupNeuralNetworkWeights(d + "/weights.%03zu.data");
    m.setupSymmetryFunctionStatistics(false, false, false, false);
}

static void printArray(char const* name, std::vector<double> const& v, bool last = false)
{
    std::printf("\"%s\": [", name);
    for (size_t k = 0; k < v.size(); ++k) std::printf("%s%.17g", k ? ", " : "", v[k]);
    std::printf("]%s\n", last ? "" : ",");
}

static int errors(std::string const& d)
{
    int failures = 0;
    {
        Mode m(0);
        m.initialize();
        try
        {
            m.loadSettingsFile(d + "/does_not_exist.nn");
            ++failures;
        }
        catch (std::runtime_error const&)
        {
        }
    }
    {
        Mode m(0);
        setup(m, d);
        Structure s;
        s.readFromFile(d + "/input.data");
        try
        {
            s.calculateNeighborList(m.getMaxCutoffRadius(), true);   // sorted lists: 4G only
            ++failures;
        }
        catch (std::invalid_argument const&)
        {
        }
        try
        {
            s.readFromFile(d + "/input.data", 1000000);
            ++failures;
        }
        catch (std::runtime_error const&)
        {
        }
        std::printf("{\"numAtoms\": %zu, \"maxCutoffRadius\": %.17g, \"failures\": %d}\n", s.numAtoms,
                    m.getMaxCutoffRadius(), failures);
    }
    return failures;
}

static int predict(std::string const& d)
{
    Mode m(0);
    setup(m, d);
    Structure s;
    s.readFromFile(d + "/input.data");
    // Prediction::predict: evaluateNNP (the neighbour list inside, Mode.cpp:2029-2077)
    m.evaluateNNP(s);
    std::vector<double> F1, F2, G, dEdG, nbr;
    for (auto const& a : s.atoms)
        for (int c = 0; c < 3; ++c) F1.push_back(a.f[c]);
    const double E1 = s.energy;
    // the stages one by one on a second structure object
    Structure t;
    t.readFromFile(d + "/input.data");
    t.calculateNeighborList(m.getMaxCutoffRadius());
    m.calculateSymmetryFunctionGroups(t, true);
    m.calculateAtomicNeuralNetworks(t, true);
    m.calculateEnergy(t);
    m.calculateForces(t);
    for (auto const& a : t.atoms)
    {
        for (int c = 0; c < 3; ++c) F2.push_back(a.f[c]);
        G.insert(G.end(), a.G.begin(), a.G.end());
        dEdG.insert(dEdG.end(), a.dEdG.begin(), a.dEdG.end());
        nbr.push_back((double)a.numNeighbors);
    }
    // a repeated evaluateNNP on unchanged positions reuses the cached symmetry functions
    m.evaluateNNP(s);
    const double E3 = s.energy;
    // moved atoms: recomputed
    Structure u;
    u.readFromFile(d + "/input.data");
    m.evaluateNNP(u);
    u.atoms[0].r[0] += 0.01;
    m.evaluateNNP(u);
    const double E4 = u.energy;
    std::printf("{\"energy\": %.17g, \"energy_stages\": %.17g, \"energy_again\": %.17g, \"energy_moved\": %.17g,\n",
                E1, t.energy, E3, E4);
    printArray("forces", F1);
    printArray("forces_stages", F2);
    printArray("G", G);
    printArray("dEdG", dEdG);
    printArray("num_neighbors", nbr, true);
    std::printf("}\n");
    return 0;
}

int main(int argc, char** argv)
{
    if (argc != 3) return 2;
    try
    {
        std::string what = argv[1];
        if (what == "errors") return errors(argv[2]);
        if (what == "predict") return predict(argv[2]);
    }
    catch (std::exception const& e)
    {
        std::fprintf(stderr, "%s", e.what());
        return 1;
    }
    return 2;
}
