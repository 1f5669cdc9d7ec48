// Host-side model setup for the 2G short-range HDNNP path.
//
// Mirrors the setup half of nnp::Mode (reference src/libnnp/Mode.cpp:162-1547):
// input.nn keyword parsing, the element map, the symmetry-function table and
// its canonical order, per-neighbour-element derivative tables, scaling, the
// per-element network topology and the weights files.  Everything here runs
// once per model on the host; the result is flattened into the device model
// (device_model.hpp) that the sm_100a kernels read.
#pragma once

#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "device_model.hpp"

namespace n2p2b200 {

constexpr int kMaxElements = 8;

// "input.nn" contents: keyword -> (argument string, line index), in file
// order; a keyword may repeat (symfunction_short, atom_energy, ...).
// Follows Settings::parseLines (Settings.cpp:324-390).
class Settings
{
public:
    void loadFile(std::string const& fileName);
    void parseText(std::string const& text);
    bool keywordExists(std::string const& key) const;
    std::string const& value(std::string const& key) const;   // first instance
    std::vector<std::pair<std::string, std::size_t>> values(std::string const& key) const;
    std::vector<std::string> const& warnings() const { return warnings_; }

private:
    std::multimap<std::string, std::pair<std::string, std::size_t>> contents_;
    std::vector<std::string> warnings_;
};

// Symbols sorted by atomic number (ElementMap::registerElements,
// ElementMap.cpp:36-54).
struct ElementMap
{
    std::vector<std::string> symbols;
    int index(std::string const& symbol) const;  // throws if unknown
    static std::size_t atomicNumber(std::string const& symbol);
};

// Core functions of the compact symmetry functions (CoreFunction::Type,
// CoreFunction.h:40-52, numbered as the cutoff cores).
enum CompactCore { CORE_EXP = CT_EXP, CORE_POLY1 = CT_POLY1, CORE_POLY2, CORE_POLY3, CORE_POLY4 };

// One symmetry function: Gaussian types 2, 3, 9 or compact types 20, 22.
struct SymFunc
{
    int    type = 0;          // 2 radial, 3 angular narrow, 9 angular wide; compact: 20 radial,
                              // 21 angular narrow, 22 angular wide, 23 radial weighted,
                              // 24 angular narrow weighted, 25 angular wide weighted
    int    ec = 0, e1 = 0, e2 = 0;
    double eta = 0.0, rs = 0.0, zeta = 0.0, lambda = 0.0, rc = 0.0;
    int    cutoffType = CT_HARD;
    double cutoffAlpha = 0.0;
    std::size_t lineNumber = 0;
    int    index = 0;          // position in the element's sorted list
    int    zetaInt = 0;
    bool   useIntegerPow = false;
    int    indexPerElement[kMaxElements];   // derivative row per neighbour element, -1 if irrelevant
    // scaling (SymFnc::setScalingType, SymFnc.cpp:52-98)
    int    scalingType = ST_NONE;
    double Smin = 0.0, Smax = 0.0, Gmin = 0.0, Gmax = 0.0, Gmean = 0.0, Gsigma = 0.0;
    double scalingFactor = 1.0;

    // compact functions (SymFncBaseComp / SymFncBaseCompAng::setParameters)
    double rl = 0.0;                      // lower radial boundary
    std::string subtype;                  // "p1".."p4", optionally + "a" (asymmetric), or "e..."
    int    core = CORE_POLY2;
    bool   asymmetric = false;
    double angleLeft = 0.0, angleRight = 0.0;   // degrees

    bool compact() const { return type >= 20; }
    bool radial() const { return type == 2 || type == 20 || type == 23; }
    // element-weighted compact functions (SymFncCompRadWeighted, SymFncBaseCompAngWeighted):
    // every neighbour counts, weighted by its atomic number
    bool weighted() const { return type >= 23; }
    bool relevant(int e) const { return weighted() || (radial() ? e == e1 : (e == e1 || e == e2)); }
    double scale(double value) const;
    double unscale(double value) const;
};

// Members sharing (ec, type, cutoff, rc, e1[, e2]) are evaluated in one
// neighbour pass (Element::setupSymmetryFunctionGroups, Element.cpp:194-287).
struct SymGroup
{
    int type = 0, ec = 0, e1 = 0, e2 = 0;
    double rc = 0.0;
    int cutoffType = CT_HARD;
    double cutoffAlpha = 0.0;
    std::vector<int> members;            // SF indices of the element, member order
    std::vector<char> calculateExp;      // recompute the Gaussian for this member
    std::vector<char> calculateComp;     // compact narrow angular: recompute the r_jk radial part
                                         // (SymGrpCompAngn::sortMembers, SymGrpCompAngn.cpp:110-126)
    std::vector<double> factorNorm;      // 2^(1-zeta) * scalingFactor (angular)
    std::vector<double> factorDeriv;     // 2 eta / zeta / lambda (angular)
};

struct NetworkTopology
{
    int numLayers = 0;
    std::vector<int> neurons;
    std::vector<int> activations;
};

struct ElementSetup
{
    std::string symbol;
    std::size_t atomicNumber = 0;
    double atomicEnergyOffset = 0.0;
    std::vector<SymFunc> sf;                       // sorted
    std::vector<SymGroup> groups;                  // Gaussian types
    std::vector<SymGroup> compactGroups;           // compact types: (type, e1[, e2]), weighted types: (type)
                                                   // (SymGrpComp*::operator==)
    std::vector<std::vector<int>> table;           // table[e] = SF indices with a derivative row for neighbour element e
    NetworkTopology topology;
    // weights[l] is layer l+1: W (neurons[l+1] x neurons[l], row major) then b
    std::vector<std::vector<double>> W;
    std::vector<std::vector<double>> b;
    bool hasWeights = false;
};

class Model
{
public:
    // Mode::loadSettingsFile (Mode.cpp:162-211)
    void loadSettingsFile(std::string const& fileName);
    void loadSettingsText(std::string const& text);
    // Mode::setupGeneric (Mode.cpp:213-237), 2G branch
    void setupGeneric();
    // Mode::setupSymmetryFunctionScaling (Mode.cpp:781-909)
    void setupSymmetryFunctionScaling(std::string const& fileName);
    // Mode::setupSymmetryFunctionScalingNone (Mode.cpp:761-779)
    void setupSymmetryFunctionScalingNone();
    // Mode::setupNeuralNetworkWeights (Mode.cpp:1520-1547) with a printf-style
    // format taking the atomic number, e.g. "dir/weights.%03zu.data".
    void setupNeuralNetworkWeights(std::string const& fileNameFormat);
    // Direct weight upload in the weights-file order (NeuralNetwork::setConnections).
    void setConnections(int element, std::vector<double> const& connections);

    std::size_t numElements() const { return elements.size(); }
    double maxCutoffRadius = 0.0;
    bool normalize = false;
    double meanEnergy = 0.0, convEnergy = 1.0, convLength = 1.0;
    bool normalizeNeurons = false;
    int cutoffType = CT_HARD;
    double cutoffAlpha = 0.0;
    int scalingType = ST_NONE;
    bool setupDone = false;
    bool scalingDone = false;
    ElementMap elementMap;
    std::vector<ElementSetup> elements;
    Settings settings;

private:
    void setupNormalization();
    void setupElementMap();
    void setupElements();
    void setupCutoff();
    void setupSymmetryFunctions();
    void setupSymmetryFunctionMemory();
    void setupSymmetryFunctionGroups();
    void setupNeuralNetwork();
};

int activationFromString(std::string const& c);
std::vector<std::string> splitWords(std::string const& line);
std::string reduceLine(std::string const& line);

} // namespace n2p2b200
