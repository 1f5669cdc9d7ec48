// Host side of the LAMMPS interface for 2G models: the state and unit
// handling of nnp::InterfaceLammps (reference
// src/libnnpif/LAMMPS/InterfaceLammps.{h,cpp}), with the local atoms' lists
// staged for one device evaluation through external neighbour lists
// (Batch::setExternalNeighbors) instead of per-atom Atom::Neighbor objects.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "engine.hpp"
#include "host_model.hpp"

namespace n2p2b200 {

class LammpsInterface
{
public:
    // InterfaceLammps::initialize (InterfaceLammps.cpp:51-255) after the
    // model's set-up: unit factors, the cutoff consistency check and the
    // LAMMPS type -> element map ("1:H,2:O"; empty = type t is element t-1).
    void initialize(Model const& model, std::string const& emap, double cflength, double cfenergy, double lammpsCutoff,
                    int lammpsNtypes, int myRank);
    bool isInitialized() const { return initialized_; }
    // InterfaceLammps::getMaxCutoffRadius (InterfaceLammps.cpp:528-532), LAMMPS units.
    double maxCutoffRadius() const;

    // InterfaceLammps::setLocalAtoms (InterfaceLammps.cpp:267-304): local
    // atoms of mapped types become centres, in LAMMPS order.
    void setLocalAtoms(int numAtomsLocal, const int* atomType);
    // InterfaceLammps::addNeighbor (InterfaceLammps.cpp:410-441): neighbour j
    // (LAMMPS index, local or ghost) of local atom i, r_i - r_j and its
    // squared length in LAMMPS units.
    void addNeighbor(int i, int j, int type, double dx, double dy, double dz, double d2);
    // PairHDNNP::transferNeighborList (pair_hdnnp.cpp:274-290) in one call:
    // every neighbour within the pair style's cutoff of every listed atom.
    // The raw lists (candidates, positions and types of the atoms they
    // name) are staged in pinned memory and filtered on the device; one step
    // uses either this or addNeighbor.
    void transferNeighborList(int inum, const int* ilist, const int* numneigh, const int* const* firstneigh,
                              const double* const* x, const int* type, double pairCutoff);

    // Hands the staged lists to `batch` (when they changed since the last
    // call) and evaluates energies and forces; InterfaceLammps::process
    // (InterfaceLammps.cpp:463-500).
    void process(Batch& batch, int precision, bool checkExtrapolation);
    // InterfaceLammps::getEnergy / getAtomicEnergy (InterfaceLammps.cpp:550-570), LAMMPS units.
    double energy() const { return energy_ / cfenergy_; }
    double atomicEnergy(Batch& batch, int index);
    // InterfaceLammps::getForces (InterfaceLammps.cpp:679-740): adds the
    // forces on every local and ghost atom named by the lists to atomF.
    void addForces(Batch& batch, double* const* atomF);
    int numCenters() const { return (int)center_.size(); }

    LammpsInterface() = default;
    LammpsInterface(LammpsInterface const&) = delete;
    LammpsInterface& operator=(LammpsInterface const&) = delete;
    ~LammpsInterface();

private:
    // page-locked host staging (grown on demand)
    struct Pinned
    {
        void* p = nullptr;
        size_t bytes = 0;
        void* ensure(size_t n);
        ~Pinned();
    };
    bool initialized_ = false;
    double cflength_ = 1.0, cfenergy_ = 1.0;
    double convLength_ = 1.0, convEnergy_ = 1.0, meanEnergy_ = 0.0;
    bool normalize_ = false;
    double rcmax_ = 0.0;          // largest symmetry-function cutoff, internal units
    int myRank_ = 0;
    std::map<int, int> typeToElement_;
    std::vector<bool> ignoreType_;   // [type], 1-based
    std::vector<double> offsets_;    // atomic energy offset per element
    std::vector<int> typeElement_;   // [type] element or -1 (ignored), type 0 unused
    // local atoms and their lists (staged)
    std::vector<int> indexMap_;      // LAMMPS local index -> centre, -1 if ignored
    std::vector<int> center_;        // centre -> LAMMPS local index
    std::vector<int> centerElement_;
    enum { LISTS_NONE, LISTS_ADDED, LISTS_TRANSFERRED } lists_ = LISTS_NONE;
    // addNeighbor: entries in call order
    std::vector<int> eCenter_, eJ_, eElem_;
    std::vector<double> eDr_, eD_;
    bool eOrdered_ = true;           // centres of the entries never decrease
    // transferNeighborList: candidates per centre and the atoms they name
    Pinned candBuf_, candOffBuf_, xBuf_, typeBuf_;
    int64_t numCand_ = 0;
    int numAll_ = 0;
    double pairCut2_ = 0.0;
    bool dirty_ = true;
    double energy_ = 0.0;            // physical units of the model, offsets included
    std::vector<double> atomicEnergy_;
    bool haveAtomic_ = false;
};

} // namespace n2p2b200
