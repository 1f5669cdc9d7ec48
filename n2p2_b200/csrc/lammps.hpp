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

private:
    bool initialized_ = false;
    double cflength_ = 1.0, cfenergy_ = 1.0;
    double convLength_ = 1.0, convEnergy_ = 1.0, meanEnergy_ = 0.0;
    bool normalize_ = false;
    double rcmax_ = 0.0;          // largest symmetry-function cutoff, internal units
    int myRank_ = 0;
    std::map<int, int> typeToElement_;
    std::vector<bool> ignoreType_;   // [type], 1-based
    std::vector<double> offsets_;    // atomic energy offset per element
    // local atoms and their lists (staged)
    std::vector<int> indexMap_;      // LAMMPS local index -> centre, -1 if ignored
    std::vector<int> center_;        // centre -> LAMMPS local index
    std::vector<int> centerElement_;
    std::vector<std::vector<int>> nbrJ_, nbrElem_;
    std::vector<std::vector<double>> nbrDr_, nbrD_;
    bool dirty_ = true;
    double energy_ = 0.0;            // physical units of the model, offsets included
    std::vector<double> atomicEnergy_;
    bool haveAtomic_ = false;
};

} // namespace n2p2b200
