// Device-side engine: the uploaded model, batches of structures and the
// evaluation sequence of Mode::evaluateNNP (Mode.cpp:2029-2077) on one GPU.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "device_model.hpp"
#include "host_model.hpp"
#include "kernels.hpp"

namespace n2p2b200 {

enum Precision { PREC_FP64 = 0, PREC_MIXED = 1 };

// Evaluation flags (bit set).
enum EvalFlags : int {
    EVAL_FORCES = 1,          // forces (else energies only)
    EVAL_STORE_DGDR = 2,      // keep dG/dr per neighbour row (API form)
    EVAL_NO_GRAPH = 4,        // launch kernels directly instead of replaying a CUDA graph
    EVAL_SF_ONLY = 8,         // symmetry functions (and the extrapolation check) only
};

void cudaCheck(cudaError_t e, char const* what);

// Whether the model's networks fit the tensor-core kernel of the mixed form
// (two hidden layers of <= 64 neurons, <= 64 inputs, linear output, no
// normalize_nodes).
bool networkTCSupported(Model const& m);

// Device memory cache of one batch: blocks given back by put() are handed out
// again for requests of up to their size (at most twice the request's size
// class), so re-setting structures of similar size allocates nothing.  Every user of a batch's memory works on
// the batch's stream, so reuse is ordered after the previous users.
class DevicePool
{
public:
    ~DevicePool();
    void* get(size_t bytes);
    void put(void* p);
    void trim();   // cudaFree every cached block

private:
    std::map<size_t, std::vector<void*>> free_;
    std::unordered_map<void*, size_t> size_;
};

// Device copy of a set-up model.
class DeviceModel
{
public:
    ~DeviceModel();
    void upload(Model const& m);
    DevModel view;
    DevGroupTable groupTable{};          // the groups again, passed by value to the specialised kernels
    int maxSF = 0;
    size_t numWeights = 0;               // entries of the flat weight array
    uint64_t fingerprint = 0;            // hash of the evaluation plan (groups, members, cutoffs)
    bool tcNetwork = false;              // mixed form runs the networks on the tensor cores
    bool networksSet = true;             // every element has weights (else symmetry functions only)
    std::string missingWeights;
    double* weightsDevice() const { return weights_; }
    double* weightsTDevice() const { return weightsT_; }
    int* transIndexDevice() const { return transIndex_; }
    std::vector<int> transIndexHost;     // weight index -> index in the transposed copy

private:
    void release();
    DevGroup* groups_ = nullptr;
    DevMember* members_ = nullptr;
    DevScaling* scaling_ = nullptr;
    int* rowTable_ = nullptr;
    double* weights_ = nullptr;
    double* weightsT_ = nullptr;
    int* transIndex_ = nullptr;
    DevCompactGroup* compactGroups_ = nullptr;
    DevCompactMember* compactMembers_ = nullptr;
    DevCompactFn* compactFns_ = nullptr;
};

struct StructureInput
{
    int numAtoms = 0;
    double box[9] = {0};      // physical units, rows = box vectors
    int periodic = 0;
};

class Batch
{
public:
    Batch(Model const& model, DeviceModel const& dmodel, cudaStream_t stream, int sms);
    ~Batch();

    // Structures and atoms.  Positions are physical units (as in input.data);
    // `remap` folds periodic positions into the cell (Structure::remap),
    // normalisation (if the model uses it) is applied on the device.
    void setStructures(std::vector<StructureInput> const& s, const int* elements, int remap);
    // External neighbour lists instead of structures (the LAMMPS interface,
    // InterfaceLammps::setLocalAtoms / addNeighbor, InterfaceLammps.cpp:267-441):
    // `numCenters` atoms of one system with their elements; centre i's entries
    // are [offsets[i], offsets[i+1]) with, per entry, the neighbour's index
    // among `numTargets` atoms (the caller's numbering, ghosts included), its
    // element, r_i - r_j ([E][3]) and |r_i - r_j|, internal units, every
    // |r_i - r_j| <= the model's largest cutoff.  centerTarget[i] is centre
    // i's own index among the targets.  evaluate() then skips the position
    // and neighbour stages and gathers the forces of all targets
    // (targetForces).  Stored dG/dr is not available in this form.
    void setExternalNeighbors(int numCenters, const int* elements, int64_t numEntries, const int64_t* offsets,
                              int numTargets, const int* target, const int* targetElement, const double* dr,
                              const double* d, const int* centerTarget);
    // The same from an MD code's own full neighbour lists (positions and
    // types of all its atoms, candidates per centre): the entries are built
    // on the device (k_external.cu).  The host arrays are read by
    // asynchronous copies: keep them unchanged until the next call that
    // synchronises (evaluate's results, targetForces).
    struct ExternalLists
    {
        int numCenters = 0;
        const int* centerElement = nullptr;   // [numCenters]
        const int* centerIndex = nullptr;     // [numCenters] index among all atoms
        const int64_t* candOffset = nullptr;  // [numCenters + 1]
        const int* cand = nullptr;            // [numCand] indices among all atoms
        int64_t numCand = 0;
        int numAll = 0;
        const double* x = nullptr;            // [numAll][3], the MD code's units
        const int* type = nullptr;            // [numAll], 1-based
        const int* typeElement = nullptr;     // [numTypes + 1], -1 = ignored
        int numTypes = 0;
        double cflength = 1.0, convLength = 1.0;
        bool normalize = false;
        double pairCut2 = 0.0;
    };
    void setExternalLists(ExternalLists const& lists);
    bool external() const { return external_; }
    int numTargets() const { return numTargets_; }
    void targetForces(double* out);   // [numTargets][3], internal units (synchronises)
    // Positions host -> device (pinned or pageable host memory), async on the stream.
    void setPositionsHost(const double* r);
    void setPositionsDevice(const double* r);
    // Mode::evaluateNNP; asynchronous unless the neighbour capacity must be
    // (re)established, which happens on the first call and after overflow.
    // A graph replay runs with the buffers sized at the first call: when new
    // positions make the lists longer, the kernels skip the atoms whose
    // entries do not fit, so every reader of the results calls verify()
    // first, which detects that, grows the buffers and evaluates again.
    void evaluate(int flags, int precision, int checkExtrapolation);
    // Synchronises; after a truncated evaluation, grows the neighbour
    // buffers and repeats the evaluation directly (the reference's list never
    // truncates, Structure.cpp:287-398).  Idempotent until the next evaluate.
    void verify();
    // Evaluations repeated by verify() since the batch was created.
    int64_t overflowRecoveries() const { return overflowRecoveries_; }
    int64_t neighborCapacity() const { return capacity_; }
    // The stages of Mode::evaluateNNP as separate calls (Mode.h:298-378),
    // launched directly on the batch's stream (no CUDA graph) with the same
    // kernels, so a sequence of them gives the bits evaluate() gives.
    //   calculateNeighborList          Structure::calculateNeighborList(rc, false)
    //                                  (Structure.cpp:287-398); synchronises to
    //                                  size the buffers
    //   calculateSymmetryFunctions     Mode::calculateSymmetryFunction[Groups]
    //                                  (Mode.cpp:1549-1709); derivatives 0 = values,
    //                                  1 = values with derivatives (contracted by
    //                                  calculateForces, nothing stored), 2 = dG/dr
    //                                  stored (Atom::dGdr, Atom::Neighbor::dGdr; FP64)
    //   calculateAtomicNeuralNetworks  Mode.cpp:1711-1732 (2G): E_i, and dE/dG with
    //                                  derivatives
    //   calculateEnergy                Mode.cpp:1876-1901
    //   calculateForces                Mode.cpp:1922-1984 (needs derivatives of both)
    // The symmetry-function call keeps the reference's caching flags
    // (Structure::hasSymmetryFunctions / hasSymmetryFunctionDerivatives,
    // Mode.cpp:1634-1635): it returns at once when its results exist.  New
    // structures or positions clear every flag; evaluate() sets them.  A stage
    // whose inputs are missing throws std::runtime_error (the reference would
    // read empty vectors).
    void calculateNeighborList();
    void calculateSymmetryFunctions(int derivatives, int precision, int checkExtrapolation);
    void calculateAtomicNeuralNetworks(int derivatives, int precision);
    void calculateEnergy();
    void calculateForces();
    struct StageState
    {
        bool neighbors = false, sf = false, sfDerivatives = false, sfStored = false, networks = false,
             dEdG = false, energy = false, forces = false;
        int sfPrecision = 0;
    };
    StageState const& stageState() const { return stage_; }

    // Host-side results (synchronise first).
    void energies(double* out);       // physical units, with atomic energy offsets
    // Inverse of the conversions of energies() / forces(): physical energies
    // (with offsets) to internal network sums, and the factor that takes
    // physical forces to internal ones.
    void energiesToInternal(const double* phys, double* out) const;
    double forceToInternal() const;
    void forces(double* out);         // physical units, [N][3]
    void synchronize();
    DevStatus status();   // verify(), then the device status word

    int numAtoms() const { return N_; }
    int numStructures() const { return S_; }
    int64_t numNeighborEntries();
    BatchView const& view() const { return v_; }
    cudaStream_t stream() const { return stream_; }
    int launchesPerEvaluate() const { return launches_; }

    // Autotuning of the symmetry-function passes' first-tier shape (stage
    // capacity x warps per block, kSFShapeCount variants): every shape of both
    // passes is timed on this batch's own inputs and the fastest kept, or the
    // choice is read from the on-disk cache (N2P2_B200_TUNE_CACHE, default
    // ~/.cache/n2p2_b200/autotune.json) keyed by GPU, model plan, precision
    // and workload class.  Runs by itself before the first graph capture of a
    // precision unless disabled.
    struct TuneResult
    {
        int values = 1, forces = 1;
        double valuesMs[kSFShapeCount] = {0}, forcesMs[kSFShapeCount] = {0};
        bool fromCache = false;
    };
    TuneResult autotune(int precision, int checkExtrapolation, bool useCache);
    void setShapes(int precision, int values, int forces);
    TuneResult lastTune(int precision) const { return lastTune_[precision]; }
    bool autotuneEnabled = true;

    // One direct evaluation with CUDA events between the stages; returns
    // (stage name, milliseconds) in launch order.
    std::vector<std::pair<std::string, double>> profileStages(int flags, int precision, int checkExtrapolation);
    // Algorithmic work counters of the current neighbour lists (10 values,
    // see kCountWork).
    void countWork(int64_t* counts);

    // Internal-unit results for inspection (neighbour lists, G, dEdG, dGdr).
    void copyNeighbors(int64_t* offsets, int* index, int* image, double* d, double* dr);
    void copyG(double* out);          // [N][numSF of the atom's element], concatenated
    void copyDEdG(double* out);
    void copyAtomicEnergies(double* out);
    void copyDGdr(double* self, double* nbr);   // self [sum numSF][3], nbr [sum rows][3]
    void copyPositions(double* out);  // internal units after remap/normalisation
    void copyAtomWarnings(int* out);
    // Symmetry-function statistics of the last evaluation (SymFncStatistics,
    // as nnp-scaling collects them): per element its atom count and, per
    // function, min, max, sum and sum of squares of the unscaled G, in atom
    // order.  counts [numElements], stats [numElements][4][maxSF].
    void sfStatistics(int64_t* counts, double* stats);
    int maxSF() const { return dmodel_.maxSF; }

private:
    void allocateAtoms();
    void allocateNeighbors(int64_t capacity);
    void allocateScratch(int64_t entries);
    void setStride(int64_t stride);
    void allocateDGdr();
    struct Mark
    {
        std::string name;
        cudaEvent_t event;
    };
    enum Stage
    {
        STAGE_NEIGHBORS = 1,   // positions, neighbour lists, cutoff values
        STAGE_SF = 2,          // symmetry functions (+ candidate masks, extrapolation check)
        STAGE_NETWORKS = 4,    // atomic networks (+ dE/dG with EVAL_FORCES)
        STAGE_ENERGY = 8,      // structure energies
        STAGE_FORCES = 16,     // force pass + gather (with EVAL_FORCES)
        STAGE_ALL = 31
    };
    void record(int flags, int precision, int checkExtrapolation, std::vector<Mark>* marks = nullptr,
                int stages = STAGE_ALL);
    DevStatus readStatus();   // the device status word as it is (synchronises)
    void releaseGraph();
    void releaseAll();

    Model const& model_;
    DeviceModel const& dmodel_;
public:
    Model const& model() const { return model_; }
    DeviceModel const& deviceModel() const { return dmodel_; }
    std::vector<int> const& structBegin() const { return structBegin_; }
private:
    cudaStream_t stream_;
    int sms_;
    int N_ = 0, S_ = 0;
    std::vector<StructureInput> structs_;
    std::vector<int> elemHost_;
    std::vector<int> structBegin_;
    std::vector<int> numAtomsPerElement_;   // [S][numElements]
    int remap_ = 1;
    BatchView v_{};
    double* rin_ = nullptr;                 // raw positions (physical)
    DevStructInfo* infoDev_ = nullptr;
    int* atomStructDev_ = nullptr;
    int* elemDev_ = nullptr;
    int* structBeginDev_ = nullptr;
    int64_t capacity_ = 0;
    bool capacityVerified_ = false;
    bool pendingVerify_ = false;      // an evaluation ran that verify() has not checked
    StageState stage_;                // results the separate stage calls (or evaluate) produced
    void requireStructures();
    int lastFlags_ = 0, lastPrecision_ = 0, lastCheck_ = 0;
    int64_t overflowRecoveries_ = 0;
    bool dgdrAllocated_ = false;
    cudaGraphExec_t graphExec_ = nullptr;
    int graphKey_ = -1;
    int launches_ = 0;
    int sfShape_[2][2] = {{1, 1}, {1, 1}};   // [values, forces][precision]: first-tier shape variant
    bool tuned_[2] = {false, false};
    TuneResult lastTune_[2];
    std::string tuneKey(int precision);
    DevicePool pool_;
    std::vector<void*> owned_;
    std::vector<void*> ownedNbr_;
    std::vector<void*> ownedScr_;     // neighbour-build scratch (unordered entries)
    int64_t scrEntries_ = 0;
    int64_t nbrStride_ = 0;           // > 0: one-pass neighbour search into fixed-stride scratch
    int64_t strideWanted_ = 0;        // the stride the next evaluation sets (0: two passes)
    std::vector<void*> ownedDGdr_;
    std::vector<void*> ownedMask_;
    uint32_t* maskBuf_ = nullptr;
    int64_t maskCap_ = 0;
    void uploadElementLists();
    // external neighbour lists
    void beginExternal(int numCenters, const int* elements, int numTargets, const int* centerTarget, int64_t capacity);
    bool external_ = false;
    bool extRaw_ = false;           // entries built on the device from raw lists (raw_)
    ExtRawView raw_{};
    int numTargets_ = 0;
    int* tCount_ = nullptr;         // [numTargets] entries naming each target
    int* tFill_ = nullptr;
    int64_t* tOffset_ = nullptr;    // [numTargets + 1]
    int64_t* tEntryTmp_ = nullptr;  // [capacity]
    int64_t* tEntry_ = nullptr;     // [capacity] per target, in entry order
    int* targetCenter_ = nullptr;   // [numTargets] centre index or -1
    int* centerIndex_ = nullptr;    // [N] each centre's index among the targets
    int64_t* tScanTmp_ = nullptr;
    double* Ftarget_ = nullptr;     // [numTargets][3]
    int64_t* entriesDev_ = nullptr; // host-built entries: their count, copied into the status by every evaluation
};

} // namespace n2p2b200
