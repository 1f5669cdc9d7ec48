// Device views of a batch and the kernel launch entry points.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_model.hpp"

namespace n2p2b200 {

// Raw device pointers of one batch of structures.  Atoms of all structures
// are concatenated; neighbour lists are one CSR over all atoms.
struct BatchView
{
    int N = 0;                 // atoms
    int S = 0;                 // structures
    int numCells = 0;
    int gStride = 0;           // row stride of G / dEdG (>= max SF count)
    const int* atomStruct = nullptr;
    const int* elem = nullptr;
    const int* structAtomBegin = nullptr;   // S+1
    const DevStructInfo* info = nullptr;
    double* px = nullptr;
    double* py = nullptr;
    double* pz = nullptr;
    // cell list
    int* atomCell = nullptr;
    int* atomSlot = nullptr;
    int* cellCount = nullptr;
    int* cellStart = nullptr;
    int64_t* cellStart64 = nullptr;
    int* cellAtoms = nullptr;
    const int* elemAtoms = nullptr;    // atoms grouped by element (ascending within an element)
    // Acceptance ballots of the G pass's candidate pairs (two words per
    // 64-candidate step, groups in order), read back by the force pass.
    uint32_t* candMask = nullptr;
    int* maskWords = nullptr;          // per atom
    int64_t* maskOffset = nullptr;     // N+1
    int64_t maskCapacity = 0;
    int elemBegin[kDevMaxElements + 1] = {0};
    double4* cellPos = nullptr;        // cell-ordered (x, y, z, atom index)
    int64_t* scanTmp = nullptr;
    // neighbour CSR
    int* nbrCount = nullptr;
    int64_t* nbrOffset = nullptr;      // N+1
    int64_t nbrCapacity = 0;
    int64_t scrStride = 0;             // > 0: one search pass writes atom i's entries at i * scrStride
                                       // (no count pass); 0: count, scan, then fill at nbrOffset[i]
    int64_t* scrKey = nullptr;
    double* scrD = nullptr;
    double* scrDx = nullptr;
    double* scrDy = nullptr;
    double* scrDz = nullptr;
    int* nbrJ = nullptr;
    int* nbrCode = nullptr;
    uint8_t* nbrElem = nullptr;        // element of each entry's neighbour
    double* nbrD = nullptr;
    double* nbrDx = nullptr;
    double* nbrDy = nullptr;
    double* nbrDz = nullptr;
    int64_t* rev = nullptr;
    double* nbrFc = nullptr;           // [slot][entry]
    double* nbrDfc = nullptr;
    // symmetry functions and networks
    double* G = nullptr;               // [atom][gStride]
    double* dEdG = nullptr;
    double* dGdr = nullptr;            // [row][entry][3] (stored form only)
    double* dGdrSelf = nullptr;        // [atom][gStride][3] (stored form only)
    double* Eatom = nullptr;
    double* Estruct = nullptr;
    double* hx = nullptr;              // force of E_i on neighbour entry (i -> j)
    double* hy = nullptr;
    double* hz = nullptr;
    double* fSelf = nullptr;           // [atom][3]
    double* F = nullptr;               // [atom][3]
    int* atomWarnings = nullptr;
    DevStatus* status = nullptr;
};

// Cell grid of one structure: periodic copies (Structure::calculatePbcCopies,
// Structure.cpp:485-516), cells per axis and the search stencil, from
// d.box, d.numAtoms and the cutoff radius.
void structureGeometry(DevStructInfo& d, double rc);
// Structure::calculateInverseBox (Structure.cpp:518-544).
void inverseBoxOf(double const* box, double* invbox);

// Throws std::runtime_error("CUDA error in ...") on failure.
void cudaCheck(cudaError_t e, char const* what);

// Raise a kernel's dynamic shared-memory limit to `bytes` on the current
// device (a no-op when an earlier call already set as much).
void setDynamicSmemOnce(const void* kernel, size_t bytes);

// neighbour list
void launchPreparePositions(BatchView const& b, const double* rin, int doRemap, int doNormalize, double convLength,
                            cudaStream_t st);
void launchNeighborBuild(BatchView const& b, double rc2, cudaStream_t st);
void launchExclusiveScan(int n, const int* in, int64_t* out, int64_t* tileSums, int64_t* total, cudaStream_t st);
int scanTileCount(int n);
__global__ void kCast64to32(int n, const int64_t* __restrict__ in, int* __restrict__ out);

// symmetry functions
void launchCutoffValues(DevModel const& m, BatchView const& b, int sms, cudaStream_t st);
// Symmetry-function passes; `variant` (0 .. kSFShapeCount-1) picks the first
// tier's (stage capacity, warps per block) in the model-specialised kernels:
// (128, 4), (160, 4), (192, 2).
constexpr int kSFShapeCount = 3;
void launchSFValues(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int precision, int sms,
                    cudaStream_t st, int variant);
void launchSFForces(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int precision, int sms,
                    cudaStream_t st, int variant);
void launchSFValuesF64(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st,
                       int variant);
void launchSFForcesF64(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st,
                       int variant);
void launchSFValuesF32(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st,
                       int variant);
void launchSFForcesF32(DevModel const& m, DevGroupTable const& gt, BatchView const& b, int sms, cudaStream_t st,
                       int variant);
void launchSFDerivatives(DevModel const& m, BatchView const& b, int sms, cudaStream_t st);
void launchContractStored(DevModel const& m, BatchView const& b, int sms, cudaStream_t st);

// networks, energies, forces
void launchNetworkFP64(DevModel const& m, BatchView const& b, int derivatives, int sms, cudaStream_t st);
// Per-atom acceptance-word counts of the angular groups and their offsets.
void launchMaskOffsets(DevModel const& m, BatchView const& b, int sms, cudaStream_t st);
// Tensor-core (tcgen05, split bfloat16) networks of the mixed form; models
// with two hidden layers of <= 64 neurons, <= 64 inputs, linear output.
void launchNetworkTC(DevModel const& m, BatchView const& b, int derivatives, int sms, cudaStream_t st);
void launchEnergySum(BatchView const& b, cudaStream_t st);
void launchGatherForces(BatchView const& b, int sms, cudaStream_t st);
// Compact symmetry functions (types 20-25; k_compact.cu): G of their
// members, then (after the Gaussian force pass) their forces added to h and
// the self forces.  Both return the number of kernels launched.
int launchCompactValues(DevModel const& m, BatchView const& b, int sms, cudaStream_t st);
int launchCompactForces(DevModel const& m, BatchView const& b, int sms, cudaStream_t st);
// Per element and function: min, max, sum, sum of squares of the unscaled G
// (result [numElements][4][maxSF]; partial [numElements][maxChunks][4][maxSF],
// maxChunks = ceil(largest element count / 1024)).
void launchSFStatistics(DevModel const& m, BatchView const& b, int numElements, int maxChunks, int maxSF,
                        double* partial, double* result, cudaStream_t st);
void launchGatherTargets(BatchView const& b, int numTargets, const int64_t* tOffset, const int64_t* tEntry,
                         const int* targetCenter, double* F, int sms, cudaStream_t st);

// An MD code's own neighbour lists on the device (k_external.cu): positions
// and types of all its atoms (local and ghost, its units), per centre the
// candidate neighbours (its indices), the type -> element map (-1: ignored)
// and the unit handling of InterfaceLammps::addNeighbor.
struct ExtRawView
{
    const double* x = nullptr;          // [numAll][3]
    const int* type = nullptr;          // [numAll], 1-based types
    const int* typeElement = nullptr;   // [numTypes + 1]
    int numTypes = 0;
    int numAll = 0;
    const int* centerIndex = nullptr;   // [N] the centre's own index among all atoms
    const int64_t* candOffset = nullptr;   // [N + 1]
    const int* cand = nullptr;
    double cflength = 1.0, convLength = 1.0;
    int normalize = 0;
    double pairCut2 = 0.0;              // the pair style's cutoff squared (its units)
    double rcmax = 0.0;                 // the model's largest cutoff (internal units)
};
// Entries of every centre (count, scan into nbrOffset and the status's
// entry count, fill).
void launchExternalEntries(ExtRawView const& r, BatchView const& b, int64_t* scanTmp, int sms, cudaStream_t st);
// Transposed lists of the entries (per target, entry order) and the
// target -> centre map.
void launchExternalTranspose(BatchView const& b, int numTargets, const int* centerIndex, int* tCount, int* tFill,
                             int64_t* tOffset, int64_t* tEntryTmp, int64_t* tEntry, int* targetCenter,
                             int64_t* scanTmp, int sms, cudaStream_t st);
void launchExtrapolationCheck(DevModel const& m, BatchView const& b, int sms, cudaStream_t st);

// neighbour list of one structure into caller buffers, no device allocation
// (during stream capture the launches only; the status call then reads the
// count and the limit checks after a replay)
void neighborListNoAlloc(const double* positions, int64_t numAtoms, const double* box, double cutoff,
                         int64_t capacity, int64_t* offsets, int32_t* index, int32_t* image, double* d, double* dr,
                         int64_t* numEntries, cudaStream_t st);
void neighborListNoAllocStatus(int64_t numAtoms, const int64_t* offsets, int64_t capacity, int64_t* numEntries,
                               cudaStream_t st);

// instrumentation
void launchCountWork(DevModel const& m, BatchView const& b, unsigned long long* counts, int sms, cudaStream_t st);
double measureFmaPeak(int fp64, int sms);
// CutoffFunction::fdf of type 0..8 at n radii on the current device (FP64, or
// the FP32 per-triplet form of the mixed kernels with fp32 != 0).
void cutoffFunctionValues(int type, double rc, double alpha, int fp32, const double* r, int64_t n, double* f,
                          double* df);

} // namespace n2p2b200
