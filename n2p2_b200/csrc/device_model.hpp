// Plain-old-data layout of the model and of a batch of structures as the
// sm_100a kernels see them.  Shared by host (.cpp) and device (.cu) code.
#pragma once

#include <cstdint>

namespace n2p2b200 {

// Numbering follows the reference enums (CutoffFunction.h:44-72,
// SymFnc.h:43-65, NeuralNetwork.h:32-56) so stored codes read the same.
enum CutoffType { CT_HARD = 0, CT_COS, CT_TANHU, CT_TANH, CT_EXP, CT_POLY1, CT_POLY2, CT_POLY3, CT_POLY4 };
enum ScalingType { ST_NONE = 0, ST_SCALE, ST_CENTER, ST_SCALECENTER, ST_SCALESIGMA };
enum Activation {
    AF_UNSET = 0, AF_IDENTITY, AF_TANH, AF_LOGISTIC, AF_SOFTPLUS, AF_RELU,
    AF_GAUSSIAN, AF_COS, AF_REVLOGISTIC, AF_EXP, AF_HARMONIC
};

constexpr int kDevMaxElements = 8;
constexpr int kDevMaxLayers = 6;
constexpr int kMaxMembers = 32;     // members of one symmetry-function group
constexpr int kMaxSFPerElement = 512;
constexpr int kMaxNeurons = 128;    // widest layer of an atomic network

// One member of a symmetry-function group (SymGrpExpRad / SymGrpExpAngn /
// SymGrpExpAngw member arrays, e.g. SymGrpExpAngn.cpp:108-148).
struct DevMember
{
    double eta, rs, lambda, zeta;
    double factorNorm;     // angular: 2^(1-zeta)*scalingFactor; radial: scalingFactor
    double factorDeriv;    // angular: 2*eta/zeta/lambda
    double zetaLambda;     // zeta*lambda
    double gNorm;          // angular: factorNorm/scalingFactor (final G prefactor)
    int    sf;             // index of the symmetry function in its element
    int    rowE1, rowE2;   // derivative row in the neighbour-element tables of e1 / e2
    int    zetaInt;
    int    useIntPow;
    int    calcExp;        // recompute the Gaussian for this member
    int    expBase;        // Gaussian exp(-eta r^2) = base^expPow; -1: evaluate directly
    int    expPow;
};

struct DevGroup
{
    int    type;           // 2, 3, 9
    int    e1, e2;
    int    cutoffType;
    int    cutoffSlot;     // which precomputed f_c/df_c set this group uses
    int    memberBegin, memberCount;
    int    numBases;       // distinct exp(-eta r^2) bases of the group (<= kMaxBases)
    int    fast;           // all members rs == 0 and planned on staged bases
    double rc, rc2;
    double baseEta[4];
    // Member grid of an angular group: every member is one (eta, lambda,
    // zeta) combination of at most 2 x 2 x 4 slots, integer zeta, rs = 0.
    int    grid;           // 0: generic member loop
    int    gridNZ;         // zeta slots in use (<= 4)
    int    etaBase[2], etaPow[2];   // eta slot -> staged base and integer power
    int    zetaM1[4];      // zeta - 1 per zeta slot
    int    etaBits;        // binary digits of the largest etaPow (squares the eta slots share)
    int    zetaBits;       // binary digits of the largest zetaM1 in use (squares the zeta slots share)
    double lambdaVal[2];
    float  baseEtaF[4], lambdaValF[2];   // FP32 copies (the mixed form's per-triplet arithmetic)
    signed char comboMember[16];    // (etaSlot * 2 + lambdaSlot) * 4 + zetaSlot -> member, -1 if absent
};

// One compact symmetry function (SymFncCompRad, SymFncCompAngw): compact
// radial function on (rl, rc) (CompactFunction: center, 1/width), and for the
// angular type a compact function of the angle on (aLeft, aRight) radians.
struct DevCompactMember
{
    int    sf;             // index of the symmetry function in its element
    int    core;           // CompactCore
    int    asym;           // asymmetric polynomial ((2 - x) x argument)
    int    calcComp;       // narrow angular: recompute the r_jk radial part (else carry the last one)
    int    rIdx, aIdx;     // angular groups: the member's radial and angular part in the group's grid
    int    impure;         // narrow groups: index among the members whose carried j-k radial part may
                           // come from another radial part (see DevCompactGroup::walkBegin), else -1
    double rl, rc, rCenter, rScale;
    double aLeft, aRight, aCenter, aScale;
};

// Compact members sharing (type, e1[, e2]) (SymGrpCompRad / SymGrpCompAngn / SymGrpCompAngw), or
// all members of one weighted type (SymGrpCompRadWeighted / SymGrpCompAng{n,w}Weighted).
struct DevCompactGroup
{
    int    type;           // 20 radial, 21 angular narrow, 22 angular wide, 23 radial weighted,
                           // 24 angular narrow weighted, 25 angular wide weighted
    int    e1, e2;
    int    memberBegin, memberCount;
    int    nR, nA;         // angular groups: distinct radial and angular parts of the members
    int    fnBegin;        // into compactFns: the nR radial parts, then the nA angular parts
    int    walkBegin, walkEnd;   // narrow groups: the members replayed per pair for the carried j-k
                                 // radial part of the impure members (empty when there are none)
    int    numImpure;
    double rmin, rmax;     // group radial window (SymGrpComp*::addMember: rmin stays 0, rmax the
                           // largest upper boundary)
};

constexpr int kCorePoly2 = 6;   // core type "p2" (CoreFunction::Type, numbering of coreFdf)

// Limits of the staged compact angular kernels (k_compact.cu): distinct
// radial / angular parts per grid chunk, and for the narrow types (one chunk)
// the impure members and the members replayed per pair.
constexpr int kCompactStageRows = 10;
constexpr int kCompactStageCols = 8;
constexpr int kCompactImpure = 6;
constexpr int kCompactWalk = 16;

// One distinct part of an angular group's members: a radial part (core,
// asymmetric flag, window (left, right) = (rl, rc)) or an angular part (core,
// window in radians); center and scale as in CompactFunction::setLeftRight
// (CompactFunction.cpp:62-76).  Every member's value over a pair is the
// product of its radial part at r_ij and r_ik and its angular part at theta.
struct alignas(16) DevCompactFn
{
    double left, right, center, scale;
    int    core, asym;
};

// The groups of a model as a kernel argument (constant bank: warp-uniform
// loads, no per-thread copy) for the model-specialised symmetry-function
// kernels; models with more groups run the generic kernels.
constexpr int kParamGroups = 40;
struct DevGroupTable
{
    int count;
    int pad_;
    DevGroup g[kParamGroups];
};

constexpr int kMaxBases = 4;        // exponential bases per group
constexpr int kMaxStagedBases = 2;  // bases staged per neighbour for angular groups

// Cutoff function parameters (CutoffFunction::setCutoffRadius/Parameter,
// CutoffFunction.cpp:95-112).
struct DevCutoff
{
    int    type;
    int    pad_;
    double rc, rcinv, rci, iw, alpha;
    double tanhPre;        // CutoffFunction::TANH_PRE (CutoffFunction.cpp:28)
    float  rcF, rciF, iwF, pad2_;   // FP32 copies for the mixed form's per-triplet f_c(r_jk)
};

// Per symmetry function scaling (SymFnc::scale / unscale, SymFnc.cpp:169-223).
struct DevScaling
{
    int    type;
    int    pad_;
    double Smin, Gmin, Gmax, Gmean, scalingFactor;
};

struct DevElement
{
    int numSF;
    int sfBegin;                      // into the scaling array
    int groupBegin, groupCount;
    int compactBegin, compactCount;   // compact groups
    int rows[kDevMaxElements];        // derivative rows per neighbour element
    int tableBegin[kDevMaxElements];  // into rowTable: SF index of each row
    // atomic network
    int numLayers;
    int neurons[kDevMaxLayers];
    int activation[kDevMaxLayers];
    int wOffset[kDevMaxLayers];       // layer l (1..) weights W[l] (n_l x n_{l-1}) in `weights`
    int bOffset[kDevMaxLayers];
};

struct DevModel
{
    int numElements;
    int numCutoffSlots;
    int maxSF;
    int maxRows;
    int normalizeNeurons;
    int sortByDistance;   // an angular group has a cutoff below the largest: stage blocks sorted by r
    int allFast;          // 0, or the zeta slots (2, 4) when every group is planned (rs = 0 bases) and every
                          // angular group is on the member grid
    int powBits;          // binary digits of the largest integer power (eta or zeta) of any member grid
    double maxCutoff, maxCutoff2;
    DevElement el[kDevMaxElements];
    DevCutoff cutoff[4];
    const DevGroup*   groups;
    const DevMember*  members;
    const DevScaling* scaling;
    const int*        rowTable;
    const double*     weights;
    const double*     weightsT;       // weights with every matrix transposed ([n_{l-1}][n_l]), same offsets
    int numCompactGroups;
    int compactTypes;     // bit (type - 20) set for every compact type present
    double atomicNumber[kDevMaxElements];   // neighbour weights of the weighted compact functions
    const DevCompactGroup*  compactGroups;
    const DevCompactMember* compactMembers;
    const DevCompactFn*     compactFns;
    int compactRows;      // largest nR of a wide angular group
    int compactAngCore;   // the core of every angular part of the staged angular groups, or 0 if they differ
    int compactNarrowStaged;   // every narrow group fits the staged kernels (one grid chunk, a short walk)
    int compactCols;      // largest nA of a staged angular group
};

// Per structure geometry for the neighbour build.
struct DevStructInfo
{
    double box[9];        // normalised units, row k = box vector k
    double invbox[9];
    double boxPhys[9];    // physical units (for the optional remap)
    double invboxPhys[9];
    int    pbc[3];        // Structure::calculatePbcCopies (Structure.cpp:485-516)
    int    periodic;
    int    nc[3];         // cell grid
    int    stencil[3];    // cells searched on each side
    int    atomBegin, numAtoms;
    int    cellBegin;
    int    pad_;
};

// Status words written by kernels and read by the host after a launch.
struct DevStatus
{
    int overflowNeighbors;   // neighbour capacity exceeded
    int maxNeighbors;
    int64_t totalNeighbors;
    int extrapolationWarnings;
    int badInput;
    int tensorCoreTimeout;   // a tensor-core network tile gave up waiting for its MMAs
    int pad_;
    int64_t maskWords;       // candidate-acceptance words the evaluation needs (Batch::allocateMasks)
};

} // namespace n2p2b200
