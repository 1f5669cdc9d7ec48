/*
 * n2p2_b200.h -- C ABI of the B200 short-range (2G) HDNNP energy/force path.
 *
 * The entry points replace the short-range evaluation path of nnp::Mode
 * (reference: src/libnnp/Mode.h and Mode.cpp of n2p2).  A handle of type
 * n2p2_mode carries what an nnp::Mode object carries after setup (settings,
 * elements, symmetry functions, scaling, networks); a handle of type
 * n2p2_batch carries one or many nnp::Structure objects resident on the GPU.
 * Each function names the reference member function it stands for.
 *
 * Conventions
 *  - Every function returns an n2p2_status; 0 is success.  The message of the
 *    last failure on the calling thread is returned by n2p2_last_error().
 *    The status codes map the reference's exception types (see below); the
 *    C ABI itself never throws.
 *  - All arrays are plain host pointers unless a function says otherwise.
 *    Lengths are in elements.  Positions, forces and neighbour vectors are
 *    [atom][3] row-major doubles.  Boxes are [structure][3][3] with row k the
 *    k-th cell vector (Structure::box).
 *  - Element indices follow the element map of the settings file, i.e. the
 *    elements sorted by atomic number (ElementMap::registerElements).
 *  - Physical units are those of input.data; if the settings file defines
 *    mean_energy/conv_energy/conv_length the library normalises internally
 *    exactly like Prediction::readStructureFromFile / predict.
 */
#ifndef N2P2_B200_H
#define N2P2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int n2p2_status;

#define N2P2_OK 0
#define N2P2_ERR_RUNTIME 1          /* std::runtime_error (settings, files, state)  */
#define N2P2_ERR_RANGE 2            /* std::range_error                               */
#define N2P2_ERR_OUT_OF_RANGE 3     /* std::out_of_range (stop on extrapolation)      */
#define N2P2_ERR_INVALID_ARGUMENT 4 /* std::invalid_argument (cutoff parameters)      */
#define N2P2_ERR_CUDA 5             /* CUDA runtime failure                           */
#define N2P2_ERR_NULL 6             /* null handle or pointer                         */

/* Precision of the symmetry-function and network stages. */
#define N2P2_PRECISION_FP64 0       /* plain FP64 throughout                          */
#define N2P2_PRECISION_MIXED 1      /* FP32 descriptors, FP64 cutoff/scaling/sums     */

/* Flags of n2p2_batch_evaluate. */
#define N2P2_EVAL_FORCES 1          /* Mode::evaluateNNP(useForces = true)            */
#define N2P2_EVAL_STORE_DGDR 2      /* keep dG/dr per neighbour (Atom::Neighbor::dGdr) */
#define N2P2_EVAL_NO_GRAPH 4        /* launch kernels one by one (no CUDA graph)      */
#define N2P2_EVAL_SYMMETRY_FUNCTIONS_ONLY 8  /* Mode::calculateSymmetryFunctionGroups alone */

typedef struct n2p2_mode n2p2_mode;
typedef struct n2p2_batch n2p2_batch;
typedef struct n2p2_trainer n2p2_trainer;
typedef struct n2p2_training n2p2_training;
typedef struct n2p2_lammps n2p2_lammps;
typedef struct n2p2_structures n2p2_structures;

/* Message of the last failure on this thread ("" if none). */
const char* n2p2_last_error(void);

/* Library version string. */
const char* n2p2_version(void);

/* ---- model set-up: nnp::Mode ------------------------------------------------ */

/* new nnp::Mode bound to CUDA device `device` (Mode::Mode, Mode.cpp:43-54).
 * The device is first used when a batch is created; the set-up functions
 * work without a GPU. */
n2p2_status n2p2_mode_create(n2p2_mode** mode, int device);
n2p2_status n2p2_mode_destroy(n2p2_mode* mode);

/* Mode::initialize (Mode.cpp:56-160): prints nothing, kept for call parity. */
n2p2_status n2p2_mode_initialize(n2p2_mode* mode);

/* Mode::loadSettingsFile (Mode.cpp:162-211). */
n2p2_status n2p2_mode_load_settings_file(n2p2_mode* mode, const char* fileName);

/* Mode::setupGeneric (Mode.cpp:213-237), 2G-HDNNP path: normalisation,
 * element map, elements, cutoff, symmetry functions (sorted), derivative
 * tables, groups, network topology. */
n2p2_status n2p2_mode_setup_generic(n2p2_mode* mode);

/* Mode::setupSymmetryFunctionScaling (Mode.cpp:781-909). */
n2p2_status n2p2_mode_setup_symmetry_function_scaling(n2p2_mode* mode, const char* fileName);

/* Mode::setupSymmetryFunctionScalingNone (Mode.cpp:761-779). */
n2p2_status n2p2_mode_setup_symmetry_function_scaling_none(n2p2_mode* mode);

/* Mode::setupNeuralNetworkWeights (Mode.cpp:1514-1547); `fileNameFormat` is
 * a printf format taking the atomic number, e.g. "weights.%03zu.data". */
n2p2_status n2p2_mode_setup_neural_network_weights(n2p2_mode* mode, const char* fileNameFormat);

/* NeuralNetwork::setConnections (NeuralNetwork.cpp:147-169) for one element,
 * values in weights-file order. */
n2p2_status n2p2_mode_set_connections(n2p2_mode* mode, int element, const double* connections, int64_t count);

/* Mode::setupSymmetryFunctionStatistics (Mode.cpp:1172-1210).  Any non-zero
 * flag enables the extrapolation check of every evaluation; with
 * stopOnExtrapolationWarnings a warning makes evaluation fail with
 * N2P2_ERR_OUT_OF_RANGE, with writeExtrapolationWarnings one line per atom is
 * written to stderr. */
n2p2_status n2p2_mode_setup_symmetry_function_statistics(n2p2_mode* mode, int collectStatistics,
                                                         int collectExtrapolationWarnings,
                                                         int writeExtrapolationWarnings,
                                                         int stopOnExtrapolationWarnings);

/* Precision of later evaluations (N2P2_PRECISION_*). */
n2p2_status n2p2_mode_set_precision(n2p2_mode* mode, int precision);

/* Mode::getMaxCutoffRadius (Mode.h:513). */
n2p2_status n2p2_mode_get_max_cutoff_radius(n2p2_mode* mode, double* radius);

/* Number of elements; symbol and index of element e (ElementMap). */
n2p2_status n2p2_mode_get_num_elements(n2p2_mode* mode, int* count);
n2p2_status n2p2_mode_get_element_symbol(n2p2_mode* mode, int element, char* buffer, int capacity);
n2p2_status n2p2_mode_get_element_index(n2p2_mode* mode, const char* symbol, int* element);

/* Element::numSymmetryFunctions (Element.h:161). */
n2p2_status n2p2_mode_get_num_symmetry_functions(n2p2_mode* mode, int element, int* count);

/* Element::getSymmetryFunction(index) (Element.h:176): parameters of the
 * index-th symmetry function of `element` in the reference's sorted order:
 * type, e1, e2 and params = {eta, rs, lambda, zeta, rc, scalingFactor}
 * (internal length units). */
n2p2_status n2p2_mode_get_symmetry_function(n2p2_mode* mode, int element, int index, int* type, int* e1, int* e2,
                                            double* params);

/* Element::getSymmetryFunctionNumTable()[neighborElement] (Element.h:188):
 * dG/dr rows stored for a neighbour of element `neighborElement` around a
 * centre of element `element`. */
n2p2_status n2p2_mode_get_num_derivative_rows(n2p2_mode* mode, int element, int neighborElement, int* rows);
/* The atomic network of `element` (NeuralNetwork::getNumNeuronsPerLayer and the
 * layers' activation types, NeuralNetwork.h:32-56 numbering): *numLayers layers
 * including input and output; neurons[l] and activations[l] for l < capacity. */
n2p2_status n2p2_mode_get_network_topology(n2p2_mode* mode, int element, int capacity, int* numLayers, int* neurons,
                                           int* activations);

/* ---- structures on the GPU: nnp::Structure ---------------------------------- */

n2p2_status n2p2_batch_create(n2p2_mode* mode, n2p2_batch** batch);
n2p2_status n2p2_batch_destroy(n2p2_batch* batch);

/* Define the structures of the batch (Structure::readFromLines,
 * Structure.cpp:142-271, without the text parsing).  numAtoms[s] atoms per
 * structure, elements[atom], boxes[s][3][3] in physical units and
 * periodic[s] (0 = isolated cluster).  With remap != 0 periodic positions are
 * folded into the cell on the device exactly like Structure::remap
 * (Structure.cpp:1224-1248). */
n2p2_status n2p2_batch_set_structures(n2p2_batch* batch, int64_t numStructures, const int64_t* numAtoms,
                                      const int32_t* elements, const double* boxes, const int32_t* periodic,
                                      int remap);

/* Positions [atom][3] in physical units; `onDevice` says whether `positions`
 * is a device pointer.  Asynchronous on the batch's stream. */
n2p2_status n2p2_batch_set_positions(n2p2_batch* batch, const double* positions, int onDevice);

/* Mode::evaluateNNP (Mode.cpp:2029-2077) on every structure: neighbour list,
 * symmetry functions, networks, energies and (flag) forces.  Asynchronous
 * except for the first call after n2p2_batch_set_structures.  Later calls
 * replay the work with the neighbour buffers sized by the first; if new
 * positions make the lists longer than those buffers, the next call that
 * reads results (any n2p2_batch_get_*, n2p2_batch_synchronize,
 * n2p2_batch_evaluate_host) grows them and evaluates again before it returns,
 * so no result ever comes from a truncated list (the reference's list never
 * truncates, Structure.cpp:287-398). */
n2p2_status n2p2_batch_evaluate(n2p2_batch* batch, int flags);

/* ---- the stages of Mode::evaluateNNP as separate calls ----
 *
 * Same kernels as n2p2_batch_evaluate, launched one stage at a time on the
 * batch's stream, so the sequence neighbour list -> symmetry functions
 * (derivatives) -> atomic networks (derivatives) -> energy -> forces gives
 * the same bits as one evaluation.  The symmetry-function call keeps the
 * reference's caching flags (Structure::hasSymmetryFunctions /
 * hasSymmetryFunctionDerivatives, Mode.cpp:1634-1635): it returns at once
 * when the requested results exist.  New structures or positions clear every
 * flag; n2p2_batch_evaluate sets them.  A stage whose inputs were not
 * calculated fails with N2P2_ERR_RUNTIME. */
#define N2P2_DERIVATIVES_NONE 0     /* values only                                      */
#define N2P2_DERIVATIVES 1          /* derivatives, contracted with dE/dG by calculate_forces */
#define N2P2_DERIVATIVES_STORED 2   /* derivatives stored as Atom::dGdr / Atom::Neighbor::dGdr
                                       (n2p2_batch_get_dGdr; FP64, Gaussian functions only) */

/* Structure::calculateNeighborList(maxCutoffRadius, false)
 * (Structure.cpp:287-398) on every structure (with external lists: their
 * entries).  Synchronises (the entry count sizes the buffers). */
n2p2_status n2p2_batch_calculate_neighbor_list(n2p2_batch* batch);

/* Mode::calculateSymmetryFunctions (Mode.cpp:1549-1628) and
 * Mode::calculateSymmetryFunctionGroups (Mode.cpp:1630-1709): Atom::G of
 * every atom, the extrapolation check when statistics are set up, and
 * derivatives as `derivatives` says.  Both names compute the same values
 * (the reference's two loops differ only in how they visit the functions). */
n2p2_status n2p2_batch_calculate_symmetry_functions(n2p2_batch* batch, int derivatives);
n2p2_status n2p2_batch_calculate_symmetry_function_groups(n2p2_batch* batch, int derivatives);

/* Mode::calculateAtomicNeuralNetworks (Mode.cpp:1711-1732, 2G): Atom::energy
 * and, with derivatives != 0, Atom::dEdG. */
n2p2_status n2p2_batch_calculate_atomic_neural_networks(n2p2_batch* batch, int derivatives);

/* Mode::calculateEnergy (Mode.cpp:1876-1901): Structure::energy, read with
 * n2p2_batch_get_energies. */
n2p2_status n2p2_batch_calculate_energy(n2p2_batch* batch);

/* Mode::calculateForces (Mode.cpp:1922-1984): Atom::f, read with
 * n2p2_batch_get_forces; needs symmetry-function derivatives and dE/dG. */
n2p2_status n2p2_batch_calculate_forces(n2p2_batch* batch);

/* Wait for the batch's stream; reports device-side input errors. */
n2p2_status n2p2_batch_synchronize(n2p2_batch* batch);

/* Neighbour entries the batch's buffers hold now, and how many evaluations
 * were repeated because new positions outgrew them (no counterpart in the
 * reference, whose lists are std::vectors). */
n2p2_status n2p2_batch_get_neighbor_capacity(n2p2_batch* batch, int64_t* capacity, int64_t* recoveries);

/* Structure::energy per structure after Prediction::predict's conversion
 * (physical units, atomic energy offsets added). */
n2p2_status n2p2_batch_get_energies(n2p2_batch* batch, double* energies);

/* Atom::f of every atom in physical units, [atom][3]. */
n2p2_status n2p2_batch_get_forces(n2p2_batch* batch, double* forces);

/* End-to-end: copy positions from host memory, evaluate, copy energies and
 * forces back, all on the batch's stream (forces may be NULL without the
 * force flag).  Pinned host memory from n2p2_host_alloc gives the fastest copies. */
n2p2_status n2p2_batch_evaluate_host(n2p2_batch* batch, const double* positions, double* energies,
                                     double* forces, int flags);

/* Sizes. */
n2p2_status n2p2_batch_get_num_atoms(n2p2_batch* batch, int64_t* atoms);
n2p2_status n2p2_batch_get_num_neighbor_entries(n2p2_batch* batch, int64_t* entries);

/* Neighbour lists in internal units (Atom::neighbors): offsets[N+1],
 * index[M] (atom index in the batch), image[M] (periodic image code,
 * ((bc0+p0)(2p1+1) + (bc1+p1))(2p2+1) + (bc2+p2)), d[M], dr[M][3].
 * Any pointer may be NULL. */
n2p2_status n2p2_batch_get_neighbors(n2p2_batch* batch, int64_t* offsets, int32_t* index, int32_t* image,
                                     double* d, double* dr);

/* Atom::G, Atom::dEdG (concatenated per atom, numSymmetryFunctions values each)
 * and Atom::energy (internal units). */
n2p2_status n2p2_batch_get_symmetry_functions(n2p2_batch* batch, double* G);
n2p2_status n2p2_batch_get_dEdG(n2p2_batch* batch, double* dEdG);
n2p2_status n2p2_batch_get_atomic_energies(n2p2_batch* batch, double* energies);

/* Symmetry-function statistics of the last evaluation, as nnp-scaling
 * collects them (SymFncStatistics::addValue, SymFncStatistics.cpp:80-89, over
 * the unscaled G of every atom; Dataset::collectSymmetryFunctionStatistics):
 * counts[e] = atoms of element e; stats = per element e, four arrays of
 * numSymmetryFunctions(e) values: minimum, maximum, sum, sum of squares.
 * Sums are taken in atom order in chunks of 1024 atoms, the chunks added in
 * order (the same result on every run). */
n2p2_status n2p2_batch_get_symmetry_function_statistics(n2p2_batch* batch, int64_t* counts, double* stats);

/* Atom::dGdr (self, [sum numSF][3]) and Atom::Neighbor::dGdr (per entry,
 * numDerivativeRows of the pair, [rows][3]); needs N2P2_EVAL_STORE_DGDR. */
n2p2_status n2p2_batch_get_dGdr(n2p2_batch* batch, double* selfDGdr, double* neighborDGdr);

/* Positions after remap and normalisation (internal units), [atom][3]. */
n2p2_status n2p2_batch_get_internal_positions(n2p2_batch* batch, double* positions);

/* Extrapolation warnings of the last evaluation: total and per atom (may be NULL). */
n2p2_status n2p2_batch_get_extrapolation_warnings(n2p2_batch* batch, int64_t* total, int32_t* perAtom);

/* Kernel launches issued by one evaluation with the last flags. */
n2p2_status n2p2_batch_get_launch_count(n2p2_batch* batch, int* launches);

/* ---- allocation-free neighbour list (no counterpart in the reference) ---- */

/* Neighbour list of ONE structure, written into device buffers the caller
 * owns, for callers that cannot call cudaMalloc where they need the list: a
 * code whose device memory belongs to its own pool allocator, or a step loop
 * that must not pay cudaMalloc's device-wide synchronisation.  Nothing is allocated: the scratch (cell
 * lists, counts, scan partials) is one fixed array in the library's device
 * memory (about 0.7 MB, held by every GPU that loads the library until the
 * process exits), shared by all calls.  Calls that overlap on the GPU race
 * on it; the first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and should come before any stream capture.  That
 * address is kept per device for the life of the process: after a
 * cudaDeviceReset in the host process it is stale, and the entry point must
 * not be called again in that process.
 *
 * positions: device [numAtoms][3], internal units, inside the cell (e.g.
 * n2p2_batch_get_internal_positions); box: host [3][3] in the same units, or
 * NULL for a cluster; offsets: device [numAtoms+1]; index, image, d: device
 * [capacity]; dr: device [capacity][3].  Entries are those of
 * n2p2_batch_get_neighbors (same order and bit-identical values).  Limits:
 * numAtoms <= 8192, at most 32768 cells, at most 256 neighbours per atom;
 * larger inputs are rejected with N2P2_ERR_RUNTIME.  The call waits for its
 * stream (`stream` is a cudaStream_t, NULL = default stream) and stores the
 * entry count in *numEntries.
 *
 * While `stream` is being captured into a CUDA graph the call only records
 * its work (no host copy, no wait: neither may be captured) and sets
 * *numEntries to -1; host-side rejections (atom count, cutoff, cell count)
 * still happen at capture.  After a replay of the graph,
 * n2p2_neighbor_list_noalloc_status reads the count and the device-side
 * checks (atoms outside the cell, more than 256 neighbours, capacity) of the
 * last run on the device, waiting for `stream`, with the same errors. */
n2p2_status n2p2_neighbor_list_noalloc(const double* positions, int64_t numAtoms, const double* box, double cutoff,
                                       int64_t capacity, int64_t* offsets, int32_t* index, int32_t* image,
                                       double* d, double* dr, int64_t* numEntries, void* stream);
n2p2_status n2p2_neighbor_list_noalloc_status(int64_t numAtoms, const int64_t* offsets, int64_t capacity,
                                              int64_t* numEntries, void* stream);

/* ---- structure files --------------------------------------------------------
 * input.data read in one pass: Structure::readFromLines (Structure.cpp:142-271)
 * on every begin..end block, numbers through strtod (bit-identical to the
 * reference's), the reference's error messages (N2P2_ERR_RUNTIME; a short
 * atom line N2P2_ERR_OUT_OF_RANGE).  A trailing block without "end" is not
 * read.  limit < 0 reads every structure. */
n2p2_status n2p2_structures_read_file(const char* fileName, int64_t limit, n2p2_structures** structures);
n2p2_status n2p2_structures_read_text(const char* text, int64_t length, int64_t limit,
                                      n2p2_structures** structures);
n2p2_status n2p2_structures_destroy(n2p2_structures* structures);
n2p2_status n2p2_structures_get_count(n2p2_structures* structures, int64_t* numStructures, int64_t* numAtoms);
/* Per structure: atoms, box [3][3] (rows = lattice vectors; zeros without
 * one), periodic flag, reference energy and total charge (any pointer may be NULL). */
n2p2_status n2p2_structures_get_structure_arrays(n2p2_structures* structures, int64_t* numAtoms, double* boxes,
                                                 int32_t* periodic, double* energies, double* charges);
/* Per atom, all structures concatenated: position [3], element symbol
 * (4 bytes, NUL-padded), charge, reference force [3] (any pointer may be NULL). */
n2p2_status n2p2_structures_get_atom_arrays(n2p2_structures* structures, double* positions, char* elements,
                                            double* charges, double* forces);
n2p2_status n2p2_structures_get_comment(n2p2_structures* structures, int64_t index, char* buffer,
                                        int32_t capacity);

/* ---- LAMMPS interface ------------------------------------------------------
 * nnp::InterfaceLammps (src/libnnpif/LAMMPS/InterfaceLammps.h:31-333), the
 * object `pair_style hdnnp` (src/interface/LAMMPS/src/ML-HDNNP/pair_hdnnp.cpp)
 * drives every MD step: local atoms and their full neighbour lists (local and
 * ghost neighbours, LAMMPS indices) in, energy and forces on local AND ghost
 * atoms out (LAMMPS folds the ghost forces back to their owners).  2G models.
 * Units: LAMMPS units in and out, converted with cflength/cfenergy as the
 * reference does.  The neighbours' forces are gathered on the device per
 * target atom in a fixed order (no atomics).  Extra over the reference:
 * n2p2_lammps_set_precision and n2p2_lammps_transfer_neighbor_list. */
n2p2_status n2p2_lammps_create(n2p2_lammps** lammps, int device);
n2p2_status n2p2_lammps_destroy(n2p2_lammps* lammps);
/* InterfaceLammps::initialize (InterfaceLammps.cpp:51-255): reads
 * directory/input.nn, scaling.data and weights.%03zu.data; emap "1:H,2:O"
 * maps LAMMPS types to elements (empty: type t is element t-1, requires
 * lammpsNtypes == number of elements; unmapped types are ignored); errors
 * of the reference (cutoff smaller than the largest symmetry-function cutoff,
 * inconsistent or invalid map) as N2P2_ERR_RUNTIME.  Extrapolation warnings
 * are counted when showew, showewsum > 0 or maxew >= 0; resetew, showewsum,
 * maxew and myRank are the pair style's business (kept for the signature). */
n2p2_status n2p2_lammps_initialize(n2p2_lammps* lammps, const char* directory, const char* emap, int32_t showew,
                                   int32_t resetew, int32_t showewsum, int32_t maxew, double cflength,
                                   double cfenergy, double lammpsCutoff, int32_t lammpsNtypes, int32_t myRank);
/* N2P2_PRECISION_FP64 (default) or N2P2_PRECISION_MIXED. */
n2p2_status n2p2_lammps_set_precision(n2p2_lammps* lammps, int precision);
/* InterfaceLammps::getMaxCutoffRadius (InterfaceLammps.cpp:528-532), LAMMPS units. */
n2p2_status n2p2_lammps_get_max_cutoff_radius(n2p2_lammps* lammps, double* radius);
/* InterfaceLammps::setLocalAtoms (InterfaceLammps.cpp:267-304): atomType[i]
 * = LAMMPS type (1-based) of local atom i; clears the neighbour lists. */
n2p2_status n2p2_lammps_set_local_atoms(n2p2_lammps* lammps, int32_t numAtomsLocal, const int32_t* atomType);
/* InterfaceLammps::addNeighbor (InterfaceLammps.cpp:410-441): neighbour j
 * (LAMMPS index, local or ghost) of local atom i, with j's tag and type,
 * dx = x_i - x_j (LAMMPS units) and d2 = |dx|^2.  Tags are not used by 2G
 * models.  Neighbours beyond the largest symmetry-function cutoff are dropped
 * (they contribute nothing in the reference either). */
n2p2_status n2p2_lammps_add_neighbor(n2p2_lammps* lammps, int32_t i, int32_t j, int64_t tag, int32_t type,
                                     double dx, double dy, double dz, double d2);
/* PairHDNNP::transferNeighborList (pair_hdnnp.cpp:274-290) in one call,
 * with LAMMPS's own arrays: list->inum, ilist, numneigh, firstneigh
 * (special-bond bits masked as NEIGHMASK does), atom->x, atom->type; every
 * pair with d2 <= maxCutoffRadius^2 (the pair style's cutoff) is added. */
n2p2_status n2p2_lammps_transfer_neighbor_list(n2p2_lammps* lammps, int32_t inum, const int32_t* ilist,
                                               const int32_t* numneigh, const int32_t* const* firstneigh,
                                               const double* const* x, const int32_t* type,
                                               double maxCutoffRadius);
/* InterfaceLammps::process (InterfaceLammps.cpp:463-500): symmetry
 * functions, networks, energy and the force pass on the device. */
n2p2_status n2p2_lammps_process(n2p2_lammps* lammps);
/* InterfaceLammps::getEnergy / getAtomicEnergy (InterfaceLammps.cpp:550-570),
 * LAMMPS units; `index` counts the local atoms of mapped types. */
n2p2_status n2p2_lammps_get_energy(n2p2_lammps* lammps, double* energy);
n2p2_status n2p2_lammps_get_atomic_energy(n2p2_lammps* lammps, int32_t index, double* energy);
/* InterfaceLammps::getForces (InterfaceLammps.cpp:679-740): ADDS the forces
 * (LAMMPS units) on every local and ghost atom named by the lists to
 * atomF[k][0..2] (LAMMPS's atom->f rows). */
n2p2_status n2p2_lammps_get_forces(n2p2_lammps* lammps, double* const* atomF);
/* Mode::getNumExtrapolationWarnings: out-of-range (atom, symmetry function)
 * occurrences summed over process() calls since the last
 * clearExtrapolationWarnings (InterfaceLammps.cpp:1049-1058; the pair style
 * clears after every step). */
n2p2_status n2p2_lammps_get_num_extrapolation_warnings(n2p2_lammps* lammps, int64_t* count);
n2p2_status n2p2_lammps_clear_extrapolation_warnings(n2p2_lammps* lammps);

/* ---- training on energies and forces --------------------------------------
 * The reference trains with nnp::Training (libnnptrain/Training.cpp) on the
 * CPU; these entry points train a mode's networks on the GPU instead (used for
 * the distilled student model): the loss
 *   L = wE/S sum_s ((E_s - E_s^ref)/N_s)^2 + wF/(3N) sum_k |F_k - F_k^ref|^2
 * in internal units, its exact gradient (through dE/dG for the force term)
 * and Adam steps as in GradientDescent::update (GradientDescent.cpp:89-113).
 * Supported networks: at most two hidden layers of <= 32 neurons, <= 128
 * symmetry functions per element, activations l, t, s, p, no normalize_nodes
 * (N2P2_ERR_INVALID_ARGUMENT otherwise).  The trainer updates the mode's
 * device weights in place; evaluations of the mode's batches use them. */
n2p2_status n2p2_trainer_create(n2p2_mode* mode, n2p2_trainer** trainer);
n2p2_status n2p2_trainer_destroy(n2p2_trainer* trainer);
/* Adam parameters (defaults 1e-3, 0.9, 0.999, 1e-8). */
n2p2_status n2p2_trainer_set_adam(n2p2_trainer* trainer, double eta, double beta1, double beta2, double epsilon);
/* Step size of the following Adam updates (moments and bias correction kept). */
n2p2_status n2p2_trainer_set_learning_rate(n2p2_trainer* trainer, double eta);
/* Loss weights wE, wF (defaults 1, 10). */
n2p2_status n2p2_trainer_set_loss_weights(n2p2_trainer* trainer, double energyWeight, double forceWeight);
n2p2_status n2p2_trainer_get_num_parameters(n2p2_trainer* trainer, int64_t* count);
/* All weights and biases, element by element in weight-file order
 * (NeuralNetwork::setConnections, NeuralNetwork.cpp:147-169). */
n2p2_status n2p2_trainer_get_parameters(n2p2_trainer* trainer, double* parameters);
n2p2_status n2p2_trainer_set_parameters(n2p2_trainer* trainer, const double* parameters);
/* Evaluates `batch` (a batch of the trainer's mode, positions set) with
 * forces, computes the loss against energies[S] (physical units, with atomic
 * energy offsets) and forces[N][3] (physical units) and, if `update`, takes
 * one Adam step.  loss[3] = {total, energy term, force term} and the gradient
 * (weight-file order) are written when the pointers are not NULL. */
n2p2_status n2p2_trainer_step(n2p2_trainer* trainer, n2p2_batch* batch, const double* energies,
                              const double* forces, int32_t update, double* loss, double* gradient);

/* ---- training updates (libnnptrain Training::update, KalmanFilter,
 * GradientDescent) -----------------------------------------------------------
 * Replaces the update loop of the reference's nnp-train
 * (src/libnnptrain/Training.cpp:2256-3169) for the 2G networks with the
 * combined update strategy and one update candidate per update (observation
 * size 1), and its updaters (KalmanFilter.cpp:126-238,
 * GradientDescent.cpp:81-118).  The training set is the batch's structures:
 * their symmetry functions and dG/dr are computed at creation and stay on the
 * device; the networks' weights are the mode's device weights, which the
 * updates change in place (every later evaluation of the mode's batches uses
 * them). */
#define N2P2_TRAINING_ENERGY 0
#define N2P2_TRAINING_FORCE 1
n2p2_status n2p2_training_create(n2p2_batch* set, n2p2_training** training);
n2p2_status n2p2_training_destroy(n2p2_training* training);
/* energies[S] (physical units, with offsets) and forces[N][3]: the references
 * of the set's structures (Structure::energyRef, Atom::fRef). */
n2p2_status n2p2_training_set_references(n2p2_training* training, const double* energies, const double* forces);
/* force_weight (Training.cpp:2910-2923): scales force errors and Jacobians. */
n2p2_status n2p2_training_set_force_weight(n2p2_training* training, double weight);
/* update_strategy (0 combined: one updater over all weights; 1 element: one updater per element over its
 * network's weights, the error shared by the element's fraction of the structure's atoms or of the observed
 * atom's neighbours, Training.cpp:2900-2922).  Set it before the updater; it resets the updater. */
#define N2P2_TRAINING_COMBINED 0
#define N2P2_TRAINING_ELEMENT 1
n2p2_status n2p2_training_set_update_strategy(n2p2_training* training, int32_t strategy);
/* jacobian_mode (0, 1: a task batch's candidates summed into one observation; 2: every candidate its own
 * observation, one Kalman update with an m x m gain, KalmanFilter.cpp:130-162 with sizeObservation m;
 * combined strategy, Kalman filter, at most 16 candidates per update). */
n2p2_status n2p2_training_set_jacobian_mode(n2p2_training* training, int32_t mode);
/* task_batch_size_energy / task_batch_size_force (Training.cpp:2277-2279 with jacobian_mode 0 or 1 on one
 * process): that many consecutive candidates form one observation (errors and Jacobians summed at the same
 * weights) and one updater step. */
n2p2_status n2p2_training_set_task_batch_size(n2p2_training* training, int32_t energy, int32_t force);
/* KalmanFilter::setParametersStandard / setParametersFadingMemory (P = I / epsilon). */
n2p2_status n2p2_training_set_kalman_standard(n2p2_training* training, double epsilon, double q0, double qtau,
                                              double qmin, double eta0, double etatau, double etamax);
n2p2_status n2p2_training_set_kalman_fading_memory(n2p2_training* training, double epsilon, double q0, double qtau,
                                                   double qmin, double lambda, double nu);
/* GradientDescent::setParametersFixed / setParametersAdam. */
n2p2_status n2p2_training_set_gradient_fixed(n2p2_training* training, double eta);
n2p2_status n2p2_training_set_gradient_adam(n2p2_training* training, double eta, double beta1, double beta2,
                                            double epsilon);
/* `count` candidates in order, one update per task batch of them (count a
 * multiple of the task batch size).  property N2P2_TRAINING_ENERGY: the energy of
 * structure[k]; N2P2_TRAINING_FORCE: component component[k] (0..2) of atom
 * atom[k] (index inside the structure) of structure[k]; atom and component
 * may be NULL for energy updates.  errors[k] (optional): reference minus
 * prediction before update k, internal units. */
n2p2_status n2p2_training_update(n2p2_training* training, int32_t property, int32_t count, const int32_t* structure,
                                 const int32_t* atom, const int32_t* component, double* errors);
/* The error (reference minus prediction, internal units) and Jacobian
 * (weight-file order; the force weight applied to force observations) of one
 * observation at the current weights, without an update: the quantities
 * Training::update hands to its updater. */
n2p2_status n2p2_training_observe(n2p2_training* training, int32_t property, int32_t structure, int32_t atom,
                                  int32_t component, double* error, double* jacobian);
/* selection_mode 2 (threshold, Training.cpp:2288-2527): num_updates updates; each tries the candidates
 * of the list in order (wrapping), at most `trials`, until one's |error| exceeds threshold x rmse (rmse:
 * the training RMSE in internal units -- energy per atom times the structure's atoms, or force component);
 * the update uses the candidate the trials stopped at (the reference's behaviour also when none exceeds).
 * *consumed receives the number of candidates taken from the list, errors[u] the used one's error. */
n2p2_status n2p2_training_update_threshold(n2p2_training* training, int32_t property, int32_t num_updates,
                                           int32_t num_candidates, const int32_t* structure, const int32_t* atom,
                                           const int32_t* component, double threshold, int32_t trials, double rmse,
                                           int32_t* consumed, double* errors);
/* Training errors at the current weights, internal units (Training::calculateError): RMSE of the energy
 * per atom and of the force components over the set; errors[2]. */
n2p2_status n2p2_training_get_errors(n2p2_training* training, double* errors);
/* KalmanFilter::status: {numUpdates, mean |P_ii|, mean |P_ij| (i != j),
 * mean |K|, q, eta (standard) or lambda (fading memory), gamma}. */
n2p2_status n2p2_training_get_kalman_status(n2p2_training* training, double* status);
n2p2_status n2p2_training_get_num_weights(n2p2_training* training, int64_t* count);
/* All elements' connections, weight-file order (NeuralNetwork::getConnections). */
n2p2_status n2p2_training_get_weights(n2p2_training* training, double* weights);
n2p2_status n2p2_training_set_weights(n2p2_training* training, const double* weights);

/* ---- the training program's shuffles ----------------------------------------
 * The reference's training loop orders its update candidates and its epoch
 * schedule with std::shuffle driven by std::mt19937_64 generators
 * (Training::rngNew / rngGlobalNew, Training.h:577-579; shuffleUpdateCandidates
 * and setEpochSchedule, Training.cpp:2062-2111), seeded from its GSL
 * generators.  These calls run that standard-library code, so a host driver
 * of the training loop draws the same permutations as the reference built
 * with the same C++ library. */
typedef struct n2p2_shuffle_rng n2p2_shuffle_rng;
/* std::mt19937_64 seeded with `seed` (std::mt19937_64::seed). */
n2p2_status n2p2_shuffle_rng_create(uint64_t seed, n2p2_shuffle_rng** rng);
n2p2_status n2p2_shuffle_rng_destroy(n2p2_shuffle_rng* rng);
/* std::shuffle(values, values + count, generator). */
n2p2_status n2p2_shuffle_rng_shuffle(n2p2_shuffle_rng* rng, int64_t* values, int64_t count);

/* ---- autotuning (no counterpart in the reference) -------------------------
 * The symmetry-function passes run their first tier of atoms with one of
 * three kernel shapes (stage capacity x warps per block: 0 = 128 x 4,
 * 1 = 160 x 4, 2 = 192 x 2).  Before a batch's first graph capture in a
 * precision the shapes are chosen per pass by timing all three on the batch
 * (or taken from the cache file N2P2_B200_TUNE_CACHE, default
 * ~/.cache/n2p2_b200/autotune.json).  Results do not depend on the shape. */
/* Enable (default) or disable the automatic tuning for the mode's batches. */
n2p2_status n2p2_mode_set_autotune(n2p2_mode* mode, int32_t enabled);
/* Tune now for the mode's current precision (the batch must have been
 * evaluated once); shapes[2] = {G pass, force pass}, ms[6] = the measured
 * times per shape (zeros when taken from the cache), *fromCache. */
n2p2_status n2p2_batch_autotune(n2p2_batch* batch, int32_t useCache, int32_t* shapes, double* ms,
                                int32_t* fromCache);
/* Fix the shapes for the mode's current precision (no tuning). */
n2p2_status n2p2_batch_set_shapes(n2p2_batch* batch, int32_t valuesShape, int32_t forcesShape);

/* ---- instrumentation (no counterpart in the reference) ------------------- */

/* The CUDA stream (cudaStream_t) the batch's kernels run on, for event timing. */
n2p2_status n2p2_batch_get_stream(n2p2_batch* batch, void** stream);

/* One direct (non-graph) evaluation with CUDA events between the stages.
 * Writes up to `capacity` stage names (32 bytes each, NUL-terminated) and
 * their durations in milliseconds; *count receives the number of stages. */
n2p2_status n2p2_batch_profile_stages(n2p2_batch* batch, int flags, int capacity, char* names, double* ms,
                                      int* count);

/* Algorithmic work of the batch's current neighbour lists, 10 counters:
 * entries, radial pair-members, radial pairs, narrow triplets, narrow
 * triplet-members, wide pairs, wide pair-members, G values, atoms,
 * derivative rows. */
n2p2_status n2p2_batch_count_work(n2p2_batch* batch, int64_t* counts);

/* Measured fused-multiply-add throughput of the device (TFLOP/s), the
 * compute roofline of the FP64 and FP32 symmetry-function kernels. */
n2p2_status n2p2_device_fma_peak(int device, double* fp64Tflops, double* fp32Tflops);

/* CutoffFunction::fdf (CutoffFunction.h:210-220; setCutoffRadius and
 * setCutoffParameter, CutoffFunction.cpp:95-112) of cutoff type 0..8 (hard,
 * cos, tanhU, tanh, exp, poly1..poly4; the settings file's cutoff_type) at n
 * radii, evaluated on the device as the symmetry-function kernels evaluate
 * it: N2P2_PRECISION_FP64 is the every-pair form, N2P2_PRECISION_MIXED the
 * FP32 form of the mixed kernels' per-triplet f_c(r_jk).  A diagnostic;
 * 0 <= alpha < 1 as in the reference (N2P2_ERR_INVALID_ARGUMENT otherwise). */
n2p2_status n2p2_cutoff_function(int device, int type, double rc, double alpha, int precision, const double* r,
                                  int64_t n, double* f, double* df);

/* Pinned (page-locked) host memory for fast transfers. */
n2p2_status n2p2_host_alloc(void** ptr, size_t bytes);
n2p2_status n2p2_host_free(void* ptr);

#ifdef __cplusplus
}
#endif

#endif /* N2P2_B200_H */
