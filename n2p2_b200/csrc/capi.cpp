// extern "C" boundary; see include/n2p2_b200.h.  Exceptions of the C++ layer
// are turned into status codes here and never cross the ABI.
#include "../../include/n2p2_b200.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "engine.hpp"
#include "host_model.hpp"
#include "lammps.hpp"
#include "structure_io.hpp"
#include "trainer.hpp"

using namespace n2p2b200;

struct n2p2_mode
{
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    Model model;
    DeviceModel dmodel;
    bool uploaded = false;
    int precision = PREC_FP64;
    bool checkExtrapolation = false;
    bool autotune = true;
    bool writeWarnings = false;
    bool stopOnWarnings = false;
};

struct n2p2_trainer
{
    n2p2_mode* mode = nullptr;
    std::unique_ptr<Trainer> trainer;
};

struct n2p2_training
{
    n2p2_mode* mode = nullptr;
    n2p2_batch* set = nullptr;
    std::unique_ptr<Training> training;
};

struct n2p2_lammps
{
    n2p2_mode mode;                  // the model, its device copy and the stream
    std::unique_ptr<Batch> batch;    // created by the first process()
    LammpsInterface iface;
    int64_t warnings = 0;
};

struct n2p2_structures
{
    StructureSet set;
};

struct n2p2_batch
{
    n2p2_mode* mode = nullptr;
    std::unique_ptr<Batch> batch;
    int lastFlags = 0;
    int64_t lastWarnings = 0;
};

namespace {

thread_local std::string g_error;

n2p2_status fail(int code, std::string const& msg)
{
    g_error = msg;
    return code;
}

template <class F>
n2p2_status guard(F&& f)
{
    try
    {
        f();
        return N2P2_OK;
    }
    catch (std::out_of_range const& e)
    {
        return fail(N2P2_ERR_OUT_OF_RANGE, e.what());
    }
    catch (std::range_error const& e)
    {
        return fail(N2P2_ERR_RANGE, e.what());
    }
    catch (std::invalid_argument const& e)
    {
        return fail(N2P2_ERR_INVALID_ARGUMENT, e.what());
    }
    catch (std::runtime_error const& e)
    {
        std::string m = e.what();
        return fail(m.rfind("CUDA error", 0) == 0 ? N2P2_ERR_CUDA : N2P2_ERR_RUNTIME, m);
    }
    catch (std::exception const& e)
    {
        return fail(N2P2_ERR_RUNTIME, e.what());
    }
}

// The device is touched only when the first batch is created, so the
// set-up half of the API (settings, symmetry functions, scaling, weights)
// also works on a host without a GPU.
void setDevice(n2p2_mode* m)
{
    cudaCheck(cudaSetDevice(m->device), "cudaSetDevice");
    if (!m->stream)
    {
        cudaDeviceProp p{};
        cudaCheck(cudaGetDeviceProperties(&p, m->device), "cudaGetDeviceProperties");
        m->sms = p.multiProcessorCount;
        cudaCheck(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    }
}

void ensureUploaded(n2p2_mode* m)
{
    setDevice(m);
    if (!m->uploaded)
    {
        m->dmodel.upload(m->model);
        m->uploaded = true;
    }
}

#define N2P2_REQUIRE(p)                                                      \
    do                                                                       \
    {                                                                        \
        if (!(p)) return fail(N2P2_ERR_NULL, "null handle or pointer: " #p); \
    } while (0)

void afterEvaluate(n2p2_batch* b)
{
    n2p2_mode* m = b->mode;
    if (!m->checkExtrapolation) return;
    DevStatus st = b->batch->status();
    b->lastWarnings = st.extrapolationWarnings;
    if (st.extrapolationWarnings > 0)
    {
        if (m->writeWarnings)
        {
            std::vector<int> w(b->batch->numAtoms());
            b->batch->copyAtomWarnings(w.data());
            for (size_t a = 0; a < w.size(); ++a)
                if (w[a] > 0)
                    std::fprintf(stderr, "### NNP EXTRAPOLATION WARNING ### ATOM: %9zu SYMFUNCS OUT OF RANGE: %d\n", a,
                                 w[a]);
        }
        if (m->stopOnWarnings)
            throw std::out_of_range("### NNP EXTRAPOLATION WARNING ### ERROR: Symmetry function value out of range.\n");
    }
}

} // namespace

extern "C" {

const char* n2p2_last_error(void) { return g_error.c_str(); }

const char* n2p2_version(void) { return "n2p2_b200 0.1 (sm_100a)"; }

n2p2_status n2p2_mode_create(n2p2_mode** mode, int device)
{
    N2P2_REQUIRE(mode);
    return guard([&] {
        auto m = std::make_unique<n2p2_mode>();
        m->device = device;
        *mode = m.release();
    });
}

n2p2_status n2p2_mode_destroy(n2p2_mode* mode)
{
    if (!mode) return N2P2_OK;
    return guard([&] {
        cudaStream_t s = mode->stream;
        if (s) cudaSetDevice(mode->device);
        delete mode;
        if (s) cudaStreamDestroy(s);
    });
}

n2p2_status n2p2_mode_initialize(n2p2_mode* mode)
{
    N2P2_REQUIRE(mode);
    return N2P2_OK;
}

n2p2_status n2p2_mode_load_settings_file(n2p2_mode* mode, const char* fileName)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(fileName);
    return guard([&] {
        mode->model.loadSettingsFile(fileName);
        mode->uploaded = false;
    });
}

n2p2_status n2p2_mode_setup_generic(n2p2_mode* mode)
{
    N2P2_REQUIRE(mode);
    return guard([&] {
        mode->model.setupGeneric();
        mode->uploaded = false;
    });
}

n2p2_status n2p2_mode_setup_symmetry_function_scaling(n2p2_mode* mode, const char* fileName)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(fileName);
    return guard([&] {
        mode->model.setupSymmetryFunctionScaling(fileName);
        mode->uploaded = false;
    });
}

n2p2_status n2p2_mode_setup_symmetry_function_scaling_none(n2p2_mode* mode)
{
    N2P2_REQUIRE(mode);
    return guard([&] {
        mode->model.setupSymmetryFunctionScalingNone();
        mode->uploaded = false;
    });
}

n2p2_status n2p2_mode_setup_neural_network_weights(n2p2_mode* mode, const char* fileNameFormat)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(fileNameFormat);
    return guard([&] {
        mode->model.setupNeuralNetworkWeights(fileNameFormat);
        mode->uploaded = false;
    });
}

n2p2_status n2p2_mode_set_connections(n2p2_mode* mode, int element, const double* connections, int64_t count)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(connections);
    return guard([&] {
        if (element < 0 || element >= (int)mode->model.numElements())
            throw std::runtime_error("ERROR: element index out of range.\n");
        mode->model.setConnections(element, std::vector<double>(connections, connections + count));
        mode->uploaded = false;
    });
}

n2p2_status n2p2_mode_setup_symmetry_function_statistics(n2p2_mode* mode, int collectStatistics,
                                                         int collectExtrapolationWarnings,
                                                         int writeExtrapolationWarnings,
                                                         int stopOnExtrapolationWarnings)
{
    N2P2_REQUIRE(mode);
    mode->checkExtrapolation =
        collectStatistics || collectExtrapolationWarnings || writeExtrapolationWarnings || stopOnExtrapolationWarnings;
    mode->writeWarnings = writeExtrapolationWarnings != 0;
    mode->stopOnWarnings = stopOnExtrapolationWarnings != 0;
    return N2P2_OK;
}

n2p2_status n2p2_mode_set_precision(n2p2_mode* mode, int precision)
{
    N2P2_REQUIRE(mode);
    if (precision != N2P2_PRECISION_FP64 && precision != N2P2_PRECISION_MIXED)
        return fail(N2P2_ERR_INVALID_ARGUMENT, "unknown precision");
    mode->precision = precision;
    return N2P2_OK;
}

n2p2_status n2p2_mode_get_max_cutoff_radius(n2p2_mode* mode, double* radius)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(radius);
    *radius = mode->model.maxCutoffRadius;
    return N2P2_OK;
}

n2p2_status n2p2_mode_get_num_elements(n2p2_mode* mode, int* count)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(count);
    *count = (int)mode->model.numElements();
    return N2P2_OK;
}

n2p2_status n2p2_mode_get_element_symbol(n2p2_mode* mode, int element, char* buffer, int capacity)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(buffer);
    return guard([&] {
        std::string const& s = mode->model.elements.at(element).symbol;
        if ((int)s.size() + 1 > capacity) throw std::runtime_error("buffer too small");
        std::memcpy(buffer, s.c_str(), s.size() + 1);
    });
}

n2p2_status n2p2_mode_get_element_index(n2p2_mode* mode, const char* symbol, int* element)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(symbol);
    N2P2_REQUIRE(element);
    return guard([&] { *element = mode->model.elementMap.index(symbol); });
}

n2p2_status n2p2_mode_get_num_symmetry_functions(n2p2_mode* mode, int element, int* count)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(count);
    return guard([&] { *count = (int)mode->model.elements.at(element).sf.size(); });
}

n2p2_status n2p2_mode_get_symmetry_function(n2p2_mode* mode, int element, int index, int* type, int* e1, int* e2,
                                            double* params)
{
    N2P2_REQUIRE(mode);
    return guard([&] {
        SymFunc const& s = mode->model.elements.at(element).sf.at(index);
        if (type) *type = s.type;
        if (e1) *e1 = s.e1;
        if (e2) *e2 = s.e2;
        if (params)
        {
            params[0] = s.eta;
            params[1] = s.rs;
            params[2] = s.lambda;
            params[3] = s.zeta;
            params[4] = s.rc;
            params[5] = s.scalingFactor;
        }
    });
}

n2p2_status n2p2_mode_get_num_derivative_rows(n2p2_mode* mode, int element, int neighborElement, int* rows)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(rows);
    return guard([&] { *rows = (int)mode->model.elements.at(element).table.at(neighborElement).size(); });
}

n2p2_status n2p2_mode_get_network_topology(n2p2_mode* mode, int element, int capacity, int* numLayers, int* neurons,
                                           int* activations)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(numLayers);
    return guard([&] {
        NetworkTopology const& t = mode->model.elements.at(element).topology;
        *numLayers = t.numLayers;
        for (int l = 0; l < t.numLayers && l < capacity; ++l)
        {
            if (neurons) neurons[l] = t.neurons.at(l);
            if (activations) activations[l] = t.activations.at(l);
        }
    });
}

struct n2p2_shuffle_rng
{
    std::mt19937_64 generator;
};

n2p2_status n2p2_shuffle_rng_create(uint64_t seed, n2p2_shuffle_rng** rng)
{
    N2P2_REQUIRE(rng);
    return guard([&] {
        auto r = std::make_unique<n2p2_shuffle_rng>();
        r->generator.seed(seed);
        *rng = r.release();
    });
}

n2p2_status n2p2_shuffle_rng_destroy(n2p2_shuffle_rng* rng)
{
    delete rng;
    return N2P2_OK;
}

n2p2_status n2p2_shuffle_rng_shuffle(n2p2_shuffle_rng* rng, int64_t* values, int64_t count)
{
    N2P2_REQUIRE(rng);
    if (count > 0) N2P2_REQUIRE(values);
    return guard([&] {
        if (count < 0) throw std::invalid_argument("ERROR: negative count.\n");
        std::shuffle(values, values + count, rng->generator);
    });
}

n2p2_status n2p2_batch_create(n2p2_mode* mode, n2p2_batch** batch)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(batch);
    return guard([&] {
        ensureUploaded(mode);
        auto b = std::make_unique<n2p2_batch>();
        b->mode = mode;
        b->batch = std::make_unique<Batch>(mode->model, mode->dmodel, mode->stream, mode->sms);
        *batch = b.release();
    });
}

n2p2_status n2p2_batch_destroy(n2p2_batch* batch)
{
    if (!batch) return N2P2_OK;
    return guard([&] {
        setDevice(batch->mode);
        delete batch;
    });
}

n2p2_status n2p2_batch_set_structures(n2p2_batch* batch, int64_t numStructures, const int64_t* numAtoms,
                                      const int32_t* elements, const double* boxes, const int32_t* periodic,
                                      int remap)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(numAtoms);
    N2P2_REQUIRE(elements);
    return guard([&] {
        setDevice(batch->mode);
        if (!batch->mode->uploaded)
            throw std::runtime_error("ERROR: model changed after the batch was created; create a new batch.\n");
        std::vector<StructureInput> s((size_t)numStructures);
        for (int64_t k = 0; k < numStructures; ++k)
        {
            s[k].numAtoms = (int)numAtoms[k];
            s[k].periodic = periodic ? periodic[k] : (boxes ? 1 : 0);
            if (s[k].periodic)
            {
                if (!boxes) throw std::runtime_error("ERROR: periodic structure without box.\n");
                std::memcpy(s[k].box, boxes + 9 * k, sizeof(double) * 9);
            }
        }
        batch->batch->setStructures(s, elements, remap);
    });
}

n2p2_status n2p2_batch_set_positions(n2p2_batch* batch, const double* positions, int onDevice)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(positions);
    return guard([&] {
        setDevice(batch->mode);
        if (onDevice) batch->batch->setPositionsDevice(positions);
        else batch->batch->setPositionsHost(positions);
    });
}

n2p2_status n2p2_batch_evaluate(n2p2_batch* batch, int flags)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        batch->lastFlags = flags;
        batch->batch->autotuneEnabled = batch->mode->autotune;
        batch->batch->evaluate(flags, batch->mode->precision, batch->mode->checkExtrapolation ? 1 : 0);
        afterEvaluate(batch);
    });
}

n2p2_status n2p2_batch_synchronize(n2p2_batch* batch)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->status();
    });
}

n2p2_status n2p2_batch_calculate_neighbor_list(n2p2_batch* batch)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->calculateNeighborList();
    });
}

n2p2_status n2p2_batch_calculate_symmetry_function_groups(n2p2_batch* batch, int derivatives)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->calculateSymmetryFunctions(derivatives, batch->mode->precision,
                                                 batch->mode->checkExtrapolation ? 1 : 0);
        afterEvaluate(batch);
    });
}

n2p2_status n2p2_batch_calculate_symmetry_functions(n2p2_batch* batch, int derivatives)
{
    return n2p2_batch_calculate_symmetry_function_groups(batch, derivatives);
}

n2p2_status n2p2_batch_calculate_atomic_neural_networks(n2p2_batch* batch, int derivatives)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->calculateAtomicNeuralNetworks(derivatives, batch->mode->precision);
    });
}

n2p2_status n2p2_batch_calculate_energy(n2p2_batch* batch)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->calculateEnergy();
    });
}

n2p2_status n2p2_batch_calculate_forces(n2p2_batch* batch)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->calculateForces();
    });
}

n2p2_status n2p2_batch_get_neighbor_capacity(n2p2_batch* batch, int64_t* capacity, int64_t* recoveries)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->verify();
        if (capacity) *capacity = batch->batch->neighborCapacity();
        if (recoveries) *recoveries = batch->batch->overflowRecoveries();
    });
}

n2p2_status n2p2_batch_get_energies(n2p2_batch* batch, double* energies)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(energies);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->energies(energies);
    });
}

n2p2_status n2p2_batch_get_forces(n2p2_batch* batch, double* forces)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(forces);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->forces(forces);
    });
}

n2p2_status n2p2_batch_evaluate_host(n2p2_batch* batch, const double* positions, double* energies, double* forces,
                                     int flags)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(positions);
    N2P2_REQUIRE(energies);
    return guard([&] {
        setDevice(batch->mode);
        batch->lastFlags = flags;
        batch->batch->setPositionsHost(positions);
        batch->batch->autotuneEnabled = batch->mode->autotune;
        batch->batch->evaluate(flags, batch->mode->precision, batch->mode->checkExtrapolation ? 1 : 0);
        afterEvaluate(batch);
        batch->batch->energies(energies);
        if (forces && (flags & N2P2_EVAL_FORCES)) batch->batch->forces(forces);
    });
}

n2p2_status n2p2_batch_get_num_atoms(n2p2_batch* batch, int64_t* atoms)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(atoms);
    *atoms = batch->batch->numAtoms();
    return N2P2_OK;
}

n2p2_status n2p2_batch_get_num_neighbor_entries(n2p2_batch* batch, int64_t* entries)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(entries);
    return guard([&] {
        setDevice(batch->mode);
        *entries = batch->batch->numNeighborEntries();
    });
}

n2p2_status n2p2_batch_get_neighbors(n2p2_batch* batch, int64_t* offsets, int32_t* index, int32_t* image,
                                     double* d, double* dr)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->synchronize();
        batch->batch->copyNeighbors(offsets, index, image, d, dr);
    });
}

n2p2_status n2p2_batch_get_symmetry_function_statistics(n2p2_batch* batch, int64_t* counts, double* stats)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(counts);
    N2P2_REQUIRE(stats);
    return guard([&] {
        setDevice(batch->mode);
        Batch& b = *batch->batch;
        const int ne = (int)batch->mode->model.numElements();
        const int maxSF = std::max(b.maxSF(), 1);
        std::vector<double> raw((size_t)ne * 4 * maxSF);
        b.sfStatistics(counts, raw.data());
        size_t at = 0;
        for (int e = 0; e < ne; ++e)
        {
            const int nsf = (int)batch->mode->model.elements[e].sf.size();
            for (int q = 0; q < 4; ++q)
                for (int f = 0; f < nsf; ++f) stats[at++] = raw[((size_t)e * 4 + q) * maxSF + f];
        }
    });
}

n2p2_status n2p2_batch_get_symmetry_functions(n2p2_batch* batch, double* G)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(G);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->synchronize();
        batch->batch->copyG(G);
    });
}

n2p2_status n2p2_batch_get_dEdG(n2p2_batch* batch, double* dEdG)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(dEdG);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->synchronize();
        batch->batch->copyDEdG(dEdG);
    });
}

n2p2_status n2p2_batch_get_atomic_energies(n2p2_batch* batch, double* energies)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(energies);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->synchronize();
        batch->batch->copyAtomicEnergies(energies);
    });
}

n2p2_status n2p2_batch_get_dGdr(n2p2_batch* batch, double* selfDGdr, double* neighborDGdr)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->synchronize();
        batch->batch->copyDGdr(selfDGdr, neighborDGdr);
    });
}

n2p2_status n2p2_batch_get_internal_positions(n2p2_batch* batch, double* positions)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(positions);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->synchronize();
        batch->batch->copyPositions(positions);
    });
}

n2p2_status n2p2_batch_get_extrapolation_warnings(n2p2_batch* batch, int64_t* total, int32_t* perAtom)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        DevStatus st = batch->batch->status();
        if (total) *total = st.extrapolationWarnings;
        if (perAtom) batch->batch->copyAtomWarnings(perAtom);
    });
}

n2p2_status n2p2_batch_get_launch_count(n2p2_batch* batch, int* launches)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(launches);
    *launches = batch->batch->launchesPerEvaluate();
    return N2P2_OK;
}

n2p2_status n2p2_neighbor_list_noalloc(const double* positions, int64_t numAtoms, const double* box, double cutoff,
                                       int64_t capacity, int64_t* offsets, int32_t* index, int32_t* image,
                                       double* d, double* dr, int64_t* numEntries, void* stream)
{
    N2P2_REQUIRE(positions);
    N2P2_REQUIRE(offsets);
    N2P2_REQUIRE(index);
    N2P2_REQUIRE(image);
    N2P2_REQUIRE(d);
    N2P2_REQUIRE(dr);
    return guard([&] {
        neighborListNoAlloc(positions, numAtoms, box, cutoff, capacity, offsets, index, image, d, dr, numEntries,
                            static_cast<cudaStream_t>(stream));
    });
}

n2p2_status n2p2_neighbor_list_noalloc_status(int64_t numAtoms, const int64_t* offsets, int64_t capacity,
                                              int64_t* numEntries, void* stream)
{
    N2P2_REQUIRE(offsets);
    return guard([&] {
        neighborListNoAllocStatus(numAtoms, offsets, capacity, numEntries, static_cast<cudaStream_t>(stream));
    });
}

n2p2_status n2p2_batch_get_stream(n2p2_batch* batch, void** stream)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(stream);
    *stream = (void*)batch->batch->stream();
    return N2P2_OK;
}

n2p2_status n2p2_batch_profile_stages(n2p2_batch* batch, int flags, int capacity, char* names, double* ms,
                                      int* count)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(count);
    return guard([&] {
        setDevice(batch->mode);
        auto st = batch->batch->profileStages(flags, batch->mode->precision, batch->mode->checkExtrapolation ? 1 : 0);
        *count = (int)st.size();
        for (int k = 0; k < (int)st.size() && k < capacity; ++k)
        {
            if (names)
            {
                std::memset(names + 32 * k, 0, 32);
                std::strncpy(names + 32 * k, st[k].first.c_str(), 31);
            }
            if (ms) ms[k] = st[k].second;
        }
    });
}

n2p2_status n2p2_batch_count_work(n2p2_batch* batch, int64_t* counts)
{
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(counts);
    return guard([&] {
        setDevice(batch->mode);
        batch->batch->countWork(counts);
    });
}

n2p2_status n2p2_device_fma_peak(int device, double* fp64Tflops, double* fp32Tflops)
{
    return guard([&] {
        cudaCheck(cudaSetDevice(device), "cudaSetDevice");
        cudaDeviceProp p{};
        cudaCheck(cudaGetDeviceProperties(&p, device), "cudaGetDeviceProperties");
        if (fp64Tflops) *fp64Tflops = measureFmaPeak(1, p.multiProcessorCount);
        if (fp32Tflops) *fp32Tflops = measureFmaPeak(0, p.multiProcessorCount);
        cudaCheck(cudaGetLastError(), "fma probe");
    });
}

n2p2_status n2p2_cutoff_function(int device, int type, double rc, double alpha, int precision, const double* r,
                                  int64_t n, double* f, double* df)
{
    N2P2_REQUIRE(r);
    N2P2_REQUIRE(f);
    N2P2_REQUIRE(df);
    return guard([&] {
        cudaCheck(cudaSetDevice(device), "cudaSetDevice");
        cutoffFunctionValues(type, rc, alpha, precision == N2P2_PRECISION_MIXED ? 1 : 0, r, n, f, df);
    });
}

n2p2_status n2p2_mode_set_autotune(n2p2_mode* mode, int32_t enabled)
{
    N2P2_REQUIRE(mode);
    return guard([&] { mode->autotune = enabled != 0; });
}

n2p2_status n2p2_batch_autotune(n2p2_batch* batch, int32_t useCache, int32_t* shapes, double* ms,
                                int32_t* fromCache)
{
    N2P2_REQUIRE(batch);
    return guard([&] {
        setDevice(batch->mode);
        Batch::TuneResult r = batch->batch->autotune(batch->mode->precision, batch->mode->checkExtrapolation ? 1 : 0,
                                                     useCache != 0);
        if (shapes)
        {
            shapes[0] = r.values;
            shapes[1] = r.forces;
        }
        if (ms)
            for (int v = 0; v < kSFShapeCount; ++v)
            {
                ms[v] = r.valuesMs[v];
                ms[kSFShapeCount + v] = r.forcesMs[v];
            }
        if (fromCache) *fromCache = r.fromCache ? 1 : 0;
    });
}

n2p2_status n2p2_batch_set_shapes(n2p2_batch* batch, int32_t valuesShape, int32_t forcesShape)
{
    N2P2_REQUIRE(batch);
    return guard([&] { batch->batch->setShapes(batch->mode->precision, valuesShape, forcesShape); });
}

n2p2_status n2p2_trainer_create(n2p2_mode* mode, n2p2_trainer** trainer)
{
    N2P2_REQUIRE(mode);
    N2P2_REQUIRE(trainer);
    return guard([&] {
        ensureUploaded(mode);
        auto t = std::make_unique<n2p2_trainer>();
        t->mode = mode;
        t->trainer = std::make_unique<Trainer>(mode->model, mode->dmodel, mode->sms);
        *trainer = t.release();
    });
}

n2p2_status n2p2_trainer_destroy(n2p2_trainer* trainer)
{
    if (!trainer) return N2P2_OK;
    return guard([&] {
        setDevice(trainer->mode);
        delete trainer;
    });
}

n2p2_status n2p2_trainer_set_adam(n2p2_trainer* trainer, double eta, double beta1, double beta2, double epsilon)
{
    N2P2_REQUIRE(trainer);
    return guard([&] {
        if (!(eta > 0.0) || !(beta1 >= 0.0 && beta1 < 1.0) || !(beta2 >= 0.0 && beta2 < 1.0) || !(epsilon > 0.0))
            throw std::invalid_argument("ERROR: invalid Adam parameters.\n");
        trainer->trainer->setAdam(eta, beta1, beta2, epsilon);
    });
}

n2p2_status n2p2_trainer_set_learning_rate(n2p2_trainer* trainer, double eta)
{
    N2P2_REQUIRE(trainer);
    return guard([&] {
        if (!(eta > 0.0)) throw std::invalid_argument("ERROR: the learning rate must be positive.\n");
        trainer->trainer->setLearningRate(eta);
    });
}

n2p2_status n2p2_trainer_set_loss_weights(n2p2_trainer* trainer, double energyWeight, double forceWeight)
{
    N2P2_REQUIRE(trainer);
    return guard([&] {
        if (!(energyWeight >= 0.0) || !(forceWeight >= 0.0))
            throw std::invalid_argument("ERROR: loss weights must be non-negative.\n");
        trainer->trainer->setLossWeights(energyWeight, forceWeight);
    });
}

n2p2_status n2p2_trainer_get_num_parameters(n2p2_trainer* trainer, int64_t* count)
{
    N2P2_REQUIRE(trainer);
    N2P2_REQUIRE(count);
    return guard([&] { *count = trainer->trainer->numParameters(); });
}

n2p2_status n2p2_trainer_get_parameters(n2p2_trainer* trainer, double* parameters)
{
    N2P2_REQUIRE(trainer);
    N2P2_REQUIRE(parameters);
    return guard([&] {
        setDevice(trainer->mode);
        trainer->trainer->getParameters(parameters, trainer->mode->stream);
    });
}

n2p2_status n2p2_trainer_set_parameters(n2p2_trainer* trainer, const double* parameters)
{
    N2P2_REQUIRE(trainer);
    N2P2_REQUIRE(parameters);
    return guard([&] {
        setDevice(trainer->mode);
        if (!trainer->mode->uploaded) throw std::runtime_error("ERROR: the mode was changed after the trainer was created.\n");
        trainer->trainer->setParameters(parameters, trainer->mode->stream);
        trainer->trainer->syncHostModel(trainer->mode->stream);
    });
}

n2p2_status n2p2_trainer_step(n2p2_trainer* trainer, n2p2_batch* batch, const double* energies,
                              const double* forces, int32_t update, double* loss, double* gradient)
{
    N2P2_REQUIRE(trainer);
    N2P2_REQUIRE(batch);
    N2P2_REQUIRE(energies);
    N2P2_REQUIRE(forces);
    return guard([&] {
        setDevice(trainer->mode);
        if (batch->mode != trainer->mode) throw std::invalid_argument("ERROR: batch belongs to another mode.\n");
        if (!trainer->mode->uploaded) throw std::runtime_error("ERROR: the mode was changed after the trainer was created.\n");
        trainer->trainer->step(*batch->batch, energies, forces, update != 0, loss, gradient);
        if (update) trainer->trainer->syncHostModel(trainer->mode->stream);
    });
}

n2p2_status n2p2_training_create(n2p2_batch* set, n2p2_training** training)
{
    N2P2_REQUIRE(set);
    N2P2_REQUIRE(training);
    return guard([&] {
        setDevice(set->mode);
        ensureUploaded(set->mode);
        auto t = std::make_unique<n2p2_training>();
        t->mode = set->mode;
        t->set = set;
        t->training = std::make_unique<Training>(set->mode->model, set->mode->dmodel, *set->batch, set->mode->sms);
        *training = t.release();
    });
}

n2p2_status n2p2_training_destroy(n2p2_training* training)
{
    if (!training) return N2P2_OK;
    return guard([&] {
        setDevice(training->mode);
        delete training;
    });
}

n2p2_status n2p2_training_set_references(n2p2_training* training, const double* energies, const double* forces)
{
    N2P2_REQUIRE(training);
    N2P2_REQUIRE(energies);
    N2P2_REQUIRE(forces);
    return guard([&] {
        setDevice(training->mode);
        training->training->setReferences(energies, forces);
    });
}

n2p2_status n2p2_training_set_force_weight(n2p2_training* training, double weight)
{
    N2P2_REQUIRE(training);
    return guard([&] {
        if (!(weight >= 0.0)) throw std::invalid_argument("ERROR: the force weight must be non-negative.\n");
        training->training->setForceWeight(weight);
    });
}

n2p2_status n2p2_training_set_update_strategy(n2p2_training* training, int32_t strategy)
{
    N2P2_REQUIRE(training);
    return guard([&] { training->training->setUpdateStrategy(strategy); });
}

n2p2_status n2p2_training_set_jacobian_mode(n2p2_training* training, int32_t mode)
{
    N2P2_REQUIRE(training);
    return guard([&] {
        if (mode < 0 || mode > 2) throw std::invalid_argument("ERROR: unknown Jacobian mode.\n");
        training->training->setFullJacobian(mode == 2);
    });
}

n2p2_status n2p2_training_set_task_batch_size(n2p2_training* training, int32_t energy, int32_t force)
{
    N2P2_REQUIRE(training);
    return guard([&] {
        if (energy < 1 || force < 1) throw std::invalid_argument("ERROR: task batch sizes must be positive.\n");
        training->training->setTaskBatchSize(energy, force);
    });
}

n2p2_status n2p2_training_set_kalman_standard(n2p2_training* training, double epsilon, double q0, double qtau,
                                              double qmin, double eta0, double etatau, double etamax)
{
    N2P2_REQUIRE(training);
    return guard([&] {
        if (!(epsilon > 0.0) || !(eta0 > 0.0)) throw std::invalid_argument("ERROR: invalid Kalman filter parameters.\n");
        setDevice(training->mode);
        training->training->setKalmanStandard(epsilon, q0, qtau, qmin, eta0, etatau, etamax);
    });
}

n2p2_status n2p2_training_set_kalman_fading_memory(n2p2_training* training, double epsilon, double q0, double qtau,
                                                   double qmin, double lambda, double nu)
{
    N2P2_REQUIRE(training);
    return guard([&] {
        if (!(epsilon > 0.0) || !(lambda > 0.0)) throw std::invalid_argument("ERROR: invalid Kalman filter parameters.\n");
        setDevice(training->mode);
        training->training->setKalmanFadingMemory(epsilon, q0, qtau, qmin, lambda, nu);
    });
}

n2p2_status n2p2_training_set_gradient_fixed(n2p2_training* training, double eta)
{
    N2P2_REQUIRE(training);
    return guard([&] {
        if (!(eta > 0.0)) throw std::invalid_argument("ERROR: the step size must be positive.\n");
        training->training->setGradientFixed(eta);
    });
}

n2p2_status n2p2_training_set_gradient_adam(n2p2_training* training, double eta, double beta1, double beta2,
                                            double epsilon)
{
    N2P2_REQUIRE(training);
    return guard([&] {
        if (!(eta > 0.0) || !(beta1 >= 0.0 && beta1 < 1.0) || !(beta2 >= 0.0 && beta2 < 1.0) || !(epsilon > 0.0))
            throw std::invalid_argument("ERROR: invalid Adam parameters.\n");
        setDevice(training->mode);
        training->training->setGradientAdam(eta, beta1, beta2, epsilon);
    });
}

n2p2_status n2p2_training_update(n2p2_training* training, int32_t property, int32_t count, const int32_t* structure,
                                 const int32_t* atom, const int32_t* component, double* errors)
{
    N2P2_REQUIRE(training);
    N2P2_REQUIRE(count >= 0);
    N2P2_REQUIRE(count == 0 || structure);
    N2P2_REQUIRE(property != N2P2_TRAINING_FORCE || count == 0 || (atom && component));
    return guard([&] {
        setDevice(training->mode);
        if (!training->mode->uploaded)
            throw std::runtime_error("ERROR: the mode was changed after the training was created.\n");
        training->training->update(property, count, structure, atom, component, errors);
    });
}

n2p2_status n2p2_training_observe(n2p2_training* training, int32_t property, int32_t structure, int32_t atom,
                                  int32_t component, double* error, double* jacobian)
{
    N2P2_REQUIRE(training);
    N2P2_REQUIRE(error);
    N2P2_REQUIRE(jacobian);
    return guard([&] {
        setDevice(training->mode);
        training->training->observe(property, structure, atom, component, error, jacobian);
    });
}

n2p2_status n2p2_training_update_threshold(n2p2_training* training, int32_t property, int32_t num_updates,
                                           int32_t num_candidates, const int32_t* structure, const int32_t* atom,
                                           const int32_t* component, double threshold, int32_t trials, double rmse,
                                           int32_t* consumed, double* errors)
{
    N2P2_REQUIRE(training);
    N2P2_REQUIRE(structure);
    N2P2_REQUIRE(num_updates >= 0);
    N2P2_REQUIRE(property != N2P2_TRAINING_FORCE || (atom && component));
    return guard([&] {
        setDevice(training->mode);
        if (!(rmse > 0.0)) throw std::invalid_argument("ERROR: the training RMSE must be positive.\n");
        const int n = training->training->updateThreshold(property, num_updates, num_candidates, structure, atom,
                                                          component, threshold, trials, rmse, errors);
        if (consumed) *consumed = n;
    });
}

n2p2_status n2p2_training_get_errors(n2p2_training* training, double* errors)
{
    N2P2_REQUIRE(training);
    N2P2_REQUIRE(errors);
    return guard([&] {
        setDevice(training->mode);
        training->training->trainingErrors(errors, errors + 1);
    });
}

n2p2_status n2p2_training_get_kalman_status(n2p2_training* training, double* status)
{
    N2P2_REQUIRE(training);
    N2P2_REQUIRE(status);
    return guard([&] {
        setDevice(training->mode);
        training->training->kalmanStatus(status);
    });
}

n2p2_status n2p2_training_get_num_weights(n2p2_training* training, int64_t* count)
{
    N2P2_REQUIRE(training);
    N2P2_REQUIRE(count);
    return guard([&] { *count = training->training->numWeights(); });
}

n2p2_status n2p2_training_get_weights(n2p2_training* training, double* weights)
{
    N2P2_REQUIRE(training);
    N2P2_REQUIRE(weights);
    return guard([&] {
        setDevice(training->mode);
        training->training->getWeights(weights);
    });
}

n2p2_status n2p2_training_set_weights(n2p2_training* training, const double* weights)
{
    N2P2_REQUIRE(training);
    N2P2_REQUIRE(weights);
    return guard([&] {
        setDevice(training->mode);
        training->training->setWeights(weights);
    });
}

n2p2_status n2p2_host_alloc(void** ptr, size_t bytes)
{
    N2P2_REQUIRE(ptr);
    return guard([&] { cudaCheck(cudaHostAlloc(ptr, bytes, cudaHostAllocDefault), "cudaHostAlloc"); });
}

n2p2_status n2p2_host_free(void* ptr)
{
    if (!ptr) return N2P2_OK;
    return guard([&] { cudaCheck(cudaFreeHost(ptr), "cudaFreeHost"); });
}

n2p2_status n2p2_lammps_create(n2p2_lammps** lammps, int device)
{
    N2P2_REQUIRE(lammps);
    return guard([&] {
        auto l = std::make_unique<n2p2_lammps>();
        l->mode.device = device;
        *lammps = l.release();
    });
}

n2p2_status n2p2_lammps_destroy(n2p2_lammps* lammps)
{
    if (!lammps) return N2P2_OK;
    return guard([&] {
        cudaStream_t s = lammps->mode.stream;
        if (s) cudaSetDevice(lammps->mode.device);
        lammps->batch.reset();
        delete lammps;
        if (s) cudaStreamDestroy(s);
    });
}

n2p2_status n2p2_lammps_initialize(n2p2_lammps* lammps, const char* directory, const char* emap, int32_t showew,
                                   int32_t resetew, int32_t showewsum, int32_t maxew, double cflength,
                                   double cfenergy, double lammpsCutoff, int32_t lammpsNtypes, int32_t myRank)
{
    N2P2_REQUIRE(lammps);
    N2P2_REQUIRE(directory);
    (void)resetew;
    return guard([&] {
        if (lammps->iface.isInitialized() || lammps->mode.model.setupDone)
            throw std::runtime_error("ERROR: the LAMMPS interface is already initialized.\n");
        std::string dir(directory);
        if (dir.empty() || dir.back() != '/') dir += '/';
        n2p2_mode& m = lammps->mode;
        m.model.loadSettingsFile(dir + "input.nn");
        m.model.setupGeneric();
        m.model.setupSymmetryFunctionScaling(dir + "scaling.data");
        m.checkExtrapolation = showew || showewsum > 0 || maxew >= 0;
        m.model.setupNeuralNetworkWeights(dir + "weights.%03zu.data");
        m.uploaded = false;
        lammps->iface.initialize(m.model, emap ? emap : "", cflength, cfenergy, lammpsCutoff, lammpsNtypes, myRank);
    });
}

n2p2_status n2p2_lammps_set_precision(n2p2_lammps* lammps, int precision)
{
    N2P2_REQUIRE(lammps);
    return n2p2_mode_set_precision(&lammps->mode, precision);
}

n2p2_status n2p2_lammps_get_max_cutoff_radius(n2p2_lammps* lammps, double* radius)
{
    N2P2_REQUIRE(lammps);
    N2P2_REQUIRE(radius);
    return guard([&] {
        if (!lammps->iface.isInitialized()) throw std::runtime_error("ERROR: the LAMMPS interface is not initialized.\n");
        *radius = lammps->iface.maxCutoffRadius();
    });
}

n2p2_status n2p2_lammps_set_local_atoms(n2p2_lammps* lammps, int32_t numAtomsLocal, const int32_t* atomType)
{
    N2P2_REQUIRE(lammps);
    if (numAtomsLocal > 0) N2P2_REQUIRE(atomType);
    return guard([&] { lammps->iface.setLocalAtoms(numAtomsLocal, atomType); });
}

n2p2_status n2p2_lammps_add_neighbor(n2p2_lammps* lammps, int32_t i, int32_t j, int64_t tag, int32_t type,
                                     double dx, double dy, double dz, double d2)
{
    N2P2_REQUIRE(lammps);
    (void)tag;
    return guard([&] { lammps->iface.addNeighbor(i, j, type, dx, dy, dz, d2); });
}

n2p2_status n2p2_lammps_transfer_neighbor_list(n2p2_lammps* lammps, int32_t inum, const int32_t* ilist,
                                               const int32_t* numneigh, const int32_t* const* firstneigh,
                                               const double* const* x, const int32_t* type, double maxCutoffRadius)
{
    N2P2_REQUIRE(lammps);
    if (inum > 0)
    {
        N2P2_REQUIRE(ilist);
        N2P2_REQUIRE(numneigh);
        N2P2_REQUIRE(firstneigh);
        N2P2_REQUIRE(x);
        N2P2_REQUIRE(type);
    }
    return guard([&] {
        setDevice(&lammps->mode);   // the staging is page-locked host memory
        lammps->iface.transferNeighborList(inum, ilist, numneigh, firstneigh, x, type, maxCutoffRadius);
    });
}

n2p2_status n2p2_lammps_process(n2p2_lammps* lammps)
{
    N2P2_REQUIRE(lammps);
    return guard([&] {
        n2p2_mode& m = lammps->mode;
        ensureUploaded(&m);
        if (!lammps->batch) lammps->batch = std::make_unique<Batch>(m.model, m.dmodel, m.stream, m.sms);
        lammps->batch->autotuneEnabled = m.autotune;
        lammps->iface.process(*lammps->batch, m.precision, m.checkExtrapolation);
        if (m.checkExtrapolation && lammps->iface.numCenters() > 0)
            lammps->warnings += lammps->batch->status().extrapolationWarnings;
    });
}

n2p2_status n2p2_lammps_get_energy(n2p2_lammps* lammps, double* energy)
{
    N2P2_REQUIRE(lammps);
    N2P2_REQUIRE(energy);
    *energy = lammps->iface.energy();
    return N2P2_OK;
}

n2p2_status n2p2_lammps_get_atomic_energy(n2p2_lammps* lammps, int32_t index, double* energy)
{
    N2P2_REQUIRE(lammps);
    N2P2_REQUIRE(energy);
    return guard([&] {
        if (!lammps->batch) throw std::runtime_error("ERROR: process() has not run.\n");
        setDevice(&lammps->mode);
        *energy = lammps->iface.atomicEnergy(*lammps->batch, index);
    });
}

n2p2_status n2p2_lammps_get_forces(n2p2_lammps* lammps, double* const* atomF)
{
    N2P2_REQUIRE(lammps);
    N2P2_REQUIRE(atomF);
    return guard([&] {
        if (!lammps->batch) throw std::runtime_error("ERROR: process() has not run.\n");
        setDevice(&lammps->mode);
        lammps->iface.addForces(*lammps->batch, atomF);
    });
}

n2p2_status n2p2_lammps_get_num_extrapolation_warnings(n2p2_lammps* lammps, int64_t* count)
{
    N2P2_REQUIRE(lammps);
    N2P2_REQUIRE(count);
    *count = lammps->warnings;
    return N2P2_OK;
}

n2p2_status n2p2_lammps_clear_extrapolation_warnings(n2p2_lammps* lammps)
{
    N2P2_REQUIRE(lammps);
    lammps->warnings = 0;
    return N2P2_OK;
}

n2p2_status n2p2_structures_read_file(const char* fileName, int64_t limit, n2p2_structures** structures)
{
    N2P2_REQUIRE(fileName);
    N2P2_REQUIRE(structures);
    return guard([&] {
        auto s = std::make_unique<n2p2_structures>();
        readStructuresFile(fileName, limit, s->set);
        *structures = s.release();
    });
}

n2p2_status n2p2_structures_read_text(const char* text, int64_t length, int64_t limit,
                                      n2p2_structures** structures)
{
    N2P2_REQUIRE(text);
    N2P2_REQUIRE(structures);
    return guard([&] {
        auto s = std::make_unique<n2p2_structures>();
        const std::string copy(text, (size_t)length);   // NUL-terminated for strtod
        readStructures(copy.c_str(), copy.size(), limit, s->set);
        *structures = s.release();
    });
}

n2p2_status n2p2_structures_destroy(n2p2_structures* structures)
{
    delete structures;
    return N2P2_OK;
}

n2p2_status n2p2_structures_get_count(n2p2_structures* structures, int64_t* numStructures, int64_t* numAtoms)
{
    N2P2_REQUIRE(structures);
    if (numStructures) *numStructures = structures->set.numStructures();
    if (numAtoms) *numAtoms = structures->set.numAtoms();
    return N2P2_OK;
}

n2p2_status n2p2_structures_get_structure_arrays(n2p2_structures* structures, int64_t* numAtoms, double* boxes,
                                                 int32_t* periodic, double* energies, double* charges)
{
    N2P2_REQUIRE(structures);
    StructureSet const& t = structures->set;
    const size_t S = (size_t)t.numStructures();
    for (size_t k = 0; k < S; ++k)
        if (numAtoms) numAtoms[k] = t.atomBegin[k + 1] - t.atomBegin[k];
    if (boxes && S) std::memcpy(boxes, t.boxes.data(), sizeof(double) * 9 * S);
    if (periodic && S) std::memcpy(periodic, t.periodic.data(), sizeof(int32_t) * S);
    if (energies && S) std::memcpy(energies, t.energies.data(), sizeof(double) * S);
    if (charges && S) std::memcpy(charges, t.charges.data(), sizeof(double) * S);
    return N2P2_OK;
}

n2p2_status n2p2_structures_get_atom_arrays(n2p2_structures* structures, double* positions, char* elements,
                                            double* charges, double* forces)
{
    N2P2_REQUIRE(structures);
    return guard([&] {
        StructureSet const& t = structures->set;
        const size_t N = (size_t)t.numAtoms();
        if (positions && N) std::memcpy(positions, t.positions.data(), sizeof(double) * 3 * N);
        if (forces && N) std::memcpy(forces, t.forces.data(), sizeof(double) * 3 * N);
        if (charges && N) std::memcpy(charges, t.atomCharges.data(), sizeof(double) * N);
        if (elements)
            for (size_t a = 0; a < N; ++a)
            {
                std::string const& e = t.elements[a];
                if (e.size() > 3) throw std::runtime_error("ERROR: element symbol longer than 3 characters.\n");
                std::memset(elements + 4 * a, 0, 4);
                std::memcpy(elements + 4 * a, e.data(), e.size());
            }
    });
}

n2p2_status n2p2_structures_get_comment(n2p2_structures* structures, int64_t index, char* buffer,
                                        int32_t capacity)
{
    N2P2_REQUIRE(structures);
    N2P2_REQUIRE(buffer);
    return guard([&] {
        std::string const& c = structures->set.comments.at((size_t)index);
        if ((int64_t)c.size() + 1 > capacity) throw std::runtime_error("buffer too small");
        std::memcpy(buffer, c.c_str(), c.size() + 1);
    });
}

} // extern "C"
