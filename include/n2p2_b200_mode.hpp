/*
 * n2p2_b200_mode.hpp -- header-only C++ facade of nnp::Mode, nnp::Structure
 * and nnp::Atom over the C ABI of n2p2_b200.h (link with -ln2p2b200).
 *
 * For C++ callers of the reference's evaluation path (nnp-predict's
 * Prediction, a training or analysis program) that want to keep their code:
 * the class and member names, argument meanings and exception types are the
 * reference's (src/libnnp/Mode.h:87-699, Structure.h, Atom.h); the work runs
 * on the GPU.  What differs, and why:
 *
 *  - Structure and Atom carry the public fields callers read (atoms[].r,
 *    .element, .energy, .f, .G, .dEdG, .dGdr, .neighbors[] with index, d,
 *    dr, dGdr; Structure::energy, box, numAtoms, the has* flags).  Each
 *    Structure is mirrored on the device by one batch the Mode creates at the
 *    first call; positions are uploaded again when atoms[].r changed.
 *  - Structure::calculateNeighborList(cutoffRadius) only marks the list as
 *    wanted: the device builds it at the model's largest cutoff at the next
 *    Mode call (the same entries; a smaller radius would drop neighbours that
 *    symmetry functions use and is rejected with std::invalid_argument).
 *    Atom::neighbors is filled from the device list.  Changed positions
 *    clear the structure's result flags (the reference keeps them until
 *    Structure::reset and would reuse the old symmetry functions).
 *  - Structure::energy and Atom::f are in the units of the input (the values
 *    Prediction::predict leaves after Structure::toPhysicalUnits and
 *    Mode::addEnergyOffset, Prediction.cpp:67-78); G, dE/dG and dG/dr are in
 *    the model's internal units, as in the reference.
 *  - Derivatives of symmetry functions are contracted with dE/dG on the GPU
 *    (calculateForces) without storing dG/dr; setStoreDerivatives(true) keeps
 *    them (FP64 form, Gaussian function types) and fills Atom::dGdr and
 *    Atom::Neighbor::dGdr as the reference does.
 *
 * The C ABI never throws; this header turns its status codes back into
 * std::runtime_error, std::range_error, std::out_of_range and
 * std::invalid_argument, the reference's exception types.
 */
#ifndef N2P2_B200_MODE_HPP
#define N2P2_B200_MODE_HPP

#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "n2p2_b200.h"

namespace n2p2b200 {
namespace nnp {

inline void check(n2p2_status s)
{
    if (s == N2P2_OK) return;
    std::string m = n2p2_last_error();
    switch (s)
    {
    case N2P2_ERR_RANGE: throw std::range_error(m);
    case N2P2_ERR_OUT_OF_RANGE: throw std::out_of_range(m);
    case N2P2_ERR_INVALID_ARGUMENT: throw std::invalid_argument(m);
    default: throw std::runtime_error(m);
    }
}

/* nnp::Vec3D (Vec3D.h): three doubles. */
struct Vec3D
{
    double r[3] = {0.0, 0.0, 0.0};
    double& operator[](std::size_t i) { return r[i]; }
    double const& operator[](std::size_t i) const { return r[i]; }
};

/* nnp::Atom (Atom.h:30-480), the fields the evaluation path fills. */
struct Atom
{
    struct Neighbor   // Atom::Neighbor (Atom.h:35-88)
    {
        std::size_t index = 0;
        std::size_t element = 0;
        double d = 0.0;
        Vec3D dr;
        std::vector<Vec3D> dGdr;
    };
    std::size_t index = 0;
    std::size_t indexStructure = 0;
    std::size_t element = 0;
    std::size_t numNeighbors = 0;
    std::size_t numSymmetryFunctions = 0;
    double energy = 0.0;
    Vec3D r;
    Vec3D f;
    std::vector<double> G;
    std::vector<double> dEdG;
    std::vector<Vec3D> dGdr;
    std::vector<Neighbor> neighbors;
    bool hasNeighborList = false;
    bool hasSymmetryFunctions = false;
    bool hasSymmetryFunctionDerivatives = false;
};

class Mode;

/* nnp::Structure (Structure.h:37-600), the fields and calls of the
 * evaluation path. */
struct Structure
{
    std::size_t index = 0;
    std::size_t numAtoms = 0;
    bool isPeriodic = false;
    bool hasNeighborList = false;
    bool hasSymmetryFunctions = false;
    bool hasSymmetryFunctionDerivatives = false;
    double energy = 0.0;
    double energyRef = 0.0;
    Vec3D box[3];
    std::string comment;
    std::vector<std::string> elementSymbols;   // per atom, as read
    std::vector<Atom> atoms;

    /* Structure::readFromFile (Structure.cpp:117-140) for the structure at
     * position `index` (0 = first) of an input.data file. */
    void readFromFile(std::string const& fileName = "input.data", std::size_t index = 0)
    {
        n2p2_structures* h = nullptr;
        check(n2p2_structures_read_file(fileName.c_str(), (int64_t)index + 1, &h));
        std::unique_ptr<n2p2_structures, n2p2_status (*)(n2p2_structures*)> guard(h, n2p2_structures_destroy);
        int64_t S = 0, N = 0;
        check(n2p2_structures_get_count(h, &S, &N));
        if ((int64_t)index >= S) throw std::runtime_error("ERROR: structure index beyond the end of the file.\n");
        std::vector<int64_t> na((size_t)S);
        std::vector<double> boxes(9 * (size_t)S), E((size_t)S);
        std::vector<int32_t> per((size_t)S);
        check(n2p2_structures_get_structure_arrays(h, na.data(), boxes.data(), per.data(), E.data(), nullptr));
        std::vector<double> pos(3 * (size_t)N);
        std::vector<char> sym(4 * (size_t)N);
        check(n2p2_structures_get_atom_arrays(h, pos.data(), sym.data(), nullptr, nullptr));
        std::vector<char> text(1 << 16);
        check(n2p2_structures_get_comment(h, (int64_t)index, text.data(), (int32_t)text.size()));
        int64_t a0 = 0;
        for (size_t k = 0; k < index; ++k) a0 += na[k];
        this->index = index;
        comment = text.data();
        numAtoms = (size_t)na[index];
        isPeriodic = per[index] != 0;
        energyRef = E[index];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) box[i][j] = boxes[9 * index + 3 * i + j];
        atoms.assign(numAtoms, Atom{});
        elementSymbols.assign(numAtoms, std::string());
        device_.reset();
        for (size_t a = 0; a < numAtoms; ++a)
        {
            atoms[a].index = a;
            atoms[a].indexStructure = index;
            for (int c = 0; c < 3; ++c) atoms[a].r[c] = pos[3 * (a0 + a) + c];
            elementSymbols[a] = std::string(&sym[4 * (a0 + a)], strnlen(&sym[4 * (a0 + a)], 4));
        }
        reset();
    }

    /* Structure::calculateNeighborList(cutoffRadius, sortByDistance)
     * (Structure.cpp:287-398): marks the list as wanted; the next Mode call
     * builds it on the device. */
    void calculateNeighborList(double cutoffRadius, bool sortByDistance = false)
    {
        if (sortByDistance)
            throw std::invalid_argument("ERROR: distance-sorted neighbour lists are a 4G feature.\n");
        listCutoff_ = cutoffRadius;
        hasNeighborList = true;
    }

    /* Structure::reset (Structure.cpp:1170-1210) as far as the evaluation
     * path is concerned: every result flag cleared. */
    void reset()
    {
        hasNeighborList = hasSymmetryFunctions = hasSymmetryFunctionDerivatives = false;
        listStale_ = true;
        for (auto& a : atoms) a.hasNeighborList = a.hasSymmetryFunctions = a.hasSymmetryFunctionDerivatives = false;
    }

private:
    friend class Mode;
    struct Device
    {
        n2p2_batch* batch = nullptr;
        void const* owner = nullptr;   // the Mode that created the batch
        std::size_t numAtoms = 0;
        std::vector<double> uploaded;
        ~Device()
        {
            if (batch) n2p2_batch_destroy(batch);
        }
    };
    std::shared_ptr<Device> device_;
    double listCutoff_ = 0.0;
    bool listStale_ = true;
};

/* nnp::Mode (Mode.h:87-699): set-up and the evaluation stages. */
class Mode
{
public:
    explicit Mode(int device = 0) { check(n2p2_mode_create(&mode_, device)); }
    ~Mode()
    {
        // the structures' device batches belong to this mode: release them first
        for (auto& w : devices_)
            if (auto d = w.lock())
                if (d->batch)
                {
                    n2p2_batch_destroy(d->batch);
                    d->batch = nullptr;
                    d->uploaded.clear();
                }
        if (mode_) n2p2_mode_destroy(mode_);
    }
    Mode(Mode const&) = delete;
    Mode& operator=(Mode const&) = delete;

    // -- set-up (Mode.cpp:56-1547) ------------------------------------------
    void initialize() { check(n2p2_mode_initialize(mode_)); }
    void loadSettingsFile(std::string const& fileName = "input.nn")
    {
        check(n2p2_mode_load_settings_file(mode_, fileName.c_str()));
    }
    void setupGeneric(std::string const& /*nnpDir*/ = "", bool /*skipNormalize*/ = false,
                      bool /*initialHardness*/ = false)
    {
        check(n2p2_mode_setup_generic(mode_));
    }
    void setupSymmetryFunctionScaling(std::string const& fileName = "scaling.data")
    {
        check(n2p2_mode_setup_symmetry_function_scaling(mode_, fileName.c_str()));
    }
    void setupSymmetryFunctionScalingNone() { check(n2p2_mode_setup_symmetry_function_scaling_none(mode_)); }
    void setupNeuralNetworkWeights(std::string const& fileNameFormat = "weights.%03zu.data")
    {
        check(n2p2_mode_setup_neural_network_weights(mode_, fileNameFormat.c_str()));
    }
    void setupSymmetryFunctionStatistics(bool collectStatistics, bool collectExtrapolationWarnings,
                                         bool writeExtrapolationWarnings, bool stopOnExtrapolationWarnings)
    {
        check(n2p2_mode_setup_symmetry_function_statistics(mode_, collectStatistics, collectExtrapolationWarnings,
                                                           writeExtrapolationWarnings,
                                                           stopOnExtrapolationWarnings));
    }
    double getMaxCutoffRadius() const
    {
        double r = 0.0;
        check(n2p2_mode_get_max_cutoff_radius(mode_, &r));
        return r;
    }
    std::size_t getNumExtrapolationWarnings() const { return numExtrapolationWarnings_; }
    void resetExtrapolationWarnings() { numExtrapolationWarnings_ = 0; }
    // Extra over the reference: N2P2_PRECISION_FP64 (default) or _MIXED, and
    // whether derivatives of symmetry functions are stored (see the file comment).
    void setPrecision(int precision) { check(n2p2_mode_set_precision(mode_, precision)); }
    void setStoreDerivatives(bool store) { storeDerivatives_ = store; }

    // -- evaluation stages (Mode.h:298-387) -----------------------------------
    void calculateSymmetryFunctions(Structure& structure, bool const derivatives)
    {
        calculateSymmetryFunctionGroups(structure, derivatives);
    }
    void calculateSymmetryFunctionGroups(Structure& structure, bool const derivatives)
    {
        n2p2_batch* b = bind(structure);
        // Mode.cpp:1634-1635
        if (structure.hasSymmetryFunctionDerivatives) return;
        if (structure.hasSymmetryFunctions && !derivatives) return;
        const int d = derivatives ? (storeDerivatives_ ? N2P2_DERIVATIVES_STORED : N2P2_DERIVATIVES)
                                  : N2P2_DERIVATIVES_NONE;
        check(n2p2_batch_calculate_symmetry_function_groups(b, d));
        int64_t warnings = 0;
        check(n2p2_batch_get_extrapolation_warnings(b, &warnings, nullptr));
        numExtrapolationWarnings_ += (std::size_t)warnings;
        std::vector<double> G(sfTotal(structure));
        check(n2p2_batch_get_symmetry_functions(b, G.data()));
        size_t at = 0;
        for (auto& a : structure.atoms)
        {
            a.numSymmetryFunctions = (size_t)numSF_[a.element];
            a.G.assign(G.begin() + at, G.begin() + at + a.numSymmetryFunctions);
            at += a.numSymmetryFunctions;
            a.hasSymmetryFunctions = true;
            a.hasSymmetryFunctionDerivatives = derivatives;
        }
        if (derivatives && storeDerivatives_) fillDerivatives(structure, b);
        structure.hasSymmetryFunctions = true;
        if (derivatives) structure.hasSymmetryFunctionDerivatives = true;
    }
    void calculateAtomicNeuralNetworks(Structure& structure, bool const derivatives, std::string id = "")
    {
        if (!id.empty() && id != "short")
            throw std::runtime_error("ERROR: only the short-range network exists in a 2G model.\n");
        n2p2_batch* b = bind(structure);
        check(n2p2_batch_calculate_atomic_neural_networks(b, derivatives ? 1 : 0));
        std::vector<double> e(structure.numAtoms);
        check(n2p2_batch_get_atomic_energies(b, e.data()));
        std::vector<double> dEdG;
        if (derivatives)
        {
            dEdG.resize(sfTotal(structure));
            check(n2p2_batch_get_dEdG(b, dEdG.data()));
        }
        size_t at = 0;
        for (size_t i = 0; i < structure.numAtoms; ++i)
        {
            Atom& a = structure.atoms[i];
            a.energy = e[i];
            const size_t n = (size_t)numSF_[a.element];
            if (derivatives) a.dEdG.assign(dEdG.begin() + at, dEdG.begin() + at + n);
            at += n;
        }
    }
    void calculateEnergy(Structure& structure) const
    {
        n2p2_batch* b = boundBatch(structure);
        check(n2p2_batch_calculate_energy(b));
        check(n2p2_batch_get_energies(b, &structure.energy));
    }
    void calculateForces(Structure& structure) const
    {
        n2p2_batch* b = boundBatch(structure);
        check(n2p2_batch_calculate_forces(b));
        std::vector<double> f(3 * structure.numAtoms);
        check(n2p2_batch_get_forces(b, f.data()));
        for (size_t i = 0; i < structure.numAtoms; ++i)
            for (int c = 0; c < 3; ++c) structure.atoms[i].f[c] = f[3 * i + c];
    }
    /* Mode::evaluateNNP (Mode.cpp:2029-2077). */
    void evaluateNNP(Structure& structure, bool useForces = true, bool useDEdG = true)
    {
        useDEdG = useForces || useDEdG;
        structure.calculateNeighborList(getMaxCutoffRadius(), false);
        calculateSymmetryFunctionGroups(structure, useForces);
        calculateAtomicNeuralNetworks(structure, useDEdG);
        calculateEnergy(structure);
        if (useForces) calculateForces(structure);
    }

    n2p2_mode* handle() const { return mode_; }

private:
    n2p2_mode* mode_ = nullptr;
    std::vector<std::weak_ptr<Structure::Device>> devices_;
    std::vector<int> numSF_;
    std::size_t numExtrapolationWarnings_ = 0;
    bool storeDerivatives_ = false;

    size_t sfTotal(Structure const& s) const
    {
        size_t n = 0;
        for (auto const& a : s.atoms) n += (size_t)numSF_[a.element];
        return n;
    }

    n2p2_batch* boundBatch(Structure const& s) const
    {
        if (!s.device_ || !s.device_->batch) throw std::runtime_error("ERROR: structure has no results yet.\n");
        return s.device_->batch;
    }

    // The structure's device batch: created at the first call, positions
    // uploaded when they changed, the neighbour list built when wanted.
    n2p2_batch* bind(Structure& s)
    {
        if (numSF_.empty())
        {
            int ne = 0;
            check(n2p2_mode_get_num_elements(mode_, &ne));
            numSF_.resize((size_t)ne);
            for (int e = 0; e < ne; ++e) check(n2p2_mode_get_num_symmetry_functions(mode_, e, &numSF_[e]));
        }
        if (!s.hasNeighborList) throw std::runtime_error("ERROR: neighbour list not calculated.\n");
        if (s.listCutoff_ < getMaxCutoffRadius())
            throw std::invalid_argument("ERROR: neighbour list cutoff below the largest symmetry-function cutoff.\n");
        if (!s.device_ || !s.device_->batch || s.device_->owner != this || s.device_->numAtoms != s.numAtoms)
        {
            auto d = std::make_shared<Structure::Device>();
            d->owner = this;
            d->numAtoms = s.numAtoms;
            check(n2p2_batch_create(mode_, &d->batch));
            devices_.push_back(d);
            const int64_t n = (int64_t)s.numAtoms;
            std::vector<int32_t> el(s.numAtoms);
            for (size_t a = 0; a < s.numAtoms; ++a)
            {
                int e = 0;
                check(n2p2_mode_get_element_index(mode_, s.elementSymbols[a].c_str(), &e));
                el[a] = e;
                s.atoms[a].element = (size_t)e;
            }
            double box[9];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) box[3 * i + j] = s.box[i][j];
            const int32_t per = s.isPeriodic ? 1 : 0;
            check(n2p2_batch_set_structures(d->batch, 1, &n, el.data(), box, &per, 1));
            s.device_ = d;
        }
        std::vector<double> r(3 * s.numAtoms);
        for (size_t a = 0; a < s.numAtoms; ++a)
            for (int c = 0; c < 3; ++c) r[3 * a + c] = s.atoms[a].r[c];
        Structure::Device& d = *s.device_;
        if (d.uploaded != r)
        {
            // new positions: results of the old ones are not reused (the
            // reference would keep using them until Structure::reset)
            check(n2p2_batch_set_positions(d.batch, r.data(), 0));
            check(n2p2_batch_synchronize(d.batch));
            d.uploaded = r;
            s.listStale_ = true;
            s.hasSymmetryFunctions = s.hasSymmetryFunctionDerivatives = false;
        }
        if (s.listStale_)
        {
            check(n2p2_batch_calculate_neighbor_list(d.batch));
            fillNeighbors(s, d.batch);
            s.listStale_ = false;
        }
        return d.batch;
    }

    void fillNeighbors(Structure& s, n2p2_batch* b) const
    {
        int64_t M = 0;
        check(n2p2_batch_get_num_neighbor_entries(b, &M));
        std::vector<int64_t> off(s.numAtoms + 1);
        std::vector<int32_t> idx((size_t)M), img((size_t)M);
        std::vector<double> d((size_t)M), dr(3 * (size_t)M);
        check(n2p2_batch_get_neighbors(b, off.data(), idx.data(), img.data(), d.data(), dr.data()));
        for (size_t i = 0; i < s.numAtoms; ++i)
        {
            Atom& a = s.atoms[i];
            a.neighbors.resize((size_t)(off[i + 1] - off[i]));
            for (int64_t k = off[i]; k < off[i + 1]; ++k)
            {
                Atom::Neighbor& n = a.neighbors[(size_t)(k - off[i])];
                n.index = (size_t)idx[k];
                n.element = s.atoms[n.index].element;
                n.d = d[k];
                for (int c = 0; c < 3; ++c) n.dr[c] = dr[3 * k + c];
                n.dGdr.clear();
            }
            a.numNeighbors = a.neighbors.size();
            a.hasNeighborList = true;
        }
    }

    void fillDerivatives(Structure& s, n2p2_batch* b) const
    {
        size_t rows = 0;
        for (auto const& a : s.atoms)
            for (auto const& n : a.neighbors)
            {
                int r = 0;
                check(n2p2_mode_get_num_derivative_rows(mode_, (int)a.element, (int)n.element, &r));
                rows += (size_t)r;
            }
        std::vector<double> self(3 * sfTotal(s)), nbr(3 * rows);
        check(n2p2_batch_get_dGdr(b, self.data(), nbr.data()));
        size_t at = 0, atRow = 0;
        for (auto& a : s.atoms)
        {
            a.dGdr.resize(a.numSymmetryFunctions);
            for (size_t k = 0; k < a.numSymmetryFunctions; ++k, ++at)
                for (int c = 0; c < 3; ++c) a.dGdr[k][c] = self[3 * at + c];
            for (auto& n : a.neighbors)
            {
                int r = 0;
                check(n2p2_mode_get_num_derivative_rows(mode_, (int)a.element, (int)n.element, &r));
                n.dGdr.resize((size_t)r);
                for (int k = 0; k < r; ++k, ++atRow)
                    for (int c = 0; c < 3; ++c) n.dGdr[(size_t)k][c] = nbr[3 * atRow + c];
            }
        }
    }
};

} // namespace nnp
} // namespace n2p2b200

#endif
