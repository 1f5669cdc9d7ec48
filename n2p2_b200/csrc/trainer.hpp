// Device training of an HDNNP on energies and forces (loss adjoints, the
// second-order parameter gradient of the force term, Adam).
#pragma once

#include <vector>

#include "engine.hpp"

namespace n2p2b200 {

class Trainer
{
public:
    Trainer(Model& model, DeviceModel& dmodel, int sms);
    ~Trainer();
    Trainer(Trainer const&) = delete;
    Trainer& operator=(Trainer const&) = delete;

    int numParameters() const { return P_; }
    void setAdam(double eta, double beta1, double beta2, double eps);
    void setLearningRate(double eta) { eta0_ = eta; }
    void setLossWeights(double wE, double wF)
    {
        wE_ = wE;
        wF_ = wF;
    }
    // One evaluation of `batch` (positions already set) with the current
    // weights, the loss against the physical-unit labels (energies per
    // structure with offsets, forces [N][3]) and its gradient; `update` takes
    // an Adam step.  loss[3] = {total, energy term, force term}; the gradient
    // is returned in weight-file order (NeuralNetwork::setConnections, element
    // by element) when `gradFileOrder` is given.
    void step(Batch& batch, const double* energiesPhys, const double* forcesPhys, bool update, double* loss,
              double* gradFileOrder);
    void getParameters(double* fileOrder, cudaStream_t st) const;
    void setParameters(const double* fileOrder, cudaStream_t st);
    // Host model weights <- device weights (for writing weight files).
    void syncHostModel(cudaStream_t st);
    int steps() const { return steps_; }

private:
    void reserve(int S, int N, int stride);

    Model& model_;
    DeviceModel& dmodel_;
    int sms_;
    int P_ = 0;
    int warps_ = 0;
    std::vector<int> fileToDevice_;
    double wE_ = 1.0, wF_ = 10.0;
    double eta0_ = 1e-3, beta1_ = 0.9, beta2_ = 0.999, eps_ = 1e-8, beta1t_ = 0.9, beta2t_ = 0.999;
    int steps_ = 0;
    double* grad_ = nullptr;
    double* m_ = nullptr;
    double* v_ = nullptr;
    double* gradPart_ = nullptr;
    double* loss_ = nullptr;
    int capS_ = 0, capN_ = 0;
    size_t capG_ = 0;
    double* eRef_ = nullptr;
    double* fRef_ = nullptr;
    double* aStruct_ = nullptr;
    double* u_ = nullptr;
    double* g_ = nullptr;
    double* lossE_ = nullptr;
    double* lossF_ = nullptr;
};

// Weight updates of the reference's training program, one observation per
// update (Training::update, libnnptrain/Training.cpp:2256-3169, with the
// combined update strategy and one update candidate per update): the error of
// a structure's energy or of one force component at the current weights, its
// Jacobian with respect to all weights, and the Kalman filter
// (KalmanFilter::update, KalmanFilter.cpp:126-197) or gradient descent
// (GradientDescent::update, GradientDescent.cpp:81-118) step -- all on the
// device, without host round trips between updates.
//
// The symmetry functions and their derivatives do not depend on the weights:
// they are computed once for the whole training set and stay resident; an
// update runs the networks and the Jacobian over one structure's atoms only.
// The filter's covariance P (weights x weights, FP64) is stored and updated
// in its lower half only, the half the reference reads
// (P.selfadjointView<Lower>()).
class Training
{
public:
    enum Property { ENERGY = 0, FORCE = 1 };
    enum UpdaterType { KF_STANDARD = 0, KF_FADING_MEMORY = 1, GD_FIXED = 2, GD_ADAM = 3 };
    enum UpdateStrategy { US_COMBINED = 0, US_ELEMENT = 1 };

    Training(Model& model, DeviceModel& dmodel, Batch& set, int sms);
    ~Training();
    Training(Training const&) = delete;
    Training& operator=(Training const&) = delete;

    int numWeights() const { return P_; }
    // Reference energies per structure and forces [N][3] (physical units, with offsets).
    void setReferences(const double* energiesPhys, const double* forcesPhys);
    void setForceWeight(double w) { forceWeight_ = w; }
    // task_batch_size_energy / _force: candidates summed into one observation per update.
    // update_strategy (Training.cpp, US_COMBINED / US_ELEMENT): one updater over
    // all weights, or one per element over its networks' weights with the
    // error shared by the element's fraction of the atoms (energies) or of the
    // observed atom's neighbours (forces).  Set it before the updater.
    void setUpdateStrategy(int strategy);
    // jacobian_mode 2: every candidate of a task batch is its own observation
    // (the Kalman filter with the combined strategy; at most 16 per update).
    void setFullJacobian(bool full) { fullJacobian_ = full; }
    void setTaskBatchSize(int energy, int force)
    {
        taskBatchEnergy_ = energy;
        taskBatchForce_ = force;
    }
    void setKalmanStandard(double epsilon, double q0, double qtau, double qmin, double eta0, double etatau,
                           double etamax);
    void setKalmanFadingMemory(double epsilon, double q0, double qtau, double qmin, double lambda, double nu);
    void setGradientFixed(double eta);
    void setGradientAdam(double eta, double beta1, double beta2, double epsilon);
    // `count` candidates in order, task-batch-size consecutive candidates per
    // update: energy of structure[k], or force component
    // component[k] of atom atom[k] (index inside the structure) of
    // structure[k].  errors[k] (optional) receives ref - prediction before the
    // update, internal units.
    void update(int property, int count, const int* structure, const int* atom, const int* component,
                double* errors);
    // Error (ref - prediction, internal units) and Jacobian (weight-file order,
    // force weight applied for forces) of one observation, no update.
    void observe(int property, int structure, int atom, int component, double* error, double* jacobianFileOrder);
    // selection_mode 2 (threshold, Training.cpp:2288-2447): `numUpdates`
    // updates; each tries candidates from the list in order (wrapping) until
    // one's error exceeds `threshold` times the training RMSE (`rmse`: energy
    // per atom, or force component; internal units), at most `trials`; the
    // update uses the candidate the trials stopped at.  Returns the
    // candidates consumed; errors[u] is the used candidate's error.
    int updateThreshold(int property, int numUpdates, int numCandidates, const int* structure, const int* atom,
                        const int* component, double threshold, int trials, double rmse, double* errors);
    // Training errors at the current weights, internal units (Training::calculateError):
    // RMSE of the energy per atom and of the force components over the set.
    void trainingErrors(double* rmseEnergyPerAtom, double* rmseForce);
    // KalmanFilter::status: numUpdates, mean |P_ii|, mean |P_ij| (i != j),
    // mean |K|, q, eta (standard) or lambda (fading memory), gamma.
    void kalmanStatus(double* out);
    void getWeights(double* fileOrder);
    void setWeights(const double* fileOrder);
    int updaterType() const { return type_; }

private:
    void observation(int property, int s, int a, int c, int t, bool accumulate, bool last, int column = 0);
    void flushKalman();
    void initKalman(double epsilon);
    void step(int property, int s, int a, int m);
    struct Block
    {
        int begin, count;     // device weights [begin, begin + count)
        size_t pOffset;       // its covariance (count x count) inside Pm_
    };
    int strategy_ = US_COMBINED;
    std::vector<Block> blocks_;
    std::vector<std::pair<int, int>> elemRange_;
    std::vector<int> atomsPerElement_;   // [S][elements]
    std::vector<int> nbrPerElement_;     // [N][elements]
    std::vector<int> nbrCount_;          // [N]
    std::vector<int64_t> nearOffset_;    // [N+1] into near_
    int* near_ = nullptr;                // per atom: itself and its distinct neighbours, ascending

    Model& model_;
    DeviceModel& dmodel_;
    Batch& set_;
    int sms_;
    int P_ = 0, N_ = 0, S_ = 0;
    std::vector<int> fileToDevice_;
    std::vector<int> atomBegin_;
    double forceWeight_ = 1.0;
    int taskBatchEnergy_ = 1, taskBatchForce_ = 1;
    bool fullJacobian_ = false;
    int pendingRank_ = 1;
    std::vector<double> eRefHost_, fRefHost_;   // references, internal units
    int type_ = -1;
    // Kalman filter state (host scalars as in KalmanFilter)
    double epsilon_ = 0.0, q_ = 0.0, q0_ = 0.0, qtau_ = 0.0, qmin_ = 0.0, eta_ = 0.0, eta0_ = 0.0, etatau_ = 0.0,
           etamax_ = 0.0, lambda_ = 0.0, nu_ = 0.0, gamma_ = 0.0;
    long numUpdates_ = 0;
    // gradient descent
    double gdEta_ = 0.0, beta1_ = 0.0, beta2_ = 0.0, gdEps_ = 0.0, beta1t_ = 0.0, beta2t_ = 0.0;
    int maxWarps_ = 0;
    double* eRef_ = nullptr;     // [S] internal units
    double* fRef_ = nullptr;     // [3N]
    double* u_ = nullptr;        // [3N] force adjoint (one unit entry during a force update)
    double* g_ = nullptr;        // [N][gStride]
    double* gradPart_ = nullptr; // [maxWarps][P]
    double* predPart_ = nullptr; // [maxWarps]
    double* H_ = nullptr;        // [P] Jacobian of the observation
    double* xi_ = nullptr;       // observation error (scaled by the force weight)
    double* err_ = nullptr;      // [capacity] raw errors of the last update call
    int errCap_ = 0;
    double* Pm_ = nullptr;       // [P][P] covariance
    double* Xb_[2] = {nullptr, nullptr};   // [P] X of the last two updates (alternating)
    double* Kb_[2] = {nullptr, nullptr};   // [P] K of the last two updates
    int cur_ = 0;                // buffer of the latest update
    bool pending_ = false;       // the latest update's P - K X^T (* scale, + q I) not applied yet
    double pendingScale_ = 1.0, pendingQ_ = 0.0;
    double* m_ = nullptr;        // Adam moments
    double* v_ = nullptr;
    double* stat_ = nullptr;     // status partial sums
    int* singular_ = nullptr;    // full-Jacobian updates skipped for a singular m x m matrix
    double* img_ = nullptr;      // [gStride] self-image part of the observed atom's adjoint
    double* rowPart_ = nullptr;  // [tiles][64] row partial sums of X = P H
    double* colPart_ = nullptr;  // [tiles][64] column partial sums (the upper half's share)
};

} // namespace n2p2b200
