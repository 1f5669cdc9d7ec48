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

} // namespace n2p2b200
