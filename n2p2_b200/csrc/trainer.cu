// Training of a (small) HDNNP on energies and forces: loss, its adjoints, the
// parameter gradient through the force term, and Adam -- all on the device.
//
// Loss of a batch of S structures with N atoms (internal units):
//   L = wE / S * sum_s ((E_s - E_s^ref) / N_s)^2 + wF / (3N) * sum_k |F_k - F_k^ref|^2
// The forces F_k = -sum_i sum_s dE_i/dG_is dG_is/dr_k depend on the weights
// through dE/dG, so
//   dL/dtheta = sum_i [ a_i dE_i/dtheta + d/dtheta (sum_s g_is dE_i/dG_is) ]
// with a_i = dL/dE_s(i) and g_is = -sum_k u_k . dG_is/dr_k, u_k = dL/dF_k.
// The second term is the parameter gradient of the directional derivative of
// E_i along g_i: a forward pass carries (value, tangent) through the network,
// a reverse pass differentiates both (second derivatives of the activations
// enter through the tangents).
//
// The forward pass (G, dG/dr, dE/dG, E, F) is the engine's own evaluation
// with stored dG/dr.  Parameter gradients are summed per warp into private
// slices and the slices in a fixed order: results do not depend on timing.
// Adam follows GradientDescent::update (libnnptrain/GradientDescent.cpp:89-113)
// in its bias-corrected step-size form.
#include "trainer.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "kernels_common.cuh"

namespace n2p2b200 {

namespace {

constexpr int kTrainWarps = 4;
constexpr int kTrainMaxLayers = 4;   // input, two hidden, output
constexpr int kTrainMaxWidth = 32;   // neurons of a hidden or output layer
constexpr int kTrainMaxInput = 128;  // symmetry functions of an element

// Value, first and second derivative of the activations the trainer supports.
__device__ __forceinline__ void activate2(int af, double x, double& f, double& f1, double& f2)
{
    switch (af)
    {
    case AF_IDENTITY: f = x; f1 = 1.0; f2 = 0.0; return;
    case AF_TANH:
    {
        const double t = tanh(x);
        f = t;
        f1 = 1.0 - t * t;
        f2 = -2.0 * t * f1;
        return;
    }
    case AF_LOGISTIC:
    {
        const double t = 1.0 / (1.0 + exp(-x));
        f = t;
        f1 = t * (1.0 - t);
        f2 = f1 * (1.0 - 2.0 * t);
        return;
    }
    case AF_SOFTPLUS:
    {
        // log(1 + e^x) with the reference's linear/zero tails (|x| > 35)
        if (x > 35.0) { f = x; f1 = 1.0; f2 = 0.0; return; }
        if (x < -35.0) { f = 0.0; f1 = 0.0; f2 = 0.0; return; }
        const double t = exp(x);
        f = log(1.0 + t);
        const double sg = 1.0 / (1.0 + 1.0 / t);
        f1 = sg;
        f2 = sg * (1.0 - sg);
        return;
    }
    }
    f = f1 = f2 = 0.0;
}

// a_s = dL/dE_s and wE ((E_s - E_ref) / N_s)^2 / S per structure.
__global__ void kEnergyResidual(BatchView b, const double* __restrict__ eRef, double wE,
                                double* __restrict__ aStruct, double* __restrict__ lossE)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < b.S; s += gridDim.x * blockDim.x)
    {
        const double n = (double)(b.structAtomBegin[s + 1] - b.structAtomBegin[s]);
        const double d = b.Estruct[s] - eRef[s];
        aStruct[s] = 2.0 * wE * d / (n * n * b.S);
        lossE[s] = wE * (d / n) * (d / n) / b.S;
    }
}

// u_k = dL/dF_k and wF |F_k - F_ref|^2 / (3N) per atom.
__global__ void kForceResidual(BatchView b, const double* __restrict__ fRef, double wF, double* __restrict__ u,
                               double* __restrict__ lossF)
{
    const double c = wF / (3.0 * b.N);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < b.N; k += gridDim.x * blockDim.x)
    {
        double l = 0.0;
        for (int q = 0; q < 3; ++q)
        {
            const double d = b.F[3 * (size_t)k + q] - fRef[3 * (size_t)k + q];
            u[3 * (size_t)k + q] = 2.0 * c * d;
            l += d * d;
        }
        lossF[k] = c * l;
    }
}

// One block: out[0] = sum lossE[0..S), out[1] = sum lossF[0..N), fixed order.
__global__ void __launch_bounds__(256) kLossSum(const double* __restrict__ lossE, int S,
                                                const double* __restrict__ lossF, int N, double* __restrict__ out)
{
    __shared__ double part[2][256];
    double a = 0.0, c = 0.0;
    for (int s = threadIdx.x; s < S; s += 256) a += lossE[s];
    for (int k = threadIdx.x; k < N; k += 256) c += lossF[k];
    part[0][threadIdx.x] = a;
    part[1][threadIdx.x] = c;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1)
    {
        if (threadIdx.x < w)
        {
            part[0][threadIdx.x] += part[0][threadIdx.x + w];
            part[1][threadIdx.x] += part[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        out[0] = part[0][0] + part[1][0];
        out[1] = part[0][0];
        out[2] = part[1][0];
    }
}

// g_is = -(u_i . dG_is/dr_i + sum_{e = (i -> j)} u_j . dG_is/dr_j): the
// transpose of the stored-dG/dr force contraction.  Lanes own the rows of an
// entry (distinct SFs), entries are visited in list order.
__global__ void __launch_bounds__(kTrainWarps * 32) kSFAdjoint(DevModel model, BatchView b,
                                                               const double* __restrict__ u, double* __restrict__ g)
{
    __shared__ double acc[kTrainWarps][kTrainMaxInput];
    const int lane = threadIdx.x & 31;
    double* a = acc[threadIdx.x >> 5];
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < b.N; i += warpsPerGrid)
    {
        const int ec = b.elem[i];
        DevElement const& E = model.el[ec];
        const double ux = u[3 * (size_t)i + 0], uy = u[3 * (size_t)i + 1], uz = u[3 * (size_t)i + 2];
        __syncwarp();
        for (int s = lane; s < E.numSF; s += 32)
        {
            const double* p = b.dGdrSelf + ((size_t)i * b.gStride + s) * 3;
            a[s] = -(p[0] * ux + p[1] * uy + p[2] * uz);
        }
        __syncwarp();
        for (int64_t e = b.nbrOffset[i]; e < b.nbrOffset[i + 1]; ++e)
        {
            const int j = b.nbrJ[e];
            const int en = b.elem[j];
            const double vx = u[3 * (size_t)j + 0], vy = u[3 * (size_t)j + 1], vz = u[3 * (size_t)j + 2];
            const int* table = model.rowTable + E.tableBegin[en];
            for (int r = lane; r < E.rows[en]; r += 32)
            {
                const double* p = b.dGdr + ((size_t)r * b.nbrCapacity + e) * 3;
                a[table[r]] -= p[0] * vx + p[1] * vy + p[2] * vz;
            }
            __syncwarp();
        }
        for (int s = lane; s < E.numSF; s += 32) g[(size_t)i * b.gStride + s] = a[s];
    }
}

struct ParamSmem
{
    double x0[kTrainMaxInput], xd0[kTrainMaxInput];                   // G and g
    double x[kTrainMaxLayers][kTrainMaxWidth];                        // layer outputs
    double xd[kTrainMaxLayers][kTrainMaxWidth];                       // their tangents along g
    __device__ __forceinline__ double in(int l, int j) const { return l == 1 ? x0[j] : x[l - 1][j]; }
    __device__ __forceinline__ double ind(int l, int j) const { return l == 1 ? xd0[j] : xd[l - 1][j]; }
    double zd[kTrainMaxLayers][kTrainMaxWidth];
    double f1[kTrainMaxLayers][kTrainMaxWidth];
    double f2[kTrainMaxLayers][kTrainMaxWidth];
    double zb[kTrainMaxWidth], zdb[kTrainMaxWidth];
    double xb[kTrainMaxWidth], xdb[kTrainMaxWidth];
};

// Per-atom parameter gradient of a_i E_i + (dE_i/dG_i . g_i), summed into the
// warp's slice gradPart[warp][P] (parameter layout of the device weights).
__global__ void __launch_bounds__(kTrainWarps * 32) kParamGrad(DevModel model, BatchView b,
                                                               const double* __restrict__ aStruct,
                                                               const double* __restrict__ g, int P,
                                                               double* __restrict__ gradPart)
{
    __shared__ ParamSmem smem[kTrainWarps];
    ParamSmem& S = smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    double* slice = gradPart + (size_t)warp * P;
    for (int p = lane; p < P; p += 32) slice[p] = 0.0;
    __syncwarp();
    for (int i = warp; i < b.N; i += warpsPerGrid)
    {
        const int ec = b.elem[i];
        DevElement const& E = model.el[ec];
        const int L = E.numLayers;
        const double a = aStruct[b.atomStruct[i]];
        for (int j = lane; j < E.neurons[0]; j += 32)
        {
            S.x0[j] = b.G[(size_t)i * b.gStride + j];
            S.xd0[j] = g[(size_t)i * b.gStride + j];
        }
        __syncwarp();
        for (int l = 1; l < L; ++l)
        {
            const int nin = E.neurons[l - 1], nout = E.neurons[l];
            const double* W = model.weights + E.wOffset[l];
            const double* bias = model.weights + E.bOffset[l];
            if (lane < nout)
            {
                double z = bias[lane], zd = 0.0;
                const double* row = W + (size_t)lane * nin;
                for (int j = 0; j < nin; ++j)
                {
                    z += row[j] * S.in(l, j);
                    zd += row[j] * S.ind(l, j);
                }
                double f, f1, f2;
                activate2(E.activation[l], z, f, f1, f2);
                S.x[l][lane] = f;
                S.xd[l][lane] = f1 * zd;
                S.zd[l][lane] = zd;
                S.f1[l][lane] = f1;
                S.f2[l][lane] = f2;
            }
            __syncwarp();
        }
        // reverse: seed d(a E + Edot)/dE = a, d/dEdot = 1 on the output neuron
        if (lane == 0)
        {
            S.xb[0] = a;
            S.xdb[0] = 1.0;
        }
        __syncwarp();
        for (int l = L - 1; l >= 1; --l)
        {
            const int nin = E.neurons[l - 1], nout = E.neurons[l];
            const double* W = model.weights + E.wOffset[l];
            if (lane < nout)
            {
                const double xb = S.xb[lane], xdb = S.xdb[lane];
                const double zb = xb * S.f1[l][lane] + xdb * S.f2[l][lane] * S.zd[l][lane];
                const double zdb = xdb * S.f1[l][lane];
                S.zb[lane] = zb;
                S.zdb[lane] = zdb;
                double* gw = slice + E.wOffset[l] + (size_t)lane * nin;
                for (int j = 0; j < nin; ++j) gw[j] += zb * S.in(l, j) + zdb * S.ind(l, j);
                slice[E.bOffset[l] + lane] += zb;
            }
            __syncwarp();
            if (l > 1)
            {
                if (lane < nin)
                {
                    double xb = 0.0, xdb = 0.0;
                    for (int k = 0; k < nout; ++k)
                    {
                        const double w = W[(size_t)k * nin + lane];
                        xb += w * S.zb[k];
                        xdb += w * S.zdb[k];
                    }
                    S.xb[lane] = xb;
                    S.xdb[lane] = xdb;
                }
                __syncwarp();
            }
        }
    }
}

// grad[p] = sum over warps w (in order) of gradPart[w][p].
__global__ void kReduceGrad(const double* __restrict__ gradPart, int warps, int P, double* __restrict__ grad)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x)
    {
        double s = 0.0;
        for (int w = 0; w < warps; ++w) s += gradPart[(size_t)w * P + p];
        grad[p] = s;
    }
}

// Adam (GradientDescent::update, DT_ADAM): m, v moments, step
// eta0 sqrt(1 - beta2^t) / (1 - beta1^t); the transposed weight copy is
// refreshed as well.
__global__ void kAdam(int P, const double* __restrict__ grad, double* __restrict__ m, double* __restrict__ v,
                      double* __restrict__ w, double* __restrict__ wT, const int* __restrict__ tidx, double beta1,
                      double beta2, double eta, double eps)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x)
    {
        const double gp = grad[p];
        const double mp = beta1 * m[p] + (1.0 - beta1) * gp;
        const double vp = beta2 * v[p] + (1.0 - beta2) * gp * gp;
        m[p] = mp;
        v[p] = vp;
        const double wp = w[p] - eta * mp / (sqrt(vp) + eps);
        w[p] = wp;
        wT[tidx[p]] = wp;
    }
}

template <typename T>
T* tAlloc(size_t n)
{
    void* p = nullptr;
    cudaCheck(cudaMalloc(&p, sizeof(T) * (n ? n : 1)), "cudaMalloc");
    return static_cast<T*>(p);
}

} // namespace

Trainer::Trainer(Model& model, DeviceModel& dmodel, int sms) : model_(model), dmodel_(dmodel), sms_(sms)
{
    DevModel const& v = dmodel_.view;
    if (v.normalizeNeurons) throw std::invalid_argument("ERROR: training with normalize_nodes is not supported.\n");
    for (int e = 0; e < v.numElements; ++e)
    {
        DevElement const& E = v.el[e];
        if (E.numLayers > kTrainMaxLayers)
            throw std::invalid_argument("ERROR: training supports at most two hidden layers.\n");
        if (E.neurons[0] > kTrainMaxInput)
            throw std::invalid_argument("ERROR: training supports at most 128 symmetry functions per element.\n");
        for (int l = 1; l < E.numLayers; ++l)
        {
            if (E.neurons[l] > kTrainMaxWidth)
                throw std::invalid_argument("ERROR: training supports layers of at most 32 neurons.\n");
            const int af = E.activation[l];
            if (af != AF_IDENTITY && af != AF_TANH && af != AF_LOGISTIC && af != AF_SOFTPLUS)
                throw std::invalid_argument("ERROR: activation not supported for training (l, t, s, p are).\n");
        }
    }
    P_ = (int)dmodel_.numWeights;
    // file order (NeuralNetwork::setConnections, per element) -> device index
    for (int e = 0; e < v.numElements; ++e)
    {
        DevElement const& E = v.el[e];
        for (int l = 1; l < E.numLayers; ++l)
        {
            const int nin = E.neurons[l - 1], nout = E.neurons[l];
            for (int j = 0; j < nin; ++j)
                for (int k = 0; k < nout; ++k) fileToDevice_.push_back(E.wOffset[l] + k * nin + j);
            for (int k = 0; k < nout; ++k) fileToDevice_.push_back(E.bOffset[l] + k);
        }
    }
    if ((int)fileToDevice_.size() != P_) throw std::runtime_error("ERROR: weight layout mismatch.\n");
    warps_ = sms_ * 8 * kTrainWarps;
    grad_ = tAlloc<double>(P_);
    m_ = tAlloc<double>(P_);
    v_ = tAlloc<double>(P_);
    gradPart_ = tAlloc<double>((size_t)warps_ * P_);
    loss_ = tAlloc<double>(3);
    cudaCheck(cudaMemset(m_, 0, sizeof(double) * P_), "memset");
    cudaCheck(cudaMemset(v_, 0, sizeof(double) * P_), "memset");
}

Trainer::~Trainer()
{
    for (void* p : {(void*)grad_, (void*)m_, (void*)v_, (void*)gradPart_, (void*)loss_, (void*)eRef_, (void*)fRef_,
                    (void*)aStruct_, (void*)u_, (void*)g_, (void*)lossE_, (void*)lossF_})
        cudaFree(p);
}

void Trainer::setAdam(double eta, double beta1, double beta2, double eps)
{
    eta0_ = eta;
    beta1_ = beta1;
    beta2_ = beta2;
    eps_ = eps;
    beta1t_ = beta1;
    beta2t_ = beta2;
}

void Trainer::reserve(int S, int N, int stride)
{
    if (S > capS_)
    {
        cudaFree(eRef_);
        cudaFree(aStruct_);
        cudaFree(lossE_);
        capS_ = S;
        eRef_ = tAlloc<double>(S);
        aStruct_ = tAlloc<double>(S);
        lossE_ = tAlloc<double>(S);
    }
    if (N > capN_ || (size_t)N * stride > capG_)
    {
        cudaFree(fRef_);
        cudaFree(u_);
        cudaFree(g_);
        cudaFree(lossF_);
        capN_ = std::max(N, capN_);
        capG_ = std::max((size_t)N * stride, capG_);
        fRef_ = tAlloc<double>(3 * (size_t)capN_);
        u_ = tAlloc<double>(3 * (size_t)capN_);
        g_ = tAlloc<double>(capG_);
        lossF_ = tAlloc<double>(capN_);
    }
}

void Trainer::step(Batch& batch, const double* energiesPhys, const double* forcesPhys, bool update, double* loss,
                   double* gradFileOrder)
{
    if (&batch.deviceModel() != &dmodel_) throw std::invalid_argument("ERROR: batch belongs to another mode.\n");
    const int S = batch.numStructures(), N = batch.numAtoms();
    if (N == 0) throw std::runtime_error("ERROR: no structures set.\n");
    cudaStream_t st = batch.stream();
    batch.evaluate(EVAL_FORCES | EVAL_STORE_DGDR | EVAL_NO_GRAPH, PREC_FP64, 0);
    BatchView const& b = batch.view();
    reserve(S, N, b.gStride);
    // labels to internal units
    std::vector<double> e(S), f(3 * (size_t)N);
    batch.energiesToInternal(energiesPhys, e.data());
    const double cf = batch.forceToInternal();
    for (size_t q = 0; q < f.size(); ++q) f[q] = forcesPhys[q] * cf;
    cudaCheck(cudaMemcpyAsync(eRef_, e.data(), sizeof(double) * S, cudaMemcpyHostToDevice, st), "H2D");
    cudaCheck(cudaMemcpyAsync(fRef_, f.data(), sizeof(double) * f.size(), cudaMemcpyHostToDevice, st), "H2D");
    DevModel const& m = dmodel_.view;
    const int tb = 256;
    kEnergyResidual<<<(S + tb - 1) / tb, tb, 0, st>>>(b, eRef_, wE_, aStruct_, lossE_);
    kForceResidual<<<(N + tb - 1) / tb, tb, 0, st>>>(b, fRef_, wF_, u_, lossF_);
    kLossSum<<<1, 256, 0, st>>>(lossE_, S, lossF_, N, loss_);
    const int blocks = warps_ / kTrainWarps;
    kSFAdjoint<<<blocks, kTrainWarps * 32, 0, st>>>(m, b, u_, g_);
    kParamGrad<<<blocks, kTrainWarps * 32, 0, st>>>(m, b, aStruct_, g_, P_, gradPart_);
    kReduceGrad<<<(P_ + tb - 1) / tb, tb, 0, st>>>(gradPart_, warps_, P_, grad_);
    cudaCheck(cudaGetLastError(), "trainer launch");
    if (update)
    {
        const double eta = eta0_ * std::sqrt(1.0 - beta2t_) / (1.0 - beta1t_);
        kAdam<<<(P_ + tb - 1) / tb, tb, 0, st>>>(P_, grad_, m_, v_, dmodel_.weightsDevice(), dmodel_.weightsTDevice(),
                                                 dmodel_.transIndexDevice(), beta1_, beta2_, eta, eps_);
        cudaCheck(cudaGetLastError(), "adam launch");
        beta1t_ *= beta1_;
        beta2t_ *= beta2_;
        ++steps_;
    }
    if (loss)
        cudaCheck(cudaMemcpyAsync(loss, loss_, sizeof(double) * 3, cudaMemcpyDeviceToHost, st), "D2H");
    if (gradFileOrder)
    {
        std::vector<double> gd(P_);
        cudaCheck(cudaMemcpyAsync(gd.data(), grad_, sizeof(double) * P_, cudaMemcpyDeviceToHost, st), "D2H");
        cudaCheck(cudaStreamSynchronize(st), "sync");
        for (int q = 0; q < P_; ++q) gradFileOrder[q] = gd[fileToDevice_[q]];
    }
    cudaCheck(cudaStreamSynchronize(st), "sync");
}

void Trainer::getParameters(double* fileOrder, cudaStream_t st) const
{
    std::vector<double> w(P_);
    cudaCheck(cudaMemcpyAsync(w.data(), dmodel_.weightsDevice(), sizeof(double) * P_, cudaMemcpyDeviceToHost, st),
              "D2H");
    cudaCheck(cudaStreamSynchronize(st), "sync");
    for (int q = 0; q < P_; ++q) fileOrder[q] = w[fileToDevice_[q]];
}

void Trainer::setParameters(const double* fileOrder, cudaStream_t st)
{
    std::vector<double> w(P_), wt(P_);
    for (int q = 0; q < P_; ++q) w[fileToDevice_[q]] = fileOrder[q];
    for (int q = 0; q < P_; ++q) wt[dmodel_.transIndexHost[q]] = w[q];
    cudaCheck(cudaMemcpyAsync(dmodel_.weightsDevice(), w.data(), sizeof(double) * P_, cudaMemcpyHostToDevice, st),
              "H2D");
    cudaCheck(cudaMemcpyAsync(dmodel_.weightsTDevice(), wt.data(), sizeof(double) * P_, cudaMemcpyHostToDevice, st),
              "H2D");
    cudaCheck(cudaStreamSynchronize(st), "sync");
}

void Trainer::syncHostModel(cudaStream_t st)
{
    std::vector<double> w(P_);
    getParameters(w.data(), st);
    size_t pos = 0;
    for (size_t e = 0; e < model_.elements.size(); ++e)
    {
        NetworkTopology const& t = model_.elements[e].topology;
        size_t need = 0;
        for (int l = 1; l < t.numLayers; ++l) need += (size_t)t.neurons[l] * t.neurons[l - 1] + t.neurons[l];
        std::vector<double> c(w.begin() + pos, w.begin() + pos + need);
        model_.setConnections((int)e, c);
        pos += need;
    }
}

} // namespace n2p2b200
