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
// Atoms [a0, a1) only.  With img, the part of g_imgAtom that comes from the
// atom's own periodic images (entries with j == i) is also written to
// img[0..numSF): Mode::calculateForces skips those entries
// (neighborsUnique.begin() + 1, Mode.cpp:1957) while Training::collectDGdxia
// (Training.cpp:3604-3615) keeps them.
// With `list`, atoms list[0..a1) instead of [a0, a1).
__global__ void __launch_bounds__(kTrainWarps * 32) kSFAdjoint(DevModel model, BatchView b, int a0, int a1,
                                                               const double* __restrict__ u, double* __restrict__ g,
                                                               int imgAtom = -1, double* __restrict__ img = nullptr,
                                                               const int* __restrict__ list = nullptr)
{
    __shared__ double acc[kTrainWarps][kTrainMaxInput];
    __shared__ double accImg[kTrainWarps][kTrainMaxInput];
    const int lane = threadIdx.x & 31;
    double* a = acc[threadIdx.x >> 5];
    double* ai = accImg[threadIdx.x >> 5];
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int k = a0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < a1; k += warpsPerGrid)
    {
        const int i = list ? list[k] : k;
        const int ec = b.elem[i];
        DevElement const& E = model.el[ec];
        const double ux = u[3 * (size_t)i + 0], uy = u[3 * (size_t)i + 1], uz = u[3 * (size_t)i + 2];
        __syncwarp();
        const bool track = img && i == imgAtom;
        for (int s = lane; s < E.numSF; s += 32)
        {
            const double* p = b.dGdrSelf + ((size_t)i * b.gStride + s) * 3;
            a[s] = -(p[0] * ux + p[1] * uy + p[2] * uz);
            ai[s] = 0.0;
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
                const double d = p[0] * vx + p[1] * vy + p[2] * vz;
                a[table[r]] -= d;
                if (track && j == i) ai[table[r]] -= d;
            }
            __syncwarp();
        }
        for (int s = lane; s < E.numSF; s += 32)
        {
            g[(size_t)i * b.gStride + s] = a[s];
            if (track) img[s] = ai[s];
        }
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

// Per-atom parameter gradient of L_i = a_i E_i + (dE_i/dG_i . g_i) over atoms
// [a0, a1), summed into the warp's slice gradPart[warp][P] (parameter layout
// of the device weights).  a_i = aStruct[structure of i], or aConst without
// aStruct; no g means g = 0.  With predPart, the warp's sum of L_i goes to
// predPart[warp] (the value whose gradient this is).  TANGENT false: g must be
// null (no tangent is carried; the zero-tangent terms are skipped).
template <bool TANGENT>
__global__ void __launch_bounds__(kTrainWarps * 32) kParamGrad(DevModel model, BatchView b, int a0, int a1,
                                                               const double* __restrict__ aStruct, double aConst,
                                                               const double* __restrict__ g, int P,
                                                               double* __restrict__ gradPart,
                                                               double* __restrict__ predPart,
                                                               int imgAtom = -1,
                                                               const double* __restrict__ img = nullptr,
                                                               const int* __restrict__ list = nullptr)
{
    __shared__ ParamSmem smem[kTrainWarps];
    ParamSmem& S = smem[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    double* slice = gradPart + (size_t)warp * P;
    for (int p = lane; p < P; p += 32) slice[p] = 0.0;
    double pred = 0.0;
    __syncwarp();
    for (int k = a0 + warp; k < a1; k += warpsPerGrid)
    {
        const int i = list ? list[k] : k;
        const int ec = b.elem[i];
        DevElement const& E = model.el[ec];
        const int L = E.numLayers;
        const double a = aStruct ? aStruct[b.atomStruct[i]] : aConst;
        for (int j = lane; j < E.neurons[0]; j += 32)
        {
            S.x0[j] = b.G[(size_t)i * b.gStride + j];
            S.xd0[j] = g ? g[(size_t)i * b.gStride + j] : 0.0;
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
                    if (TANGENT) zd += row[j] * S.ind(l, j);
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
        // the prediction leaves out the tangent along the atom's self-image part
        // of g (see kSFAdjoint); the gradient keeps it
        if (img && i == imgAtom)
        {
            for (int l = 1; l < L; ++l)
            {
                const int nin = E.neurons[l - 1], nout = E.neurons[l];
                const double* W = model.weights + E.wOffset[l];
                double t = 0.0;
                if (lane < nout)
                {
                    const double* row = W + (size_t)lane * nin;
                    for (int j = 0; j < nin; ++j) t += row[j] * (l == 1 ? img[j] : S.zb[j]);
                    t *= S.f1[l][lane];
                }
                __syncwarp();
                if (lane < nout) S.zb[lane] = t;
                __syncwarp();
            }
            if (lane == 0) pred -= S.zb[0];
            __syncwarp();
        }
        // reverse: seed d(a E + Edot)/dE = a, d/dEdot = 1 on the output neuron
        if (lane == 0)
        {
            S.xb[0] = a;
            S.xdb[0] = 1.0;
            pred += a * S.x[L - 1][0] + S.xd[L - 1][0];
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
                if (TANGENT)
                    for (int j = 0; j < nin; ++j) gw[j] += zb * S.in(l, j) + zdb * S.ind(l, j);
                else
                    for (int j = 0; j < nin; ++j) gw[j] += zb * S.in(l, j);
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
                        if (TANGENT) xdb += w * S.zdb[k];
                    }
                    S.xb[lane] = xb;
                    S.xdb[lane] = xdb;
                }
                __syncwarp();
            }
        }
    }
    if (predPart && lane == 0) predPart[warp] = pred;
}

// grad[p] = scale * sum over warps w (in order) of gradPart[w][p].
__global__ void kReduceGrad(const double* __restrict__ gradPart, int warps, int P, double* __restrict__ grad,
                            double scale = 1.0)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x)
    {
        double s = 0.0;
        for (int w = 0; w < warps; ++w) s += gradPart[(size_t)w * P + p];
        grad[p] = scale == 1.0 ? s : s * scale;
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
    kSFAdjoint<<<blocks, kTrainWarps * 32, 0, st>>>(m, b, 0, N, u_, g_);
    kParamGrad<true><<<blocks, kTrainWarps * 32, 0, st>>>(m, b, 0, N, aStruct_, 0.0, g_, P_, gradPart_, nullptr);
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

namespace {

__global__ void kSetEntry(double* p, int64_t k, double v) { p[k] = v; }

// The observation's prediction (sum of the warps' values, fixed order) and
// error: err = ref - prediction, xi = scale * err (Training.cpp:2879-2898,
// the force weight at :2910-2923).
// xi[1] keeps the unscaled sum over a task batch's candidates (accumulate),
// xi[0] that sum times the scale.
__global__ void kObsError(const double* __restrict__ predPart, int warps, const double* __restrict__ ref,
                          int64_t refIndex, double scale, double* __restrict__ xi, double* __restrict__ err,
                          int accumulate)
{
    const int lane = threadIdx.x;
    double p = 0.0;
    for (int w = lane; w < warps; w += 32) p += predPart[w];
    p = warpSum(p);
    if (lane == 0)
    {
        const double e = ref[refIndex] - p;
        *err = e;
        const double sum = accumulate ? xi[1] + e : e;
        xi[1] = sum;
        xi[0] = scale == 1.0 ? sum : sum * scale;
    }
}

// out[p] = scale * sum over slices w of part[w][p] in a fixed order: thread
// row r sums w = r, r + 8, ... in turn, the 8 partial sums are then added in
// row order.  32 parameters x 8 slice rows per block.
// With `accumulate` the sum is added to out's previous value before scaling
// (task batches: the candidates' Jacobians are summed, then scaled once).
__global__ void __launch_bounds__(256) kReduceSlices(const double* __restrict__ part, int slices, int P,
                                                     double* __restrict__ out, double scale, int accumulate)
{
    __shared__ double acc[8][32];
    const int lx = threadIdx.x & 31, r = threadIdx.x >> 5;
    const int p = blockIdx.x * 32 + lx;
    double s = 0.0;
    if (p < P)
        for (int w = r; w < slices; w += 8) s += part[(size_t)w * P + p];
    acc[r][lx] = s;
    __syncthreads();
    if (r == 0 && p < P)
    {
        double t = acc[0][lx];
        for (int k = 1; k < 8; ++k) t += acc[k][lx];
        if (accumulate) t = out[p] + t;
        out[p] = scale == 1.0 ? t : t * scale;
    }
}

constexpr int kTile = 64;   // lower-triangle tiles of the covariance

// Lower-triangle pass over P (the reference reads only that half,
// P.selfadjointView<Lower>()): one CTA per 64 x 64 tile (I >= J) applies the
// previous update's pending change (P_ic - K_i X_c) * scale (+ q on the
// diagonal) to its elements i >= c, and writes two fixed-order partial sums
// for this update's X = P H: rowPart[tile][r] = sum_c P_ic H_c over its
// columns, colPart[tile][c] = sum_(i > c) P_ic H_i over its rows (the upper
// half's contribution, by symmetry).  kKalmanXSum adds them up per row.
__global__ void __launch_bounds__(256) kKalmanTiles(double* __restrict__ Pm, const double* __restrict__ Kp,
                                                    const double* __restrict__ Xp, int n, int pending, double scale,
                                                    double q, const double* __restrict__ H,
                                                    double* __restrict__ rowPart, double* __restrict__ colPart,
                                                    int rank = 1, int ld = 0)
{
    __shared__ double rowS[kTile][kTile + 1];
    __shared__ double colS[4][kTile];
    const int t = blockIdx.x;
    // tile index t = I (I + 1) / 2 + J, J <= I
    int I = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((I + 1) * (I + 2) / 2 <= t) ++I;
    while (I * (I + 1) / 2 > t) --I;
    const int J = t - I * (I + 1) / 2;
    const int tx = threadIdx.x & (kTile - 1), ty = threadIdx.x >> 6;
    const int c = J * kTile + tx;
    const bool cIn = c < n;
    const double Hc = cIn ? H[c] : 0.0;
    const double Xc = cIn && pending ? Xp[c] : 0.0;
    double colAcc = 0.0;
    for (int r = ty; r < kTile; r += 4)
    {
        const int i = I * kTile + r;
        double contrib = 0.0;
        if (cIn && i < n && c <= i)
        {
            double* pe = Pm + (size_t)i * n + c;
            double v = *pe;
            if (pending)
            {
                v = v - Kp[i] * Xc;
                for (int o = 1; o < rank; ++o) v = v - Kp[i + (size_t)o * ld] * Xp[c + (size_t)o * ld];
                if (scale != 1.0) v *= scale;
                if (c == i) v += q;
                *pe = v;
            }
            contrib = v * Hc;
            if (c < i) colAcc += v * H[i];
        }
        rowS[r][tx] = contrib;
    }
    colS[ty][tx] = colAcc;
    __syncthreads();
    if (threadIdx.x < kTile)
    {
        const int r = threadIdx.x;
        double a = 0.0;
        for (int k = 0; k < kTile; ++k) a += rowS[r][k];
        rowPart[(size_t)t * kTile + r] = a;
        colPart[(size_t)t * kTile + r] = ((colS[0][r] + colS[1][r]) + colS[2][r]) + colS[3][r];
    }
}

// X_i = the row partials of the tiles of row block I plus the column
// partials of the tiles of column block I (rows I..T-1): one warp per row,
// lanes over the partials, fixed shuffle-tree order.
__global__ void __launch_bounds__(256) kKalmanXSum(const double* __restrict__ rowPart,
                                                   const double* __restrict__ colPart, int n, int T,
                                                   double* __restrict__ X)
{
    const int lane = threadIdx.x & 31;
    const int warpsPerGrid = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warpsPerGrid)
    {
        const int I = i / kTile, r = i % kTile;
        double a = 0.0;
        for (int J = lane; J <= I; J += 32) a += rowPart[((size_t)I * (I + 1) / 2 + J) * kTile + r];
        for (int I2 = I + lane; I2 < T; I2 += 32) a += colPart[((size_t)I2 * (I2 + 1) / 2 + I) * kTile + r];
        a = warpSum(a);
        if (lane == 0) X[i] = a;
    }
}

// The updater's error: xi as it is (div == 0), or the per-element share
// (xi * mul) / div * post (Training.cpp:2900-2922 with update_strategy 1:
// mul / div the element's atoms / all atoms, or the atom's neighbours of the
// element / all its neighbours; post the force weight).
__device__ __forceinline__ double updaterError(const double* xi, double mul, double div, double post)
{
    const double e = *xi;
    return div == 0.0 ? e : e * mul / div * post;
}

// A = H^T X + diag (one observation), K = X A^-1, w += K xi (the transposed
// weight copy follows).  One block, fixed reduction order.
__global__ void __launch_bounds__(1024) kKalmanGain(const double* __restrict__ H, const double* __restrict__ X, int n,
                                                    double diag, const double* __restrict__ xi, double mul,
                                                    double div, double post, double* __restrict__ K,
                                                    double* __restrict__ w, double* __restrict__ wT,
                                                    const int* __restrict__ tidx)
{
    __shared__ double part[1024];
    double a = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) a += H[i] * X[i];
    part[threadIdx.x] = a;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1)
    {
        if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    const double inv = 1.0 / (part[0] + diag);
    const double e = updaterError(xi, mul, div, post);
    for (int i = threadIdx.x; i < n; i += blockDim.x)
    {
        const double k = X[i] * inv;
        K[i] = k;
        const double wi = w[i] + k * e;
        w[i] = wi;
        wT[tidx[i]] = wi;
    }
}

constexpr int kMaxObs = 16;   // observations per update with the full Jacobian

// Several observations (jacobian_mode 2): A = H^T X + diag I (m x m), its
// inverse by Gauss-Jordan elimination with partial pivoting, K = X A^-1,
// w += K xi (xi[2 o] the scaled error of observation o).  One block.
__global__ void __launch_bounds__(1024) kKalmanGainFull(const double* __restrict__ H, const double* __restrict__ X,
                                                        int n, int ld, int m, double diag,
                                                        const double* __restrict__ xi, double* __restrict__ K,
                                                        double* __restrict__ w, double* __restrict__ wT,
                                                        const int* __restrict__ tidx, int* __restrict__ singular)
{
    __shared__ double part[1024];
    __shared__ double A[kMaxObs][2 * kMaxObs];
    __shared__ int bad;
    for (int a = 0; a < m; ++a)
        for (int c = 0; c < m; ++c)
        {
            double s = 0.0;
            for (int i = threadIdx.x; i < n; i += blockDim.x) s += H[i + (size_t)a * ld] * X[i + (size_t)c * ld];
            part[threadIdx.x] = s;
            __syncthreads();
            for (int st = blockDim.x / 2; st > 0; st >>= 1)
            {
                if (threadIdx.x < st) part[threadIdx.x] += part[threadIdx.x + st];
                __syncthreads();
            }
            if (threadIdx.x == 0)
            {
                A[a][c] = part[0] + (a == c ? diag : 0.0);
                A[a][m + c] = a == c ? 1.0 : 0.0;
            }
            __syncthreads();
        }
    if (threadIdx.x == 0)
    {
        // A = H^T P H + diag I is symmetric positive definite while P is; a
        // pivot that is not finite, or negligible against the largest
        // diagonal entry (linearly dependent observations with a degenerate
        // P), makes the inverse meaningless: the update is skipped and counted
        double scaleA = 0.0;
        for (int c = 0; c < m; ++c) scaleA = fmax(scaleA, fabs(A[c][c]));
        bad = !(scaleA > 0.0) || !isfinite(scaleA);
        for (int c = 0; c < m && !bad; ++c)
        {
            int piv = c;
            for (int r = c + 1; r < m; ++r)
                if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
            if (piv != c)
                for (int k = 0; k < 2 * m; ++k)
                {
                    const double t = A[c][k];
                    A[c][k] = A[piv][k];
                    A[piv][k] = t;
                }
            if (!isfinite(A[c][c]) || !(fabs(A[c][c]) > 1e-14 * scaleA))
            {
                bad = 1;
                break;
            }
            const double d = 1.0 / A[c][c];
            for (int k = 0; k < 2 * m; ++k) A[c][k] *= d;
            for (int r = 0; r < m; ++r)
                if (r != c)
                {
                    const double f = A[r][c];
                    for (int k = 0; k < 2 * m; ++k) A[r][k] -= f * A[c][k];
                }
        }
        if (bad) atomicAdd(singular, 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
    {
        double wi = w[i];
        for (int c = 0; c < m; ++c)
        {
            double k = 0.0;
            if (!bad)
                for (int a = 0; a < m; ++a) k += X[i + (size_t)a * ld] * A[a][m + c];
            K[i + (size_t)c * ld] = k;   // a skipped update leaves P's change at zero
            wi += k * xi[2 * c];
        }
        if (!bad)
        {
            w[i] = wi;
            wT[tidx[i]] = wi;
        }
    }
}

// P = (P - K X^T) * scale + q I, every element with the formula of its lower
// twin (row max(i, j), column min(i, j)), so P stays exactly symmetric.
__global__ void __launch_bounds__(256) kKalmanP(double* __restrict__ Pm, const double* __restrict__ K,
                                                const double* __restrict__ X, int n, double scale, double q,
                                                int rank = 1, int ld = 0)
{
    const int i = blockIdx.y;
    const double Ki = K[i], Xi = X[i];
    double* row = Pm + (size_t)i * n;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j <= i && j < n; j += gridDim.x * blockDim.x)
    {
        double v = row[j] - Ki * X[j];
        for (int o = 1; o < rank; ++o) v = v - K[i + (size_t)o * ld] * X[j + (size_t)o * ld];
        if (scale != 1.0) v *= scale;
        if (j == i) v += q;
        row[j] = v;
    }
    (void)Xi;
}

__global__ void kKalmanInit(double* __restrict__ Pm, int n, double d)
{
    const size_t total = (size_t)n * n;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x)
        Pm[k] = (k / n == k % n) ? d : 0.0;
}

// GradientDescent::update, DT_FIXED: state -= eta * error * -gradient.
__global__ void kGradFixed(int n, const double* __restrict__ H, const double* __restrict__ xi, double mul,
                           double div, double post, double eta, double* __restrict__ w, double* __restrict__ wT,
                           const int* __restrict__ tidx)
{
    const double e = updaterError(xi, mul, div, post);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const double wi = w[i] - eta * e * -H[i];
        w[i] = wi;
        wT[tidx[i]] = wi;
    }
}

// GradientDescent::update, DT_ADAM, with g = error * -gradient.
__global__ void kGradAdam(int n, const double* __restrict__ H, const double* __restrict__ xi, double mul, double div,
                          double post, double beta1, double beta2, double eta, double eps, double* __restrict__ m,
                          double* __restrict__ v, double* __restrict__ w, double* __restrict__ wT,
                          const int* __restrict__ tidx)
{
    const double e = updaterError(xi, mul, div, post);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const double gi = e * -H[i];
        const double mi = beta1 * m[i] + (1.0 - beta1) * gi;
        const double vi = beta2 * v[i] + (1.0 - beta2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const double wi = w[i] - eta * mi / (sqrt(vi) + eps);
        w[i] = wi;
        wT[tidx[i]] = wi;
    }
}

// Partial sums for KalmanFilter::status: per block sum |P_ii|, sum |P_ij|, sum |K_i|.
__global__ void __launch_bounds__(256) kKalmanStat(const double* __restrict__ Pm, const double* __restrict__ K, int n,
                                                   double* __restrict__ out)
{
    __shared__ double part[3][256];
    double d = 0.0, a = 0.0, k = 0.0;
    const size_t total = (size_t)n * n;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
    {
        const size_t i = e / n, j = e % n;
        if (j > i) continue;   // the lower half is the stored one; the upper mirrors it
        const double v = fabs(Pm[e]);
        a += i == j ? v : 2.0 * v;
        if (i == j) d += v;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) k += fabs(K[i]);
    part[0][threadIdx.x] = d;
    part[1][threadIdx.x] = a;
    part[2][threadIdx.x] = k;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1)
    {
        if (threadIdx.x < s)
            for (int c = 0; c < 3; ++c) part[c][threadIdx.x] += part[c][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; ++c) out[3 * blockIdx.x + c] = part[c][0];
}

constexpr int kStatBlocks = 256;

std::vector<int> fileOrderToDevice(DevModel const& v)
{
    std::vector<int> map;
    for (int e = 0; e < v.numElements; ++e)
    {
        DevElement const& E = v.el[e];
        for (int l = 1; l < E.numLayers; ++l)
        {
            const int nin = E.neurons[l - 1], nout = E.neurons[l];
            for (int j = 0; j < nin; ++j)
                for (int k = 0; k < nout; ++k) map.push_back(E.wOffset[l] + k * nin + j);
            for (int k = 0; k < nout; ++k) map.push_back(E.bOffset[l] + k);
        }
    }
    return map;
}

} // namespace

Training::Training(Model& model, DeviceModel& dmodel, Batch& set, int sms)
    : model_(model), dmodel_(dmodel), set_(set), sms_(sms)
{
    if (&set.deviceModel() != &dmodel_) throw std::invalid_argument("ERROR: batch belongs to another mode.\n");
    if (set.external()) throw std::invalid_argument("ERROR: training needs structures, not external lists.\n");
    DevModel const& v = dmodel_.view;
    if (v.numCompactGroups > 0)
        throw std::invalid_argument("ERROR: training needs stored dG/dr, which compact functions do not provide.\n");
    // the network limits of the gradient kernels
    Trainer probe(model_, dmodel_, 1);
    (void)probe;
    P_ = (int)dmodel_.numWeights;
    fileToDevice_ = fileOrderToDevice(v);
    if ((int)fileToDevice_.size() != P_) throw std::runtime_error("ERROR: weight layout mismatch.\n");
    N_ = set.numAtoms();
    S_ = set.numStructures();
    if (N_ == 0) throw std::runtime_error("ERROR: no structures set.\n");
    // G and dG/dr of the whole set, once (they do not depend on the weights)
    set.evaluate(EVAL_FORCES | EVAL_STORE_DGDR | EVAL_NO_GRAPH, PREC_FP64, 0);
    BatchView const& b = set.view();
    cudaStream_t st = set.stream();
    atomBegin_.resize((size_t)S_ + 1);
    cudaCheck(cudaMemcpyAsync(atomBegin_.data(), b.structAtomBegin, sizeof(int) * (S_ + 1), cudaMemcpyDeviceToHost, st),
              "D2H");
    cudaCheck(cudaStreamSynchronize(st), "sync");
    int maxAtoms = 0;
    for (int k = 0; k < S_; ++k) maxAtoms = std::max(maxAtoms, atomBegin_[k + 1] - atomBegin_[k]);
    // per element: its contiguous block of device weights, atoms per structure, neighbours per atom
    const int ne = v.numElements;
    size_t fpos = 0;
    for (int e = 0; e < ne; ++e)
    {
        DevElement const& E = v.el[e];
        int cnt = 0;
        for (int l = 1; l < E.numLayers; ++l) cnt += E.neurons[l] * E.neurons[l - 1] + E.neurons[l];
        int lo = P_, hi = 0;
        for (int q = 0; q < cnt; ++q)
        {
            lo = std::min(lo, fileToDevice_[fpos + q]);
            hi = std::max(hi, fileToDevice_[fpos + q] + 1);
        }
        if (hi - lo != cnt) throw std::runtime_error("ERROR: element weights are not contiguous.\n");
        elemRange_.push_back({lo, cnt});
        fpos += cnt;
    }
    {
        std::vector<int> elem(N_);
        std::vector<int64_t> off((size_t)N_ + 1);
        cudaCheck(cudaMemcpyAsync(elem.data(), b.elem, sizeof(int) * N_, cudaMemcpyDeviceToHost, st), "D2H");
        cudaCheck(cudaMemcpyAsync(off.data(), b.nbrOffset, sizeof(int64_t) * (N_ + 1), cudaMemcpyDeviceToHost, st),
                  "D2H");
        cudaCheck(cudaStreamSynchronize(st), "sync");
        std::vector<int> nj((size_t)off[N_]);
        if (!nj.empty())
            cudaCheck(cudaMemcpyAsync(nj.data(), b.nbrJ, sizeof(int) * nj.size(), cudaMemcpyDeviceToHost, st), "D2H");
        cudaCheck(cudaStreamSynchronize(st), "sync");
        atomsPerElement_.assign((size_t)S_ * ne, 0);
        for (int k = 0; k < S_; ++k)
            for (int i = atomBegin_[k]; i < atomBegin_[k + 1]; ++i) ++atomsPerElement_[(size_t)k * ne + elem[i]];
        nbrPerElement_.assign((size_t)N_ * ne, 0);
        nbrCount_.assign(N_, 0);
        for (int i = 0; i < N_; ++i)
        {
            nbrCount_[i] = (int)(off[i + 1] - off[i]);
            for (int64_t q = off[i]; q < off[i + 1]; ++q) ++nbrPerElement_[(size_t)i * ne + elem[nj[q]]];
        }
        // per atom: itself and its distinct neighbours, ascending (the neighbour relation is
        // symmetric, so these are the atoms whose functions depend on its position)
        std::vector<int> nearList;
        nearOffset_.assign((size_t)N_ + 1, 0);
        std::vector<int> tmp;
        for (int i = 0; i < N_; ++i)
        {
            tmp.assign(nj.begin() + off[i], nj.begin() + off[i + 1]);
            tmp.push_back(i);
            std::sort(tmp.begin(), tmp.end());
            tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
            nearList.insert(nearList.end(), tmp.begin(), tmp.end());
            nearOffset_[i + 1] = (int64_t)nearList.size();
        }
        near_ = tAlloc<int>(nearList.size());
        cudaCheck(cudaMemcpyAsync(near_, nearList.data(), sizeof(int) * nearList.size(), cudaMemcpyHostToDevice, st),
                  "H2D");
        cudaCheck(cudaStreamSynchronize(st), "sync");
    }
    blocks_.push_back({0, P_, 0});
    maxWarps_ = std::min(maxAtoms, sms_ * 8);
    maxWarps_ = (maxWarps_ + kTrainWarps - 1) / kTrainWarps * kTrainWarps;
    eRef_ = tAlloc<double>(S_);
    fRef_ = tAlloc<double>(3 * (size_t)N_);
    u_ = tAlloc<double>(3 * (size_t)N_);
    g_ = tAlloc<double>((size_t)N_ * b.gStride);
    gradPart_ = tAlloc<double>((size_t)maxWarps_ * P_);
    predPart_ = tAlloc<double>(maxWarps_);
    H_ = tAlloc<double>((size_t)P_ * kMaxObs);
    xi_ = tAlloc<double>(2 * kMaxObs);
    for (int k = 0; k < 2; ++k)
    {
        Xb_[k] = tAlloc<double>((size_t)P_ * kMaxObs);
        Kb_[k] = tAlloc<double>((size_t)P_ * kMaxObs);
    }
    stat_ = tAlloc<double>(3 * kStatBlocks);
    singular_ = tAlloc<int>(1);
    cudaCheck(cudaMemsetAsync(singular_, 0, sizeof(int), st), "memset");
    {
        const int T = (P_ + kTile - 1) / kTile;
        rowPart_ = tAlloc<double>((size_t)T * (T + 1) / 2 * kTile);
        colPart_ = tAlloc<double>((size_t)T * (T + 1) / 2 * kTile);
    }
    img_ = tAlloc<double>(b.gStride);
    cudaCheck(cudaMemsetAsync(u_, 0, sizeof(double) * 3 * (size_t)N_, st), "memset");
    for (int k = 0; k < 2; ++k) cudaCheck(cudaMemsetAsync(Kb_[k], 0, sizeof(double) * P_ * kMaxObs, st), "memset");
    cudaCheck(cudaMemsetAsync(eRef_, 0, sizeof(double) * S_, st), "memset");
    cudaCheck(cudaMemsetAsync(fRef_, 0, sizeof(double) * 3 * (size_t)N_, st), "memset");
    cudaCheck(cudaStreamSynchronize(st), "sync");
}

Training::~Training()
{
    for (void* p : {(void*)eRef_, (void*)fRef_, (void*)u_, (void*)g_, (void*)gradPart_, (void*)predPart_, (void*)H_,
                    (void*)xi_, (void*)err_, (void*)Pm_, (void*)Xb_[0], (void*)Xb_[1], (void*)Kb_[0], (void*)Kb_[1], (void*)m_, (void*)v_, (void*)stat_, (void*)singular_, (void*)img_, (void*)rowPart_, (void*)colPart_,
                    (void*)near_})
        cudaFree(p);
}

void Training::setReferences(const double* energiesPhys, const double* forcesPhys)
{
    std::vector<double> e(S_), f(3 * (size_t)N_);
    set_.energiesToInternal(energiesPhys, e.data());
    const double cf = set_.forceToInternal();
    for (size_t q = 0; q < f.size(); ++q) f[q] = forcesPhys[q] * cf;
    cudaStream_t st = set_.stream();
    eRefHost_ = e;
    fRefHost_ = f;
    cudaCheck(cudaMemcpyAsync(eRef_, e.data(), sizeof(double) * S_, cudaMemcpyHostToDevice, st), "H2D");
    cudaCheck(cudaMemcpyAsync(fRef_, f.data(), sizeof(double) * f.size(), cudaMemcpyHostToDevice, st), "H2D");
    cudaCheck(cudaStreamSynchronize(st), "sync");
}

void Training::setKalmanStandard(double epsilon, double q0, double qtau, double qmin, double eta0, double etatau,
                                 double etamax)
{
    // KalmanFilter::KalmanFilter (P = I) and setParametersStandard (P /= epsilon), KalmanFilter.cpp:62-117, 199-218
    initKalman(epsilon);
    type_ = KF_STANDARD;
    epsilon_ = epsilon;
    q0_ = q0;
    qtau_ = qtau;
    qmin_ = qmin;
    eta0_ = eta0;
    etatau_ = etatau;
    etamax_ = etamax;
    q_ = q0;
    eta_ = eta0;
    numUpdates_ = 0;
}

void Training::setKalmanFadingMemory(double epsilon, double q0, double qtau, double qmin, double lambda, double nu)
{
    // KalmanFilter::setParametersFadingMemory, KalmanFilter.cpp:220-238
    initKalman(epsilon);
    type_ = KF_FADING_MEMORY;
    epsilon_ = epsilon;
    q0_ = q0;
    qtau_ = qtau;
    qmin_ = qmin;
    lambda_ = lambda;
    nu_ = nu;
    q_ = q0;
    gamma_ = 1.0;
    numUpdates_ = 0;
}

void Training::setGradientFixed(double eta)
{
    type_ = GD_FIXED;
    gdEta_ = eta;
    numUpdates_ = 0;
}

void Training::setGradientAdam(double eta, double beta1, double beta2, double epsilon)
{
    // GradientDescent::setParametersAdam: moments 0, beta1t = beta1, beta2t = beta2
    if (!m_) m_ = tAlloc<double>(P_);
    if (!v_) v_ = tAlloc<double>(P_);
    cudaCheck(cudaMemsetAsync(m_, 0, sizeof(double) * P_, set_.stream()), "memset");
    cudaCheck(cudaMemsetAsync(v_, 0, sizeof(double) * P_, set_.stream()), "memset");
    type_ = GD_ADAM;
    gdEta_ = eta;
    beta1_ = beta1;
    beta2_ = beta2;
    gdEps_ = epsilon;
    beta1t_ = beta1;
    beta2t_ = beta2;
    numUpdates_ = 0;
}

// Error and Jacobian of one observation at the current weights
// (Training.cpp:2551-2681 for the 2G networks): the energy of structure s
// (sum of dE_i/dc over its atoms) or force component c of its atom a (the
// second-order gradient with the force adjoint e_{a,c}); force errors and
// Jacobians carry the force weight.
void Training::observation(int property, int s, int a, int c, int t, bool accumulate, bool last, int column)
{
    const int acc = accumulate ? 1 : 0;
    double* H = H_ + (size_t)column * P_;   // the full Jacobian keeps one column per observation
    double* xi = xi_ + 2 * column;
    cudaStream_t st = set_.stream();
    BatchView const& b = set_.view();
    DevModel const& m = dmodel_.view;
    const int a0 = atomBegin_[s], a1 = atomBegin_[s + 1];
    const int warps = std::min(maxWarps_, (a1 - a0 + kTrainWarps - 1) / kTrainWarps * kTrainWarps);
    const int blocks = warps / kTrainWarps;
    if (property == ENERGY)
    {
        kParamGrad<false><<<blocks, kTrainWarps * 32, 0, st>>>(m, b, a0, a1, nullptr, 1.0, nullptr, P_, gradPart_,
                                                               predPart_);
        kReduceSlices<<<(P_ + 31) / 32, 256, 0, st>>>(gradPart_, warps, P_, H, 1.0, acc);
        kObsError<<<1, 32, 0, st>>>(predPart_, warps, eRef_, s, 1.0, xi, err_ + t, acc);
    }
    else
    {
        // only the atom and its neighbours carry a nonzero adjoint: the passes run over that list
        const int64_t k = 3 * (int64_t)(a0 + a) + c;
        const int l0 = (int)nearOffset_[a0 + a], l1 = (int)nearOffset_[a0 + a + 1];
        const int fw = std::min(maxWarps_, (l1 - l0 + kTrainWarps - 1) / kTrainWarps * kTrainWarps);
        const int fb = fw / kTrainWarps;
        kSetEntry<<<1, 1, 0, st>>>(u_, k, 1.0);
        kSFAdjoint<<<fb, kTrainWarps * 32, 0, st>>>(m, b, l0, l1, u_, g_, a0 + a, img_, near_);
        kSetEntry<<<1, 1, 0, st>>>(u_, k, 0.0);
        kParamGrad<true><<<fb, kTrainWarps * 32, 0, st>>>(m, b, l0, l1, nullptr, 0.0, g_, P_, gradPart_, predPart_, a0 + a,
                                                    img_, near_);
        kReduceSlices<<<(P_ + 31) / 32, 256, 0, st>>>(gradPart_, fw, P_, H, last ? forceWeight_ : 1.0, acc);
        kObsError<<<1, 32, 0, st>>>(predPart_, fw, fRef_, k, forceWeight_, xi, err_ + t, acc);
    }
    cudaCheck(cudaGetLastError(), "observation launch");
}

// The updaters' step with the observation in H_ / xi_: one updater over all
// weights (combined strategy) or one per element over its block of weights
// (element strategy), each with its share of the error.
void Training::step(int property, int s, int a, int m)
{
    cudaStream_t st = set_.stream();
    double* w = dmodel_.weightsDevice();
    double* wT = dmodel_.weightsTDevice();
    const int* tidx = dmodel_.transIndexDevice();
    const int tb = 256;
    const int ne = (int)blocks_.size();
    const bool element = strategy_ == US_ELEMENT;
    auto share = [&](int e, double& mul, double& div) {
        if (!element)
        {
            mul = 1.0;
            div = 0.0;
        }
        else if (property == ENERGY)
        {
            mul = (double)atomsPerElement_[(size_t)s * ne + e];
            div = (double)(atomBegin_[s + 1] - atomBegin_[s]);
        }
        else
        {
            const size_t k = (size_t)(atomBegin_[s] + a);
            mul = (double)nbrPerElement_[k * ne + e];
            div = (double)nbrCount_[k];
        }
    };
    // the combined path reads the scaled error; the element path scales the raw one itself
    const double* xiPtr = element ? xi_ + 1 : xi_;
    const double post = element && property == FORCE ? forceWeight_ : 1.0;
    if (type_ == KF_STANDARD || type_ == KF_FADING_MEMORY)
    {
        // KalmanFilter::update (KalmanFilter.cpp:126-197), one observation per updater; the
        // updaters advance in lockstep, so their eta, q, lambda and gamma are shared scalars
        double diag, scale = 1.0;
        if (type_ == KF_STANDARD)
        {
            if (eta_ < etamax_) eta_ *= std::exp(etatau_);
            diag = 1.0 / eta_;
        }
        else
        {
            diag = lambda_;
            scale = 1.0 / lambda_;
        }
        // this update's X with the previous update's P update applied on the way
        const int cur = cur_ ^ 1;
        if (m > 1)
        {
            // jacobian_mode 2 (combined strategy): X column by column, the pending change applied
            // by the first pass, then the m x m gain
            const int n = P_, T = (n + kTile - 1) / kTile;
            for (int o = 0; o < m; ++o)
            {
                kKalmanTiles<<<T * (T + 1) / 2, 256, 0, st>>>(Pm_, Kb_[cur_], Xb_[cur_], n, (o == 0 && pending_) ? 1 : 0,
                                                               pendingScale_, pendingQ_, H_ + (size_t)o * n, rowPart_,
                                                               colPart_, pendingRank_, n);
                kKalmanXSum<<<(n + 7) / 8, 256, 0, st>>>(rowPart_, colPart_, n, T, Xb_[cur] + (size_t)o * n);
            }
            kKalmanGainFull<<<1, 1024, 0, st>>>(H_, Xb_[cur], n, n, m, diag, xi_, Kb_[cur], w, wT, tidx, singular_);
        }
        else
        for (int e = 0; e < ne; ++e)
        {
            Block const& B = blocks_[e];
            double mul, div;
            share(e, mul, div);
            const int T = (B.count + kTile - 1) / kTile;
            const int tiles = T * (T + 1) / 2;
            kKalmanTiles<<<tiles, 256, 0, st>>>(Pm_ + B.pOffset, Kb_[cur_] + B.begin, Xb_[cur_] + B.begin, B.count,
                                                pending_ ? 1 : 0, pendingScale_, pendingQ_, H_ + B.begin, rowPart_,
                                                colPart_, pendingRank_, P_);
            kKalmanXSum<<<(B.count + 7) / 8, 256, 0, st>>>(rowPart_, colPart_, B.count, T, Xb_[cur] + B.begin);
            kKalmanGain<<<1, 1024, 0, st>>>(H_ + B.begin, Xb_[cur] + B.begin, B.count, diag, xiPtr, mul, div, post,
                                            Kb_[cur] + B.begin, w + B.begin, wT, tidx + B.begin);
        }
        cur_ = cur;
        pending_ = true;   // P - K X^T, * scale, + q I: applied by the next pass over P
        pendingRank_ = m;
        pendingScale_ = scale;
        pendingQ_ = q_;
        if (q_ > qmin_) q_ *= std::exp(-qtau_);
        if (type_ == KF_FADING_MEMORY)
        {
            lambda_ = nu_ * lambda_ + 1.0 - nu_;
            gamma_ = 1.0 / (1.0 + lambda_ / gamma_);
        }
    }
    else if (m > 1)
        throw std::invalid_argument("ERROR: the full Jacobian needs the Kalman filter.\n");
    else if (type_ == GD_FIXED)
    {
        for (int e = 0; e < ne; ++e)
        {
            Block const& B = blocks_[e];
            double mul, div;
            share(e, mul, div);
            kGradFixed<<<(B.count + tb - 1) / tb, tb, 0, st>>>(B.count, H_ + B.begin, xiPtr, mul, div, post, gdEta_,
                                                               w + B.begin, wT, tidx + B.begin);
        }
    }
    else
    {
        const double eta = gdEta_ * std::sqrt(1.0 - beta2t_) / (1.0 - beta1t_);
        for (int e = 0; e < ne; ++e)
        {
            Block const& B = blocks_[e];
            double mul, div;
            share(e, mul, div);
            kGradAdam<<<(B.count + tb - 1) / tb, tb, 0, st>>>(B.count, H_ + B.begin, xiPtr, mul, div, post, beta1_,
                                                              beta2_, eta, gdEps_, m_ + B.begin, v_ + B.begin,
                                                              w + B.begin, wT, tidx + B.begin);
        }
        beta1t_ *= beta1_;
        beta2t_ *= beta2_;
    }
    cudaCheck(cudaGetLastError(), "updater launch");
    ++numUpdates_;
}

void Training::setUpdateStrategy(int strategy)
{
    if (strategy != US_COMBINED && strategy != US_ELEMENT) throw std::invalid_argument("ERROR: unknown update strategy.\n");
    strategy_ = strategy;
    blocks_.clear();
    if (strategy == US_COMBINED) blocks_.push_back({0, P_, 0});
    else
    {
        size_t off = 0;
        for (auto const& r : elemRange_)
        {
            blocks_.push_back({r.first, r.second, off});
            off += (size_t)r.second * r.second;
        }
    }
    type_ = -1;   // the updater is set up again for the new blocks
}

void Training::initKalman(double epsilon)
{
    if (!Pm_) Pm_ = tAlloc<double>((size_t)P_ * P_);
    for (Block const& B : blocks_)
        kKalmanInit<<<sms_ * 8, 256, 0, set_.stream()>>>(Pm_ + B.pOffset, B.count, 1.0 / epsilon);
    cudaCheck(cudaGetLastError(), "kalman init");
    pending_ = false;
    pendingRank_ = 1;
    cudaCheck(cudaMemsetAsync(Kb_[cur_], 0, sizeof(double) * P_ * kMaxObs, set_.stream()), "memset");
}

void Training::update(int property, int count, const int* structure, const int* atom, const int* component,
                      double* errors)
{
    if (type_ < 0) throw std::runtime_error("ERROR: no updater set.\n");
    if (property != ENERGY && property != FORCE) throw std::invalid_argument("ERROR: unknown property.\n");
    for (int t = 0; t < count; ++t)
    {
        const int s = structure[t];
        if (s < 0 || s >= S_) throw std::out_of_range("ERROR: structure index out of range.\n");
        if (property == FORCE)
        {
            if (atom[t] < 0 || atom[t] >= atomBegin_[s + 1] - atomBegin_[s])
                throw std::out_of_range("ERROR: atom index out of range.\n");
            if (component[t] < 0 || component[t] > 2) throw std::out_of_range("ERROR: force component out of range.\n");
        }
    }
    cudaStream_t st = set_.stream();
    if (count > errCap_)
    {
        cudaFree(err_);
        errCap_ = count;
        err_ = tAlloc<double>(count);
    }
    // a task batch of candidates forms one observation: errors and Jacobians
    // summed at the same weights, then one updater step (Training.cpp:2879-2923)
    const int batch = property == ENERGY ? taskBatchEnergy_ : taskBatchForce_;
    if (strategy_ == US_ELEMENT && batch != 1)
        throw std::invalid_argument("ERROR: the element update strategy needs task batches of one candidate.\n");
    if (fullJacobian_ && batch > kMaxObs)
        throw std::invalid_argument("ERROR: the full Jacobian takes at most 16 candidates per update.\n");
    if (fullJacobian_ && batch > 1 && type_ != KF_STANDARD && type_ != KF_FADING_MEMORY)
        throw std::invalid_argument("ERROR: the full Jacobian needs the Kalman filter.\n");
    if (count % batch != 0)
        throw std::invalid_argument("ERROR: the number of candidates is not a multiple of the task batch size.\n");
    for (int t = 0; t < count; ++t)
    {
        const int q = t % batch;
        if (fullJacobian_)   // one observation per candidate
            observation(property, structure[t], property == FORCE ? atom[t] : 0, property == FORCE ? component[t] : 0,
                        t, false, true, q);
        else
            observation(property, structure[t], property == FORCE ? atom[t] : 0, property == FORCE ? component[t] : 0,
                        t, q > 0, q == batch - 1);
        if (q == batch - 1) step(property, structure[t], property == FORCE ? atom[t] : 0, fullJacobian_ ? batch : 1);
    }
    if (errors)
        cudaCheck(cudaMemcpyAsync(errors, err_, sizeof(double) * count, cudaMemcpyDeviceToHost, st), "D2H");
    int skipped = 0;
    if (fullJacobian_ && batch > 1)
    {
        cudaCheck(cudaMemcpyAsync(&skipped, singular_, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
        cudaCheck(cudaMemsetAsync(singular_, 0, sizeof(int), st), "memset");
    }
    cudaCheck(cudaStreamSynchronize(st), "sync");
    if (skipped > 0)
        throw std::runtime_error("ERROR: " + std::to_string(skipped) +
                                 " update(s) skipped: the m x m matrix of the full Jacobian was singular "
                                 "(linearly dependent observations in one task batch); their weights are "
                                 "unchanged.\n");
}

int Training::updateThreshold(int property, int numUpdates, int numCandidates, const int* structure, const int* atom,
                              const int* component, double threshold, int trials, double rmse, double* errors)
{
    if (type_ < 0) throw std::runtime_error("ERROR: no updater set.\n");
    if (property != ENERGY && property != FORCE) throw std::invalid_argument("ERROR: unknown property.\n");
    if ((property == ENERGY ? taskBatchEnergy_ : taskBatchForce_) != 1)
        throw std::invalid_argument("ERROR: threshold selection needs task batches of one candidate.\n");
    if (numCandidates < 1 || trials < 1) throw std::invalid_argument("ERROR: no candidates or trials.\n");
    for (int t = 0; t < numCandidates; ++t)
    {
        const int s = structure[t];
        if (s < 0 || s >= S_) throw std::out_of_range("ERROR: structure index out of range.\n");
        if (property == FORCE && (atom[t] < 0 || atom[t] >= atomBegin_[s + 1] - atomBegin_[s] || component[t] < 0 ||
                                  component[t] > 2))
            throw std::out_of_range("ERROR: atom or component out of range.\n");
    }
    if (errCap_ < 1)
    {
        errCap_ = 1;
        err_ = tAlloc<double>(1);
    }
    cudaStream_t st = set_.stream();
    int pos = 0;
    auto obs = [&](int k) {
        observation(property, structure[k], property == FORCE ? atom[k] : 0, property == FORCE ? component[k] : 0, 0,
                    false, true, 0);
        double e = 0.0;
        cudaCheck(cudaMemcpyAsync(&e, err_, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        cudaCheck(cudaStreamSynchronize(st), "sync");
        return e;
    };
    for (int u = 0; u < numUpdates; ++u)
    {
        // When no trial exceeds the threshold the reference records the best
        // candidate but updates with the one it tried last (the candidate
        // pointer c is not reset to indexBest, Training.cpp:2492-2505, and
        // c->s is the structure used at :2527); so does this loop.
        int chosen = -1;
        double chosenErr = 0.0;
        for (int il = 0; il < trials; ++il)
        {
            const int k = pos % numCandidates;
            const double e = obs(k);
            const int s = structure[k];
            const double frac =
                property == ENERGY ? std::fabs(e) / ((atomBegin_[s + 1] - atomBegin_[s]) * rmse) : std::fabs(e) / rmse;
            ++pos;
            chosen = k;
            chosenErr = e;
            if (frac > threshold) break;
        }
        step(property, structure[chosen], property == FORCE ? atom[chosen] : 0, 1);
        if (errors) errors[u] = chosenErr;
    }
    cudaCheck(cudaStreamSynchronize(st), "sync");
    return pos;
}

void Training::trainingErrors(double* rmseEnergyPerAtom, double* rmseForce)
{
    if (eRefHost_.empty()) throw std::runtime_error("ERROR: no references set.\n");
    flushKalman();
    set_.evaluate(EVAL_FORCES | EVAL_STORE_DGDR | EVAL_NO_GRAPH, PREC_FP64, 0);
    BatchView const& b = set_.view();
    cudaStream_t st = set_.stream();
    std::vector<double> E(S_), F(3 * (size_t)N_);
    cudaCheck(cudaMemcpyAsync(E.data(), b.Estruct, sizeof(double) * S_, cudaMemcpyDeviceToHost, st), "D2H");
    cudaCheck(cudaMemcpyAsync(F.data(), b.F, sizeof(double) * F.size(), cudaMemcpyDeviceToHost, st), "D2H");
    cudaCheck(cudaStreamSynchronize(st), "sync");
    // Structure::updateError / Atom::updateError summed, Training::collectError
    double se = 0.0, sf = 0.0;
    for (int k = 0; k < S_; ++k)
    {
        const double n = (double)(atomBegin_[k + 1] - atomBegin_[k]);
        const double d = eRefHost_[k] - E[k];
        se += d * d / (n * n);
    }
    for (size_t q = 0; q < F.size(); ++q)
    {
        const double d = fRefHost_[q] - F[q];
        sf += d * d;
    }
    *rmseEnergyPerAtom = std::sqrt(se / S_);
    *rmseForce = std::sqrt(sf / (double)F.size());
}

void Training::observe(int property, int structure, int atom, int component, double* error,
                       double* jacobianFileOrder)
{
    if (property != ENERGY && property != FORCE) throw std::invalid_argument("ERROR: unknown property.\n");
    if (structure < 0 || structure >= S_) throw std::out_of_range("ERROR: structure index out of range.\n");
    if (property == FORCE && (atom < 0 || atom >= atomBegin_[structure + 1] - atomBegin_[structure] ||
                              component < 0 || component > 2))
        throw std::out_of_range("ERROR: atom or component out of range.\n");
    if (errCap_ < 1)
    {
        errCap_ = 1;
        err_ = tAlloc<double>(1);
    }
    cudaStream_t st = set_.stream();
    observation(property, structure, atom, component, 0, false, true, 0);
    std::vector<double> h(P_);
    cudaCheck(cudaMemcpyAsync(h.data(), H_, sizeof(double) * P_, cudaMemcpyDeviceToHost, st), "D2H");
    cudaCheck(cudaMemcpyAsync(error, err_, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    cudaCheck(cudaStreamSynchronize(st), "sync");
    for (int q = 0; q < P_; ++q) jacobianFileOrder[q] = h[fileToDevice_[q]];
}

void Training::flushKalman()
{
    if (!pending_) return;
    for (Block const& B : blocks_)
    {
        dim3 grid((B.count + 255) / 256, B.count);
        kKalmanP<<<grid, 256, 0, set_.stream()>>>(Pm_ + B.pOffset, Kb_[cur_] + B.begin, Xb_[cur_] + B.begin, B.count,
                                                  pendingScale_, pendingQ_, pendingRank_, P_);
    }
    cudaCheck(cudaGetLastError(), "kalman flush");
    pending_ = false;
}

void Training::kalmanStatus(double* out)
{
    flushKalman();
    out[0] = (double)numUpdates_;
    out[1] = out[2] = out[3] = 0.0;
    if (Pm_ && (type_ == KF_STANDARD || type_ == KF_FADING_MEMORY))
    {
        // over all updaters' covariance blocks (one block for the combined strategy)
        cudaStream_t st = set_.stream();
        double d = 0.0, a = 0.0, k = 0.0, offCount = 0.0;
        std::vector<double> part(3 * kStatBlocks);
        for (Block const& B : blocks_)
        {
            kKalmanStat<<<kStatBlocks, 256, 0, st>>>(Pm_ + B.pOffset, Kb_[cur_] + B.begin, B.count, stat_);
            cudaCheck(cudaMemcpyAsync(part.data(), stat_, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st),
                      "D2H");
            cudaCheck(cudaStreamSynchronize(st), "sync");
            for (int bIdx = 0; bIdx < kStatBlocks; ++bIdx)
            {
                d += part[3 * bIdx];
                a += part[3 * bIdx + 1];
                k += part[3 * bIdx + 2];
            }
            offCount += (double)B.count * (B.count - 1.0);
        }
        const double n = (double)P_;
        out[1] = d / n;
        out[2] = (a - d) / offCount;
        out[3] = k / n;
    }
    out[4] = q_;
    out[5] = type_ == KF_FADING_MEMORY ? lambda_ : eta_;
    out[6] = gamma_;
}

void Training::getWeights(double* fileOrder)
{
    std::vector<double> w(P_);
    cudaStream_t st = set_.stream();
    cudaCheck(cudaMemcpyAsync(w.data(), dmodel_.weightsDevice(), sizeof(double) * P_, cudaMemcpyDeviceToHost, st),
              "D2H");
    cudaCheck(cudaStreamSynchronize(st), "sync");
    for (int q = 0; q < P_; ++q) fileOrder[q] = w[fileToDevice_[q]];
}

void Training::setWeights(const double* fileOrder)
{
    std::vector<double> w(P_), wt(P_);
    for (int q = 0; q < P_; ++q) w[fileToDevice_[q]] = fileOrder[q];
    for (int q = 0; q < P_; ++q) wt[dmodel_.transIndexHost[q]] = w[q];
    cudaStream_t st = set_.stream();
    cudaCheck(cudaMemcpyAsync(dmodel_.weightsDevice(), w.data(), sizeof(double) * P_, cudaMemcpyHostToDevice, st),
              "H2D");
    cudaCheck(cudaMemcpyAsync(dmodel_.weightsTDevice(), wt.data(), sizeof(double) * P_, cudaMemcpyHostToDevice, st),
              "H2D");
    cudaCheck(cudaStreamSynchronize(st), "sync");
}

} // namespace n2p2b200
