// Host side of the learned block-match proposals: the MLP object behind the
// vnlbgpu_mlp_* entry points of include/vnlbgpu.h (no reference counterpart).
// It owns the FP32 weights, their BF16 copies, Adam's moments, and the
// activation and gradient buffers of batches up to max_batch rows.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/vnlbgpu.h"
#include "learned.h"

namespace vnlbgpu {

void set_last_error(const std::string& message);

namespace {

void check(cudaError_t status, const char* what) {
    if (status != cudaSuccess) throw std::runtime_error(std::string("VNLB CUDA: ") + what + " failed: " +
                                                        cudaGetErrorString(status));
}

template <typename T> T* device_alloc(size_t n, const char* what) {
    T* p = nullptr;
    check(cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T)), what);
    return p;
}

}  // namespace
}  // namespace vnlbgpu

struct vnlbgpu_mlp {
    int device = 0;
    int inputs = 0, hidden = 0, layers = 0, outputs = 0, max_batch = 0;
    int step = 0;
    cudaStream_t stream = nullptr;
    vnlbgpu::MlpDevice net{};
    float* w[vnlbgpu::kMlpMaxLayers + 1] = {};   // FP32 weights
    float* gw[vnlbgpu::kMlpMaxLayers + 1] = {};
    float* gb[vnlbgpu::kMlpMaxLayers + 1] = {};
    float* mw[vnlbgpu::kMlpMaxLayers + 1] = {};
    float* vw[vnlbgpu::kMlpMaxLayers + 1] = {};
    float* mb[vnlbgpu::kMlpMaxLayers + 1] = {};
    float* vb[vnlbgpu::kMlpMaxLayers + 1] = {};
    float* acts[vnlbgpu::kMlpMaxLayers] = {};
    float* dacts[vnlbgpu::kMlpMaxLayers] = {};
    float* logits = nullptr;
    float* loss = nullptr;
    int* status = nullptr;  // the inference kernels' status word

    int fan_in(int l) const { return l == 0 ? inputs : hidden; }
    int fan_out(int l) const { return l == layers ? outputs : hidden; }
    size_t weights(int l) const { return static_cast<size_t>(fan_out(l)) * fan_in(l); }
    size_t parameters() const {
        size_t n = 0;
        for (int l = 0; l <= layers; ++l) n += weights(l) + fan_out(l);
        return n;
    }

    ~vnlbgpu_mlp() {
        if (stream) cudaStreamSynchronize(stream);
        for (int l = 0; l <= vnlbgpu::kMlpMaxLayers; ++l)
            for (void* p : {static_cast<void*>(w[l]), static_cast<void*>(net.w16[l]), static_cast<void*>(net.b[l]),
                            static_cast<void*>(gw[l]), static_cast<void*>(gb[l]), static_cast<void*>(mw[l]),
                            static_cast<void*>(vw[l]), static_cast<void*>(mb[l]), static_cast<void*>(vb[l])})
                if (p) cudaFree(p);
        for (int l = 0; l < vnlbgpu::kMlpMaxLayers; ++l) {
            if (acts[l]) cudaFree(acts[l]);
            if (dacts[l]) cudaFree(dacts[l]);
        }
        if (logits) cudaFree(logits);
        if (loss) cudaFree(loss);
        if (status) cudaFree(status);
        if (stream) cudaStreamDestroy(stream);
    }

    void check_batch(int batch) const {
        if (batch <= 0 || batch > max_batch)
            throw std::invalid_argument("VNLB CUDA: batch must be in 1.." + std::to_string(max_batch));
    }

    // forward, then the gradients of the mean loss; returns the mean loss
    float gradients(const float* x, const int* targets, int batch, int tk) {
        check_batch(batch);
        vnlbgpu::check(vnlbgpu::mlp_forward(net, x, batch, acts, logits, stream), "MLP forward");
        vnlbgpu::check(vnlbgpu::mlp_backward(net, x, batch, acts, logits, targets, tk, loss, dacts, gw, gb, stream),
                       "MLP backward");
        std::vector<float> l(static_cast<size_t>(batch));
        vnlbgpu::check(cudaMemcpyAsync(l.data(), loss, l.size() * sizeof(float), cudaMemcpyDeviceToHost, stream),
                       "cudaMemcpyAsync(loss)");
        vnlbgpu::check(cudaStreamSynchronize(stream), "cudaStreamSynchronize(MLP)");
        double s = 0.0;
        for (float v : l) s += v;
        return static_cast<float>(s / batch);
    }
};

namespace vnlbgpu {
MlpDevice mlp_device(const vnlbgpu_mlp* mlp) { return mlp->net; }
}  // namespace vnlbgpu

namespace {

template <typename Fn> int guarded_mlp(Fn&& fn) {
    try {
        fn();
        return 0;
    } catch (const std::exception& error) {
        vnlbgpu::set_last_error(error.what());
        return -1;
    }
}

}  // namespace

extern "C" {

int vnlbgpu_mlp_create(int inputs, int hidden, int layers, int outputs, int max_batch, unsigned seed, int device_id,
                       vnlbgpu_mlp** out) {
    return guarded_mlp([&]() {
        if (!out) throw std::invalid_argument("VNLB CUDA: null argument");
        if (inputs <= 0 || hidden <= 0 || outputs <= 0 || layers < 1 || layers > vnlbgpu::kMlpMaxLayers ||
            max_batch <= 0)
            throw std::invalid_argument("VNLB CUDA: the MLP needs positive sizes and 1..4 hidden layers");
        vnlbgpu::check(cudaSetDevice(device_id), "cudaSetDevice");
        auto m = std::make_unique<vnlbgpu_mlp>();
        m->device = device_id;
        m->inputs = inputs;
        m->hidden = hidden;
        m->layers = layers;
        m->outputs = outputs;
        m->max_batch = max_batch;
        m->net.inputs = inputs;
        m->net.hidden = hidden;
        m->net.layers = layers;
        m->net.outputs = outputs;
        vnlbgpu::check(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        std::mt19937 rng(seed);
        for (int l = 0; l <= layers; ++l) {
            const size_t nw = m->weights(l), nb = static_cast<size_t>(m->fan_out(l));
            m->w[l] = vnlbgpu::device_alloc<float>(nw, "cudaMalloc(MLP weights)");
            m->net.w16[l] = vnlbgpu::device_alloc<__nv_bfloat16>(nw, "cudaMalloc(MLP weights)");
            m->net.b[l] = vnlbgpu::device_alloc<float>(nb, "cudaMalloc(MLP biases)");
            m->gw[l] = vnlbgpu::device_alloc<float>(nw, "cudaMalloc(MLP gradients)");
            m->gb[l] = vnlbgpu::device_alloc<float>(nb, "cudaMalloc(MLP gradients)");
            m->mw[l] = vnlbgpu::device_alloc<float>(nw, "cudaMalloc(Adam moments)");
            m->vw[l] = vnlbgpu::device_alloc<float>(nw, "cudaMalloc(Adam moments)");
            m->mb[l] = vnlbgpu::device_alloc<float>(nb, "cudaMalloc(Adam moments)");
            m->vb[l] = vnlbgpu::device_alloc<float>(nb, "cudaMalloc(Adam moments)");
            // He initialisation for the ReLU layers, a smaller scale for the logits
            std::normal_distribution<float> dist(0.0f, std::sqrt((l == layers ? 1.0f : 2.0f) / m->fan_in(l)));
            std::vector<float> hw(nw), hb(nb, 0.0f);
            for (float& v : hw) v = dist(rng);
            vnlbgpu::check(cudaMemcpy(m->w[l], hw.data(), nw * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy");
            vnlbgpu::check(cudaMemcpy(m->net.b[l], hb.data(), nb * sizeof(float), cudaMemcpyHostToDevice),
                           "cudaMemcpy");
            for (float* p : {m->mw[l], m->vw[l]})
                vnlbgpu::check(cudaMemset(p, 0, nw * sizeof(float)), "cudaMemset");
            for (float* p : {m->mb[l], m->vb[l]})
                vnlbgpu::check(cudaMemset(p, 0, nb * sizeof(float)), "cudaMemset");
            vnlbgpu::check(vnlbgpu::weights_to_bf16(m->w[l], m->net.w16[l], nw, m->stream), "BF16 weights");
        }
        for (int l = 0; l < layers; ++l) {
            m->acts[l] = vnlbgpu::device_alloc<float>(static_cast<size_t>(max_batch) * hidden, "cudaMalloc(MLP)");
            m->dacts[l] = vnlbgpu::device_alloc<float>(static_cast<size_t>(max_batch) * hidden, "cudaMalloc(MLP)");
        }
        m->logits = vnlbgpu::device_alloc<float>(static_cast<size_t>(max_batch) * outputs, "cudaMalloc(MLP logits)");
        m->status = vnlbgpu::device_alloc<int>(1, "cudaMalloc(MLP status)");
        vnlbgpu::check(cudaMemset(m->status, 0, sizeof(int)), "cudaMemset(MLP status)");
        m->loss = vnlbgpu::device_alloc<float>(static_cast<size_t>(max_batch), "cudaMalloc(MLP loss)");
        vnlbgpu::check(cudaStreamSynchronize(m->stream), "cudaStreamSynchronize(MLP)");
        *out = m.release();
    });
}

void vnlbgpu_mlp_destroy(vnlbgpu_mlp* mlp) {
    if (!mlp) return;
    cudaSetDevice(mlp->device);
    delete mlp;
}

long long vnlbgpu_mlp_parameters(const vnlbgpu_mlp* mlp) { return mlp ? static_cast<long long>(mlp->parameters()) : 0; }

int vnlbgpu_mlp_get_weights(vnlbgpu_mlp* mlp, float* host) {
    return guarded_mlp([&]() {
        if (!mlp || !host) throw std::invalid_argument("VNLB CUDA: null argument");
        vnlbgpu::check(cudaSetDevice(mlp->device), "cudaSetDevice");
        vnlbgpu::check(cudaStreamSynchronize(mlp->stream), "cudaStreamSynchronize(MLP)");
        size_t off = 0;
        for (int l = 0; l <= mlp->layers; ++l) {
            vnlbgpu::check(cudaMemcpy(host + off, mlp->w[l], mlp->weights(l) * sizeof(float), cudaMemcpyDeviceToHost),
                           "cudaMemcpy(weights)");
            off += mlp->weights(l);
            vnlbgpu::check(cudaMemcpy(host + off, mlp->net.b[l], mlp->fan_out(l) * sizeof(float),
                                      cudaMemcpyDeviceToHost),
                           "cudaMemcpy(biases)");
            off += mlp->fan_out(l);
        }
    });
}

int vnlbgpu_mlp_set_weights(vnlbgpu_mlp* mlp, const float* host) {
    return guarded_mlp([&]() {
        if (!mlp || !host) throw std::invalid_argument("VNLB CUDA: null argument");
        vnlbgpu::check(cudaSetDevice(mlp->device), "cudaSetDevice");
        vnlbgpu::check(cudaStreamSynchronize(mlp->stream), "cudaStreamSynchronize(MLP)");
        size_t off = 0;
        for (int l = 0; l <= mlp->layers; ++l) {
            vnlbgpu::check(cudaMemcpy(mlp->w[l], host + off, mlp->weights(l) * sizeof(float), cudaMemcpyHostToDevice),
                           "cudaMemcpy(weights)");
            vnlbgpu::check(vnlbgpu::weights_to_bf16(mlp->w[l], mlp->net.w16[l], mlp->weights(l), mlp->stream),
                           "BF16 weights");
            off += mlp->weights(l);
            vnlbgpu::check(cudaMemcpy(mlp->net.b[l], host + off, mlp->fan_out(l) * sizeof(float),
                                      cudaMemcpyHostToDevice),
                           "cudaMemcpy(biases)");
            off += mlp->fan_out(l);
        }
        vnlbgpu::check(cudaStreamSynchronize(mlp->stream), "cudaStreamSynchronize(MLP)");
    });
}

int vnlbgpu_mlp_gradients(vnlbgpu_mlp* mlp, const float* x, const int* targets, int batch, int tk, float* host_grads,
                          float* mean_loss) {
    return guarded_mlp([&]() {
        if (!mlp || !x || !targets) throw std::invalid_argument("VNLB CUDA: null argument");
        vnlbgpu::check(cudaSetDevice(mlp->device), "cudaSetDevice");
        const float l = mlp->gradients(x, targets, batch, tk);
        if (mean_loss) *mean_loss = l;
        if (host_grads) {
            size_t off = 0;
            for (int k = 0; k <= mlp->layers; ++k) {
                vnlbgpu::check(cudaMemcpy(host_grads + off, mlp->gw[k], mlp->weights(k) * sizeof(float),
                                          cudaMemcpyDeviceToHost),
                               "cudaMemcpy(gradients)");
                off += mlp->weights(k);
                vnlbgpu::check(cudaMemcpy(host_grads + off, mlp->gb[k], mlp->fan_out(k) * sizeof(float),
                                          cudaMemcpyDeviceToHost),
                               "cudaMemcpy(gradients)");
                off += mlp->fan_out(k);
            }
        }
    });
}

int vnlbgpu_mlp_train_step(vnlbgpu_mlp* mlp, const float* x, const int* targets, int batch, int tk, float lr,
                           float* mean_loss) {
    return guarded_mlp([&]() {
        if (!mlp || !x || !targets) throw std::invalid_argument("VNLB CUDA: null argument");
        vnlbgpu::check(cudaSetDevice(mlp->device), "cudaSetDevice");
        const float l = mlp->gradients(x, targets, batch, tk);
        mlp->step += 1;
        vnlbgpu::check(vnlbgpu::mlp_adam(mlp->net, mlp->gw, mlp->gb, mlp->mw, mlp->vw, mlp->mb, mlp->vb, mlp->w, lr,
                                         mlp->step, mlp->stream),
                       "Adam");
        if (mean_loss) *mean_loss = l;
    });
}

int vnlbgpu_mlp_logits(vnlbgpu_mlp* mlp, const float* x, int batch, float* logits) {
    return guarded_mlp([&]() {
        if (!mlp || !x || !logits) throw std::invalid_argument("VNLB CUDA: null argument");
        vnlbgpu::check(cudaSetDevice(mlp->device), "cudaSetDevice");
        mlp->check_batch(batch);
        vnlbgpu::check(vnlbgpu::mlp_forward(mlp->net, x, batch, mlp->acts, logits, mlp->stream), "MLP forward");
        vnlbgpu::check(cudaStreamSynchronize(mlp->stream), "cudaStreamSynchronize(MLP)");
    });
}

int vnlbgpu_mlp_shortlist(vnlbgpu_mlp* mlp, const float* x, int batch, int k, int* out) {
    return guarded_mlp([&]() {
        if (!mlp || !x || !out) throw std::invalid_argument("VNLB CUDA: null argument");
        vnlbgpu::check(cudaSetDevice(mlp->device), "cudaSetDevice");
        if (k <= 0 || k > mlp->outputs) throw std::invalid_argument("VNLB CUDA: shortlist size out of range");
        for (int b0 = 0; b0 < batch; b0 += mlp->max_batch) {
            const int n = std::min(mlp->max_batch, batch - b0);
            vnlbgpu::check(vnlbgpu::mlp_infer(mlp->net, x + static_cast<size_t>(b0) * mlp->inputs, n, mlp->acts,
                                              mlp->logits, mlp->status, mlp->stream),
                           "MLP inference");
            vnlbgpu::check(vnlbgpu::logits_topk(mlp->logits, n, mlp->outputs, k, out + static_cast<size_t>(b0) * k,
                                                mlp->stream),
                           "shortlist");
        }
        int st = 0;
        vnlbgpu::check(cudaMemcpyAsync(&st, mlp->status, sizeof(int), cudaMemcpyDeviceToHost, mlp->stream),
                       "cudaMemcpyAsync(status)");
        vnlbgpu::check(cudaStreamSynchronize(mlp->stream), "cudaStreamSynchronize(MLP)");
        if (st != 0) {
            vnlbgpu::check(cudaMemset(mlp->status, 0, sizeof(int)), "cudaMemset(status)");
            throw std::runtime_error("VNLB CUDA: the network's tensor-core output layer timed out waiting for its MMAs");
        }
    });
}

}  // extern "C"
