// Learned per-partition variant selector.
//
// A small MLP (kMlpIn -> 64 -> 64 -> PC_NUM_VARIANTS, ReLU, fp32) predicts
// log(milliseconds) of every TC kernel variant on a planning unit from the
// unit's features.  Training data are timings the library measures itself
// (pc_selector_collect runs each feasible variant on each unit alone;
// pc_selector_collect_insitu runs each variant on all units at once and
// charges every unit its share of the run, measured by per-item cycle
// counters -- the cost that matters when the units share the GPU).  The
// network is trained on the GPU by the kernels below (forward, backward and
// Adam in one single-CTA launch per training run); inference also runs on the
// GPU.  The plain autotuned heuristic stays the fallback and the judge: the
// learned choice replaces the heuristic's only when the model is inside its
// training range and predicts a gain.  Either way every variant returns the
// exact count, so selection changes speed, never results.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>

#include "synth_rng.h"
#include "selector.cuh"

namespace pc {

// ---- features ----------------------------------------------------------------

void raw_to_features(const unsigned long long* r, float* f) {
    const double np = std::max<double>(1.0, (double)r[0]);
    const double mean_ld = (double)r[6] / 1024.0 / np;
    const double var_ld = std::max(0.0, (double)r[7] / 1024.0 / np - mean_ld * mean_ld);
    f[0] = (float)r[0];
    f[1] = (float)r[1];
    f[2] = (float)r[2];
    f[3] = (float)r[3];
    f[4] = (float)r[4];
    f[5] = (float)r[5];
    f[6] = (float)mean_ld;
    f[7] = (float)var_ld;
    f[8] = r[1] ? (float)((double)r[8] / (double)r[1]) : 0.f;
    f[9] = (float)((double)r[1] / np);
}

void features_to_inputs(const float* f, float* x) {
    const double ein = std::max(1.0, (double)f[1]);
    const double np = std::max(1.0, (double)f[0]);
    const double mean_scan = (double)f[5] / ein;
    const double mean_set = (double)f[2] / np;
    x[0] = (float)std::log1p((double)f[0]);
    x[1] = (float)std::log1p((double)f[1]);
    x[2] = (float)std::log1p((double)f[2]);
    x[3] = (float)std::log1p((double)f[3]);
    x[4] = (float)(std::log2(1.0 + (double)f[4]) / 32.0);
    x[5] = (float)std::log1p((double)f[5]);
    x[6] = f[6];
    x[7] = f[7];
    x[8] = f[8];
    x[9] = (float)std::log1p((double)f[9]);
    x[10] = (float)std::log1p(mean_scan);
    x[11] = (float)(std::log1p(mean_scan) - std::log1p(mean_set));  // neighbour-list length ratio
}

// ---- heuristic parameters ---------------------------------------------------------

static std::mutex g_mu;
static HeuristicParams g_hp;

HeuristicParams heuristic_params() {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_hp;
}
void bump_version_locked();
void set_heuristic_params(const HeuristicParams& hp) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_hp = hp;
    bump_version_locked();
}

// ---- MLP kernels ---------------------------------------------------------------
// Parameter layout (row-major, out x in): W1[H][In] b1[H] W2[H][H] b2[H]
// W3[Out][H] b3[Out].

constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kMlpOut * kMlpHidden;
static_assert(kOffB3 + kMlpOut == kMlpParams, "parameter layout");

constexpr int kTrainThreads = 256;
constexpr int kChunkS = 8;  // samples processed together

struct TrainSmem {
    float P[kMlpParams];
    float G[kMlpParams];
    float x[kChunkS][kMlpIn];
    float t[kChunkS][kMlpOut];
    float msk[kChunkS][kMlpOut];
    float w[kChunkS];
    float h1[kChunkS][kMlpHidden];
    float h2[kChunkS][kMlpHidden];
    float y[kChunkS][kMlpOut];
    float dy[kChunkS][kMlpOut];
    float dh2[kChunkS][kMlpHidden];
    float dh1[kChunkS][kMlpHidden];
    float lpart[kChunkS * kMlpOut];
    float loss;
};

// Full-batch training: `steps` iterations of forward, backward (mean squared
// error over masked outputs, each sample's terms weighted by W[s], 1 when W
// is null) and Adam.  With steps == 0 the kernel evaluates the loss and
// gradient at `params` (gradient check) without updating.
__global__ void __launch_bounds__(kTrainThreads) k_mlp_train(float* __restrict__ params, float* __restrict__ adam_m,
                                                             float* __restrict__ adam_v, const float* __restrict__ X,
                                                             const float* __restrict__ Y,
                                                             const uint8_t* __restrict__ M,
                                                             const float* __restrict__ W, int batch, float inv_count,
                                                             int steps, float lr, float* __restrict__ loss_out,
                                                             float* __restrict__ grad_out) {
    extern __shared__ float4 smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    const int tid = threadIdx.x;
    for (int i = tid; i < kMlpParams; i += blockDim.x) S.P[i] = params[i];
    const int iters = steps > 0 ? steps : 1;
    const float b1c = 0.9f, b2c = 0.999f, eps = 1e-8f;
    float b1t = 1.f, b2t = 1.f;
    for (int step = 0; step < iters; ++step) {
        for (int i = tid; i < kMlpParams; i += blockDim.x) S.G[i] = 0.f;
        if (tid == 0) S.loss = 0.f;
        __syncthreads();
        for (int c0 = 0; c0 < batch; c0 += kChunkS) {
            const int ns = min(kChunkS, batch - c0);
            for (int i = tid; i < kChunkS * kMlpIn; i += blockDim.x) {
                const int s = i / kMlpIn, k = i % kMlpIn;
                S.x[s][k] = s < ns ? X[(size_t)(c0 + s) * kMlpIn + k] : 0.f;
            }
            for (int i = tid; i < kChunkS * kMlpOut; i += blockDim.x) {
                const int s = i / kMlpOut, o = i % kMlpOut;
                S.t[s][o] = s < ns ? Y[(size_t)(c0 + s) * kMlpOut + o] : 0.f;
                S.msk[s][o] = (s < ns && M[(size_t)(c0 + s) * kMlpOut + o]) ? 1.f : 0.f;
            }
            for (int s = tid; s < kChunkS; s += blockDim.x) S.w[s] = s < ns ? (W ? W[c0 + s] : 1.f) : 0.f;
            __syncthreads();
            for (int i = tid; i < kChunkS * kMlpHidden; i += blockDim.x) {
                const int s = i / kMlpHidden, j = i % kMlpHidden;
                float z = S.P[kOffB1 + j];
                for (int k = 0; k < kMlpIn; ++k) z += S.P[kOffW1 + j * kMlpIn + k] * S.x[s][k];
                S.h1[s][j] = z > 0.f ? z : 0.f;
            }
            __syncthreads();
            for (int i = tid; i < kChunkS * kMlpHidden; i += blockDim.x) {
                const int s = i / kMlpHidden, j = i % kMlpHidden;
                float z = S.P[kOffB2 + j];
                for (int k = 0; k < kMlpHidden; ++k) z += S.P[kOffW2 + j * kMlpHidden + k] * S.h1[s][k];
                S.h2[s][j] = z > 0.f ? z : 0.f;
            }
            __syncthreads();
            for (int i = tid; i < kChunkS * kMlpOut; i += blockDim.x) {
                const int s = i / kMlpOut, o = i % kMlpOut;
                float z = S.P[kOffB3 + o];
                for (int k = 0; k < kMlpHidden; ++k) z += S.P[kOffW3 + o * kMlpHidden + k] * S.h2[s][k];
                S.y[s][o] = z;
                const float d = (z - S.t[s][o]) * S.msk[s][o];
                S.dy[s][o] = 2.f * S.w[s] * d * inv_count;
                S.lpart[i] = S.w[s] * d * d * inv_count;
            }
            __syncthreads();
            if (tid == 0) {
                float l = 0.f;
                for (int i = 0; i < kChunkS * kMlpOut; ++i) l += S.lpart[i];
                S.loss += l;
            }
            for (int i = tid; i < kMlpOut * kMlpHidden; i += blockDim.x) {
                const int o = i / kMlpHidden, k = i % kMlpHidden;
                float g = 0.f;
                for (int s = 0; s < kChunkS; ++s) g += S.dy[s][o] * S.h2[s][k];
                S.G[kOffW3 + i] += g;
            }
            if (tid < kMlpOut) {
                float g = 0.f;
                for (int s = 0; s < kChunkS; ++s) g += S.dy[s][tid];
                S.G[kOffB3 + tid] += g;
            }
            for (int i = tid; i < kChunkS * kMlpHidden; i += blockDim.x) {
                const int s = i / kMlpHidden, k = i % kMlpHidden;
                float g = 0.f;
                for (int o = 0; o < kMlpOut; ++o) g += S.P[kOffW3 + o * kMlpHidden + k] * S.dy[s][o];
                S.dh2[s][k] = S.h2[s][k] > 0.f ? g : 0.f;
            }
            __syncthreads();
            for (int i = tid; i < kMlpHidden * kMlpHidden; i += blockDim.x) {
                const int j = i / kMlpHidden, k = i % kMlpHidden;
                float g = 0.f;
                for (int s = 0; s < kChunkS; ++s) g += S.dh2[s][j] * S.h1[s][k];
                S.G[kOffW2 + i] += g;
            }
            if (tid < kMlpHidden) {
                float g = 0.f;
                for (int s = 0; s < kChunkS; ++s) g += S.dh2[s][tid];
                S.G[kOffB2 + tid] += g;
            }
            for (int i = tid; i < kChunkS * kMlpHidden; i += blockDim.x) {
                const int s = i / kMlpHidden, k = i % kMlpHidden;
                float g = 0.f;
                for (int j = 0; j < kMlpHidden; ++j) g += S.P[kOffW2 + j * kMlpHidden + k] * S.dh2[s][j];
                S.dh1[s][k] = S.h1[s][k] > 0.f ? g : 0.f;
            }
            __syncthreads();
            for (int i = tid; i < kMlpHidden * kMlpIn; i += blockDim.x) {
                const int j = i / kMlpIn, k = i % kMlpIn;
                float g = 0.f;
                for (int s = 0; s < kChunkS; ++s) g += S.dh1[s][j] * S.x[s][k];
                S.G[kOffW1 + i] += g;
            }
            if (tid < kMlpHidden) {
                float g = 0.f;
                for (int s = 0; s < kChunkS; ++s) g += S.dh1[s][tid];
                S.G[kOffB1 + tid] += g;
            }
            __syncthreads();
        }
        if (steps > 0) {
            b1t *= b1c;
            b2t *= b2c;
            for (int i = tid; i < kMlpParams; i += blockDim.x) {
                const float g = S.G[i];
                const float m = b1c * adam_m[i] + (1.f - b1c) * g;
                const float v = b2c * adam_v[i] + (1.f - b2c) * g * g;
                adam_m[i] = m;
                adam_v[i] = v;
                const float mh = m / (1.f - b1t), vh = v / (1.f - b2t);
                S.P[i] -= lr * mh / (sqrtf(vh) + eps);
            }
        }
        __syncthreads();
    }
    for (int i = tid; i < kMlpParams; i += blockDim.x) {
        params[i] = S.P[i];
        if (grad_out) grad_out[i] = S.G[i];
    }
    if (tid == 0 && loss_out) *loss_out = S.loss;
}

// Inference: one CTA of kMlpHidden threads per sample.
__global__ void k_mlp_forward(const float* __restrict__ params, const float* __restrict__ X, int batch,
                              float* __restrict__ Yout) {
    __shared__ float x[kMlpIn], h1[kMlpHidden], h2[kMlpHidden];
    const int s = blockIdx.x, j = threadIdx.x;
    if (s >= batch) return;
    if (j < kMlpIn) x[j] = X[(size_t)s * kMlpIn + j];
    __syncthreads();
    float z = params[kOffB1 + j];
    for (int k = 0; k < kMlpIn; ++k) z += params[kOffW1 + j * kMlpIn + k] * x[k];
    h1[j] = z > 0.f ? z : 0.f;
    __syncthreads();
    z = params[kOffB2 + j];
    for (int k = 0; k < kMlpHidden; ++k) z += params[kOffW2 + j * kMlpHidden + k] * h1[k];
    h2[j] = z > 0.f ? z : 0.f;
    __syncthreads();
    if (j < kMlpOut) {
        z = params[kOffB3 + j];
        for (int k = 0; k < kMlpHidden; ++k) z += params[kOffW3 + j * kMlpHidden + k] * h2[k];
        Yout[(size_t)s * kMlpOut + j] = z;
    }
}

// ---- model state -----------------------------------------------------------------

struct Model {
    bool trained = false;
    bool enabled = true;
    std::vector<float> params;       // kMlpParams
    float mean[kMlpIn] = {0}, stdv[kMlpIn] = {0};
    float lo[kMlpIn] = {0}, hi[kMlpIn] = {0};  // training range (standardised)
    // The judge: the learned choice replaces the heuristic's only when it is
    // predicted faster by more than this (log ratio).  Chosen by
    // leave-one-group-out validation at training; +inf keeps the heuristic.
    float judge_log_margin = 0.0487902f;  // log(1.05) until validated
    double heldout_gain = 0.0;            // plain / judged cost on held-out groups (0: not validated)
    // samples
    std::vector<float> feats;   // kNumFeatures per sample (raw)
    std::vector<float> logms;   // kMlpOut per sample
    std::vector<uint8_t> mask;  // kMlpOut per sample
    std::vector<int32_t> group; // one id per collection call (validation folds)
    int32_t next_group = 0;
};

// Per-sample work scale: the model predicts log(ms) - log(1 + in-edges +
// prefix ids), the cost per unit of work, so units of other sizes than the
// training units stay comparable.  It cancels in the per-unit argmin.
static float log_work(const float* f) { return (float)std::log(1.0 + (double)f[1] + (double)f[5]); }
static Model g_model;

static size_t train_smem_bytes() { return sizeof(TrainSmem) + 16; }

// Runs the training kernel on the current device.
static pc_status run_train_kernel(std::vector<float>& params, const std::vector<float>& X, const std::vector<float>& Y,
                                  const std::vector<uint8_t>& M, const std::vector<float>* W, int batch, int steps,
                                  float lr, float* loss, std::vector<float>* grad) {
    size_t cnt = 0;
    for (int i = 0; i < batch * kMlpOut; ++i) cnt += M[i] ? 1 : 0;
    if (cnt == 0) return fail(PC_ERR_INVALID_INPUT, "no masked targets to train on");
    DevBuf dP, dm, dv, dX, dY, dM, dW, dL, dG;
    PC_TRY(dP.alloc(kMlpParams * 4, "mlp params"));
    PC_TRY(dm.alloc(kMlpParams * 4, "adam m"));
    PC_TRY(dv.alloc(kMlpParams * 4, "adam v"));
    PC_TRY(dX.alloc((size_t)batch * kMlpIn * 4, "mlp inputs"));
    PC_TRY(dY.alloc((size_t)batch * kMlpOut * 4, "mlp targets"));
    PC_TRY(dM.alloc((size_t)batch * kMlpOut, "mlp mask"));
    PC_TRY(dL.alloc(4, "mlp loss"));
    PC_TRY(dG.alloc(kMlpParams * 4, "mlp grad"));
    PC_CUDA(cudaMemcpy(dP.p, params.data(), kMlpParams * 4, cudaMemcpyHostToDevice));
    PC_CUDA(cudaMemset(dm.p, 0, kMlpParams * 4));
    PC_CUDA(cudaMemset(dv.p, 0, kMlpParams * 4));
    PC_CUDA(cudaMemcpy(dX.p, X.data(), (size_t)batch * kMlpIn * 4, cudaMemcpyHostToDevice));
    PC_CUDA(cudaMemcpy(dY.p, Y.data(), (size_t)batch * kMlpOut * 4, cudaMemcpyHostToDevice));
    PC_CUDA(cudaMemcpy(dM.p, M.data(), (size_t)batch * kMlpOut, cudaMemcpyHostToDevice));
    if (W) {
        PC_TRY(dW.alloc((size_t)batch * 4, "mlp sample weights"));
        PC_CUDA(cudaMemcpy(dW.p, W->data(), (size_t)batch * 4, cudaMemcpyHostToDevice));
    }
    const size_t smem = train_smem_bytes();
    PC_CUDA(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_mlp_train<<<1, kTrainThreads, smem>>>(dP.as<float>(), dm.as<float>(), dv.as<float>(), dX.as<float>(),
                                            dY.as<float>(), dM.as<uint8_t>(), W ? dW.as<float>() : nullptr, batch,
                                            1.0f / (float)cnt, steps, lr,
                                            dL.as<float>(), dG.as<float>());
    PC_LAUNCHED();
    PC_CUDA(cudaDeviceSynchronize());
    PC_CUDA(cudaMemcpy(params.data(), dP.p, kMlpParams * 4, cudaMemcpyDeviceToHost));
    if (loss) PC_CUDA(cudaMemcpy(loss, dL.p, 4, cudaMemcpyDeviceToHost));
    if (grad) {
        grad->resize(kMlpParams);
        PC_CUDA(cudaMemcpy(grad->data(), dG.p, kMlpParams * 4, cudaMemcpyDeviceToHost));
    }
    return PC_OK;
}

static pc_status run_forward(const std::vector<float>& params, const float* X, int batch, float* Y) {
    if (batch <= 0) return PC_OK;
    DevBuf dP, dX, dY;
    PC_TRY(dP.alloc(kMlpParams * 4, "mlp params"));
    PC_TRY(dX.alloc((size_t)batch * kMlpIn * 4, "mlp inputs"));
    PC_TRY(dY.alloc((size_t)batch * kMlpOut * 4, "mlp outputs"));
    PC_CUDA(cudaMemcpy(dP.p, params.data(), kMlpParams * 4, cudaMemcpyHostToDevice));
    PC_CUDA(cudaMemcpy(dX.p, X, (size_t)batch * kMlpIn * 4, cudaMemcpyHostToDevice));
    k_mlp_forward<<<batch, kMlpHidden>>>(dP.as<float>(), dX.as<float>(), batch, dY.as<float>());
    PC_LAUNCHED();
    PC_CUDA(cudaMemcpy(Y, dY.p, (size_t)batch * kMlpOut * 4, cudaMemcpyDeviceToHost));
    return PC_OK;
}

static void standardise(const Model& md, const float* raw, float* x) {
    float in[kMlpIn];
    features_to_inputs(raw, in);
    for (int k = 0; k < kMlpIn; ++k) x[k] = (in[k] - md.mean[k]) / md.stdv[k];
}

static uint64_t g_version = 1;

bool selector_ready(int) {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_model.trained && g_model.enabled;
}

uint64_t selector_version() {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_version;
}

void bump_version_locked() { ++g_version; }

// Learned choices, judged against the heuristic: for a unit the model must be
// inside its training range (with a margin) and predict the heuristic's
// choice slower than its own by more than the validated judge margin;
// otherwise the heuristic's choice stands.  (The per-unit work scale of the
// predictions cancels in these comparisons.)
pc_status selector_choose_batch(const std::vector<float>& feat, size_t U, std::vector<int8_t>* choice) {
    Model md;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_model.trained) return fail(PC_ERR_UNSUPPORTED, "the selector is not trained");
        md.params = g_model.params;
        memcpy(md.mean, g_model.mean, sizeof(md.mean));
        memcpy(md.stdv, g_model.stdv, sizeof(md.stdv));
        memcpy(md.lo, g_model.lo, sizeof(md.lo));
        memcpy(md.hi, g_model.hi, sizeof(md.hi));
        md.judge_log_margin = g_model.judge_log_margin;
    }
    const HeuristicParams hp = heuristic_params();
    choice->assign(U, -1);
    const bool use_model = std::isfinite(md.judge_log_margin);  // +inf: validation kept the heuristic
    std::vector<size_t> idx;
    std::vector<float> X;
    for (size_t u = 0; u < U; ++u) {
        const float* f = &feat[u * kNumFeatures];
        const int h = tc::heuristic_choice(f, hp);
        (*choice)[u] = (int8_t)h;
        if (h < 0) continue;
        float x[kMlpIn];
        standardise(md, f, x);
        bool inside = true;
        for (int k = 0; k < kMlpIn; ++k) {
            const float span = md.hi[k] - md.lo[k];
            if (x[k] < md.lo[k] - 0.25f * span - 0.5f || x[k] > md.hi[k] + 0.25f * span + 0.5f) inside = false;
        }
        if (!inside || !use_model) continue;
        idx.push_back(u);
        X.insert(X.end(), x, x + kMlpIn);
    }
    if (idx.empty()) return PC_OK;
    std::vector<float> Y(idx.size() * kMlpOut);
    PC_TRY(run_forward(md.params, X.data(), (int)idx.size(), Y.data()));
    for (size_t i = 0; i < idx.size(); ++i) {
        const size_t u = idx[i];
        const float* f = &feat[u * kNumFeatures];
        const float* y = &Y[i * kMlpOut];
        const int h = (*choice)[u];
        int best = -1;
        for (int v = 0; v < kMlpOut; ++v)
            if (tc::variant_feasible(v, f) && (best < 0 || y[v] < y[best])) best = v;
        if (best >= 0 && y[h] - y[best] > md.judge_log_margin) (*choice)[u] = (int8_t)best;
    }
    return PC_OK;
}

}  // namespace pc

using namespace pc;

extern "C" {

int32_t pc_mlp_num_params(void) { return kMlpParams; }

pc_status pc_mlp_forward(const float* params, const float* x, int32_t batch, float* y) {
    clear_error();
    if (!params || !x || !y || batch < 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    if (pc_device_count() == 0) return fail(PC_ERR_NO_DEVICE, "no CUDA device is visible");
    std::vector<float> p(params, params + kMlpParams);
    return run_forward(p, x, batch, y);
}

pc_status pc_mlp_loss_grad(const float* params, const float* x, const float* y, const uint8_t* mask, int32_t batch,
                           float* loss, float* grad) {
    return pc_mlp_loss_grad_weighted(params, x, y, mask, nullptr, batch, loss, grad);
}

pc_status pc_mlp_loss_grad_weighted(const float* params, const float* x, const float* y, const uint8_t* mask,
                                    const float* weights, int32_t batch, float* loss, float* grad) {
    clear_error();
    if (!params || !x || !y || !mask || batch <= 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    if (pc_device_count() == 0) return fail(PC_ERR_NO_DEVICE, "no CUDA device is visible");
    std::vector<float> p(params, params + kMlpParams);
    std::vector<float> X(x, x + (size_t)batch * kMlpIn), Y(y, y + (size_t)batch * kMlpOut);
    std::vector<uint8_t> M(mask, mask + (size_t)batch * kMlpOut);
    std::vector<float> W;
    if (weights) W.assign(weights, weights + batch);
    std::vector<float> g;
    PC_TRY(run_train_kernel(p, X, Y, M, weights ? &W : nullptr, batch, 0, 0.f, loss, &g));
    if (grad) memcpy(grad, g.data(), kMlpParams * 4);
    return PC_OK;
}

pc_status pc_mlp_train_steps(float* params, const float* x, const float* y, const uint8_t* mask, int32_t batch,
                             int32_t steps, float lr, float* final_loss) {
    clear_error();
    if (!params || !x || !y || !mask || batch <= 0 || steps <= 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    if (pc_device_count() == 0) return fail(PC_ERR_NO_DEVICE, "no CUDA device is visible");
    std::vector<float> p(params, params + kMlpParams);
    std::vector<float> X(x, x + (size_t)batch * kMlpIn), Y(y, y + (size_t)batch * kMlpOut);
    std::vector<uint8_t> M(mask, mask + (size_t)batch * kMlpOut);
    PC_TRY(run_train_kernel(p, X, Y, M, nullptr, batch, steps, lr, final_loss, nullptr));
    memcpy(params, p.data(), kMlpParams * 4);
    return PC_OK;
}

pc_status pc_tc_units(pc_pgraph* pg, int32_t* nunits) {
    clear_error();
    if (!pg || !nunits) return fail(PC_ERR_INVALID_INPUT, "null argument");
    PC_TRY(use_device(pg->g));
    PC_TRY(tc_ensure_features(pg));
    *nunits = (int32_t)pg->unit_lo.size();
    return PC_OK;
}

pc_status pc_tc_unit_features(pc_pgraph* pg, float* feats, int32_t cap) {
    clear_error();
    if (!pg || !feats) return fail(PC_ERR_INVALID_INPUT, "null argument");
    PC_TRY(use_device(pg->g));
    PC_TRY(tc_ensure_features(pg));
    const size_t U = pg->unit_lo.size();
    if ((size_t)cap < U) return fail(PC_ERR_INVALID_INPUT, "feature buffer too small");
    memcpy(feats, pg->part_features.data(), U * kNumFeatures * sizeof(float));
    return PC_OK;
}

pc_status pc_tc_plan(pc_pgraph* pg, int32_t variant, int8_t* assign, int32_t cap) {
    clear_error();
    if (!pg || !assign) return fail(PC_ERR_INVALID_INPUT, "null argument");
    PC_TRY(use_device(pg->g));
    PC_TRY(tc_ensure_features(pg));
    const size_t U = pg->unit_lo.size();
    if ((size_t)cap < U) return fail(PC_ERR_INVALID_INPUT, "plan buffer too small");
    std::vector<int8_t> a;
    int sel = 0;
    PC_TRY(tc_assign(pg, variant, pg->part_features, U, &a, &sel));
    memcpy(assign, a.data(), U);
    return PC_OK;
}

pc_status pc_tc_time_unit(pc_pgraph* pg, int32_t unit, int32_t variant, double* ms, uint64_t* count) {
    clear_error();
    if (!pg || !ms || !count || unit < 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    if (variant < 0 || variant >= PC_NUM_VARIANTS) return fail(PC_ERR_INVALID_INPUT, "unknown variant");
    PC_TRY(use_device(pg->g));
    PC_TRY(tc_ensure_features(pg));
    if ((size_t)unit >= pg->unit_lo.size()) return fail(PC_ERR_INVALID_INPUT, "unit index out of range");
    if (!tc::variant_feasible(variant, &pg->part_features[(size_t)unit * kNumFeatures]))
        return fail(PC_ERR_UNSUPPORTED, "variant not feasible on this unit");
    return tc_time_unit(pg, (size_t)unit, variant, ms, count);
}

pc_status pc_selector_collect(pc_pgraph* pg, int32_t max_units, int32_t repeats, int32_t* added) {
    clear_error();
    if (!pg || max_units <= 0 || repeats <= 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    PC_TRY(use_device(pg->g));
    PC_TRY(tc_ensure_features(pg));
    const size_t U = pg->unit_lo.size();
    std::vector<size_t> work;
    for (size_t u = 0; u < U; ++u) {
        const float* f = &pg->part_features[u * kNumFeatures];
        if (f[1] > 0 && f[2] > 0) work.push_back(u);
    }
    // heaviest units first, then an even stride over the rest
    std::sort(work.begin(), work.end(), [&](size_t a, size_t b) {
        return pg->part_features[a * kNumFeatures + 5] > pg->part_features[b * kNumFeatures + 5];
    });
    std::vector<size_t> pick;
    if ((int32_t)work.size() <= max_units) {
        pick = work;
    } else {
        const size_t head = (size_t)max_units / 2;
        for (size_t i = 0; i < head; ++i) pick.push_back(work[i]);
        const size_t rest = work.size() - head, want = (size_t)max_units - head;
        for (size_t i = 0; i < want; ++i) pick.push_back(work[head + i * rest / want]);
    }
    int32_t n_added = 0;
    int32_t gid = -1;
    for (size_t u : pick) {
        const float* f = &pg->part_features[u * kNumFeatures];
        float logms[kMlpOut];
        uint8_t msk[kMlpOut];
        uint64_t ref = 0;
        bool have_ref = false;
        for (int v = 0; v < kMlpOut; ++v) {
            msk[v] = 0;
            logms[v] = 0.f;
            if (!tc::variant_feasible(v, f)) continue;
            double best = 1e30;
            for (int r = 0; r < repeats; ++r) {
                double ms = 0;
                uint64_t c = 0;
                PC_TRY(tc_time_unit(pg, u, v, &ms, &c));
                if (!have_ref) { ref = c; have_ref = true; }
                if (c != ref) {
                    char buf[160];
                    snprintf(buf, sizeof(buf), "variant %d counted %llu on unit %zu, expected %llu", v,
                             (unsigned long long)c, u, (unsigned long long)ref);
                    return fail(PC_ERR_CUDA, buf);
                }
                best = std::min(best, ms);
            }
            logms[v] = (float)std::log(std::max(best, 1e-4));
            msk[v] = 1;
        }
        std::lock_guard<std::mutex> lk(g_mu);
        if (gid < 0) gid = g_model.next_group++;
        g_model.feats.insert(g_model.feats.end(), f, f + kNumFeatures);
        g_model.logms.insert(g_model.logms.end(), logms, logms + kMlpOut);
        g_model.mask.insert(g_model.mask.end(), msk, msk + kMlpOut);
        g_model.group.push_back(gid);
        ++n_added;
    }
    if (added) *added = n_added;
    return PC_OK;
}

pc_status pc_selector_collect_insitu(pc_pgraph* pg, int32_t repeats, int32_t* added) {
    clear_error();
    if (!pg || repeats <= 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    PC_TRY(use_device(pg->g));
    PC_TRY(tc_ensure_features(pg));
    const size_t U = pg->unit_lo.size();
    std::vector<std::vector<double>> best(kMlpOut, std::vector<double>(U, 1e30));
    // counts agree among the variants that ran on the same units: the bitmap
    // variants (ids within the bitmap), the matrix form (ids below 2^16) and
    // the others (every unit with work)
    uint64_t ref[3] = {0, 0, 0};
    bool have[3] = {false, false, false};
    for (int v = 0; v < kMlpOut; ++v) {
        const int cls = v == PC_VARIANT_MATRIX ? 2
                         : (v == PC_VARIANT_BITMAP_WARP || v == PC_VARIANT_BITMAP_GROUP8 || v == PC_VARIANT_BITMAP_LANE)
                               ? 1
                               : 0;
        for (int r = 0; r < repeats; ++r) {
            std::vector<double> ms;
            uint64_t c = 0;
            PC_TRY(tc_profile_variant(pg, v, &ms, &c));
            if (!have[cls]) { ref[cls] = c; have[cls] = true; }
            if (c != ref[cls]) {
                char buf[160];
                snprintf(buf, sizeof(buf), "variant %d counted %llu in a profiling run, expected %llu", v,
                         (unsigned long long)c, (unsigned long long)ref[cls]);
                return fail(PC_ERR_CUDA, buf);
            }
            for (size_t u = 0; u < U; ++u)
                if (ms[u] >= 0) best[v][u] = std::min(best[v][u], ms[u]);
        }
    }
    int32_t n_added = 0;
    std::lock_guard<std::mutex> lk(g_mu);
    const int32_t gid = g_model.next_group++;
    for (size_t u = 0; u < U; ++u) {
        const float* f = &pg->part_features[u * kNumFeatures];
        if (!(f[1] > 0 && f[2] > 0)) continue;
        float logms[kMlpOut];
        uint8_t msk[kMlpOut];
        for (int v = 0; v < kMlpOut; ++v) {
            msk[v] = best[v][u] < 1e29 ? 1 : 0;
            logms[v] = msk[v] ? (float)std::log(std::max(best[v][u], 1e-6)) : 0.f;
        }
        g_model.feats.insert(g_model.feats.end(), f, f + kNumFeatures);
        g_model.logms.insert(g_model.logms.end(), logms, logms + kMlpOut);
        g_model.mask.insert(g_model.mask.end(), msk, msk + kMlpOut);
        g_model.group.push_back(gid);
        ++n_added;
    }
    if (added) *added = n_added;
    return PC_OK;
}

int32_t pc_selector_num_samples(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    return (int32_t)(g_model.feats.size() / kNumFeatures);
}

pc_status pc_selector_get_samples(float* feats, float* log_ms, uint8_t* mask, int32_t cap) {
    clear_error();
    std::lock_guard<std::mutex> lk(g_mu);
    const size_t n = g_model.feats.size() / kNumFeatures;
    if ((size_t)cap < n) return fail(PC_ERR_INVALID_INPUT, "buffer too small");
    if (feats) memcpy(feats, g_model.feats.data(), n * kNumFeatures * 4);
    if (log_ms) memcpy(log_ms, g_model.logms.data(), n * kMlpOut * 4);
    if (mask) memcpy(mask, g_model.mask.data(), n * kMlpOut);
    return PC_OK;
}

pc_status pc_selector_add_samples(const float* feats, const float* log_ms, const uint8_t* mask, int32_t count) {
    clear_error();
    if (!feats || !log_ms || !mask || count < 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    std::lock_guard<std::mutex> lk(g_mu);
    g_model.feats.insert(g_model.feats.end(), feats, feats + (size_t)count * kNumFeatures);
    g_model.logms.insert(g_model.logms.end(), log_ms, log_ms + (size_t)count * kMlpOut);
    g_model.mask.insert(g_model.mask.end(), mask, mask + (size_t)count * kMlpOut);
    g_model.group.insert(g_model.group.end(), (size_t)count, g_model.next_group++);
    return PC_OK;
}

pc_status pc_selector_clear(void) {
    clear_error();
    std::lock_guard<std::mutex> lk(g_mu);
    g_model = Model();
    bump_version_locked();
    return PC_OK;
}

int32_t pc_selector_trained(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_model.trained ? 1 : 0;
}

pc_status pc_selector_enable(int32_t on) {
    clear_error();
    std::lock_guard<std::mutex> lk(g_mu);
    g_model.enabled = on != 0;
    bump_version_locked();
    return PC_OK;
}

}  // extern "C"

namespace pc {

// Fits a model to the samples idx of `data` (standardisation, He-uniform
// initialisation from the counter-based generator, full-batch Adam on the GPU).
// Each sample's squared errors are weighted by the measured time of its
// unit's fastest variant (normalised to mean 1 over the fit): the quantity
// the selector minimises is the summed time, so the few units that hold most
// of it -- the hub units, a handful among hundreds -- must be predicted
// well, not just the many light ones.
static pc_status fit_model(const Model& data, const std::vector<size_t>& idx, int32_t steps, float lr, uint64_t seed,
                           Model* md, float* loss) {
    const int n = (int)idx.size();
    std::vector<float> X((size_t)n * kMlpIn), Y((size_t)n * kMlpOut), W((size_t)n, 1.f);
    std::vector<uint8_t> M((size_t)n * kMlpOut);
    double wsum = 0.0;
    for (int i = 0; i < n; ++i) {
        const float* f = &data.feats[idx[i] * kNumFeatures];
        features_to_inputs(f, &X[(size_t)i * kMlpIn]);
        const float lw = log_work(f);
        float best = INFINITY;
        for (int o = 0; o < kMlpOut; ++o) {
            const float lm = data.logms[idx[i] * kMlpOut + o];
            const uint8_t mk = data.mask[idx[i] * kMlpOut + o];
            Y[(size_t)i * kMlpOut + o] = lm - lw;
            M[(size_t)i * kMlpOut + o] = mk;
            if (mk) best = std::min(best, lm);
        }
        W[i] = std::isfinite(best) ? (float)std::exp((double)best) : 0.f;
        wsum += W[i];
    }
    if (wsum > 0.0)
        for (int i = 0; i < n; ++i) W[i] = (float)(W[i] * n / wsum);
    else
        std::fill(W.begin(), W.end(), 1.f);
    for (int k = 0; k < kMlpIn; ++k) {
        double m = 0, v = 0;
        for (int i = 0; i < n; ++i) m += X[(size_t)i * kMlpIn + k];
        m /= n;
        for (int i = 0; i < n; ++i) v += (X[(size_t)i * kMlpIn + k] - m) * (X[(size_t)i * kMlpIn + k] - m);
        v /= n;
        md->mean[k] = (float)m;
        md->stdv[k] = (float)std::max(1e-3, std::sqrt(v));
        md->lo[k] = 1e30f;
        md->hi[k] = -1e30f;
        for (int i = 0; i < n; ++i) {
            float& z = X[(size_t)i * kMlpIn + k];
            z = (z - md->mean[k]) / md->stdv[k];
            md->lo[k] = std::min(md->lo[k], z);
            md->hi[k] = std::max(md->hi[k], z);
        }
    }
    md->params.assign(kMlpParams, 0.f);
    const uint64_t key = pc_graph_key(seed, 99);
    auto init = [&](int off, int fan_in, int count) {
        const double a = std::sqrt(6.0 / fan_in);
        for (int i = 0; i < count; ++i) {
            const double u = (double)(pc_draw(key, (uint64_t)(off + i)) >> 11) * (1.0 / 9007199254740992.0);
            md->params[off + i] = (float)((2.0 * u - 1.0) * a);
        }
    };
    init(kOffW1, kMlpIn, kMlpHidden * kMlpIn);
    init(kOffW2, kMlpHidden, kMlpHidden * kMlpHidden);
    init(kOffW3, kMlpHidden, kMlpOut * kMlpHidden);
    return run_train_kernel(md->params, X, Y, M, &W, n, steps, lr, loss, nullptr);
}

// Predicted log(ms) per variant for the samples idx of `data` under model md.
static pc_status predict_samples(const Model& md, const Model& data, const std::vector<size_t>& idx,
                                 std::vector<float>* out) {
    const int n = (int)idx.size();
    std::vector<float> X((size_t)n * kMlpIn);
    for (int i = 0; i < n; ++i) standardise(md, &data.feats[idx[i] * kNumFeatures], &X[(size_t)i * kMlpIn]);
    out->assign((size_t)n * kMlpOut, 0.f);
    PC_TRY(run_forward(md.params, X.data(), n, out->data()));
    for (int i = 0; i < n; ++i) {
        const float lw = log_work(&data.feats[idx[i] * kNumFeatures]);
        for (int o = 0; o < kMlpOut; ++o) (*out)[(size_t)i * kMlpOut + o] += lw;
    }
    return PC_OK;
}

}  // namespace pc

extern "C" {

pc_status pc_selector_train(int32_t steps, float lr, uint64_t seed, float* final_loss) {
    clear_error();
    if (steps <= 0 || !(lr > 0.f)) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    if (pc_device_count() == 0) return fail(PC_ERR_NO_DEVICE, "no CUDA device is visible");
    Model data;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        data.feats = g_model.feats;
        data.logms = g_model.logms;
        data.mask = g_model.mask;
        data.group = g_model.group;
    }
    const size_t n = data.feats.size() / kNumFeatures;
    if (n < 2) return fail(PC_ERR_INVALID_INPUT, "collect at least two samples before training");
    const HeuristicParams hp = heuristic_params();
    // Judge margin by leave-one-group-out validation: for every collection
    // group, a model fitted on the other groups plans the held-out units;
    // the margin that gives the lowest measured total over all held-out
    // units wins, +inf (keep the heuristic) when none beats the heuristic.
    const float margins[] = {0.0f, 0.0487902f, 0.0953102f, 0.1823216f, 0.3364722f, INFINITY};
    constexpr int kM = sizeof(margins) / sizeof(margins[0]);
    double cost[kM] = {0};
    std::vector<int32_t> gids(data.group.begin(), data.group.end());
    std::sort(gids.begin(), gids.end());
    gids.erase(std::unique(gids.begin(), gids.end()), gids.end());
    bool validated = false;
    if (gids.size() >= 2) {
        for (int32_t g : gids) {
            std::vector<size_t> tr, te;
            for (size_t i = 0; i < n; ++i) (data.group[i] == g ? te : tr).push_back(i);
            if (tr.size() < 2 || te.empty()) continue;
            Model md;
            PC_TRY(fit_model(data, tr, steps, lr, seed, &md, nullptr));
            std::vector<float> Y;
            PC_TRY(predict_samples(md, data, te, &Y));
            for (size_t i = 0; i < te.size(); ++i) {
                const size_t sidx = te[i];
                const float* f = &data.feats[sidx * kNumFeatures];
                const float* meas = &data.logms[sidx * kMlpOut];
                const uint8_t* msk = &data.mask[sidx * kMlpOut];
                const int h = tc::heuristic_choice(f, hp);
                if (h < 0 || !msk[h]) continue;
                float x[kMlpIn];
                standardise(md, f, x);
                bool inside = true;
                for (int k = 0; k < kMlpIn; ++k) {
                    const float span = md.hi[k] - md.lo[k];
                    if (x[k] < md.lo[k] - 0.25f * span - 0.5f || x[k] > md.hi[k] + 0.25f * span + 0.5f) inside = false;
                }
                const float* y = &Y[i * kMlpOut];
                int best = -1;
                for (int v = 0; v < kMlpOut; ++v)
                    if (tc::variant_feasible(v, f) && msk[v] && (best < 0 || y[v] < y[best])) best = v;
                for (int k = 0; k < kM; ++k) {
                    const int c = (inside && best >= 0 && y[h] - y[best] > margins[k]) ? best : h;
                    cost[k] += std::exp((double)meas[c]);
                }
            }
            validated = true;
        }
    }
    int pick = validated ? kM - 1 : 1;  // unvalidated: the default 5 % margin
    if (validated)
        for (int k = kM - 2; k >= 0; --k)
            if (cost[k] < cost[pick] * 0.999) pick = k;
    std::vector<size_t> all(n);
    for (size_t i = 0; i < n; ++i) all[i] = i;
    Model md;
    float loss = 0.f;
    PC_TRY(fit_model(data, all, steps, lr, seed, &md, &loss));
    if (final_loss) *final_loss = loss;
    std::lock_guard<std::mutex> lk(g_mu);
    g_model.params = md.params;
    memcpy(g_model.mean, md.mean, sizeof(md.mean));
    memcpy(g_model.stdv, md.stdv, sizeof(md.stdv));
    memcpy(g_model.lo, md.lo, sizeof(md.lo));
    memcpy(g_model.hi, md.hi, sizeof(md.hi));
    g_model.judge_log_margin = margins[pick];
    g_model.heldout_gain = validated && cost[pick] > 0 ? cost[kM - 1] / cost[pick] : 0.0;
    g_model.trained = true;
    bump_version_locked();
    return PC_OK;
}

pc_status pc_selector_judge(double* log_margin, double* heldout_gain) {
    clear_error();
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_model.trained) return fail(PC_ERR_UNSUPPORTED, "the selector is not trained");
    if (log_margin) *log_margin = g_model.judge_log_margin;
    if (heldout_gain) *heldout_gain = g_model.heldout_gain;
    return PC_OK;
}

pc_status pc_selector_predict(const float* feats, int32_t count, float* log_ms) {
    clear_error();
    if (!feats || !log_ms || count < 0) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    Model md;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_model.trained) return fail(PC_ERR_UNSUPPORTED, "the selector is not trained");
        md.params = g_model.params;
        memcpy(md.mean, g_model.mean, sizeof(md.mean));
        memcpy(md.stdv, g_model.stdv, sizeof(md.stdv));
    }
    std::vector<float> X((size_t)count * kMlpIn);
    for (int s = 0; s < count; ++s) standardise(md, feats + (size_t)s * kNumFeatures, &X[(size_t)s * kMlpIn]);
    PC_TRY(run_forward(md.params, X.data(), count, log_ms));
    for (int s = 0; s < count; ++s) {
        const float lw = log_work(feats + (size_t)s * kNumFeatures);
        for (int o = 0; o < kMlpOut; ++o) log_ms[(size_t)s * kMlpOut + o] += lw;
    }
    return PC_OK;
}

pc_status pc_selector_get_heuristic(double* p) {
    clear_error();
    if (!p) return fail(PC_ERR_INVALID_INPUT, "null argument");
    const HeuristicParams hp = heuristic_params();
    p[0] = hp.min_in_per_pivot_cta;
    p[1] = hp.warp_scan;
    p[2] = hp.group_scan;
    p[3] = hp.matrix_scan;
    return PC_OK;
}

pc_status pc_selector_set_heuristic(const double* p) {
    clear_error();
    if (!p) return fail(PC_ERR_INVALID_INPUT, "null argument");
    HeuristicParams hp;
    hp.min_in_per_pivot_cta = p[0];
    hp.warp_scan = p[1];
    hp.group_scan = p[2];
    hp.matrix_scan = p[3];
    set_heuristic_params(hp);
    return PC_OK;
}

// Autotuner of the plain heuristic: grid search of its four thresholds that
// minimises the summed measured time of its choices over the collected samples.
}  // extern "C"

namespace pc {

// Thresholds of the heuristic ranked by the proxy objective: the sum over all
// collected samples of the in-situ cost of the variant the rule picks.  Grid
// points that pick the same variants everywhere tie; the first of each total
// (grid order) represents it.  Returns up to k distinct totals, best first.
static pc_status autotune_rank(size_t k, std::vector<HeuristicParams>* out, std::vector<double>* proxy) {
    std::vector<float> feats, logms;
    std::vector<uint8_t> mask;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        feats = g_model.feats;
        logms = g_model.logms;
        mask = g_model.mask;
    }
    const size_t n = feats.size() / kNumFeatures;
    if (n == 0) return fail(PC_ERR_INVALID_INPUT, "no samples collected");
    const double grid_in[] = {1, 2, 4, 8, 16, 32, 64, 128, 256, 1e30};
    const double grid_scan[] = {0, 2, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 1e30};
    auto total = [&](const HeuristicParams& hp) {
        double t = 0;
        for (size_t s = 0; s < n; ++s) {
            int v = tc::heuristic_choice(&feats[s * kNumFeatures], hp);
            if (v < 0) continue;
            if (!mask[s * kMlpOut + v]) return 1e300;
            t += std::exp((double)logms[s * kMlpOut + v]);
        }
        return t;
    };
    std::vector<std::pair<double, HeuristicParams>> all;
    for (double a : grid_in)
        for (double w : grid_scan)
            for (double g : grid_scan) {
                if (g > w) continue;
                for (double mx : grid_scan) {
                    HeuristicParams hp{a, w, g, mx};
                    const double t = total(hp);
                    if (t < 1e299) all.emplace_back(t, hp);
                }
            }
    std::stable_sort(all.begin(), all.end(),
                     [](const std::pair<double, HeuristicParams>& x, const std::pair<double, HeuristicParams>& y) {
                         return x.first < y.first;
                     });
    out->clear();
    proxy->clear();
    for (const auto& e : all) {
        if (out->size() >= k) break;
        if (!proxy->empty() && e.first == proxy->back()) continue;
        out->push_back(e.second);
        proxy->push_back(e.first);
    }
    if (out->empty()) return fail(PC_ERR_INVALID_INPUT, "no threshold set can run every sample");
    return PC_OK;
}

static void params_out(const HeuristicParams& hp, double* p) {
    p[0] = hp.min_in_per_pivot_cta;
    p[1] = hp.warp_scan;
    p[2] = hp.group_scan;
    p[3] = hp.matrix_scan;
}

}  // namespace pc

extern "C" {

pc_status pc_selector_autotune(double* tuned) {
    clear_error();
    std::vector<HeuristicParams> cand;
    std::vector<double> proxy;
    PC_TRY(autotune_rank(1, &cand, &proxy));
    set_heuristic_params(cand[0]);
    if (tuned) params_out(cand[0], tuned);
    return PC_OK;
}

pc_status pc_selector_autotune_measured(pc_pgraph* const* pgs, int32_t npg, int32_t k, int32_t repeats,
                                        double* tuned, double* measured_ms) {
    clear_error();
    if (!pgs || npg < 1 || k < 1 || repeats < 1) return fail(PC_ERR_INVALID_INPUT, "bad argument");
    for (int32_t i = 0; i < npg; ++i)
        if (!pgs[i]) return fail(PC_ERR_INVALID_INPUT, "null graph view");
    std::vector<HeuristicParams> cand;
    std::vector<double> proxy;
    PC_TRY(autotune_rank((size_t)k, &cand, &proxy));
    // the thresholds in force before tuning compete too
    cand.push_back(heuristic_params());
    const HeuristicParams before = heuristic_params();
    // ms[c * npg + i]: median counting time of candidate c on view i
    std::vector<double> ms(cand.size() * (size_t)npg, 0.0);
    for (size_t c = 0; c < cand.size(); ++c) {
        set_heuristic_params(cand[c]);
        for (int32_t i = 0; i < npg; ++i) {
            PC_TRY(use_device(pgs[i]->g));
            std::vector<double> t;
            uint64_t cnt0 = 0;
            for (int32_t r = 0; r <= repeats; ++r) {  // the first call plans and warms up
                uint64_t cnt = 0;
                pc_tc_stats st;
                const pc_status e = tc_count(pgs[i], PC_VARIANT_HEURISTIC, &cnt, &st);
                if (e != PC_OK) {
                    set_heuristic_params(before);
                    return e;
                }
                if (r == 0) cnt0 = cnt;
                else t.push_back(st.kernel_ms);
                if (cnt != cnt0) {
                    set_heuristic_params(before);
                    return fail(PC_ERR_INVALID_INPUT, "autotune: counts differ between calls");
                }
            }
            std::sort(t.begin(), t.end());
            ms[c * npg + i] = t[t.size() / 2];
        }
    }
    // each view weighs alike: a candidate scores the sum over views of its time
    // over the fastest candidate's time on that view
    std::vector<double> fastest(npg, INFINITY);
    for (size_t c = 0; c < cand.size(); ++c)
        for (int32_t i = 0; i < npg; ++i) fastest[i] = std::min(fastest[i], ms[c * npg + i]);
    double best_score = INFINITY;
    size_t best = 0;
    for (size_t c = 0; c < cand.size(); ++c) {
        double score = 0;
        for (int32_t i = 0; i < npg; ++i) score += ms[c * npg + i] / std::max(fastest[i], 1e-9);
        if (score < best_score) {
            best_score = score;
            best = c;
        }
    }
    set_heuristic_params(cand[best]);
    if (tuned) params_out(cand[best], tuned);
    if (measured_ms) {
        double sum = 0;
        for (int32_t i = 0; i < npg; ++i) sum += ms[best * npg + i];
        *measured_ms = sum;
    }
    return PC_OK;
}

pc_status pc_selector_save(const char* path) {
    clear_error();
    if (!path) return fail(PC_ERR_INVALID_INPUT, "null path");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_model.trained) return fail(PC_ERR_UNSUPPORTED, "the selector is not trained");
    FILE* f = fopen(path, "wb");
    if (!f) return fail(PC_ERR_INVALID_INPUT, std::string("cannot write ") + path);
    const uint32_t magic = 0x50434D32u, np = kMlpParams;
    fwrite(&magic, 4, 1, f);
    fwrite(&np, 4, 1, f);
    fwrite(g_model.params.data(), 4, kMlpParams, f);
    fwrite(g_model.mean, 4, kMlpIn, f);
    fwrite(g_model.stdv, 4, kMlpIn, f);
    fwrite(g_model.lo, 4, kMlpIn, f);
    fwrite(g_model.hi, 4, kMlpIn, f);
    fwrite(&g_model.judge_log_margin, 4, 1, f);
    fclose(f);
    return PC_OK;
}

pc_status pc_selector_load(const char* path) {
    clear_error();
    if (!path) return fail(PC_ERR_INVALID_INPUT, "null path");
    FILE* f = fopen(path, "rb");
    if (!f) return fail(PC_ERR_INVALID_INPUT, std::string("cannot read ") + path);
    uint32_t magic = 0, np = 0;
    Model md;
    md.params.resize(kMlpParams);
    bool ok = fread(&magic, 4, 1, f) == 1 && fread(&np, 4, 1, f) == 1 && magic == 0x50434D32u && np == kMlpParams &&
              fread(md.params.data(), 4, kMlpParams, f) == (size_t)kMlpParams &&
              fread(md.mean, 4, kMlpIn, f) == (size_t)kMlpIn && fread(md.stdv, 4, kMlpIn, f) == (size_t)kMlpIn &&
              fread(md.lo, 4, kMlpIn, f) == (size_t)kMlpIn && fread(md.hi, 4, kMlpIn, f) == (size_t)kMlpIn &&
              fread(&md.judge_log_margin, 4, 1, f) == 1;
    fclose(f);
    if (!ok) return fail(PC_ERR_INVALID_INPUT, "not a selector model file");
    std::lock_guard<std::mutex> lk(g_mu);
    g_model.params = md.params;
    memcpy(g_model.mean, md.mean, sizeof(md.mean));
    memcpy(g_model.stdv, md.stdv, sizeof(md.stdv));
    memcpy(g_model.lo, md.lo, sizeof(md.lo));
    memcpy(g_model.hi, md.hi, sizeof(md.hi));
    g_model.judge_log_margin = md.judge_log_margin;
    g_model.trained = true;
    bump_version_locked();
    return PC_OK;
}

}  // extern "C"
