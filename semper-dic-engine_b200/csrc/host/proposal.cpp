// The learned seed proposal network: host side (proposal.hpp).
#include "proposal.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <stdexcept>

namespace semper_b200 {

ProposalNet::ProposalNet(int max_batch) : max_batch_(max_batch) {
    if (max_batch <= 0) throw std::invalid_argument("proposal: batch");
    check(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "stream");
    const size_t n = param_count();
    for (DevBuf<float>* b : {&params_, &grads_, &m_, &v_}) b->ensure(n);
    target_.ensure((size_t)max_batch * dic::kPpOut);
    centres_.ensure((size_t)max_batch * 8);
    check(cudaHostAlloc(&h_maps_, (size_t)max_batch * 8 * sizeof(float), cudaHostAllocDefault), "pinned maps");
    check(cudaHostAlloc(&h_out_, (size_t)max_batch * 6 * sizeof(float), cudaHostAllocDefault), "pinned out");
    work_.ensure(dic::pp_work_bytes(max_batch));
    dic::pp_work_carve(w_, work_.p, max_batch);
    init(0);
}

ProposalNet::~ProposalNet() {
    if (st_) {
        cudaStreamSynchronize(st_);
        cudaStreamDestroy(st_);
    }
    drop_graphs();
    if (h_maps_) cudaFreeHost(h_maps_);
    if (h_out_) cudaFreeHost(h_out_);
}

void ProposalNet::drop_graphs() {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
}

size_t ProposalNet::param_count() { return dic::pp_layout().total; }

void ProposalNet::set_params(const float* host) {
    check(cudaMemcpyAsync(params_.p, host, param_count() * 4, cudaMemcpyHostToDevice, st_), "H2D params");
    check(cudaMemsetAsync(m_.p, 0, param_count() * 4, st_), "memset");
    check(cudaMemsetAsync(v_.p, 0, param_count() * 4, st_), "memset");
    check(cudaStreamSynchronize(st_), "sync");
    adam_t_ = 0;
}

void ProposalNet::get_params(float* host) const {
    check(cudaMemcpyAsync(host, params_.p, param_count() * 4, cudaMemcpyDeviceToHost, st_), "D2H params");
    check(cudaStreamSynchronize(st_), "sync");
}

void ProposalNet::init(uint64_t seed) {
    const dic::PpLayout L = dic::pp_layout();
    std::vector<float> p(L.total, 0.0f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    for (int l = 0; l < 5; ++l) {
        const int ci = dic::kPpChannels[l], co = dic::kPpChannels[l + 1];
        const float s = std::sqrt(2.0f / (9.0f * ci));
        for (size_t i = 0; i < (size_t)co * 9 * ci; ++i) p[L.w[l] + i] = nd(rng) * s;
    }
    const float s5 = std::sqrt(2.0f / dic::kPpFc0), s6 = 0.1f * std::sqrt(1.0f / dic::kPpFc1);
    for (size_t i = 0; i < (size_t)dic::kPpFc1 * dic::kPpFc0; ++i) p[L.w[5] + i] = nd(rng) * s5;
    for (size_t i = 0; i < (size_t)dic::kPpOut * dic::kPpFc1; ++i) p[L.w[6] + i] = nd(rng) * s6;
    set_params(p.data());
}

namespace {

// Host floats to bfloat16 bits (nearest even), as the device rounds.
uint16_t host_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    const uint32_t lsb = (u >> 16) & 1u;
    return (uint16_t)((u + 0x7fffu + lsb) >> 16);
}
float host_from_bf16(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

}  // namespace

void ProposalNet::forward_host(const float* x, int B, float* out) {
    if (B <= 0 || B > max_batch_) throw std::invalid_argument("proposal: batch");
    std::vector<uint16_t> xb((size_t)B * 8192);
    for (size_t i = 0; i < xb.size(); ++i) xb[i] = host_bf16(x[i]);
    check(cudaMemcpyAsync(w_.act[0], xb.data(), xb.size() * 2, cudaMemcpyHostToDevice, st_), "H2D x");
    check(dic::pp_forward(params_.p, w_, B, st_), "proposal forward");
    check(cudaMemcpyAsync(out, w_.out, (size_t)B * 6 * 4, cudaMemcpyDeviceToHost, st_), "D2H out");
    check(cudaStreamSynchronize(st_), "sync");
}

float ProposalNet::gradients_host(const float* x, const float* target, int B, float* grads) {
    if (B <= 0 || B > max_batch_) throw std::invalid_argument("proposal: batch");
    std::vector<uint16_t> xb((size_t)B * 8192);
    for (size_t i = 0; i < xb.size(); ++i) xb[i] = host_bf16(x[i]);
    check(cudaMemcpyAsync(w_.act[0], xb.data(), xb.size() * 2, cudaMemcpyHostToDevice, st_), "H2D x");
    check(cudaMemcpyAsync(target_.p, target, (size_t)B * 6 * 4, cudaMemcpyHostToDevice, st_), "H2D target");
    check(dic::pp_forward(params_.p, w_, B, st_), "proposal forward");
    check(dic::pp_loss(w_, target_.p, B, st_), "proposal loss");
    check(dic::pp_backward(params_.p, w_, B, grads_.p, st_), "proposal backward");
    float loss = 0.0f;
    check(cudaMemcpyAsync(&loss, w_.loss, 4, cudaMemcpyDeviceToHost, st_), "D2H loss");
    check(cudaMemcpyAsync(grads, grads_.p, param_count() * 4, cudaMemcpyDeviceToHost, st_), "D2H grads");
    check(cudaStreamSynchronize(st_), "sync");
    return loss;
}

void ProposalNet::upload_speckle(const uint8_t* speckle, int W, int H) {
    const size_t n = (size_t)W * H;
    std::vector<float> f(n);
    for (size_t i = 0; i < n; ++i) f[i] = (float)speckle[i];
    speckle_f_.ensure(std::max(speckle_f_.n, n));
    check(cudaMemcpyAsync(speckle_f_.p, f.data(), n * 4, cudaMemcpyHostToDevice, st_), "H2D speckle");
    check(cudaStreamSynchronize(st_), "sync");
}

void ProposalNet::synth_host(const uint8_t* speckle, int W, int H, const dic::PpSynth& cfg, uint64_t seed, int B,
                             float* x, float* target) {
    if (B <= 0 || B > max_batch_) throw std::invalid_argument("proposal: batch");
    upload_speckle(speckle, W, H);
    check(dic::pp_synth_pairs(speckle_f_.p, W, H, cfg, seed, B, w_.act[0], target_.p, st_), "synth pairs");
    std::vector<uint16_t> xb((size_t)B * 8192);
    check(cudaMemcpyAsync(xb.data(), w_.act[0], xb.size() * 2, cudaMemcpyDeviceToHost, st_), "D2H x");
    check(cudaMemcpyAsync(target, target_.p, (size_t)B * 6 * 4, cudaMemcpyDeviceToHost, st_), "D2H target");
    check(cudaStreamSynchronize(st_), "sync");
    for (size_t i = 0; i < xb.size(); ++i) x[i] = host_from_bf16(xb[i]);
}

void ProposalNet::train(const uint8_t* speckle, int W, int H, const dic::PpSynth& cfg, int steps, int B, float lr,
                        uint64_t seed, float* losses) {
    if (B <= 0 || B > max_batch_ || steps < 0) throw std::invalid_argument("proposal: batch");
    upload_speckle(speckle, W, H);
    DevBuf<float> dl;
    dl.ensure((size_t)std::max(steps, 1));
    for (int s = 0; s < steps; ++s) {
        check(dic::pp_synth_pairs(speckle_f_.p, W, H, cfg, seed * 1000003ull + (uint64_t)s, B, w_.act[0], target_.p,
                                  st_),
              "synth pairs");
        check(dic::pp_forward(params_.p, w_, B, st_), "proposal forward");
        check(dic::pp_loss(w_, target_.p, B, st_), "proposal loss");
        check(dic::pp_backward(params_.p, w_, B, grads_.p, st_), "proposal backward");
        check(dic::pp_adam(params_.p, grads_.p, m_.p, v_.p, param_count(), ++adam_t_, lr, st_), "adam");
        check(cudaMemcpyAsync(dl.p + s, w_.loss, 4, cudaMemcpyDeviceToDevice, st_), "loss");
    }
    if (losses && steps > 0)
        check(cudaMemcpyAsync(losses, dl.p, (size_t)steps * 4, cudaMemcpyDeviceToHost, st_), "D2H losses");
    check(cudaStreamSynchronize(st_), "sync");
}

void ProposalNet::predict_device(const uint8_t* d_ref, const uint8_t* d_def, int W, int H, int pitch,
                                 const float* centres, int K, int f, float* out, cudaStream_t st) {
    if (K <= 0 || K > max_batch_) throw std::invalid_argument("proposal: batch");
    centres_.ensure(std::max(centres_.n, (size_t)K * 4));
    check(cudaMemcpyAsync(centres_.p, centres, (size_t)K * 16, cudaMemcpyHostToDevice, st), "H2D centres");
    check(dic::pp_cut_pairs(d_ref, d_def, W, H, pitch, centres_.p, K, f, w_.act[0], st), "cut pairs");
    check(dic::pp_forward(params_.p, w_, K, st), "proposal forward");
    check(cudaMemcpyAsync(out, w_.out, (size_t)K * 6 * 4, cudaMemcpyDeviceToHost, st), "D2H out");
    check(cudaStreamSynchronize(st), "sync");
}

void ProposalNet::predict_warped(const uint8_t* d_ref, const uint8_t* d_def, int W, int H, int pitch,
                                 const float* maps, int K, int f, float* out, cudaStream_t st) {
    if (K <= 0 || K > max_batch_) throw std::invalid_argument("proposal: batch");
    if (W < 2 || H < 2 || pitch < W || f < 1 || f > 16) throw std::invalid_argument("proposal: frame or factor");
    // one graph launch instead of 16 launches and two pageable copies: the
    // cascade of the learned seeding makes about a dozen of these calls a
    // frame, each waiting for its predictions
    std::memcpy(h_maps_, maps, (size_t)K * 32);
    const GraphKey key{d_ref, d_def, W, H, pitch, K, f, st};
    auto it = graphs_.find(key);
    if (it == graphs_.end()) {
        if (graphs_.size() >= 64) drop_graphs();
        cudaGraph_t g = nullptr;
        check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
        cudaError_t e = cudaMemcpyAsync(centres_.p, h_maps_, (size_t)K * 32, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = dic::pp_cut_warped(d_ref, d_def, W, H, pitch, centres_.p, K, f, w_.act[0], w_.y, st);
        if (e == cudaSuccess) e = dic::pp_forward(params_.p, w_, K, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_out_, w_.out, (size_t)K * 6 * 4, cudaMemcpyDeviceToHost, st);
        const cudaError_t ee = cudaStreamEndCapture(st, &g);
        if ((e != cudaSuccess || ee != cudaSuccess) && g) cudaGraphDestroy(g);
        check(e, "proposal capture");
        check(ee, "capture end");
        cudaGraphExec_t x = nullptr;
        e = cudaGraphInstantiate(&x, g, 0);
        cudaGraphDestroy(g);
        check(e, "graph instantiate");
        it = graphs_.emplace(key, x).first;
    }
    check(cudaGraphLaunch(it->second, st), "graph launch");
    check(cudaStreamSynchronize(st), "sync");
    std::memcpy(out, h_out_, (size_t)K * 6 * 4);
}

void ProposalNet::predict_warped_host(const uint8_t* ref, const uint8_t* def, int W, int H, const float* maps, int K,
                                      int f, float* out) {
    if (W < 2 || H < 2) throw std::invalid_argument("proposal: frame size");
    const size_t n = (size_t)W * H;
    frames_.ensure(std::max(frames_.n, 2 * n));
    check(cudaMemcpyAsync(frames_.p, ref, n, cudaMemcpyHostToDevice, st_), "H2D ref");
    check(cudaMemcpyAsync(frames_.p + n, def, n, cudaMemcpyHostToDevice, st_), "H2D def");
    predict_warped(frames_.p, frames_.p + n, W, H, W, maps, K, f, out, st_);
}

}  // namespace semper_b200
