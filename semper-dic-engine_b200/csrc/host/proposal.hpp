// The learned seed proposal network on the host side: parameters and
// optimiser state in device memory, batched forward and backward on the
// kernels of kernels/proposal.cu, training on synthetic pairs made on the
// device, and inference on patch pairs cut from frames in device memory.
#pragma once
#include <cstddef>
#include <cstdint>
#include <map>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../kernels/proposal.cuh"
#include "engine.hpp"

namespace semper_b200 {

class ProposalNet {
public:
    explicit ProposalNet(int max_batch = 256);
    ~ProposalNet();
    ProposalNet(const ProposalNet&) = delete;
    ProposalNet& operator=(const ProposalNet&) = delete;

    static size_t param_count();
    void set_params(const float* host);
    void get_params(float* host) const;
    // He-normal weights and zero biases from a seed (host generator).
    void init(uint64_t seed);
    int max_batch() const { return max_batch_; }

    // x: host [B, 64, 64, 2] floats (rounded to bfloat16); out: host [B, 6].
    void forward_host(const float* x, int B, float* out);
    // The loss of targets [B, 6] and every parameter's gradient (host).
    float gradients_host(const float* x, const float* target, int B, float* grads);
    // Synthetic pairs from a u8 speckle image (host), as the training makes
    // them: x [B, 64, 64, 2] and target [B, 6] to the host.
    void synth_host(const uint8_t* speckle, int W, int H, const dic::PpSynth& cfg, uint64_t seed, int B, float* x,
                    float* target);
    // Adam on synthetic pairs: `steps` batches of B pairs (pair seeds from
    // `seed`); losses[i] (host, may be null) the loss of batch i.
    void train(const uint8_t* speckle, int W, int H, const dic::PpSynth& cfg, int steps, int B, float lr,
               uint64_t seed, float* losses);
    // Predictions for K pairs cut from device frames on `st` (centres host
    // [K, 4]: ref x, y, def x, y) at box factor f; out host [K, 6].
    void predict_device(const uint8_t* d_ref, const uint8_t* d_def, int W, int H, int pitch, const float* centres,
                        int K, int f, float* out, cudaStream_t st);

    // The same with each pair's second patch sampled through an affine map
    // (maps host [K, 8]: ref centre x, y, then a00 a01 a10 a11 bx by).
    void predict_warped(const uint8_t* d_ref, const uint8_t* d_def, int W, int H, int pitch, const float* maps,
                        int K, int f, float* out, cudaStream_t st);
    // predict_warped on u8 frames in host memory (W x H, packed rows), on the
    // network's own stream.
    void predict_warped_host(const uint8_t* ref, const uint8_t* def, int W, int H, const float* maps, int K, int f,
                             float* out);

private:
    void upload_speckle(const uint8_t* speckle, int W, int H);
    int max_batch_;
    cudaStream_t st_ = nullptr;
    DevBuf<float> params_, grads_, m_, v_, target_, centres_, speckle_f_;
    DevBuf<unsigned char> work_, frames_;
    dic::PpWork w_;
    int adam_t_ = 0;
    // predict_warped as one CUDA graph per (frames, size, batch, factor,
    // stream): the map upload from pinned staging, the patch cut, the
    // forward and the prediction download, captured on first use. The
    // graphs hold the device buffers' addresses, which stay fixed (centres_
    // is sized for max_batch up front).
    struct GraphKey {
        const void* ref;
        const void* def;
        int W, H, pitch, K, f;
        cudaStream_t st;
        bool operator<(const GraphKey& o) const {
            return std::tie(ref, def, W, H, pitch, K, f, st) < std::tie(o.ref, o.def, o.W, o.H, o.pitch, o.K, o.f, o.st);
        }
    };
    std::map<GraphKey, cudaGraphExec_t> graphs_;
    float* h_maps_ = nullptr;  // pinned, max_batch x 8
    float* h_out_ = nullptr;   // pinned, max_batch x 6
    void drop_graphs();
};

}  // namespace semper_b200
