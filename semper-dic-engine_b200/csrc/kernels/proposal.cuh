// The learned seed proposal network on the device (proposal.cu): BF16
// tensor-core convolutions and MLP, forward and backward, FP32 accumulation,
// Adam on FP32 master weights, and the generator of synthetic training pairs.
//
// Network: two 64x64 patches stacked as two channels (NHWC); five 3x3
// convolutions, stride 2, padding 1, to 16, 32, 64, 128, 128 channels, each
// with ReLU; the 128 x 2 x 2 features flattened (h, w, c); 512 -> 128 (ReLU)
// -> 6. The six outputs are the affine map of centred patch coordinates from
// the first patch to the second, A = I + [[o0, o1], [o2, o3]], t = 16 (o4, o5).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace dic {

constexpr int kPpSide = 64;  // patch side
constexpr int kPpChannels[6] = {2, 16, 32, 64, 128, 128};
constexpr int kPpFc0 = 512, kPpFc1 = 128, kPpOut = 6;
constexpr float kPpTScale = 16.0f;

// Flat parameter layout (floats): w0 b0 w1 b1 ... w4 b4 w5 b5 w6 b6, conv
// weights [co][kh][kw][ci], FC weights [out][in].
struct PpLayout {
    size_t w[7], b[7];
    size_t total;
};
PpLayout pp_layout();

// Device workspace of one batch (activations bf16 NHWC per layer, FP32
// scratch for pre-activations and gradients), sized for up to max_batch pairs.
struct PpWork {
    int max_batch = 0;
    uint16_t* act[6] = {};  // bf16: input, then the five conv outputs
    uint16_t* h = nullptr;  // bf16 [B, 128]
    float* y = nullptr;     // FP32 scratch: the largest pre-activation / gradient
    float* dy = nullptr;    // FP32 scratch
    float* out = nullptr;   // [B, 6]
    float* gout = nullptr;  // [B, 6]
    float* loss = nullptr;  // [1]
};
size_t pp_work_bytes(int max_batch);
void pp_work_carve(PpWork& w, void* base, int max_batch);

// Forward: x (w.act[0], bf16 [B, 64, 64, 2]) -> w.out [B, 6]; params FP32.
cudaError_t pp_forward(const float* params, PpWork& w, int B, cudaStream_t st);
// Loss (mean squared displacement of the affine map at a 3x3 grid of patch
// points) and its gradient w.r.t. the outputs: w.loss, w.gout.
cudaError_t pp_loss(PpWork& w, const float* target, int B, cudaStream_t st);
// Backward from w.gout: grads (FP32, zeroed by the call) of every parameter.
cudaError_t pp_backward(const float* params, PpWork& w, int B, float* grads, cudaStream_t st);
// One Adam step on the FP32 parameters (m, v: moment buffers; t >= 1).
cudaError_t pp_adam(float* params, const float* grads, float* m, float* v, size_t n, int t, float lr,
                    cudaStream_t st);

// Patch pairs into the network's input (bf16 [B, 64, 64, 2]), each patch
// normalised to zero mean and unit deviation: pair k takes the box average
// of f x f pixels of `ref` around centre (ax_k, ay_k) and of `def` around
// (bx_k, by_k) (centres [B][4]; u8 frames of width W, height H, row pitch
// `pitch`); patch pixel (u, v) covers the f x f pixels from
// centre + f (u - 32, v - 32); pixels outside the frame read its nearest edge.
cudaError_t pp_cut_pairs(const uint8_t* ref, const uint8_t* def, int W, int H, int pitch, const float* centres,
                         int B, int f, uint16_t* x, cudaStream_t st);

// The same with the second patch sampled through an affine map: pair k's
// second patch takes, for each sample X of its first patch (the f x f pixels
// around centre (ax_k, ay_k)), `def` at x' = A_k X + b_k (bilinear, clamped
// to the frame); maps [B][8] = ax, ay, a00, a01, a10, a11, bx, by. With the
// map the true one, the two patches show the same material. scratch: B x 8192
// floats for the values before normalisation.
cudaError_t pp_cut_warped(const uint8_t* ref, const uint8_t* def, int W, int H, int pitch, const float* maps, int B,
                          int f, uint16_t* x, float* scratch, cudaStream_t st);

// Synthetic training pairs from a float speckle image S (W x H): pair k gets
// a random centre c, rotation, small stretch and shear and translation t; its
// first patch is S box-averaged by f around c, its second the warped image
// x = o + t + A (X - o) (o = c - 0.5, the patches' common origin) sampled
// bilinearly with Gaussian noise of `noise` gray levels per full-resolution
// sample, box-averaged by f around c; target [B, 6] the affine map in patch
// coordinates (A, t / f). Deterministic in (seed, k).
struct PpSynth {
    float max_rot;      // rotation drawn in [0, max_rot) radians
    float max_stretch;  // per-axis stretch in [-max_stretch, max_stretch]
    float max_shear;
    float max_shift;    // translation per axis in [-max_shift, max_shift] full-resolution px
    float noise;
    int f;              // box-average factor
};
cudaError_t pp_synth_pairs(const float* S, int W, int H, const PpSynth& cfg, uint64_t seed, int B, uint16_t* x,
                           float* target, cudaStream_t st);

}  // namespace dic
