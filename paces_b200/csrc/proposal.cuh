// Learned candidate proposal: a small MLP that scores every image ("event") of the
// truncated basis during expansion, so that images unlikely to matter are dropped before
// they are merged, sorted and built into H.  No counterpart in the reference.
//
// Events.  For a basis X (nx states) the events are e = (j - 1) * nx + i for the four
// off-diagonal runs j = 1..4 (FROM_LEFT: the exciton of state i hops right, FROM_RIGHT:
// hops left, UP: one phonon created at the exciton site, DOWN: one annihilated) -- the
// merge's runs, indexed by source state.  An event is invalid where the image does not
// exist (open-chain end, occupation ceiling, floor).
//
// Features (16, rounded to bf16) of event (j, i) with image state (p', n'):
//   f[0..8]  n'_{p'+d} * fp32(1 / (max_ho_dim_{p'+d} - 1)), d = -4..4 (ring: wrapped; open
//            chain: 0 outside the chain)
//   f[9]     sum_s n'_s / 16
//   f[10]    (log max(|psi_i|, 1e-30) - log max(cut, 1e-30)) / 16: the source state's
//            amplitude relative to the cut of the truncation that kept it (the smallest
//            kept |psi|), which makes the feature stationary as the wavefunction spreads
//   f[11..13] one-hot term type: hop, create, annihilate
//   f[14]    log max(|H_image,source|, 1e-30) / 4: J for a hop, g sqrt(n') for a creation,
//            g sqrt(n' + 1) for an annihilation (n' the image's occupation at the site)
//   f[15]    0
// Network: h1 = bf16(relu(W1 f + b1)), h2 = relu(W2 h1 + b2), logit = w3 . h2 + b3, with
// W1 [64][16] and W2 [64][64] in bf16, everything else fp32; the image is kept when
// logit > threshold.  A truncation that dropped nothing has no cut (0): then every
// existing image is kept.
#pragma once

#include "common.cuh"

namespace paces {

constexpr int kMlpIn = 16;
constexpr int kMlpHid = 64;
// packed inference parameters (device): bf16 W1 [64][16], bf16 W2 [64][64], f32 b1, b2, w3 [64], f32 b3
constexpr size_t kMlpOffW1 = 0;
constexpr size_t kMlpOffW2 = kMlpOffW1 + size_t(kMlpHid) * kMlpIn * 2;
constexpr size_t kMlpOffB1 = kMlpOffW2 + size_t(kMlpHid) * kMlpHid * 2;
constexpr size_t kMlpOffB2 = kMlpOffB1 + kMlpHid * 4;
constexpr size_t kMlpOffW3 = kMlpOffB2 + kMlpHid * 4;
constexpr size_t kMlpOffB3 = kMlpOffW3 + kMlpHid * 4;
constexpr size_t kMlpParamBytes = 11264;
// fp32 master weights and gradients: W1 [64*16], W2 [64*64], b1 [64], b2 [64], w3 [64], b3
constexpr int kMlpMW1 = 0;
constexpr int kMlpMW2 = kMlpMW1 + kMlpHid * kMlpIn;
constexpr int kMlpMB1 = kMlpMW2 + kMlpHid * kMlpHid;
constexpr int kMlpMB2 = kMlpMB1 + kMlpHid;
constexpr int kMlpMW3 = kMlpMB2 + kMlpHid;
constexpr int kMlpMB3 = kMlpMW3 + kMlpHid;
constexpr int kMlpMasterFloats = kMlpMB3 + 1;

struct ProposalOut {
    uint8_t* keep;       // [kRuns][keep_cap] (row 0 unused) or null
    int64_t keep_cap;
    float* logits;       // [4 * nx] or null
    int* counts;         // [2] valid events, kept events (accumulated) or null
};

int launch_proposal_score(int nw, const ModelDev& m, const uint64_t* x_keys, const int* x_blk,
                          const float* x_w, const float* cut, const void* params, float threshold,
                          const ProposalOut& out, int* status, int num_sms, cudaStream_t st);
int launch_proposal_features(int nw, const ModelDev& m, const uint64_t* x_keys, const int* x_blk,
                             const float* x_w, const float* cut, uint16_t* feats, uint8_t* valid, int num_sms,
                             cudaStream_t st);
int launch_proposal_labels(int nw, const ModelDev& m, const uint64_t* x_keys, const int* x_blk,
                           const uint64_t* y_keys, const int* y_blk, uint8_t* labels, int num_sms,
                           cudaStream_t st);
int launch_mlp_pack(const float* master, void* params, cudaStream_t st);
int launch_mlp_forward(const void* params, const uint16_t* x, int64_t n, float* logits, int num_sms,
                       cudaStream_t st);
int launch_mlp_backward(const void* params, const uint16_t* x, const float* y, const float* sw, int64_t n,
                        float inv_norm, float* grads, double* loss, int num_sms, cudaStream_t st);
int launch_mlp_adam(float* master, float* m1, float* m2, float* grads, int t, float lr, float beta1,
                    float beta2, float eps, void* params, cudaStream_t st);

}  // namespace paces
