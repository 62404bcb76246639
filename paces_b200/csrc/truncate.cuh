// Amplitude-ranked truncation to `maxstates` states.
//
// Reference (paces/core/time_evolution.py:833-910): stable ascending argsort of |psi|,
// keep the last `maxstates` entries (among equal values the highest indices), lexsort
// the kept rows.  With shuffle_seed set and a tie at the cut, the tied states at the
// cut are drawn at random.
//
// B200 design: no sort.  The weights |psi| are non-negative doubles, so their bit
// patterns order like the values; a radix select (12-bit digits, shared-memory
// histograms) finds the threshold value v* and the number of states equal to v* that
// must be kept.  Because the basis is already sorted, keeping the selected states in
// index order *is* the lexsorted result: one order-preserving compaction writes the
// new basis (keys and block offsets).  Tie rule as in the reference: the states equal
// to v* with the highest indices; with shuffling, the tied states whose 64-bit hash of
// (seed, step, index) is smallest -- a uniformly random subset, like the reference's
// random permutation, but not the same stream (parity unpinned for that branch).
#pragma once

#include "common.cuh"

namespace paces {

struct TruncWs {
    unsigned* hist;              // [4096]
    unsigned long long* cand;    // [cap] candidate weight bits (or hashes)
    int* cand_idx;               // [cap]
    long long* sel;              // selection state, see truncate.cu
    int* tile_cnt;               // [ntiles_cap][3]
    int* tile_pre;               // [ntiles_cap][3]
    int64_t cap;
    int ntiles_cap;
};

constexpr int kTruncTile = 4096;

inline int trunc_tiles_cap(int64_t cap) { return int(cap / kTruncTile + 2); }

// Radix rounds (12-bit digits from the top) of the weight selection for a weight kind (0
// complex128 |psi|, 1 complex64 |psi|, 2 precomputed fp64 weights): a complex64 weight is
// an fp32 value widened to a double, so its bits 28..0 are zero and rounds 0-2 (bits
// 63..28) decide it.
inline int weight_rounds(int wk) { return wk == 1 ? 3 : 6; }
// Kernels one truncation enqueues.
inline int trunc_launches(int wk, bool shuffle) { return 5 + 2 * weight_rounds(wk) + (shuffle ? 14 : 0); }

// weights (optional, one non-negative double per state): rank by these instead of |psi|
// (the look-ahead weighting, lookahead.cu).
// scratch (optional, without weights: 4 bytes per state for complex64, 8 for complex128):
// the first radix round stores |psi| there and the later passes read it instead of the
// amplitudes, so |psi| is computed once per state.
// out_w (optional, out_cap + 1 floats): the ranked weight (|psi|) of every kept state in the
// new basis' order, and at out_w[out_cap] the cut -- the weight of the smallest kept state, 0
// when nothing was dropped.
int launch_truncate(int nw, bool c64, const ModelDev& m, const uint64_t* x_keys, const int* x_blk,
                    const void* psi, const double* weights, void* scratch, int64_t maxstates, int shuffle, uint64_t seed,
                    uint64_t step, const TruncWs& ws, uint64_t* out_keys, int* out_blk, int64_t out_cap, float* out_w,
                    int* n_tied_out, int* n_kept_out, int* status, int num_sms, cudaStream_t st);

}  // namespace paces
