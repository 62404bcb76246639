// Declarations shared between the stage kernels and the C ABI layer.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "merge.cuh"
#include "truncate.cuh"

namespace paces {

// Largest r with off[r] <= s (off non-decreasing with n+1 entries, s < off[n]).
__device__ __forceinline__ int find_segment(const int* off, int n, int s) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= s) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---- remap ------------------------------------------------------------------------------
struct RemapWs {
    int* tile_off;  // [L+1]
    int* counters;  // [0] tiles
    int* split;     // [tile_cap][2] old-basis split of each tile's first and last diagonal
    int tile_cap;
};
// diagonals per remap tile: 1024 measured faster than 2048 for one or two key words (0.30 -> 0.25 ms
// at 2^22, eight blocks' worth of tiles per SM)
__host__ __device__ constexpr int remap_tile(int nw) { return nw <= 4 ? 1024 : 512; }
inline int remap_tile_cap(int64_t cap, int nw, int L) { return int((2 * cap) / remap_tile(nw) + L + 8); }
int launch_remap(int nw, bool c64, const ModelDev& m, const uint64_t* ok, const int* ob,
                 const void* opsi, const uint64_t* nk, const int* nb, void* npsi, const RemapWs& ws,
                 int* status, int num_sms, cudaStream_t st);
// Workspace of the remap in the library's static device scratch (current device).
int remap_static_ws(RemapWs* ws, const char** err);
int remap_static_tile_cap();

// ---- Taylor -----------------------------------------------------------------------------
struct TaylorOut {
    int* converged;
    int* final_m;
    double* c1_plus_c2;
    double* term_ratio;
};
struct TaylorWs {
    void* ta;            // [cap] complex
    void* tb;            // [cap] complex
    double* partials;    // [2][max_grid][4]
    unsigned* barrier;   // [2]
    uint64_t wait_ns;    // grid-barrier wait limit (kWaitLimitNs unless a test shortens it)
    int skip_block;      // test hook: this block skips its first grid-barrier arrival (-1: none)
    double* diag;        // null, or [diag_groups(rows)][3]: see diag_group
};
int taylor_max_grid(bool c64, int num_sms);

// ---- diagnostics of the input state, from the first Taylor sweep ---------------------------
// The first sweep of the series forms (H v)_r for every row, so the post-adaptation norm and
// energy <v|H|v> come out of it: each warp folds the rows of one 64-row group (rows 64 g + l and
// 64 g + 32 + l on lane l, in every kernel and schedule: the lane adds its two rows, then a fixed
// butterfly), and diag_final sums the groups in a fixed order.  The result depends on the rows
// only -- not on the grid, the row schedule or whether the trajectory runs alone or in a batch.
constexpr int kDiagGroup = 64;
constexpr int kDiagChunk = 2048;  // groups per block of the first reduction
__host__ __device__ inline int64_t diag_groups(int64_t rows) { return (rows + kDiagGroup - 1) / kDiagGroup; }
inline int64_t diag_chunks(int64_t rows) { return (diag_groups(rows) + kDiagChunk - 1) / kDiagChunk; }
// doubles of a diag buffer for up to `cap` rows: the group sums, then the chunk sums
inline size_t diag_doubles(int64_t cap) { return size_t(diag_groups(cap) + diag_chunks(cap)) * 3; }

// |v_r|^2, Re and Im of conj(v_r) (H v)_r of one row (zero when it does not exist).
template <typename C>
__device__ __forceinline__ void diag_row(bool valid, const C& a, const C& y, double& n2, double& er, double& ei) {
    n2 = er = ei = 0.0;
    if (valid) {
        const double ar = double(a.x), ai = double(a.y), yr = double(y.x), yi = double(y.y);
        n2 = fma(ar, ar, __dmul_rn(ai, ai));
        er = fma(ar, yr, __dmul_rn(ai, yi));
        ei = fma(ar, yi, -__dmul_rn(ai, yr));
    }
}

// Called by all 32 lanes of a warp for group g, whose rows 64 g + lane (valid0: it exists; a0,
// y0: v_r and (H v)_r) and 64 g + 32 + lane (valid1, a1, y1) this lane holds.
template <typename C>
__device__ __forceinline__ void diag_group(double* __restrict__ diag, int64_t g, bool valid0, const C& a0,
                                           const C& y0, bool valid1, const C& a1, const C& y1) {
    double n2, er, ei, n2b, erb, eib;
    diag_row(valid0, a0, y0, n2, er, ei);
    diag_row(valid1, a1, y1, n2b, erb, eib);
    n2 = __dadd_rn(n2, n2b);
    er = __dadd_rn(er, erb);
    ei = __dadd_rn(ei, eib);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n2 = __dadd_rn(n2, __shfl_xor_sync(0xffffffffu, n2, o));
        er = __dadd_rn(er, __shfl_xor_sync(0xffffffffu, er, o));
        ei = __dadd_rn(ei, __shfl_xor_sync(0xffffffffu, ei, o));
    }
    if ((threadIdx.x & 31) == 0) {
        diag[g * 3] = n2;
        diag[g * 3 + 1] = er;
        diag[g * 3 + 2] = ei;
    }
}

// ---- Lanczos ----------------------------------------------------------------------------
constexpr int kMaxLanczosOrder = PACES_MAX_LANCZOS_ORDER;
struct LanczosWs {
    void* u;             // [order+1][cap] complex: the Krylov vectors q_i (columns of V)
    void* w0;            // [cap] complex: the recurrence's w, double-buffered
    void* w1;
    double* partials;    // [2][max_grid][4]
    unsigned* barrier;   // [2]
    int64_t cap;         // rows of each vector
    int max_grid;
    int skip_block;      // test hook (see TaylorWs)
    uint64_t wait_ns;
};
int lanczos_max_grid(int num_sms);

// ---- rows of uint32 words (host API helpers) ---------------------------------------------
size_t rows_sort_ws_bytes(int64_t n);
int launch_rows_lower_bound(const uint32_t* pb, int64_t n, const uint32_t* q, int64_t nq, int words, int must,
                            int64_t* out, int* missing, int num_sms, cudaStream_t st);
int launch_rows_sort_unique(const uint32_t* rows, int64_t n, int words, uint32_t* out, int64_t* count, void* ws,
                            int num_sms, cudaStream_t st);
int launch_lanczos(bool c64, const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta,
                   const void* v_in, void* res, double dt, int order, const LanczosWs& ws, const TaylorOut& out,
                   int* status, int num_sms, cudaStream_t st);
// blocks_per_sm: 0 = as many as fit (the grid never exceeds taylor_max_grid);
// variant: 0 = direct grid-stride rows, 1 = chunks prefetched by bulk TMA copies
int launch_taylor(bool c64, const ModelDev& m, const int* blk, const int* nbr, int64_t nbr_cap,
                  const uint32_t* meta, const void* v_in, void* res, double dt, int m_star,
                  double tol, const TaylorWs& ws, const TaylorOut& out, int* status, int num_sms,
                  int blocks_per_sm, int variant, cudaStream_t st);

// ---- scaling and squaring (expm.cu) ---------------------------------------------------------
// out[0] = trace(H), out[1] = max row 1-norm of H - *shift I (0 when shift is null),
// out[2] = trace / n; part holds 2 * nparts doubles.
int launch_hnorms(const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta, const double* shift,
                  double* part, int nparts, double* out, cudaStream_t st);
int launch_expm_scaled(bool c64, const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta,
                       const void* v_in, void* res, double t, double shift, int m_star, int stages, double tol,
                       double eta_re, double eta_im, const TaylorWs& ws, const TaylorOut& out, int* status,
                       int num_sms, int max_grid, cudaStream_t st);

// ---- look-ahead truncation weights (lookahead.cu) -------------------------------------------
// w[r] for every row of the basis (blk[L] rows): kind is PACES_WEIGHT_COHERENCE, _NORM or
// _HAM_ONES.
int launch_lookahead(bool c64, const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta,
                     const void* psi, double tau, int kind, double* w, int* status, int num_sms, cudaStream_t st);

// ---- batched Taylor: many trajectories in one persistent launch ---------------------------
constexpr int kMaxBatch = 128;  // trajectories per launch (the descriptors travel as kernel parameters)
// batches whose every evolving trajectory has room for at least this many states step their
// Taylor series through the single-trajectory kernel, one launch per trajectory
constexpr int64_t kBatchSingleCap = PACES_BATCH_SINGLE_CAP;
constexpr int kSqrtTable = 260; // sqrt(k) * g for k < 260 (occupations up to 255, plus one)
// One trajectory of a batched Taylor launch: its H (neighbour table + metadata), vectors,
// model constants and where its results go.  Field names follow ModelDev so the row
// helpers take either.
struct TaylorItem {
    const int* blk;            // [L+1]; blk[L] = rows
    const int* nbr;            // [rows][4]
    const uint32_t* meta;      // [rows]
    const void* v_in;          // input state
    void* res;                 // output state
    void* ta;                  // term buffers [cap]
    void* tb;
    const double* site_eps;    // [L] device (read when has_site_eps)
    const double* sq;          // [kSqrtTable] sqrt(k) * g, fp64
    const float* sqf;          // [kSqrtTable] the same rounded to fp32
    int* status;               // the trajectory's status word
    double* diag;              // null, or the trajectory's diag buffer (first-sweep diagnostics)
    TaylorOut out;
    double dt, tol, eps_sys, hbar_omega, delta_eps, J;
    int L, has_site_eps, m_star, pad;
};
struct TaylorBatch {
    TaylorItem items[kMaxBatch];
    int n;
    int max_m_star;
};
struct TaylorBatchWs {
    unsigned* barrier;             // [2]
    unsigned long long* maxima;    // [3][kMaxBatch][4] per-term maxima (fp64 bit patterns)
    uint64_t wait_ns;              // grid-barrier wait limit (kWaitLimitNs unless a test shortens it)
    int skip_block;                // test hook: this block skips its first grid-barrier arrival (-1: none)
};
constexpr size_t kTaylorBatchWsBytes = 256 + size_t(3) * kMaxBatch * 4 * 8;
int taylor_batch_max_grid(bool c64, int num_sms);
int launch_taylor_batch(bool c64, const TaylorBatch& bt, const TaylorBatchWs& ws, int num_sms,
                        int blocks_per_sm, cudaStream_t st);

// ---- observables --------------------------------------------------------------------------
struct ObsTarget {
    double* norm;        // may be null
    double* energy_re;
    double* energy_im;
    double* n_exc;       // [L] or null
    double* n_pho;       // [L] or null
};
// Norm and energy from a diag buffer filled by the first sweep of a Taylor launch (rows:
// blk[L]; cap: the buffer's row capacity).  Two launches.
int launch_diag_final(const double* diag, const int* blk, int L, int64_t cap, const ObsTarget& out, cudaStream_t st);
constexpr int kObsGridPerSm = 4;
inline int obs_max_grid(int num_sms) { return num_sms * kObsGridPerSm; }
int launch_observables(int nw, bool c64, const ModelDev& m, const uint64_t* keys, const int* blk,
                       const int* nbr, int64_t nbr_cap, const uint32_t* meta, const void* psi,
                       int what, double* partials, const ObsTarget& out, int num_sms,
                       cudaStream_t st);
int launch_scale(bool c64, const ModelDev& m, const int* blk, void* psi, const double* norm,
                 int num_sms, cudaStream_t st);
// Per exciton position the hopping and vibronic energies (re, im) and the phonon-vacuum
// amplitude sum: out[4L + 2] = hop re[L], hop im[L], vib re[L], vib im[L], vacuum re, im.
int launch_term_energies(bool c64, const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta,
                         const void* psi, double* partials, double* out, int num_sms, cudaStream_t st);
int launch_apply_h(bool c64, const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta,
                   const void* x, void* y, int num_sms, cudaStream_t st);

// ---- lookup and layout conversion -------------------------------------------------------
struct RefLayout {
    int words;                    // uint32 words per reference row
    int nfields;                  // L + 1 (field 0 = exciton position)
    int off[kMaxSites + 1];       // bit offset of each field from the row's MSB
    int bits[kMaxSites + 1];
};
constexpr int kMaxRefWords = 40;
int launch_lookup(int nw, const ModelDev& m, const uint64_t* pk, const int* pblk,
                  const uint64_t* qk, const int* qpos, int64_t nq, int must_exist, int64_t* out,
                  int* status, int num_sms, cudaStream_t st);
int launch_keys_to_ref(int nw, const ModelDev& m, const RefLayout& rl, const uint64_t* keys,
                       const int* blk, uint32_t* ref, int num_sms, cudaStream_t st);
int launch_keys_from_ref(int nw, const ModelDev& m, const RefLayout& rl, const uint32_t* ref,
                         int64_t n, uint64_t* keys, int* pos, int* status, int num_sms,
                         cudaStream_t st);

}  // namespace paces
