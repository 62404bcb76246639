/*
 * paces_b200.h -- C ABI of libpaces_b200.so, the sm_100a implementation of the
 * paces adaptive-basis time step (truncate -> expand -> sort/unique -> lookup ->
 * assemble H -> expm-multiply -> observables) for the single-exciton Holstein chain.
 *
 * Conventions
 *   - Every entry point returns an int status (PACES_OK == 0).  Errors raised
 *     inside kernels (capacity overflow, failed lookup, non-finite values, a
 *     bounded wait that ran out) are written to the device-side status word of
 *     the step record / context and returned by the next call that reads it.
 *   - Device buffers are owned by the caller.  No entry point allocates device
 *     memory except paces_create (4 KB of status words and model constants) and
 *     paces_batch_create (a few KB of Taylor scratch).
 *     Scratch comes from a caller-provided workspace sized by
 *     paces_workspace_bytes.
 *   - All work is enqueued on the caller's stream; nothing synchronises the
 *     host except paces_read_record-style helpers the caller invokes itself.
 *   - A context is not re-entrant: one host thread/stream per context.
 *
 * Basis layout (device)
 *   A basis is a set of states (pos, n_0..n_{N-1}) sorted lexicographically,
 *   stored blocked by exciton position: keys[i] holds only the phonon
 *   occupations, packed MSB-first into `nw` uint64 words (fields never
 *   straddle a word); blk[p] is the index of the first state with pos == p and
 *   blk[nchain] is the number of states.  Within a block, uint64-word order is
 *   the lexicographic order of (n_0, ..., n_{N-1}), so (pos, words) order is
 *   the reference's MSB-first uint32 row order.  paces_keys_to_ref /
 *   paces_keys_from_ref convert to and from the reference's whoami layout.
 *
 * Reference interfaces replaced (paths within rkevk/paces 1.2.0):
 *   paces_expand       HamiltonianFramework.enlarge_basis_set  paces/core/hamiltonian.py:550-577
 *                      + cupy_unique                          paces/aux/helpers.py:63-75
 *   paces_assemble     HamiltonianFramework.generate_mel       paces/core/hamiltonian.py:383-547
 *                      + TimeEvolutionFramework.create_matrices paces/core/time_evolution.py:365-372
 *   paces_truncate     _determine_select_whoami                paces/core/time_evolution.py:833-910
 *   paces_truncate_weighted  the same with use_weight_function     paces/core/time_evolution.py:854-857
 *   paces_lookahead_weights  coherence_weighting_func / norm_weighting_func / total_ham_ones
 *                                                             paces/core/time_evolution.py:464-476, :403-420
 *   paces_remap        vector remap in _generate_new_hilbert_space_cupy
 *                                                             paces/core/time_evolution.py:781-797
 *   paces_taylor       _simple_taylor + total_ham              paces/core/time_evolution.py:482-512, :382-400
 *   paces_term_energies calculate_hopping / calculate_coupling / calculate_mu_to_0 sums
 *                                                             paces/models/holstein.py:325-377
 *   paces_observables  calculate_n_exc / calculate_n_pho / calculate_total_energy / norm
 *                      paces/models/holstein.py:299-322, paces/core/observables.py:95-99,
 *                      paces/core/time_evolution.py:585-602
 *   paces_lookup       searchsorted_full_binary                paces/aux/cupy_search.py:78-93
 *   paces_step         TimeEvolutionFramework._evolve_single_step / _perform_first_step
 *                      paces/core/time_evolution.py:552-650
 */
#ifndef PACES_B200_H
#define PACES_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *paces_stream_t; /* a cudaStream_t */

enum paces_status {
    PACES_OK = 0,
    PACES_ERR_CAPACITY = 1,   /* a result did not fit the caller's buffers: grow and retry */
    PACES_ERR_LOOKUP = 2,     /* a state that must be present in a basis was not found */
    PACES_ERR_NONFINITE = 3,  /* NaN/Inf amplitudes */
    PACES_ERR_TIMEOUT = 4,    /* a bounded device-side wait ran out */
    PACES_ERR_BADARG = 5,
    PACES_ERR_CUDA = 6,       /* a CUDA runtime call failed (see paces_last_error) */
    PACES_ERR_EXPLOSION = 7,  /* norm above ExpmParams.explosion_cutoff */
    PACES_ERR_SHUFFLE = 8     /* tie shuffle would touch > 90% of the states */
};

enum paces_precision {
    PACES_C128 = 0, /* complex128 amplitudes, float64 matrix elements (reference precision) */
    PACES_C64 = 1   /* complex64 amplitudes/SpMV with fp32 accumulation; fp64 norms and scalars */
};

#define PACES_MAX_SITES 128
/* largest ExpmParams.lanczos_order (Krylov vectors: order + 1) */
#define PACES_MAX_LANCZOS_ORDER 63
#define PACES_BATCH_SINGLE_CAP (1 << 25)

typedef struct paces_model_desc {
    int32_t nchain;            /* number of sites L (1D chain), 1 <= L <= 128 */
    int32_t periodic;          /* 0: open chain (reference); 1: ring (L >= 3) */
    int32_t precision;         /* enum paces_precision */
    int32_t reserved;
    const int32_t *max_ho_dims; /* host array, nchain entries, 2..256 */
    double eps_sys;            /* use_terms["diag"]["eps_sys"] */
    double hbar_omega;         /* use_terms["diag"]["hbar_omega"] */
    double delta_eps;          /* use_terms["diag"]["delta_eps"] */
    double J;                  /* use_terms["hopping"]["J"] (real) */
    double g;                  /* use_terms["vib_coupling"]["g"] (real) */
    const double *site_eps;    /* host array of nchain per-site energies, or NULL */
    /* lattices (paces/models/holstein.py:24-51, :150-240): geo_dim (0 or 1: chain) lattice
     * dimensions of side l = nchain^(1/geo_dim), hopping along every dimension; hopping2 != 0
     * adds the next-nearest-neighbour term use_terms["hopping2"]["J2"] (needs l >= 3).  Both
     * need open boundaries. */
    int32_t geo_dim;
    int32_t hopping2;
    double J2;
} paces_model_desc;

typedef struct paces_ctx paces_ctx;

typedef struct paces_basis {
    uint64_t *keys; /* device [cap][nw] */
    int32_t *blk;   /* device [nchain+1]; blk[nchain] = number of states */
    int64_t cap;    /* capacity in states */
} paces_basis;

/* H on a basis: neighbour table + per-row metadata.  nbr[4*r + k] (16 bytes per row) is the
 * row index of the k-th neighbour of row r (k: 0 = exciton one site left, 1 = right, 2 = one phonon
 * less at the exciton site, 3 = one phonon more), or -1 when that coupling is absent from
 * the reference's H (both rows outside the enlarged basis, or a boundary/ceiling/floor).
 * meta[r] = pos | n_exc << 8 | n_total << 16, from which the diagonal element is
 * eps_sys + hbar_omega*n_total (+ delta_eps*pos) (+ site_eps[pos]). */
typedef struct paces_hmat {
    int32_t *nbr;
    uint32_t *meta;
    int64_t cap;
    /* lattices with more than one hopping channel (paces_hop_channels > 1): the other
     * channels' neighbours, xnbr[2*(c-1)*cap + 2*r + {0,1}] = row of the state with the
     * exciton moved by -/+ the distance of channel c (-1: absent); NULL otherwise */
    int32_t *xnbr;
} paces_hmat;

typedef struct paces_step_params {
    int64_t maxstates;       /* TimeEvoParams.maxstates */
    int32_t enlarge_steps;   /* TimeEvoParams.enlarge_steps */
    int32_t evolve;          /* 0: first step (no propagation), 1: propagate by dt */
    double dt;
    int32_t m_star;          /* ExpmParams.m_star */
    int32_t diagnostics;     /* TimeEvoParams.diagnostics: post-remap norm and energy */
    double tol;              /* Taylor stop tolerance (2^-53 for C128, 2^-24 for C64) */
    int32_t shuffle;         /* 1: shuffle equal-weight states at the cut (shuffle_seed set) */
    int32_t renormalize;     /* ExpmParams.renormalize */
    uint64_t shuffle_seed;
    uint64_t step_index;     /* mixes into the shuffle stream */
    double explosion_cutoff; /* ExpmParams.explosion_cutoff */
    /* learned proposal (no counterpart in the reference): with proposal != 0 the first
     * enlargement keeps only the images the MLP at proposal_params (paces_mlp_param_bytes
     * bytes, device) scores above proposal_threshold */
    int32_t proposal;
    float proposal_threshold;
    const void *proposal_params;
    /* look-ahead weighting (TimeEvoParams.weighting_name / tau; the reference applies it
     * from the second time step on, time_evolution.py:560): weighting = PACES_WEIGHT_NONE
     * ranks the states by |psi|, PACES_WEIGHT_COHERENCE / PACES_WEIGHT_NORM by the weights
     * paces_lookahead_weights computes with tau (non-zero) and old_h, the neighbour table of
     * old_basis (what the previous step wrote into its h).  old_h may be h itself: the step
     * reads it before it writes h, but then a step that fails leaves no table to retry from.
     * Not combined with the learned proposal. */
    int32_t weighting;
    int32_t reserved0;
    double tau;
    const paces_hmat *old_h;
    /* ExpmParams.lanczos_order: with lanczos_order > 0 the propagation is the Lanczos step
     * (paces_lanczos) in the caller's Krylov workspace krylov (paces_lanczos_bytes for the
     * new basis' capacity and this order); the record's Taylor fields are 0, as the
     * reference's placeholder diagnostics. */
    int32_t lanczos_order;
    int32_t reserved1;
    void *krylov;
    size_t krylov_bytes;
    /* NULL, or a CUDA event (cudaEvent_t) that the step records on its stream as soon as
     * new_b (keys, block offsets) and h are final, after the assembly and before the remap
     * and the propagation, which no longer write them.  Another stream that waits on it can
     * copy the new basis to the host while the propagation runs.  Under stream capture
     * the record is an external event node, recorded at every replay.  A step that fails
     * before that point does not record it. */
    void *basis_ready;
} paces_step_params;

/* Written on the device by paces_step; the caller copies it back (one transfer per step). */
typedef struct paces_step_record {
    int32_t status;          /* first error raised by a kernel of this step */
    int32_t n_select;        /* states kept by the truncation */
    int32_t n_enlarged;      /* size of the enlarged basis the matrix elements come from */
    int32_t n_states;        /* size of the new basis (numstates) */
    int32_t converged;       /* Taylor: stop criterion met */
    int32_t final_m;         /* Taylor: index of the last term (j_ind) */
    int32_t ceiling_hits;    /* enlarged-basis states at the phonon ceiling */
    int32_t n_tied;          /* states tied with the truncation threshold */
    int32_t n_candidates;    /* proposal: images scored (existing ones) */
    int32_t n_candidates_kept; /* proposal: images kept */
    double c1_plus_c2;
    double term_ratio;
    double post_adapt_norm;  /* -1 when diagnostics are off */
    double post_adapt_energy_re;
    double post_adapt_energy_im;
    double norm;
    double energy_re;
    double energy_im;
    double n_exc[PACES_MAX_SITES];
    double n_pho[PACES_MAX_SITES];
} paces_step_record;

/* Taylor diagnostics (device), as returned by _simple_taylor (time_evolution.py:510-511). */
typedef struct paces_expm_info {
    int32_t converged;
    int32_t final_m;
    double c1_plus_c2;
    double term_ratio;
} paces_expm_info;

/* Observables (device output of paces_observables): [0] norm, [1] energy re, [2] energy im,
 * [3 .. 3+L) n_exc, [3+L .. 3+2L) n_pho.  `what` is a bit set of PACES_OBS_*. */
enum { PACES_OBS_NORM = 1, PACES_OBS_ENERGY = 2, PACES_OBS_SITES = 4 };

/* Truncation weights (paces_lookahead_weights, paces_step_params.weighting):
 *   COHERENCE  |psi|^2 + tau^2 |psi|^2 (H 1)^2   coherence_weighting_func  time_evolution.py:464-469
 *   NORM       |psi - 1j tau H psi|              norm_weighting_func       time_evolution.py:472-476
 *   HAM_ONES   H 1 (signed; not a ranking)       total_ham_ones            time_evolution.py:403-420 */
enum { PACES_WEIGHT_NONE = 0, PACES_WEIGHT_COHERENCE = 1, PACES_WEIGHT_NORM = 2, PACES_WEIGHT_HAM_ONES = 3 };

/* ---- context ----------------------------------------------------------------------- */
int paces_create(const paces_model_desc *desc, paces_ctx **out);
/* Hopping channels of the context's model: geo_dim for the hopping term, twice that with
 * hopping2 (1 for the chain).  An H table of a model with more than one needs xnbr. */
int paces_hop_channels(const paces_ctx *ctx);
int paces_destroy(paces_ctx *ctx);
const char *paces_last_error(const paces_ctx *ctx);
int paces_key_words(const paces_ctx *ctx);         /* nw: uint64 words per key */
int paces_ref_words(const paces_ctx *ctx);         /* uint32 words per reference row */
/* Internal key layout, nchain entries each: word index, LSB position, field width of site s. */
int paces_key_layout(const paces_ctx *ctx, int32_t *word, int32_t *shift, int32_t *bits);
int paces_version(void);                            /* 10000*major + 100*minor + patch */
/* Copy the context's device status word (errors raised by kernels of the stage entry points)
 * to the host, synchronising `stream`, and clear it. */
int paces_read_status(paces_ctx *ctx, paces_stream_t stream, int32_t *host_status);
/* Rows of `words` uint32 (1..16) in the reference's whoami layout, compared lexicographically
 * (word 0 most significant); no context needed.  For the host API (the time step itself
 * never searches or sorts rows).
 * paces_rows_lower_bound replaces searchsorted_full_binary (paces/aux/cupy_search.py:78-93):
 * out[i] = lower bound of query row i in the sorted rows of pb (n when beyond the end); with
 * allow_escapes == 0 a query that is not present sets *dev_missing (device int) to 1 instead
 * of the reference's device assert (:205-228).
 * paces_rows_sort_unique replaces cupy_unique (paces/aux/helpers.py:63-75): the sorted unique
 * rows of `rows` into out (room for n rows) and their number into *dev_count (device),
 * using a caller-owned workspace of paces_rows_sort_bytes(n) bytes; n < 2^31. */
int paces_rows_lower_bound(const uint32_t *pb, int64_t n, const uint32_t *q, int64_t nq, int32_t words,
                           int32_t allow_escapes, int64_t *out, int32_t *dev_missing, paces_stream_t stream);
size_t paces_rows_sort_bytes(int64_t n);
int paces_rows_sort_unique(const uint32_t *rows, int64_t n, int32_t words, uint32_t *out, int64_t *dev_count,
                           void *ws, size_t ws_bytes, paces_stream_t stream);
/* Lanczos propagation: replaces _lanczos (paces/core/time_evolution.py:515-549), selected
 * by ExpmParams.lanczos_order = order (1 .. PACES_MAX_LANCZOS_ORDER, :577-578).  psi_out =
 * |psi| V exp(-i dt T) e_0 from order + 1 Lanczos vectors of H on the basis (fewer when
 * the Krylov space closes, beta < 1e-15), all in one cooperative launch: the Krylov
 * vectors in the precision of the context, alpha, beta and the small exponential in fp64.
 * dev_info (device, may be NULL) receives the reference's placeholder diagnostics
 * [0, 0, 0, 0].  krylov is a caller-owned device buffer of paces_lanczos_bytes(cap,
 * order) bytes with cap >= basis->cap; no other workspace is needed. */
int paces_lanczos_bytes(const paces_ctx *ctx, int64_t cap, int32_t order, size_t *bytes);
int paces_lanczos(paces_ctx *ctx, const paces_basis *basis, const paces_hmat *h, const void *psi_in,
                  void *psi_out, double dt, int32_t order, paces_expm_info *dev_info, void *krylov,
                  size_t krylov_bytes, paces_stream_t stream);
/* Test hook for the bounded device waits that replace the reference's device assert
 * (paces/aux/cupy_search.py:205-228 traps; this library raises PACES_ERR_TIMEOUT and returns).
 * wait_limit_ns (0 = the default 2 s, at most 2 s) bounds each grid-barrier wait of this
 * context's Taylor and scaling-and-squaring kernels; skip_barrier_block >= 0 makes that block
 * give up at its first grid barrier without arriving, so every other block's wait runs out
 * (-1 = off); the Lanczos kernel's grid barriers obey the same hooks.  Results are
 * unaffected while the hooks are off. */
int paces_set_test_hooks(paces_ctx *ctx, uint64_t wait_limit_ns, int32_t skip_barrier_block);
/* Stage timing (no counterpart in the reference, which only prints wall-clock times):
 * with profiling on, paces_step records CUDA events between its stages, and
 * paces_stage_times waits for the last step and returns 7 durations in ms: truncate,
 * expand, assemble, remap, diagnostics, Taylor, observables. */
int paces_set_profiling(paces_ctx *ctx, int32_t on);
int paces_stage_times(paces_ctx *ctx, float *ms);
/* Number of kernels paces_step has enqueued on this context so far. */
unsigned long long paces_kernel_launches(const paces_ctx *ctx);
/* Launch shapes (no counterpart in the reference): the merge tiles' splitter strides
 * (tile size = 17 * stride elements; one for the expansions, one for the assembly), the
 * Taylor kernel's blocks per SM and its row schedule.  Results do
 * not depend on them; paces_b200.autotune picks them by timing the live workload.
 * paces_get_tuning also reports the allowed ranges; paces_set_tuning rejects values
 * outside them with PACES_ERR_BADARG. */
typedef struct paces_tuning {
    int32_t merge_stride;              /* multiple of 16 in [merge_stride_min, merge_stride_max] */
    int32_t taylor_blocks_per_sm;      /* 0 = as many as fit, else 1..taylor_blocks_per_sm_max */
    int32_t merge_stride_min;          /* read only */
    int32_t merge_stride_max;          /* read only */
    int32_t taylor_blocks_per_sm_max;  /* read only */
    int32_t taylor_variant;            /* 0: rows read directly; 1: 512-row chunks prefetched by bulk copies */
    int32_t assemble_stride;           /* the assembly's stride, same range; 0 on set: merge_stride */
    int32_t reserved[1];
} paces_tuning;
int paces_get_tuning(const paces_ctx *ctx, paces_tuning *t);
int paces_set_tuning(paces_ctx *ctx, const paces_tuning *t);
/* Workspace bytes for every entry point on bases of up to `cap` states. */
int paces_workspace_bytes(const paces_ctx *ctx, int64_t cap, size_t *bytes);

/* ---- layout conversion --------------------------------------------------------------- */
/* Reference rows (pos in the leading bits, MSB-first uint32 words, ref_words per row) ->
 * keys + positions.  Rows need not be sorted. */
int paces_keys_from_ref(paces_ctx *ctx, const uint32_t *ref, int64_t n, int32_t ref_words,
                        uint64_t *keys_out, int32_t *pos_out, paces_stream_t stream);
/* A basis -> reference rows (ref_words uint32 per row). */
int paces_keys_to_ref(paces_ctx *ctx, const paces_basis *b, int32_t ref_words, uint32_t *ref_out,
                      paces_stream_t stream);

/* ---- stages -------------------------------------------------------------------------- */
/* Every stage uses its workspace `ws` as scratch: no input or output may lie inside it. */
int paces_expand(paces_ctx *ctx, const paces_basis *in, paces_basis *out, void *ws,
                 size_t ws_bytes, paces_stream_t stream);
int paces_assemble(paces_ctx *ctx, const paces_basis *in, paces_basis *out, paces_hmat *h,
                   int32_t *dev_ceiling_hits, void *ws, size_t ws_bytes, paces_stream_t stream);
int paces_truncate(paces_ctx *ctx, const paces_basis *in, const void *psi, int64_t maxstates,
                   int32_t shuffle, uint64_t shuffle_seed, uint64_t step_index,
                   paces_basis *out, void *ws, size_t ws_bytes, paces_stream_t stream);
/* The look-ahead weights of the states of b (dev_weights: one double per state) from psi
 * and b's neighbour table h; `weighting` is a PACES_WEIGHT_* other than NONE. */
int paces_lookahead_weights(paces_ctx *ctx, const paces_basis *b, const paces_hmat *h, const void *psi,
                            double tau, int32_t weighting, double *dev_weights, paces_stream_t stream);
/* paces_truncate ranking by dev_weights (non-negative, one per state of `in`) instead of
 * |psi|: _determine_select_whoami with use_weight_function (time_evolution.py:854-857). */
int paces_truncate_weighted(paces_ctx *ctx, const paces_basis *in, const double *dev_weights,
                            int64_t maxstates, int32_t shuffle, uint64_t shuffle_seed,
                            uint64_t step_index, paces_basis *out, void *ws, size_t ws_bytes,
                            paces_stream_t stream);
int paces_remap(paces_ctx *ctx, const paces_basis *old_b, const void *old_psi,
                const paces_basis *new_b, void *new_psi, void *ws, size_t ws_bytes,
                paces_stream_t stream);
/* paces_remap without a workspace.  No counterpart in the reference (which allocates
 * through CuPy's pool on every call).  For callers that cannot allocate device memory
 * at all: a host application that owns the whole device through its own memory pool, or
 * a latency-critical loop that must not call cudaMalloc (it can synchronise the device).
 * The scratch is a 512 KiB array in the library's static device memory, held by every
 * GPU that loads the library until the process exits; it bounds the two bases together
 * to about 64M states (1024 per remap tile for keys of 1-4 words, 512 beyond).  Capacities beyond that return PACES_ERR_CAPACITY before anything is
 * launched.  The first call in each CUDA context (a device's primary context, or one the
 * host made current) looks up the array's device address in that context: make it before
 * any stream capture.  A context destroyed and replaced by a new one at the same handle
 * keeps the cached address, so do not call this after destroying a context.  All calls share the one array, so
 * calls that overlap on the GPU (other streams, other threads) race: serialise them. */
int paces_remap_noalloc(paces_ctx *ctx, const paces_basis *old_b, const void *old_psi,
                        const paces_basis *new_b, void *new_psi, paces_stream_t stream);
int paces_taylor(paces_ctx *ctx, const paces_basis *b, const paces_hmat *h, const void *psi_in,
                 void *psi_out, double dt, int32_t m_star, double tol,
                 paces_expm_info *dev_info, void *ws, size_t ws_bytes, paces_stream_t stream);
int paces_observables(paces_ctx *ctx, const paces_basis *b, const paces_hmat *h, const void *psi,
                      int32_t what, double *dev_out, void *ws, size_t ws_bytes,
                      paces_stream_t stream);
/* Per exciton position p (0..L-1) the energies of the hopping term and of the vibronic
 * coupling, sum over the rows r of block p of conj(psi_r) (H_term psi)_r, and the sum of the
 * amplitudes of the phonon-vacuum states: dev_out[4L + 2] = hop re[L], hop im[L], vib re[L],
 * vib im[L], vacuum re, vacuum im.  The partitioned sums of calculate_hopping /
 * calculate_coupling and the value of calculate_mu_to_0 (paces/models/holstein.py:325-377). */
int paces_term_energies(paces_ctx *ctx, const paces_basis *b, const paces_hmat *h, const void *psi,
                        double *dev_out, void *ws, size_t ws_bytes, paces_stream_t stream);
/* Norms for the scaling-and-squaring propagation: dev_out[0] = trace of H, dev_out[1] =
 * the largest row 1-norm of H - (*dev_shift) I (0 when dev_shift is NULL), dev_out[2] =
 * trace / n (three doubles, device).  Reference: _trace and _exact_1_norm,
 * paces/aux/_scipy/_expm_multiply.py:23-40, applied to 1j * H in expm_multiply_simple
 * (:106-160); H is symmetric, so its column and row 1-norms agree. */
int paces_hnorms(paces_ctx *ctx, const paces_basis *b, const paces_hmat *h, const double *dev_shift,
                 double *dev_out, void *ws, size_t ws_bytes, paces_stream_t stream);
/* psi_out = exp(t A) psi_in with A = 1j * (H - shift I), by `stages` stages of at most
 * m_star Taylor terms each, stopping a stage by the inf-norm test at tol, and multiplying
 * by eta = eta_re + 1j eta_im (exp(t mu / stages) for the removed mean mu = 1j * shift)
 * after every stage.  dev_info gets converged, final_m (terms over all stages), the last
 * c1 + c2 and term ratio.  Reference: _expm_multiply_simple_core,
 * paces/aux/_scipy/_expm_multiply.py:163-202, called with 1j * H and t = dt by
 * paces/core/time_evolution.py:579-581.  The host picks stages and m_star
 * (paces_b200.expm). */
int paces_expm_scaled(paces_ctx *ctx, const paces_basis *b, const paces_hmat *h, const void *psi_in,
                      void *psi_out, double t, double shift, int32_t m_star, int32_t stages, double tol,
                      double eta_re, double eta_im, paces_expm_info *dev_info, void *ws, size_t ws_bytes,
                      paces_stream_t stream);
/* y = H x on a basis (x and y distinct).  Reference: TimeEvolutionFramework.total_ham,
 * paces/core/time_evolution.py:382-400. */
int paces_apply_h(paces_ctx *ctx, const paces_basis *b, const paces_hmat *h, const void *x, void *y,
                  paces_stream_t stream);
/* Lower-bound lookup of (pos, key) queries in a basis; out[i] = row index or -1 if absent.
 * With must_exist != 0 a miss also raises PACES_ERR_LOOKUP (reference: noesc kernel). */
int paces_lookup(paces_ctx *ctx, const paces_basis *phonebook, const uint64_t *q_keys,
                 const int32_t *q_pos, int64_t nq, int32_t must_exist, int64_t *out,
                 void *ws, size_t ws_bytes, paces_stream_t stream);

/* One full time step: truncate(old) -> expand^enlarge_steps -> assemble -> remap ->
 * [diagnostics] -> [Taylor] -> observables.  The old basis and amplitudes are read only;
 * the new basis, new amplitudes, h and rec are written.
 * Returns PACES_OK once enqueued; kernel-side errors land in rec->status. */
int paces_step(paces_ctx *ctx, const paces_basis *old_b, const void *old_psi, paces_basis *new_b,
               void *new_psi, paces_hmat *h, const paces_step_params *prm,
               paces_step_record *dev_rec, void *ws, size_t ws_bytes, paces_stream_t stream);

/* ---- learned proposal (no counterpart in the reference) ------------------------------
 * Events of a basis X (nx states): e = (j-1)*nx + i, the image of state i under run j =
 * 1 (exciton hops right), 2 (hops left), 3 (phonon created at the exciton site), 4
 * (annihilated).  Features, network and keep rule are documented in
 * paces_b200/csrc/proposal.cuh.  The MLP's packed inference parameters are
 * paces_mlp_param_bytes() bytes of device memory; its fp32 master weights (and
 * gradients, and Adam moments) paces_mlp_master_floats() floats. */
size_t paces_mlp_param_bytes(void);
int32_t paces_mlp_master_floats(void);
/* The truncated basis of the last paces_step that used this workspace, its amplitudes
 * |psi| (float, one per state) and the cut (one float: the smallest kept |psi|, 0 when the
 * truncation dropped nothing); views into the workspace, valid until its next use. */
int paces_selected_view(const paces_ctx *ctx, void *ws, size_t ws_bytes, paces_basis *sel, float **weights,
                        float **cut);
/* Score every event of X with the MLP on the tensor cores: keep[j*keep_cap + i] (j = 1..4)
 * = logit > threshold (every existing image when *cut == 0), logits[e] (optional),
 * counts[0..1] += existing / kept events (optional).  Any of keep, logits, counts may be
 * NULL; weights and cut are device pointers. */
int paces_proposal_score(paces_ctx *ctx, const paces_basis *x, const float *weights, const float *cut,
                         const void *params, float threshold, uint8_t *keep, int64_t keep_cap, float *logits,
                         int32_t *counts, paces_stream_t stream);
/* Features of every event as bf16 [4*nx][16] and whether the image exists [4*nx]. */
int paces_proposal_features(paces_ctx *ctx, const paces_basis *x, const float *weights, const float *cut,
                            uint16_t *feats, uint8_t *valid, paces_stream_t stream);
/* Training labels of X's events against the next truncated basis Y: 1 image in Y, 0 not,
 * 255 image already in X (not a candidate), 254 image does not exist. */
int paces_proposal_labels(paces_ctx *ctx, const paces_basis *x, const paces_basis *y, uint8_t *labels,
                          paces_stream_t stream);
/* fp32 master weights -> packed inference parameters. */
int paces_mlp_pack(const float *master, void *params, paces_stream_t stream);
/* logits of n feature rows (bf16 [n][16]) -- CUDA cores, the reference for the scorer. */
int paces_mlp_forward(const void *params, const uint16_t *x, int64_t n, float *logits, paces_stream_t stream);
/* grads += d/dw of inv_norm * sum_s sw[s] * BCE(logit_s, y[s]); loss += that loss (double). */
int paces_mlp_backward(const void *params, const uint16_t *x, const float *y, const float *sw, int64_t n,
                       float inv_norm, float *grads, double *loss, paces_stream_t stream);
/* One Adam step (step t >= 1) on the master weights; writes the packed parameters and
 * clears the gradients. */
int paces_mlp_adam(float *master, float *m1, float *m2, float *grads, int32_t t, float lr, float beta1,
                   float beta2, float eps, void *params, paces_stream_t stream);

/* ---- batched trajectories (no counterpart in the reference, which runs one trajectory
 * per process) ------------------------------------------------------------------------
 * paces_batch_step advances up to 128 independent trajectories -- each with its own
 * context (model, key width, dt, maxstates), buffers and record -- by one time step.
 * The per-trajectory truncation, enlargement, assembly, remap and observables are spread
 * over the batch's own streams (forked from and joined back into `stream`, so the whole
 * call can be captured into one CUDA graph); the Taylor series of every trajectory runs
 * in ONE persistent cooperative launch -- unless every evolving trajectory's new basis
 * has room for PACES_BATCH_SINGLE_CAP states or more, when each runs through paces_step's
 * kernel in turn (its schedule streams long row ranges faster).  Each trajectory's results
 * are bit-identical to paces_step on the same inputs.  All contexts share one precision and device.  Item
 * errors land in each record's status; a non-OK return names the item in
 * paces_batch_last_error. */
typedef struct paces_batch paces_batch;
typedef struct paces_batch_item {
    paces_ctx *ctx;
    const paces_basis *old_basis;
    const void *old_psi;
    paces_basis *new_basis;
    void *new_psi;
    paces_hmat *h;
    const paces_step_params *params;
    paces_step_record *record;   /* device */
    void *workspace;
    size_t workspace_bytes;
} paces_batch_item;
/* max_items <= 128; n_streams in [1, 64] (allocates the Taylor scratch, a few KB). */
int paces_batch_create(int32_t max_items, int32_t n_streams, paces_batch **out);
int paces_batch_destroy(paces_batch *batch);
int paces_batch_step(paces_batch *batch, const paces_batch_item *items, int32_t n,
                     paces_stream_t stream);
const char *paces_batch_last_error(const paces_batch *batch);
/* Number of kernels paces_batch_step has enqueued on this batch so far. */
unsigned long long paces_batch_kernel_launches(const paces_batch *batch);
/* With profiling on (not under stream capture), paces_batch_step records events around
 * its three phases; paces_batch_stage_times waits for the last step and returns their
 * durations in ms: per-trajectory front stages, the batched Taylor launch, back stages. */
int paces_batch_set_profiling(paces_batch *batch, int32_t on);
/* The same test hook for the batch's persistent Taylor launch (paces_set_test_hooks). */
int paces_batch_set_test_hooks(paces_batch *batch, uint64_t wait_limit_ns, int32_t skip_barrier_block);
int paces_batch_stage_times(paces_batch *batch, float *ms);

#ifdef __cplusplus
}
#endif
#endif /* PACES_B200_H */
