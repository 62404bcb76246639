// C ABI of libpaces_b200 (declared in include/paces_b200.h).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "kernels.cuh"
#include "proposal.cuh"

using namespace paces;

struct paces_ctx {
    ModelDev m;
    RefLayout rl;
    int nw;
    int precision;
    int device;
    int num_sms;
    int taylor_grid;
    int merge_stride;     // tuning: elements per splitter of the expansions' merge tiles
    int assemble_stride;  // tuning: the same for the assembly
    int taylor_bps;    // tuning: Taylor blocks per SM (0 = as many as fit)
    int taylor_variant;  // tuning: 0 direct rows, 1 bulk-prefetched chunks
    int* d_status;  // device status word for the stage entry points (start of the constants block)
    double* d_site_eps;  // [kMaxSites] per-site energies, device copy (batched Taylor)
    double* d_sq;        // [kSqrtTable] sqrt(k) * g
    float* d_sqf;        // [kSqrtTable] the same rounded to fp32
    int profiling;  // record stage events in paces_step
    cudaEvent_t ev[8];
    unsigned long long launches;  // kernels launched by paces_step since creation
    uint64_t test_wait_ns;   // test hook: grid-barrier wait limit of the Taylor kernels (0: kWaitLimitNs)
    int test_skip_block;     // test hook: block that skips its grid-barrier arrival (-1: none)
    char err[512];
};


struct paces_batch {
    int max_items;
    int n_streams;
    int device;
    int num_sms;
    cudaStream_t* streams;
    cudaEvent_t fork;
    cudaEvent_t* join;
    void* d_ws;                   // TaylorBatchWs: barrier words + per-term maxima
    TaylorBatch* desc;            // host staging of the launch descriptors
    int profiling;                // record events around the three phases of a batch step
    cudaEvent_t ev[4];
    unsigned long long launches;  // kernels enqueued by paces_batch_step
    uint64_t test_wait_ns;        // test hook: grid-barrier wait limit (0: kWaitLimitNs)
    int test_skip_block;          // test hook: block that skips its grid-barrier arrival (-1: none)
    char err[512];
};

namespace {

int fail(const paces_ctx* c, int code, const char* fmt, ...) {
    if (c) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(const_cast<paces_ctx*>(c)->err, sizeof(c->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

int cuda_fail(const paces_ctx* c, const char* where) {
    const cudaError_t e = cudaGetLastError();
    return fail(c, PACES_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

#define PACES_CHECK_LAUNCH(c, rc, where)                          \
    do {                                                          \
        const int _rc = (rc);                                     \
        if (_rc == PACES_ERR_CUDA) return cuda_fail((c), (where)); \
        if (_rc != PACES_OK) return fail((c), _rc, "%s failed", (where)); \
    } while (0)

// Workspace regions for bases of up to `cap` states.
struct Layout {
    size_t total = 0;
    int64_t cap = 0;
    size_t keysA, blkA, keysB, blkB, maps;
    size_t m_run_lo, m_run_len, m_split_off, m_tile_off, m_counters, m_split_co, m_split_rank, m_ord_co,
        m_tile_state, m_tile_desc;
    int64_t split_cap, tile_cap;
    size_t t_hist, t_cand, t_cand_idx, t_sel, t_tile_cnt, t_tile_pre;
    int t_tiles;
    size_t r_tile_off, r_counters, r_split;
    int r_tiles;
    size_t v_V, v_TA, v_TB, v_partials, v_bar;
    size_t o_partials, o_out;
    size_t aw, keep;  // kept amplitudes of the truncation, proposal keep mask [kRuns][cap]
    size_t maps_e, keysN, blkN, n2b;  // split expansion: its maps, the new part, new part -> output
    size_t maps_x;                    // lattices: maps of the assembly's passes 2 and 3
    size_t diag;                      // diagnostics folded by the first Taylor sweep (diag_group)
};

Layout make_layout(const paces_ctx* c, int64_t cap) {
    Layout l;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) & ~size_t(255);
        return o;
    };
    const int L = c->m.L, nw = c->nw;
    const size_t cs = c->precision == PACES_C64 ? 8 : 16;
    const size_t ucap = size_t(cap);
    l.cap = cap;
    l.keysA = take(ucap * nw * 8);
    l.blkA = take(size_t(L + 1) * 4);
    l.keysB = take(ucap * nw * 8);
    l.blkB = take(size_t(L + 1) * 4);
    l.maps = take(size_t(kRuns) * ucap * 4);
    l.split_cap = merge_split_cap(cap, nw, L);
    l.tile_cap = merge_tile_cap(l.split_cap, L);
    l.m_run_lo = take(size_t(L) * kRuns * 4);
    l.m_run_len = take(size_t(L) * kRuns * 4);
    l.m_split_off = take((size_t(L) * kRuns + 1) * 4);
    l.m_tile_off = take(size_t(L + 1) * 4);
    l.m_counters = take(16 * 4);
    l.m_split_co = take(size_t(l.split_cap) * kRuns * 4);
    l.m_split_rank = take(size_t(l.split_cap) * 4);
    l.m_ord_co = take(size_t(l.split_cap) * kRuns * 4);
    l.m_tile_state = take(size_t(l.tile_cap) * 8);
    l.m_tile_desc = take(size_t(l.tile_cap) * merge_desc_bytes());
    l.t_tiles = trunc_tiles_cap(cap);
    l.t_hist = take(4096 * 4);
    l.t_cand = take(ucap * 8);
    l.t_cand_idx = take(ucap * 4);
    l.t_sel = take(16 * 8);
    l.t_tile_cnt = take(size_t(l.t_tiles) * 3 * 4);
    l.t_tile_pre = take(size_t(l.t_tiles) * 3 * 4);
    l.r_tiles = remap_tile_cap(cap, nw, L);
    l.r_tile_off = take(size_t(L + 1) * 4);
    l.r_counters = take(16);
    l.r_split = take(size_t(l.r_tiles) * 2 * 4);
    l.v_V = take(ucap * cs);
    l.v_TA = take(ucap * cs);
    l.v_TB = take(ucap * cs);
    l.v_partials = take(size_t(2) * c->taylor_grid * 4 * 8);
    l.v_bar = take(16);
    l.o_partials = take(size_t(obs_max_grid(c->num_sms)) * (4 + 2 * L) * 8);
    l.o_out = take(size_t(3 + 2 * L) * 8);
    l.aw = take((ucap + 1) * 4);
    l.keep = take(size_t(kRuns) * ucap);
    l.maps_e = take(size_t(kRuns) * ucap * 4);
    const int passes = merge_passes(c->m);
    l.maps_x = take(passes > 2 ? size_t(passes - 2) * kRuns * ucap * 4 : 0);
    l.keysN = take(ucap * nw * 8);
    l.blkN = take(size_t(L + 1) * 4);
    l.n2b = take(ucap * 4);
    l.diag = take(diag_doubles(cap) * 8);
    l.total = off;
    return l;
}

// Largest capacity whose layout fits `bytes`.
Layout fit_layout(const paces_ctx* c, size_t bytes) {
    int64_t lo = 0, hi = int64_t(bytes / 8) + 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) / 2;
        if (make_layout(c, mid).total <= bytes) lo = mid; else hi = mid - 1;
    }
    return make_layout(c, lo);
}

template <typename T>
T* at(void* ws, size_t off) {
    return reinterpret_cast<T*>(static_cast<unsigned char*>(ws) + off);
}

// The model of a launch that reads the H table h: the extra channels' neighbours travel with it.
ModelDev with_h(const paces_ctx* c, const paces_hmat* h) {
    ModelDev m = c->m;
    m.xnbr = h ? reinterpret_cast<const int2*>(h->xnbr) : nullptr;
    m.xcap = h ? h->cap : 0;
    return m;
}

MergeWs merge_ws(const paces_ctx* c, const Layout& l, void* ws) {
    MergeWs w;
    w.run_lo = at<int>(ws, l.m_run_lo);
    w.run_len = at<int>(ws, l.m_run_len);
    w.split_off = at<int>(ws, l.m_split_off);
    w.tile_off = at<int>(ws, l.m_tile_off);
    w.counters = at<int>(ws, l.m_counters);
    w.split_co = at<int>(ws, l.m_split_co);
    w.split_rank = at<int>(ws, l.m_split_rank);
    w.ord_co = at<int>(ws, l.m_ord_co);
    w.tile_state = at<unsigned long long>(ws, l.m_tile_state);
    w.tile_desc = at<unsigned char>(ws, l.m_tile_desc);
    w.split_cap = int(l.split_cap);
    w.tile_cap = int(l.tile_cap);
    w.keep = nullptr;
    w.keep_cap = 0;
    merge_spec_standard(w, c->m);
    return w;
}

TruncWs trunc_ws(const Layout& l, void* ws) {
    TruncWs w;
    w.hist = at<unsigned>(ws, l.t_hist);
    w.cand = at<unsigned long long>(ws, l.t_cand);
    w.cand_idx = at<int>(ws, l.t_cand_idx);
    w.sel = at<long long>(ws, l.t_sel);
    w.tile_cnt = at<int>(ws, l.t_tile_cnt);
    w.tile_pre = at<int>(ws, l.t_tile_pre);
    w.cap = l.cap;
    w.ntiles_cap = l.t_tiles;
    return w;
}

RemapWs remap_ws(const Layout& l, void* ws) {
    RemapWs w;
    w.tile_off = at<int>(ws, l.r_tile_off);
    w.counters = at<int>(ws, l.r_counters);
    w.split = at<int>(ws, l.r_split);
    w.tile_cap = l.r_tiles;
    return w;
}

TaylorWs taylor_ws(const paces_ctx* c, const Layout& l, void* ws) {
    TaylorWs w;
    w.ta = at<void>(ws, l.v_TA);
    w.tb = at<void>(ws, l.v_TB);
    w.partials = at<double>(ws, l.v_partials);
    w.barrier = at<unsigned>(ws, l.v_bar);
    w.wait_ns = c->test_wait_ns ? c->test_wait_ns : kWaitLimitNs;
    w.skip_block = c->test_skip_block;
    w.diag = nullptr;
    return w;
}

// The post-adaptation diagnostics come out of the Taylor launch's first sweep when the step
// propagates by the Taylor series; otherwise (no propagation, Lanczos) from their own pass.
bool diag_in_taylor(const paces_step_params* prm) {
    return prm->diagnostics && prm->evolve && prm->lanczos_order == 0;
}

// Output rows the assembly can flag in the Taylor term buffer (one byte each).
int64_t self_flag_cap(const paces_ctx* c, const Layout& l) {
    return l.cap * int64_t(c->precision == PACES_C64 ? 8 : 16);
}

// The caller's Krylov workspace of the Lanczos step: order+1 vectors, two w buffers, the
// per-block partial sums and the barrier words.
struct KrylovLayout {
    size_t u, w0, w1, partials, barrier, total;
    int max_grid;
};

KrylovLayout krylov_layout(const paces_ctx* c, int64_t cap, int order) {
    KrylovLayout k;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) & ~size_t(255);
        return o;
    };
    const size_t cs = c->precision == PACES_C64 ? 8 : 16;
    k.max_grid = lanczos_max_grid(c->num_sms);
    k.u = take(size_t(order + 1) * size_t(cap) * cs);
    k.w0 = take(size_t(cap) * cs);
    k.w1 = take(size_t(cap) * cs);
    k.partials = take(size_t(2) * k.max_grid * 4 * 8);
    k.barrier = take(16);
    k.total = off;
    return k;
}

// Largest capacity whose Krylov layout fits `bytes` (0 when none does).
int64_t krylov_cap(const paces_ctx* c, size_t bytes, int order) {
    int64_t lo = 0, hi = int64_t(bytes / 8) + 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) / 2;
        if (krylov_layout(c, mid, order).total <= bytes) lo = mid; else hi = mid - 1;
    }
    return lo;
}

LanczosWs lanczos_ws(const paces_ctx* c, void* krylov, int64_t cap, int order) {
    const KrylovLayout k = krylov_layout(c, cap, order);
    LanczosWs w;
    w.u = at<void>(krylov, k.u);
    w.w0 = at<void>(krylov, k.w0);
    w.w1 = at<void>(krylov, k.w1);
    w.partials = at<double>(krylov, k.partials);
    w.barrier = at<unsigned>(krylov, k.barrier);
    w.cap = cap;
    w.max_grid = k.max_grid;
    w.skip_block = c->test_skip_block;
    w.wait_ns = c->test_wait_ns ? c->test_wait_ns : kWaitLimitNs;
    return w;
}

bool valid_basis(const paces_basis* b) { return b && b->keys && b->blk && b->cap >= 0; }

__global__ void record_init_kernel(paces_step_record* rec, int diagnostics) {
    if (threadIdx.x != 0) return;
    memset(rec, 0, sizeof(paces_step_record));
    rec->post_adapt_norm = -1.0;
    rec->post_adapt_energy_re = __longlong_as_double(0x7ff8000000000000ll);
    rec->post_adapt_energy_im = 0.0;
    (void)diagnostics;
}

// (n_select is written by the truncation: with several merge passes its buffer is reused)
__global__ void record_counts_kernel(paces_step_record* rec, const int* enl_blk, const int* new_blk, int L) {
    if (threadIdx.x != 0) return;
    rec->n_enlarged = enl_blk[L];
    rec->n_states = new_blk[L];
}

// Expansion (assemble = false) or assembly of X over every hopping channel of a lattice:
// merge_passes passes, pass 0 with the five standard runs, pass k >= 1 with the self run (the
// previous pass's output) and the images of X under channels 2k-1 and 2k.  Passes before the
// last write tmp[k & 1] (neither may alias X or fin's output); the last writes fin.  An
// assembly's pass k writes its maps to the k-th map array of the layout, its last pass the
// H rows of fin, and then the neighbour table (both parts) is filled from the maps.
int merge_all_channels(paces_ctx* c, bool assemble, const Layout& l, void* ws, const paces_basis& X,
                       const paces_basis* tmp, const MergeOut& fin, int* xnbr, int* ceiling, int* status,
                       cudaStream_t st) {
    const int P = merge_passes(c->m);
    int* pass_maps[4] = {at<int>(ws, l.maps), at<int>(ws, l.maps_e), nullptr, nullptr};
    if (P > 2) pass_maps[2] = at<int>(ws, l.maps_x);
    if (P > 3) pass_maps[3] = at<int>(ws, l.maps_x) + size_t(kRuns) * l.cap;
    const paces_basis* prev = nullptr;
    for (int k = 0; k < P; ++k) {
        const bool last = k == P - 1;
        MergeWs mws = merge_ws(c, l, ws);
        if (k > 0) merge_spec_hops(mws, c->m, 2 * k - 1, 2 * k < c->m.nhop ? 2 * k : -1);
        MergeOut mo{};
        if (last) {
            mo = fin;
        } else {
            mo.keys = tmp[k & 1].keys;
            mo.blk = tmp[k & 1].blk;
            mo.cap = tmp[k & 1].cap;
        }
        if (assemble) {
            mo.maps = pass_maps[k];
            mo.map_cap = l.cap;
        }
        const int rc = launch_merge(c->nw, assemble ? MERGE_ASSEMBLE : MERGE_EXPAND, assemble ? c->assemble_stride : c->merge_stride, c->m,
                                    k == 0 ? X.keys : prev->keys, k == 0 ? X.blk : prev->blk,
                                    k == 0 ? nullptr : X.keys, k == 0 ? nullptr : X.blk, mws, mo,
                                    k == 0 ? ceiling : nullptr, 0, status, c->num_sms, st);
        if (rc != PACES_OK) return rc;
        prev = last ? nullptr : &tmp[k & 1];
    }
    if (assemble && P > 1)
        return launch_nbr_fill_multi(c->m, X.blk, pass_maps, P, l.cap, fin.nbr, xnbr, fin.nbr_cap, c->num_sms, st);
    return PACES_OK;
}

// ---- the time step, in the pieces the single and the batched step share ---------------------
struct StepPlan {
    Layout l;
    const paces_basis* old_b;
    const void* old_psi;
    paces_basis* new_b;
    void* new_psi;
    paces_hmat* h;
    const paces_step_params* prm;
    paces_step_record* rec;
    void* ws;
    paces_basis A, B;   // truncated basis, enlargement ping-pong
    paces_basis* cur;   // the enlarged basis (A or B after enlarge_steps merges)
    const int* enl_blk; // block offsets of the enlarged basis (step_front)
    void* target;       // remapped amplitudes (the Taylor input when evolving)
};

int plan_step(paces_ctx* c, const paces_basis* old_b, const void* old_psi, paces_basis* new_b, void* new_psi,
              paces_hmat* h, const paces_step_params* prm, paces_step_record* rec, void* ws, size_t ws_bytes,
              StepPlan* p) {
    if (!c) return PACES_ERR_BADARG;
    if (!valid_basis(old_b) || !valid_basis(new_b) || !old_psi || !new_psi || !h || !h->nbr || !h->meta ||
        !prm || !rec || !ws)
        return fail(c, PACES_ERR_BADARG, "paces_step: null argument");
    if (prm->maxstates < 1 || prm->enlarge_steps < 0 || (prm->evolve && prm->m_star < 1))
        return fail(c, PACES_ERR_BADARG, "paces_step: bad parameters");
    if (prm->proposal && !prm->proposal_params)
        return fail(c, PACES_ERR_BADARG, "paces_step: proposal without MLP parameters");
    if (prm->lanczos_order < 0 || prm->lanczos_order > kMaxLanczosOrder)
        return fail(c, PACES_ERR_BADARG, "paces_step: lanczos_order %d outside 0..%d", int(prm->lanczos_order),
                    kMaxLanczosOrder);
    if (prm->evolve && prm->lanczos_order > 0) {
        if (!prm->krylov) return fail(c, PACES_ERR_BADARG, "paces_step: the Lanczos step needs a Krylov workspace");
        if (krylov_cap(c, prm->krylov_bytes, prm->lanczos_order) < new_b->cap)
            return fail(c, PACES_ERR_CAPACITY, "paces_step: the Krylov workspace holds fewer than %lld states",
                        (long long)new_b->cap);
    }
    if (c->m.nhop > 1) {
        if (!h->xnbr) return fail(c, PACES_ERR_BADARG, "paces_step: the lattice's H table needs xnbr");
        if (prm->proposal) return fail(c, PACES_ERR_BADARG, "paces_step: the learned proposal needs the chain model");
        if (prm->weighting && (!prm->old_h || !prm->old_h->xnbr))
            return fail(c, PACES_ERR_BADARG, "paces_step: the lattice's old H table needs xnbr");
    }
    if (prm->weighting) {
        if (prm->weighting != PACES_WEIGHT_COHERENCE && prm->weighting != PACES_WEIGHT_NORM)
            return fail(c, PACES_ERR_BADARG, "paces_step: unknown weighting %d", int(prm->weighting));
        if (!(prm->tau != 0.0 && std::isfinite(prm->tau)))
            return fail(c, PACES_ERR_BADARG, "paces_step: the look-ahead weighting needs a non-zero finite tau");
        if (!prm->old_h || !prm->old_h->nbr || !prm->old_h->meta || prm->old_h->cap < old_b->cap)
            return fail(c, PACES_ERR_BADARG, "paces_step: the look-ahead weighting needs the old basis' table");
        if (prm->proposal)
            return fail(c, PACES_ERR_BADARG, "paces_step: the look-ahead weighting and the proposal exclude each other");
    }
    p->l = fit_layout(c, ws_bytes);
    const Layout& l = p->l;
    if (old_b->cap > l.cap || new_b->cap > l.cap || h->cap > l.cap)
        return fail(c, PACES_ERR_CAPACITY, "workspace holds %lld states; bases hold %lld/%lld", (long long)l.cap,
                    (long long)old_b->cap, (long long)new_b->cap);
    p->old_b = old_b;
    p->old_psi = old_psi;
    p->new_b = new_b;
    p->new_psi = new_psi;
    p->h = h;
    p->prm = prm;
    p->rec = rec;
    p->ws = ws;
    p->A = paces_basis{at<uint64_t>(ws, l.keysA), at<int32_t>(ws, l.blkA), l.cap};
    p->B = paces_basis{at<uint64_t>(ws, l.keysB), at<int32_t>(ws, l.blkB), l.cap};
    p->cur = (prm->enlarge_steps & 1) ? &p->B : &p->A;
    p->target = prm->evolve ? at<void>(ws, l.v_V) : new_psi;
    return PACES_OK;
}

// Kernels one step enqueues (merge: 4 per pass, +1 for the neighbour table; truncation: see
// trunc_launches, +1 with look-ahead weights; remap 2; observables 2 or 3; Taylor 1;
// renormalisation 3; record 2).
unsigned long long step_launches(const paces_step_params& prm, bool c64, bool with_taylor, int passes) {
    const int wk = prm.weighting ? 2 : (c64 ? 1 : 0);
    return 2 + (prm.weighting ? 1 : 0) + trunc_launches(wk, prm.shuffle != 0) +
           (prm.proposal && prm.enlarge_steps > 0 ? 1 : 0) + 4ull * passes * (prm.enlarge_steps + 1) + 1 +
           2 + (prm.diagnostics ? 2 : 0) +
           (prm.evolve ? (with_taylor ? 1 : 0) + (prm.renormalize ? 3 : 0) : 0) + 3;
}

// Record, truncation, enlargement, new basis + H, remap, post-adaptation diagnostics.
int step_front(paces_ctx* c, StepPlan& p, cudaStream_t st, bool marks) {
    const bool c64 = c->precision == PACES_C64;
    const paces_step_params* prm = p.prm;
    paces_step_record* rec = p.rec;
    int* status = &rec->status;
    void* ws = p.ws;
    const Layout& l = p.l;
    auto mark = [&](int i) {
        if (marks && c->profiling) cudaEventRecord(c->ev[i], st);
    };
    record_init_kernel<<<1, 32, 0, st>>>(rec, prm->diagnostics);
    mark(0);
    // 1. truncation of the old state (ranked by the look-ahead weights, in the Taylor term
    //    buffer, which is free until the propagation)
    const double* weights = nullptr;
    if (prm->weighting) {
        double* w = at<double>(ws, l.v_TA);
        PACES_CHECK_LAUNCH(c, launch_lookahead(c64, with_h(c, prm->old_h), p.old_b->blk, prm->old_h->nbr, prm->old_h->meta, p.old_psi,
                                               prm->tau, prm->weighting, w, status, c->num_sms, st),
                           "step/weights");
        weights = w;
    }
    // without look-ahead weights the same buffer holds |psi| after the first radix round
    void* wscratch = weights ? nullptr : at<void>(ws, l.v_TA);
    PACES_CHECK_LAUNCH(c, launch_truncate(c->nw, c64, c->m, p.old_b->keys, p.old_b->blk, p.old_psi, weights, wscratch,
                                          prm->maxstates,
                                          prm->shuffle, prm->shuffle_seed, prm->step_index, trunc_ws(l, ws), p.A.keys,
                                          p.A.blk, p.A.cap, at<float>(ws, l.aw), &rec->n_tied, &rec->n_select, status, c->num_sms, st),
                       "step/truncate");
    // 1b. learned proposal: score the truncated basis' images
    const bool propose = prm->proposal && prm->enlarge_steps > 0;
    if (propose) {
        ProposalOut po{};
        po.keep = at<uint8_t>(ws, l.keep);
        po.keep_cap = l.cap;
        po.counts = &rec->n_candidates;
        PACES_CHECK_LAUNCH(c, launch_proposal_score(c->nw, c->m, p.A.keys, p.A.blk, at<float>(ws, l.aw),
                                                    at<float>(ws, l.aw) + l.cap, prm->proposal_params,
                                                    prm->proposal_threshold, po, status, c->num_sms, st),
                           "step/proposal");
    }
    mark(1);
    // 2. enlargement (enlarge_steps times; the first one filtered by the proposal).  Without
    //    the proposal the last enlargement B = P + images(P) is split: it also records where
    //    P's images landed and which states of B are new (N = B \ P), so the assembly merges
    //    B with the images of N only -- the images of P are in B already.
    const bool multi = c->m.nhop > 1;
    const bool split = prm->enlarge_steps > 0 && !propose && !multi;
    paces_basis* cur = &p.A;
    paces_basis* other = &p.B;
    paces_basis nbasis{at<uint64_t>(ws, l.keysN), at<int32_t>(ws, l.blkN), l.cap};
    if (multi) {
        // lattices: every expansion and the assembly in merge_passes passes, rotating three
        // buffers (the truncated basis starts in A)
        paces_basis bufs[3] = {p.A, p.B, nbasis};
        int ci = 0;
        const int P = merge_passes(c->m);
        for (int e = 0; e < prm->enlarge_steps; ++e) {
            const int o0 = (ci + 1) % 3, o1 = (ci + 2) % 3;
            const paces_basis tmp[2] = {bufs[o0], bufs[o1]};
            const int outi = ((P - 1) & 1) ? o1 : o0;
            MergeOut fin{};
            fin.keys = bufs[outi].keys;
            fin.blk = bufs[outi].blk;
            fin.cap = bufs[outi].cap;
            PACES_CHECK_LAUNCH(c, merge_all_channels(c, false, l, ws, bufs[ci], tmp, fin, nullptr, nullptr, status, st),
                               "step/expand");
            ci = outi;
        }
        mark(2);
        const paces_basis tmp[2] = {bufs[(ci + 1) % 3], bufs[(ci + 2) % 3]};
        MergeOut fin{};
        fin.keys = p.new_b->keys;
        fin.blk = p.new_b->blk;
        fin.cap = p.new_b->cap < p.h->cap ? p.new_b->cap : p.h->cap;
        fin.meta = p.h->meta;
        fin.nbr = p.h->nbr;
        fin.nbr_cap = p.h->cap;
        PACES_CHECK_LAUNCH(c, merge_all_channels(c, true, l, ws, bufs[ci], tmp, fin, p.h->xnbr, &rec->ceiling_hits,
                                                 status, st),
                           "step/assemble");
        p.enl_blk = bufs[ci].blk;
    }
    for (int e = 0; e < prm->enlarge_steps && !multi; ++e) {
        MergeWs mws = merge_ws(c, l, ws);
        if (propose && e == 0) {
            mws.keep = at<uint8_t>(ws, l.keep);
            mws.keep_cap = l.cap;
        }
        const bool last_split = split && e == prm->enlarge_steps - 1;
        MergeOut mo{};
        mo.keys = other->keys;
        mo.blk = other->blk;
        mo.cap = other->cap;
        if (last_split) {
            mo.maps = at<int>(ws, l.maps_e);
            mo.map_cap = l.cap;
            mo.new_keys = nbasis.keys;
            mo.new_blk = nbasis.blk;
            mo.new_to_out = at<int>(ws, l.n2b);
            mo.new_cap = nbasis.cap;
        }
        PACES_CHECK_LAUNCH(c, launch_merge(c->nw, last_split ? MERGE_EXPAND_SPLIT : MERGE_EXPAND, c->merge_stride, c->m,
                                           cur->keys, cur->blk, nullptr, nullptr, mws, mo,
                                           last_split ? &rec->ceiling_hits : nullptr, 0, status, c->num_sms, st),
                           "step/expand");
        paces_basis* t = cur;
        cur = other;
        other = t;
    }
    // 3. new basis + H
    if (!multi) {
        mark(2);
        p.enl_blk = cur->blk;
        MergeOut mo{};
        mo.keys = p.new_b->keys;
        mo.blk = p.new_b->blk;
        mo.cap = p.new_b->cap < p.h->cap ? p.new_b->cap : p.h->cap;
        mo.meta = p.h->meta;
        mo.nbr = p.h->nbr;
        mo.nbr_cap = p.h->cap;
        mo.maps = at<int>(ws, l.maps);
        mo.map_cap = l.cap;
        mo.self_rows_filled = split ? 1 : 0;  // nbr_fill_split writes the rows of the enlarged basis
        // which rows those are, for the neighbour fill (the Taylor term buffer is free until
        // the propagation; S bytes)
        mo.self_flag = at<uint8_t>(ws, l.v_TA);
        if (mo.cap > self_flag_cap(c, l)) mo.cap = self_flag_cap(c, l);
        PACES_CHECK_LAUNCH(c, launch_merge(c->nw, MERGE_ASSEMBLE, c->assemble_stride, c->m, cur->keys, cur->blk,
                                           split ? nbasis.keys : nullptr, split ? nbasis.blk : nullptr, merge_ws(c, l, ws),
                                           mo, &rec->ceiling_hits, split ? 1 : 0, status, c->num_sms, st),
                           "step/assemble");
        if (split)
            PACES_CHECK_LAUNCH(c, launch_nbr_fill_split(c->m, other->blk, nbasis.blk, at<int>(ws, l.maps_e),
                                                        at<int>(ws, l.maps), at<int>(ws, l.n2b), mo.self_flag, l.cap,
                                                        p.h->nbr, p.h->cap, c->num_sms, st),
                               "step/neighbours");
    }
    mark(3);
    // the new basis and its table are final: a caller may start copying them out
    if (prm->basis_ready) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cs) != cudaSuccess ||
            cudaEventRecordWithFlags(static_cast<cudaEvent_t>(prm->basis_ready), st,
                                     cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal
                                                                         : cudaEventRecordDefault) != cudaSuccess)
            return cuda_fail(c, "step/basis_ready");
    }
    // 4. amplitudes into the new basis
    PACES_CHECK_LAUNCH(c, launch_remap(c->nw, c64, c->m, p.old_b->keys, p.old_b->blk, p.old_psi, p.new_b->keys,
                                       p.new_b->blk, p.target, remap_ws(l, ws), status, c->num_sms, st),
                       "step/remap");
    mark(4);
    // 5. post-adaptation diagnostics (unless the Taylor launch folds them)
    if (prm->diagnostics && !diag_in_taylor(prm)) {
        ObsTarget t{&rec->post_adapt_norm, &rec->post_adapt_energy_re, &rec->post_adapt_energy_im, nullptr, nullptr};
        PACES_CHECK_LAUNCH(c, launch_observables(c->nw, c64, with_h(c, p.h), p.new_b->keys, p.new_b->blk, p.h->nbr,
                                                 p.h->cap, p.h->meta, p.target, PACES_OBS_NORM | PACES_OBS_ENERGY,
                                                 at<double>(ws, l.o_partials), t, c->num_sms, st),
                           "step/diagnostics");
    }
    mark(5);
    return PACES_OK;
}

// Renormalisation, observables of the new state, sizes into the record.
int step_back(paces_ctx* c, StepPlan& p, cudaStream_t st, bool marks) {
    const bool c64 = c->precision == PACES_C64;
    const paces_step_params* prm = p.prm;
    paces_step_record* rec = p.rec;
    double* opart = at<double>(p.ws, p.l.o_partials);
    auto mark = [&](int i) {
        if (marks && c->profiling) cudaEventRecord(c->ev[i], st);
    };
    if (diag_in_taylor(prm)) {
        ObsTarget t{&rec->post_adapt_norm, &rec->post_adapt_energy_re, &rec->post_adapt_energy_im, nullptr, nullptr};
        PACES_CHECK_LAUNCH(c, launch_diag_final(at<double>(p.ws, p.l.diag), p.new_b->blk, c->m.L, p.l.cap, t, st),
                           "step/diagnostics");
    }
    if (prm->evolve && prm->renormalize) {
        ObsTarget t{&rec->norm, nullptr, nullptr, nullptr, nullptr};
        PACES_CHECK_LAUNCH(c, launch_observables(c->nw, c64, with_h(c, p.h), p.new_b->keys, p.new_b->blk, p.h->nbr, p.h->cap,
                                                 p.h->meta, p.new_psi, PACES_OBS_NORM, opart, t, c->num_sms, st),
                           "step/norm");
        PACES_CHECK_LAUNCH(c, launch_scale(c64, c->m, p.new_b->blk, p.new_psi, &rec->norm, c->num_sms, st),
                           "step/renormalize");
    }
    mark(6);
    // 7. observables of the new state
    {
        ObsTarget t{&rec->norm, &rec->energy_re, &rec->energy_im, rec->n_exc, rec->n_pho};
        PACES_CHECK_LAUNCH(c, launch_observables(c->nw, c64, with_h(c, p.h), p.new_b->keys, p.new_b->blk, p.h->nbr, p.h->cap,
                                                 p.h->meta, p.new_psi,
                                                 PACES_OBS_NORM | PACES_OBS_ENERGY | PACES_OBS_SITES, opart, t,
                                                 c->num_sms, st),
                           "step/observables");
    }
    record_counts_kernel<<<1, 32, 0, st>>>(rec, p.enl_blk, p.new_b->blk, c->m.L);
    mark(7);
    if (cudaGetLastError() != cudaSuccess) return cuda_fail(c, "step/record");
    return PACES_OK;
}

}  // namespace

extern "C" {

int paces_version(void) { return 10300; }

int paces_hop_channels(const paces_ctx* c) { return c ? c->m.nhop : 0; }

int paces_create(const paces_model_desc* d, paces_ctx** out) {
    if (!out) return PACES_ERR_BADARG;
    *out = nullptr;
    if (!d || !d->max_ho_dims) return PACES_ERR_BADARG;
    const int L = d->nchain;
    if (L < 2 || L > kMaxSites) return PACES_ERR_BADARG;
    if (d->periodic && L < 3) return PACES_ERR_BADARG;
    if (d->precision != PACES_C128 && d->precision != PACES_C64) return PACES_ERR_BADARG;
    paces_ctx* c = new paces_ctx();
    std::memset(c, 0, sizeof(*c));
    ModelDev& m = c->m;
    m.L = L;
    m.periodic = d->periodic ? 1 : 0;
    m.eps_sys = d->eps_sys;
    m.hbar_omega = d->hbar_omega;
    m.delta_eps = d->delta_eps;
    m.J = d->J;
    m.g = d->g;
    m.has_site_eps = d->site_eps ? 1 : 0;
    // hopping channels (paces/models/holstein.py:150-240): per term (hopping, then hopping2),
    // one channel per lattice dimension d, moving the exciton by order * l^d
    {
        const int geo = d->geo_dim > 0 ? d->geo_dim : 1;
        const int l = int(std::lround(std::pow(double(L), 1.0 / geo)));  // lattice_l, holstein.py:49
        long long lp = 1;
        for (int k = 0; k < geo; ++k) lp *= l;
        if (geo > 3 || lp != L || (d->hopping2 && l - 1 < 2) || (d->periodic && (geo != 1 || d->hopping2))) {
            delete c;
            return PACES_ERR_BADARG;
        }
        m.J2 = d->hopping2 ? d->J2 : 0.0;
        m.nhop = 0;
        for (int t = 0; t < (d->hopping2 ? 2 : 1); ++t) {
            long long ld = 1;
            for (int k = 0; k < geo; ++k, ld *= l) {
                m.hop_dist[m.nhop] = int((t + 1) * ld);
                m.hop_mod[m.nhop] = int(ld * l);
                m.hop_term[m.nhop] = t;
                ++m.nhop;
            }
        }
        // per term: neighbours below p (largest distance first), then above (smallest first)
        for (int t = 0; t < 2; ++t) {
            int n = 0;
            for (int k = m.nhop - 1; k >= 0; --k)
                if (m.hop_term[k] == t) m.hop_ord[t][n++] = int8_t(k << 1);
            for (int k = 0; k < m.nhop; ++k)
                if (m.hop_term[k] == t) m.hop_ord[t][n++] = int8_t((k << 1) | 1);
            m.hop_n[t] = n;
        }
    }
    int word = 0, used = 0, total_bits = 0;
    for (int s = 0; s < L; ++s) {
        const int md = d->max_ho_dims[s];
        if (md < 2 || md > 256) {
            delete c;
            return PACES_ERR_BADARG;
        }
        int b = 0;
        while ((1 << b) < md) ++b;  // ceil(log2(max_dim)), paces/core/hamiltonian.py:155
        if (used + b > 64) {
            ++word;
            used = 0;
        }
        m.word[s] = uint8_t(word);
        m.shift[s] = uint8_t(64 - used - b);
        m.bits[s] = uint8_t(b);
        m.maxd[s] = uint16_t(md);
        m.site_eps[s] = d->site_eps ? d->site_eps[s] : 0.0;
        used += b;
        total_bits += b;
    }
    c->nw = word + 1;
    m.nw = c->nw;
    if (c->nw > kMaxKeyWords) {
        delete c;
        return PACES_ERR_BADARG;
    }
    m.max_bits = 0;
    for (int s = 0; s < L; ++s) {
        if (m.bits[s] > m.max_bits) m.max_bits = m.bits[s];
        for (int b = 0; b < m.bits[s]; ++b) m.plane[m.word[s]][b] |= uint64_t(1) << (m.shift[s] + b);
    }
    // reference row layout: position field first, then the sites (hamiltonian.py:140-160)
    int pb = 0;
    while ((1 << pb) < L) ++pb;
    c->rl.nfields = L + 1;
    c->rl.off[0] = 0;
    c->rl.bits[0] = pb;
    for (int s = 0; s < L; ++s) {
        c->rl.off[s + 1] = c->rl.off[s] + c->rl.bits[s];
        c->rl.bits[s + 1] = m.bits[s];
    }
    c->rl.words = (pb + total_bits + 31) / 32;
    if (c->rl.words > kMaxRefWords) {
        delete c;
        return PACES_ERR_BADARG;
    }
    c->precision = d->precision;
    if (cudaGetDevice(&c->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess) {
        delete c;
        return PACES_ERR_CUDA;
    }
    c->taylor_grid = taylor_max_grid(c->precision == PACES_C64, c->num_sms);
    c->merge_stride = merge_default_stride(c->nw);
    c->assemble_stride = merge_default_assemble_stride(c->nw);
    c->taylor_bps = 0;
    c->taylor_variant = 1;
    c->test_wait_ns = 0;
    c->test_skip_block = -1;
    // constants block: status words, per-site energies and the sqrt(k) * g tables
    {
        const size_t o_eps = 64, o_sq = o_eps + kMaxSites * 8, o_sqf = o_sq + kSqrtTable * 8;
        const size_t bytes = o_sqf + kSqrtTable * 4;
        alignas(8) unsigned char host[o_sqf + kSqrtTable * 4];
        std::memset(host, 0, sizeof(host));
        double* eps = reinterpret_cast<double*>(host + o_eps);
        double* sq = reinterpret_cast<double*>(host + o_sq);
        float* sqf = reinterpret_cast<float*>(host + o_sqf);
        for (int s = 0; s < L; ++s) eps[s] = m.site_eps[s];
        // IEEE sqrt and product, rounded to nearest: the values the kernels compute themselves
        for (int k = 0; k < kSqrtTable; ++k) {
            sq[k] = std::sqrt(double(k)) * m.g;
            sqf[k] = float(sq[k]);
        }
        void* d = nullptr;
        if (cudaMalloc(&d, bytes) != cudaSuccess || cudaMemcpy(d, host, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            if (d) cudaFree(d);
            delete c;
            return PACES_ERR_CUDA;
        }
        unsigned char* base = static_cast<unsigned char*>(d);
        c->d_status = reinterpret_cast<int*>(base);
        c->d_site_eps = reinterpret_cast<double*>(base + o_eps);
        c->d_sq = reinterpret_cast<double*>(base + o_sq);
        c->d_sqf = reinterpret_cast<float*>(base + o_sqf);
    }
    *out = c;
    return PACES_OK;
}

int paces_set_test_hooks(paces_ctx* c, uint64_t wait_limit_ns, int32_t skip_barrier_block) {
    if (!c || skip_barrier_block < -1) return PACES_ERR_BADARG;
    if (wait_limit_ns > kWaitLimitNs) return fail(c, PACES_ERR_BADARG, "wait limit above %llu ns", (unsigned long long)kWaitLimitNs);
    c->test_wait_ns = wait_limit_ns;
    c->test_skip_block = skip_barrier_block;
    return PACES_OK;
}

int paces_set_profiling(paces_ctx* c, int32_t on) {
    if (!c) return PACES_ERR_BADARG;
    if (on && !c->profiling) {
        for (int i = 0; i < 8; ++i)
            if (cudaEventCreate(&c->ev[i]) != cudaSuccess) return cuda_fail(c, "paces_set_profiling");
    }
    if (!on && c->profiling) {
        for (int i = 0; i < 8; ++i) cudaEventDestroy(c->ev[i]);
    }
    c->profiling = on ? 1 : 0;
    return PACES_OK;
}

int paces_stage_times(paces_ctx* c, float* ms) {
    if (!c || !ms || !c->profiling) return PACES_ERR_BADARG;
    if (cudaEventSynchronize(c->ev[7]) != cudaSuccess) return cuda_fail(c, "paces_stage_times");
    for (int i = 0; i < 7; ++i)
        if (cudaEventElapsedTime(&ms[i], c->ev[i], c->ev[i + 1]) != cudaSuccess)
            return cuda_fail(c, "paces_stage_times");
    return PACES_OK;
}

unsigned long long paces_kernel_launches(const paces_ctx* c) { return c ? c->launches : 0ull; }

int paces_destroy(paces_ctx* c) {
    if (!c) return PACES_OK;
    if (c->profiling) paces_set_profiling(c, 0);
    if (c->d_status) cudaFree(c->d_status);
    delete c;
    return PACES_OK;
}

const char* paces_last_error(const paces_ctx* c) { return c ? c->err : "no context"; }

int paces_key_words(const paces_ctx* c) { return c ? c->nw : 0; }

int paces_ref_words(const paces_ctx* c) { return c ? c->rl.words : 0; }

int paces_key_layout(const paces_ctx* c, int32_t* word, int32_t* shift, int32_t* bits) {
    if (!c) return PACES_ERR_BADARG;
    for (int s = 0; s < c->m.L; ++s) {
        if (word) word[s] = c->m.word[s];
        if (shift) shift[s] = c->m.shift[s];
        if (bits) bits[s] = c->m.bits[s];
    }
    return PACES_OK;
}

int paces_get_tuning(const paces_ctx* c, paces_tuning* t) {
    if (!c || !t) return PACES_ERR_BADARG;
    std::memset(t, 0, sizeof(*t));
    t->merge_stride = c->merge_stride;
    t->assemble_stride = c->assemble_stride;
    t->merge_stride_max = merge_stride(c->nw);
    t->merge_stride_min = kMinMergeStride;
    t->taylor_blocks_per_sm = c->taylor_bps;
    t->taylor_blocks_per_sm_max = c->taylor_grid / c->num_sms;
    t->taylor_variant = c->taylor_variant;
    return PACES_OK;
}

int paces_set_tuning(paces_ctx* c, const paces_tuning* t) {
    if (!c || !t) return PACES_ERR_BADARG;
    if (t->merge_stride < kMinMergeStride || t->merge_stride > merge_stride(c->nw) || t->merge_stride % 16)
        return fail(c, PACES_ERR_BADARG, "merge_stride %d: a multiple of 16 in [%d, %d]", t->merge_stride,
                    kMinMergeStride, merge_stride(c->nw));
    const int as = t->assemble_stride ? t->assemble_stride : t->merge_stride;
    if (as < kMinMergeStride || as > merge_stride(c->nw) || as % 16)
        return fail(c, PACES_ERR_BADARG, "assemble_stride %d: 0 or a multiple of 16 in [%d, %d]", t->assemble_stride,
                    kMinMergeStride, merge_stride(c->nw));
    if (t->taylor_blocks_per_sm < 0 || t->taylor_blocks_per_sm > c->taylor_grid / c->num_sms)
        return fail(c, PACES_ERR_BADARG, "taylor_blocks_per_sm %d: 0..%d", t->taylor_blocks_per_sm,
                    c->taylor_grid / c->num_sms);
    if (t->taylor_variant < 0 || t->taylor_variant > 1)
        return fail(c, PACES_ERR_BADARG, "taylor_variant %d: 0 or 1", t->taylor_variant);
    c->merge_stride = t->merge_stride;
    c->assemble_stride = as;
    c->taylor_bps = t->taylor_blocks_per_sm;
    c->taylor_variant = t->taylor_variant;
    return PACES_OK;
}

int paces_workspace_bytes(const paces_ctx* c, int64_t cap, size_t* bytes) {
    if (!c || !bytes || cap < 0) return PACES_ERR_BADARG;
    *bytes = make_layout(c, cap).total;
    return PACES_OK;
}

int paces_read_status(paces_ctx* c, paces_stream_t stream, int32_t* host_status) {
    if (!c || !host_status) return PACES_ERR_BADARG;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(host_status, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess || cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), st) != cudaSuccess)
        return cuda_fail(c, "paces_read_status");
    return PACES_OK;
}

int paces_keys_from_ref(paces_ctx* c, const uint32_t* ref, int64_t n, int32_t ref_words,
                        uint64_t* keys_out, int32_t* pos_out, paces_stream_t stream) {
    if (!c) return PACES_ERR_BADARG;
    if (ref_words != c->rl.words) return fail(c, PACES_ERR_BADARG, "reference rows have %d words, model needs %d", ref_words, c->rl.words);
    PACES_CHECK_LAUNCH(c, launch_keys_from_ref(c->nw, c->m, c->rl, ref, n, keys_out, pos_out, c->d_status,
                                               c->num_sms, reinterpret_cast<cudaStream_t>(stream)),
                       "keys_from_ref");
    return PACES_OK;
}

int paces_keys_to_ref(paces_ctx* c, const paces_basis* b, int32_t ref_words, uint32_t* ref_out,
                      paces_stream_t stream) {
    if (!c || !valid_basis(b) || !ref_out) return PACES_ERR_BADARG;
    if (ref_words != c->rl.words) return fail(c, PACES_ERR_BADARG, "reference rows have %d words, model needs %d", ref_words, c->rl.words);
    PACES_CHECK_LAUNCH(c, launch_keys_to_ref(c->nw, c->m, c->rl, b->keys, b->blk, ref_out, c->num_sms,
                                             reinterpret_cast<cudaStream_t>(stream)),
                       "keys_to_ref");
    return PACES_OK;
}

int paces_expand(paces_ctx* c, const paces_basis* in, paces_basis* out, void* ws, size_t ws_bytes,
                 paces_stream_t stream) {
    if (!c || !valid_basis(in) || !valid_basis(out) || !ws) return PACES_ERR_BADARG;
    const Layout l = fit_layout(c, ws_bytes);
    if (in->cap > l.cap) return fail(c, PACES_ERR_CAPACITY, "workspace holds %lld states, input basis %lld", (long long)l.cap, (long long)in->cap);
    MergeOut mo{};
    mo.keys = out->keys;
    mo.blk = out->blk;
    mo.cap = out->cap;
    if (c->m.nhop > 1) {
        const paces_basis tmp[2] = {{at<uint64_t>(ws, l.keysA), at<int32_t>(ws, l.blkA), l.cap},
                                    {at<uint64_t>(ws, l.keysB), at<int32_t>(ws, l.blkB), l.cap}};
        PACES_CHECK_LAUNCH(c, merge_all_channels(c, false, l, ws, *in, tmp, mo, nullptr, nullptr, c->d_status,
                                                 reinterpret_cast<cudaStream_t>(stream)),
                           "expand");
        return PACES_OK;
    }
    PACES_CHECK_LAUNCH(c, launch_merge(c->nw, MERGE_EXPAND, c->merge_stride, c->m, in->keys, in->blk, nullptr, nullptr,
                                       merge_ws(c, l, ws), mo, nullptr, 0,
                                       c->d_status, c->num_sms, reinterpret_cast<cudaStream_t>(stream)),
                       "expand");
    return PACES_OK;
}

int paces_assemble(paces_ctx* c, const paces_basis* in, paces_basis* out, paces_hmat* h,
                   int32_t* dev_ceiling_hits, void* ws, size_t ws_bytes, paces_stream_t stream) {
    if (!c || !valid_basis(in) || !valid_basis(out) || !h || !h->nbr || !h->meta || !ws) return PACES_ERR_BADARG;
    const Layout l = fit_layout(c, ws_bytes);
    if (in->cap > l.cap) return fail(c, PACES_ERR_CAPACITY, "workspace holds %lld states, input basis %lld", (long long)l.cap, (long long)in->cap);
    MergeOut mo{};
    mo.keys = out->keys;
    mo.blk = out->blk;
    mo.cap = out->cap;
    mo.meta = h->meta;
    mo.nbr = h->nbr;
    mo.nbr_cap = h->cap;
    mo.maps = at<int>(ws, l.maps);
    mo.map_cap = l.cap;
    mo.self_flag = at<uint8_t>(ws, l.v_TA);  // S bytes of the workspace's Taylor term buffer
    if (h->cap < out->cap) mo.cap = h->cap;
    // the tile kernel flags every output row in that buffer: an output larger than it raises
    // PACES_ERR_CAPACITY instead of writing past it
    if (mo.cap > self_flag_cap(c, l)) mo.cap = self_flag_cap(c, l);
    if (c->m.nhop > 1) {
        if (!h->xnbr) return fail(c, PACES_ERR_BADARG, "paces_assemble: the model's H needs xnbr");
        const paces_basis tmp[2] = {{at<uint64_t>(ws, l.keysA), at<int32_t>(ws, l.blkA), l.cap},
                                    {at<uint64_t>(ws, l.keysB), at<int32_t>(ws, l.blkB), l.cap}};
        PACES_CHECK_LAUNCH(c, merge_all_channels(c, true, l, ws, *in, tmp, mo, h->xnbr, dev_ceiling_hits, c->d_status,
                                                 reinterpret_cast<cudaStream_t>(stream)),
                           "assemble");
        return PACES_OK;
    }
    PACES_CHECK_LAUNCH(c, launch_merge(c->nw, MERGE_ASSEMBLE, c->assemble_stride, c->m, in->keys, in->blk, nullptr, nullptr,
                                       merge_ws(c, l, ws), mo, dev_ceiling_hits, 0,
                                       c->d_status, c->num_sms, reinterpret_cast<cudaStream_t>(stream)),
                       "assemble");
    return PACES_OK;
}

int paces_truncate(paces_ctx* c, const paces_basis* in, const void* psi, int64_t maxstates, int32_t shuffle,
                   uint64_t shuffle_seed, uint64_t step_index, paces_basis* out, void* ws, size_t ws_bytes,
                   paces_stream_t stream) {
    if (!c || !valid_basis(in) || !valid_basis(out) || !psi || !ws || maxstates < 1) return PACES_ERR_BADARG;
    const Layout l = fit_layout(c, ws_bytes);
    if (in->cap > l.cap) return fail(c, PACES_ERR_CAPACITY, "workspace holds %lld states, input basis %lld", (long long)l.cap, (long long)in->cap);
    PACES_CHECK_LAUNCH(c, launch_truncate(c->nw, c->precision == PACES_C64, c->m, in->keys, in->blk, psi, nullptr,
                                          at<void>(ws, l.v_TA), maxstates, shuffle, shuffle_seed, step_index, trunc_ws(l, ws), out->keys,
                                          out->blk, out->cap, nullptr, nullptr, nullptr, c->d_status, c->num_sms,
                                          reinterpret_cast<cudaStream_t>(stream)),
                       "truncate");
    return PACES_OK;
}

int paces_truncate_weighted(paces_ctx* c, const paces_basis* in, const double* weights, int64_t maxstates,
                            int32_t shuffle, uint64_t shuffle_seed, uint64_t step_index, paces_basis* out, void* ws,
                            size_t ws_bytes, paces_stream_t stream) {
    if (!c || !valid_basis(in) || !valid_basis(out) || !weights || !ws || maxstates < 1) return PACES_ERR_BADARG;
    const Layout l = fit_layout(c, ws_bytes);
    if (in->cap > l.cap) return fail(c, PACES_ERR_CAPACITY, "workspace holds %lld states, input basis %lld", (long long)l.cap, (long long)in->cap);
    PACES_CHECK_LAUNCH(c, launch_truncate(c->nw, c->precision == PACES_C64, c->m, in->keys, in->blk, nullptr, weights,
                                          nullptr, maxstates, shuffle, shuffle_seed, step_index, trunc_ws(l, ws), out->keys,
                                          out->blk, out->cap, nullptr, nullptr, nullptr, c->d_status, c->num_sms,
                                          reinterpret_cast<cudaStream_t>(stream)),
                       "truncate_weighted");
    return PACES_OK;
}

int paces_lookahead_weights(paces_ctx* c, const paces_basis* b, const paces_hmat* h, const void* psi, double tau,
                            int32_t weighting, double* w, paces_stream_t stream) {
    if (!c || !valid_basis(b) || !h || !h->nbr || !h->meta || !psi || !w || h->cap < b->cap) return PACES_ERR_BADARG;
    if (weighting != PACES_WEIGHT_COHERENCE && weighting != PACES_WEIGHT_NORM && weighting != PACES_WEIGHT_HAM_ONES)
        return fail(c, PACES_ERR_BADARG, "paces_lookahead_weights: unknown weighting %d", int(weighting));
    if (!std::isfinite(tau)) return fail(c, PACES_ERR_BADARG, "paces_lookahead_weights: tau is not finite");
    PACES_CHECK_LAUNCH(c, launch_lookahead(c->precision == PACES_C64, with_h(c, h), b->blk, h->nbr, h->meta, psi, tau, weighting,
                                           w, c->d_status, c->num_sms, reinterpret_cast<cudaStream_t>(stream)),
                       "lookahead_weights");
    return PACES_OK;
}

int paces_remap(paces_ctx* c, const paces_basis* old_b, const void* old_psi, const paces_basis* new_b,
                void* new_psi, void* ws, size_t ws_bytes, paces_stream_t stream) {
    if (!c || !valid_basis(old_b) || !valid_basis(new_b) || !old_psi || !new_psi || !ws) return PACES_ERR_BADARG;
    const Layout l = fit_layout(c, ws_bytes);
    if (old_b->cap > l.cap || new_b->cap > l.cap)
        return fail(c, PACES_ERR_CAPACITY, "workspace holds %lld states", (long long)l.cap);
    PACES_CHECK_LAUNCH(c, launch_remap(c->nw, c->precision == PACES_C64, c->m, old_b->keys, old_b->blk, old_psi,
                                       new_b->keys, new_b->blk, new_psi, remap_ws(l, ws), c->d_status, c->num_sms,
                                       reinterpret_cast<cudaStream_t>(stream)),
                       "remap");
    return PACES_OK;
}

int paces_remap_noalloc(paces_ctx* c, const paces_basis* old_b, const void* old_psi, const paces_basis* new_b,
                        void* new_psi, paces_stream_t stream) {
    if (!c || !valid_basis(old_b) || !valid_basis(new_b) || !old_psi || !new_psi) return PACES_ERR_BADARG;
    // the tile table must fit the static scratch for any contents of the two bases
    const int64_t tiles = (old_b->cap + new_b->cap) / remap_tile(c->nw) + c->m.L + 8;
    if (tiles > remap_static_tile_cap())
        return fail(c, PACES_ERR_CAPACITY,
                    "paces_remap_noalloc: bases of %lld + %lld states need %lld remap tiles; the static "
                    "scratch holds %d (at most %lld states in total with %d key words)",
                    (long long)old_b->cap, (long long)new_b->cap, (long long)tiles, remap_static_tile_cap(),
                    (long long)(remap_static_tile_cap() - c->m.L - 8) * remap_tile(c->nw), c->nw);
    RemapWs ws{};
    const char* err = nullptr;
    const int rc = remap_static_ws(&ws, &err);
    if (rc != PACES_OK) return fail(c, rc, "paces_remap_noalloc: %s", err ? err : "set-up failed");
    PACES_CHECK_LAUNCH(c, launch_remap(c->nw, c->precision == PACES_C64, c->m, old_b->keys, old_b->blk, old_psi,
                                       new_b->keys, new_b->blk, new_psi, ws, c->d_status, c->num_sms,
                                       reinterpret_cast<cudaStream_t>(stream)),
                       "remap_noalloc");
    return PACES_OK;
}

int paces_taylor(paces_ctx* c, const paces_basis* b, const paces_hmat* h, const void* psi_in, void* psi_out,
                 double dt, int32_t m_star, double tol, paces_expm_info* dev_info, void* ws, size_t ws_bytes,
                 paces_stream_t stream) {
    if (!c || !valid_basis(b) || !h || !psi_in || !psi_out || psi_in == psi_out || !ws || m_star < 1)
        return PACES_ERR_BADARG;
    const Layout l = fit_layout(c, ws_bytes);
    if (h->cap > l.cap) return fail(c, PACES_ERR_CAPACITY, "workspace holds %lld states", (long long)l.cap);
    TaylorOut o{};
    if (dev_info) {
        o.converged = &dev_info->converged;
        o.final_m = &dev_info->final_m;
        o.c1_plus_c2 = &dev_info->c1_plus_c2;
        o.term_ratio = &dev_info->term_ratio;
    }
    PACES_CHECK_LAUNCH(c, launch_taylor(c->precision == PACES_C64, with_h(c, h), b->blk, h->nbr, h->cap, h->meta, psi_in,
                                        psi_out, dt, m_star, tol, taylor_ws(c, l, ws), o, c->d_status, c->num_sms,
                                        c->taylor_bps, c->taylor_variant, reinterpret_cast<cudaStream_t>(stream)),
                       "taylor");
    return PACES_OK;
}

namespace {
int current_sms() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
        return 0;
    return sms;
}
}  // namespace

int paces_rows_lower_bound(const uint32_t* pb, int64_t n, const uint32_t* q, int64_t nq, int32_t words,
                           int32_t allow_escapes, int64_t* out, int32_t* dev_missing, paces_stream_t stream) {
    if (n < 0 || nq < 0 || (nq > 0 && (!q || !out)) || (n > 0 && !pb) || (!allow_escapes && !dev_missing))
        return PACES_ERR_BADARG;
    const int sms = current_sms();
    if (!sms) return PACES_ERR_CUDA;
    return launch_rows_lower_bound(pb, n, q, nq, words, allow_escapes ? 0 : 1, out, dev_missing, sms,
                                   reinterpret_cast<cudaStream_t>(stream));
}

size_t paces_rows_sort_bytes(int64_t n) { return n < 0 ? 0 : rows_sort_ws_bytes(n); }

int paces_rows_sort_unique(const uint32_t* rows, int64_t n, int32_t words, uint32_t* out, int64_t* dev_count,
                           void* ws, size_t ws_bytes, paces_stream_t stream) {
    if (n < 0 || !dev_count || (n > 0 && (!rows || !out || !ws))) return PACES_ERR_BADARG;
    if (n > 0 && ws_bytes < rows_sort_ws_bytes(n)) return PACES_ERR_CAPACITY;
    const int sms = current_sms();
    if (!sms) return PACES_ERR_CUDA;
    return launch_rows_sort_unique(rows, n, words, out, dev_count, ws, sms, reinterpret_cast<cudaStream_t>(stream));
}

int paces_lanczos_bytes(const paces_ctx* c, int64_t cap, int32_t order, size_t* bytes) {
    if (!c || !bytes || cap < 0 || order < 1 || order > kMaxLanczosOrder) return PACES_ERR_BADARG;
    *bytes = krylov_layout(c, cap, order).total;
    return PACES_OK;
}

int paces_lanczos(paces_ctx* c, const paces_basis* b, const paces_hmat* h, const void* psi_in, void* psi_out,
                  double dt, int32_t order, paces_expm_info* dev_info, void* krylov, size_t krylov_bytes,
                  paces_stream_t stream) {
    if (!c || !valid_basis(b) || !h || !h->nbr || !h->meta || !psi_in || !psi_out || psi_in == psi_out || !krylov)
        return PACES_ERR_BADARG;
    if (order < 1 || order > kMaxLanczosOrder)
        return fail(c, PACES_ERR_BADARG, "paces_lanczos: order %d outside 1..%d", int(order), kMaxLanczosOrder);
    if (c->m.nhop > 1 && !h->xnbr) return fail(c, PACES_ERR_BADARG, "paces_lanczos: the lattice's H needs xnbr");
    const int64_t kcap = krylov_cap(c, krylov_bytes, order);
    if (kcap < b->cap) return fail(c, PACES_ERR_CAPACITY, "Krylov workspace holds %lld states, basis %lld", (long long)kcap, (long long)b->cap);
    TaylorOut o{};
    if (dev_info) {
        o.converged = &dev_info->converged;
        o.final_m = &dev_info->final_m;
        o.c1_plus_c2 = &dev_info->c1_plus_c2;
        o.term_ratio = &dev_info->term_ratio;
    }
    PACES_CHECK_LAUNCH(c, launch_lanczos(c->precision == PACES_C64, with_h(c, h), b->blk, h->nbr, h->meta, psi_in, psi_out,
                                         dt, order, lanczos_ws(c, krylov, kcap, order), o, c->d_status, c->num_sms,
                                         reinterpret_cast<cudaStream_t>(stream)),
                       "lanczos");
    return PACES_OK;
}

int paces_hnorms(paces_ctx* c, const paces_basis* b, const paces_hmat* h, const double* dev_shift, double* dev_out,
                 void* ws, size_t ws_bytes, paces_stream_t stream) {
    if (!c || !valid_basis(b) || !h || !h->nbr || !h->meta || !dev_out || !ws) return PACES_ERR_BADARG;
    const Layout l = fit_layout(c, ws_bytes);
    const int nparts = c->num_sms * 2;  // the observables' partials hold far more than 2 * nparts doubles
    PACES_CHECK_LAUNCH(c, launch_hnorms(with_h(c, h), b->blk, h->nbr, h->meta, dev_shift, at<double>(ws, l.o_partials), nparts,
                                        dev_out, reinterpret_cast<cudaStream_t>(stream)),
                       "hnorms");
    return PACES_OK;
}

int paces_expm_scaled(paces_ctx* c, const paces_basis* b, const paces_hmat* h, const void* psi_in, void* psi_out,
                      double t, double shift, int32_t m_star, int32_t stages, double tol, double eta_re, double eta_im,
                      paces_expm_info* dev_info, void* ws, size_t ws_bytes, paces_stream_t stream) {
    if (!c || !valid_basis(b) || !h || !h->nbr || !h->meta || !psi_in || !psi_out || psi_in == psi_out || !ws ||
        m_star < 0 || stages < 1)
        return PACES_ERR_BADARG;
    const Layout l = fit_layout(c, ws_bytes);
    if (h->cap > l.cap) return fail(c, PACES_ERR_CAPACITY, "workspace holds %lld states", (long long)l.cap);
    TaylorOut o{};
    if (dev_info) {
        o.converged = &dev_info->converged;
        o.final_m = &dev_info->final_m;
        o.c1_plus_c2 = &dev_info->c1_plus_c2;
        o.term_ratio = &dev_info->term_ratio;
    }
    PACES_CHECK_LAUNCH(c, launch_expm_scaled(c->precision == PACES_C64, with_h(c, h), b->blk, h->nbr, h->meta, psi_in, psi_out,
                                             t, shift, m_star, stages, tol, eta_re, eta_im, taylor_ws(c, l, ws), o,
                                             c->d_status, c->num_sms, c->taylor_grid,
                                             reinterpret_cast<cudaStream_t>(stream)),
                       "expm_scaled");
    return PACES_OK;
}

int paces_observables(paces_ctx* c, const paces_basis* b, const paces_hmat* h, const void* psi, int32_t what,
                      double* dev_out, void* ws, size_t ws_bytes, paces_stream_t stream) {
    if (!c || !valid_basis(b) || !h || !psi || !dev_out || !ws) return PACES_ERR_BADARG;
    const Layout l = fit_layout(c, ws_bytes);
    const int L = c->m.L;
    ObsTarget t{dev_out, dev_out + 1, dev_out + 2, dev_out + 3, dev_out + 3 + L};
    PACES_CHECK_LAUNCH(c, launch_observables(c->nw, c->precision == PACES_C64, with_h(c, h), b->keys, b->blk, h->nbr, h->cap,
                                             h->meta, psi, what, at<double>(ws, l.o_partials), t, c->num_sms,
                                             reinterpret_cast<cudaStream_t>(stream)),
                       "observables");
    return PACES_OK;
}

int paces_term_energies(paces_ctx* c, const paces_basis* b, const paces_hmat* h, const void* psi, double* dev_out,
                        void* ws, size_t ws_bytes, paces_stream_t stream) {
    if (!c || !valid_basis(b) || !h || !h->nbr || !h->meta || !psi || !dev_out || !ws) return PACES_ERR_BADARG;
    if (c->m.nhop > 1 && !h->xnbr) return fail(c, PACES_ERR_BADARG, "paces_term_energies: the lattice's H needs xnbr");
    const Layout l = fit_layout(c, ws_bytes);
    PACES_CHECK_LAUNCH(c, launch_term_energies(c->precision == PACES_C64, with_h(c, h), b->blk, h->nbr, h->meta, psi,
                                               at<double>(ws, l.o_partials), dev_out, c->num_sms,
                                               reinterpret_cast<cudaStream_t>(stream)),
                       "term_energies");
    return PACES_OK;
}

int paces_apply_h(paces_ctx* c, const paces_basis* b, const paces_hmat* h, const void* x, void* y,
                  paces_stream_t stream) {
    if (!c || !valid_basis(b) || !h || !h->nbr || !h->meta || !x || !y || x == y) return PACES_ERR_BADARG;
    PACES_CHECK_LAUNCH(c, launch_apply_h(c->precision == PACES_C64, with_h(c, h), b->blk, h->nbr, h->meta, x, y, c->num_sms,
                                         reinterpret_cast<cudaStream_t>(stream)),
                       "apply_h");
    return PACES_OK;
}

int paces_lookup(paces_ctx* c, const paces_basis* pb, const uint64_t* q_keys, const int32_t* q_pos, int64_t nq,
                 int32_t must_exist, int64_t* out, void* ws, size_t ws_bytes, paces_stream_t stream) {
    (void)ws;
    (void)ws_bytes;
    if (!c || !valid_basis(pb) || (nq > 0 && (!q_keys || !q_pos || !out))) return PACES_ERR_BADARG;
    PACES_CHECK_LAUNCH(c, launch_lookup(c->nw, c->m, pb->keys, pb->blk, q_keys, q_pos, nq, must_exist, out,
                                        c->d_status, c->num_sms, reinterpret_cast<cudaStream_t>(stream)),
                       "lookup");
    return PACES_OK;
}

int paces_step(paces_ctx* c, const paces_basis* old_b, const void* old_psi, paces_basis* new_b, void* new_psi,
               paces_hmat* h, const paces_step_params* prm, paces_step_record* rec, void* ws, size_t ws_bytes,
               paces_stream_t stream) {
    StepPlan p;
    const int rc = plan_step(c, old_b, old_psi, new_b, new_psi, h, prm, rec, ws, ws_bytes, &p);
    if (rc != PACES_OK) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    c->launches += step_launches(*prm, c->precision == PACES_C64, true, merge_passes(c->m));
    int r = step_front(c, p, st, true);
    if (r != PACES_OK) return r;
    if (prm->evolve) {
        TaylorOut o{&rec->converged, &rec->final_m, &rec->c1_plus_c2, &rec->term_ratio};
        if (prm->lanczos_order > 0) {
            const int64_t kcap = krylov_cap(c, prm->krylov_bytes, prm->lanczos_order);
            PACES_CHECK_LAUNCH(c, launch_lanczos(c->precision == PACES_C64, with_h(c, h), new_b->blk, h->nbr, h->meta,
                                                 p.target, new_psi, prm->dt, prm->lanczos_order,
                                                 lanczos_ws(c, prm->krylov, kcap, prm->lanczos_order), o, &rec->status,
                                                 c->num_sms, st),
                               "step/lanczos");
        } else {
            TaylorWs tw = taylor_ws(c, p.l, ws);
            if (diag_in_taylor(prm)) tw.diag = at<double>(ws, p.l.diag);
            PACES_CHECK_LAUNCH(c, launch_taylor(c->precision == PACES_C64, with_h(c, h), new_b->blk, h->nbr, h->cap,
                                                h->meta, p.target, new_psi, prm->dt, prm->m_star, prm->tol, tw, o,
                                                &rec->status, c->num_sms, c->taylor_bps, c->taylor_variant, st),
                               "step/taylor");
        }
    }
    return step_back(c, p, st, true);
}


// ---- learned proposal ----------------------------------------------------------------------
size_t paces_mlp_param_bytes(void) { return kMlpParamBytes; }

int32_t paces_mlp_master_floats(void) { return kMlpMasterFloats; }

int paces_selected_view(const paces_ctx* c, void* ws, size_t ws_bytes, paces_basis* sel, float** weights,
                        float** cut) {
    if (!c || !ws || !sel) return PACES_ERR_BADARG;
    const Layout l = fit_layout(c, ws_bytes);
    *sel = paces_basis{at<uint64_t>(ws, l.keysA), at<int32_t>(ws, l.blkA), l.cap};
    if (weights) *weights = at<float>(ws, l.aw);
    if (cut) *cut = at<float>(ws, l.aw) + l.cap;
    return PACES_OK;
}

int paces_proposal_score(paces_ctx* c, const paces_basis* x, const float* weights, const float* cut, const void* params,
                         float threshold, uint8_t* keep, int64_t keep_cap, float* logits, int32_t* counts,
                         paces_stream_t stream) {
    if (!c || !valid_basis(x) || !weights || !params || (keep && keep_cap < x->cap)) return PACES_ERR_BADARG;
    ProposalOut po{keep, keep_cap, logits, counts};
    PACES_CHECK_LAUNCH(c, launch_proposal_score(c->nw, c->m, x->keys, x->blk, weights, cut, params, threshold, po,
                                                c->d_status, c->num_sms, reinterpret_cast<cudaStream_t>(stream)),
                       "proposal_score");
    return PACES_OK;
}

int paces_proposal_features(paces_ctx* c, const paces_basis* x, const float* weights, const float* cut,
                            uint16_t* feats, uint8_t* valid, paces_stream_t stream) {
    if (!c || !valid_basis(x) || !weights || !feats || !valid) return PACES_ERR_BADARG;
    PACES_CHECK_LAUNCH(c, launch_proposal_features(c->nw, c->m, x->keys, x->blk, weights, cut, feats, valid, c->num_sms,
                                                   reinterpret_cast<cudaStream_t>(stream)),
                       "proposal_features");
    return PACES_OK;
}

int paces_proposal_labels(paces_ctx* c, const paces_basis* x, const paces_basis* y, uint8_t* labels,
                          paces_stream_t stream) {
    if (!c || !valid_basis(x) || !valid_basis(y) || !labels) return PACES_ERR_BADARG;
    PACES_CHECK_LAUNCH(c, launch_proposal_labels(c->nw, c->m, x->keys, x->blk, y->keys, y->blk, labels, c->num_sms,
                                                 reinterpret_cast<cudaStream_t>(stream)),
                       "proposal_labels");
    return PACES_OK;
}

namespace {
int device_sms() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    return sms;
}
}  // namespace

int paces_mlp_pack(const float* master, void* params, paces_stream_t stream) {
    if (!master || !params) return PACES_ERR_BADARG;
    return launch_mlp_pack(master, params, reinterpret_cast<cudaStream_t>(stream));
}

int paces_mlp_forward(const void* params, const uint16_t* x, int64_t n, float* logits, paces_stream_t stream) {
    if (!params || n < 0 || (n > 0 && (!x || !logits))) return PACES_ERR_BADARG;
    const int sms = device_sms();
    if (sms < 1) return PACES_ERR_CUDA;
    return launch_mlp_forward(params, x, n, logits, sms, reinterpret_cast<cudaStream_t>(stream));
}

int paces_mlp_backward(const void* params, const uint16_t* x, const float* y, const float* sw, int64_t n,
                       float inv_norm, float* grads, double* loss, paces_stream_t stream) {
    if (!params || !grads || n < 0 || (n > 0 && (!x || !y || !sw))) return PACES_ERR_BADARG;
    const int sms = device_sms();
    if (sms < 1) return PACES_ERR_CUDA;
    return launch_mlp_backward(params, x, y, sw, n, inv_norm, grads, loss, sms, reinterpret_cast<cudaStream_t>(stream));
}

int paces_mlp_adam(float* master, float* m1, float* m2, float* grads, int32_t t, float lr, float beta1, float beta2,
                   float eps, void* params, paces_stream_t stream) {
    if (!master || !m1 || !m2 || !grads || !params || t < 1) return PACES_ERR_BADARG;
    return launch_mlp_adam(master, m1, m2, grads, t, lr, beta1, beta2, eps, params,
                           reinterpret_cast<cudaStream_t>(stream));
}

// ---- batched trajectories ------------------------------------------------------------------
int paces_batch_create(int32_t max_items, int32_t n_streams, paces_batch** out) {
    if (!out) return PACES_ERR_BADARG;
    *out = nullptr;
    if (max_items < 1 || max_items > kMaxBatch || n_streams < 1 || n_streams > 64) return PACES_ERR_BADARG;
    paces_batch* b = new paces_batch();
    b->max_items = max_items;
    b->n_streams = n_streams;
    b->streams = new cudaStream_t[n_streams]();
    b->join = new cudaEvent_t[n_streams]();
    b->desc = new TaylorBatch();
    b->test_wait_ns = 0;
    b->test_skip_block = -1;
    bool ok = cudaGetDevice(&b->device) == cudaSuccess &&
              cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaMalloc(&b->d_ws, kTaylorBatchWsBytes) == cudaSuccess;
    for (int k = 0; ok && k < n_streams; ++k)
        ok = cudaStreamCreateWithFlags(&b->streams[k], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        paces_batch_destroy(b);
        return PACES_ERR_CUDA;
    }
    *out = b;
    return PACES_OK;
}

int paces_batch_destroy(paces_batch* b) {
    if (!b) return PACES_OK;
    for (int k = 0; k < b->n_streams; ++k) {
        if (b->streams && b->streams[k]) cudaStreamDestroy(b->streams[k]);
        if (b->join && b->join[k]) cudaEventDestroy(b->join[k]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->profiling) paces_batch_set_profiling(b, 0);
    if (b->d_ws) cudaFree(b->d_ws);
    delete[] b->streams;
    delete[] b->join;
    delete b->desc;
    delete b;
    return PACES_OK;
}

const char* paces_batch_last_error(const paces_batch* b) { return b ? b->err : "no batch"; }

int paces_batch_set_test_hooks(paces_batch* b, uint64_t wait_limit_ns, int32_t skip_barrier_block) {
    if (!b || skip_barrier_block < -1 || wait_limit_ns > kWaitLimitNs) return PACES_ERR_BADARG;
    b->test_wait_ns = wait_limit_ns;
    b->test_skip_block = skip_barrier_block;
    return PACES_OK;
}

int paces_batch_set_profiling(paces_batch* b, int32_t on) {
    if (!b) return PACES_ERR_BADARG;
    if (on && !b->profiling)
        for (int i = 0; i < 4; ++i)
            if (cudaEventCreate(&b->ev[i]) != cudaSuccess) return PACES_ERR_CUDA;
    if (!on && b->profiling)
        for (int i = 0; i < 4; ++i) cudaEventDestroy(b->ev[i]);
    b->profiling = on ? 1 : 0;
    return PACES_OK;
}

int paces_batch_stage_times(paces_batch* b, float* ms) {
    if (!b || !ms || !b->profiling) return PACES_ERR_BADARG;
    if (cudaEventSynchronize(b->ev[3]) != cudaSuccess) return PACES_ERR_CUDA;
    for (int i = 0; i < 3; ++i)
        if (cudaEventElapsedTime(&ms[i], b->ev[i], b->ev[i + 1]) != cudaSuccess) return PACES_ERR_CUDA;
    return PACES_OK;
}

unsigned long long paces_batch_kernel_launches(const paces_batch* b) { return b ? b->launches : 0ull; }

int paces_batch_step(paces_batch* b, const paces_batch_item* items, int32_t n, paces_stream_t stream) {
    if (!b) return PACES_ERR_BADARG;
    auto bfail = [&](int code, const char* fmt, ...) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(b->err, sizeof(b->err), fmt, ap);
        va_end(ap);
        return code;
    };
    if (!items || n < 1 || n > b->max_items) return bfail(PACES_ERR_BADARG, "paces_batch_step: %d items (max %d)", n, b->max_items);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int precision = items[0].ctx ? items[0].ctx->precision : -1;
    StepPlan* plans = new StepPlan[n];
    struct Cleanup {
        StepPlan* p;
        ~Cleanup() { delete[] p; }
    } cleanup{plans};
    unsigned long long launches = 0;
    int n_evolve = 0;
    for (int i = 0; i < n; ++i) {
        const paces_batch_item& it = items[i];
        if (!it.ctx) return bfail(PACES_ERR_BADARG, "item %d: no context", i);
        if (it.ctx->precision != precision) return bfail(PACES_ERR_BADARG, "item %d: mixed precisions in one batch", i);
        if (it.ctx->device != b->device) return bfail(PACES_ERR_BADARG, "item %d: context on another device", i);
        if (it.ctx->m.nhop > 1) return bfail(PACES_ERR_BADARG, "item %d: batched steps take chain models only", i);
        if (it.params && it.params->lanczos_order > 0)
            return bfail(PACES_ERR_BADARG, "item %d: batched steps propagate by the Taylor series only", i);
        const int rc = plan_step(it.ctx, it.old_basis, it.old_psi, it.new_basis, it.new_psi, it.h, it.params,
                                 it.record, it.workspace, it.workspace_bytes, &plans[i]);
        if (rc != PACES_OK) return bfail(rc, "item %d: %s", i, it.ctx->err);
        launches += step_launches(*it.params, it.ctx->precision == PACES_C64, false, merge_passes(it.ctx->m));
        n_evolve += it.params->evolve ? 1 : 0;
    }
    auto fork = [&]() -> bool {
        if (cudaEventRecord(b->fork, st) != cudaSuccess) return false;
        for (int k = 0; k < b->n_streams; ++k)
            if (cudaStreamWaitEvent(b->streams[k], b->fork, 0) != cudaSuccess) return false;
        return true;
    };
    auto join = [&]() -> bool {
        for (int k = 0; k < b->n_streams; ++k)
            if (cudaEventRecord(b->join[k], b->streams[k]) != cudaSuccess ||
                cudaStreamWaitEvent(st, b->join[k], 0) != cudaSuccess)
                return false;
        return true;
    };
    auto mark = [&](int i) {
        if (b->profiling) cudaEventRecord(b->ev[i], st);
    };
    // 1. every trajectory's truncation, enlargement, assembly, remap and diagnostics,
    //    spread over the batch's streams
    mark(0);
    if (!fork()) return bfail(PACES_ERR_CUDA, "fork: %s", cudaGetErrorString(cudaGetLastError()));
    for (int i = 0; i < n; ++i) {
        const int rc = step_front(items[i].ctx, plans[i], b->streams[i % b->n_streams], false);
        if (rc != PACES_OK) {
            join();
            return bfail(rc, "item %d: %s", i, items[i].ctx->err);
        }
    }
    if (!join()) return bfail(PACES_ERR_CUDA, "join: %s", cudaGetErrorString(cudaGetLastError()));
    mark(1);
    // 2. the Taylor series.  Batches of large trajectories (every evolving one with room for at
    //    least kBatchSingleCap states) run them one after the other through the single-trajectory
    //    kernel, whose bulk-copy schedule streams long row ranges faster (0.85 against 0.61 of
    //    HBM on 64M-row trajectories); otherwise one persistent launch serves all.  Both give
    //    the same results.  Test hooks on the batch keep the batched launch.
    bool per_item = n_evolve > 0 && b->test_wait_ns == 0 && b->test_skip_block < 0;
    for (int i = 0; i < n && per_item; ++i)
        if (items[i].params->evolve && plans[i].new_b->cap < kBatchSingleCap) per_item = false;
    if (per_item) {
        for (int i = 0; i < n; ++i) {
            const paces_step_params* prm = items[i].params;
            if (!prm->evolve) continue;
            paces_ctx* c = items[i].ctx;
            StepPlan& p = plans[i];
            TaylorWs tw = taylor_ws(c, p.l, p.ws);
            if (diag_in_taylor(prm)) tw.diag = at<double>(p.ws, p.l.diag);
            TaylorOut o{&p.rec->converged, &p.rec->final_m, &p.rec->c1_plus_c2, &p.rec->term_ratio};
            if (launch_taylor(c->precision == PACES_C64, with_h(c, p.h), p.new_b->blk, p.h->nbr, p.h->cap, p.h->meta,
                              p.target, p.new_psi, prm->dt, prm->m_star, prm->tol, tw, o, &p.rec->status, c->num_sms,
                              c->taylor_bps, c->taylor_variant, st) != PACES_OK)
                return bfail(PACES_ERR_CUDA, "item %d: Taylor: %s", i, cudaGetErrorString(cudaGetLastError()));
            launches += 1;
        }
    } else if (n_evolve > 0) {
        TaylorBatch& bt = *b->desc;
        bt.n = 0;
        bt.max_m_star = 0;
        for (int i = 0; i < n; ++i) {
            const paces_step_params* prm = items[i].params;
            if (!prm->evolve) continue;
            paces_ctx* c = items[i].ctx;
            const StepPlan& p = plans[i];
            const TaylorWs tw = taylor_ws(c, p.l, p.ws);
            TaylorItem& ti = bt.items[bt.n++];
            ti.blk = p.new_b->blk;
            ti.nbr = p.h->nbr;
            ti.meta = p.h->meta;
            ti.v_in = p.target;
            ti.res = p.new_psi;
            ti.ta = tw.ta;
            ti.tb = tw.tb;
            ti.site_eps = c->d_site_eps;
            ti.sq = c->d_sq;
            ti.sqf = c->d_sqf;
            ti.status = &p.rec->status;
            ti.diag = diag_in_taylor(prm) ? at<double>(p.ws, p.l.diag) : nullptr;
            ti.out = TaylorOut{&p.rec->converged, &p.rec->final_m, &p.rec->c1_plus_c2, &p.rec->term_ratio};
            ti.dt = prm->dt;
            ti.tol = prm->tol;
            ti.eps_sys = c->m.eps_sys;
            ti.hbar_omega = c->m.hbar_omega;
            ti.delta_eps = c->m.delta_eps;
            ti.J = c->m.J;
            ti.L = c->m.L;
            ti.has_site_eps = c->m.has_site_eps;
            ti.m_star = prm->m_star;
            ti.pad = 0;
            if (prm->m_star > bt.max_m_star) bt.max_m_star = prm->m_star;
        }
        TaylorBatchWs tws;
        tws.barrier = static_cast<unsigned*>(b->d_ws);
        tws.maxima = reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(b->d_ws) + 256);
        tws.wait_ns = b->test_wait_ns ? b->test_wait_ns : kWaitLimitNs;
        tws.skip_block = b->test_skip_block;
        if (launch_taylor_batch(precision == PACES_C64, bt, tws, b->num_sms, items[0].ctx->taylor_bps, st) != PACES_OK)
            return bfail(PACES_ERR_CUDA, "batched Taylor: %s", cudaGetErrorString(cudaGetLastError()));
        launches += 1;
    }
    mark(2);
    // 3. renormalisation, observables and records, again spread over the streams
    if (!fork()) return bfail(PACES_ERR_CUDA, "fork: %s", cudaGetErrorString(cudaGetLastError()));
    for (int i = 0; i < n; ++i) {
        const int rc = step_back(items[i].ctx, plans[i], b->streams[i % b->n_streams], false);
        if (rc != PACES_OK) {
            join();
            return bfail(rc, "item %d: %s", i, items[i].ctx->err);
        }
    }
    if (!join()) return bfail(PACES_ERR_CUDA, "join: %s", cudaGetErrorString(cudaGetLastError()));
    mark(3);
    b->launches += launches;
    return PACES_OK;
}

}  // extern "C"
