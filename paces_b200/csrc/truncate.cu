// Amplitude-ranked truncation (see truncate.cuh).
#include <type_traits>

#include "truncate.cuh"

namespace paces {

namespace {

// selection state words (TruncWs.sel)
enum : int {
    SEL_S = 0,        // number of input states
    SEL_ALL = 1,      // 1: keep everything (S <= maxstates)
    SEL_W = 2,        // weight select: [2] prefix [3] mask [4] need [5] active
    SEL_H = 6,        // hash select:   [6] prefix [7] mask [8] need [9] active
    SEL_CAND = 10,    // candidate count
    SEL_TIES = 11,    // states equal to the threshold
    SEL_SHUFFLE = 12, // 1: ties at the cut are shuffled
    SEL_WORDS = 16
};

constexpr int kRounds = 6;
__host__ __device__ constexpr int round_shift(int r) { return r < 5 ? 52 - 12 * r : 0; }
__host__ __device__ constexpr int round_bits(int r) { return r < 5 ? 12 : 4; }

// The ranked weight of state i: WK 0 = |psi| of complex128 amplitudes, 1 = |psi| of
// complex64 amplitudes, 2 = precomputed non-negative fp64 weights (the look-ahead
// weighting, or |psi| of complex128 amplitudes stored by the first radix round), 3 = |psi|
// of complex64 amplitudes stored as fp32 by the first round (exact: hypotf's result,
// widened like WK 1 widens it).  Non-negative doubles order like their bit patterns.  The
// load and the conversion are separate so that loops can issue several loads before the
// first use.
template <int WK>
using RawW = typename std::conditional<
    WK == 0, double2,
    typename std::conditional<WK == 1, float2, typename std::conditional<WK == 2, double, float>::type>::type>::type;

// the kind the first round stores for later passes (WK 0 -> 2, WK 1 -> 3)
__host__ __device__ constexpr int stored_kind(int wk) { return wk == 1 ? 3 : 2; }

template <int WK>
__device__ __forceinline__ RawW<WK> load_raw(const void* psi, int64_t i) {
    return __ldcs(reinterpret_cast<const RawW<WK>*>(psi) + i);
}

template <int WK>
__device__ __forceinline__ unsigned long long raw_bits(const RawW<WK>& z, int* status) {
    double w;
    if constexpr (WK == 1) w = double(hypotf(z.x, z.y));
    else if constexpr (WK == 0) w = hypot(z.x, z.y);
    else w = double(z);
    if (!(w <= 1.7976931348623157e308)) raise_status(status, PACES_ERR_NONFINITE);
    return (unsigned long long)__double_as_longlong(w);
}

template <int WK>
__device__ __forceinline__ unsigned long long weight_bits(const void* psi, int64_t i, int* status) {
    return raw_bits<WK>(load_raw<WK>(psi, i), status);
}

// splitmix64 finaliser applied to (index + stream offset): a bijection of the index, so
// hashes of distinct states never collide.
__device__ __forceinline__ unsigned long long tie_hash(uint64_t seed, uint64_t step, int64_t i) {
    unsigned long long z = (unsigned long long)i + seed * 0x9E3779B97F4A7C15ull + step * 0xD1B54A32D192ED03ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return ~z;  // keep the largest ~hash == the smallest hash
}

__global__ void trunc_init_kernel(ModelDev m, const int* __restrict__ x_blk, int64_t maxstates,
                                  TruncWs ws) {
    const int tid = threadIdx.x;
    for (int b = tid; b < 4096; b += blockDim.x) ws.hist[b] = 0;
    if (tid == 0) {
        const long long S = x_blk[m.L];
        for (int k = 0; k < SEL_WORDS; ++k) ws.sel[k] = 0;
        ws.sel[SEL_S] = S;
        ws.sel[SEL_ALL] = S <= maxstates ? 1 : 0;
        ws.sel[SEL_W + 2] = maxstates;
        ws.sel[SEL_W + 3] = S <= maxstates ? 0 : 1;
    }
}

// One radix round: find the digit holding the need-th largest key, narrow the prefix;
// on the final round (record_ties) the chosen bin's count is the number of tied states.
__global__ void __launch_bounds__(1024) trunc_select_kernel(TruncWs ws, int base, int round,
                                                            int record_ties) {
    __shared__ long long s_warp[32];
    __shared__ int s_bin;
    __shared__ long long s_above;
    if (!ws.sel[base + 3]) return;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int bits = round_bits(round), shift = round_shift(round);
    const int nb = 1 << bits;
    const int per = (nb + 1023) / 1024;  // 4 or 1
    const long long need = ws.sel[base + 2];
    long long mine = 0;
    for (int q = 0; q < per; ++q) {
        const int b = tid * per + q;
        if (b < nb) mine += ws.hist[b];
    }
    // suffix sums: threads above me
    long long incl = mine;  // inclusive suffix within the warp (lanes >= lane)
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long v = __shfl_down_sync(0xffffffffu, incl, o);
        if (lane + o < 32) incl += v;
    }
    if (lane == 0) s_warp[wid] = incl;
    if (tid == 0) s_bin = -1;
    __syncthreads();
    long long warps_above = 0;
    for (int w = wid + 1; w < 32; ++w) warps_above += s_warp[w];
    const long long above_me = warps_above + (incl - mine);  // sum of bins above my range
    if (mine > 0 && above_me < need && need <= above_me + mine) {
        long long acc = above_me;
        for (int q = per - 1; q >= 0; --q) {
            const int b = tid * per + q;
            if (b >= nb) continue;
            const long long hb = ws.hist[b];
            if (acc < need && need <= acc + hb) {
                s_bin = b;
                s_above = acc;
                break;
            }
            acc += hb;
        }
    }
    __syncthreads();
    if (tid == 0 && s_bin >= 0) {
        const int b = s_bin;
        ws.sel[base + 2] = need - s_above;
        ws.sel[base + 0] |= (long long)((unsigned long long)b << shift);
        ws.sel[base + 1] |= (long long)((unsigned long long)(nb - 1) << shift);
        if (record_ties) ws.sel[SEL_TIES] = ws.hist[b];
    }
    __syncthreads();
    for (int b = tid; b < 4096; b += blockDim.x) ws.hist[b] = 0;
}

// One radix round over all states: histogram of the round's digit among the states whose
// higher digits equal the prefix chosen so far (round 0: every state).  A full streaming
// pass per round -- no candidate list, so no global counter and no scattered writes.  Lanes
// with the same digit add to the shared histogram once (warp-aggregated: in round 0 most
// states share a few binades).
// STORE (round 0 of |psi| kinds): also write every state's weight to `wout` in the stored
// kind, which the later passes read instead of recomputing |psi|.
template <int WK, bool STORE>
__global__ void __launch_bounds__(256) trunc_hist_pass_kernel(const void* __restrict__ psi, TruncWs ws, int round,
                                                              void* __restrict__ wout, int* status) {
    __shared__ unsigned h[4096];
    if (!ws.sel[SEL_W + 3]) return;
    const int bits = round_bits(round), shift = round_shift(round);
    const unsigned long long dm = (1ull << bits) - 1;
    for (int b = threadIdx.x; b < (1 << bits); b += blockDim.x) h[b] = 0;
    __syncthreads();
    const int64_t S = ws.sel[SEL_S];
    const unsigned long long pre = (unsigned long long)ws.sel[SEL_W + 0];
    const unsigned long long msk = (unsigned long long)ws.sel[SEL_W + 1];
    const int lane = threadIdx.x & 31;
    // warp chunks of 4 x 32 states: the four loads of a lane are in flight together
    constexpr int kU = 4;
    const int64_t nwarps = int64_t(gridDim.x) * (blockDim.x >> 5);
    for (int64_t c = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); c * 32 * kU < S; c += nwarps) {
        RawW<WK> z[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int64_t i = (c * kU + u) * 32 + lane;
            if (i < S) z[u] = load_raw<WK>(psi, i);
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int64_t i = (c * kU + u) * 32 + lane;
            bool match = false;
            unsigned bin = 0xffffffffu;
            if (i < S) {
                const unsigned long long k = raw_bits<WK>(z[u], status);
                if constexpr (STORE) {
                    const double wv = __longlong_as_double((long long)k);
                    if constexpr (stored_kind(WK) == 3) reinterpret_cast<float*>(wout)[i] = float(wv);
                    else reinterpret_cast<double*>(wout)[i] = wv;
                }
                match = (k & msk) == pre;
                if (match) bin = unsigned((k >> shift) & dm);
            }
            const unsigned peers = __match_any_sync(0xffffffffu, bin);
            if (match && lane == __ffs(peers) - 1) atomicAdd(&h[bin], unsigned(__popc(peers)));
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < (1 << bits); b += blockDim.x)
        if (h[b]) atomicAdd(&ws.hist[b], h[b]);
}

__global__ void __launch_bounds__(256) trunc_hist_cand_kernel(TruncWs ws, int base, int round) {
    __shared__ unsigned h[4096];
    if (!ws.sel[base + 3]) return;
    const int bits = round_bits(round), shift = round_shift(round);
    const unsigned long long dm = (1ull << bits) - 1;
    for (int b = threadIdx.x; b < 4096; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const long long nc = min(ws.sel[SEL_CAND], (long long)ws.cap);
    const unsigned long long pre = (unsigned long long)ws.sel[base + 0];
    const unsigned long long msk = (unsigned long long)ws.sel[base + 1];
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = ws.cand[c];
        if ((k & msk) == pre) atomicAdd(&h[(k >> shift) & dm], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < (1 << bits); b += blockDim.x)
        if (h[b]) atomicAdd(&ws.hist[b], h[b]);
}

// Decide whether the tie at the cut is shuffled; if so, collect the tied states' hashes.
__global__ void trunc_shuffle_prep_kernel(TruncWs ws, int* status) {
    if (threadIdx.x != 0) return;
    const long long ties = ws.sel[SEL_TIES];
    const long long need = ws.sel[SEL_W + 2];
    const bool active = ws.sel[SEL_W + 3] && ties > need;
    ws.sel[SEL_SHUFFLE] = active ? 1 : 0;
    if (active && double(ties) > 0.9 * double(ws.sel[SEL_S])) raise_status(status, PACES_ERR_SHUFFLE);
    ws.sel[SEL_H + 0] = 0;
    ws.sel[SEL_H + 1] = 0;
    ws.sel[SEL_H + 2] = need;
    ws.sel[SEL_H + 3] = active ? 1 : 0;
    ws.sel[SEL_CAND] = 0;
}

template <int WK>
__global__ void __launch_bounds__(256) trunc_collect_ties_kernel(const void* __restrict__ psi, TruncWs ws,
                                                                 uint64_t seed, uint64_t step, int* status) {
    if (!ws.sel[SEL_H + 3]) return;
    const int64_t S = ws.sel[SEL_S];
    const unsigned long long vstar = (unsigned long long)ws.sel[SEL_W + 0];
    const int lane = threadIdx.x & 31;
    for (int64_t i0 = blockIdx.x * int64_t(blockDim.x); i0 < S; i0 += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = i0 + threadIdx.x;
        bool take = false;
        if (i < S) take = weight_bits<WK>(psi, i, status) == vstar;
        const unsigned ballot = __ballot_sync(0xffffffffu, take);
        if (!ballot) continue;
        int basei = 0;
        if (lane == 0) basei = int(atomicAdd(reinterpret_cast<unsigned long long*>(&ws.sel[SEL_CAND]),
                                            (unsigned long long)__popc(ballot)));
        basei = __shfl_sync(0xffffffffu, basei, 0);
        if (take) {
            const int slot = basei + __popc(ballot & ((1u << lane) - 1));
            if (slot < ws.cap) {
                ws.cand[slot] = tie_hash(seed, step, i);
                ws.cand_idx[slot] = int(i);
            }
        }
    }
}

// Per tile: states above the threshold, tied states, tied states kept by the hash rule.
template <int WK>
__global__ void __launch_bounds__(256) trunc_count_kernel(const void* __restrict__ psi, TruncWs ws,
                                                          uint64_t seed, uint64_t step, int* status) {
    __shared__ int s_c[3];
    const int64_t S = ws.sel[SEL_S];
    const int ntiles = int((S + kTruncTile - 1) / kTruncTile);
    if (ws.sel[SEL_ALL]) return;
    const unsigned long long vstar = (unsigned long long)ws.sel[SEL_W + 0];
    const bool shuf = ws.sel[SEL_SHUFFLE] != 0;
    const unsigned long long hstar = (unsigned long long)ws.sel[SEL_H + 0];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        if (threadIdx.x < 3) s_c[threadIdx.x] = 0;
        __syncthreads();
        int a = 0, ti = 0, hk = 0;
        const int64_t i1 = min(S, int64_t(t + 1) * kTruncTile);
        constexpr int kU = 4;  // loads in flight per thread
        for (int64_t i0 = int64_t(t) * kTruncTile + threadIdx.x; i0 < i1; i0 += kU * int64_t(blockDim.x)) {
            RawW<WK> z[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (i0 + u * int64_t(blockDim.x) < i1) z[u] = load_raw<WK>(psi, i0 + u * int64_t(blockDim.x));
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int64_t i = i0 + u * int64_t(blockDim.x);
                if (i >= i1) break;
                const unsigned long long k = raw_bits<WK>(z[u], status);
                a += k > vstar;
                if (k == vstar) {
                    ++ti;
                    if (shuf) hk += tie_hash(seed, step, i) >= hstar;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            ti += __shfl_xor_sync(0xffffffffu, ti, o);
            hk += __shfl_xor_sync(0xffffffffu, hk, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&s_c[0], a);
            atomicAdd(&s_c[1], ti);
            atomicAdd(&s_c[2], hk);
        }
        __syncthreads();
        if (threadIdx.x < 3) ws.tile_cnt[t * 3 + threadIdx.x] = s_c[threadIdx.x];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(1024) trunc_scan_kernel(TruncWs ws) {
    __shared__ int s_w[32][3];
    if (ws.sel[SEL_ALL]) return;
    const int64_t S = ws.sel[SEL_S];
    const int ntiles = int((S + kTruncTile - 1) / kTruncTile);
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int per = (ntiles + 1023) / 1024;
    const int t0 = min(tid * per, ntiles), t1 = min(t0 + per, ntiles);
    int c[3] = {0, 0, 0};
    for (int t = t0; t < t1; ++t)
        for (int k = 0; k < 3; ++k) c[k] += ws.tile_cnt[t * 3 + k];
    int incl[3];
    for (int k = 0; k < 3; ++k) {
        incl[k] = c[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl[k], o);
            if (lane >= o) incl[k] += v;
        }
        if (lane == 31) s_w[wid][k] = incl[k];
    }
    __syncthreads();
    if (tid < 3) {
        int acc = 0;
        for (int w = 0; w < 32; ++w) {
            const int v = s_w[w][tid];
            s_w[w][tid] = acc;
            acc += v;
        }
    }
    __syncthreads();
    int run[3];
    for (int k = 0; k < 3; ++k) run[k] = s_w[wid][k] + incl[k] - c[k];
    for (int t = t0; t < t1; ++t)
        for (int k = 0; k < 3; ++k) {
            ws.tile_pre[t * 3 + k] = run[k];
            run[k] += ws.tile_cnt[t * 3 + k];
        }
}

// The compaction: every warp owns kTruncTile / 8 consecutive states of the tile.  Pass 1
// counts, per warp, the states above the threshold, the tied ones and the tied ones the
// hash keeps (ballots); pass 2 walks the same states 32 at a time and places every kept
// state at its rank among the kept ones (ballot prefixes).  Lanes read consecutive keys
// and the kept ones write consecutive outputs, so both sides coalesce.
// The weights come from `wsrc` (kind WK); when every state is kept the selection rounds
// did not run, so the out_w weights come from `psi` (kind WKA).
template <int NW, int WK, int WKA>
__global__ void __launch_bounds__(256) trunc_write_kernel(ModelDev m, const uint64_t* __restrict__ x_keys,
                                                          const int* __restrict__ x_blk,
                                                          const void* __restrict__ wsrc,
                                                          const void* __restrict__ psi, TruncWs ws,
                                                          uint64_t seed, uint64_t step,
                                                          uint64_t* __restrict__ out_keys,
                                                          int* __restrict__ out_blk, int64_t out_cap,
                                                          float* __restrict__ out_w, int* status) {
    constexpr int kWarps = 8;
    constexpr int kSeg = kTruncTile / kWarps;
    __shared__ unsigned long long s_k[kTruncTile];
    __shared__ int s_blk[kMaxSites + 1];
    __shared__ int s_w[kWarps][3];
    const int L = m.L;
    for (int i = threadIdx.x; i <= L; i += blockDim.x) s_blk[i] = x_blk[i];
    const int64_t S = ws.sel[SEL_S];
    const bool all = ws.sel[SEL_ALL] != 0;
    const int ntiles = int((S + kTruncTile - 1) / kTruncTile);
    const unsigned long long vstar = (unsigned long long)ws.sel[SEL_W + 0];
    const long long need = ws.sel[SEL_W + 2];
    const long long ties = ws.sel[SEL_TIES];
    const long long skip_ties = ties - need;  // tied states dropped (the lowest indices)
    const bool shuf = ws.sel[SEL_SHUFFLE] != 0;
    const unsigned long long hstar = (unsigned long long)ws.sel[SEL_H + 0];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    __syncthreads();
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t i0 = int64_t(t) * kTruncTile;
        const int n = int(min(int64_t(kTruncTile), S - i0));
        const int q_lo = min(wid * kSeg, n), q_hi = min(q_lo + kSeg, n);
        // pass 1: weights into shared memory, per-warp counts
        int ca = 0, ct = 0, ch = 0;
        if (!all || out_w) {
            constexpr int kU = 4;  // loads in flight per lane
            if (WK != WKA && all) {
                // every state kept (early steps only): out_w from the amplitudes
                for (int q = q_lo + lane; q < q_hi; q += 32) s_k[q] = raw_bits<WKA>(load_raw<WKA>(psi, i0 + q), status);
            } else {
                for (int q0 = q_lo; q0 < q_hi; q0 += 32 * kU) {
                    RawW<WK> z[kU];
#pragma unroll
                    for (int u = 0; u < kU; ++u) {
                        const int q = q0 + 32 * u + lane;
                        if (q < q_hi) z[u] = load_raw<WK>(wsrc, i0 + q);
                    }
#pragma unroll
                    for (int u = 0; u < kU; ++u) {
                        const int q = q0 + 32 * u + lane;
                        if (q < q_hi) s_k[q] = raw_bits<WK>(z[u], status);
                    }
                }
            }
            __syncwarp();
            if (!all)
                for (int q0 = q_lo; q0 < q_hi; q0 += 32) {
                    const int q = q0 + lane;
                    const bool v = q < q_hi;
                    const unsigned long long k = v ? s_k[q] : 0ull;
                    const bool tie = v && k == vstar;
                    ca += __popc(__ballot_sync(0xffffffffu, v && k > vstar));
                    ct += __popc(__ballot_sync(0xffffffffu, tie));
                    if (shuf) ch += __popc(__ballot_sync(0xffffffffu, tie && tie_hash(seed, step, i0 + q) >= hstar));
                }
        }
        if (lane == 0) {
            s_w[wid][0] = ca;
            s_w[wid][1] = ct;
            s_w[wid][2] = ch;
        }
        __syncthreads();
        long long A = 0, T = 0, H = 0;
        if (!all) {
            A = ws.tile_pre[t * 3 + 0];
            T = ws.tile_pre[t * 3 + 1];
            H = ws.tile_pre[t * 3 + 2];
            for (int w = 0; w < wid; ++w) {
                A += s_w[w][0];
                T += s_w[w][1];
                H += s_w[w][2];
            }
        }
        // pass 2: ranks among the kept states, block starts, copies; four slices of 32 per
        // round, their key loads in flight together.  Exciton blocks start in few of the
        // warp's segments: a warp whose segment holds no block start skips their search.
        bool starts = false;
        for (int p = lane; p < L; p += 32) {
            const int64_t b0 = s_blk[p];
            starts |= b0 >= i0 + q_lo && b0 < i0 + q_hi && b0 < s_blk[p + 1];
        }
        starts = __any_sync(0xffffffffu, starts);
        constexpr int kU = 4;
        for (int qb = q_lo; qb < q_hi; qb += 32 * kU) {
            bool keep[kU];
            long long out[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int q0 = qb + 32 * u;
                const int q = q0 + lane;
                const bool v = q < q_hi;
                const int64_t i = i0 + q;
                if (all) {
                    keep[u] = v;
                    out[u] = i;
                } else {
                    const unsigned long long k = v ? s_k[q] : 0ull;
                    const bool above = v && k > vstar;
                    const bool tie = v && k == vstar;
                    const bool hk = shuf && tie && tie_hash(seed, step, i) >= hstar;
                    const unsigned ba = __ballot_sync(0xffffffffu, above);
                    const unsigned bt = __ballot_sync(0xffffffffu, tie);
                    const unsigned bh = __ballot_sync(0xffffffffu, hk);
                    const long long a_l = A + __popc(ba & lt_mask);
                    const long long t_l = T + __popc(bt & lt_mask);
                    const long long h_l = H + __popc(bh & lt_mask);
                    out[u] = a_l + (shuf ? h_l : max(0ll, t_l - skip_ties));
                    keep[u] = above || (tie && (shuf ? hk : t_l >= skip_ties));
                    A += __popc(ba);
                    T += __popc(bt);
                    H += __popc(bh);
                }
                // block starts among these 32 states: the number of kept states before them
                for (int p0 = 0; starts && p0 < L; p0 += 32) {
                    const int p = p0 + lane;
                    const int e = p < L ? int(int64_t(s_blk[p]) - (i0 + q0)) : -1;
                    const long long o = __shfl_sync(0xffffffffu, out[u], (e >= 0 && e < 32) ? e : 0);
                    if (p < L && e >= 0 && e < 32 && q0 + e < q_hi && s_blk[p] < s_blk[p + 1]) out_blk[p] = int(o);
                }
            }
            Key<NW> kk[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (keep[u] && out[u] < out_cap) kk[u] = load_key<NW>(x_keys, i0 + qb + 32 * u + lane);
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                if (!keep[u]) continue;
                if (out[u] < out_cap) {
                    store_key<NW>(out_keys, out[u], kk[u]);
                    if (out_w) out_w[out[u]] = float(__longlong_as_double((long long)s_k[qb + 32 * u + lane]));
                } else {
                    raise_status(status, PACES_ERR_CAPACITY);
                }
            }
        }
        __syncthreads();
    }
}

__global__ void trunc_finalize_kernel(ModelDev m, const int* __restrict__ x_blk, int64_t maxstates,
                                      TruncWs ws, int* out_blk, int64_t out_cap, int* n_tied_out, int* n_kept_out,
                                      float* cut_out, int* status) {
    if (threadIdx.x != 0) return;
    // the cut: |psi| of the smallest kept state when states were dropped, else 0
    if (cut_out) *cut_out = ws.sel[SEL_ALL] ? 0.f : float(__longlong_as_double(ws.sel[SEL_W + 0]));
    const int L = m.L;
    const long long S = ws.sel[SEL_S];
    long long total = ws.sel[SEL_ALL] ? S : maxstates;
    if (total > out_cap) {
        raise_status(status, PACES_ERR_CAPACITY);
        total = out_cap;
    }
    if (ws.sel[SEL_CAND] > ws.cap) raise_status(status, PACES_ERR_CAPACITY);
    out_blk[L] = int(total);
    for (int p = L - 1; p >= 0; --p)
        if (x_blk[p] == x_blk[p + 1]) out_blk[p] = out_blk[p + 1];
    if (n_tied_out) *n_tied_out = int(ws.sel[SEL_ALL] ? 0 : ws.sel[SEL_TIES]);
    if (n_kept_out) *n_kept_out = int(total);
}

// WK: the kind of `psi`.  WKS: the kind the passes after round 0 read from `src` -- WK
// itself reading `psi`, or the stored kind reading the weights round 0 wrote to scratch.
template <int NW, int WK, int WKS>
int launch_truncate_t(const ModelDev& m, const uint64_t* x_keys, const int* x_blk, const void* psi, void* scratch,
                      int64_t maxstates, int shuffle, uint64_t seed, uint64_t step, const TruncWs& ws,
                      uint64_t* out_keys, int* out_blk, int64_t out_cap, float* out_w, int* n_tied_out, int* n_kept_out,
                      int* status, int num_sms, cudaStream_t st) {
    constexpr bool kStore = WKS != WK;
    const void* src = kStore ? scratch : psi;
    const int g = grid_for(ws.cap, 1024, num_sms * 4);          // streaming passes
    const int gt = grid_for(ws.cap, kTruncTile, num_sms * 4);   // passes over 4096-state tiles
    const int rounds = weight_rounds(WK);
    trunc_init_kernel<<<1, 1024, 0, st>>>(m, x_blk, maxstates, ws);
    for (int r = 0; r < rounds; ++r) {
        if (r == 0) trunc_hist_pass_kernel<WK, kStore><<<g, 256, 0, st>>>(psi, ws, r, scratch, status);
        else trunc_hist_pass_kernel<WKS, false><<<g, 256, 0, st>>>(src, ws, r, nullptr, status);
        trunc_select_kernel<<<1, 1024, 0, st>>>(ws, SEL_W, r, r == rounds - 1);
    }
    if (shuffle) {
        trunc_shuffle_prep_kernel<<<1, 32, 0, st>>>(ws, status);
        trunc_collect_ties_kernel<WKS><<<g, 256, 0, st>>>(src, ws, seed, step, status);
        for (int r = 0; r < kRounds; ++r) {
            trunc_hist_cand_kernel<<<g, 256, 0, st>>>(ws, SEL_H, r);
            trunc_select_kernel<<<1, 1024, 0, st>>>(ws, SEL_H, r, 0);
        }
    }
    trunc_count_kernel<WKS><<<gt, 256, 0, st>>>(src, ws, seed, step, status);
    trunc_scan_kernel<<<1, 1024, 0, st>>>(ws);
    trunc_write_kernel<NW, WKS, WK><<<gt, 256, 0, st>>>(m, x_keys, x_blk, src, psi, ws, seed, step, out_keys,
                                                        out_blk, out_cap, out_w, status);
    trunc_finalize_kernel<<<1, 32, 0, st>>>(m, x_blk, maxstates, ws, out_blk, out_cap, n_tied_out, n_kept_out,
                                            out_w ? out_w + out_cap : nullptr, status);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

template <int NW>
int dispatch_prec(bool c64, const ModelDev& m, const uint64_t* x_keys, const int* x_blk,
                  const void* psi, const double* weights, void* scratch, int64_t maxstates, int shuffle, uint64_t seed,
                  uint64_t step, const TruncWs& ws, uint64_t* out_keys, int* out_blk, int64_t out_cap,
                  float* out_w, int* n_tied_out, int* n_kept_out, int* status, int num_sms, cudaStream_t st) {
#define PACES_TRUNC_LAUNCH(WK, WKS, SRC)                                                                     \
    return launch_truncate_t<NW, WK, WKS>(m, x_keys, x_blk, SRC, scratch, maxstates, shuffle, seed, step, ws, \
                                          out_keys, out_blk, out_cap, out_w, n_tied_out, n_kept_out, status,  \
                                          num_sms, st)
    if (weights) PACES_TRUNC_LAUNCH(2, 2, weights);
    if (c64) {
        if (scratch) PACES_TRUNC_LAUNCH(1, stored_kind(1), psi);
        PACES_TRUNC_LAUNCH(1, 1, psi);
    }
    if (scratch) PACES_TRUNC_LAUNCH(0, stored_kind(0), psi);
    PACES_TRUNC_LAUNCH(0, 0, psi);
#undef PACES_TRUNC_LAUNCH
}

}  // namespace

int launch_truncate(int nw, bool c64, const ModelDev& m, const uint64_t* x_keys, const int* x_blk,
                    const void* psi, const double* weights, void* scratch, int64_t maxstates, int shuffle, uint64_t seed,
                    uint64_t step, const TruncWs& ws, uint64_t* out_keys, int* out_blk, int64_t out_cap, float* out_w,
                    int* n_tied_out, int* n_kept_out, int* status, int num_sms, cudaStream_t st) {
#define PACES_TRUNC_CASE(N)                                                                       \
    case N:                                                                                       \
        return dispatch_prec<N>(c64, m, x_keys, x_blk, psi, weights, scratch, maxstates, shuffle, seed, step, ws, \
                                out_keys, out_blk, out_cap, out_w, n_tied_out, n_kept_out, status, num_sms, st);
    switch (nw) {
        PACES_TRUNC_CASE(1)
        PACES_TRUNC_CASE(2)
        PACES_TRUNC_CASE(3)
        PACES_TRUNC_CASE(4)
        PACES_TRUNC_CASE(5)
        PACES_TRUNC_CASE(6)
        PACES_TRUNC_CASE(7)
        PACES_TRUNC_CASE(8)
        default: return PACES_ERR_BADARG;
    }
#undef PACES_TRUNC_CASE
}

}  // namespace paces
