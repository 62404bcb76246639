// Structured k-way merge kernels (see merge.cuh for the design).
#include "kernels.cuh"
#include "tc.cuh"

namespace paces {

namespace {

constexpr int kTileThreads = 256;
constexpr unsigned long long kLbAgg = 1ull << 62;
constexpr unsigned long long kLbInc = 2ull << 62;
constexpr unsigned long long kLbMask = (1ull << 62) - 1;

// Source block of run j of output block p, or -1.  A hop run reads the block its images come
// from when that block's hop stays inside its lattice row (the ring wraps instead).
__device__ __forceinline__ int run_source(const ModelDev& m, const MergeWs& ws, int p, int j) {
    const int kind = ws.run_kind[j];
    if (kind == RK_FROM_LOWER) {
        const int s = p - ws.run_dist[j];
        if (m.periodic) return s >= 0 ? s : s + m.L;
        return (s >= 0 && s % ws.run_mod[j] < ws.run_mod[j] - ws.run_dist[j]) ? s : -1;
    }
    if (kind == RK_FROM_UPPER) {
        const int s = p + ws.run_dist[j];
        if (m.periodic) return s < m.L ? s : s - m.L;
        return (s < m.L && s % ws.run_mod[j] >= ws.run_dist[j]) ? s : -1;
    }
    if (kind == RK_EMPTY) return -1;
    return p;
}

// Element `src` of X as it appears in run j of block p: key and order flag
// (0 = floor hole, 1 = real, 2 = ceiling hole).
template <int NW>
__device__ __forceinline__ void run_transform(const ModelDev& m, const MergeWs& ws, int p, int j, int64_t src,
                                              Key<NW>& k, int& flag) {
    flag = 1;
    if (ws.keep && j != RUN_SELF && src < ws.keep_cap && !__ldg(ws.keep + j * ws.keep_cap + src)) flag = 2;
    const int kind = ws.run_kind[j];
    if (kind == RK_UP || kind == RK_DOWN) {
        const int w = m.word[p];
        const int sh = m.shift[p];
        const uint32_t n = get_field(m, k, p);
        const uint64_t low = sh == 0 ? 0ull : ((uint64_t(1) << sh) - 1);
        if (kind == RK_UP) {
            if (n + 1 >= m.maxd[p]) {
                flag = 2;
#pragma unroll
                for (int q = 0; q < NW; ++q)
                    k.w[q] = (k.w[q] | (low & (0ull - uint64_t(q == w)))) | (0ull - uint64_t(q > w));
            } else {
                add_field(m, k, p, +1);
            }
        } else {
            if (n == 0) {
                flag = 0;
#pragma unroll
                for (int q = 0; q < NW; ++q)
                    k.w[q] = (k.w[q] & ~(low & (0ull - uint64_t(q == w)))) & ~(0ull - uint64_t(q > w));
            } else {
                add_field(m, k, p, -1);
            }
        }
    }
}

template <int NW>
__device__ __forceinline__ void run_elem(const ModelDev& m, const uint64_t* __restrict__ X,
                                         const uint64_t* __restrict__ Y, const MergeWs& ws, int p, int j,
                                         int64_t src, Key<NW>& k, int& flag) {
    k = load_key<NW>(j == RUN_SELF ? X : Y, src);
    run_transform<NW>(m, ws, p, j, src, k, flag);
}

template <int NW>
__device__ __forceinline__ int cmp_kf(const Key<NW>& a, int fa, const Key<NW>& b, int fb) {
    int c = key_cmp(a, b);
    return c != 0 ? c : (fa - fb);
}

// Tile keys in shared memory, element-major (w[e*NW + q]): a probe of an element reads its
// whole key with 16-byte loads (NW even) instead of one load per word.
template <int NW>
struct SKeys {
    uint64_t* w;
    __device__ __forceinline__ Key<NW> get(int e) const {
        Key<NW> k;
        if constexpr (NW % 2 == 0) {
            const ulonglong2* p = reinterpret_cast<const ulonglong2*>(w + size_t(e) * NW);
#pragma unroll
            for (int q = 0; q < NW / 2; ++q) {
                const ulonglong2 v = p[q];
                k.w[2 * q] = v.x;
                k.w[2 * q + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int q = 0; q < NW; ++q) k.w[q] = w[size_t(e) * NW + q];
        }
        return k;
    }
    __device__ __forceinline__ void set(int e, const Key<NW>& k) const {
        if constexpr (NW % 2 == 0) {
            ulonglong2* p = reinterpret_cast<ulonglong2*>(w + size_t(e) * NW);
#pragma unroll
            for (int q = 0; q < NW / 2; ++q) p[q] = make_ulonglong2(k.w[2 * q], k.w[2 * q + 1]);
        } else {
#pragma unroll
            for (int q = 0; q < NW; ++q) w[size_t(e) * NW + q] = k.w[q];
        }
    }
};

// (key, flag) pairs held in registers: a strictly below b.  Branch-free fold from the least
// significant word, so a warp's lanes never diverge on where their keys first differ.
template <int NW>
__device__ __forceinline__ bool reg_less(const Key<NW>& a, int fa, const Key<NW>& b, int fb) {
    bool lt = fa < fb;
#pragma unroll
    for (int q = NW - 1; q >= 0; --q) lt = (a.w[q] < b.w[q]) | ((a.w[q] == b.w[q]) & lt);
    return lt;
}

template <int NW>
__device__ __forceinline__ bool reg_eq(const Key<NW>& a, const Key<NW>& b) {
    bool eq = true;
#pragma unroll
    for (int q = 0; q < NW; ++q) eq &= a.w[q] == b.w[q];
    return eq;
}

// Entries of a merged level (and of the tile's merged order): the element's index in the tile
// in the low kEntBits bits, its order flag above them, so that reading an entry gives both.
constexpr int kEntBits = 12;
constexpr int kEntMask = (1 << kEntBits) - 1;
static_assert(merge_tmax(merge_stride(1)) <= (1 << kEntBits), "tile element index must fit an entry");

__device__ __forceinline__ uint16_t make_ent(int e, int f) { return uint16_t(e | (f << kEntBits)); }

// A sorted sequence of tile elements: a run segment (element k is base + k, its flag in the
// tile's flag array) or a merged level (entry k of ptr).  Which of the two a sequence is, is a
// template argument of every function that reads one (ARR: a merged level).
struct Seq {
    const uint16_t* ptr;
    int base;
    int n;
};

template <bool ARR>
__device__ __forceinline__ void seq_at(const Seq& s, const uint8_t* flags, int k, int& e, int& f) {
    if constexpr (ARR) {
        const int v = s.ptr[k];
        e = v & kEntMask;
        f = v >> kEntBits;
    } else {
        e = s.base + k;
        f = flags[e];
    }
}

// Merge-path frontier tables of a tile: for each sub-merge of the tree (A = runs [ja, jb),
// B = runs [jb, jc)) and each splitter frontier k = 0 .. nsp (the last the tile's end), the
// number of A elements | B elements << 16 before the frontier.  Every sub-merge's path passes
// through these points.
enum SubMerge : int { SM_01 = 0, SM_23 = 1, SM_0123 = 2, SM_ALL = 3, kSubMerges = 4 };
constexpr int kFrontiers = kMergeGroup + 1;

__device__ __forceinline__ void frontier_table(const uint16_t (*sc)[kRuns], int nsp, uint32_t (*ft)[kFrontiers],
                                               int idx) {
    if (idx >= kSubMerges * kFrontiers) return;
    const int c = idx / kFrontiers, k = idx % kFrontiers;
    const int ja = c == SM_23 ? 2 : 0;
    const int jb = c == SM_01 ? 1 : (c == SM_23 ? 3 : (c == SM_0123 ? 2 : 4));
    const int jc = c == SM_01 ? 2 : (c == SM_ALL ? 5 : 4);
    const int kk = k <= nsp ? k : nsp;  // unused points repeat the end
    int a = 0, b = 0;
    for (int j = ja; j < jb; ++j) a += sc[kk][j];
    for (int j = jb; j < jc; ++j) b += sc[kk][j];
    ft[c][k] = uint32_t(a) | (uint32_t(b) << 16);
}

// Bounds [lo, hi] on the number of A elements before merged position d0 of a sub-merge (A and B
// of lengths An, Bn): the frontier interval that holds d0 (a binary search over the frontier
// points, whose positions a + b do not decrease).
__device__ __forceinline__ void frontier_bounds(const uint32_t* ft, int d0, int An, int Bn, int& lo, int& hi) {
    int k0 = -1, k1 = kFrontiers;  // last point at or before d0, first point after it
    while (k1 - k0 > 1) {
        const int mid = (k0 + k1) >> 1;
        const uint32_t v = ft[mid];
        if (int(v & 0xffffu) + int(v >> 16) <= d0) k0 = mid; else k1 = mid;
    }
    int a0 = 0, b0 = 0, a1 = An, b1 = Bn;
    if (k0 >= 0) {
        a0 = int(ft[k0] & 0xffffu);
        b0 = int(ft[k0] >> 16);
    }
    if (k1 < kFrontiers) {
        a1 = int(ft[k1] & 0xffffu);
        b1 = int(ft[k1] >> 16);
    }
    lo = max(max(0, d0 - Bn), max(a0, d0 - b1));
    hi = min(min(d0, An), min(a1, d0 - b0));
    if (lo > hi) lo = hi;  // cannot happen for consistent frontiers
}

// Output positions [d0, d1) of the merge of two sorted sequences of tile elements, A and B;
// an element of A precedes an equal element of B (A always holds the lower run indices).
// Merge-path split, then a sequential merge that keeps both heads (key, flag, element) in
// registers and per step reads only the next element of the side it took, without branches.
// Writes entries (element | flag) to out.
template <int NW, bool AARR, bool BARR>
__device__ __forceinline__ void merge_range(const SKeys<NW>& keys, const uint8_t* flags, const Seq& A, const Seq& B,
                                            int d0, int d1, uint16_t* out, int lo, int hi) {
    // [lo, hi] brackets the number of A elements before d0 (see frontier_bounds)
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        int ea, fa, eb, fb;
        seq_at<BARR>(B, flags, d0 - 1 - mid, eb, fb);
        seq_at<AARR>(A, flags, mid, ea, fa);
        if (!reg_less<NW>(keys.get(eb), fb, keys.get(ea), fa)) lo = mid + 1; else hi = mid;
    }
    int i = lo, j = d0 - lo;
    bool va = i < A.n, vb = j < B.n;
    // an exhausted side's head is element 0, never taken
    int ea = 0, fa = 0, eb = 0, fb = 0;
    if (va) seq_at<AARR>(A, flags, i, ea, fa);
    if (vb) seq_at<BARR>(B, flags, j, eb, fb);
    Key<NW> ka = keys.get(ea), kb = keys.get(eb);
    for (int d = d0; d < d1; ++d) {
        const bool take_a = va & (!vb | !reg_less<NW>(kb, fb, ka, fa));
        out[d] = take_a ? make_ent(ea, fa) : make_ent(eb, fb);
        const int k = take_a ? ++i : ++j;
        const bool valid = k < (take_a ? A.n : B.n);
        const int kk = valid ? k : 0;  // entry 0 of the side taken exists (it was not empty)
        int en, fn;
        if constexpr (AARR == BARR) {
            Seq s;
            s.ptr = take_a ? A.ptr : B.ptr;
            s.base = take_a ? A.base : B.base;
            seq_at<AARR>(s, flags, kk, en, fn);
        } else {
            int e1, f1, e2, f2;
            seq_at<AARR>(A, flags, take_a ? kk : 0, e1, f1);
            seq_at<BARR>(B, flags, take_a ? 0 : kk, e2, f2);
            en = take_a ? e1 : e2;
            fn = take_a ? f1 : f2;
        }
        const Key<NW> kn = keys.get(en);
        if (take_a) {
            ea = en;
            fa = fn;
            ka = kn;
            va = valid;
        } else {
            eb = en;
            fb = fn;
            kb = kn;
            vb = valid;
        }
    }
}

// The last merge level, fused with the dedup: output positions [d0, d1) of the merge of A (a
// merged level) and B (a run segment), as merge_range, and for each position whether it holds
// the first real element of its key -- a real element whose predecessor in merged order (held
// in registers; at d0 the later of the two heads' predecessors, at 0 the tile's merged
// predecessor) is not a real element with the same key.  cnt[d] = running count of firsts in
// [d0, d] | first << 15; with SPLIT the same for the firsts of the new part (element index >=
// o1: the group has no self-run element) into cntn.  Returns the counts (firsts | new-part
// firsts << 16).
template <int NW, bool SPLIT>
__device__ __forceinline__ int merge_range_first(const SKeys<NW>& keys, const uint8_t* flags, const Seq& A,
                                                 const Seq& B, int d0, int d1, uint16_t* out, uint16_t* cnt,
                                                 uint16_t* cntn, int o1, bool tile_has_pred,
                                                 const Key<NW>& tile_pred, int tile_pred_flag, int lo, int hi) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        int ea, fa, eb, fb;
        seq_at<false>(B, flags, d0 - 1 - mid, eb, fb);
        seq_at<true>(A, flags, mid, ea, fa);
        if (!reg_less<NW>(keys.get(eb), fb, keys.get(ea), fa)) lo = mid + 1; else hi = mid;
    }
    int i = lo, j = d0 - lo;
    // the predecessor of position d0
    bool have = false;
    Key<NW> pk = tile_pred;
    int pf = tile_pred_flag;
    if (d0 == 0) {
        have = tile_has_pred;
    } else {
        int xa = 0, fa = 0, xb = 0, fb = 0;
        if (i > 0) seq_at<true>(A, flags, i - 1, xa, fa);
        if (j > 0) seq_at<false>(B, flags, j - 1, xb, fb);
        int pe = xb;
        pf = fb;
        if (i > 0 && (j == 0 || reg_less<NW>(keys.get(xb), fb, keys.get(xa), fa))) {  // equal: B's comes later
            pe = xa;
            pf = fa;
        }
        pk = keys.get(pe);
        have = true;
    }
    bool va = i < A.n, vb = j < B.n;
    int ea = 0, fa = 0, eb = 0, fb = 0;
    if (va) seq_at<true>(A, flags, i, ea, fa);
    if (vb) seq_at<false>(B, flags, j, eb, fb);
    Key<NW> ka = keys.get(ea), kb = keys.get(eb);
    int c = 0, cn = 0;
    for (int d = d0; d < d1; ++d) {
        const bool take_a = va & (!vb | !reg_less<NW>(kb, fb, ka, fa));
        const int e = take_a ? ea : eb;
        const int f = take_a ? fa : fb;
        Key<NW> k;
#pragma unroll
        for (int q = 0; q < NW; ++q) k.w[q] = take_a ? ka.w[q] : kb.w[q];
        out[d] = make_ent(e, f);
        const int first = (f == 1) & !(have & (pf == 1) & reg_eq<NW>(k, pk));
        c += first;
        cnt[d] = uint16_t(c | (first << 15));
        if constexpr (SPLIT) {
            const int fnew = first & (e >= o1);
            cn += fnew;
            cntn[d] = uint16_t(cn | (fnew << 15));
        }
        pk = k;
        pf = f;
        have = true;
        // the next head of the side taken
        const int kq = take_a ? ++i : ++j;
        const bool valid = kq < (take_a ? A.n : B.n);
        const int kk = valid ? kq : 0;
        int e1, f1, e2, f2;
        seq_at<true>(A, flags, take_a ? kk : 0, e1, f1);
        seq_at<false>(B, flags, take_a ? 0 : kk, e2, f2);
        const int en = take_a ? e1 : e2;
        const int fn = take_a ? f1 : f2;
        const Key<NW> kn = keys.get(en);
        if (take_a) {
            ea = en;
            fa = fn;
            ka = kn;
            va = valid;
        } else {
            eb = en;
            fb = fn;
            kb = kn;
            vb = valid;
        }
    }
    return c | (cn << 16);
}

// Splitters every `stride` elements of each run, with their co-ranks in the block's other
// runs.  The plan comes first and every block derives it from the block offsets: the runs'
// extents, the splitter prefix over (block, run) and the tile prefix over blocks (a tile is
// kMergeGroup splitter intervals of one block).  Block 0 publishes it, sets the counters and
// every block clears its share of the look-back words for the tile kernel.
template <int NW>
__global__ void __launch_bounds__(256) merge_split_kernel(ModelDev m, const uint64_t* __restrict__ X,
                                                          const uint64_t* __restrict__ Y,
                                                          const int* __restrict__ x_blk,
                                                          const int* __restrict__ y_blk, MergeWs ws, int stride,
                                                          int* status) {
    __shared__ int s_lo[kMaxSites * kRuns];
    __shared__ int s_len[kMaxSites * kRuns];
    __shared__ int s_off[kMaxSites * kRuns + 1];
    __shared__ int s_pos[kMaxSites + 1];  // splitters per block, then their prefix
    __shared__ int s_toff[kMaxSites + 1];
    __shared__ int s_total, s_tiles;
    const int L = m.L;
    const int nr = L * kRuns;
    for (int idx = threadIdx.x; idx < nr; idx += blockDim.x) {
        const int p = idx / kRuns, j = idx % kRuns;
        const int src = run_source(m, ws, p, j);
        const int* sb = j == RUN_SELF ? x_blk : y_blk;
        int lo = 0, len = 0;
        if (src >= 0) {
            lo = sb[src];
            len = sb[src + 1] - lo;
        }
        s_lo[idx] = lo;
        s_len[idx] = len;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < L; p += blockDim.x) {
        int c = 0;
#pragma unroll
        for (int j = 0; j < kRuns; ++j) c += (s_len[p * kRuns + j] + stride - 1) / stride;
        s_pos[p] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0, tacc = 0;
        for (int p = 0; p < L; ++p) {
            const int c = s_pos[p];
            s_pos[p] = acc;
            s_toff[p] = tacc;
            acc += c;
            tacc += (c + kMergeGroup - 1) / kMergeGroup;
        }
        s_pos[L] = acc;
        s_toff[L] = tacc;
        const bool ok = acc <= ws.split_cap && tacc <= ws.tile_cap;
        s_total = ok ? acc : 0;
        s_tiles = ok ? tacc : 0;
        if (blockIdx.x == 0) {
            if (!ok) raise_status(status, PACES_ERR_CAPACITY);
            ws.counters[0] = s_total;
            ws.counters[1] = s_tiles;
            ws.counters[2] = 0;
            ws.counters[3] = 0;
            ws.counters[4] = 0;
            ws.counters[5] = 0;
        }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < L; p += blockDim.x) {
        int acc = s_pos[p];
#pragma unroll
        for (int j = 0; j < kRuns; ++j) {
            s_off[p * kRuns + j] = acc;
            acc += (s_len[p * kRuns + j] + stride - 1) / stride;
        }
    }
    if (threadIdx.x == 0) s_off[nr] = s_pos[L];
    __syncthreads();
    if (blockIdx.x == 0) {
        for (int idx = threadIdx.x; idx < nr; idx += blockDim.x) {
            ws.run_lo[idx] = s_lo[idx];
            ws.run_len[idx] = s_len[idx];
            ws.split_off[idx] = s_off[idx];
        }
        for (int p = threadIdx.x; p <= L; p += blockDim.x) ws.tile_off[p] = s_toff[p];
        if (threadIdx.x == 0) ws.split_off[nr] = s_off[nr];
    }
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < s_tiles; t += gridDim.x * blockDim.x)
        ws.tile_state[t] = 0ull;

    const int total = s_total;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < total; s += gridDim.x * blockDim.x) {
        const int r = find_segment(s_off, nr, s);
        const int p = r / kRuns, j = r % kRuns;
        const int i = (s - s_off[r]) * stride;
        Key<NW> k;
        int f;
        run_elem<NW>(m, X, Y, ws, p, j, s_lo[r] + i, k, f);
        // the bounds in the other runs: all searches advance one step per round, so their
        // dependent loads are in flight together
        int lo_[kRuns], a_[kRuns], b_[kRuns];
#pragma unroll
        for (int jj = 0; jj < kRuns; ++jj) {
            lo_[jj] = s_lo[p * kRuns + jj];
            a_[jj] = 0;
            b_[jj] = jj == j ? 0 : s_len[p * kRuns + jj];
        }
        for (;;) {
            bool any = false;
#pragma unroll
            for (int jj = 0; jj < kRuns; ++jj) {
                if (a_[jj] >= b_[jj]) continue;
                any = true;
                const int mid = (a_[jj] + b_[jj]) >> 1;
                Key<NW> k2;
                int f2;
                run_elem<NW>(m, X, Y, ws, p, jj, lo_[jj] + mid, k2, f2);
                const int c = cmp_kf(k2, f2, k, f);
                if ((jj < j) ? (c <= 0) : (c < 0)) a_[jj] = mid + 1; else b_[jj] = mid;
            }
            if (!any) break;
        }
        int rank = 0;
#pragma unroll
        for (int jj = 0; jj < kRuns; ++jj) {
            const int co = jj == j ? i : a_[jj];
            ws.split_co[int64_t(s) * kRuns + jj] = co;
            rank += co;
        }
        ws.split_rank[s] = rank;
    }
}

__global__ void __launch_bounds__(256) merge_order_kernel(ModelDev m, MergeWs ws) {
    const int total = ws.counters[0];
    const int nr = m.L * kRuns;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < total; s += gridDim.x * blockDim.x) {
        const int r = find_segment(ws.split_off, nr, s);
        const int p = r / kRuns, j = r % kRuns;
        const int own = s - ws.split_off[r];
        const int rank = ws.split_rank[s];
        int o = own;
        int a_[kRuns], b_[kRuns], base_[kRuns];
#pragma unroll
        for (int jj = 0; jj < kRuns; ++jj) {
            a_[jj] = base_[jj] = ws.split_off[p * kRuns + jj];
            b_[jj] = jj == j ? a_[jj] : ws.split_off[p * kRuns + jj + 1];
        }
        for (;;) {  // lockstep searches, as in the split kernel
            bool any = false;
#pragma unroll
            for (int jj = 0; jj < kRuns; ++jj) {
                if (a_[jj] >= b_[jj]) continue;
                any = true;
                const int mid = (a_[jj] + b_[jj]) >> 1;
                if (ws.split_rank[mid] < rank) a_[jj] = mid + 1; else b_[jj] = mid;
            }
            if (!any) break;
        }
#pragma unroll
        for (int jj = 0; jj < kRuns; ++jj) o += a_[jj] - base_[jj];
        const int64_t dst = int64_t(ws.split_off[p * kRuns]) + o;
        if (dst >= ws.split_off[(p + 1) * kRuns]) continue;  // inconsistent ranks: cannot happen for sorted runs
#pragma unroll
        for (int jj = 0; jj < kRuns; ++jj) ws.ord_co[dst * kRuns + jj] = ws.split_co[int64_t(s) * kRuns + jj];
    }
}

// Exclusive prefix of `count` over tiles taken in ticket order: decoupled look-back by one
// warp, kLbPerLane consecutive predecessors per lane and probe (relaxed loads).  The look-back
// of a tile almost always ends within its first probe, so a probe's latency is what the block
// waits for: a probe of 256 predecessors (eight per lane) made the merge tiles 25 % slower
// than one of 32.  Called by all lanes of one warp; returns the prefix.  A count packs two
// 31-bit counters (output states | new-part states << 31), which add without carrying into
// each other.
constexpr int kPackShift = 31;
constexpr long long kPackLow = (1ll << kPackShift) - 1;
constexpr int kLbPerLane = 1;

__device__ __forceinline__ unsigned long long load_relaxed(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ long long lookback_warp(unsigned long long* state, int t, long long count, int* status) {
    const int lane = threadIdx.x & 31;
    if (t == 0) {
        if (lane == 0) atomicExch(&state[0], kLbInc | (unsigned long long)count);
        return 0;
    }
    if (lane == 0) atomicExch(&state[t], kLbAgg | (unsigned long long)count);
    long long excl = 0;
    int top = t - 1;  // window: lane l reads top - 8l - k, k = 0..7 (lane 0, k = 0 the most recent)
    const uint64_t t0 = global_ns();
    while (top >= 0) {
        unsigned long long v[kLbPerLane];
#pragma unroll
        for (int k = 0; k < kLbPerLane; ++k) {
            const int idx = top - lane * kLbPerLane - k;
            v[k] = idx >= 0 ? load_relaxed(state + idx) : kLbInc;  // before tile 0: an inclusive 0
        }
        // this lane's predecessors in recency order, up to its first inclusive prefix: their
        // sum, and whether one of them has published nothing yet
        bool found = false, notready = false;
        long long sum = 0;
#pragma unroll
        for (int k = 0; k < kLbPerLane; ++k) {
            if (found) continue;
            const unsigned long long fl = v[k] >> 62;
            notready |= fl == 0;
            sum += (long long)(v[k] & kLbMask);
            found = fl == 2;
        }
        const unsigned inc = __ballot_sync(0xffffffffu, found);
        const unsigned nr = __ballot_sync(0xffffffffu, notready);
        const int first_inc = inc ? __ffs(inc) - 1 : 32;  // the lane holding the newest inclusive
        const unsigned need = first_inc >= 31 ? 0xffffffffu : ((2u << first_inc) - 1u);
        if (nr & need) {
            if (global_ns() - t0 > kWaitLimitNs) {
                if (lane == 0) raise_status(status, PACES_ERR_TIMEOUT);
                break;
            }
            __nanosleep(32);
            continue;
        }
        long long val = lane <= first_inc ? sum : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
        excl += val;
        if (first_inc < 32) break;
        top -= 32 * kLbPerLane;
    }
    if (lane == 0) {
        __threadfence();
        atomicExch(&state[t], kLbInc | (unsigned long long)(excl + count));
    }
    return excl;
}

// Everything a tile needs before it loads its elements: its block, segments and merged
// predecessor (the largest element before the start of any run).  Computed for all tiles at
// once by merge_desc_kernel, read by the tile kernel with one coalesced load.
template <int NW>
struct TileDesc {
    int p, tl, n, has_pred, pred_flag, nsp;
    int start[kRuns], off[kRuns + 1], lo[kRuns];
    int pad2;
    uint64_t pred[NW];
    // the merge frontier at the tile's splitters k = 0 .. nsp-1 and at its end (k = nsp): how
    // many elements of each run's segment precede it (every sub-merge of the tile passes
    // through these points)
    uint16_t sc[kMergeGroup + 1][kRuns];
};
static_assert(sizeof(TileDesc<kMaxKeyWords>) <= merge_desc_bytes(), "tile descriptor size");

template <int NW>
__global__ void __launch_bounds__(256) merge_desc_kernel(ModelDev m, const uint64_t* __restrict__ X,
                                                         const uint64_t* __restrict__ Y, MergeWs ws, int tmax,
                                                         int* status) {
    const int ntiles = ws.counters[1];
    const int L = m.L;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
        TileDesc<NW> d;
        const int p = find_segment(ws.tile_off, L, t);
        const int tl = t - __ldg(ws.tile_off + p);
        const int ob = __ldg(ws.split_off + p * kRuns);
        const int nsb = __ldg(ws.split_off + (p + 1) * kRuns) - ob;
        const int a = ob + tl * kMergeGroup;
        const int bidx = tl * kMergeGroup + kMergeGroup;
        d.p = p;
        d.tl = tl;
        d.pad2 = 0;
        const int nsp = min(kMergeGroup, nsb - tl * kMergeGroup);
        d.nsp = nsp;
        int n = 0, has = 0, pf = 0;
        Key<NW> pk;
#pragma unroll
        for (int q = 0; q < NW; ++q) pk.w[q] = 0;
        for (int j = 0; j < kRuns; ++j) {
            const int st = __ldcg(ws.ord_co + int64_t(a) * kRuns + j);
            const int en = bidx < nsb ? __ldcg(ws.ord_co + int64_t(ob + bidx) * kRuns + j)
                                      : __ldg(ws.run_len + p * kRuns + j);
            const int lo = __ldg(ws.run_lo + p * kRuns + j);
            d.start[j] = st;
            d.lo[j] = lo;
            d.off[j] = n;
            n += en - st;
            for (int k = 0; k <= kMergeGroup; ++k) {
                int c = en - st;  // the end (and unused points)
                if (k < nsp) c = __ldcg(ws.ord_co + int64_t(a + k) * kRuns + j) - st;
                d.sc[k][j] = uint16_t(min(max(c, 0), en - st));
            }
            if (st > 0) {
                Key<NW> k;
                int f;
                run_elem<NW>(m, X, Y, ws, p, j, int64_t(lo) + st - 1, k, f);
                // a later run wins ties: it sorts after the earlier one
                if (!has || cmp_kf(k, f, pk, pf) >= 0) {
                    pk = k;
                    pf = f;
                    has = 1;
                }
            }
        }
        d.off[kRuns] = n;
        d.n = n;
        if (n > tmax) {
            // cannot happen for sorted runs (see merge_tmax); flag it and emit nothing
            raise_status(status, PACES_ERR_CAPACITY);
            for (int j = 0; j <= kRuns; ++j) d.off[j] = 0;
            d.n = 0;
            has = 0;
        }
        d.has_pred = has;
        d.pred_flag = pf;
#pragma unroll
        for (int q = 0; q < NW; ++q) d.pred[q] = pk.w[q];
        *reinterpret_cast<TileDesc<NW>*>(ws.tile_desc + size_t(t) * merge_desc_bytes()) = d;
    }
}

// Output block offsets for blocks without tiles, the output count, capacity check (split:
// the same for the new part).
// Run by one thread of the tile block that finishes last.
__device__ void merge_finalize(const ModelDev& m, const MergeWs& ws, const MergeOut& out, int* ceiling_out,
                               int ceiling_add, int split, int* status) {
    const int L = m.L;
    const int ntiles = __ldcg(ws.counters + 1);
    long long packed = 0;
    if (ntiles > 0) packed = (long long)(__ldcg(ws.tile_state + ntiles - 1) & kLbMask);
    long long total = packed & kPackLow, total_n = packed >> kPackShift;
    if (total > out.cap) {
        raise_status(status, PACES_ERR_CAPACITY);
        total = out.cap;
    }
    out.blk[L] = int(total);
    for (int p = L - 1; p >= 0; --p) {
        if (ntiles == 0 || __ldcg(ws.tile_off + p) == __ldcg(ws.tile_off + p + 1)) out.blk[p] = out.blk[p + 1];
        if (out.blk[p] > total) out.blk[p] = int(total);
    }
    if (split) {
        if (total_n > out.new_cap) {
            raise_status(status, PACES_ERR_CAPACITY);
            total_n = out.new_cap;
        }
        out.new_blk[L] = int(total_n);
        for (int p = L - 1; p >= 0; --p) {
            if (ntiles == 0 || __ldcg(ws.tile_off + p) == __ldcg(ws.tile_off + p + 1)) out.new_blk[p] = out.new_blk[p + 1];
            if (out.new_blk[p] > total_n) out.new_blk[p] = int(total_n);
        }
    }
    ws.counters[4] = int(total);
    if (ceiling_out) *ceiling_out = (ceiling_add ? *ceiling_out : 0) + __ldcg(ws.counters + 3);
}

template <int NW, int MODE>
__global__ void __launch_bounds__(kTileThreads)
merge_tile_kernel(ModelDev m, const uint64_t* __restrict__ X, const uint64_t* __restrict__ Y, MergeWs ws,
                  int tmax, MergeOut out, int* ceiling_out, int ceiling_add, int* status) {
    constexpr bool ASM = MODE == MERGE_ASSEMBLE;
    constexpr bool SPLIT = MODE == MERGE_EXPAND_SPLIT;
    constexpr bool MAPS = ASM || SPLIT;
    extern __shared__ __align__(16) unsigned char smem[];
    const SKeys<NW> s_key{reinterpret_cast<uint64_t*>(smem)};
    uint8_t* s_flag = smem + size_t(tmax) * NW * 8;
    uint16_t* s_perm = reinterpret_cast<uint16_t*>(s_flag + ((tmax + 15) & ~15));  // merged pos -> entry
    uint16_t* s_lv1 = s_perm + tmax;   // first merge level; then the per-thread counts of firsts
    uint16_t* s_lv2 = s_lv1 + tmax;    // second merge level
    uint16_t* s_cnt = s_lv1;           // after level 2: running count of firsts | first << 15
    uint16_t* s_cntn = s_lv2 + tmax;   // split only: the same for the new part
    __shared__ int s_t;
    __shared__ long long s_base;
    __shared__ int s_thr[kTileThreads], s_thrn[kTileThreads];  // exclusive count before each thread
    __shared__ int s_warp[kTileThreads / 32], s_warpn[kTileThreads / 32];
    __shared__ int s_ceil;
    __shared__ __align__(16) TileDesc<NW> s_d;
    __shared__ uint32_t s_ft[kSubMerges][kFrontiers];
    __shared__ __align__(8) uint64_t s_mbar;  // completion of the tile's bulk copies
    __shared__ int s_abort;
    const int* s_start = s_d.start;
    const int* s_off = s_d.off;
    const int* s_lo = s_d.lo;

    const int tid = threadIdx.x;
    const int lane = tid & 31, wid = tid >> 5;
    const int ntiles = ws.counters[1];
    constexpr int kDescWords = int(sizeof(TileDesc<NW>) / 4);

    // tiles are taken by ticket when a block starts them (the order the decoupled look-back
    // waits in): the next ticket is drawn at the end of each tile, before its last barrier
    if (tid == 0) {
        s_t = atomicAdd(&ws.counters[2], 1);
        s_ceil = 0;
        s_abort = 0;
        if constexpr (NW % 2 == 0) tc::mbar_init(tc::smem_addr(&s_mbar), 1);
    }
    __syncthreads();
    uint32_t parity = 0;  // phase of s_mbar
    for (;;) {
        const int t = s_t;
        if (t >= ntiles) break;
        // tile set-up: the precomputed descriptor
        if (tid < kDescWords)
            reinterpret_cast<int*>(&s_d)[tid] =
                __ldcg(reinterpret_cast<const int*>(ws.tile_desc + size_t(t) * merge_desc_bytes()) + tid);
        __syncthreads();
        const int n = min(s_d.n, tmax);
        const int p = s_d.p;
        const int s_tl = s_d.tl;
        Key<NW> s_pred;
#pragma unroll
        for (int q = 0; q < NW; ++q) s_pred.w[q] = s_d.pred[q];

        // 1. the tile's segments into shared memory, transforms applied
        if constexpr (NW % 2 == 0) {
            // keys of 16-byte multiples: one bulk copy per run segment (completion on the
            // mbarrier, bounded wait), then the transforms in place
            const uint32_t mb = tc::smem_addr(&s_mbar);
            if (tid == 0 && n > 0) {
                // the block's reads of the previous tile's keys precede the copies' writes
                tc::fence_proxy_async();
                tc::mbar_expect_tx(mb, uint32_t(n) * uint32_t(NW * 8));
                for (int j = 0; j < kRuns; ++j) {
                    const int len = s_off[j + 1] - s_off[j];
                    if (len <= 0) continue;
                    const uint64_t* src = (j == RUN_SELF ? X : Y) + (int64_t(s_lo[j]) + s_start[j]) * NW;
                    tc::bulk_g2s(tc::smem_addr(s_key.w + size_t(s_off[j]) * NW), src, uint32_t(len) * (NW * 8), mb);
                }
            }
            if (n > 0) {
                if (!tc::mbar_wait(mb, parity) && lane == 0) s_abort = 1;
                parity ^= 1u;
            }
            for (int e = tid; e < n; e += kTileThreads) {
                int j = 0;
#pragma unroll
                for (int q = 1; q < kRuns; ++q) j += (e >= s_off[q]);
                int kind = ws.run_kind[0];
#pragma unroll
                for (int q = 1; q < kRuns; ++q) kind = j == q ? ws.run_kind[q] : kind;
                int f = 1;
                if (kind == RK_UP || kind == RK_DOWN || (ws.keep && j != RUN_SELF)) {
                    Key<NW> k = s_key.get(e);
                    run_transform<NW>(m, ws, p, j, int64_t(s_lo[j]) + s_start[j] + (e - s_off[j]), k, f);
                    s_key.set(e, k);
                }
                s_flag[e] = uint8_t(f);
            }
        } else {
            for (int e = tid; e < n; e += kTileThreads) {
                int j = 0;
#pragma unroll
                for (int q = 1; q < kRuns; ++q) j += (e >= s_off[q]);
                Key<NW> k;
                int f;
                run_elem<NW>(m, X, Y, ws, p, j, int64_t(s_lo[j]) + s_start[j] + (e - s_off[j]), k, f);
                s_key.set(e, k);
                s_flag[e] = uint8_t(f);
            }
        }
        frontier_table(s_d.sc, s_d.nsp, s_ft, tid);
        __syncthreads();

        // 2. merged order: pairwise merge tree (runs 0+1, 2+3) -> (0123) -> (01234) in shared
        //    memory; every thread merges a contiguous output range after a merge-path split.  The
        //    last level also flags and counts the first occurrences (the dedup).
        const int o1 = s_off[1], o2 = s_off[2], o3 = s_off[3], o4 = s_off[4];
        const int per = max((n + kTileThreads - 1) / kTileThreads, 1);
        int cnt = 0, cntn = 0;
        {
            const int n01 = o2, n0123 = o4;
            auto ident = [](int base, int len) { return Seq{nullptr, base, len}; };
            auto arr = [](const uint16_t* x, int len) { return Seq{x, 0, len}; };
            const int per4 = (n0123 + kTileThreads - 1) / kTileThreads;
            int lo, hi;
            int d0 = min(tid * per4, n0123), d1 = min(d0 + per4, n0123);
            if (d0 < n01) {
                frontier_bounds(s_ft[SM_01], d0, o1, o2 - o1, lo, hi);
                merge_range<NW, false, false>(s_key, s_flag, ident(0, o1), ident(o1, o2 - o1), d0, min(d1, n01), s_lv1, lo, hi);
            }
            if (d1 > n01) {
                const int e0 = max(d0, n01) - n01;
                frontier_bounds(s_ft[SM_23], e0, o3 - o2, o4 - o3, lo, hi);
                merge_range<NW, false, false>(s_key, s_flag, ident(o2, o3 - o2), ident(o3, o4 - o3), e0, d1 - n01, s_lv1 + n01, lo,
                                hi);
            }
            __syncthreads();
            if (d0 < d1) {
                frontier_bounds(s_ft[SM_0123], d0, n01, n0123 - n01, lo, hi);
                merge_range<NW, true, true>(s_key, s_flag, arr(s_lv1, n01), arr(s_lv1 + n01, n0123 - n01), d0, d1, s_lv2, lo, hi);
            }
            __syncthreads();
            d0 = min(tid * per, n);
            d1 = min(d0 + per, n);
            if (d0 < d1) {
                frontier_bounds(s_ft[SM_ALL], d0, n0123, n - o4, lo, hi);
                const int c = merge_range_first<NW, SPLIT>(s_key, s_flag, arr(s_lv2, n0123), ident(o4, n - o4), d0,
                                                           d1, s_perm, s_cnt, s_cntn, o1, s_d.has_pred != 0, s_pred,
                                                           s_d.pred_flag, lo, hi);
                cnt = c & 0xffff;
                cntn = c >> 16;
            }
        }

        // 3. block exclusive scan of the per-thread counts (and of the new part's)
        int incl = cnt, incln = cntn;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            const int vn = __shfl_up_sync(0xffffffffu, incln, o);
            if (lane >= o) {
                incl += v;
                incln += vn;
            }
        }
        if (lane == 31) {
            s_warp[wid] = incl;
            s_warpn[wid] = incln;
        }
        s_thr[tid] = incl - cnt;  // exclusive inside the warp; the warp's offset is added below
        s_thrn[tid] = incln - cntn;
        __syncthreads();
        if (wid == 0) {
            int v = lane < kTileThreads / 32 ? s_warp[lane] : 0;
            int vn = lane < kTileThreads / 32 ? s_warpn[lane] : 0;
            int tot = v, totn = vn;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int a = __shfl_up_sync(0xffffffffu, tot, o);
                const int an = __shfl_up_sync(0xffffffffu, totn, o);
                if (lane >= o) {
                    tot += a;
                    totn += an;
                }
            }
            if (lane < kTileThreads / 32) {
                s_warp[lane] = tot - v;    // exclusive over warps
                s_warpn[lane] = totn - vn;
            }
            const int all = __shfl_sync(0xffffffffu, tot, 31);
            const int alln = __shfl_sync(0xffffffffu, totn, 31);
            const long long b = lookback_warp(ws.tile_state, t, (long long)all | ((long long)alln << kPackShift),
                                              status);
            if (lane == 0) {
                s_base = b;
                if (s_tl == 0) {
                    out.blk[p] = int(b & kPackLow);
                    if constexpr (SPLIT) out.new_blk[p] = int(b >> kPackShift);
                }
            }
        }
        __syncthreads();
        const int base = int(s_base & kPackLow);
        const int basen = int(s_base >> kPackShift);

        // 4. one pass over the merged positions, consecutive threads -> consecutive outputs: the
        //    new keys (and H rows, or the new part) at first occurrences, and every element's
        //    index map (its group's output: the running count at its merged position)
        int ceil_local = 0;
        // q / per as a multiply and shift: exact for q < 2^kEntBits and per <= 16, which covers
        // every tile (n <= 4080 over 256 threads); the rounded-up reciprocal's error stays below
        // 1 / per, and every (q, per) pair in that range was checked
        static_assert(merge_tmax(merge_stride(1)) <= 16 * kTileThreads, "per <= 16");
        const uint32_t per_inv = (65536u + uint32_t(per) - 1u) / uint32_t(per);
        for (int q = tid; q < n; q += kTileThreads) {
            const int owner = int((uint32_t(q) * per_inv) >> 16);
            const unsigned raw = s_cnt[q];
            const int c = int(raw & 0x7fffu) + s_thr[owner] + s_warp[owner >> 5];  // firsts in the tile up to q
            const int ent = s_perm[q];
            const int e = ent & kEntMask;
            if (e >= n) {  // every position is written by level 3: cannot happen
                raise_status(status, PACES_ERR_BADARG);
                continue;
            }
            const int64_t u = int64_t(base) + c - 1;
            if (raw >> 15) {
                if (u < out.cap) {
                    const Key<NW> k = s_key.get(e);
                    store_key<NW>(out.keys, u, k);
                    if constexpr (ASM) {
                        const uint32_t nex = get_field(m, k, p);
                        const uint32_t ntot = total_phonons(m, k);
                        if (u < out.nbr_cap) {
                            out.meta[u] = uint32_t(p) | (nex << 8) | (ntot << 16);
                            // a group's first element is its self-run element when it has one
                            if (!out.self_rows_filled || e >= o1)
                                reinterpret_cast<int4*>(out.nbr)[u] = make_int4(-1, -1, -1, -1);
                            if (out.self_flag) out.self_flag[u] = uint8_t(e < o1);
                        }
                    }
                    if constexpr (SPLIT) {
                        const unsigned rawn = s_cntn[q];
                        if (rawn >> 15) {
                            const int64_t v =
                                int64_t(basen) + int(rawn & 0x7fffu) + s_thrn[owner] + s_warpn[owner >> 5] - 1;
                            if (v < out.new_cap) {
                                store_key<NW>(out.new_keys, v, k);
                                out.new_to_out[v] = int(u);
                            } else {
                                raise_status(status, PACES_ERR_CAPACITY);
                            }
                        }
                    }
                } else {
                    raise_status(status, PACES_ERR_CAPACITY);
                }
            }
            if constexpr (MAPS) {
                int j = 0;
#pragma unroll
                for (int qq = 1; qq < kRuns; ++qq) j += (e >= s_off[qq]);
                const int64_t src = int64_t(s_lo[j]) + s_start[j] + (e - s_off[j]);
                const int f = ent >> kEntBits;
                ceil_local += (f == 2);
                if (src < out.map_cap) out.maps[int64_t(j) * out.map_cap + src] = f == 1 ? int(u) : -1;
            }
        }
        if constexpr (MAPS) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) ceil_local += __shfl_xor_sync(0xffffffffu, ceil_local, o);
            if (lane == 0 && ceil_local) atomicAdd(&s_ceil, ceil_local);
            __syncthreads();
            if (tid == 0) {
                if (s_ceil) atomicAdd(&ws.counters[3], s_ceil);
                s_ceil = 0;
            }
        }
        // every thread has read this tile's ticket and descriptor: draw the next one (none
        // after a copy that did not complete in time)
        if (tid == 0) s_t = s_abort ? ntiles : atomicAdd(&ws.counters[2], 1);
        __syncthreads();
    }
    if (s_abort && tid == 0) {
        // wait (bounded) for the late copy before the block's shared memory is released
        raise_status(status, PACES_ERR_TIMEOUT);
        tc::mbar_wait(tc::smem_addr(&s_mbar), parity ^ 1u);
    }
    // the block that finishes last writes the block offsets and the totals: every block makes
    // its tiles' words and counts visible before it takes its exit ticket
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(&ws.counters[5], 1) == int(gridDim.x) - 1) {
            __threadfence();
            merge_finalize(m, ws, out, ceiling_out, ceiling_add, SPLIT ? 1 : 0, status);
        }
    }
}

// H neighbour table from the per-source index maps (assemble only).  Source i of the
// enlarged basis landed at row q; its four images (when coupled) at s_k.  Row q is exactly
// (s_left, s_right, s_down, s_up): one 16-byte store, q ascending with i.  Each image row
// gets the reverse entry (a 4-byte store); where an image row is itself a source row, both
// writers store the same value.
__global__ void __launch_bounds__(256) nbr_fill_kernel(ModelDev m, const int* __restrict__ x_blk,
                                                       MergeOut out) {
    __shared__ int s_blk[kMaxSites + 1];
    const int L = m.L;
    for (int i = threadIdx.x; i <= L; i += blockDim.x) s_blk[i] = x_blk[i];
    __syncthreads();
    const int nx = s_blk[L];
    const int64_t mc = out.map_cap, nc = out.nbr_cap;
    const int* map = out.maps;
    int* nb = out.nbr;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
        const int p = block_of(s_blk, L, i);
        const int q = __ldcs(map + i);
        if (q < 0 || q >= nc) continue;
        auto ok = [&](int s) { return s >= 0 && s < nc; };
        int sr = hop_exists(m, 0, p, 1) ? __ldcs(map + int64_t(RUN_FROM_LEFT) * mc + i) : -1;
        int sl = hop_exists(m, 0, p, 0) ? __ldcs(map + int64_t(RUN_FROM_RIGHT) * mc + i) : -1;
        int su = __ldcs(map + int64_t(RUN_UP) * mc + i);
        int sd = __ldcs(map + int64_t(RUN_DOWN) * mc + i);
        sr = ok(sr) ? sr : -1;
        sl = ok(sl) ? sl : -1;
        su = ok(su) ? su : -1;
        sd = ok(sd) ? sd : -1;
        int4 row;
        row.x = sl;  // NB_LEFT
        row.y = sr;  // NB_RIGHT
        row.z = sd;  // NB_DOWN
        row.w = su;  // NB_UP
        reinterpret_cast<int4*>(nb)[q] = row;
        // a row of an X state gets its own store above: reverse entries only into the others
        // when the assembly flagged them
        const uint8_t* sf = out.self_flag;
        if (sr >= 0 && !(sf && __ldg(sf + sr))) nb[4 * int64_t(sr) + NB_LEFT] = q;
        if (sl >= 0 && !(sf && __ldg(sf + sl))) nb[4 * int64_t(sl) + NB_RIGHT] = q;
        if (su >= 0 && !(sf && __ldg(sf + su))) nb[4 * int64_t(su) + NB_DOWN] = q;
        if (sd >= 0 && !(sf && __ldg(sf + sd))) nb[4 * int64_t(sd) + NB_UP] = q;
    }
}

template <int NW>
size_t tile_smem_bytes(int tmax, int mode) {
    // keys, order flags, then uint16 arrays: merged order, two merge levels (the first becomes
    // the running counts) and, for the split expansion, the new part's running counts
    return size_t(tmax) * sizeof(Key<NW>) + size_t((tmax + 15) & ~15) +
           size_t(tmax) * (mode == MERGE_EXPAND_SPLIT ? 8 : 6);
}

template <int NW, int MODE>
void launch_tile(int tmax, const ModelDev& m, const uint64_t* X, const uint64_t* Y, const MergeWs& ws,
                 const MergeOut& out, int* ceiling_out, int ceiling_add, int* status, int num_sms, cudaStream_t st) {
    const size_t smem = tile_smem_bytes<NW>(tmax, MODE);
    auto kfn = merge_tile_kernel<NW, MODE>;
    cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kTileThreads, smem);
    const int grid = num_sms * max(per_sm, 1);
    kfn<<<grid < ws.tile_cap ? grid : max(ws.tile_cap, 1), kTileThreads, smem, st>>>(m, X, Y, ws, tmax, out, ceiling_out,
                                                                                  ceiling_add, status);
}

template <int NW>
int launch_merge_t(int mode, int stride, const ModelDev& m, const uint64_t* X, const int* x_blk, const uint64_t* Y,
                   const int* y_blk, const MergeWs& ws, const MergeOut& out, int* ceiling_out, int ceiling_add,
                   int* status, int num_sms, cudaStream_t st) {
    if (stride < kMinMergeStride || stride > merge_stride(NW) || stride % 16) return PACES_ERR_BADARG;
    if (mode < MERGE_EXPAND || mode > MERGE_EXPAND_SPLIT) return PACES_ERR_BADARG;
    if (mode == MERGE_EXPAND_SPLIT && (!out.maps || !out.new_keys || !out.new_blk || !out.new_to_out))
        return PACES_ERR_BADARG;
    const bool split_input = Y != nullptr && Y != X;
    if (!Y) {
        Y = X;
        y_blk = x_blk;
    }
    const int tmax = merge_tmax(stride);
    MergeOut o = out;
    if (mode == MERGE_ASSEMBLE && !split_input && out.nbr) o.self_rows_filled = 1;  // nbr_fill_kernel below
    const int g = grid_for(ws.split_cap, 256, num_sms * 8);
    merge_split_kernel<NW><<<g, 256, 0, st>>>(m, X, Y, x_blk, y_blk, ws, stride, status);
    merge_order_kernel<<<g, 256, 0, st>>>(m, ws);
    merge_desc_kernel<NW><<<grid_for(ws.tile_cap, 256, num_sms * 8), 256, 0, st>>>(m, X, Y, ws, tmax, status);
    if (mode == MERGE_ASSEMBLE)
        launch_tile<NW, MERGE_ASSEMBLE>(tmax, m, X, Y, ws, o, ceiling_out, ceiling_add, status, num_sms, st);
    else if (mode == MERGE_EXPAND_SPLIT)
        launch_tile<NW, MERGE_EXPAND_SPLIT>(tmax, m, X, Y, ws, o, ceiling_out, ceiling_add, status, num_sms, st);
    else
        launch_tile<NW, MERGE_EXPAND>(tmax, m, X, Y, ws, o, ceiling_out, ceiling_add, status, num_sms, st);
    if (mode == MERGE_ASSEMBLE && !split_input && out.nbr)
        nbr_fill_kernel<<<grid_for(out.map_cap, 256, num_sms * 8), 256, 0, st>>>(m, x_blk, o);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

// Neighbour table after a split expansion: sources are the expansion's input P (images
// through the expansion's maps into its output B, then through the assembly's self map into
// S) and the new part N (images through the assembly's maps).  Every row of B gets its
// 16-byte store as in nbr_fill_kernel; reverse entries go only from N's rows, since those of
// P's rows land in rows of B, which carry them already.
__global__ void __launch_bounds__(256) nbr_fill_split_kernel(ModelDev m, const int* __restrict__ p_blk,
                                                             const int* __restrict__ n_blk,
                                                             const int* __restrict__ maps_e,
                                                             const int* __restrict__ maps_s,
                                                             const int* __restrict__ new_to_out,
                                                             const uint8_t* __restrict__ self_flag, int64_t mc,
                                                             int* __restrict__ nb, int64_t nc) {
    __shared__ int s_pb[kMaxSites + 1], s_nb[kMaxSites + 1];
    const int L = m.L;
    for (int i = threadIdx.x; i <= L; i += blockDim.x) {
        s_pb[i] = p_blk[i];
        s_nb[i] = n_blk[i];
    }
    __syncthreads();
    const int np_ = s_pb[L], nn = s_nb[L];
    const int64_t total = int64_t(np_) + nn;
    auto fill = [&](int64_t x) {
        const bool from_p = x < np_;
        const int i = int(from_p ? x : x - np_);
        const int p = from_p ? block_of(s_pb, L, i) : block_of(s_nb, L, i);
        // the S index of a map entry of run j for this source (-1: no coupling)
        auto img = [&](int j) -> int {
            if (from_p) {
                const int b = __ldcs(maps_e + int64_t(j) * mc + i);
                return (b >= 0 && b < mc) ? __ldg(maps_s + b) : -1;
            }
            return __ldcs(maps_s + int64_t(j) * mc + i);
        };
        int q;
        if (from_p) {
            q = img(RUN_SELF);
        } else {
            const int b = __ldcs(new_to_out + i);
            q = (b >= 0 && b < mc) ? __ldg(maps_s + b) : -1;
        }
        auto ok = [&](int s) { return s >= 0 && s < nc; };
        int sr = hop_exists(m, 0, p, 1) ? img(RUN_FROM_LEFT) : -1;
        int sl = hop_exists(m, 0, p, 0) ? img(RUN_FROM_RIGHT) : -1;
        int su = img(RUN_UP);
        int sd = img(RUN_DOWN);
        if (q < 0 || q >= nc) return;
        sr = ok(sr) ? sr : -1;
        sl = ok(sl) ? sl : -1;
        su = ok(su) ? su : -1;
        sd = ok(sd) ? sd : -1;
        int4 row;
        row.x = sl;  // NB_LEFT
        row.y = sr;  // NB_RIGHT
        row.z = sd;  // NB_DOWN
        row.w = su;  // NB_UP
        reinterpret_cast<int4*>(nb)[q] = row;
        // the images of P are states of the enlarged basis, sources themselves, whose own row
        // holds the reverse entry: only the images of N can lie outside it, and only those
        // outside it (no self-run element) need the entry from here
        if (from_p) return;
        if (sr >= 0 && !__ldg(self_flag + sr)) nb[4 * int64_t(sr) + NB_LEFT] = q;
        if (sl >= 0 && !__ldg(self_flag + sl)) nb[4 * int64_t(sl) + NB_RIGHT] = q;
        if (su >= 0 && !__ldg(self_flag + su)) nb[4 * int64_t(su) + NB_DOWN] = q;
        if (sd >= 0 && !__ldg(self_flag + sd)) nb[4 * int64_t(sd) + NB_UP] = q;
    };
    // two sources a grid stride apart per iteration: their map reads are in flight together
    const int64_t gs = int64_t(gridDim.x) * blockDim.x;
    int64_t x = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    for (; x + gs < total; x += 2 * gs) {
        fill(x);
        fill(x + gs);
    }
    if (x < total) fill(x);
}

// Neighbour table of a lattice with several hopping channels, after the assembly's passes
// (merge_passes): pass 0 mapped the enlarged basis X (five standard runs) into S_0; pass k >= 1
// mapped S_{k-1} (its self run) and the images of X under channels 2k-1, 2k into S_k; S is
// the last S_k.  An index of S_k becomes one of S through the self maps of the later passes.
// Channel 0 and the phonon neighbours go to the int4 rows, channel c >= 1 to xnbr[c-1].
struct PassMaps {
    const int* maps[4];
    int n;
};

__global__ void __launch_bounds__(256) nbr_fill_multi_kernel(ModelDev m, const int* __restrict__ x_blk, PassMaps pm,
                                                             int64_t mc, int* __restrict__ nb, int2* __restrict__ xnb,
                                                             int64_t nc) {
    __shared__ int s_blk[kMaxSites + 1];
    const int L = m.L;
    for (int i = threadIdx.x; i <= L; i += blockDim.x) s_blk[i] = x_blk[i];
    __syncthreads();
    const int nx = s_blk[L];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx; i += gridDim.x * blockDim.x) {
        const int p = block_of(s_blk, L, i);
        // entry (run j) of pass k for source i, carried to an index of S
        auto final_index = [&](int k, int j) -> int {
            int v = __ldcs(pm.maps[k] + int64_t(j) * mc + i);
            for (int kk = k + 1; kk < pm.n && v >= 0; ++kk) v = v < mc ? __ldg(pm.maps[kk] + v) : -1;
            return (v >= 0 && v < nc) ? v : -1;
        };
        const int q = final_index(0, RUN_SELF);
        if (q < 0) continue;
        int4 row;
        row.x = hop_exists(m, 0, p, 0) ? final_index(0, RUN_FROM_RIGHT) : -1;  // NB_LEFT
        row.y = hop_exists(m, 0, p, 1) ? final_index(0, RUN_FROM_LEFT) : -1;   // NB_RIGHT
        row.z = final_index(0, RUN_DOWN);                                      // NB_DOWN
        row.w = final_index(0, RUN_UP);                                        // NB_UP
        reinterpret_cast<int4*>(nb)[q] = row;
        if (row.y >= 0) nb[4 * int64_t(row.y) + NB_LEFT] = q;
        if (row.x >= 0) nb[4 * int64_t(row.x) + NB_RIGHT] = q;
        if (row.w >= 0) nb[4 * int64_t(row.w) + NB_DOWN] = q;
        if (row.z >= 0) nb[4 * int64_t(row.z) + NB_UP] = q;
        for (int c = 1; c < m.nhop; ++c) {
            const int k = 1 + (c - 1) / 2;
            const int jl = (c - 1) % 2 == 0 ? 1 : 3;  // the pass's from-below run of channel c; from-above next
            int2 e;
            e.y = hop_exists(m, c, p, 1) ? final_index(k, jl) : -1;      // the +dist image: upper neighbour
            e.x = hop_exists(m, c, p, 0) ? final_index(k, jl + 1) : -1;  // the -dist image: lower neighbour
            int2* t = xnb + int64_t(c - 1) * nc;
            t[q] = e;
            if (e.y >= 0) reinterpret_cast<int*>(t + e.y)[0] = q;
            if (e.x >= 0) reinterpret_cast<int*>(t + e.x)[1] = q;
        }
    }
}

}  // namespace

int launch_nbr_fill_multi(const ModelDev& m, const int* x_blk, const int* const* pass_maps, int passes, int64_t map_cap,
                          int* nbr, int* xnbr, int64_t nbr_cap, int num_sms, cudaStream_t st) {
    if (passes < 1 || passes > 4 || !xnbr) return PACES_ERR_BADARG;
    PassMaps pm{};
    for (int k = 0; k < passes; ++k) pm.maps[k] = pass_maps[k];
    pm.n = passes;
    if (cudaMemsetAsync(xnbr, 0xff, size_t(m.nhop - 1) * size_t(nbr_cap) * 8, st) != cudaSuccess) return PACES_ERR_CUDA;
    nbr_fill_multi_kernel<<<grid_for(map_cap, 256, num_sms * 8), 256, 0, st>>>(m, x_blk, pm, map_cap, nbr,
                                                                              reinterpret_cast<int2*>(xnbr),
                                                       nbr_cap);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

int launch_merge(int nw, int mode, int stride, const ModelDev& m, const uint64_t* x_keys, const int* x_blk,
                 const uint64_t* y_keys, const int* y_blk, const MergeWs& ws, const MergeOut& out,
                 int* ceiling_out, int ceiling_add, int* status, int num_sms, cudaStream_t st) {
#define PACES_MERGE_CASE(W)                                                                                    \
    case W:                                                                                                    \
        return launch_merge_t<W>(mode, stride, m, x_keys, x_blk, y_keys, y_blk, ws, out, ceiling_out, ceiling_add, \
                                 status, num_sms, st);
    switch (nw) {
        PACES_MERGE_CASE(1)
        PACES_MERGE_CASE(2)
        PACES_MERGE_CASE(3)
        PACES_MERGE_CASE(4)
        PACES_MERGE_CASE(5)
        PACES_MERGE_CASE(6)
        PACES_MERGE_CASE(7)
        PACES_MERGE_CASE(8)
        default: return PACES_ERR_BADARG;
    }
#undef PACES_MERGE_CASE
}

int launch_nbr_fill_split(const ModelDev& m, const int* p_blk, const int* n_blk, const int* maps_e,
                          const int* maps_s, const int* new_to_out, const uint8_t* self_flag, int64_t map_cap,
                          int* nbr, int64_t nbr_cap, int num_sms, cudaStream_t st) {
    if (!self_flag) return PACES_ERR_BADARG;
    nbr_fill_split_kernel<<<grid_for(map_cap, 512, num_sms * 8), 256, 0, st>>>(m, p_blk, n_blk, maps_e, maps_s,
                                                                              new_to_out, self_flag, map_cap, nbr,
                                                                              nbr_cap);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
