// Generic helpers over rows of uint32 words in the reference's whoami layout (MSB-first
// words, rows compared lexicographically, word 0 most significant), for the host API of the
// drop-in.  The time step never calls them (its lookups are the merge's index maps).
//
// Reference: searchsorted_full_binary (paces/aux/cupy_search.py:78-93, kernel :149-228), one
// thread per query and a plain binary search; cupy_unique (paces/aux/helpers.py:63-75), a
// lexsort -- one stable sort per word, last word first -- and an adjacent-row dedup.
//
// Here the lower bound caches 512 evenly spaced rows of the sorted array in shared memory
// (the upper levels of the search tree) and finishes in global memory; the sort is the same
// lexsort, each word a stable LSD radix sort of 8-bit digits (per-block digit histograms, a
// digit-major exclusive scan, and an order-preserving scatter that ranks equal digits inside
// each warp with __match_any_sync), followed by a first-occurrence flag, a scan and the
// compaction of the unique rows.
#include "kernels.cuh"

namespace paces {

namespace {

constexpr int kRowsMaxWords = 16;
constexpr int kRowSamples = 512;
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;  // rows per thread per block tile
constexpr int kSortTile = kSortThreads * kSortItems;

__device__ __forceinline__ int row_cmp(const uint32_t* a, const uint32_t* b, int w) {
    for (int k = 0; k < w; ++k)
        if (a[k] != b[k]) return a[k] < b[k] ? -1 : 1;
    return 0;
}

__global__ void __launch_bounds__(256) rows_lower_bound_kernel(const uint32_t* __restrict__ pb, int64_t n,
                                                               const uint32_t* __restrict__ q, int64_t nq, int w,
                                                               int must, int64_t* __restrict__ out,
                                                               int* __restrict__ missing) {
    __shared__ uint32_t s_rows[kRowSamples * 8];
    const bool cached = w <= 8 && n > 0;
    if (cached)
        for (int k = threadIdx.x; k < kRowSamples; k += blockDim.x) {
            const int64_t idx = (int64_t(k) * n) / kRowSamples;
            for (int c = 0; c < w; ++c) s_rows[k * 8 + c] = pb[idx * w + c];
        }
    __syncthreads();
    uint32_t key[kRowsMaxWords];
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nq; i += int64_t(gridDim.x) * blockDim.x) {
        for (int c = 0; c < w; ++c) key[c] = q[i * w + c];
        int64_t lo = 0, hi = n;
        if (cached) {
            int a = 0, b = kRowSamples;  // first sample with row >= key
            while (a < b) {
                const int mid = (a + b) >> 1;
                if (row_cmp(s_rows + mid * 8, key, w) < 0) a = mid + 1; else b = mid;
            }
            if (a > 0) lo = (int64_t(a - 1) * n) / kRowSamples + 1;
            if (a < kRowSamples) hi = (int64_t(a) * n) / kRowSamples;
            if (lo > hi) lo = hi;
        }
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (row_cmp(pb + mid * w, key, w) < 0) lo = mid + 1; else hi = mid;
        }
        out[i] = lo;
        if (must && (lo >= n || row_cmp(pb + lo * w, key, w) != 0)) atomicExch(missing, 1);
    }
}

// digit of the row at `idx`: (word w >> shift) & 255
__device__ __forceinline__ unsigned row_digit(const uint32_t* rows, int words, int64_t idx, int w, int shift) {
    return (rows[idx * words + w] >> shift) & 255u;
}

__global__ void __launch_bounds__(kSortThreads) rows_hist_kernel(const uint32_t* __restrict__ rows, int words,
                                                                 const int* __restrict__ perm, int64_t n, int w,
                                                                 int shift, unsigned* __restrict__ hist) {
    __shared__ unsigned s_h[256];
    s_h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = int64_t(blockIdx.x) * kSortTile;
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + int64_t(k) * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&s_h[row_digit(rows, words, perm[i], w, shift)], 1u);
    }
    __syncthreads();
    hist[size_t(threadIdx.x) * gridDim.x + blockIdx.x] = s_h[threadIdx.x];  // digit-major
}

// In-place exclusive scan of m values by one block.
__global__ void __launch_bounds__(1024) rows_scan_kernel(unsigned* __restrict__ v, int64_t m) {
    __shared__ unsigned s_w[32];
    __shared__ unsigned s_carry;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (int64_t c = 0; c < m; c += 1024) {
        const int64_t i = c + tid;
        const unsigned x = i < m ? v[i] : 0u;
        unsigned incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_w[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            unsigned t = s_w[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            s_w[lane] = t;  // inclusive over warps
        }
        __syncthreads();
        const unsigned before = s_carry + (wid > 0 ? s_w[wid - 1] : 0u) + incl - x;
        if (i < m) v[i] = before;
        __syncthreads();
        if (tid == 0) s_carry += s_w[31];
        __syncthreads();
    }
}

// Order-preserving scatter of perm by digit: rows are ranked in tile order (items, warps,
// lanes), equal digits inside a warp by their lane order.
__global__ void __launch_bounds__(kSortThreads) rows_scatter_kernel(const uint32_t* __restrict__ rows, int words,
                                                                    const int* __restrict__ perm_in,
                                                                    int* __restrict__ perm_out, int64_t n, int w,
                                                                    int shift, const unsigned* __restrict__ offs) {
    constexpr int kWarps = kSortThreads / 32;
    __shared__ unsigned s_base[256];
    __shared__ unsigned s_cnt[kWarps][256];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    s_base[tid] = offs[size_t(tid) * gridDim.x + blockIdx.x];
    const int64_t base = int64_t(blockIdx.x) * kSortTile;
    const unsigned lt = (1u << lane) - 1u;
    for (int k = 0; k < kSortItems; ++k) {
        for (int x = 0; x < kWarps; ++x) s_cnt[x][tid] = 0;
        __syncthreads();
        const int64_t i = base + int64_t(k) * kSortThreads + tid;
        const bool ok = i < n;
        const int p = ok ? perm_in[i] : 0;
        const unsigned d = ok ? row_digit(rows, words, p, w, shift) : 256u + lane;  // no peers when out of range
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned rank = __popc(peers & lt);
        if (ok && rank == 0) s_cnt[wid][d] = __popc(peers);
        __syncthreads();
        // per digit: offsets of the warps in order, and the running base
        {
            unsigned run = s_base[tid];
            for (int x = 0; x < kWarps; ++x) {
                const unsigned c = s_cnt[x][tid];
                s_cnt[x][tid] = run;
                run += c;
            }
            s_base[tid] = run;
        }
        __syncthreads();
        if (ok) perm_out[s_cnt[wid][d] + rank] = p;
        __syncthreads();
    }
}

__global__ void rows_iota_kernel(int* __restrict__ perm, int64_t n) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        perm[i] = int(i);
}

// First occurrences of the sorted order (row perm[i] differs from row perm[i-1]) and the
// per-block counts of them.
__global__ void __launch_bounds__(kSortThreads) rows_first_kernel(const uint32_t* __restrict__ rows, int words,
                                                                  const int* __restrict__ perm, int64_t n,
                                                                  unsigned* __restrict__ flag,
                                                                  unsigned* __restrict__ block_cnt) {
    __shared__ unsigned s_c;
    if (threadIdx.x == 0) s_c = 0;
    __syncthreads();
    const int64_t base = int64_t(blockIdx.x) * kSortTile;
    unsigned c = 0;
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + int64_t(k) * kSortThreads + threadIdx.x;
        if (i >= n) continue;
        const unsigned f =
            i == 0 || row_cmp(rows + int64_t(perm[i]) * words, rows + int64_t(perm[i - 1]) * words, words) != 0;
        flag[i] = f;
        c += f;
    }
    atomicAdd(&s_c, c);
    __syncthreads();
    if (threadIdx.x == 0) block_cnt[blockIdx.x] = s_c;
}

// Unique rows in order: block b's first occurrences go to [block_off[b], ...), ranked in tile
// order through a block scan of the flags.
__global__ void __launch_bounds__(kSortThreads) rows_compact_kernel(const uint32_t* __restrict__ rows, int words,
                                                                    const int* __restrict__ perm, int64_t n,
                                                                    const unsigned* __restrict__ flag,
                                                                    const unsigned* __restrict__ block_off,
                                                                    uint32_t* __restrict__ out, int64_t* count) {
    constexpr int kWarps = kSortThreads / 32;
    __shared__ unsigned s_w[kWarps];
    __shared__ unsigned s_run;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) s_run = block_off[blockIdx.x];
    __syncthreads();
    const int64_t base = int64_t(blockIdx.x) * kSortTile;
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + int64_t(k) * kSortThreads + tid;
        const unsigned f = i < n ? flag[i] : 0u;
        const unsigned b = __ballot_sync(0xffffffffu, f);
        if (lane == 0) s_w[wid] = __popc(b);
        __syncthreads();
        unsigned before = s_run;
        for (int x = 0; x < wid; ++x) before += s_w[x];
        before += __popc(b & ((1u << lane) - 1u));
        if (f) {
            const int64_t src = int64_t(perm[i]) * words;
            for (int c = 0; c < words; ++c) out[int64_t(before) * words + c] = rows[src + c];
        }
        __syncthreads();
        if (tid == 0) {
            unsigned t = 0;
            for (int x = 0; x < kWarps; ++x) t += s_w[x];
            s_run += t;
        }
        __syncthreads();
    }
    if (blockIdx.x == gridDim.x - 1 && tid == 0) *count = s_run;
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

// Workspace of launch_rows_sort_unique: two permutations, the flags, the digit histogram and
// the block counts.
size_t rows_sort_ws_bytes(int64_t n) {
    const int64_t blocks = (n + kSortTile - 1) / kSortTile;
    return 3 * align256(size_t(n) * 4) + align256(size_t(blocks) * 256 * 4) + align256(size_t(blocks) * 4);
}

int launch_rows_lower_bound(const uint32_t* pb, int64_t n, const uint32_t* q, int64_t nq, int words, int must,
                            int64_t* out, int* missing, int num_sms, cudaStream_t st) {
    if (words < 1 || words > kRowsMaxWords) return PACES_ERR_BADARG;
    if (nq <= 0) return PACES_OK;
    rows_lower_bound_kernel<<<grid_for(nq, 256, num_sms * 4), 256, 0, st>>>(pb, n, q, nq, words, must, out, missing);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

int launch_rows_sort_unique(const uint32_t* rows, int64_t n, int words, uint32_t* out, int64_t* count, void* ws,
                            int num_sms, cudaStream_t st) {
    if (words < 1 || words > kRowsMaxWords || n < 0 || n > (int64_t(1) << 31) - 1) return PACES_ERR_BADARG;
    if (n == 0) return cudaMemsetAsync(count, 0, sizeof(int64_t), st) == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
    const int64_t blocks = (n + kSortTile - 1) / kSortTile;
    unsigned char* p = static_cast<unsigned char*>(ws);
    const size_t vec = align256(size_t(n) * 4);
    int* perm[2] = {reinterpret_cast<int*>(p), reinterpret_cast<int*>(p + vec)};
    unsigned* flag = reinterpret_cast<unsigned*>(p + 2 * vec);
    unsigned* hist = reinterpret_cast<unsigned*>(p + 3 * vec);
    unsigned* bcnt = reinterpret_cast<unsigned*>(p + 3 * vec + align256(size_t(blocks) * 256 * 4));
    rows_iota_kernel<<<grid_for(n, 256, num_sms * 4), 256, 0, st>>>(perm[0], n);
    int cur = 0;
    // lexsort: a stable sort per word, the least significant word first
    for (int w = words - 1; w >= 0; --w)
        for (int shift = 0; shift < 32; shift += 8) {
            rows_hist_kernel<<<int(blocks), kSortThreads, 0, st>>>(rows, words, perm[cur], n, w, shift, hist);
            rows_scan_kernel<<<1, 1024, 0, st>>>(hist, blocks * 256);
            rows_scatter_kernel<<<int(blocks), kSortThreads, 0, st>>>(rows, words, perm[cur], perm[cur ^ 1], n, w,
                                                                      shift, hist);
            cur ^= 1;
        }
    rows_first_kernel<<<int(blocks), kSortThreads, 0, st>>>(rows, words, perm[cur], n, flag, bcnt);
    rows_scan_kernel<<<1, 1024, 0, st>>>(bcnt, blocks);
    rows_compact_kernel<<<int(blocks), kSortThreads, 0, st>>>(rows, words, perm[cur], n, flag, bcnt, out, count);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
