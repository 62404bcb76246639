// Amplitude remap into the new basis.
//
// Reference (paces/core/time_evolution.py:781-797): for every new state, binary-search
// the old basis; where the state exists, copy its old amplitude, else 0 (states that
// the previous truncation dropped but the expansion re-created get their old amplitude
// back).
//
// B200 design: both bases are sorted and blocked by exciton position, so the lookup is
// a merge-path sorted search per block.  A first kernel splits every block's merged
// (old + new) sequence into tiles along diagonals, one thread per diagonal; the tile
// kernel stages the tile's old keys in shared memory and resolves each new key by a
// shared-memory upper bound (old before new on equal keys; a match is the old element
// just before the new one).
#include <mutex>

#include "kernels.cuh"

namespace paces {

namespace {

template <int NW>
__device__ int merge_path(const uint64_t* __restrict__ A, int na, const uint64_t* __restrict__ B, int nb,
                          int diag) {
    int begin = max(0, diag - nb), end = min(diag, na);
    while (begin < end) {
        const int mid = (begin + end) >> 1;
        const Key<NW> a = load_key<NW>(A, mid);
        const Key<NW> b = load_key<NW>(B, diag - 1 - mid);
        if (!(key_cmp(b, a) < 0)) begin = mid + 1; else end = mid;
    }
    return begin;
}

// split[2t] / split[2t+1]: old elements before the tile's first / past its last diagonal.
// Every block first derives the tile offsets per exciton block (tiles of `tile` diagonals of
// the merged old + new block) from the block offsets; block 0 publishes them and the tile
// count for the tile kernel.
template <int NW>
__global__ void __launch_bounds__(256) remap_split_kernel(ModelDev m, const uint64_t* __restrict__ old_keys,
                                                          const int* __restrict__ ob,
                                                          const uint64_t* __restrict__ new_keys,
                                                          const int* __restrict__ nb, RemapWs ws, int tile,
                                                          int* status) {
    __shared__ int s_toff[kMaxSites + 1];
    __shared__ int s_ntiles;
    for (int p = threadIdx.x; p < m.L; p += blockDim.x) {
        const int tot = (ob[p + 1] - ob[p]) + (nb[p + 1] - nb[p]);
        s_toff[p] = (tot + tile - 1) / tile;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int p = 0; p < m.L; ++p) {
            const int c = s_toff[p];
            s_toff[p] = acc;
            acc += c;
        }
        s_toff[m.L] = acc;
        const bool ok = acc <= ws.tile_cap;
        s_ntiles = ok ? acc : 0;
        if (blockIdx.x == 0) {
            if (!ok) raise_status(status, PACES_ERR_CAPACITY);
            ws.counters[0] = s_ntiles;
        }
    }
    __syncthreads();
    if (blockIdx.x == 0)
        for (int p = threadIdx.x; p <= m.L; p += blockDim.x) ws.tile_off[p] = s_toff[p];
    const int ntiles = s_ntiles;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * ntiles; i += gridDim.x * blockDim.x) {
        const int t = i >> 1;
        const int p = find_segment(s_toff, m.L, t);
        const int tl = t - s_toff[p];
        const int o0 = ob[p], no = ob[p + 1] - o0;
        const int n0 = nb[p], nn = nb[p + 1] - n0;
        const int d = (i & 1) ? min((tl + 1) * tile, no + nn) : tl * tile;
        ws.split[i] = merge_path<NW>(old_keys + int64_t(o0) * NW, no, new_keys + int64_t(n0) * NW, nn, d);
    }
}

constexpr int kRThreads = 256;

template <int NW, bool C64>
__global__ void __launch_bounds__(kRThreads) remap_tile_kernel(ModelDev m, const uint64_t* __restrict__ old_keys,
                                                         const int* __restrict__ ob,
                                                         const void* __restrict__ old_psi,
                                                         const uint64_t* __restrict__ new_keys,
                                                         const int* __restrict__ nb, void* __restrict__ new_psi,
                                                         RemapWs ws) {
    using C = typename std::conditional<C64, float2, double2>::type;
    constexpr int kTile = remap_tile(NW);
    constexpr int kPer = kTile / kRThreads;  // new keys per thread at most
    __shared__ Key<NW> s_old[kTile + 1];
    const int ntiles = ws.counters[0];
    const C* op = reinterpret_cast<const C*>(old_psi);
    C* np = reinterpret_cast<C*>(new_psi);
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int p = find_segment(ws.tile_off, m.L, t);
        const int tl = t - ws.tile_off[p];
        const int o0 = ob[p], no = ob[p + 1] - o0;
        const int n0 = nb[p], nn = nb[p + 1] - n0;
        const uint64_t* O = old_keys + int64_t(o0) * NW;
        const uint64_t* N = new_keys + int64_t(n0) * NW;
        const int d0 = tl * kTile, d1 = min(d0 + kTile, no + nn);
        const int a0 = ws.split[2 * t], a1 = ws.split[2 * t + 1];
        const int h = a0 > 0 ? 1 : 0;  // halo: the old element before the tile
#pragma unroll 4
        for (int e = threadIdx.x; e < a1 - a0 + h; e += blockDim.x) s_old[e] = load_key<NW>(O, a0 - h + e);
        __syncthreads();
        const int b0 = d0 - a0, b1 = d1 - a1;
        const int nold = a1 - a0;
        // every thread resolves a run of consecutive new keys: the first by a binary search,
        // the next ones by stepping forward from the previous bound (new keys ascend, and
        // few old keys lie between two of them), falling back to a binary search of the rest
        const int per = (b1 - b0 + kRThreads - 1) / kRThreads;  // <= kPer
        const int x0 = min(b0 + int(threadIdx.x) * per, b1), x1 = min(x0 + per, b1);
        // 1. the old index of every new key of the run (-1: not in the old basis); the next
        //    key's load is issued before the current key is searched
        int found[kPer];
        int lo = 0;  // upper bound among s_old[h .. h+nold) of the previous key
        Key<NW> kn;
        if (x0 < x1) kn = load_key<NW>(N, x0);
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            found[u] = -1;
            const int x = x0 + u;
            if (x >= x1) continue;
            const Key<NW> k = kn;
            if (x + 1 < x1) kn = load_key<NW>(N, x + 1);
            int hi = nold;
            if (u == 0) {
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (key_cmp(s_old[h + mid], k) <= 0) lo = mid + 1; else hi = mid;
                }
            } else {
                int steps = 0;
                while (lo < nold && steps < 8 && key_cmp(s_old[h + lo], k) <= 0) {
                    ++lo;
                    ++steps;
                }
                if (steps == 8)
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (key_cmp(s_old[h + mid], k) <= 0) lo = mid + 1; else hi = mid;
                    }
            }
            const int aa = a0 + lo;  // old elements before k in merged order
            if (aa > 0 && key_eq(s_old[h + lo - 1], k)) found[u] = o0 + aa - 1;
        }
        // 2. the amplitudes: all gathers of the run in flight together
        C v[kPer];
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            v[u].x = 0;
            v[u].y = 0;
            if (found[u] >= 0) v[u] = op[found[u]];
        }
#pragma unroll
        for (int u = 0; u < kPer; ++u)
            if (x0 + u < x1) np[int64_t(n0) + x0 + u] = v[u];
        __syncthreads();
    }
}

template <int NW, bool C64>
int launch_remap_t(const ModelDev& m, const uint64_t* ok, const int* ob, const void* opsi,
                   const uint64_t* nk, const int* nb, void* npsi, const RemapWs& ws, int* status,
                   int num_sms, cudaStream_t st) {
    remap_split_kernel<NW><<<grid_for(int64_t(ws.tile_cap) * 2, 256, num_sms * 2), 256, 0, st>>>(m, ok, ob, nk, nb, ws,
                                                                                                remap_tile(NW), status);
    remap_tile_kernel<NW, C64><<<grid_for(ws.tile_cap, 1, num_sms * 8), kRThreads, 0, st>>>(m, ok, ob, opsi, nk, nb, npsi,
                                                                                            ws);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

// Scratch of the workspace-free remap (paces_remap_noalloc): block tile offsets, the tile
// counter and two splits per tile, 512 KiB in total.  Every GPU that loads the library
// holds one copy until the process exits.  Nothing in it has to start at zero: the split
// kernel rewrites the offsets, the counter and every split it uses.
constexpr size_t kStaticRemapBytes = size_t(512) << 10;
constexpr size_t kStaticHeaderBytes = 1024;  // tile_off[kMaxSites+1] and counters

}  // namespace

static __device__ __align__(256) unsigned char g_remap_scratch[kStaticRemapBytes];

int remap_static_tile_cap() { return int((kStaticRemapBytes - kStaticHeaderBytes) / (2 * sizeof(int))); }

// The array's device address belongs to a CUDA context: the cache below is keyed on the
// context current at the call (the device's primary context, or one the host created), read
// through the CUDA driver API's cuCtxGetCurrent.
using CtxGetCurrentFn = int (*)(void**);

void* current_context() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

int remap_static_ws(RemapWs* ws, const char** err) {
    constexpr int kSlots = 64;
    static std::mutex mu;
    static void* ctx_of[kSlots] = {};
    static void* addr_of[kSlots] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        *err = "no current CUDA device";
        return PACES_ERR_CUDA;
    }
    // host code cannot use the array's name as a device address: ask the runtime, once per
    // context, with that context current
    void* p = nullptr;
    auto lookup = [&]() {
        if (cudaGetSymbolAddress(&p, g_remap_scratch) != cudaSuccess || !p) {
            *err = "cudaGetSymbolAddress of the static remap scratch failed";
            return false;
        }
        return true;
    };
    void* ctx = current_context();
    if (!ctx) {
        // no context yet: the lookup makes the device's primary context current
        if (!lookup()) return PACES_ERR_CUDA;
        ctx = current_context();
        if (!ctx) {
            *err = "cuCtxGetCurrent is unavailable or reports no current context";
            return PACES_ERR_CUDA;
        }
    }
    std::lock_guard<std::mutex> lock(mu);
    int slot = -1;
    for (int s = 0; s < kSlots && slot < 0; ++s)
        if (ctx_of[s] == ctx) slot = s;
    if (slot < 0) {
        if (!p && !lookup()) return PACES_ERR_CUDA;
        for (int s = 0; s < kSlots && slot < 0; ++s)
            if (!ctx_of[s]) slot = s;
        if (slot < 0) {
            *err = "more than 64 CUDA contexts have called paces_remap_noalloc";
            return PACES_ERR_CUDA;
        }
        ctx_of[slot] = ctx;
        addr_of[slot] = p;
    }
    unsigned char* base = static_cast<unsigned char*>(addr_of[slot]);
    ws->tile_off = reinterpret_cast<int*>(base);
    ws->counters = reinterpret_cast<int*>(base + sizeof(int) * (kMaxSites + 8));
    ws->split = reinterpret_cast<int*>(base + kStaticHeaderBytes);
    ws->tile_cap = remap_static_tile_cap();
    return PACES_OK;
}

int launch_remap(int nw, bool c64, const ModelDev& m, const uint64_t* ok, const int* ob,
                 const void* opsi, const uint64_t* nk, const int* nb, void* npsi, const RemapWs& ws,
                 int* status, int num_sms, cudaStream_t st) {
#define PACES_REMAP_CASE(N)                                                                         \
    case N:                                                                                         \
        return c64 ? launch_remap_t<N, true>(m, ok, ob, opsi, nk, nb, npsi, ws, status, num_sms, st) \
                   : launch_remap_t<N, false>(m, ok, ob, opsi, nk, nb, npsi, ws, status, num_sms, st);
    switch (nw) {
        PACES_REMAP_CASE(1)
        PACES_REMAP_CASE(2)
        PACES_REMAP_CASE(3)
        PACES_REMAP_CASE(4)
        PACES_REMAP_CASE(5)
        PACES_REMAP_CASE(6)
        PACES_REMAP_CASE(7)
        PACES_REMAP_CASE(8)
        default: return PACES_ERR_BADARG;
    }
#undef PACES_REMAP_CASE
}

}  // namespace paces
