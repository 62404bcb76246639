// Lookup of arbitrary (pos, key) queries in a basis, and conversion to/from the
// reference's uint32 row layout.
//
// Reference: searchsorted_full_binary (paces/aux/cupy_search.py:78-93, kernel :149-228):
// one thread per query, plain lower-bound binary search over multi-word rows; the
// `noesc` variant asserts on a miss.  Here each block first caches a sample of the key
// array (the upper levels of the search tree) in shared memory, narrows every query to
// one sample interval there, and finishes the lower bound in global memory inside the
// query's exciton block.  A miss returns -1 and, when the state must exist, raises
// PACES_ERR_LOOKUP through the status word instead of trapping.
#include "kernels.cuh"

namespace paces {

namespace {

template <int NW>
constexpr int samples_for() { return NW > 4 ? 512 : 1024; }

template <int NW>
__global__ void __launch_bounds__(256) lookup_kernel(ModelDev m, const uint64_t* __restrict__ pk,
                                                     const int* __restrict__ pblk,
                                                     const uint64_t* __restrict__ qk,
                                                     const int* __restrict__ qpos, int64_t nq,
                                                     int must, int64_t* __restrict__ out, int* status) {
    constexpr int kSamples = samples_for<NW>();
    __shared__ Key<NW> s_key[kSamples];
    __shared__ int s_blk[kMaxSites + 1];
    const int L = m.L;
    for (int i = threadIdx.x; i <= L; i += blockDim.x) s_blk[i] = pblk[i];
    __syncthreads();
    const int64_t S = s_blk[L];
    // sample k sits at index (k * S) / kSamples
    for (int k = threadIdx.x; k < kSamples; k += blockDim.x) {
        const int64_t idx = (int64_t(k) * S) / kSamples;
        if (idx < S) s_key[k] = load_key<NW>(pk, idx);
    }
    __syncthreads();
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nq; i += int64_t(gridDim.x) * blockDim.x) {
        const int p = qpos[i];
        int64_t res = -1;
        if (p >= 0 && p < L && S > 0) {
            const Key<NW> key = load_key<NW>(qk, i);
            int64_t lo = s_blk[p], hi = s_blk[p + 1];
            // samples whose index lies in [lo, hi): k in [klo, khi)
            const int klo = int((lo * kSamples + S - 1) / S);
            const int khi = int((hi * kSamples + S - 1) / S);
            int a = klo, b = min(khi, kSamples);
            while (a < b) {  // first sample in range with key > query
                const int mid = (a + b) >> 1;
                if (key_cmp(s_key[mid], key) <= 0) a = mid + 1; else b = mid;
            }
            if (a > klo) lo = max(lo, (int64_t(a - 1) * S) / kSamples);
            if (a < min(khi, kSamples)) hi = min(hi, (int64_t(a) * S) / kSamples + 1);
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (key_cmp(load_key<NW>(pk, mid), key) < 0) lo = mid + 1; else hi = mid;
            }
            if (lo < s_blk[p + 1] && key_eq(load_key<NW>(pk, lo), key)) res = lo;
        }
        if (res < 0 && must) raise_status(status, PACES_ERR_LOOKUP);
        out[i] = res;
    }
}

template <int NW>
__global__ void keys_to_ref_kernel(ModelDev m, RefLayout rl, const uint64_t* __restrict__ keys,
                                   const int* __restrict__ blk, uint32_t* __restrict__ ref) {
    __shared__ int s_blk[kMaxSites + 1];
    const int L = m.L;
    for (int i = threadIdx.x; i <= L; i += blockDim.x) s_blk[i] = blk[i];
    __syncthreads();
    const int64_t S = s_blk[L];
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < S; i += int64_t(gridDim.x) * blockDim.x) {
        uint32_t row[kMaxRefWords];
        for (int w = 0; w < rl.words; ++w) row[w] = 0;
        const Key<NW> k = load_key<NW>(keys, i);
        const int p = block_of(s_blk, L, i);
        for (int f = 0; f < rl.nfields; ++f) {
            const uint64_t v = f == 0 ? uint64_t(p) : uint64_t(get_field(m, k, f - 1));
            const int off = rl.off[f], bits = rl.bits[f];
            if (bits == 0) continue;
            const int wi = off >> 5;
            const int n2 = off + bits - 32 * wi;  // end bit inside the 64-bit window (wi, wi+1)
            const uint64_t win = v << (64 - n2);
            row[wi] |= uint32_t(win >> 32);
            if (n2 > 32) row[wi + 1] |= uint32_t(win & 0xffffffffu);
        }
        for (int w = 0; w < rl.words; ++w) ref[i * rl.words + w] = row[w];
    }
}

template <int NW>
__global__ void keys_from_ref_kernel(ModelDev m, RefLayout rl, const uint32_t* __restrict__ ref, int64_t n,
                                     uint64_t* __restrict__ keys, int* __restrict__ pos, int* status) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        Key<NW> k;
#pragma unroll
        for (int q = 0; q < NW; ++q) k.w[q] = 0;
        int p = 0;
        for (int f = 0; f < rl.nfields; ++f) {
            const int off = rl.off[f], bits = rl.bits[f];
            if (bits == 0) continue;
            const int wi = off >> 5;
            const int n2 = off + bits - 32 * wi;
            uint64_t win = uint64_t(ref[i * rl.words + wi]) << 32;
            if (wi + 1 < rl.words) win |= ref[i * rl.words + wi + 1];
            const uint64_t v = (win >> (64 - n2)) & ((uint64_t(1) << bits) - 1);
            if (f == 0) {
                p = int(v);
            } else {
                const int s = f - 1;
                if (v >= m.maxd[s]) raise_status(status, PACES_ERR_BADARG);
#pragma unroll
                for (int q = 0; q < NW; ++q)
                    if (q == m.word[s]) k.w[q] |= v << m.shift[s];
            }
        }
        if (p >= m.L) raise_status(status, PACES_ERR_BADARG);
        store_key<NW>(keys, i, k);
        pos[i] = p;
    }
}

}  // namespace

#define PACES_NW_SWITCH(CALL)        \
    switch (nw) {                    \
        case 1: { constexpr int N = 1; CALL; } break; \
        case 2: { constexpr int N = 2; CALL; } break; \
        case 3: { constexpr int N = 3; CALL; } break; \
        case 4: { constexpr int N = 4; CALL; } break; \
        case 5: { constexpr int N = 5; CALL; } break; \
        case 6: { constexpr int N = 6; CALL; } break; \
        case 7: { constexpr int N = 7; CALL; } break; \
        case 8: { constexpr int N = 8; CALL; } break; \
        default: return PACES_ERR_BADARG;             \
    }

int launch_lookup(int nw, const ModelDev& m, const uint64_t* pk, const int* pblk,
                  const uint64_t* qk, const int* qpos, int64_t nq, int must_exist, int64_t* out,
                  int* status, int num_sms, cudaStream_t st) {
    if (nq <= 0) return PACES_OK;
    PACES_NW_SWITCH((lookup_kernel<N><<<num_sms * 4, 256, 0, st>>>(m, pk, pblk, qk, qpos, nq, must_exist, out, status)))
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

int launch_keys_to_ref(int nw, const ModelDev& m, const RefLayout& rl, const uint64_t* keys,
                       const int* blk, uint32_t* ref, int num_sms, cudaStream_t st) {
    PACES_NW_SWITCH((keys_to_ref_kernel<N><<<num_sms * 4, 256, 0, st>>>(m, rl, keys, blk, ref)))
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

int launch_keys_from_ref(int nw, const ModelDev& m, const RefLayout& rl, const uint32_t* ref,
                         int64_t n, uint64_t* keys, int* pos, int* status, int num_sms,
                         cudaStream_t st) {
    if (n <= 0) return PACES_OK;
    PACES_NW_SWITCH((keys_from_ref_kernel<N><<<num_sms * 4, 256, 0, st>>>(m, rl, ref, n, keys, pos, status)))
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
