// Learned candidate proposal (see proposal.cuh): event features and labels, the MLP's
// tensor-core inference kernel (tcgen05, fused with the feature computation and the keep
// mask), and its training kernels (fp32 accumulation over bf16 inputs).
#include <cuda_bf16.h>

#include <cmath>

#include "kernels.cuh"
#include "proposal.cuh"
#include "tc.cuh"

namespace paces {

namespace {

__device__ __forceinline__ uint16_t bf16_bits(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_float(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }
__device__ __forceinline__ float bf16_round(float x) { return bf16_float(bf16_bits(x)); }

// Image of state (p, k) under run j (1..4); false when it does not exist.  The runs are the
// merge's: FROM_LEFT (the state appears in block p+1: the exciton hopped right), FROM_RIGHT
// (block p-1), UP / DOWN (one phonon more / less at the exciton site, ceiling and floor as
// in paces/models/holstein.py:242-277).
template <int NW>
__device__ __forceinline__ bool image_of(const ModelDev& m, const Key<NW>& k, int p, int j, Key<NW>& child,
                                         int& cpos) {
    child = k;
    if (j == RUN_FROM_LEFT) {
        cpos = p + 1;
        if (cpos == m.L) {
            if (!m.periodic) return false;
            cpos = 0;
        }
        return true;
    }
    if (j == RUN_FROM_RIGHT) {
        cpos = p - 1;
        if (cpos < 0) {
            if (!m.periodic) return false;
            cpos = m.L - 1;
        }
        return true;
    }
    cpos = p;
    const uint32_t n = get_field(m, k, p);
    if (j == RUN_UP) {
        if (n + 1 >= m.maxd[p]) return false;
        add_field(m, child, p, +1);
        return true;
    }
    if (n == 0) return false;
    add_field(m, child, p, -1);
    return true;
}

// Per-site constants of the features, staged in shared memory by each kernel: where the
// field lives (word, shift, mask) and 1 / (max_ho_dim - 1) rounded to fp32.
struct SiteTab {
    uint8_t word[kMaxSites];
    uint8_t shift[kMaxSites];
    uint16_t mask[kMaxSites];
    float inv[kMaxSites];
};

__device__ __forceinline__ void load_site_tab(const ModelDev& m, SiteTab& t) {
    for (int s = threadIdx.x; s < m.L; s += blockDim.x) {
        t.word[s] = m.word[s];
        t.shift[s] = m.shift[s];
        t.mask[s] = uint16_t((1u << m.bits[s]) - 1u);
        t.inv[s] = 1.0f / float(m.maxd[s] - 1);
    }
}

template <int NW>
__device__ __forceinline__ uint32_t tab_field(const SiteTab& t, const Key<NW>& k, int s) {
    uint64_t word = 0;
    const int w = t.word[s];
#pragma unroll
    for (int q = 0; q < NW; ++q)
        if (q == w) word = k.w[q];
    return uint32_t(word >> t.shift[s]) & t.mask[s];
}

template <int NW>
__device__ __forceinline__ void event_features(const ModelDev& m, const SiteTab& tab, const Key<NW>& c, int cpos,
                                               int j, float w, float log_cut, float f[kMlpIn]) {
#pragma unroll
    for (int d = -4; d <= 4; ++d) {
        int s = cpos + d;
        float v = 0.f;
        if (m.periodic) {
            // s is in [-4, L+3] and L >= 3: at most two wraps either way
            s += s < 0 ? m.L : 0;
            s += s < 0 ? m.L : 0;
            s -= s >= m.L ? m.L : 0;
            s -= s >= m.L ? m.L : 0;
            v = float(tab_field<NW>(tab, c, s)) * tab.inv[s];
        } else if (s >= 0 && s < m.L) {
            v = float(tab_field<NW>(tab, c, s)) * tab.inv[s];
        }
        f[d + 4] = v;
    }
    f[9] = float(total_phonons(m, c)) * (1.0f / 16.0f);
    f[10] = (logf(fmaxf(w, 1e-30f)) - log_cut) * (1.0f / 16.0f);
    f[11] = (j == RUN_FROM_LEFT || j == RUN_FROM_RIGHT) ? 1.f : 0.f;
    f[12] = j == RUN_UP ? 1.f : 0.f;
    f[13] = j == RUN_DOWN ? 1.f : 0.f;
    // the matrix element that carries amplitude from the source to the image
    float elem;
    if (j == RUN_FROM_LEFT || j == RUN_FROM_RIGHT) {
        elem = float(m.J);
    } else {
        const float nc = float(tab_field<NW>(tab, c, cpos));
        elem = float(m.g) * sqrtf(j == RUN_UP ? nc : nc + 1.f);
    }
    f[14] = logf(fmaxf(fabsf(elem), 1e-30f)) * 0.25f;
    f[15] = 0.f;
}

// Event e of basis X -> run, source index and image.  `s_blk` holds X's block offsets.
template <int NW>
__device__ __forceinline__ bool event_image(const ModelDev& m, const uint64_t* __restrict__ keys, const int* s_blk,
                                            int64_t nx, int64_t e, int& j, int64_t& i, Key<NW>& child, int& cpos) {
    j = 1 + int(e / nx);
    i = e - int64_t(j - 1) * nx;
    const int p = block_of(s_blk, m.L, i);
    const Key<NW> k = load_key<NW>(keys, i);
    return image_of<NW>(m, k, p, j, child, cpos);
}

template <int NW>
__device__ __forceinline__ bool contains(const uint64_t* __restrict__ keys, int lo, int hi, const Key<NW>& k) {
    const int end = hi;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (key_cmp(load_key<NW>(keys, mid), k) < 0) lo = mid + 1; else hi = mid;
    }
    return lo < end && key_eq(load_key<NW>(keys, lo), k);
}

// ---- tensor-core inference --------------------------------------------------------------
constexpr int kSThreads = 128;  // one thread per row of the 128-row MMA tile
constexpr uint32_t kSOffW1 = 0, kSOffW2 = 2048, kSOffA1 = 10240, kSOffA2 = 14336;
// Both layers accumulate into the same 64 tensor-memory columns (D1 is read out before the
// second MMA is issued).  The 30 KB of operands per CTA let at most 7 CTAs share an SM, so
// their 7 x 64 columns always fit the SM's 512 and no allocation waits.
constexpr size_t kScoreSmem = 30 * 1024;
constexpr uint32_t kTmemCols = 64;
constexpr int kScoreCtasPerSm = 7;

template <int NW>
__global__ void __launch_bounds__(kSThreads, 1)
proposal_score_kernel(ModelDev m, const uint64_t* __restrict__ keys, const int* __restrict__ blk,
                      const float* __restrict__ wts, const float* __restrict__ cut, const uint8_t* __restrict__ params,
                      float thr, ProposalOut out, int* status) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ int s_blk[kMaxSites + 1];
    __shared__ float s_b1[kMlpHid], s_b2[kMlpHid], s_w3[kMlpHid];
    __shared__ float s_b3;
    __shared__ __align__(8) uint64_t s_mbar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    __shared__ int s_cnt[2];
    __shared__ SiteTab s_tab;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int L = m.L;
    for (int i = tid; i <= L; i += kSThreads) s_blk[i] = blk[i];
    load_site_tab(m, s_tab);
    // weights into the canonical K-major layout (16-byte chunks of 8 bf16)
    for (int c = tid; c < kMlpHid * 2; c += kSThreads) {
        const int n = c >> 1, kc = c & 1;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(params + kMlpOffW1 + n * 32 + kc * 16));
        *reinterpret_cast<uint4*>(smem + kSOffW1 + tc::kmajor_offset(n, kc * 8, 16)) = v;
    }
    for (int c = tid; c < kMlpHid * 8; c += kSThreads) {
        const int n = c >> 3, kc = c & 7;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(params + kMlpOffW2 + n * 128 + kc * 16));
        *reinterpret_cast<uint4*>(smem + kSOffW2 + tc::kmajor_offset(n, kc * 8, 64)) = v;
    }
    for (int a = tid; a < kMlpHid; a += kSThreads) {
        s_b1[a] = reinterpret_cast<const float*>(params + kMlpOffB1)[a];
        s_b2[a] = reinterpret_cast<const float*>(params + kMlpOffB2)[a];
        s_w3[a] = reinterpret_cast<const float*>(params + kMlpOffW3)[a];
    }
    if (tid == 0) {
        s_b3 = *reinterpret_cast<const float*>(params + kMlpOffB3);
        s_abort = 0;
        s_cnt[0] = s_cnt[1] = 0;
        tc::mbar_init(tc::smem_addr(&s_mbar), 1);
    }
    if (warp == 0) {
        tc::alloc(tc::smem_addr(&s_tmem), kTmemCols);
        tc::relinquish();
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = s_tmem;
    const uint32_t row_lane = uint32_t(32 * warp) << 16;
    // without a cut (nothing was truncated) every existing image is kept
    const float cut_v = cut ? __ldg(cut) : 0.f;
    const bool keep_all = !(cut_v > 0.f);
    const float log_cut = logf(fmaxf(cut_v, 1e-30f));
    const int64_t nx = s_blk[L];
    const int64_t nev = 4 * nx;
    const int64_t ntiles = (nev + kSThreads - 1) / kSThreads;
    const uint32_t idesc = tc::idesc_bf16_f32(128, kMlpHid);
    const uint32_t mbar = tc::smem_addr(&s_mbar);
    const uint32_t a1 = tc::smem_addr(smem + kSOffA1), a2 = tc::smem_addr(smem + kSOffA2);
    const uint32_t w1 = tc::smem_addr(smem + kSOffW1), w2 = tc::smem_addr(smem + kSOffW2);
    uint32_t phase = 0;
    int valid_cnt = 0, kept_cnt = 0;

    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t e = t * kSThreads + tid;
        int j = 0, cpos = 0;
        int64_t i = 0;
        bool valid = false;
        float f[kMlpIn];
#pragma unroll
        for (int q = 0; q < kMlpIn; ++q) f[q] = 0.f;
        if (e < nev) {
            Key<NW> child;
            valid = event_image<NW>(m, keys, s_blk, nx, e, j, i, child, cpos);
            if (valid) event_features<NW>(m, s_tab, child, cpos, j, __ldg(wts + i), log_cut, f);
        }
        {
            uint32_t pk[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) pk[q] = uint32_t(bf16_bits(f[2 * q])) | (uint32_t(bf16_bits(f[2 * q + 1])) << 16);
            *reinterpret_cast<uint4*>(smem + kSOffA1 + tc::kmajor_offset(tid, 0, 16)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            *reinterpret_cast<uint4*>(smem + kSOffA1 + tc::kmajor_offset(tid, 8, 16)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
        tc::fence_proxy_async();
        __syncthreads();
        // layer 1: D1[128 x 64] = A1[128 x 16] . W1^T
        if (tid == 0) {
            tc::fence_after_sync();
            tc::mma_bf16(tmem, tc::smem_desc(a1, 128, 256), tc::smem_desc(w1, 128, 256), idesc, 0);
            tc::commit(mbar);
        }
        if (!tc::mbar_wait(mbar, phase)) s_abort = 1;
        phase ^= 1;
        tc::fence_after_sync();
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            uint32_t v[16];
            tc::ld16(tmem + row_lane + uint32_t(c * 16), v);
            tc::wait_ld();
            uint32_t pk[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float h0 = fmaxf(__uint_as_float(v[2 * q]) + s_b1[c * 16 + 2 * q], 0.f);
                const float h1 = fmaxf(__uint_as_float(v[2 * q + 1]) + s_b1[c * 16 + 2 * q + 1], 0.f);
                pk[q] = uint32_t(bf16_bits(h0)) | (uint32_t(bf16_bits(h1)) << 16);
            }
            *reinterpret_cast<uint4*>(smem + kSOffA2 + tc::kmajor_offset(tid, c * 16, 64)) =
                make_uint4(pk[0], pk[1], pk[2], pk[3]);
            *reinterpret_cast<uint4*>(smem + kSOffA2 + tc::kmajor_offset(tid, c * 16 + 8, 64)) =
                make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
        tc::fence_proxy_async();
        tc::fence_before_sync();
        __syncthreads();
        if (s_abort) break;
        // layer 2: D2[128 x 64] = A2[128 x 64] . W2^T, four K=16 steps
        if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
                tc::mma_bf16(tmem, tc::smem_desc(a2 + kk * 256, 128, 1024), tc::smem_desc(w2 + kk * 256, 128, 1024),
                             idesc, kk > 0 ? 1u : 0u);
            tc::commit(mbar);
        }
        if (!tc::mbar_wait(mbar, phase)) s_abort = 1;
        phase ^= 1;
        tc::fence_after_sync();
        float logit = s_b3;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            uint32_t v[16];
            tc::ld16(tmem + row_lane + uint32_t(c * 16), v);
            tc::wait_ld();
#pragma unroll
            for (int q = 0; q < 16; ++q)
                logit = fmaf(s_w3[c * 16 + q], fmaxf(__uint_as_float(v[q]) + s_b2[c * 16 + q], 0.f), logit);
        }
        if (e < nev) {
            const bool keep = valid && (keep_all || logit > thr);
            if (out.logits) out.logits[e] = logit;
            if (out.keep && i < out.keep_cap) out.keep[int64_t(j) * out.keep_cap + i] = keep ? 1 : 0;
            valid_cnt += valid;
            kept_cnt += keep;
        }
        tc::fence_before_sync();
        __syncthreads();
        if (s_abort) break;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        valid_cnt += __shfl_xor_sync(0xffffffffu, valid_cnt, o);
        kept_cnt += __shfl_xor_sync(0xffffffffu, kept_cnt, o);
    }
    if (lane == 0) {
        atomicAdd(&s_cnt[0], valid_cnt);
        atomicAdd(&s_cnt[1], kept_cnt);
    }
    __syncthreads();
    if (tid == 0) {
        if (out.counts) {
            atomicAdd(&out.counts[0], s_cnt[0]);
            atomicAdd(&out.counts[1], s_cnt[1]);
        }
        if (s_abort) raise_status(status, PACES_ERR_TIMEOUT);
    }
    if (s_abort) {
        // a commit that never arrived: give the tensor core a bounded last chance before
        // the columns are released
        tc::mbar_wait(mbar, phase);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::dealloc(tmem, kTmemCols);
    }
}

// ---- dataset kernels ----------------------------------------------------------------------
template <int NW>
__global__ void __launch_bounds__(256)
proposal_features_kernel(ModelDev m, const uint64_t* __restrict__ keys, const int* __restrict__ blk,
                         const float* __restrict__ wts, const float* __restrict__ cut, uint16_t* __restrict__ feats,
                         uint8_t* __restrict__ valid) {
    __shared__ int s_blk[kMaxSites + 1];
    __shared__ SiteTab s_tab;
    for (int i = threadIdx.x; i <= m.L; i += blockDim.x) s_blk[i] = blk[i];
    load_site_tab(m, s_tab);
    __syncthreads();
    const float log_cut = logf(fmaxf(cut ? __ldg(cut) : 0.f, 1e-30f));
    const int64_t nx = s_blk[m.L], nev = 4 * nx;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nev; e += int64_t(gridDim.x) * blockDim.x) {
        int j, cpos = 0;
        int64_t i;
        Key<NW> child;
        float f[kMlpIn];
#pragma unroll
        for (int q = 0; q < kMlpIn; ++q) f[q] = 0.f;
        const bool ok = event_image<NW>(m, keys, s_blk, nx, e, j, i, child, cpos);
        if (ok) event_features<NW>(m, s_tab, child, cpos, j, wts[i], log_cut, f);
        uint32_t pk[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) pk[q] = uint32_t(bf16_bits(f[2 * q])) | (uint32_t(bf16_bits(f[2 * q + 1])) << 16);
        uint4* dst = reinterpret_cast<uint4*>(feats + e * kMlpIn);
        dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        valid[e] = ok ? 1 : 0;
    }
}

// label of event e: 254 image does not exist, 255 image already in X (not a candidate),
// 1 image in Y (the next truncation's basis), 0 otherwise
template <int NW>
__global__ void __launch_bounds__(256)
proposal_labels_kernel(ModelDev m, const uint64_t* __restrict__ xk, const int* __restrict__ xb,
                       const uint64_t* __restrict__ yk, const int* __restrict__ yb, uint8_t* __restrict__ labels) {
    __shared__ int s_xb[kMaxSites + 1], s_yb[kMaxSites + 1];
    for (int i = threadIdx.x; i <= m.L; i += blockDim.x) {
        s_xb[i] = xb[i];
        s_yb[i] = yb[i];
    }
    __syncthreads();
    const int64_t nx = s_xb[m.L], nev = 4 * nx;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nev; e += int64_t(gridDim.x) * blockDim.x) {
        int j, cpos = 0;
        int64_t i;
        Key<NW> child;
        uint8_t lab = 254;
        if (event_image<NW>(m, xk, s_xb, nx, e, j, i, child, cpos)) {
            if (contains<NW>(xk, s_xb[cpos], s_xb[cpos + 1], child)) lab = 255;
            else lab = contains<NW>(yk, s_yb[cpos], s_yb[cpos + 1], child) ? 1 : 0;
        }
        labels[e] = lab;
    }
}

// ---- training (CUDA cores, fp32 accumulation over bf16 inputs) ----------------------------
__device__ __forceinline__ void load_params_f32(const uint8_t* __restrict__ params, float* sW1, float* sW2, float* sb1,
                                                float* sb2, float* sw3, float* sb3) {
    const uint16_t* w1 = reinterpret_cast<const uint16_t*>(params + kMlpOffW1);
    const uint16_t* w2 = reinterpret_cast<const uint16_t*>(params + kMlpOffW2);
    for (int q = threadIdx.x; q < kMlpHid * kMlpIn; q += blockDim.x) sW1[q] = bf16_float(w1[q]);
    for (int q = threadIdx.x; q < kMlpHid * kMlpHid; q += blockDim.x) sW2[q] = bf16_float(w2[q]);
    for (int a = threadIdx.x; a < kMlpHid; a += blockDim.x) {
        sb1[a] = reinterpret_cast<const float*>(params + kMlpOffB1)[a];
        sb2[a] = reinterpret_cast<const float*>(params + kMlpOffB2)[a];
        sw3[a] = reinterpret_cast<const float*>(params + kMlpOffW3)[a];
    }
    if (threadIdx.x == 0) *sb3 = *reinterpret_cast<const float*>(params + kMlpOffB3);
}

__device__ __forceinline__ void load_x(const uint16_t* __restrict__ x, int64_t s, float* xs) {
    const uint4* src = reinterpret_cast<const uint4*>(x + s * kMlpIn);
    const uint4 a = src[0], b = src[1];
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        xs[2 * q] = bf16_float(uint16_t(w[q] & 0xffffu));
        xs[2 * q + 1] = bf16_float(uint16_t(w[q] >> 16));
    }
}

__global__ void __launch_bounds__(128)
mlp_forward_kernel(const uint8_t* __restrict__ params, const uint16_t* __restrict__ x, int64_t n,
                   float* __restrict__ logits) {
    __shared__ float sW1[kMlpHid * kMlpIn], sW2[kMlpHid * kMlpHid], sb1[kMlpHid], sb2[kMlpHid], sw3[kMlpHid];
    __shared__ float sb3;
    load_params_f32(params, sW1, sW2, sb1, sb2, sw3, &sb3);
    __syncthreads();
    for (int64_t s = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; s < n; s += int64_t(gridDim.x) * blockDim.x) {
        float xs[kMlpIn], h1[kMlpHid];
        load_x(x, s, xs);
#pragma unroll 4
        for (int a = 0; a < kMlpHid; ++a) {
            float z = 0.f;
#pragma unroll
            for (int k = 0; k < kMlpIn; ++k) z = fmaf(sW1[a * kMlpIn + k], xs[k], z);
            h1[a] = bf16_round(fmaxf(z + sb1[a], 0.f));
        }
        float logit = sb3;
        for (int a = 0; a < kMlpHid; ++a) {
            float z = 0.f;
#pragma unroll
            for (int b = 0; b < kMlpHid; ++b) z = fmaf(sW2[a * kMlpHid + b], h1[b], z);
            logit = fmaf(sw3[a], fmaxf(z + sb2[a], 0.f), logit);
        }
        logits[s] = logit;
    }
}

constexpr int kGThreads = 128;
constexpr int kGPad = kMlpHid + 1;
// dynamic shared memory of mlp_backward_kernel, in floats
constexpr int kGSmemFloats = kMlpMasterFloats + 3       // parameters (fp32 copies)
                             + kGThreads * (kMlpIn + 1)  // x
                             + 3 * kGThreads * kGPad     // h1 (then dz1), h2, dz2
                             + kGThreads                 // dlogit
                             + kMlpMasterFloats + 3;     // block gradient sums

__global__ void __launch_bounds__(kGThreads)
mlp_backward_kernel(const uint8_t* __restrict__ params, const uint16_t* __restrict__ x, const float* __restrict__ y,
                    const float* __restrict__ sw, int64_t n, float inv_norm, float* __restrict__ grads,
                    double* __restrict__ loss) {
    extern __shared__ float g_smem[];
    float* sW1 = g_smem;
    float* sW2 = sW1 + kMlpHid * kMlpIn;
    float* sb1 = sW2 + kMlpHid * kMlpHid;
    float* sb2 = sb1 + kMlpHid;
    float* sw3 = sb2 + kMlpHid;
    float* sb3 = sw3 + kMlpHid;
    float* xs = g_smem + kMlpMasterFloats + 3;
    float* h1s = xs + kGThreads * (kMlpIn + 1);
    float* h2s = h1s + kGThreads * kGPad;
    float* dz2s = h2s + kGThreads * kGPad;
    float* dl = dz2s + kGThreads * kGPad;
    float* gacc = dl + kGThreads;
    __shared__ double s_loss;
    const int t = threadIdx.x;
    load_params_f32(params, sW1, sW2, sb1, sb2, sw3, sb3);
    for (int q = t; q < kMlpMasterFloats; q += kGThreads) gacc[q] = 0.f;
    if (t == 0) s_loss = 0.0;
    __syncthreads();
    double my_loss = 0.0;
    const int64_t nchunks = (n + kGThreads - 1) / kGThreads;
    for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
        const int64_t s = ch * kGThreads + t;
        const bool active = s < n;
        float* xr = xs + t * (kMlpIn + 1);
        float* h1 = h1s + t * kGPad;
        float* h2 = h2s + t * kGPad;
        float* dz2 = dz2s + t * kGPad;
        if (active) {
            float tmp[kMlpIn];
            load_x(x, s, tmp);
#pragma unroll
            for (int k = 0; k < kMlpIn; ++k) xr[k] = tmp[k];
        } else {
#pragma unroll
            for (int k = 0; k < kMlpIn; ++k) xr[k] = 0.f;
        }
        for (int a = 0; a < kMlpHid; ++a) {
            float z = 0.f;
#pragma unroll
            for (int k = 0; k < kMlpIn; ++k) z = fmaf(sW1[a * kMlpIn + k], xr[k], z);
            h1[a] = bf16_round(fmaxf(z + sb1[a], 0.f));
        }
        float logit = *sb3;
        for (int a = 0; a < kMlpHid; ++a) {
            float z = 0.f;
            for (int b = 0; b < kMlpHid; ++b) z = fmaf(sW2[a * kMlpHid + b], h1[b], z);
            z += sb2[a];
            const float h = fmaxf(z, 0.f);
            h2[a] = h;
            dz2[a] = z > 0.f ? 1.f : 0.f;
            logit = fmaf(sw3[a], h, logit);
        }
        float dlog = 0.f;
        if (active) {
            const float yy = y[s], ww = sw[s];
            const float p = 1.f / (1.f + expf(-logit));
            dlog = ww * (p - yy) * inv_norm;
            // binary cross-entropy with logits: softplus(l) - y l
            const float sp = fmaxf(logit, 0.f) + log1pf(expf(-fabsf(logit)));
            my_loss += double(ww) * double(inv_norm) * double(sp - yy * logit);
        }
        dl[t] = dlog;
        for (int a = 0; a < kMlpHid; ++a) dz2[a] *= dlog * sw3[a];
        __syncthreads();
        // dW2, db2, dw3, db3 from this chunk
        for (int o = t; o < kMlpHid * kMlpHid; o += kGThreads) {
            const int a = o >> 6, b = o & 63;
            float acc = 0.f;
            for (int q = 0; q < kGThreads; ++q) acc = fmaf(dz2s[q * kGPad + a], h1s[q * kGPad + b], acc);
            gacc[kMlpMW2 + o] += acc;
        }
        for (int a = t; a < kMlpHid; a += kGThreads) {
            float g2 = 0.f, g3 = 0.f;
            for (int q = 0; q < kGThreads; ++q) {
                g2 += dz2s[q * kGPad + a];
                g3 = fmaf(dl[q], h2s[q * kGPad + a], g3);
            }
            gacc[kMlpMB2 + a] += g2;
            gacc[kMlpMW3 + a] += g3;
        }
        if (t == 0) {
            float g = 0.f;
            for (int q = 0; q < kGThreads; ++q) g += dl[q];
            gacc[kMlpMB3] += g;
        }
        __syncthreads();
        // dz1 = (W2^T dz2) masked by h1 > 0, into h1's row
        {
            float d1[kMlpHid];
            for (int b = 0; b < kMlpHid; ++b) d1[b] = 0.f;
            for (int a = 0; a < kMlpHid; ++a) {
                const float g = dz2[a];
                for (int b = 0; b < kMlpHid; ++b) d1[b] = fmaf(sW2[a * kMlpHid + b], g, d1[b]);
            }
            for (int b = 0; b < kMlpHid; ++b) h1[b] = h1[b] > 0.f ? d1[b] : 0.f;
        }
        __syncthreads();
        for (int o = t; o < kMlpHid * kMlpIn; o += kGThreads) {
            const int b = o >> 4, k = o & 15;
            float acc = 0.f;
            for (int q = 0; q < kGThreads; ++q) acc = fmaf(h1s[q * kGPad + b], xs[q * (kMlpIn + 1) + k], acc);
            gacc[kMlpMW1 + o] += acc;
        }
        for (int b = t; b < kMlpHid; b += kGThreads) {
            float g = 0.f;
            for (int q = 0; q < kGThreads; ++q) g += h1s[q * kGPad + b];
            gacc[kMlpMB1 + b] += g;
        }
        __syncthreads();
    }
    for (int q = t; q < kMlpMasterFloats; q += kGThreads)
        if (gacc[q] != 0.f) atomicAdd(&grads[q], gacc[q]);
    atomicAdd(&s_loss, my_loss);
    __syncthreads();
    if (t == 0 && loss) atomicAdd(loss, s_loss);
}

__device__ __forceinline__ void pack_one(int q, float v, uint8_t* __restrict__ params) {
    if (q < kMlpMB1) {
        const size_t off = q < kMlpMW2 ? kMlpOffW1 + size_t(q) * 2 : kMlpOffW2 + size_t(q - kMlpMW2) * 2;
        *reinterpret_cast<uint16_t*>(params + off) = bf16_bits(v);
    } else {
        reinterpret_cast<float*>(params + kMlpOffB1)[q - kMlpMB1] = v;  // b1, b2, w3, b3 are contiguous
    }
}

__global__ void mlp_pack_kernel(const float* __restrict__ master, uint8_t* __restrict__ params) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < kMlpMasterFloats; q += gridDim.x * blockDim.x)
        pack_one(q, master[q], params);
}

// Adam (bias-corrected), then the packed inference copy; the gradients are cleared.
__global__ void mlp_adam_kernel(float* __restrict__ master, float* __restrict__ m1, float* __restrict__ m2,
                                float* __restrict__ grads, float lr, float beta1, float beta2, float eps, float c1,
                                float c2, uint8_t* __restrict__ params) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < kMlpMasterFloats; q += gridDim.x * blockDim.x) {
        const float g = grads[q];
        grads[q] = 0.f;
        const float a = beta1 * m1[q] + (1.f - beta1) * g;
        const float b = beta2 * m2[q] + (1.f - beta2) * g * g;
        m1[q] = a;
        m2[q] = b;
        const float v = master[q] - lr * (a * c1) / (sqrtf(b * c2) + eps);
        master[q] = v;
        pack_one(q, v, params);
    }
}

template <int NW>
int score_t(const ModelDev& m, const uint64_t* keys, const int* blk, const float* w, const float* cut,
            const void* params, float thr, const ProposalOut& out, int* status, int num_sms, cudaStream_t st) {
    auto kfn = proposal_score_kernel<NW>;
    if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kScoreSmem)) != cudaSuccess)
        return PACES_ERR_CUDA;
    kfn<<<num_sms * kScoreCtasPerSm, kSThreads, kScoreSmem, st>>>(m, keys, blk, w, cut, static_cast<const uint8_t*>(params), thr,
                                                    out, status);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace

#define PACES_NW_SWITCH(nw, ...)                     \
    switch (nw) {                                    \
        case 1: { constexpr int W = 1; __VA_ARGS__; } \
        case 2: { constexpr int W = 2; __VA_ARGS__; } \
        case 3: { constexpr int W = 3; __VA_ARGS__; } \
        case 4: { constexpr int W = 4; __VA_ARGS__; } \
        case 5: { constexpr int W = 5; __VA_ARGS__; } \
        case 6: { constexpr int W = 6; __VA_ARGS__; } \
        case 7: { constexpr int W = 7; __VA_ARGS__; } \
        case 8: { constexpr int W = 8; __VA_ARGS__; } \
        default: return PACES_ERR_BADARG;            \
    }

int launch_proposal_score(int nw, const ModelDev& m, const uint64_t* x_keys, const int* x_blk, const float* x_w,
                          const float* cut, const void* params, float threshold, const ProposalOut& out, int* status,
                          int num_sms, cudaStream_t st) {
    PACES_NW_SWITCH(nw, return score_t<W>(m, x_keys, x_blk, x_w, cut, params, threshold, out, status, num_sms, st))
}

int launch_proposal_features(int nw, const ModelDev& m, const uint64_t* x_keys, const int* x_blk, const float* x_w,
                             const float* cut, uint16_t* feats, uint8_t* valid, int num_sms, cudaStream_t st) {
    PACES_NW_SWITCH(nw, proposal_features_kernel<W><<<num_sms * 4, 256, 0, st>>>(m, x_keys, x_blk, x_w, cut, feats,
                                                                                 valid);
                    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA)
}

int launch_proposal_labels(int nw, const ModelDev& m, const uint64_t* x_keys, const int* x_blk, const uint64_t* y_keys,
                           const int* y_blk, uint8_t* labels, int num_sms, cudaStream_t st) {
    PACES_NW_SWITCH(nw, proposal_labels_kernel<W><<<num_sms * 4, 256, 0, st>>>(m, x_keys, x_blk, y_keys, y_blk, labels);
                    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA)
}
#undef PACES_NW_SWITCH

int launch_mlp_pack(const float* master, void* params, cudaStream_t st) {
    mlp_pack_kernel<<<(kMlpMasterFloats + 255) / 256, 256, 0, st>>>(master, static_cast<uint8_t*>(params));
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

int launch_mlp_forward(const void* params, const uint16_t* x, int64_t n, float* logits, int num_sms, cudaStream_t st) {
    if (n <= 0) return PACES_OK;
    mlp_forward_kernel<<<num_sms * 8, 128, 0, st>>>(static_cast<const uint8_t*>(params), x, n, logits);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

int launch_mlp_backward(const void* params, const uint16_t* x, const float* y, const float* sw, int64_t n,
                        float inv_norm, float* grads, double* loss, int num_sms, cudaStream_t st) {
    if (n <= 0) return PACES_OK;
    const size_t smem = size_t(kGSmemFloats) * sizeof(float);
    if (cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return PACES_ERR_CUDA;
    const int64_t chunks = (n + kGThreads - 1) / kGThreads;
    const int grid = int(chunks < num_sms ? chunks : num_sms);
    mlp_backward_kernel<<<grid, kGThreads, smem, st>>>(static_cast<const uint8_t*>(params), x, y, sw, n, inv_norm,
                                                       grads, loss);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

int launch_mlp_adam(float* master, float* m1, float* m2, float* grads, int t, float lr, float beta1, float beta2,
                    float eps, void* params, cudaStream_t st) {
    if (t < 1) return PACES_ERR_BADARG;
    const float c1 = float(1.0 / (1.0 - std::pow(double(beta1), t)));
    const float c2 = float(1.0 / (1.0 - std::pow(double(beta2), t)));
    mlp_adam_kernel<<<(kMlpMasterFloats + 255) / 256, 256, 0, st>>>(master, m1, m2, grads, lr, beta1, beta2, eps, c1, c2,
                                                                     static_cast<uint8_t*>(params));
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
