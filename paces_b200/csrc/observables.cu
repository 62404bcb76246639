// Norm, energy and per-site observables in one pass over the state.
//
// Reference: calculate_n_exc (paces/models/holstein.py:311-314, partitioned sum of
// |psi|^2 by exciton position), calculate_n_pho (holstein.py:317-322 with the CUB
// block-reduce + atomicAdd kernel _holstein_kernels.py:215-255), calculate_total_energy
// (paces/core/observables.py:95-99, <psi|H psi>) and the norms of
// paces/core/time_evolution.py:587, :602, :818.
//
// B200 design: one grid-stride sweep reads psi, the row metadata and the keys once;
// every warp broadcasts its 32 rows lane by lane and lane l accumulates the sites
// l, l+32, l+64, l+96 in registers, so n_pho needs no atomics.  Per-block partials are
// summed in a fixed order by a second tiny kernel: the result is deterministic, unlike
// the reference's floating-point atomics.
#include "hrow.cuh"
#include "kernels.cuh"

namespace paces {

namespace {

constexpr int kOThreads = 256;
constexpr int kOWarps = kOThreads / 32;

template <int NW, bool C64>
__global__ void __launch_bounds__(kOThreads)
obs_kernel(ModelDev m, const uint64_t* __restrict__ keys, const int* __restrict__ blk,
           const int* __restrict__ nbr, int64_t cap, const uint32_t* __restrict__ meta,
           const void* __restrict__ psi, int what, double* __restrict__ partials) {
    using C = typename std::conditional<C64, float2, double2>::type;
    using R = typename std::conditional<C64, float, double>::type;
    __shared__ R s_sq[260];
    __shared__ double s_site[kOWarps][2 * kMaxSites];
    __shared__ double s_red[kOWarps][3];
    const int L = m.L;
    const int nvals = 3 + 2 * L;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < 260; k += kOThreads) s_sq[k] = R(__dmul_rn(sqrt(double(k)), m.g));
    __syncthreads();
    const int64_t S = blk[L];
    const C* x = reinterpret_cast<const C*>(psi);
    const R J = R(m.J);
    const bool energy = (what & PACES_OBS_ENERGY) != 0;
    const bool sites = (what & PACES_OBS_SITES) != 0;
    double norm2 = 0.0, er = 0.0, ei = 0.0;
    double pho[4] = {0.0, 0.0, 0.0, 0.0}, exc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t base = (int64_t(blockIdx.x) * kOWarps + wid) * 32; base < S;
         base += int64_t(gridDim.x) * kOWarps * 32) {
        const int64_t r = base + lane;
        const bool valid = r < S;
        double w = 0.0;
        uint32_t mm = 0;
        Key<NW> k;
#pragma unroll
        for (int q = 0; q < NW; ++q) k.w[q] = 0;
        if (valid) {
            const C z = x[r];
            const double zr = double(z.x), zi = double(z.y);
            w = zr * zr + zi * zi;
            mm = meta[r];
            if (energy) {
                double yr, yi;
                if constexpr (C64) {
                    const float2 y = h_row_c64(m, s_sq, J, r, nbr, cap, mm, x);
                    yr = y.x;
                    yi = y.y;
                } else {
                    const double2 y = h_row_c128(m, s_sq, r, nbr, cap, mm, x);
                    yr = y.x;
                    yi = y.y;
                }
                er += zr * yr + zi * yi;
                ei += zr * yi - zi * yr;
            }
            if (sites) k = load_key<NW>(keys, r);
        }
        norm2 += w;
        if (sites) {
            unsigned act = __ballot_sync(0xffffffffu, valid && w != 0.0);
            while (act) {
                const int src = __ffs(act) - 1;
                act &= act - 1;
                const double ws = __shfl_sync(0xffffffffu, w, src);
                const int ps = __shfl_sync(0xffffffffu, int(mm & 0xffu), src);
                Key<NW> kk;
#pragma unroll
                for (int q = 0; q < NW; ++q) kk.w[q] = __shfl_sync(0xffffffffu, k.w[q], src);
#pragma unroll
                for (int qi = 0; qi < 4; ++qi) {
                    const int s = lane + 32 * qi;
                    if (s < L) {
                        pho[qi] += ws * double(get_field(m, kk, s));
                        if (ps == s) exc[qi] += ws;
                    }
                }
            }
        }
    }
    // block partials, fixed order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        norm2 += __shfl_xor_sync(0xffffffffu, norm2, o);
        er += __shfl_xor_sync(0xffffffffu, er, o);
        ei += __shfl_xor_sync(0xffffffffu, ei, o);
    }
    if (lane == 0) {
        s_red[wid][0] = norm2;
        s_red[wid][1] = er;
        s_red[wid][2] = ei;
    }
    if (sites) {
#pragma unroll
        for (int qi = 0; qi < 4; ++qi) {
            const int s = lane + 32 * qi;
            if (s < L) {
                s_site[wid][s] = exc[qi];
                s_site[wid][L + s] = pho[qi];
            }
        }
    }
    __syncthreads();
    double* out = partials + size_t(blockIdx.x) * nvals;
    for (int v = threadIdx.x; v < nvals; v += kOThreads) {
        double acc = 0.0;
        if (v < 3) {
            for (int w2 = 0; w2 < kOWarps; ++w2) acc += s_red[w2][v];
        } else if (sites) {
            for (int w2 = 0; w2 < kOWarps; ++w2) acc += s_site[w2][v - 3];
        }
        out[v] = acc;
    }
}

__global__ void obs_final_kernel(int L, int nblocks, const double* __restrict__ partials, ObsTarget t) {
    const int nvals = 3 + 2 * L;
    for (int v = threadIdx.x; v < nvals; v += blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < nblocks; ++b) acc += partials[size_t(b) * nvals + v];
        if (v == 0) {
            if (t.norm) *t.norm = sqrt(acc);
        } else if (v == 1) {
            if (t.energy_re) *t.energy_re = acc;
        } else if (v == 2) {
            if (t.energy_im) *t.energy_im = acc;
        } else if (v < 3 + L) {
            if (t.n_exc) t.n_exc[v - 3] = acc;
        } else {
            if (t.n_pho) t.n_pho[v - 3 - L] = acc;
        }
    }
}

template <bool C64>
__global__ void scale_kernel(int L, const int* __restrict__ blk, void* psi, const double* norm) {
    using C = typename std::conditional<C64, float2, double2>::type;
    const int64_t S = blk[L];
    const double nv = *norm;
    C* x = reinterpret_cast<C*>(psi);
    for (int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < S; r += int64_t(gridDim.x) * blockDim.x) {
        C z = x[r];
        if constexpr (C64) {
            z.x = float(double(z.x) / nv);
            z.y = float(double(z.y) / nv);
        } else {
            z.x = z.x / nv;
            z.y = z.y / nv;
        }
        x[r] = z;
    }
}

template <int NW, bool C64>
int launch_obs_t(const ModelDev& m, const uint64_t* keys, const int* blk, const int* nbr,
                 int64_t nbr_cap, const uint32_t* meta, const void* psi, int what, double* partials,
                 const ObsTarget& out, int num_sms, cudaStream_t st) {
    const int grid = obs_max_grid(num_sms);
    obs_kernel<NW, C64><<<grid, kOThreads, 0, st>>>(m, keys, blk, nbr, nbr_cap, meta, psi, what, partials);
    obs_final_kernel<<<1, 256, 0, st>>>(m.L, grid, partials, out);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace

int launch_observables(int nw, bool c64, const ModelDev& m, const uint64_t* keys, const int* blk,
                       const int* nbr, int64_t nbr_cap, const uint32_t* meta, const void* psi,
                       int what, double* partials, const ObsTarget& out, int num_sms,
                       cudaStream_t st) {
#define PACES_OBS_CASE(N)                                                                          \
    case N:                                                                                        \
        return c64 ? launch_obs_t<N, true>(m, keys, blk, nbr, nbr_cap, meta, psi, what, partials,  \
                                           out, num_sms, st)                                       \
                   : launch_obs_t<N, false>(m, keys, blk, nbr, nbr_cap, meta, psi, what, partials, \
                                            out, num_sms, st);
    switch (nw) {
        PACES_OBS_CASE(1)
        PACES_OBS_CASE(2)
        PACES_OBS_CASE(3)
        PACES_OBS_CASE(4)
        PACES_OBS_CASE(5)
        PACES_OBS_CASE(6)
        PACES_OBS_CASE(7)
        PACES_OBS_CASE(8)
        default: return PACES_ERR_BADARG;
    }
#undef PACES_OBS_CASE
}

int launch_scale(bool c64, const ModelDev& m, const int* blk, void* psi, const double* norm,
                 int num_sms, cudaStream_t st) {
    if (c64) scale_kernel<true><<<num_sms * 4, 256, 0, st>>>(m.L, blk, psi, norm);
    else scale_kernel<false><<<num_sms * 4, 256, 0, st>>>(m.L, blk, psi, norm);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
