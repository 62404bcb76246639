// exp(t A) psi by scaling and squaring with a truncated Taylor series per stage, for
// A = i (H - mu I) -- the propagation the reference runs with ExpmParams(use_scaling=True).
//
// Reference: paces/core/time_evolution.py:579-581 calls expm_multiply_simple(1j * H, psi,
// t=dt), paces/aux/_scipy/_expm_multiply.py:106-202 (Al-Mohy and Higham 2011, algorithm
// 3.2): mu = trace(A)/n is removed from the diagonal, the stage count s and the order
// bound m come from the 1-norm of A - mu I (fragment 3.1), and every stage runs up to m
// terms  B <- t/(s (j+1)) (A - mu I) B,  F <- F + B  with the inf-norm stop test, then
// F <- exp(t mu / s) F and B <- F.  The host chooses s and m from the two norms these
// kernels measure (`paces_b200/expm.py`).
//
// B200 design: the norms are two deterministic reductions over the neighbour table; the
// whole series -- every term of every stage and the stage-end phase factors -- is one
// persistent cooperative launch with a bounded grid barrier between sweeps, as in the
// plain Taylor kernel.  Each stage's first term reads a copy of F (made during the
// stage-end sweep), so no sweep gathers from a vector it is writing.
#include "grid.cuh"
#include "hrow.cuh"
#include "kernels.cuh"

namespace paces {

namespace {

constexpr int kEThreads = 256;
constexpr int kEWarps = kEThreads / 32;

__device__ void block_max4(double v[4], double (*red)[kEWarps], double* out) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] = fmax(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
        if (lane == 0) red[k][wid] = v[k];
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double r = 0.0;
        for (int w = 0; w < kEWarps; ++w) r = fmax(r, red[threadIdx.x][w]);
        out[threadIdx.x] = r;
    }
    __syncthreads();
}

// Per-block partials of the trace (sum of diagonal elements, [0]) and of the largest row
// 1-norm of H - shift I ([1]; only when shift is given).
__global__ void __launch_bounds__(kEThreads)
hnorm_kernel(ModelDev m, const int* __restrict__ blk, const int* __restrict__ nbr, const uint32_t* __restrict__ meta,
             const double* __restrict__ shift, double* __restrict__ part) {
    __shared__ double s_sum[kEWarps], s_max[kEWarps];
    const int64_t S = blk[m.L];
    const double d0 = shift ? *shift : 0.0;
    double sum = 0.0, mx = 0.0;
    for (int64_t r = int64_t(blockIdx.x) * kEThreads + threadIdx.x; r < S; r += int64_t(gridDim.x) * kEThreads) {
        const uint32_t mm = __ldg(meta + r);
        const double d = diag_value(m, mm);
        sum += d;
        if (shift) {
            const int4 nb = load_nbr(nbr, r);
            const int n = int((mm >> 8) & 0xffu);
            double a = fabs(d - d0);
            if (m.nhop > 1) {
                for (int t = 0; t < 2; ++t)
                    for (int e = 0; e < m.hop_n[t]; ++e)
                        if (hop_index(m, r, nb, m.hop_ord[t][e]) >= 0) a += fabs(t == 0 ? m.J : m.J2);
            } else {
                a += (nb.x >= 0 ? fabs(m.J) : 0.0) + (nb.y >= 0 ? fabs(m.J) : 0.0);
            }
            a += (nb.z >= 0 ? fabs(m.g) * sqrt(double(n)) : 0.0) + (nb.w >= 0 ? fabs(m.g) * sqrt(double(n + 1)) : 0.0);
            mx = fmax(mx, a);
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
        s_sum[wid] = sum;
        s_max[wid] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < kEWarps; ++w) {
            a += s_sum[w];
            b = fmax(b, s_max[w]);
        }
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

// Fixed-order reduction of the partials: out[0] = trace, out[1] = max row 1-norm,
// out[2] = trace / n.
__global__ void hnorm_final_kernel(const int* __restrict__ blk, int L, const double* __restrict__ part, int nparts,
                                   double* __restrict__ out) {
    if (threadIdx.x != 0) return;
    double a = 0.0, b = 0.0;
    for (int i = 0; i < nparts; ++i) {
        a += part[2 * i];
        b = fmax(b, part[2 * i + 1]);
    }
    const int64_t S = blk[L];
    out[0] = a;
    out[1] = b;
    out[2] = S > 0 ? a / double(S) : 0.0;
}

template <bool C64>
__global__ void __launch_bounds__(kEThreads, C64 ? 4 : 3)
expm_scaled_kernel(ModelDev m, const int* __restrict__ blk, const int* __restrict__ nbr,
                   const uint32_t* __restrict__ meta, const void* v_in, void* res_out, TaylorWs ws, double t,
                   double shift, int m_star, int stages, double tol, double eta_re, double eta_im, TaylorOut out,
                   int* status) {
    using C = typename std::conditional<C64, float2, double2>::type;
    using R = typename std::conditional<C64, float, double>::type;
    __shared__ R s_sq[260];
    __shared__ double s_red[4][kEWarps];
    __shared__ double s_fin[4];
    for (int k = threadIdx.x; k < 260; k += kEThreads) s_sq[k] = R(__dmul_rn(sqrt(double(k)), m.g));
    __syncthreads();
    const int64_t S = blk[m.L];
    const unsigned nblocks = gridDim.x;
    unsigned gen = 0;
    const C* v = reinterpret_cast<const C*>(v_in);
    C* res = reinterpret_cast<C*>(res_out);
    C* ta = reinterpret_cast<C*>(ws.ta);
    C* tb = reinterpret_cast<C*>(ws.tb);
    const R J = R(m.J);
    const R sh = R(shift);
    const int64_t stride = int64_t(gridDim.x) * kEThreads;
    const int64_t r0 = int64_t(blockIdx.x) * kEThreads + threadIdx.x;
    double c1 = 0.0, c1c2 = 0.0, ratio = 0.0;
    int conv = 0, final_m = 0;
    bool stop = false;

    for (int st = 0; st < stages && !stop; ++st) {
        for (int j = 0; j < m_star; ++j) {
            // stage 0 starts from the input; later stages from the copy of F in tb
            const C* src = j == 0 ? (st == 0 ? v : tb) : ((j & 1) ? ta : tb);
            C* dst = (j & 1) ? tb : ta;
            const C* rin = (st == 0 && j == 0) ? v : res;
            const double cd = t / (double(stages) * double(j + 1));
            const R c = R(cd);
            double mx[4] = {0.0, 0.0, 0.0, 0.0};  // |B|, |F|, |B at stage start|, non-finite
            for (int64_t r = r0; r < S; r += stride) {
                const uint32_t mm = __ldg(meta + r);
                C y;
                const C xr = __ldcg(src + r);
                if constexpr (C64) {
                    y = h_row_c64_any(m, s_sq, J, r, load_nbr(nbr, r), mm, __ldcg(src + r), src);
                    y.x = fmaf(-sh, xr.x, y.x);
                    y.y = fmaf(-sh, xr.y, y.y);
                } else {
                    y = h_row_c128_any(m, s_sq, r, load_nbr(nbr, r), mm, __ldcg(src + r), src);
                    y.x = __dsub_rn(y.x, __dmul_rn(sh, xr.x));
                    y.y = __dsub_rn(y.y, __dmul_rn(sh, xr.y));
                }
                // B = c * i * y
                C b, f;
                const C a = rin[r];
                if constexpr (C64) {
                    b = make_float2(-(c * y.y), c * y.x);
                    f = make_float2(a.x + b.x, a.y + b.y);
                    mx[0] = fmax(mx[0], double(fmaf(b.x, b.x, b.y * b.y)));
                    mx[1] = fmax(mx[1], double(fmaf(f.x, f.x, f.y * f.y)));
                    if (j == 0) mx[2] = fmax(mx[2], double(fmaf(xr.x, xr.x, xr.y * xr.y)));
                } else {
                    b = make_double2(-__dmul_rn(cd, y.y), __dmul_rn(cd, y.x));
                    f = make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
                    mx[0] = fmax(mx[0], fma(b.x, b.x, b.y * b.y));
                    mx[1] = fmax(mx[1], fma(f.x, f.x, f.y * f.y));
                    if (j == 0) mx[2] = fmax(mx[2], fma(xr.x, xr.x, xr.y * xr.y));
                }
                if (!(isfinite(double(f.x)) && isfinite(double(f.y)))) mx[3] = 1.0;
                dst[r] = b;
                res[r] = f;
            }
            block_max4(mx, s_red, s_fin);
            if (threadIdx.x == 0) {
                double* pp = ws.partials + (size_t((final_m & 1) * nblocks) + blockIdx.x) * 4;
                for (int k = 0; k < 4; ++k) pp[k] = s_fin[k];
            }
            if (!grid_barrier(ws.barrier, nblocks, gen, status, ws.wait_ns, int(blockIdx.x) == ws.skip_block)) {
                stop = true;
                break;
            }
            double g4[4] = {0.0, 0.0, 0.0, 0.0};
            for (unsigned bb = threadIdx.x; bb < nblocks; bb += kEThreads) {
                const double* pp = ws.partials + (size_t((final_m & 1) * nblocks) + bb) * 4;
#pragma unroll
                for (int k = 0; k < 4; ++k) g4[k] = fmax(g4[k], __ldcg(pp + k));
            }
            block_max4(g4, s_red, s_fin);
            ++final_m;
            if (s_fin[3] != 0.0) {
                if (blockIdx.x == 0 && threadIdx.x == 0) raise_status(status, PACES_ERR_NONFINITE);
                stop = true;
                break;
            }
            if (j == 0) c1 = sqrt(s_fin[2]);
            const double c2 = sqrt(s_fin[0]);
            c1c2 = c1 + c2;
            ratio = c1c2 / sqrt(s_fin[1]);
            if (ratio <= tol) {
                conv = 1;
                break;
            }
            c1 = c2;
        }
        if (stop) break;
        // F <- exp(t mu / s) F, and the next stage's B is a copy of F
        const bool phase = !(eta_re == 1.0 && eta_im == 0.0);
        for (int64_t r = r0; r < S; r += stride) {
            C f = (st == 0 && m_star == 0) ? v[r] : res[r];
            if (phase) {
                if constexpr (C64) {
                    const float er = float(eta_re), ei = float(eta_im);
                    f = make_float2(er * f.x - ei * f.y, er * f.y + ei * f.x);
                } else {
                    f = make_double2(__dsub_rn(__dmul_rn(eta_re, f.x), __dmul_rn(eta_im, f.y)),
                                     __dadd_rn(__dmul_rn(eta_re, f.y), __dmul_rn(eta_im, f.x)));
                }
            }
            res[r] = f;
            tb[r] = f;
        }
        if (st + 1 < stages && !grid_barrier(ws.barrier, nblocks, gen, status, ws.wait_ns,
                                             int(blockIdx.x) == ws.skip_block))
            break;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (out.converged) *out.converged = conv;
        if (out.final_m) *out.final_m = final_m;
        if (out.c1_plus_c2) *out.c1_plus_c2 = c1c2;
        if (out.term_ratio) *out.term_ratio = ratio;
    }
}

template <bool C64>
int expm_occupancy() {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, expm_scaled_kernel<C64>, kEThreads, 0);
    return per_sm < 1 ? 1 : (per_sm > 8 ? 8 : per_sm);
}

}  // namespace

int launch_hnorms(const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta, const double* shift,
                  double* part, int nparts, double* out, cudaStream_t st) {
    hnorm_kernel<<<nparts, kEThreads, 0, st>>>(m, blk, nbr, meta, shift, part);
    hnorm_final_kernel<<<1, 32, 0, st>>>(blk, m.L, part, nparts, out);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

int launch_expm_scaled(bool c64, const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta,
                       const void* v_in, void* res, double t, double shift, int m_star, int stages, double tol,
                       double eta_re, double eta_im, const TaylorWs& ws, const TaylorOut& out, int* status,
                       int num_sms, int max_grid, cudaStream_t st) {
    if (m_star < 0 || stages < 1) return PACES_ERR_BADARG;
    if (cudaMemsetAsync(ws.barrier, 0, 2 * sizeof(unsigned), st) != cudaSuccess) return PACES_ERR_CUDA;
    int grid = num_sms * (c64 ? expm_occupancy<true>() : expm_occupancy<false>());
    if (grid > max_grid) grid = max_grid;  // the partials buffer holds max_grid blocks
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kEThreads);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e =
        c64 ? cudaLaunchKernelEx(&cfg, expm_scaled_kernel<true>, m, blk, nbr, meta, v_in, res, ws, t, shift, m_star,
                                 stages, tol, eta_re, eta_im, out, status)
            : cudaLaunchKernelEx(&cfg, expm_scaled_kernel<false>, m, blk, nbr, meta, v_in, res, ws, t, shift, m_star,
                                 stages, tol, eta_re, eta_im, out, status);
    return e == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
