// Krylov (Lanczos) exp(-i dt H) psi as one persistent cooperative kernel.
//
// Reference: _lanczos (paces/core/time_evolution.py:515-549), selected by
// ExpmParams.lanczos_order = m > 0 (:577-578).  From q_0 = psi / |psi| the plain Lanczos
// recurrence (no re-orthogonalisation) builds m+1 vectors:
//   w = H q_i - beta_i q_{i-1},  alpha_i = vdot(w, q_i) (complex),  w -= alpha_i q_i,
//   beta_{i+1} = |w|  (stop when beta < 1e-15),  q_{i+1} = w / beta_{i+1};
// the (m+1)^2 tridiagonal T = tridiag(beta, alpha, beta) is exponentiated densely
// (scipy/cupyx expm) and psi(t + dt) = |psi| V exp(-i dt T) e_0.  The diagnostics are the
// reference's placeholder [False, 0, 0, 0].  The reference makes one host round trip per
// vector (norms, vdot) and a dense expm on the device.
//
// B200 design: the whole recurrence is one launch.  Per Krylov vector two grid-stride
// sweeps, each closed by a bounded grid barrier:
//   A_i  q_i = s / beta_i and (H q_i)_r = (H s)_r / beta_i from the unnormalised s = the
//        previous w (gathered through the neighbour table, as in the Taylor kernel), stores
//        q_i (column i of V) and w = H q_i - beta_i q_{i-1}; partial vdot(w, q_i);
//   B_i  w -= alpha_i q_i in place; partial |w|^2.
// The partial sums are fp64 (complex64 vectors too) and every block adds the per-block
// partials in the same order, so all blocks hold bit-identical alpha and beta and take the
// same stop decision.  After the recurrence every block computes the first column of
// exp(-i dt T) itself in fp64 (below), and a last sweep forms |psi| sum_i c_i q_i.
//
// The small exponential: x = exp(A) e_0 for A = -i dt T by the truncated Taylor series with
// s sub-steps, x <- sum_j (A/s)^j x / j!, s = ceil(|A|_1) so every sub-step has |A/s|_1 <= 1
// -- the stepping of Al-Mohy and Higham, "Computing the action of the matrix exponential"
// (SIAM J. Sci. Comput. 33, 2011), with the stop test of the plain Taylor path (two
// consecutive terms below 2^-53 of the sum in the inf-norm).  T is tridiagonal, so each
// term costs O(m); one warp computes it, two rows per lane.
#include "grid.cuh"
#include "hrow.cuh"
#include "kernels.cuh"

namespace paces {

namespace {

constexpr int kLThreads = 256;
constexpr int kLWarps = kLThreads / 32;
constexpr int kKrylovMax = kMaxLanczosOrder + 1;  // vectors
static_assert(kKrylovMax <= 64, "the small exponential holds two rows per lane of one warp");

// Sum of NV doubles over the block, in a fixed order (warp shuffles, then the warps in
// index order); the result is in out[0..NV) for every thread after the call.
template <int NV>
__device__ void block_sum(double v[NV], double (*red)[kLWarps], double* out) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        if (lane == 0) red[k][wid] = v[k];
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double r = 0.0;
        for (int w = 0; w < kLWarps; ++w) r += red[threadIdx.x][w];
        out[threadIdx.x] = r;
    }
    __syncthreads();
}

// Grid-wide sum of NV doubles: block partials into ws.partials[parity], the barrier, then
// every block adds all partials in the same order.  false when the barrier timed out.
template <int NV>
__device__ bool grid_sum(double v[NV], const LanczosWs& ws, int parity, unsigned& gen, int* status,
                         double (*red)[kLWarps], double* fin) {
    block_sum<NV>(v, red, fin);
    const unsigned nblocks = gridDim.x;
    if (threadIdx.x == 0) {
        double* pp = ws.partials + (size_t(parity) * ws.max_grid + blockIdx.x) * 4;
#pragma unroll
        for (int k = 0; k < NV; ++k) pp[k] = fin[k];
    }
    if (!grid_barrier(ws.barrier, nblocks, gen, status, ws.wait_ns, int(blockIdx.x) == ws.skip_block)) return false;
    double g[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) g[k] = 0.0;
    for (unsigned b = threadIdx.x; b < nblocks; b += kLThreads) {
        const double* pp = ws.partials + (size_t(parity) * ws.max_grid + b) * 4;
#pragma unroll
        for (int k = 0; k < NV; ++k) g[k] += __ldcg(pp + k);
    }
    block_sum<NV>(g, red, fin);
    return true;
}

// First column of exp(-i dt T), T = tridiag(beta[1..k-1], alpha[0..k-1], beta[1..k-1]),
// into (lre, lim); warp 0 of the block, fp64.
__device__ void small_expm_col0(int k, double dt, const double* are, const double* aim, const double* beta,
                                double* lre, double* lim, double* tre, double* tim, double* nre, double* nim) {
    const int lane = threadIdx.x;  // warp 0 only
    auto off = [&](int r) { return (r >= 1 && r < k) ? beta[r] : 0.0; };  // couples r-1 and r
    double a1 = 0.0;
    for (int r = lane; r < k; r += 32) {
        lre[r] = r == 0 ? 1.0 : 0.0;
        lim[r] = 0.0;
        a1 = fmax(a1, dt * (hypot(are[r], aim[r]) + off(r) + off(r + 1)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a1 = fmax(a1, __shfl_xor_sync(0xffffffffu, a1, o));
    const int s = a1 > 1.0 ? int(ceil(a1)) : 1;
    auto inf_norm = [&](const double* xr, const double* xi) {
        double v = 0.0;
        for (int r = lane; r < k; r += 32) v = fmax(v, hypot(xr[r], xi[r]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        return v;
    };
    for (int step = 0; step < s; ++step) {
        for (int r = lane; r < k; r += 32) {
            tre[r] = lre[r];
            tim[r] = lim[r];
        }
        __syncwarp();
        double c1 = inf_norm(tre, tim);
        for (int j = 1; j <= 80; ++j) {
            const double c = dt / (double(s) * double(j));
            // new term = -i c T term
            for (int r = lane; r < k; r += 32) {
                double yr = are[r] * tre[r] - aim[r] * tim[r];
                double yi = are[r] * tim[r] + aim[r] * tre[r];
                if (r >= 1) {
                    yr += beta[r] * tre[r - 1];
                    yi += beta[r] * tim[r - 1];
                }
                if (r + 1 < k) {
                    yr += beta[r + 1] * tre[r + 1];
                    yi += beta[r + 1] * tim[r + 1];
                }
                nre[r] = c * yi;
                nim[r] = -c * yr;
            }
            __syncwarp();
            for (int r = lane; r < k; r += 32) {
                tre[r] = nre[r];
                tim[r] = nim[r];
                lre[r] += nre[r];
                lim[r] += nim[r];
            }
            __syncwarp();
            const double c2 = inf_norm(tre, tim);
            const double f = inf_norm(lre, lim);
            if (c1 + c2 <= 1.1102230246251565e-16 * f) break;
            c1 = c2;
        }
    }
    __syncwarp();
}

template <bool C64, bool XHOP>
__global__ void __launch_bounds__(kLThreads)
lanczos_kernel(ModelDev m, const int* __restrict__ blk, const int* __restrict__ nbr, const uint32_t* __restrict__ meta,
               const void* v_in, void* res_out, LanczosWs ws, double dt, int order, TaylorOut out, int* status) {
    using C = typename std::conditional<C64, float2, double2>::type;
    using R = typename std::conditional<C64, float, double>::type;
    __shared__ R s_sq[260];
    __shared__ double s_red[4][kLWarps];
    __shared__ double s_fin[4];
    __shared__ double s_are[kKrylovMax], s_aim[kKrylovMax], s_beta[kKrylovMax + 1];
    __shared__ double s_lre[kKrylovMax], s_lim[kKrylovMax];
    __shared__ double s_w[4][kKrylovMax];
    for (int k = threadIdx.x; k < 260; k += kLThreads) s_sq[k] = R(__dmul_rn(sqrt(double(k)), m.g));
    for (int k = threadIdx.x; k <= kKrylovMax; k += kLThreads) s_beta[k] = 0.0;
    __syncthreads();

    const int64_t S = blk[m.L];
    const int64_t cap = ws.cap;
    const int64_t stride = int64_t(gridDim.x) * kLThreads;
    const int64_t r0 = int64_t(blockIdx.x) * kLThreads + threadIdx.x;
    const C* v = reinterpret_cast<const C*>(v_in);
    C* res = reinterpret_cast<C*>(res_out);
    C* U = reinterpret_cast<C*>(ws.u);
    C* Wb[2] = {reinterpret_cast<C*>(ws.w0), reinterpret_cast<C*>(ws.w1)};
    const R J = R(m.J);
    unsigned gen = 0;
    int parity = 0;
    bool ok = true;

    // |psi|
    double nv[1] = {0.0};
    for (int64_t r = r0; r < S; r += stride) {
        const C x = v[r];
        nv[0] += double(x.x) * double(x.x) + double(x.y) * double(x.y);
    }
    ok = grid_sum<1>(nv, ws, parity, gen, status, s_red, s_fin);
    parity ^= 1;
    const double nrm = sqrt(s_fin[0]);
    if (ok && !(nrm > 0.0 && nrm <= 1.7976931348623157e308)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_status(status, PACES_ERR_NONFINITE);
        ok = false;
    }
    int k = 0;             // Krylov vectors built
    double beta = nrm;     // scale of the source of the next A sweep
    for (int i = 0; ok && i <= order; ++i) {
        // A_i
        const C* src = i == 0 ? v : Wb[(i - 1) & 1];
        C* w = Wb[i & 1];
        C* qi = U + int64_t(i) * cap;
        const C* qp = i > 0 ? U + int64_t(i - 1) * cap : nullptr;
        const double bi = i > 0 ? s_beta[i] : 0.0;
        double pa[2] = {0.0, 0.0};
        // (H s)_r and s_r of one row (all its loads issued here)
        auto load_row = [&](int64_t r, C& y, C& xr) {
            const uint32_t mm = __ldg(meta + r);
            const int4 nb = load_nbr(nbr, r);
            xr = __ldcg(src + r);
            if constexpr (XHOP) {
                if constexpr (C64) y = h_row_c64_x(m, s_sq, r, nb, mm, xr, src);
                else y = h_row_c128_x(m, s_sq, r, nb, mm, xr, src);
            } else {
                if constexpr (C64) y = h_row_c64_nb(m, s_sq, J, r, nb, mm, xr, src);
                else y = h_row_c128_nb(m, s_sq, r, nb, mm, xr, src);
            }
        };
        // q_r = s_r / beta, w_r = (H s)_r / beta - beta_i q_{i-1,r}; the vdot partial
        const double rb = 1.0 / beta;
        auto finish_row = [&](int64_t r, const C& y, const C& xr, const C& p) {
            C q, wr;
            if constexpr (C64) {
                const float b = float(rb), bp = float(bi);
                q = make_float2(xr.x * b, xr.y * b);
                wr = make_float2(y.x * b, y.y * b);
                wr.x = fmaf(-bp, p.x, wr.x);
                wr.y = fmaf(-bp, p.y, wr.y);
            } else {
                q = make_double2(__dmul_rn(xr.x, rb), __dmul_rn(xr.y, rb));
                wr = make_double2(__dmul_rn(y.x, rb), __dmul_rn(y.y, rb));
                wr = make_double2(__dsub_rn(wr.x, __dmul_rn(bi, p.x)), __dsub_rn(wr.y, __dmul_rn(bi, p.y)));
            }
            qi[r] = q;
            w[r] = wr;
            // vdot(w, q) = sum conj(w) q
            pa[0] += double(wr.x) * double(q.x) + double(wr.y) * double(q.y);
            pa[1] += double(wr.x) * double(q.y) - double(wr.y) * double(q.x);
        };
        C zero;
        zero.x = 0;
        zero.y = 0;
        {
            // two rows a grid stride apart per iteration: their loads are in flight together
            int64_t r = r0;
            for (; r + stride < S; r += 2 * stride) {
                C y0, x0, y1, x1;
                load_row(r, y0, x0);
                load_row(r + stride, y1, x1);
                const C p0 = qp ? qp[r] : zero, p1 = qp ? qp[r + stride] : zero;
                finish_row(r, y0, x0, p0);
                finish_row(r + stride, y1, x1, p1);
            }
            if (r < S) {
                C y0, x0;
                load_row(r, y0, x0);
                finish_row(r, y0, x0, qp ? qp[r] : zero);
            }
        }
        if (!grid_sum<2>(pa, ws, parity, gen, status, s_red, s_fin)) {
            ok = false;
            break;
        }
        parity ^= 1;
        const double are = s_fin[0], aim = s_fin[1];
        if (!(isfinite(are) && isfinite(aim))) {
            if (blockIdx.x == 0 && threadIdx.x == 0) raise_status(status, PACES_ERR_NONFINITE);
            ok = false;
            break;
        }
        if (threadIdx.x == 0) {
            s_are[i] = are;
            s_aim[i] = aim;
        }
        k = i + 1;
        if (i == order) break;
        // B_i
        double pb[1] = {0.0};
        auto axpy_row = [&](int64_t r, const C& q, C wr) {
            if constexpr (C64) {
                const float ar = float(are), ai = float(aim);
                wr.x -= ar * q.x - ai * q.y;
                wr.y -= ar * q.y + ai * q.x;
            } else {
                const double px = __dsub_rn(__dmul_rn(are, q.x), __dmul_rn(aim, q.y));
                const double py = __dadd_rn(__dmul_rn(are, q.y), __dmul_rn(aim, q.x));
                wr = make_double2(__dsub_rn(wr.x, px), __dsub_rn(wr.y, py));
            }
            w[r] = wr;
            pb[0] += double(wr.x) * double(wr.x) + double(wr.y) * double(wr.y);
        };
        {
            int64_t r = r0;
            for (; r + stride < S; r += 2 * stride) {
                const C q0 = qi[r], w0 = w[r], q1 = qi[r + stride], w1 = w[r + stride];
                axpy_row(r, q0, w0);
                axpy_row(r + stride, q1, w1);
            }
            if (r < S) axpy_row(r, qi[r], w[r]);
        }
        if (!grid_sum<1>(pb, ws, parity, gen, status, s_red, s_fin)) {
            ok = false;
            break;
        }
        parity ^= 1;
        const double bnext = sqrt(s_fin[0]);
        if (!(bnext <= 1.7976931348623157e308)) {
            if (blockIdx.x == 0 && threadIdx.x == 0) raise_status(status, PACES_ERR_NONFINITE);
            ok = false;
            break;
        }
        if (bnext < 1e-15) break;  // the Krylov space is invariant: k vectors
        if (threadIdx.x == 0) s_beta[i + 1] = bnext;
        __syncthreads();
        beta = bnext;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (out.converged) *out.converged = 0;
        if (out.final_m) *out.final_m = 0;
        if (out.c1_plus_c2) *out.c1_plus_c2 = 0.0;
        if (out.term_ratio) *out.term_ratio = 0.0;
    }
    if (!ok) return;
    __syncthreads();
    if (threadIdx.x < 32) small_expm_col0(k, dt, s_are, s_aim, s_beta, s_lre, s_lim, s_w[0], s_w[1], s_w[2], s_w[3]);
    __syncthreads();
    // psi(t + dt) = |psi| sum_i c_i q_i
    bool finite = true;
    for (int64_t r = r0; r < S; r += stride) {
        double fr = 0.0, fi = 0.0;
        for (int i = 0; i < k; ++i) {
            const C q = U[int64_t(i) * cap + r];
            fr += s_lre[i] * double(q.x) - s_lim[i] * double(q.y);
            fi += s_lre[i] * double(q.y) + s_lim[i] * double(q.x);
        }
        fr *= nrm;
        fi *= nrm;
        if (!(isfinite(fr) && isfinite(fi))) finite = false;
        if constexpr (C64) res[r] = make_float2(float(fr), float(fi));
        else res[r] = make_double2(fr, fi);
    }
    if (!finite) raise_status(status, PACES_ERR_NONFINITE);
}

template <bool C64, bool XHOP>
int lanczos_occupancy() {
    static int cached = 0;  // per process: the kernel's resources do not change
    if (cached) return cached;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lanczos_kernel<C64, XHOP>, kLThreads, 0);
    cached = per_sm < 1 ? 1 : (per_sm > 8 ? 8 : per_sm);
    return cached;
}

}  // namespace

int lanczos_max_grid(int num_sms) {
    int best = lanczos_occupancy<true, false>();
    const int o[3] = {lanczos_occupancy<true, true>(), lanczos_occupancy<false, false>(),
                      lanczos_occupancy<false, true>()};
    for (int x : o) best = x > best ? x : best;
    return num_sms * best;
}

int launch_lanczos(bool c64, const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta,
                   const void* v_in, void* res, double dt, int order, const LanczosWs& ws, const TaylorOut& out,
                   int* status, int num_sms, cudaStream_t st) {
    if (order < 1 || order > kMaxLanczosOrder) return PACES_ERR_BADARG;
    if (m.nhop > 1 && !m.xnbr) return PACES_ERR_BADARG;
    if (cudaMemsetAsync(ws.barrier, 0, 2 * sizeof(unsigned), st) != cudaSuccess) return PACES_ERR_CUDA;
    const bool xhop = m.nhop > 1;
    const int occ = c64 ? (xhop ? lanczos_occupancy<true, true>() : lanczos_occupancy<true, false>())
                        : (xhop ? lanczos_occupancy<false, true>() : lanczos_occupancy<false, false>());
    // a fixed wave: the fp64 partial sums (and so alpha, beta) do not depend on buffer sizes
    int grid = num_sms * occ;
    if (grid > ws.max_grid) grid = ws.max_grid;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kLThreads);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e;
    if (c64) {
        e = xhop ? cudaLaunchKernelEx(&cfg, lanczos_kernel<true, true>, m, blk, nbr, meta, v_in, res, ws, dt, order, out, status)
                 : cudaLaunchKernelEx(&cfg, lanczos_kernel<true, false>, m, blk, nbr, meta, v_in, res, ws, dt, order, out, status);
    } else {
        e = xhop ? cudaLaunchKernelEx(&cfg, lanczos_kernel<false, true>, m, blk, nbr, meta, v_in, res, ws, dt, order, out, status)
                 : cudaLaunchKernelEx(&cfg, lanczos_kernel<false, false>, m, blk, nbr, meta, v_in, res, ws, dt, order, out, status);
    }
    return e == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
