// Truncated-Taylor exp(-i dt H) psi as one persistent cooperative kernel.
//
// Reference (paces/core/time_evolution.py:482-512, _simple_taylor): term_{j+1} =
// (-i dt/(j+1)) H term_j, res += term_{j+1}, stop when (|term_j|_inf + |term_{j+1}|_inf) /
// |res|_inf <= tol, at most m_star terms; one host sync per term in the reference.
//
// B200 design: every term is one grid-stride sweep over the rows (neighbour-table SpMV,
// term write, res update and the two inf-norms fused), separated by a bounded grid
// barrier; every block reduces the per-block maxima itself and takes the same stop
// decision, so the whole series runs in one launch with no host round trip.  The
// neighbour indices of consecutive rows are monotone (images of a sorted block are
// sorted), so the four gathers stream through L2.  complex128 rounds every operation
// like the reference; complex64 uses fp32 FMA with fp64 stop arithmetic.
//
// Two row schedules (a tuning choice; the results are identical because every row's
// arithmetic is the same and the maxima are exact):
//  * direct: grid-stride, two rows per thread per pass, all loads from global memory;
//  * bulk:   each block owns 512-row chunks; while it computes one chunk, one thread has
//            the next chunk's neighbour rows, metadata, result and own term elements
//            brought into the other half of a shared-memory double buffer by bulk TMA
//            copies (cp.async.bulk, completion on an mbarrier), so the streaming reads are
//            in flight while the gathers of the current chunk wait on L2.
#include "grid.cuh"
#include "hrow.cuh"
#include "kernels.cuh"
#include "tc.cuh"

namespace paces {

namespace {

constexpr int kTThreads = 256;
constexpr int kTWarps = kTThreads / 32;

// max-reduce four values over the block; result in out[0..3] (shared), valid after return.
__device__ void block_max4(double v[4], double (*red)[kTWarps], double* out) {
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
        for (int w = 0; w < kTWarps; ++w) r = fmax(r, red[threadIdx.x][w]);
        out[threadIdx.x] = r;
    }
    __syncthreads();
}

constexpr int kChunk = 2 * kTThreads;  // rows per block pass of the bulk schedule
template <bool C64>
constexpr uint32_t chunk_bytes() {  // neighbour rows, metadata, result, own term element
    return uint32_t(kChunk) * (16 + 4 + 2 * (C64 ? 8 : 16));
}

// XHOP: a lattice with several hopping channels (the channel loop of h_row_*_x).
template <bool C64, bool BULK, bool XHOP>
__global__ void __launch_bounds__(kTThreads, C64 ? 4 : 3)
taylor_kernel(ModelDev m, const int* __restrict__ blk, const int* __restrict__ nbr, int64_t cap,
              const uint32_t* __restrict__ meta, const void* v_in, void* res_out, TaylorWs ws,
              double dt, int m_star, double tol, TaylorOut out, int* status) {
    using C = typename std::conditional<C64, float2, double2>::type;
    using R = typename std::conditional<C64, float, double>::type;
    extern __shared__ __align__(128) unsigned char t_smem[];  // bulk: 2 x chunk_bytes
    __shared__ R s_sq[260];
    __shared__ double s_red[4][kTWarps];
    __shared__ double s_fin[4];
    __shared__ __align__(8) uint64_t s_mbar[2];
    __shared__ int s_abort;
    for (int k = threadIdx.x; k < 260; k += kTThreads) s_sq[k] = R(__dmul_rn(sqrt(double(k)), m.g));
    if constexpr (BULK) {
        if (threadIdx.x == 0) {
            tc::mbar_init(tc::smem_addr(&s_mbar[0]), 1);
            tc::mbar_init(tc::smem_addr(&s_mbar[1]), 1);
            s_abort = 0;
        }
    }
    __syncthreads();
    uint32_t parity = 0;    // bulk: phase parity of each buffer's mbarrier (bit b)
    uint32_t pending = 0;   // bulk, thread 0: buffers with copies issued and not yet consumed

    const int64_t S = blk[m.L];
    const unsigned nblocks = gridDim.x;
    unsigned gen = 0;
    const C* v = reinterpret_cast<const C*>(v_in);
    C* res = reinterpret_cast<C*>(res_out);
    C* ta = reinterpret_cast<C*>(ws.ta);
    C* tb = reinterpret_cast<C*>(ws.tb);
    const R J = R(m.J);
    double c1 = 0.0, c1c2 = 0.0, ratio = 0.0;
    int conv = 0, fin_j = 0;

    for (int j = 0; j < m_star; ++j) {
        const C* src = j == 0 ? v : ((j & 1) ? ta : tb);
        C* dst = (j & 1) ? tb : ta;
        const C* rin = j == 0 ? v : res;
        const double cd = dt / double(j + 1);
        const R c = R(cd);
        double mx[4] = {0.0, 0.0, 0.0, 0.0};  // |term|, |res|, |v|, non-finite
        auto hrow = [&](int64_t r) -> C {
            const uint32_t mm = __ldg(meta + r);
            if constexpr (XHOP) {
                if constexpr (C64) return h_row_c64_x(m, s_sq, r, load_nbr(nbr, r), mm, __ldcg(src + r), src);
                else return h_row_c128_x(m, s_sq, r, load_nbr(nbr, r), mm, __ldcg(src + r), src);
            } else {
                if constexpr (C64) return h_row_c64(m, s_sq, J, r, nbr, mm, src);
                else return h_row_c128(m, s_sq, r, nbr, mm, src);
            }
        };
        auto finish = [&](int64_t r, const C& y, const C& a) {
            C t, rr;
            if constexpr (C64) {
                // separate roundings (no contraction into an FMA): every kernel and schedule that
                // runs these rows -- direct, bulk, batched -- must round them alike
                t = make_float2(__fmul_rn(c, y.y), -__fmul_rn(c, y.x));
                rr = make_float2(__fadd_rn(a.x, t.x), __fadd_rn(a.y, t.y));
                mx[0] = fmax(mx[0], double(fmaf(t.x, t.x, __fmul_rn(t.y, t.y))));
                mx[1] = fmax(mx[1], double(fmaf(rr.x, rr.x, __fmul_rn(rr.y, rr.y))));
                if (j == 0) mx[2] = fmax(mx[2], double(fmaf(a.x, a.x, __fmul_rn(a.y, a.y))));
            } else {
                t = make_double2(__dmul_rn(cd, y.y), -__dmul_rn(cd, y.x));
                rr = make_double2(__dadd_rn(a.x, t.x), __dadd_rn(a.y, t.y));
                mx[0] = fmax(mx[0], fma(t.x, t.x, __dmul_rn(t.y, t.y)));
                mx[1] = fmax(mx[1], fma(rr.x, rr.x, __dmul_rn(rr.y, rr.y)));
                if (j == 0) mx[2] = fmax(mx[2], fma(a.x, a.x, __dmul_rn(a.y, a.y)));
            }
            if (!(isfinite(double(rr.x)) && isfinite(double(rr.y)))) mx[3] = 1.0;
            dst[r] = t;
            res[r] = rr;
        };
        const bool diag = j == 0 && ws.diag != nullptr;  // first sweep: fold the input's diagnostics
        const int wid = threadIdx.x >> 5;
        if constexpr (!BULK) {
            // two rows per thread per pass: all loads of both rows precede the stores
            const int64_t stride = int64_t(gridDim.x) * kTThreads;
            if (!diag) {
                int64_t r = int64_t(blockIdx.x) * kTThreads + threadIdx.x;
                for (; r + stride < S; r += 2 * stride) {
                    const C y0 = hrow(r), y1 = hrow(r + stride);
                    const C a0 = rin[r], a1 = rin[r + stride];
                    finish(r, y0, a0);
                    finish(r + stride, y1, a1);
                }
                if (r < S) finish(r, hrow(r), rin[r]);
            } else {
                // every row once, in 64-row units per warp (rows u + lane and u + 32 + lane, a
                // warp-uniform loop), so that each warp folds its 64-row groups
                const int lane = threadIdx.x & 31;
                const int64_t ustride = int64_t(gridDim.x) * kTWarps * kDiagGroup;
                for (int64_t ub = (int64_t(blockIdx.x) * kTWarps + wid) * kDiagGroup; ub < S; ub += ustride) {
                    const int64_t r0 = ub + lane, r1 = ub + 32 + lane;
                    const bool v0 = r0 < S, v1 = r1 < S;
                    C y0{}, y1{}, a0{}, a1{};
                    if (v0) {
                        y0 = hrow(r0);
                        a0 = rin[r0];
                    }
                    if (v1) {
                        y1 = hrow(r1);
                        a1 = rin[r1];
                    }
                    if (v0) finish(r0, y0, a0);
                    if (v1) finish(r1, y1, a1);
                    diag_group(ws.diag, ub / kDiagGroup, v0, a0, y0, v1, a1, y1);
                }
            }
        } else {
            constexpr uint32_t kCB = chunk_bytes<C64>();
            constexpr uint32_t kOffMeta = kChunk * 16, kOffRin = kOffMeta + kChunk * 4,
                               kOffSelf = kOffRin + kChunk * sizeof(C);
            const int64_t nch = (S + kChunk - 1) / kChunk;
            auto full = [&](int64_t c) { return (c + 1) * kChunk <= S; };
            auto issue = [&](int64_t c, int b) {  // thread 0
                const int64_t r0 = c * kChunk;
                const uint32_t base = tc::smem_addr(t_smem + b * kCB);
                const uint32_t mb = tc::smem_addr(&s_mbar[b]);
                tc::mbar_expect_tx(mb, kCB);
                tc::bulk_g2s(base, nbr + r0 * 4, kChunk * 16, mb);
                tc::bulk_g2s(base + kOffMeta, meta + r0, kChunk * 4, mb);
                tc::bulk_g2s(base + kOffRin, rin + r0, kChunk * sizeof(C), mb);
                tc::bulk_g2s(base + kOffSelf, src + r0, kChunk * sizeof(C), mb);
                pending |= 1u << b;
            };
            int64_t c = blockIdx.x;
            if (threadIdx.x == 0 && c < nch) {
                // the previous term's stores (every block's, ordered by the grid barrier) before
                // this term's bulk reads of them
                tc::fence_proxy_async_global();
                if (full(c)) issue(c, 0);
            }
            for (int k = 0; c < nch; c += gridDim.x, ++k) {
                const int b = k & 1;
                const int64_t cn = c + gridDim.x;
                if (threadIdx.x == 0 && cn < nch && full(cn)) issue(cn, b ^ 1);
                const int64_t r0 = c * kChunk;
                // chunk rows of this thread: t and t + 256, or in the first sweep with the
                // diagnostics 64 w + lane and 64 w + 32 + lane (warp w's 64-row group)
                const int t0 = diag ? kDiagGroup * wid + (threadIdx.x & 31) : threadIdx.x;
                const int t1 = diag ? t0 + 32 : threadIdx.x + kTThreads;
                if (full(c)) {
                    if (!tc::mbar_wait(tc::smem_addr(&s_mbar[b]), (parity >> b) & 1u)) s_abort = 1;
                    parity ^= 1u << b;
                    if (threadIdx.x == 0) pending &= ~(1u << b);
                    const unsigned char* base = t_smem + b * kCB;
                    const int4* snb = reinterpret_cast<const int4*>(base);
                    const uint32_t* smeta = reinterpret_cast<const uint32_t*>(base + kOffMeta);
                    const C* srin = reinterpret_cast<const C*>(base + kOffRin);
                    const C* sself = reinterpret_cast<const C*>(base + kOffSelf);
                    C y0, y1;
                    if constexpr (XHOP) {
                        if constexpr (C64) {
                            y0 = h_row_c64_x(m, s_sq, r0 + t0, snb[t0], smeta[t0], sself[t0], src);
                            y1 = h_row_c64_x(m, s_sq, r0 + t1, snb[t1], smeta[t1], sself[t1], src);
                        } else {
                            y0 = h_row_c128_x(m, s_sq, r0 + t0, snb[t0], smeta[t0], sself[t0], src);
                            y1 = h_row_c128_x(m, s_sq, r0 + t1, snb[t1], smeta[t1], sself[t1], src);
                        }
                    } else if constexpr (C64) {
                        y0 = h_row_c64_nb(m, s_sq, J, r0 + t0, snb[t0], smeta[t0], sself[t0], src);
                        y1 = h_row_c64_nb(m, s_sq, J, r0 + t1, snb[t1], smeta[t1], sself[t1], src);
                    } else {
                        y0 = h_row_c128_nb(m, s_sq, r0 + t0, snb[t0], smeta[t0], sself[t0], src);
                        y1 = h_row_c128_nb(m, s_sq, r0 + t1, snb[t1], smeta[t1], sself[t1], src);
                    }
                    finish(r0 + t0, y0, srin[t0]);
                    finish(r0 + t1, y1, srin[t1]);
                    if (diag) diag_group(ws.diag, r0 / kDiagGroup + wid, true, srin[t0], y0, true, srin[t1], y1);
                } else {
                    // the last, partial chunk: direct loads
                    const bool v0 = r0 + t0 < S, v1 = r0 + t1 < S;
                    C y0{}, y1{}, a0{}, a1{};
                    if (v0) {
                        y0 = hrow(r0 + t0);
                        a0 = rin[r0 + t0];
                        finish(r0 + t0, y0, a0);
                    }
                    if (v1) {
                        y1 = hrow(r0 + t1);
                        a1 = rin[r0 + t1];
                        finish(r0 + t1, y1, a1);
                    }
                    if (diag && r0 + kDiagGroup * wid < S)  // groups with at least one row (warp-uniform)
                        diag_group(ws.diag, r0 / kDiagGroup + wid, v0, a0, y0, v1, a1, y1);
                }
                __syncthreads();  // the buffer is free for the copy issued next iteration
                if (s_abort) break;
            }
            if (s_abort) {
                // a copy that never completed: wait (bounded) for what is still in flight
                if (threadIdx.x == 0)
                    for (int bb = 0; bb < 2; ++bb)
                        if (pending & (1u << bb)) tc::mbar_wait(tc::smem_addr(&s_mbar[bb]), (parity >> bb) & 1u);
                if (threadIdx.x == 0) raise_status(status, PACES_ERR_TIMEOUT);
                fin_j = j;
                break;
            }
        }
        block_max4(mx, s_red, s_fin);
        if (threadIdx.x == 0) {
            double* pp = ws.partials + (size_t((j & 1) * nblocks) + blockIdx.x) * 4;
            pp[0] = s_fin[0];
            pp[1] = s_fin[1];
            pp[2] = s_fin[2];
            pp[3] = s_fin[3];
        }
        if (!grid_barrier(ws.barrier, nblocks, gen, status, ws.wait_ns, int(blockIdx.x) == ws.skip_block)) {
            fin_j = j;
            break;
        }
        double g4[4] = {0.0, 0.0, 0.0, 0.0};
        for (unsigned b = threadIdx.x; b < nblocks; b += kTThreads) {
            const double* pp = ws.partials + (size_t((j & 1) * nblocks) + b) * 4;
#pragma unroll
            for (int k = 0; k < 4; ++k) g4[k] = fmax(g4[k], __ldcg(pp + k));
        }
        block_max4(g4, s_red, s_fin);
        fin_j = j;
        if (s_fin[3] != 0.0) {
            if (blockIdx.x == 0 && threadIdx.x == 0) raise_status(status, PACES_ERR_NONFINITE);
            break;
        }
        // the maxima are of |z|^2; one square root per term gives the inf-norms
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
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (out.converged) *out.converged = conv;
        if (out.final_m) *out.final_m = fin_j;
        if (out.c1_plus_c2) *out.c1_plus_c2 = c1c2;
        if (out.term_ratio) *out.term_ratio = ratio;
    }
}

template <bool C64, bool BULK>
size_t dyn_smem() {
    return BULK ? size_t(2) * chunk_bytes<C64>() : 0;
}

template <bool C64, bool BULK, bool XHOP>
int occupancy() {
    static int cached = 0;  // per process: the kernels' resources do not change
    if (cached) return cached;
    auto kfn = taylor_kernel<C64, BULK, XHOP>;
    if (BULK) cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn_smem<C64, BULK>()));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kTThreads, dyn_smem<C64, BULK>());
    cached = per_sm < 1 ? 1 : (per_sm > 8 ? 8 : per_sm);
    return cached;
}

template <bool C64>
int occupancy_any(int variant, bool xhop) {
    if (xhop) return variant == 1 ? occupancy<C64, true, true>() : occupancy<C64, false, true>();
    return variant == 1 ? occupancy<C64, true, false>() : occupancy<C64, false, false>();
}

template <bool C64, bool BULK, bool XHOP>
cudaError_t launch_one(const cudaLaunchConfig_t& cfg, const ModelDev& m, const int* blk, const int* nbr, int64_t cap,
                       const uint32_t* meta, const void* v_in, void* res, const TaylorWs& ws, double dt, int m_star,
                       double tol, const TaylorOut& out, int* status) {
    if (BULK) {  // the attribute belongs to the current device: set it on every launch
        const cudaError_t a = cudaFuncSetAttribute(taylor_kernel<C64, BULK, XHOP>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   int(dyn_smem<C64, BULK>()));
        if (a != cudaSuccess) return a;
    }
    return cudaLaunchKernelEx(&cfg, taylor_kernel<C64, BULK, XHOP>, m, blk, nbr, cap, meta, v_in, res, ws, dt, m_star,
                              tol, out, status);
}

}  // namespace

int taylor_max_grid(bool c64, int num_sms) {
    int best = 0;
    for (int v = 0; v < 2; ++v)
        for (int x = 0; x < 2; ++x) {
            const int o = c64 ? occupancy_any<true>(v, x != 0) : occupancy_any<false>(v, x != 0);
            best = o > best ? o : best;
        }
    return num_sms * best;
}

int launch_taylor(bool c64, const ModelDev& m, const int* blk, const int* nbr, int64_t nbr_cap,
                  const uint32_t* meta, const void* v_in, void* res, double dt, int m_star,
                  double tol, const TaylorWs& ws, const TaylorOut& out, int* status, int num_sms,
                  int blocks_per_sm, int variant, cudaStream_t st) {
    if (m_star < 1 || variant < 0 || variant > 1) return PACES_ERR_BADARG;
    if (m.nhop > 1 && !m.xnbr) return PACES_ERR_BADARG;
    if (cudaMemsetAsync(ws.barrier, 0, 2 * sizeof(unsigned), st) != cudaSuccess) return PACES_ERR_CUDA;
    const bool xhop = m.nhop > 1;
    const int occ = c64 ? occupancy_any<true>(variant, xhop) : occupancy_any<false>(variant, xhop);
    // a wave of blocks, or one block per 2048 rows of a small problem (fewer blocks at the grid
    // barriers; the results do not depend on the grid)
    const int grid = grid_for(nbr_cap, 2048, num_sms * (blocks_per_sm > 0 && blocks_per_sm < occ ? blocks_per_sm : occ));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kTThreads);
    cfg.dynamicSmemBytes = variant == 1 ? (c64 ? dyn_smem<true, true>() : dyn_smem<false, true>()) : 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int64_t cap = nbr_cap;
    cudaError_t e;
#define PACES_TAYLOR_ONE(C, B, X) launch_one<C, B, X>(cfg, m, blk, nbr, cap, meta, v_in, res, ws, dt, m_star, tol, out, status)
    if (c64) {
        if (xhop) e = variant == 1 ? PACES_TAYLOR_ONE(true, true, true) : PACES_TAYLOR_ONE(true, false, true);
        else e = variant == 1 ? PACES_TAYLOR_ONE(true, true, false) : PACES_TAYLOR_ONE(true, false, false);
    } else {
        if (xhop) e = variant == 1 ? PACES_TAYLOR_ONE(false, true, true) : PACES_TAYLOR_ONE(false, false, true);
        else e = variant == 1 ? PACES_TAYLOR_ONE(false, true, false) : PACES_TAYLOR_ONE(false, false, false);
    }
#undef PACES_TAYLOR_ONE
    return e == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
