// Batched truncated-Taylor series: many independent trajectories (each its own basis, H,
// dt, model constants and stop test) advance through exp(-i dt H) psi in ONE persistent
// cooperative launch.
//
// Reference: _simple_taylor (paces/core/time_evolution.py:482-512) with total_ham
// (:382-400), run once per trajectory; the reference has no batching.
//
// Design.  The rows of all trajectories form one index space (trajectory t owns rows
// [off[t], off[t] + rows_t), off computed on the device from every basis' blk[L] rounded up
// to a multiple of the 64-row unit, so the host never reads a size and no unit straddles two
// trajectories).  Each term is one sweep over that space in warp units of 64 rows (two per
// lane, all loads before the stores), assigned grid-stride so the rows of the trajectories
// still running are spread over every SM.  Lanes keep running maxima of |term|^2, |res|^2,
// |v|^2 and a non-finite flag for the warp's current trajectory and fold them into shared
// memory only when the trajectory changes.  Rows 64 u + l and 64 u + 32 + l of a trajectory
// sit on lane l of its unit, as in the single-trajectory kernel's 64-row groups, so the first
// sweep folds the input's diagnostics (diag_group) exactly as that kernel does.  Blocks then fold into
// per-trajectory global maxima with
// atomicMax on the fp64 bit patterns (non-negative doubles order like their bits), which
// is exact and order-independent, so each trajectory's stop decision -- taken by every
// block from the same global maxima -- and its arithmetic are bit-identical to the
// single-trajectory kernel.  Three rotating maxima buffers let block 0 clear the one for
// term j+2 after barrier j without racing the writers of term j+1.  A trajectory that
// converges, overflows or reaches its m_star leaves the sweep; the launch ends when none
// is left.
#include "grid.cuh"
#include "hrow.cuh"
#include "kernels.cuh"

namespace paces {

namespace {

constexpr int kBThreads = 256;
constexpr int kBWarps = kBThreads / 32;
constexpr int kUnit = 64;

__device__ __forceinline__ unsigned long long dbits(double x) {
    return static_cast<unsigned long long>(__double_as_longlong(x));
}

template <bool C64>
__global__ void __launch_bounds__(kBThreads, C64 ? 4 : 3)
taylor_batch_kernel(const __grid_constant__ TaylorBatch bt, TaylorBatchWs ws) {
    using C = typename std::conditional<C64, float2, double2>::type;
    using R = typename std::conditional<C64, float, double>::type;
    __shared__ long long s_off[kMaxBatch + 1];
    __shared__ long long s_rows[kMaxBatch];
    __shared__ unsigned long long s_max[kMaxBatch][4];
    __shared__ double s_c1[kMaxBatch], s_c1c2[kMaxBatch], s_ratio[kMaxBatch], s_cd[kMaxBatch];
    __shared__ int s_active[kMaxBatch];
    __shared__ int s_left;

    const int n = bt.n;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int i = tid; i < n; i += kBThreads) {
        const TaylorItem& I = bt.items[i];
        s_rows[i] = I.blk[I.L];
        s_off[i + 1] = (s_rows[i] + kUnit - 1) / kUnit * kUnit;
        s_active[i] = 1;
        s_c1[i] = s_c1c2[i] = s_ratio[i] = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) s_max[i][k] = 0ull;
    }
    __syncthreads();
    if (tid == 0) {
        s_off[0] = 0;
        for (int i = 0; i < n; ++i) s_off[i + 1] += s_off[i];
    }
    __syncthreads();
    const long long rows = s_off[n];
    const long long units = (rows + kUnit - 1) / kUnit;
    const long long gwarp = (long long)blockIdx.x * kBWarps + wid;
    const long long nwarps = (long long)gridDim.x * kBWarps;
    const unsigned nblocks = gridDim.x;
    unsigned gen = 0;

    auto emit = [&](int i, int j, int conv, int fin_j) {
        const TaylorOut& o = bt.items[i].out;
        if (o.converged) *o.converged = conv;
        if (o.final_m) *o.final_m = fin_j;
        if (o.c1_plus_c2) *o.c1_plus_c2 = s_c1c2[i];
        if (o.term_ratio) *o.term_ratio = s_ratio[i];
        (void)j;
    };

    for (int j = 0; j < bt.max_m_star; ++j) {
        for (int i = tid; i < n; i += kBThreads) s_cd[i] = bt.items[i].dt / double(j + 1);
        __syncthreads();
        const bool first = j == 0;

        // one row: y = H src, term t = -i cd y, res = rin + t; maxima into mx
        auto load_row = [&](const TaylorItem& I, long long l, C& y, C& a) {
            const C* src = reinterpret_cast<const C*>(first ? I.v_in : ((j & 1) ? I.ta : I.tb));
            const C* rin = reinterpret_cast<const C*>(first ? I.v_in : I.res);
            const uint32_t mm = __ldg(I.meta + l);
            if constexpr (C64) y = h_row_c64(I, I.sqf, R(I.J), l, I.nbr, mm, src);
            else y = h_row_c128(I, I.sq, l, I.nbr, mm, src);
            a = rin[l];
        };
        auto finish_row = [&](const TaylorItem& I, double cd, long long l, const C& y, const C& a, double mx[4]) {
            C* dst = reinterpret_cast<C*>((j & 1) ? I.tb : I.ta);
            C* res = reinterpret_cast<C*>(I.res);
            C t, rr;
            if constexpr (C64) {
                const R c = R(cd);
                // separate roundings, as the single-trajectory kernel (no contraction into an FMA)
                t = make_float2(__fmul_rn(c, y.y), -__fmul_rn(c, y.x));
                rr = make_float2(__fadd_rn(a.x, t.x), __fadd_rn(a.y, t.y));
                mx[0] = fmax(mx[0], double(fmaf(t.x, t.x, __fmul_rn(t.y, t.y))));
                mx[1] = fmax(mx[1], double(fmaf(rr.x, rr.x, __fmul_rn(rr.y, rr.y))));
                if (first) mx[2] = fmax(mx[2], double(fmaf(a.x, a.x, __fmul_rn(a.y, a.y))));
            } else {
                t = make_double2(__dmul_rn(cd, y.y), -__dmul_rn(cd, y.x));
                rr = make_double2(__dadd_rn(a.x, t.x), __dadd_rn(a.y, t.y));
                mx[0] = fmax(mx[0], fma(t.x, t.x, __dmul_rn(t.y, t.y)));
                mx[1] = fmax(mx[1], fma(rr.x, rr.x, __dmul_rn(rr.y, rr.y)));
                if (first) mx[2] = fmax(mx[2], fma(a.x, a.x, __dmul_rn(a.y, a.y)));
            }
            if (!(isfinite(double(rr.x)) && isfinite(double(rr.y)))) mx[3] = 1.0;
            dst[l] = t;
            res[l] = rr;
        };

        int cur = -1;             // warp-uniform: trajectory whose maxima cm[] holds
        double cm[4] = {0.0, 0.0, 0.0, 0.0};
        auto flush = [&]() {      // all lanes of the warp call this together
            if (cur < 0) return;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) cm[k] = fmax(cm[k], __shfl_xor_sync(0xffffffffu, cm[k], o));
                if (lane == 0 && cm[k] > 0.0) atomicMax(&s_max[cur][k], dbits(cm[k]));
                cm[k] = 0.0;
            }
        };
        int it = 0;
        for (long long u = gwarp; u < units; u += nwarps) {
            const long long base = u * kUnit;
            while (s_off[it + 1] <= base) ++it;
            // the whole unit is rows (or padding) of trajectory `it`
            if (!s_active[it]) continue;
            if (it != cur) {
                flush();
                cur = it;
            }
            const TaylorItem& I = bt.items[it];
            const double cd = s_cd[it];
            const long long l0 = base - s_off[it] + lane, l1 = l0 + 32;
            const long long nr = s_rows[it];
            if (first && I.diag) {
                // the first sweep with the diagnostics: the unit is one 64-row group (it holds at
                // least one row, since the padding is shorter than a unit)
                const bool v0 = l0 < nr, v1 = l1 < nr;
                C y0{}, a0{}, y1{}, a1{};
                if (v0) load_row(I, l0, y0, a0);
                if (v1) load_row(I, l1, y1, a1);
                diag_group(I.diag, (base - s_off[it]) / kDiagGroup, v0, a0, y0, v1, a1, y1);
                if (v0) finish_row(I, cd, l0, y0, a0, cm);
                if (v1) finish_row(I, cd, l1, y1, a1, cm);
            } else if (l1 < nr) {
                C y0, a0, y1, a1;
                load_row(I, l0, y0, a0);
                load_row(I, l1, y1, a1);
                finish_row(I, cd, l0, y0, a0, cm);
                finish_row(I, cd, l1, y1, a1, cm);
            } else if (l0 < nr) {
                C y0, a0;
                load_row(I, l0, y0, a0);
                finish_row(I, cd, l0, y0, a0, cm);
            }
        }
        flush();
        __syncthreads();
        unsigned long long* gmax = ws.maxima + size_t(j % 3) * kMaxBatch * 4;
        for (int e = tid; e < n * 4; e += kBThreads) {
            const unsigned long long v = s_max[e >> 2][e & 3];
            if (v) atomicMax(&gmax[e], v);
            s_max[e >> 2][e & 3] = 0ull;
        }
        if (!grid_barrier(ws.barrier, nblocks, gen, nullptr, ws.wait_ns, int(blockIdx.x) == ws.skip_block)) {
            for (int i = tid; i < n; i += kBThreads) {
                if (!s_active[i]) continue;
                raise_status(bt.items[i].status, PACES_ERR_TIMEOUT);
                if (blockIdx.x == 0) emit(i, j, 0, j);
                s_active[i] = 0;
            }
            break;
        }
        // every block takes the same per-trajectory decisions from the same maxima
        for (int i = tid; i < n; i += kBThreads) {
            if (!s_active[i]) continue;
            double g4[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) g4[k] = __longlong_as_double((long long)__ldcg(&gmax[i * 4 + k]));
            const TaylorItem& I = bt.items[i];
            if (g4[3] != 0.0) {
                if (blockIdx.x == 0) {
                    raise_status(I.status, PACES_ERR_NONFINITE);
                    emit(i, j, 0, j);
                }
                s_active[i] = 0;
                continue;
            }
            if (first) s_c1[i] = sqrt(g4[2]);
            const double c2 = sqrt(g4[0]);
            s_c1c2[i] = s_c1[i] + c2;
            s_ratio[i] = s_c1c2[i] / sqrt(g4[1]);
            if (s_ratio[i] <= I.tol) {
                if (blockIdx.x == 0) emit(i, j, 1, j);
                s_active[i] = 0;
                continue;
            }
            s_c1[i] = c2;
            if (j + 1 >= I.m_star) {
                if (blockIdx.x == 0) emit(i, j, 0, j);
                s_active[i] = 0;
            }
        }
        if (blockIdx.x == 0) {
            unsigned long long* clr = ws.maxima + size_t((j + 2) % 3) * kMaxBatch * 4;
            for (int e = tid; e < n * 4; e += kBThreads) clr[e] = 0ull;
        }
        if (tid == 0) s_left = 0;
        __syncthreads();
        for (int i = tid; i < n; i += kBThreads)
            if (s_active[i]) atomicAdd(&s_left, 1);
        __syncthreads();
        if (s_left == 0) break;
    }
}

template <bool C64>
int batch_occupancy() {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, taylor_batch_kernel<C64>, kBThreads, 0);
    return per_sm < 1 ? 1 : (per_sm > 8 ? 8 : per_sm);
}

}  // namespace

int taylor_batch_max_grid(bool c64, int num_sms) {
    return num_sms * (c64 ? batch_occupancy<true>() : batch_occupancy<false>());
}

int launch_taylor_batch(bool c64, const TaylorBatch& bt, const TaylorBatchWs& ws, int num_sms, int blocks_per_sm,
                        cudaStream_t st) {
    if (bt.n < 1 || bt.n > kMaxBatch || bt.max_m_star < 1) return PACES_ERR_BADARG;
    if (cudaMemsetAsync(ws.barrier, 0, kTaylorBatchWsBytes, st) != cudaSuccess) return PACES_ERR_CUDA;
    cudaLaunchConfig_t cfg = {};
    const int occ = c64 ? batch_occupancy<true>() : batch_occupancy<false>();
    cfg.gridDim = dim3(num_sms * (blocks_per_sm > 0 && blocks_per_sm < occ ? blocks_per_sm : occ));
    cfg.blockDim = dim3(kBThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = c64 ? cudaLaunchKernelEx(&cfg, taylor_batch_kernel<true>, bt, ws)
                        : cudaLaunchKernelEx(&cfg, taylor_batch_kernel<false>, bt, ws);
    return e == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
