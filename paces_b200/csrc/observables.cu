// Norm, energy and per-site observables.
//
// Reference: calculate_n_exc (paces/models/holstein.py:311-314, partitioned sum of
// |psi|^2 by exciton position), calculate_n_pho (holstein.py:317-322 with the CUB
// block-reduce + atomicAdd kernel _holstein_kernels.py:215-255), calculate_total_energy
// (paces/core/observables.py:95-99, <psi|H psi>) and the norms of
// paces/core/time_evolution.py:587, :602, :818.
//
// B200 design: two streaming passes with one full wave of resident blocks each.
//  * energy pass: norm and <psi|H psi> with the neighbour-table SpMV row (gathers);
//  * site pass: norm, n_exc and n_pho from psi, the keys and the row metadata only.
//    Rows are sorted by exciton position, so n_exc is a warp-segmented sum; for keys
//    whose fields all have one width >= 4 bits every thread keeps all per-site sums of
//    its rows in registers (no atomics, no shuffles per row).
// Per-block partials are summed in a fixed order by a final kernel, one block per
// output value: results are deterministic, unlike the reference's float atomics.
#include "hrow.cuh"
#include "kernels.cuh"

namespace paces {

namespace {

constexpr int kOThreads = 256;
constexpr int kOWarps = kOThreads / 32;
constexpr int kFpwMax = 16;  // register fast path: fields of >= 4 bits, at most 16 per word

template <bool C64, bool XHOP>
__global__ void __launch_bounds__(kOThreads, 4)
obs_energy_kernel(ModelDev m, const int* __restrict__ blk, const int* __restrict__ nbr, int64_t cap,
                  const uint32_t* __restrict__ meta, const void* __restrict__ psi, double* __restrict__ part) {
    using C = typename std::conditional<C64, float2, double2>::type;
    using R = typename std::conditional<C64, float, double>::type;
    __shared__ R s_sq[260];
    __shared__ double s_red[kOWarps][3];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < 260; k += kOThreads) s_sq[k] = R(__dmul_rn(sqrt(double(k)), m.g));
    __syncthreads();
    const int64_t S = blk[m.L];
    const C* x = reinterpret_cast<const C*>(psi);
    const R J = R(m.J);
    double norm2 = 0.0, er = 0.0, ei = 0.0;
    auto row = [&](int64_t r) {
        const uint32_t mm = __ldg(meta + r);
        const int4 nb = load_nbr(nbr, r);
        const C z = __ldcg(x + r);
        const double zr = double(z.x), zi = double(z.y);
        double yr, yi;
        if constexpr (C64) {
            const float2 y = XHOP ? h_row_c64_x(m, s_sq, r, nb, mm, z, x) : h_row_c64_nb(m, s_sq, J, r, nb, mm, z, x);
            yr = y.x;
            yi = y.y;
        } else {
            const double2 y = XHOP ? h_row_c128_x(m, s_sq, r, nb, mm, z, x) : h_row_c128_nb(m, s_sq, r, nb, mm, z, x);
            yr = y.x;
            yi = y.y;
        }
        norm2 += zr * zr + zi * zi;
        er += zr * yr + zi * yi;
        ei += zr * yi - zi * yr;
    };
    // four rows a grid stride apart per iteration: their loads are independent and in flight
    // together
    const int64_t gs = int64_t(gridDim.x) * kOThreads;
    int64_t r = int64_t(blockIdx.x) * kOThreads + threadIdx.x;
    for (; r + 3 * gs < S; r += 4 * gs) {
        row(r);
        row(r + gs);
        row(r + 2 * gs);
        row(r + 3 * gs);
    }
    for (; r < S; r += gs) row(r);
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
    __syncthreads();
    if (threadIdx.x < 3) {
        double acc = 0.0;
        for (int w = 0; w < kOWarps; ++w) acc += s_red[w][threadIdx.x];
        part[size_t(blockIdx.x) * 3 + threadIdx.x] = acc;
    }
}

// `uniform`: every field is `ub` bits wide and word q holds sites q*fpw .. q*fpw+fpw-1
// MSB-first (NW <= 4), so thread-private register accumulators cover all sites.  UB = 4
// (the width for occupation cut-offs up to 15) masks each field in place at a constant
// position; UB = 0 reads the width from `ub`.  A field value becomes a double exactly by
// the 2^52 offset (its bits under the exponent of 2^52, minus 2^52): two FP64-pipe
// operations instead of an integer conversion, whose pipe is a quarter as wide.
template <int NW, bool C64, int UB>
__global__ void __launch_bounds__(kOThreads, NW <= 2 ? 2 : 1)
obs_sites_kernel(ModelDev m, const uint64_t* __restrict__ keys, const int* __restrict__ blk,
                 const uint32_t* __restrict__ meta, const void* __restrict__ psi, double* __restrict__ part,
                 int uniform_in, int ub, int fpw) {
    using C = typename std::conditional<C64, float2, double2>::type;
    constexpr bool kFast = NW <= 4;
    constexpr int kAcc = kFast ? NW * kFpwMax : 1;
    __shared__ double s_site[kOWarps][2 * kMaxSites];
    __shared__ double s_red[kOWarps];
    const int L = m.L;
    const int nv = 1 + 2 * L;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const bool uniform = kFast && uniform_in;
    const uint64_t umask = (uint64_t(1) << ub) - 1;
    double racc[kAcc];
#pragma unroll
    for (int i = 0; i < kAcc; ++i) racc[i] = 0.0;
    double pho[4] = {0.0, 0.0, 0.0, 0.0}, exc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = threadIdx.x; k < kOWarps * 2 * kMaxSites; k += kOThreads) (&s_site[0][0])[k] = 0.0;
    __syncthreads();
    const int64_t S = blk[L];
    const C* x = reinterpret_cast<const C*>(psi);
    double norm2 = 0.0;
    int pcur = -1;      // uniform layouts: the warp's current exciton block (warp-uniform)
    double eacc = 0.0;  // and this lane's running sum of |psi|^2 in it
    auto flush_exc = [&]() {  // all lanes of the warp together
        if (pcur < 0) return;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) eacc += __shfl_xor_sync(0xffffffffu, eacc, o);
        if (lane == 0) s_site[wid][pcur] += eacc;
        eacc = 0.0;
        pcur = -1;
    };
    // the loads of the next 32 rows are issued before the current rows are summed (the
    // accumulators hold the occupancy at two blocks per SM, so the memory parallelism has
    // to come from within each thread)
    const int64_t gstride = int64_t(gridDim.x) * kOWarps * 32;
    int64_t base = (int64_t(blockIdx.x) * kOWarps + wid) * 32;
    C zn{};
    uint32_t mn = 0;
    Key<NW> kn;
#pragma unroll
    for (int q = 0; q < NW; ++q) kn.w[q] = 0;
    if (base + lane < S) {
        zn = __ldcs(x + base + lane);
        mn = __ldcs(meta + base + lane);
        kn = load_key<NW>(keys, base + lane);
    }
    for (; base < S; base += gstride) {
        const int64_t r = base + lane;
        const bool valid = r < S;
        const C z = zn;
        const uint32_t mm = valid ? mn : 0u;
        Key<NW> k = kn;
        {
            const int64_t rn = r + gstride;
            if (rn < S) {
                zn = __ldcs(x + rn);
                mn = __ldcs(meta + rn);
                kn = load_key<NW>(keys, rn);
            }
        }
        double w = 0.0;
        if (valid) {
            const double zr = double(z.x), zi = double(z.y);
            w = zr * zr + zi * zi;
        } else {
#pragma unroll
            for (int q = 0; q < NW; ++q) k.w[q] = 0;
        }
        norm2 += w;
        if (uniform) {
            // n_exc: the warp's rows lie in one exciton block or straddle a few; while they stay
            // in the block of the previous rows, each lane keeps adding to its own sum
            const int pme = int(mm & 0xffu);
            const int p0 = __shfl_sync(0xffffffffu, pme, 0);
            const int vlast = __shfl_sync(0xffffffffu, valid ? pme : -1, 31);
            const int p1 = vlast < 0 ? L - 1 : vlast;
            if (p0 == p1 && p0 == pcur) {
                eacc += w;
            } else {
                flush_exc();
                if (p0 == p1) {
                    pcur = p0;
                    eacc = w;
                } else {
                    for (int pp = p0; pp <= p1; ++pp) {
                        double v = (valid && pme == pp) ? w : 0.0;
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                        if (lane == 0) s_site[wid][pp] += v;
                    }
                }
            }
            if (valid && w != 0.0) {
#pragma unroll
                for (int q = 0; q < NW; ++q) {
                    const uint64_t word = k.w[q];
                    const uint32_t whi = uint32_t(word >> 32), wlo = uint32_t(word);
#pragma unroll
                    for (int f = 0; f < kFpwMax; ++f) {
                        if (UB == 4 || f < fpw) {
                            // UB = 4: the field left in place, n * 2^(28 - 4 (f mod 8)) of its
                            // 32-bit half (one AND); the sum is scaled back at the end
                            uint32_t nf;
                            if constexpr (UB == 4) nf = (f < 8 ? whi : wlo) & (15u << (28 - 4 * (f & 7)));
                            else nf = uint32_t((word >> (64 - ub * (f + 1))) & umask);
                            const double dn = __hiloint2double(0x43300000, int(nf)) - 4503599627370496.0;
                            racc[q * kFpwMax + f] = fma(w, dn, racc[q * kFpwMax + f]);
                        }
                    }
                }
            }
        } else {
            // general layout: broadcast each row; lane l owns sites l, l+32, l+64, l+96
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
    flush_exc();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) norm2 += __shfl_xor_sync(0xffffffffu, norm2, o);
    if (lane == 0) s_red[wid] = norm2;
    if (uniform) {
#pragma unroll
        for (int i = 0; i < kAcc; ++i) {
            // UB = 4 sums carry the field's position 2^(28 - 4 (f mod 8)): every product and
            // partial sum is exactly that power of two times the unscaled one (no overflow or
            // underflow at these magnitudes), so the scaled-back sum has the same bits
            double v = UB == 4 ? racc[i] * (1.0 / double(1u << (28 - 4 * ((i % kFpwMax) & 7)))) : racc[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            const int q = i / kFpwMax, f = i % kFpwMax;
            const int s = q * fpw + f;
            if (lane == 0 && f < fpw && s < L) s_site[wid][L + s] = v;
        }
    } else {
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
    double* out = part + size_t(blockIdx.x) * nv;
    for (int v = threadIdx.x; v < nv; v += kOThreads) {
        double acc = 0.0;
        if (v == 0) {
            for (int w2 = 0; w2 < kOWarps; ++w2) acc += s_red[w2];
        } else {
            for (int w2 = 0; w2 < kOWarps; ++w2) acc += s_site[w2][v - 1];
        }
        out[v] = acc;
    }
}

// One block per output value: strided partial sums then a fixed-shape tree (deterministic).
// v = 0 norm, 1-2 energy (energy pass), 3.. n_exc and n_pho (site pass).
__global__ void __launch_bounds__(256) obs_final_kernel(int L, int nb_e, const double* __restrict__ part_e,
                                                        int nb_s, const double* __restrict__ part_s,
                                                        ObsTarget t) {
    __shared__ double s_w[8];
    const int v = blockIdx.x;
    const bool from_e = v < 3 && nb_e > 0;
    const int stride = from_e ? 3 : 1 + 2 * L;
    const int col = from_e ? v : (v == 0 ? 0 : v - 2);
    const int nb = from_e ? nb_e : nb_s;
    const double* part = from_e ? part_e : part_s;
    double acc_t = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) acc_t += part[size_t(b) * stride + col];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc_t += __shfl_xor_sync(0xffffffffu, acc_t, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = acc_t;
    __syncthreads();
    if (threadIdx.x != 0) return;
    double acc = 0.0;
    for (int w = 0; w < 8; ++w) acc += s_w[w];
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

// Diagnostics from a diag buffer (diag_group): block c sums the groups [c kDiagChunk,
// (c+1) kDiagChunk) -- thread t its eight consecutive groups in order, then the warps'
// butterflies and the eight warp sums in order -- into the chunk sums that follow the groups.
__global__ void __launch_bounds__(256) diag_chunk_kernel(const double* __restrict__ groups, double* __restrict__ chunks,
                                                        const int* __restrict__ blk, int L) {
    __shared__ double s_w[8][3];
    const int64_t ng = diag_groups(blk[L]);
    const int64_t c = blockIdx.x;
    if (c * kDiagChunk >= ng) return;
    double v[3] = {0.0, 0.0, 0.0};
    const int64_t g0 = c * kDiagChunk + int64_t(threadIdx.x) * (kDiagChunk / 256);
#pragma unroll
    for (int k = 0; k < kDiagChunk / 256; ++k) {
        const int64_t g = g0 + k;
        if (g < ng) {
#pragma unroll
            for (int q = 0; q < 3; ++q) v[q] = __dadd_rn(v[q], groups[g * 3 + q]);
        }
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] = __dadd_rn(v[q], __shfl_xor_sync(0xffffffffu, v[q], o));
        if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5][q] = v[q];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double acc = 0.0;
        for (int w = 0; w < 8; ++w) acc = __dadd_rn(acc, s_w[w][threadIdx.x]);
        chunks[c * 3 + threadIdx.x] = acc;
    }
}

// The chunk sums in a fixed order -- warp q sums value q: lane l the chunks l, l + 32, ... in
// order, then the butterfly -- into the norm (square root of the sum of |v|^2) and energy.
__global__ void __launch_bounds__(96) diag_final_kernel(const double* __restrict__ chunks, const int* __restrict__ blk,
                                                        int L, ObsTarget t) {
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t nch = (diag_groups(blk[L]) + kDiagChunk - 1) / kDiagChunk;
    double acc = 0.0;
    for (int64_t c = lane; c < nch; c += 32) acc = __dadd_rn(acc, chunks[c * 3 + q]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, o));
    if (lane != 0) return;
    if (q == 0) {
        if (t.norm) *t.norm = sqrt(acc);
    } else if (q == 1) {
        if (t.energy_re) *t.energy_re = acc;
    } else {
        if (t.energy_im) *t.energy_im = acc;
    }
}

// y = H x on every row of the basis (total_ham, paces/core/time_evolution.py:382-400).
template <bool C64>
__global__ void __launch_bounds__(kOThreads) apply_h_kernel(ModelDev m, const int* __restrict__ blk,
                                                            const int* __restrict__ nbr,
                                                            const uint32_t* __restrict__ meta,
                                                            const void* __restrict__ xin, void* __restrict__ yout) {
    using C = typename std::conditional<C64, float2, double2>::type;
    using R = typename std::conditional<C64, float, double>::type;
    __shared__ R s_sq[260];
    for (int k = threadIdx.x; k < 260; k += kOThreads) s_sq[k] = R(__dmul_rn(sqrt(double(k)), m.g));
    __syncthreads();
    const int64_t S = blk[m.L];
    const C* x = reinterpret_cast<const C*>(xin);
    C* y = reinterpret_cast<C*>(yout);
    for (int64_t r = int64_t(blockIdx.x) * kOThreads + threadIdx.x; r < S; r += int64_t(gridDim.x) * kOThreads) {
        const uint32_t mm = __ldg(meta + r);
        if constexpr (C64) y[r] = h_row_c64_any(m, s_sq, float(m.J), r, load_nbr(nbr, r), mm, __ldcg(x + r), x);
        else y[r] = h_row_c128_any(m, s_sq, r, load_nbr(nbr, r), mm, __ldcg(x + r), x);
    }
}

// Per exciton position p: sum over the rows of block p of conj(psi_r) (H_hop psi)_r and of
// conj(psi_r) (H_vib psi)_r -- the partitioned sums behind calculate_hopping and
// calculate_coupling (paces/models/holstein.py:325-364, :380-396; H_hop is the "hopping"
// term, every order-1 channel) -- and the sum of the amplitudes of phonon-vacuum rows
// (calculate_mu_to_0, holstein.py:366-377).  Per-block partials [4L + 2] (hop re, im per
// p, then vib re, im per p, then the vacuum sum), summed in a fixed order afterwards.
template <bool C64>
__global__ void __launch_bounds__(kOThreads) obs_terms_kernel(ModelDev m, const int* __restrict__ blk,
                                                              const int* __restrict__ nbr,
                                                              const uint32_t* __restrict__ meta,
                                                              const void* __restrict__ psi,
                                                              double* __restrict__ part) {
    using C = typename std::conditional<C64, float2, double2>::type;
    using R = typename std::conditional<C64, float, double>::type;
    __shared__ R s_sq[260];
    __shared__ double s_acc[kOWarps][4 * kMaxSites];
    __shared__ double s_vac[kOWarps][2];
    const int L = m.L;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < 260; k += kOThreads) s_sq[k] = R(__dmul_rn(sqrt(double(k)), m.g));
    for (int k = threadIdx.x; k < kOWarps * 4 * kMaxSites; k += kOThreads) (&s_acc[0][0])[k] = 0.0;
    __syncthreads();
    const int64_t S = blk[L];
    const C* x = reinterpret_cast<const C*>(psi);
    double vac_r = 0.0, vac_i = 0.0;
    for (int64_t base = (int64_t(blockIdx.x) * kOWarps + wid) * 32; base < S;
         base += int64_t(gridDim.x) * kOWarps * 32) {
        const int64_t r = base + lane;
        const bool valid = r < S;
        double eh_r = 0.0, eh_i = 0.0, ev_r = 0.0, ev_i = 0.0;
        int pme = -1;
        if (valid) {
            const uint32_t mm = __ldg(meta + r);
            pme = int(mm & 0xffu);
            const int n = int((mm >> 8) & 0xffu);
            const int4 nb = load_nbr(nbr, r);
            const C z = __ldcg(x + r);
            double hr = 0.0, hi = 0.0, vr = 0.0, vi = 0.0;
            if constexpr (C64) {
                float2 h = make_float2(0.f, 0.f), v = make_float2(0.f, 0.f);
                if (m.nhop > 1) {
                    for (int e = 0; e < m.hop_n[0]; ++e) {
                        const int idx = hop_index(m, r, nb, m.hop_ord[0][e]);
                        if (idx < 0) continue;
                        const float2 w = __ldcg(x + idx);
                        h.x = fmaf(float(m.J), w.x, h.x);
                        h.y = fmaf(float(m.J), w.y, h.y);
                    }
                } else {
                    const float J = float(m.J);
                    if (nb.x >= 0) { const float2 w = __ldcg(x + nb.x); h.x = fmaf(J, w.x, h.x); h.y = fmaf(J, w.y, h.y); }
                    if (nb.y >= 0) { const float2 w = __ldcg(x + nb.y); h.x = fmaf(J, w.x, h.x); h.y = fmaf(J, w.y, h.y); }
                }
                if (nb.z >= 0) { const float2 w = __ldcg(x + nb.z); v.x = fmaf(s_sq[n], w.x, v.x); v.y = fmaf(s_sq[n], w.y, v.y); }
                if (nb.w >= 0) { const float2 w = __ldcg(x + nb.w); v.x = fmaf(s_sq[n + 1], w.x, v.x); v.y = fmaf(s_sq[n + 1], w.y, v.y); }
                hr = h.x; hi = h.y; vr = v.x; vi = v.y;
            } else {
                // the rows of the term matrices as the reference sums them (see hrow.cuh)
                double2 h = make_double2(0.0, 0.0);
                if (m.nhop > 1) {
                    bool any = false;
                    for (int e = 0; e < m.hop_n[0]; ++e) {
                        const int idx = hop_index(m, r, nb, m.hop_ord[0][e]);
                        if (idx < 0) continue;
                        const double2 w = __ldcg(x + idx);
                        const double2 pv = make_double2(__dmul_rn(m.J, w.x), __dmul_rn(m.J, w.y));
                        h = any ? make_double2(__dadd_rn(h.x, pv.x), __dadd_rn(h.y, pv.y)) : pv;
                        any = true;
                    }
                } else {
                    const bool swap = nb.y >= 0 && (nb.x < 0 || nb.y < nb.x);
                    const int a = swap ? nb.y : nb.x, b = swap ? nb.x : nb.y;
                    const bool ha = a >= 0, hb = b >= 0;
                    const double2 xa = ha ? __ldcg(x + a) : make_double2(0.0, 0.0);
                    const double2 xb = hb ? __ldcg(x + b) : make_double2(0.0, 0.0);
                    const double2 pa = make_double2(__dmul_rn(m.J, xa.x), __dmul_rn(m.J, xa.y));
                    const double2 pb = make_double2(__dmul_rn(m.J, xb.x), __dmul_rn(m.J, xb.y));
                    h = (ha && hb) ? make_double2(__dadd_rn(pa.x, pb.x), __dadd_rn(pa.y, pb.y))
                                   : (ha ? pa : (hb ? pb : make_double2(0.0, 0.0)));
                }
                const bool hd = nb.z >= 0, hu = nb.w >= 0;
                const double2 xd = hd ? __ldcg(x + nb.z) : make_double2(0.0, 0.0);
                const double2 xu = hu ? __ldcg(x + nb.w) : make_double2(0.0, 0.0);
                const double2 pd = make_double2(__dmul_rn(s_sq[n], xd.x), __dmul_rn(s_sq[n], xd.y));
                const double2 pu = make_double2(__dmul_rn(s_sq[n + 1], xu.x), __dmul_rn(s_sq[n + 1], xu.y));
                const double2 v = (hd && hu) ? make_double2(__dadd_rn(pd.x, pu.x), __dadd_rn(pd.y, pu.y))
                                             : (hd ? pd : (hu ? pu : make_double2(0.0, 0.0)));
                hr = h.x; hi = h.y; vr = v.x; vi = v.y;
            }
            const double zr = double(z.x), zi = double(z.y);
            // conj(z) * y
            eh_r = __dadd_rn(__dmul_rn(zr, hr), __dmul_rn(zi, hi));
            eh_i = __dsub_rn(__dmul_rn(zr, hi), __dmul_rn(zi, hr));
            ev_r = __dadd_rn(__dmul_rn(zr, vr), __dmul_rn(zi, vi));
            ev_i = __dsub_rn(__dmul_rn(zr, vi), __dmul_rn(zi, vr));
            if ((mm >> 16) == 0) {
                vac_r += zr;
                vac_i += zi;
            }
        }
        // the warp's rows span consecutive exciton blocks: segmented sums per block
        const int p0 = __shfl_sync(0xffffffffu, pme, 0);
        const int vlast = __shfl_sync(0xffffffffu, pme, 31);
        const int p1 = vlast < 0 ? L - 1 : vlast;
        for (int pp = p0; pp <= p1 && pp >= 0; ++pp) {
            double a0 = pme == pp ? eh_r : 0.0, a1 = pme == pp ? eh_i : 0.0;
            double a2 = pme == pp ? ev_r : 0.0, a3 = pme == pp ? ev_i : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                a0 += __shfl_xor_sync(0xffffffffu, a0, o);
                a1 += __shfl_xor_sync(0xffffffffu, a1, o);
                a2 += __shfl_xor_sync(0xffffffffu, a2, o);
                a3 += __shfl_xor_sync(0xffffffffu, a3, o);
            }
            if (lane == 0) {
                s_acc[wid][pp] += a0;
                s_acc[wid][L + pp] += a1;
                s_acc[wid][2 * L + pp] += a2;
                s_acc[wid][3 * L + pp] += a3;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        vac_r += __shfl_xor_sync(0xffffffffu, vac_r, o);
        vac_i += __shfl_xor_sync(0xffffffffu, vac_i, o);
    }
    if (lane == 0) {
        s_vac[wid][0] = vac_r;
        s_vac[wid][1] = vac_i;
    }
    __syncthreads();
    const int nv = 4 * L + 2;
    double* out = part + size_t(blockIdx.x) * nv;
    for (int v = threadIdx.x; v < nv; v += kOThreads) {
        double acc = 0.0;
        for (int w = 0; w < kOWarps; ++w) acc += v < 4 * L ? s_acc[w][v] : s_vac[w][v - 4 * L];
        out[v] = acc;
    }
}

// out[v] = sum over blocks of part[b][v], one block per value, fixed order.
__global__ void __launch_bounds__(256) terms_final_kernel(int nv, int nb, const double* __restrict__ part,
                                                          double* __restrict__ out) {
    __shared__ double s_w[8];
    const int v = blockIdx.x;
    double acc = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) acc += part[size_t(b) * nv + v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += s_w[w];
        out[v] = t;
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

template <typename K>
int wave_blocks(K kernel, int num_sms) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kOThreads, 0);
    per_sm = per_sm < 1 ? 1 : (per_sm > kObsGridPerSm ? kObsGridPerSm : per_sm);
    return num_sms * per_sm;
}

// The observables' grids stay a full wave whatever the problem size: the partial sums are
// summed per block, so the grid sets the order of the additions, and results must not
// change when a trajectory's buffers grow.
template <int NW, bool C64>
int launch_obs_t(const ModelDev& m, const uint64_t* keys, const int* blk, const int* nbr,
                 int64_t nbr_cap, const uint32_t* meta, const void* psi, int what, double* partials,
                 const ObsTarget& out, int num_sms, cudaStream_t st) {
    static int grid_e = 0, grid_ex = 0, grid_s = 0, grid_s4 = 0;
    if (grid_e == 0) {
        grid_e = wave_blocks(obs_energy_kernel<C64, false>, num_sms);
        grid_ex = wave_blocks(obs_energy_kernel<C64, true>, num_sms);
        grid_s = wave_blocks(obs_sites_kernel<NW, C64, 0>, num_sms);
        if constexpr (NW <= 4) grid_s4 = wave_blocks(obs_sites_kernel<NW, C64, 4>, num_sms);
    }
    const bool energy = (what & PACES_OBS_ENERGY) != 0;
    const bool sites = (what & PACES_OBS_SITES) != 0;
    double* part_e = partials;
    double* part_s = partials + size_t(obs_max_grid(num_sms)) * 3;
    int nb_e = 0, nb_s = 0;
    if (energy || !sites) {
        if (m.nhop > 1) {
            obs_energy_kernel<C64, true><<<grid_ex, kOThreads, 0, st>>>(m, blk, nbr, nbr_cap, meta, psi, part_e);
            nb_e = grid_ex;
        } else {
            obs_energy_kernel<C64, false><<<grid_e, kOThreads, 0, st>>>(m, blk, nbr, nbr_cap, meta, psi, part_e);
            nb_e = grid_e;
        }
    }
    if (sites) {
        int ub = m.bits[0];
        const int fpw = ub > 0 ? 64 / ub : 0;
        bool uniform = ub >= 4 && NW <= 4;
        for (int s = 0; s < m.L && uniform; ++s)
            uniform = m.bits[s] == ub && m.word[s] == s / fpw && m.shift[s] == 64 - ub * (s % fpw + 1);
        bool done = false;
        if constexpr (NW <= 4) {
            if (uniform && ub == 4) {
                obs_sites_kernel<NW, C64, 4><<<grid_s4, kOThreads, 0, st>>>(m, keys, blk, meta, psi, part_s, 1, ub, fpw);
                nb_s = grid_s4;
                done = true;
            }
        }
        if (!done) {
            obs_sites_kernel<NW, C64, 0><<<grid_s, kOThreads, 0, st>>>(m, keys, blk, meta, psi, part_s,
                                                                      uniform ? 1 : 0, ub, fpw);
            nb_s = grid_s;
        }
    }
    obs_final_kernel<<<sites ? 3 + 2 * m.L : 3, 256, 0, st>>>(m.L, nb_e, part_e, nb_s, part_s, out);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace

int launch_diag_final(const double* diag, const int* blk, int L, int64_t cap, const ObsTarget& out, cudaStream_t st) {
    if (!diag || cap < 0) return PACES_ERR_BADARG;
    double* chunks = const_cast<double*>(diag) + diag_groups(cap) * 3;
    const int64_t nch = diag_chunks(cap);
    diag_chunk_kernel<<<unsigned(nch > 0 ? nch : 1), 256, 0, st>>>(diag, chunks, blk, L);
    diag_final_kernel<<<1, 96, 0, st>>>(chunks, blk, L, out);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

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

int launch_term_energies(bool c64, const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta,
                         const void* psi, double* partials, double* out, int num_sms, cudaStream_t st) {
    const int grid = num_sms * 2;  // the partials hold obs_max_grid * (4 + 2L) doubles
    if (c64) obs_terms_kernel<true><<<grid, kOThreads, 0, st>>>(m, blk, nbr, meta, psi, partials);
    else obs_terms_kernel<false><<<grid, kOThreads, 0, st>>>(m, blk, nbr, meta, psi, partials);
    terms_final_kernel<<<4 * m.L + 2, 256, 0, st>>>(4 * m.L + 2, grid, partials, out);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

int launch_apply_h(bool c64, const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta,
                   const void* x, void* y, int num_sms, cudaStream_t st) {
    if (c64) apply_h_kernel<true><<<num_sms * 4, kOThreads, 0, st>>>(m, blk, nbr, meta, x, y);
    else apply_h_kernel<false><<<num_sms * 4, kOThreads, 0, st>>>(m, blk, nbr, meta, x, y);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

int launch_scale(bool c64, const ModelDev& m, const int* blk, void* psi, const double* norm,
                 int num_sms, cudaStream_t st) {
    if (c64) scale_kernel<true><<<num_sms * 4, 256, 0, st>>>(m.L, blk, psi, norm);
    else scale_kernel<false><<<num_sms * 4, 256, 0, st>>>(m.L, blk, psi, norm);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
