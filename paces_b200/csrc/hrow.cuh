// One row of H applied to a vector, from the neighbour table (one int4 per row: left,
// right, one phonon less, one phonon more; -1 = absent) and the row metadata.
//
// Reference: total_ham (paces/core/time_evolution.py:382-400) computes
//   diag * v + hopping_csr.dot(v) + vib_coupling_csr.dot(v)
// with CSR rows summed in increasing column order and float64 matrix elements
// J (hopping, paces/models/holstein.py:205-206) and g*sqrt(n) (vibronic coupling,
// holstein.py:271-274).  The complex128 form below keeps exactly that grouping and
// rounds every product and sum separately (no fused multiply-add), so it reproduces
// the reference arithmetic row by row.
//
// The rows are branch-free: every neighbour load is issued (an absent neighbour re-reads
// the row's own element, already in flight, and its term is discarded by a select), so
// the five loads of a row -- and of several rows handled by one thread -- are in flight
// together without funnelling the absent ones onto one hot cache line.
#pragma once

#include "common.cuh"

namespace paces {

// Diagonal element from the row metadata (paces/models/holstein.py:280-287).  `P` is the
// model (ModelDev) or a batched trajectory's parameters: any type with eps_sys,
// hbar_omega, delta_eps, has_site_eps, site_eps[] and J.
template <class P>
__device__ __forceinline__ double diag_value(const P& m, uint32_t meta) {
    const int pos = int(meta & 0xffu);
    const uint32_t ntot = meta >> 16;
    double d = __dadd_rn(m.eps_sys, __dmul_rn(m.hbar_omega, double(ntot)));
    if (m.delta_eps != 0.0) d = __dadd_rn(d, __dmul_rn(m.delta_eps, double(pos)));
    if (m.has_site_eps) d = __dadd_rn(d, m.site_eps[pos]);
    return d;
}

__device__ __forceinline__ int4 load_nbr(const int* __restrict__ nbr, int64_t r) {
    return __ldg(reinterpret_cast<const int4*>(nbr) + r);
}

// y = (H x)[r] in complex128 from the row's neighbour entry nb and its own element xr.
// sq[k] = sqrt(k) * g.
template <class P>
__device__ __forceinline__ double2 h_row_c128_nb(const P& m, const double* sq, int64_t r, int4 nb, uint32_t meta,
                                                 double2 xr, const double2* __restrict__ x) {
    const int n = int((meta >> 8) & 0xffu);
    // hopping columns in increasing order (a <= b), as the CSR row sum visits them
    const bool swap = nb.y >= 0 && (nb.x < 0 || nb.y < nb.x);
    const int a = swap ? nb.y : nb.x, b = swap ? nb.x : nb.y;
    const bool ha = a >= 0, hb = b >= 0, hd = nb.z >= 0, hu = nb.w >= 0;
    const double2 xa = __ldcg(x + (ha ? a : r));
    const double2 xb = __ldcg(x + (hb ? b : r));
    const double2 xd = __ldcg(x + (hd ? nb.z : r));
    const double2 xu = __ldcg(x + (hu ? nb.w : r));
    const double d = diag_value(m, meta);
    double2 y = make_double2(__dmul_rn(d, xr.x), __dmul_rn(d, xr.y));
    // hopping: (J xa) + (J xb), terms present only
    const double2 pa = make_double2(__dmul_rn(m.J, xa.x), __dmul_rn(m.J, xa.y));
    const double2 pb = make_double2(__dmul_rn(m.J, xb.x), __dmul_rn(m.J, xb.y));
    const double2 hs = (ha && hb) ? make_double2(__dadd_rn(pa.x, pb.x), __dadd_rn(pa.y, pb.y)) : (ha ? pa : pb);
    if (ha || hb) y = make_double2(__dadd_rn(y.x, hs.x), __dadd_rn(y.y, hs.y));
    // vibronic: (g sqrt(n) xd) + (g sqrt(n+1) xu); one phonon less sorts first
    const double cd = sq[n], cu = sq[n + 1];
    const double2 pd = make_double2(__dmul_rn(cd, xd.x), __dmul_rn(cd, xd.y));
    const double2 pu = make_double2(__dmul_rn(cu, xu.x), __dmul_rn(cu, xu.y));
    const double2 vs = (hd && hu) ? make_double2(__dadd_rn(pd.x, pu.x), __dadd_rn(pd.y, pu.y)) : (hd ? pd : pu);
    if (hd || hu) y = make_double2(__dadd_rn(y.x, vs.x), __dadd_rn(y.y, vs.y));
    return y;
}

template <class P>
__device__ __forceinline__ double2 h_row_c128(const P& m, const double* sq, int64_t r,
                                              const int* __restrict__ nbr, uint32_t meta,
                                              const double2* __restrict__ x) {
    return h_row_c128_nb(m, sq, r, load_nbr(nbr, r), meta, __ldcg(x + r), x);
}

// y = (H x)[r] in complex64 with fp32 accumulation.  sq[k] = float(sqrt(k) * g).
template <class P>
__device__ __forceinline__ float2 h_row_c64_nb(const P& m, const float* sq, float J, int64_t r, int4 nb,
                                               uint32_t meta, float2 xr, const float2* __restrict__ x) {
    const int n = int((meta >> 8) & 0xffu);
    const float2 xa = __ldcg(x + (nb.x >= 0 ? nb.x : r));
    const float2 xb = __ldcg(x + (nb.y >= 0 ? nb.y : r));
    const float2 xd = __ldcg(x + (nb.z >= 0 ? nb.z : r));
    const float2 xu = __ldcg(x + (nb.w >= 0 ? nb.w : r));
    const float d = float(diag_value(m, meta));
    const float ja = nb.x >= 0 ? J : 0.f, jb = nb.y >= 0 ? J : 0.f;
    const float cd = nb.z >= 0 ? sq[n] : 0.f, cu = nb.w >= 0 ? sq[n + 1] : 0.f;
    float2 y = make_float2(__fmul_rn(d, xr.x), __fmul_rn(d, xr.y));
    y.x = fmaf(ja, xa.x, y.x);
    y.y = fmaf(ja, xa.y, y.y);
    y.x = fmaf(jb, xb.x, y.x);
    y.y = fmaf(jb, xb.y, y.y);
    y.x = fmaf(cd, xd.x, y.x);
    y.y = fmaf(cd, xd.y, y.y);
    y.x = fmaf(cu, xu.x, y.x);
    y.y = fmaf(cu, xu.y, y.y);
    return y;
}

template <class P>
__device__ __forceinline__ float2 h_row_c64(const P& m, const float* sq, float J, int64_t r,
                                            const int* __restrict__ nbr, uint32_t meta,
                                            const float2* __restrict__ x) {
    return h_row_c64_nb(m, sq, J, r, load_nbr(nbr, r), meta, __ldcg(x + r), x);
}

// ---- lattices with several hopping channels (ModelDev::nhop > 1) ---------------------------
// The reference sums H x term by term -- diag * x, then the "hopping" CSR row, then the
// "hopping2" row, then the vibronic row (paces/core/time_evolution.py:382-400, the terms in
// the order of use_terms) -- and each CSR row in increasing column order, which for open
// boundaries is increasing exciton position (hop_ord).  Channel 0 lives in the int4 row
// (left = lower, right = upper), channels 1.. in m.xnbr.

__device__ __forceinline__ int hop_index(const ModelDev& m, int64_t r, int4 nb, int code) {
    const int ch = code >> 1, up = code & 1;
    if (ch == 0) return up ? nb.y : nb.x;
    const int2 e = __ldg(m.xnbr + int64_t(ch - 1) * m.xcap + r);
    return up ? e.y : e.x;
}

__device__ __forceinline__ double2 h_row_c128_x(const ModelDev& m, const double* sq, int64_t r, int4 nb, uint32_t meta,
                                                double2 xr, const double2* __restrict__ x) {
    const int n = int((meta >> 8) & 0xffu);
    const double d = diag_value(m, meta);
    double2 y = make_double2(__dmul_rn(d, xr.x), __dmul_rn(d, xr.y));
    for (int t = 0; t < 2; ++t) {
        const double Jt = t == 0 ? m.J : m.J2;
        double2 hs = make_double2(0.0, 0.0);
        bool any = false;
        for (int e = 0; e < m.hop_n[t]; ++e) {
            const int idx = hop_index(m, r, nb, m.hop_ord[t][e]);
            if (idx < 0) continue;
            const double2 v = __ldcg(x + idx);
            const double2 pv = make_double2(__dmul_rn(Jt, v.x), __dmul_rn(Jt, v.y));
            hs = any ? make_double2(__dadd_rn(hs.x, pv.x), __dadd_rn(hs.y, pv.y)) : pv;
            any = true;
        }
        if (any) y = make_double2(__dadd_rn(y.x, hs.x), __dadd_rn(y.y, hs.y));
    }
    const bool hd = nb.z >= 0, hu = nb.w >= 0;
    const double2 xd = __ldcg(x + (hd ? nb.z : r));
    const double2 xu = __ldcg(x + (hu ? nb.w : r));
    const double cd = sq[n], cu = sq[n + 1];
    const double2 pd = make_double2(__dmul_rn(cd, xd.x), __dmul_rn(cd, xd.y));
    const double2 pu = make_double2(__dmul_rn(cu, xu.x), __dmul_rn(cu, xu.y));
    const double2 vs = (hd && hu) ? make_double2(__dadd_rn(pd.x, pu.x), __dadd_rn(pd.y, pu.y)) : (hd ? pd : pu);
    if (hd || hu) y = make_double2(__dadd_rn(y.x, vs.x), __dadd_rn(y.y, vs.y));
    return y;
}

__device__ __forceinline__ float2 h_row_c64_x(const ModelDev& m, const float* sq, int64_t r, int4 nb, uint32_t meta,
                                              float2 xr, const float2* __restrict__ x) {
    const int n = int((meta >> 8) & 0xffu);
    const float d = float(diag_value(m, meta));
    float2 y = make_float2(__fmul_rn(d, xr.x), __fmul_rn(d, xr.y));
    for (int t = 0; t < 2; ++t) {
        const float Jt = float(t == 0 ? m.J : m.J2);
        for (int e = 0; e < m.hop_n[t]; ++e) {
            const int idx = hop_index(m, r, nb, m.hop_ord[t][e]);
            if (idx < 0) continue;
            const float2 v = __ldcg(x + idx);
            y.x = fmaf(Jt, v.x, y.x);
            y.y = fmaf(Jt, v.y, y.y);
        }
    }
    const float2 xd = __ldcg(x + (nb.z >= 0 ? nb.z : r));
    const float2 xu = __ldcg(x + (nb.w >= 0 ? nb.w : r));
    const float cd = nb.z >= 0 ? sq[n] : 0.f, cu = nb.w >= 0 ? sq[n + 1] : 0.f;
    y.x = fmaf(cd, xd.x, y.x);
    y.y = fmaf(cd, xd.y, y.y);
    y.x = fmaf(cu, xu.x, y.x);
    y.y = fmaf(cu, xu.y, y.y);
    return y;
}

// One row of H x for either model: the chain's fixed form, or the channel loop.
__device__ __forceinline__ double2 h_row_c128_any(const ModelDev& m, const double* sq, int64_t r, int4 nb,
                                                  uint32_t meta, double2 xr, const double2* __restrict__ x) {
    return m.nhop > 1 ? h_row_c128_x(m, sq, r, nb, meta, xr, x) : h_row_c128_nb(m, sq, r, nb, meta, xr, x);
}
__device__ __forceinline__ float2 h_row_c64_any(const ModelDev& m, const float* sq, float J, int64_t r, int4 nb,
                                                uint32_t meta, float2 xr, const float2* __restrict__ x) {
    return m.nhop > 1 ? h_row_c64_x(m, sq, r, nb, meta, xr, x) : h_row_c64_nb(m, sq, J, r, nb, meta, xr, x);
}

// H 1 of one row: diag + the row sums term by term (total_ham_ones,
// paces/core/time_evolution.py:403-420), in the order h_row_c128_x sums H x.
__device__ __forceinline__ double h_ones_row_any(const ModelDev& m, const double* sq, int64_t r, int4 nb,
                                                 uint32_t meta) {
    const int n = int((meta >> 8) & 0xffu);
    double h = diag_value(m, meta);
    if (m.nhop > 1) {
        for (int t = 0; t < 2; ++t) {
            const double Jt = t == 0 ? m.J : m.J2;
            double hs = 0.0;
            bool any = false;
            for (int e = 0; e < m.hop_n[t]; ++e) {
                if (hop_index(m, r, nb, m.hop_ord[t][e]) < 0) continue;
                hs = any ? __dadd_rn(hs, Jt) : Jt;
                any = true;
            }
            if (any) h = __dadd_rn(h, hs);
        }
    } else {
        const bool ha = nb.x >= 0, hb = nb.y >= 0;
        if (ha || hb) h = __dadd_rn(h, (ha && hb) ? __dadd_rn(m.J, m.J) : m.J);
    }
    const bool hd = nb.z >= 0, hu = nb.w >= 0;
    const double cd = sq[n], cu = sq[n + 1];
    if (hd || hu) h = __dadd_rn(h, (hd && hu) ? __dadd_rn(cd, cu) : (hd ? cd : cu));
    return h;
}

}  // namespace paces
