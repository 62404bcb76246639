// One row of H applied to a vector, from the neighbour table and the row metadata.
//
// Reference: total_ham (paces/core/time_evolution.py:382-400) computes
//   diag * v + hopping_csr.dot(v) + vib_coupling_csr.dot(v)
// with CSR rows summed in increasing column order and float64 matrix elements
// J (hopping, paces/models/holstein.py:205-206) and g*sqrt(n) (vibronic coupling,
// holstein.py:271-274).  The complex128 form below keeps exactly that grouping and
// rounds every product and sum separately (no fused multiply-add), so it reproduces
// the reference arithmetic row by row.
#pragma once

#include "common.cuh"

namespace paces {

// Diagonal element from the row metadata (paces/models/holstein.py:280-287).
__device__ __forceinline__ double diag_value(const ModelDev& m, uint32_t meta) {
    const int pos = int(meta & 0xffu);
    const uint32_t ntot = meta >> 16;
    double d = __dadd_rn(m.eps_sys, __dmul_rn(m.hbar_omega, double(ntot)));
    if (m.delta_eps != 0.0) d = __dadd_rn(d, __dmul_rn(m.delta_eps, double(pos)));
    if (m.has_site_eps) d = __dadd_rn(d, m.site_eps[pos]);
    return d;
}

// y = (H x)[r] in complex128.  sq[k] = sqrt(k) * g.
__device__ __forceinline__ double2 h_row_c128(const ModelDev& m, const double* sq, int64_t r,
                                              const int* __restrict__ nbr, int64_t cap, uint32_t meta,
                                              const double2* __restrict__ x) {
    const int n = int((meta >> 8) & 0xffu);
    const double d = diag_value(m, meta);
    const double2 xr = __ldcg(x + r);
    double2 y = make_double2(__dmul_rn(d, xr.x), __dmul_rn(d, xr.y));
    int a = __ldg(nbr + r), b = __ldg(nbr + cap + r);
    const int nd = __ldg(nbr + 2 * cap + r), nu = __ldg(nbr + 3 * cap + r);
    if (a >= 0 || b >= 0) {
        if (a < 0 || (b >= 0 && b < a)) {
            const int tmp = a;
            a = b;
            b = tmp;
        }
        const double2 xa = __ldcg(x + a);
        double2 h = make_double2(__dmul_rn(m.J, xa.x), __dmul_rn(m.J, xa.y));
        if (b >= 0) {
            const double2 xb = __ldcg(x + b);
            h.x = __dadd_rn(h.x, __dmul_rn(m.J, xb.x));
            h.y = __dadd_rn(h.y, __dmul_rn(m.J, xb.y));
        }
        y.x = __dadd_rn(y.x, h.x);
        y.y = __dadd_rn(y.y, h.y);
    }
    if (nd >= 0 || nu >= 0) {
        double2 v;
        if (nd >= 0) {
            const double c = sq[n];
            const double2 xd = __ldcg(x + nd);
            v = make_double2(__dmul_rn(c, xd.x), __dmul_rn(c, xd.y));
            if (nu >= 0) {
                const double c2 = sq[n + 1];
                const double2 xu = __ldcg(x + nu);
                v.x = __dadd_rn(v.x, __dmul_rn(c2, xu.x));
                v.y = __dadd_rn(v.y, __dmul_rn(c2, xu.y));
            }
        } else {
            const double c2 = sq[n + 1];
            const double2 xu = __ldcg(x + nu);
            v = make_double2(__dmul_rn(c2, xu.x), __dmul_rn(c2, xu.y));
        }
        y.x = __dadd_rn(y.x, v.x);
        y.y = __dadd_rn(y.y, v.y);
    }
    return y;
}

// y = (H x)[r] in complex64 with fp32 accumulation.  sq[k] = float(sqrt(k) * g).
__device__ __forceinline__ float2 h_row_c64(const ModelDev& m, const float* sq, float J, int64_t r,
                                            const int* __restrict__ nbr, int64_t cap, uint32_t meta,
                                            const float2* __restrict__ x) {
    const int n = int((meta >> 8) & 0xffu);
    const float d = float(diag_value(m, meta));
    const float2 xr = __ldcg(x + r);
    float2 y = make_float2(d * xr.x, d * xr.y);
    const int a = __ldg(nbr + r), b = __ldg(nbr + cap + r);
    const int nd = __ldg(nbr + 2 * cap + r), nu = __ldg(nbr + 3 * cap + r);
    if (a >= 0) {
        const float2 v = __ldcg(x + a);
        y.x = fmaf(J, v.x, y.x);
        y.y = fmaf(J, v.y, y.y);
    }
    if (b >= 0) {
        const float2 v = __ldcg(x + b);
        y.x = fmaf(J, v.x, y.x);
        y.y = fmaf(J, v.y, y.y);
    }
    if (nd >= 0) {
        const float2 v = __ldcg(x + nd);
        y.x = fmaf(sq[n], v.x, y.x);
        y.y = fmaf(sq[n], v.y, y.y);
    }
    if (nu >= 0) {
        const float2 v = __ldcg(x + nu);
        y.x = fmaf(sq[n + 1], v.x, y.x);
        y.y = fmaf(sq[n + 1], v.y, y.y);
    }
    return y;
}

}  // namespace paces
