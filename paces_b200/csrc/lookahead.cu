// Look-ahead weights for the truncation (TimeEvoParams.tau != 0).
//
// Reference (paces/core/time_evolution.py):
//   coherence_weighting_func (:464-469)  w = |psi|^2 + tau^2 |psi|^2 (H 1)^2
//   norm_weighting_func      (:472-476)  w = |psi - 1j tau H psi|
//   total_ham_ones           (:403-420)  H 1 = diag + row sums of each term matrix
// and _determine_select_whoami (:833-857) ranks the states by w instead of |psi| from the
// second time step on (:560).  H is the table of the basis psi lives in -- the one the
// previous step assembled.
//
// B200 design: one grid-stride pass over the rows, reading the row's neighbour entry and
// metadata (20 bytes), its amplitude and, for the norm weighting, the four neighbour
// amplitudes (the same gather as one Taylor term), writing one double.  HBM-bound like a
// Taylor term; it runs once per step, before the truncation's radix select.
//
// Bit-exactness (complex128): every product and sum is rounded separately (no fused
// multiply-add) in the reference's order.  The row sums need no order: the vibronic
// matrix has at most two elements in a row, and every element of a hopping term's row is
// the same J, so any order of their sum rounds alike.  The product
// 1j * tau * Hpsi has the real part 0 * Re(Hpsi) - tau * Im(Hpsi) = -(tau * Im(Hpsi)) and
// the imaginary part tau * Re(Hpsi), exactly, whatever the evaluation order.
#include "kernels.cuh"

#include "hrow.cuh"

namespace paces {

namespace {

template <bool C64>
__global__ void __launch_bounds__(256) lookahead_kernel(ModelDev m, const int* __restrict__ blk,
                                                        const int* __restrict__ nbr,
                                                        const uint32_t* __restrict__ meta,
                                                        const void* __restrict__ psi, double tau, double tau2,
                                                        int kind, double* __restrict__ w, int* status) {
    // sqrt(k) * g for occupations k < 260 (fields are at most 8 bits wide), as the Taylor
    // kernels build it; fp32 copies for the complex64 rows
    __shared__ double s_sq[260];
    __shared__ float s_sqf[260];
    for (int k = threadIdx.x; k < 260; k += blockDim.x) {
        s_sq[k] = __dmul_rn(sqrt(double(k)), m.g);
        s_sqf[k] = float(s_sq[k]);
    }
    __syncthreads();
    const int64_t S = blk[m.L];
    for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < S; r += int64_t(gridDim.x) * blockDim.x) {
        const int4 nb = load_nbr(nbr, r);
        const uint32_t mt = __ldg(meta + r);
        double out;
        if (kind == PACES_WEIGHT_NORM) {
            if constexpr (C64) {
                const float2* x = reinterpret_cast<const float2*>(psi);
                const float2 xr = __ldcg(x + r);
                const float2 hx = h_row_c64_any(m, s_sqf, float(m.J), r, nb, mt, xr, x);
                const float t = float(tau);
                out = double(hypotf(xr.x + t * hx.y, xr.y - t * hx.x));
            } else {
                const double2* x = reinterpret_cast<const double2*>(psi);
                const double2 xr = __ldcg(x + r);
                const double2 hx = h_row_c128_any(m, s_sq, r, nb, mt, xr, x);
                out = hypot(__dadd_rn(xr.x, __dmul_rn(tau, hx.y)), __dsub_rn(xr.y, __dmul_rn(tau, hx.x)));
            }
        } else {
            const double h1 = h_ones_row_any(m, s_sq, r, nb, mt);
            if (kind == PACES_WEIGHT_HAM_ONES) {
                out = h1;
            } else {
                double a;
                if constexpr (C64) {
                    const float2 z = __ldcg(reinterpret_cast<const float2*>(psi) + r);
                    a = double(hypotf(z.x, z.y));
                } else {
                    const double2 z = __ldcg(reinterpret_cast<const double2*>(psi) + r);
                    a = hypot(z.x, z.y);
                }
                const double psq = __dmul_rn(a, a);
                out = __dadd_rn(psq, __dmul_rn(__dmul_rn(tau2, psq), __dmul_rn(h1, h1)));
            }
        }
        if (kind != PACES_WEIGHT_HAM_ONES && !(out <= 1.7976931348623157e308)) raise_status(status, PACES_ERR_NONFINITE);
        w[r] = out;
    }
}

}  // namespace

int launch_lookahead(bool c64, const ModelDev& m, const int* blk, const int* nbr, const uint32_t* meta,
                     const void* psi, double tau, int kind, double* w, int* status, int num_sms, cudaStream_t st) {
    if (kind != PACES_WEIGHT_COHERENCE && kind != PACES_WEIGHT_NORM && kind != PACES_WEIGHT_HAM_ONES)
        return PACES_ERR_BADARG;
    const double tau2 = tau * tau;
    const int g = num_sms * 8;
    if (c64)
        lookahead_kernel<true><<<g, 256, 0, st>>>(m, blk, nbr, meta, psi, tau, tau2, kind, w, status);
    else
        lookahead_kernel<false><<<g, 256, 0, st>>>(m, blk, nbr, meta, psi, tau, tau2, kind, w, status);
    return cudaGetLastError() == cudaSuccess ? PACES_OK : PACES_ERR_CUDA;
}

}  // namespace paces
