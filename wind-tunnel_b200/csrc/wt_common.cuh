// Shared device-side definitions for libwt.so (sm_100a).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/wt.h"

namespace wt {

constexpr int Q = 19;

// D3Q19 velocity set in the reference's order (server/lbm.py:15-17).
__host__ __device__ constexpr int cx(int i) {
    constexpr int t[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[i];
}
__host__ __device__ constexpr int cy(int i) {
    constexpr int t[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
    return t[i];
}
__host__ __device__ constexpr int cz(int i) {
    constexpr int t[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
    return t[i];
}
__host__ __device__ constexpr int opp(int i) {
    constexpr int t[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
    return t[i];
}
// weights as the reference computes them, in double (server/lbm.py:18)
__host__ __device__ constexpr double wd(int i) {
    return i == 0 ? 1.0 / 3.0
                  : ((cx(i) != 0) + (cy(i) != 0) + (cz(i) != 0) == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
}

// ---- storage traits: S = stored type, T = arithmetic type ----
template <int PREC> struct Prec;
template <> struct Prec<WT_F32> {
    using S = float; using T = float; static constexpr bool shifted = false;
    __device__ static __forceinline__ float to(S v) { return v; }
    __device__ static __forceinline__ S from(float v) { return v; }
};
template <> struct Prec<WT_F16> {
    using S = __half; using T = float; static constexpr bool shifted = true;
    __device__ static __forceinline__ float to(S v) { return __half2float(v); }
    __device__ static __forceinline__ S from(float v) { return __float2half_rn(v); }
};
template <> struct Prec<WT_BF16> {
    using S = __nv_bfloat16; using T = float; static constexpr bool shifted = true;
    __device__ static __forceinline__ float to(S v) { return __bfloat162float(v); }
    __device__ static __forceinline__ S from(float v) { return __float2bfloat16_rn(v); }
};
template <> struct Prec<WT_F64> {
    using S = double; using T = double; static constexpr bool shifted = false;
    __device__ static __forceinline__ double to(S v) { return v; }
    __device__ static __forceinline__ S from(double v) { return v; }
};

// population value as the collision sees it; shifted storage holds f - e (e: the shift of
// population I, see ShiftTables)
template <class P, int I>
__device__ __forceinline__ typename P::T ld_pop(const typename P::S* p, typename P::T e) {
    if constexpr (P::shifted) return P::to(*p) + e;
    else return P::to(*p);
}
template <class P, int I>
__device__ __forceinline__ void st_pop(typename P::S* p, typename P::T v, typename P::T e) {
    if constexpr (P::shifted) *p = P::from(v - e);
    else *p = P::from(v);
}

// Shift of half-width (fp16/bf16) population storage: populations are stored as
// d_i = f_i - e_i with e_i the equilibrium at rho = 1, u = (U, 0, 0) (wt_grid.shift_u). Near
// the free stream the stored deviations are then small, which is where half precision has
// its absolute resolution. U = 0 gives e_i = w_i, the rest weights. All tables are evaluated
// in double and rounded once:
//   e_i  = w_i (1 + 3 cx_i U + 4.5 cx_i^2 U^2 - 1.5 U^2)
//   bb_i = e_opp(i) - e_i          (bounce-back in deviation form)
//   dw_i = e_i - w_i               (momentum exchange uses f_i - w_i)
//   su = U, suu = U^2, s45 = 4.5 U^2, s15 = 1.5 U^2 (moment-space collision)
struct ShiftTables {
    bool on;  // U != 0
    double e[Q], bb[Q], dw[Q];
    double su, suu, s45, s15;
};
inline ShiftTables shift_tables(double U) {
    ShiftTables t;
    t.on = U != 0.0;
    double e[Q];
    for (int i = 0; i < Q; ++i) {
        const double cu = 3.0 * cx(i) * U;
        e[i] = wd(i) * (1.0 + cu + 0.5 * cu * cu - 1.5 * U * U);
    }
    for (int i = 0; i < Q; ++i) {
        t.e[i] = t.on ? e[i] : wd(i);
        t.bb[i] = e[opp(i)] - e[i];
        t.dw[i] = e[i] - wd(i);
    }
    t.su = U;
    t.suu = U * U;
    t.s45 = 4.5 * U * U;
    t.s15 = 1.5 * U * U;
    return t;
}

// Division of non-negative 32-bit ints below 2^31 by a fixed divisor via multiply-high
// (Granlund & Montgomery, "Division by invariant integers using multiplication", 1994):
// with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1, q = (umulhi(m, n) + n) >> l.
struct FastDiv {
    uint32_t d, m, l;
    FastDiv() = default;
    __host__ explicit FastDiv(uint32_t div) : d(div) {
        l = 0;
        while ((1ull << l) < div) ++l;
        m = (uint32_t)(((1ull << 32) * ((1ull << l) - div)) / div + 1);
    }
    __device__ __forceinline__ uint32_t div(uint32_t n) const { return (__umulhi(m, n) + n) >> l; }
};

// per-cell code byte (wt_build_codes)
constexpr uint8_t CODE_SOLID = 1;  // solid byte != 0
constexpr uint8_t CODE_NEAR = 2;   // interior fluid cell with a non-fluid neighbour (slow pull path)

template <int I, int N, class F>
__device__ __forceinline__ void unroll(F&& f) {
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        unroll<I + 1, N>(f);
    }
}

}  // namespace wt

// error plumbing (wt_abi.cu)
int wt_set_error(int code, const char* fmt, ...);
int wt_cuda_check(const char* what);
