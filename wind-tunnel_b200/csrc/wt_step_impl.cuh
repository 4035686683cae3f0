// Fused D3Q19 step: pull streaming + bounce-back / moving belt + equilibrium faces +
// regularized collision with Smagorinsky eddy viscosity and outlet sponge.
// Semantics: step_kernel of RICKxxROLLING/wind-tunnel server/lbm.py:72-166.
//
// One step = two launches:
//   k_step_bulk  -- every cell except the "current-read" faces below. Each thread owns V
//                   consecutive cells of one x-row. Interior cells pull and collide; x = 0
//                   inlet cells; face cells whose interior neighbour has a LARGER linear
//                   index read that neighbour's mac from the previous step (mac_prev); the
//                   outlet cell x = nx-1 of an interior row takes the current values of its
//                   x = nx-2 neighbour from the same thread (V > 1) or the previous lane.
//   k_step_faces -- the z = nz-1 plane and the y = ny-1 rows of interior z (x > 0): their
//                   neighbour has a SMALLER linear index, so they read the mac that
//                   k_step_bulk just wrote (mac_cur).
// That is exactly the value each face cell sees when the reference launch runs in tid
// order (Warp's CPU backend), and it is deterministic, unlike the single-launch race of
// server/lbm.py:87 vs :166 on a GPU.
//
// Memory: population i of the pull source of cell idx is src[i][idx] with
// src[i] = fin + i*n - (c_ix + c_iy*nx + c_iz*nx*ny), so every load is one base pointer
// (kernel parameter, uniform) plus idx. A thread whose V cells are all plain interior fluid
// (the common case) loads each population with one aligned V-wide vector load, plus one
// scalar for the ±x-shifted ones, and stores each output population with one vector store.
//
// mac is double-buffered: the step that writes f[b] writes mac[b]. Every step writes mac
// for the shell of interior cells that faces read (coordinates 1 or n-2); with mac_all set
// (the last step before a frame) every cell writes it, as the reference does.
//
// Arithmetic keeps the reference's association order (the library is built without FMA
// contraction). Two rewrites are exact: a leading "0.0 +" of a generated sum is dropped
// (it can only turn -0.0 into +0.0, which no later operation can observe here), and the
// term 0.5*cu*cu is shared by opposite directions (cu of the opposite direction is the
// exact negation).
#pragma once

#include <algorithm>

#include "wt_common.cuh"

namespace wt {

template <class S, class T>
struct StepArgs {
    const S* src[Q];   // pull source bases, see above
    S* dst[Q];         // fout + i*n
    const S* fin;
    const T* mac_prev;
    T* mac_cur;
    const uint8_t* solid;
    const uint8_t* code;
    int32_t nx, ny, nz, n, nxy;
    FastDiv dnx, dny;
    T uin, tau, csmag;  // csmag = 25.4558441 * smag * smag, evaluated in T left to right
    int32_t mac_all;
    // streaming kernel: 16-byte aligned copy bases (src[i] rounded down) and the remainders
    const S* chunk_src[Q];
    int32_t chunk_r[Q];
    int32_t* status;           // device word for bounded-wait failures (may be null)
    int32_t test_skip_chunk;   // test hook: when > 0, chunk test_skip_chunk-1 is never loaded
    // shifted storage (ShiftTables of wt_grid.shift_u, rounded to T)
    T e[Q], bb[Q];
    T su, suu, s45, s15;
};

template <class S, class T>
inline void set_shift(StepArgs<S, T>& a, double shift_u) {
    const ShiftTables t = shift_tables(shift_u);
    for (int i = 0; i < Q; ++i) {
        a.e[i] = (T)t.e[i];
        a.bb[i] = (T)t.bb[i];
    }
    a.su = (T)t.su; a.suu = (T)t.suu; a.s45 = (T)t.s45; a.s15 = (T)t.s15;
}

// the shift constants the moment-space collision needs (a pair: broadcast to both lanes)
template <class T>
struct ShiftK {
    T su, suu, s45, s15;
};

template <class T>
__device__ __forceinline__ void store_mac(T* mac, int32_t idx, T a, T b, T c, T d) {
    if constexpr (sizeof(T) == 4) {
        reinterpret_cast<float4*>(mac)[idx] = make_float4(a, b, c, d);
    } else {
        reinterpret_cast<double2*>(mac)[2 * idx] = make_double2(a, b);
        reinterpret_cast<double2*>(mac)[2 * idx + 1] = make_double2(c, d);
    }
}
template <class T>
__device__ __forceinline__ void load_mac(const T* mac, int32_t idx, T& a, T& b, T& c, T& d) {
    if constexpr (sizeof(T) == 4) {
        const float4 v = reinterpret_cast<const float4*>(mac)[idx];
        a = v.x; b = v.y; c = v.z; d = v.w;
    } else {
        const double2 v0 = reinterpret_cast<const double2*>(mac)[2 * idx];
        const double2 v1 = reinterpret_cast<const double2*>(mac)[2 * idx + 1];
        a = v0.x; b = v0.y; c = v1.x; d = v1.y;
    }
}

template <class T>
__device__ __forceinline__ T clampv(T x, T lo, T hi) { return x < lo ? lo : (x > hi ? hi : x); }

// aligned vector of V stored values
template <class S, int V>
struct SVec {
    S v[V];
};
template <class S, int V>
__device__ __forceinline__ SVec<S, V> vload(const S* p) {
    SVec<S, V> r;
    constexpr int B = (int)sizeof(S) * V;
    static_assert(B == 4 || B == 8 || B == 16 || B == 32, "vector width");
    if constexpr (B == 4) {
        const uint32_t u = *reinterpret_cast<const uint32_t*>(p);
        memcpy(&r, &u, 4);
    } else if constexpr (B == 8) {
        const uint2 u = *reinterpret_cast<const uint2*>(p);
        memcpy(&r, &u, 8);
    } else if constexpr (B == 16) {
        const uint4 u = *reinterpret_cast<const uint4*>(p);
        memcpy(&r, &u, 16);
    } else {
        const uint4 u0 = reinterpret_cast<const uint4*>(p)[0];
        const uint4 u1 = reinterpret_cast<const uint4*>(p)[1];
        memcpy(&r, &u0, 16);
        memcpy(reinterpret_cast<char*>(&r) + 16, &u1, 16);
    }
    return r;
}
template <class S, int V>
__device__ __forceinline__ void vstore(S* p, const SVec<S, V>& r) {
    constexpr int B = (int)sizeof(S) * V;
    if constexpr (B == 4) {
        uint32_t u;
        memcpy(&u, &r, 4);
        *reinterpret_cast<uint32_t*>(p) = u;
    } else if constexpr (B == 8) {
        uint2 u;
        memcpy(&u, &r, 8);
        *reinterpret_cast<uint2*>(p) = u;
    } else if constexpr (B == 16) {
        uint4 u;
        memcpy(&u, &r, 16);
        *reinterpret_cast<uint4*>(p) = u;
    } else {
        uint4 u0, u1;
        memcpy(&u0, &r, 16);
        memcpy(&u1, reinterpret_cast<const char*>(&r) + 16, 16);
        reinterpret_cast<uint4*>(p)[0] = u0;
        reinterpret_cast<uint4*>(p)[1] = u1;
    }
}

// Equilibrium face populations from (br, bux, buy, buz) (server/lbm.py:104-107).
template <class P>
__device__ __forceinline__ void face_eq(const StepArgs<typename P::S, typename P::T>& a, int32_t idx,
                                        typename P::T br, typename P::T bux, typename P::T buy, typename P::T buz) {
    using T = typename P::T;
    const T bsq = (T)1.5 * (bux * bux + buy * buy + buz * buz);
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        T s = (T)0.0;
        if constexpr (cx(i) > 0) s = s + bux;
        if constexpr (cx(i) < 0) s = s - bux;
        if constexpr (cy(i) > 0) s = s + buy;
        if constexpr (cy(i) < 0) s = s - buy;
        if constexpr (cz(i) > 0) s = s + buz;
        if constexpr (cz(i) < 0) s = s - buz;
        const T bc = (T)3.0 * s;
        st_pop<P, i>(a.dst[i] + idx, (T)wd(i) * br * ((T)1.0 + bc + (T)0.5 * bc * bc - bsq), a.e[i]);
    });
}

// Boundary values of a face cell from its clamped interior neighbour's mac
// (server/lbm.py:87-103).
template <class T>
__device__ __forceinline__ void face_values(int32_t x, int32_t y, int32_t z, int32_t nx, int32_t ny, int32_t nz,
                                            T uin, T mx, T my, T mz, T mr, T& br, T& bux, T& buy, T& buz) {
    br = clampv(mr, (T)0.9, (T)1.1);
    bux = mx; buy = my; buz = mz;
    if (y == 0 || y == ny - 1) buy = (T)0.0;
    if (z == 0 || z == nz - 1) buz = (T)0.0;
    if (x == 0) {
        br = (T)1.0; bux = uin; buy = (T)0.0; buz = (T)0.0;
    } else if (x == nx - 1) {
        br = (T)1.0; bux = bux < (T)0.0 ? (T)0.0 : bux;
    }
}

// sum of c-signed terms in the generator's order with the leading "0.0 +" dropped
template <int AX, class T>
__device__ __forceinline__ T csum(const T (&f)[Q]) {
    T acc = (T)0.0;
    bool first = true;
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        constexpr int c = AX == 0 ? cx(i) : (AX == 1 ? cy(i) : cz(i));
        if constexpr (c != 0) {
            if (first) acc = c > 0 ? f[i] : -f[i];
            else acc = c > 0 ? acc + f[i] : acc - f[i];
            first = false;
        }
    });
    return acc;
}

// Regularized Smagorinsky collision of one cell (server/lbm.py:125-166). f holds the
// pulled populations on entry and the post-collision populations on exit.
template <class T>
__device__ __forceinline__ void collide(T (&f)[Q], int32_t x, int32_t nx, T tau, T csmag, T& oux, T& ouy, T& ouz,
                                        T& orho) {
    T rho = f[0];
    unroll<1, Q>([&](auto ic) { rho = rho + f[decltype(ic)::value]; });
    const T jx = csum<0>(f), jy = csum<1>(f), jz = csum<2>(f);
    const T ir = (T)1.0 / rho;
    T ux = jx * ir, uy = jy * ir, uz = jz * ir;
    const T um = sqrt(ux * ux + uy * uy + uz * uz);
    if (um > (T)0.35) {
        const T sc = (T)0.35 / um;
        ux = ux * sc; uy = uy * sc; uz = uz * sc;
    }
    const T usq = (T)1.5 * (ux * ux + uy * uy + uz * uz);
    T e[Q];
    // e_i = w rho (1 + cu + 0.5 cu cu - usq), d_i = f_i - e_i (f[] becomes d[])
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (i == 0) {
            e[0] = (T)wd(0) * rho * ((T)1.0 - usq);
            f[0] = f[0] - e[0];
        } else if constexpr (opp(i) > i) {  // handle the pair (i, opp(i)) together
            constexpr int o = opp(i);
            T s;
            bool first = true;
            if constexpr (cx(i) != 0) { s = cx(i) > 0 ? ux : -ux; first = false; }
            if constexpr (cy(i) != 0) {
                if (first) s = cy(i) > 0 ? uy : -uy;
                else s = cy(i) > 0 ? s + uy : s - uy;
                first = false;
            }
            if constexpr (cz(i) != 0) {
                if (first) s = cz(i) > 0 ? uz : -uz;
                else s = cz(i) > 0 ? s + uz : s - uz;
            }
            const T cu = (T)3.0 * s;
            const T q = (T)0.5 * cu * cu;
            const T wr = (T)wd(i) * rho;
            e[i] = wr * ((T)1.0 + cu + q - usq);
            e[o] = wr * ((T)1.0 - cu + q - usq);
            f[i] = f[i] - e[i];
            f[o] = f[o] - e[o];
        }
    });
    T pxx, pyy, pzz, pxy, pxz, pyz;
    {
        bool fx = true, fy = true, fz = true, fxy = true, fxz = true, fyz = true;
        pxx = pyy = pzz = pxy = pxz = pyz = (T)0.0;
        unroll<0, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            if constexpr (cx(i) != 0) { pxx = fx ? f[i] : pxx + f[i]; fx = false; }
            if constexpr (cy(i) != 0) { pyy = fy ? f[i] : pyy + f[i]; fy = false; }
            if constexpr (cz(i) != 0) { pzz = fz ? f[i] : pzz + f[i]; fz = false; }
            if constexpr (cx(i) * cy(i) != 0) {
                pxy = fxy ? (cx(i) * cy(i) > 0 ? f[i] : -f[i]) : (cx(i) * cy(i) > 0 ? pxy + f[i] : pxy - f[i]);
                fxy = false;
            }
            if constexpr (cx(i) * cz(i) != 0) {
                pxz = fxz ? (cx(i) * cz(i) > 0 ? f[i] : -f[i]) : (cx(i) * cz(i) > 0 ? pxz + f[i] : pxz - f[i]);
                fxz = false;
            }
            if constexpr (cy(i) * cz(i) != 0) {
                pyz = fyz ? (cy(i) * cz(i) > 0 ? f[i] : -f[i]) : (cy(i) * cz(i) > 0 ? pyz + f[i] : pyz - f[i]);
                fyz = false;
            }
        });
    }
    const T qn = sqrt(pxx * pxx + pyy * pyy + pzz * pzz + (T)2.0 * (pxy * pxy + pxz * pxz + pyz * pyz));
    T tau0 = tau;
    const T sp = (T)x - (T)nx + (T)24.0;
    if (sp > (T)0.0) tau0 = tau0 + sp * (T)0.015;
    const T tau_e = (T)0.5 * (tau0 + sqrt(tau0 * tau0 + csmag * qn * ir));
    const T keep = (T)1.0 - (T)1.0 / tau_e;
    const T tr3 = (pxx + pyy + pzz) * ((T)1.0 / (T)3.0);
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        // the generator's ' + '.join(terms) + ' - tr3' (server/lbm.py:157-164)
        T qp;
        if constexpr (i == 0) {
            qp = -tr3;
        } else {
            constexpr bool hx = cx(i) != 0, hy = cy(i) != 0, hz = cz(i) != 0;
            T acc = hx ? pxx : (hy ? pyy : pzz);
            if constexpr (hx && hy) acc = acc + pyy;
            if constexpr ((hx || hy) && hz) acc = acc + pzz;
            if constexpr (hx && hy) acc = acc + (T)(2 * cx(i) * cy(i)) * pxy;
            if constexpr (hx && hz) acc = acc + (T)(2 * cx(i) * cz(i)) * pxz;
            if constexpr (hy && hz) acc = acc + (T)(2 * cy(i) * cz(i)) * pyz;
            qp = acc - tr3;
        }
        f[i] = e[i] + (T)(4.5 * wd(i)) * keep * qp;
    });
    oux = ux; ouy = uy; ouz = uz; orho = rho;
}

// fused multiply-add, rounded once (explicit: the library is built without contraction)
__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }

// Moment-space form of the same regularized Smagorinsky collision (mathematically equal
// to collide(): on D3Q19 the second moment of the second-order equilibrium is
// rho (u u + I/3), so Pi_neq = sum_i f_i c_i c_i - rho (u u + I/3), and every output is
// w_i (B + 3 rho c.u + 4.5 rho (c.u)^2 + c c : A) with A = 4.5 (1 - 1/tau_e) Pi_neq and
// B = rho (1 - 1.5 u.u) - tr(A)/3). Opposite directions share all but the sign of the odd
// term. About 200 floating-point operations per cell against 330 in the reference order.
// With SHIFT the inputs and outputs are deviations v_i = f_i - w_i (the fp16/bf16 storage
// form): the constant parts cancel analytically, which keeps small numbers small.
// Reciprocals and square roots use the special-function unit (rcp_fast etc.), so results
// match the oracle's IEEE restatement of this form to within a few float ulps.
// Reciprocal and square roots for the fast form: the special-function unit's
// approximation refined by one Newton step (about 1 ulp in float); IEEE ops in double.
__device__ __forceinline__ float rcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    const float e = __fmaf_rn(-x, r, 1.0f);
    return __fmaf_rn(r, e, r);
}
__device__ __forceinline__ double rcp_fast(double x) { return 1.0 / x; }
__device__ __forceinline__ float sqrt_fast(float x) {  // x >= 0 (0 maps to 0)
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ double sqrt_fast(double x) { return sqrt(x); }
__device__ __forceinline__ float rsqrt_fast(float x) {  // x > 0
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    const float h = __fmul_rn(__fmul_rn(0.5f, x), __fmul_rn(r, r));
    return __fmul_rn(r, __fsub_rn(1.5f, h));
}
__device__ __forceinline__ double rsqrt_fast(double x) { return 1.0 / sqrt(x); }

// Two cells in one register pair. sm_100's paired fp32 instructions (FADD2, FMUL2, FFMA2)
// round each lane to nearest like the one-lane forms, so collide_fast on F2 gives each of
// the two cells exactly the bits of collide_fast on float, in about half the instructions.
struct F2 {
    float2 v;
    F2() = default;
    __device__ __forceinline__ explicit F2(double s) : v(make_float2((float)s, (float)s)) {}
    __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { F2 r; r.v = __fadd2_rn(a.v, b.v); return r; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { F2 r; r.v = __fmul2_rn(a.v, b.v); return r; }
#ifndef WT_PAIRED_SUB
#define WT_PAIRED_SUB 0
#endif
#if WT_PAIRED_SUB == 0
__device__ __forceinline__ F2 operator-(F2 a) { return F2(-a.v.x, -a.v.y); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return a + (-b); }  // x - y == x + (-y) in IEEE
#else
__device__ __forceinline__ F2 operator-(F2 a) { return a * F2(-1.0); }  // exact negation, one paired op
#if WT_PAIRED_SUB == 1
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {  // paired IEEE subtraction
    unsigned long long x, y, d;
    memcpy(&x, &a.v, 8);
    memcpy(&y, &b.v, 8);
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(x), "l"(y));
    F2 r;
    memcpy(&r.v, &d, 8);
    return r;
}
#else
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return a + b * F2(-1.0); }
#endif
#endif
__device__ __forceinline__ F2 fmaT(F2 a, F2 b, F2 c) { F2 r; r.v = __ffma2_rn(a.v, b.v, c.v); return r; }
__device__ __forceinline__ F2 rcp_fast(F2 x) {
    float r0, r1;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(x.v.x));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(x.v.y));
    const F2 r(r0, r1);
    return fmaT(r, fmaT(-x, r, F2(1.0)), r);
}
__device__ __forceinline__ F2 sqrt_fast(F2 x) { return F2(sqrt_fast(x.v.x), sqrt_fast(x.v.y)); }
__device__ __forceinline__ F2 rsqrt_fast(F2 x) {
    float r0, r1;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(x.v.x));
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r1) : "f"(x.v.y));
    const F2 r(r0, r1);
    return r * (F2(1.5) - (F2(0.5) * x) * (r * r));
}
// a > t in any lane; lane-wise a > t ? p : q
__device__ __forceinline__ bool any_gt(float a, float t) { return a > t; }
__device__ __forceinline__ bool any_gt(double a, double t) { return a > t; }
__device__ __forceinline__ bool any_gt(F2 a, F2 t) { return a.v.x > t.v.x || a.v.y > t.v.y; }
__device__ __forceinline__ float sel_gt(float a, float t, float p, float q) { return a > t ? p : q; }
__device__ __forceinline__ double sel_gt(double a, double t, double p, double q) { return a > t ? p : q; }
__device__ __forceinline__ F2 sel_gt(F2 a, F2 t, F2 p, F2 q) {
    return F2(a.v.x > t.v.x ? p.v.x : q.v.x, a.v.y > t.v.y ? p.v.y : q.v.y);
}
// x coordinate of the cell(s): x, or (x, x + 1) for a pair
template <class T>
__device__ __forceinline__ T xcoord(int32_t x) { return (T)x; }
template <>
__device__ __forceinline__ F2 xcoord<F2>(int32_t x) { return F2((float)x, (float)(x + 1)); }

// B = rho (1 - 1.5 u.u) - tr(A)/3 (with S for rho where SHIFT). The pair form evaluates it one
// lane at a time: its product-then-difference, compiled as paired operations, is fused by the
// assembler into one paired FMA (paired multiplies feeding paired adds are fused whatever the
// rounding modifiers and -fmad=false say), which rounds differently from the one-cell form;
// per-lane evaluation keeps identical bits at a cost of a few instructions. (Restating B with
// every product feeding an FMA multiplicand, k45 tr(N) times -1/3, was tried: the pair form
// still came out a last bit different from the one-cell form in some cells.)
// With SHIFT the outputs are deviations from the shift e_i, so B also carries + 1.5 U^2.
template <class T, bool SHIFT>
struct BTerm {
    __device__ static __forceinline__ T eval(T rho, T S, T usq, T axx, T ayy, T azz, T s15) {
        const T tra3 = ((axx + ayy) + azz) * (T)(1.0 / 3.0);
        const T b = fmaT(-rho, (T)1.5 * usq, SHIFT ? S : rho) - tra3;
        return SHIFT ? b + s15 : b;
    }
};
template <bool SHIFT>
struct BTerm<F2, SHIFT> {
    __device__ static __forceinline__ F2 eval(F2 rho, F2 S, F2 usq, F2 axx, F2 ayy, F2 azz, F2 s15) {
        return F2(BTerm<float, SHIFT>::eval(rho.v.x, S.v.x, usq.v.x, axx.v.x, ayy.v.x, azz.v.x, s15.v.x),
                  BTerm<float, SHIFT>::eval(rho.v.y, S.v.y, usq.v.y, axx.v.y, ayy.v.y, azz.v.y, s15.v.y));
    }
};

template <class T, bool SHIFT>
__device__ __forceinline__ void collide_fast(T (&v)[Q], int32_t x, int32_t nx, T tau, T csmag, const ShiftK<T>& sk,
                                             T& oux, T& ouy, T& ouz, T& orho) {
    const T s1 = v[1] + v[2], a1 = v[1] - v[2];
    const T s3 = v[3] + v[4], a3 = v[3] - v[4];
    const T s5 = v[5] + v[6], a5 = v[5] - v[6];
    const T s7 = v[7] + v[8], a7 = v[7] - v[8];
    const T s9 = v[9] + v[10], a9 = v[9] - v[10];
    const T s11 = v[11] + v[12], a11 = v[11] - v[12];
    const T s13 = v[13] + v[14], a13 = v[13] - v[14];
    const T s15 = v[15] + v[16], a15 = v[15] - v[16];
    const T s17 = v[17] + v[18], a17 = v[17] - v[18];
    const T d7 = s7 + s9, d11 = s11 + s13, d15 = s15 + s17;
    // with SHIFT: + U^2 in xx and + U in jx restore the moments of the shift e_i
    const T xxx0 = (s1 + d7) + d11, xyy = (s3 + d7) + d15, xzz = (s5 + d11) + d15;
    const T xxx = SHIFT ? xxx0 + sk.suu : xxx0;
    const T xxy = s7 - s9, xxz = s11 - s13, xyz = s15 - s17;
    const T S = ((v[0] + s1) + (s3 + s5)) + ((d7 + d11) + d15);
    const T jx0 = ((a1 + a7) + (a9 + a11)) + a13;
    const T jx = SHIFT ? jx0 + sk.su : jx0;
    const T jy = ((a3 + a7) - (a9 - a15)) + a17;
    const T jz = ((a5 + a11) - (a13 - a15)) - a17;
    const T rho = SHIFT ? S + (T)1.0 : S;
    const T ir = rcp_fast(rho);
    T ux = jx * ir, uy = jy * ir, uz = jz * ir;
    T usq = fmaT(uz, uz, fmaT(uy, uy, ux * ux));
    if (any_gt(usq, (T)0.1225)) {  // |u| > 0.35 (server/lbm.py:131-135)
        // a lane below the limit scales by 1 (exact) and recomputes the same usq
        const T sc = sel_gt(usq, (T)0.1225, (T)0.35 * rsqrt_fast(usq), (T)1.0);
        ux = ux * sc; uy = uy * sc; uz = uz * sc;
        usq = fmaT(uz, uz, fmaT(uy, uy, ux * ux));
    }
    const T rux = rho * ux, ruy = rho * uy, ruz = rho * uz;
    const T t3 = (SHIFT ? S : rho) * (T)(1.0 / 3.0);  // the float nearest 1/3 either way
    const T nxx = fmaT(-rux, ux, xxx - t3), nyy = fmaT(-ruy, uy, xyy - t3), nzz = fmaT(-ruz, uz, xzz - t3);
    const T nxy = fmaT(-rux, uy, xxy), nxz = fmaT(-rux, uz, xxz), nyz = fmaT(-ruy, uz, xyz);
    const T q1 = fmaT(nzz, nzz, fmaT(nyy, nyy, nxx * nxx));
    const T q2 = fmaT(nyz, nyz, fmaT(nxz, nxz, nxy * nxy));
    const T qn = sqrt_fast(fmaT((T)2.0, q2, q1));
    const T sp = xcoord<T>(x) - (T)(nx - 24);  // outlet sponge (server/lbm.py:149-151)
    const T tau0 = sel_gt(sp, (T)0.0, fmaT(sp, (T)0.015, tau), tau);
    const T tau_e = (T)0.5 * (tau0 + sqrt_fast(fmaT(tau0, tau0, csmag * qn * ir)));
    const T keep = (T)1.0 - rcp_fast(tau_e);
    const T k45 = (T)4.5 * keep, k9 = (T)9.0 * keep;
    const T axx = k45 * nxx, ayy = k45 * nyy, azz = k45 * nzz;
    const T axy = k9 * nxy, axz = k9 * nxz, ayz = k9 * nyz;  // 2 A_ab
    const T B = BTerm<T, SHIFT>::eval(rho, S, usq, axx, ayy, azz, sk.s15);
    // with SHIFT, a direction with c_x != 0 drops 3 c_x U from its odd term and 4.5 U^2 from
    // its even term (the shift's own terms): rux/rs less su, D less s45
    const T w0 = (T)wd(0), w1 = (T)wd(1), w2 = (T)wd(7);
    const T w1x3 = (T)(3.0 * wd(1)), w2x3 = (T)(3.0 * wd(7));
    v[0] = w0 * B;
    const T bxx = B + axx, byy = B + ayy;
    {
        const T D0 = fmaT((T)4.5 * rux, ux, bxx);
        const T D = SHIFT ? D0 - sk.s45 : D0, E = w1x3 * (SHIFT ? rux - sk.su : rux);
        v[1] = fmaT(w1, D, E); v[2] = fmaT(w1, D, -E);
    }
    {
        const T D = fmaT((T)4.5 * ruy, uy, byy), E = w1x3 * ruy;
        v[3] = fmaT(w1, D, E); v[4] = fmaT(w1, D, -E);
    }
    {
        const T D = fmaT((T)4.5 * ruz, uz, B + azz), E = w1x3 * ruz;
        v[5] = fmaT(w1, D, E); v[6] = fmaT(w1, D, -E);
    }
    const T pxy = bxx + ayy, pxz = bxx + azz, pyz = byy + azz;
    {
        const T su = ux + uy, rs = rux + ruy;
        const T D0 = fmaT((T)4.5 * rs, su, pxy + axy);
        const T D = SHIFT ? D0 - sk.s45 : D0, E = w2x3 * (SHIFT ? rs - sk.su : rs);
        v[7] = fmaT(w2, D, E); v[8] = fmaT(w2, D, -E);
    }
    {
        const T su = ux - uy, rs = rux - ruy;
        const T D0 = fmaT((T)4.5 * rs, su, pxy - axy);
        const T D = SHIFT ? D0 - sk.s45 : D0, E = w2x3 * (SHIFT ? rs - sk.su : rs);
        v[9] = fmaT(w2, D, E); v[10] = fmaT(w2, D, -E);
    }
    {
        const T su = ux + uz, rs = rux + ruz;
        const T D0 = fmaT((T)4.5 * rs, su, pxz + axz);
        const T D = SHIFT ? D0 - sk.s45 : D0, E = w2x3 * (SHIFT ? rs - sk.su : rs);
        v[11] = fmaT(w2, D, E); v[12] = fmaT(w2, D, -E);
    }
    {
        const T su = ux - uz, rs = rux - ruz;
        const T D0 = fmaT((T)4.5 * rs, su, pxz - axz);
        const T D = SHIFT ? D0 - sk.s45 : D0, E = w2x3 * (SHIFT ? rs - sk.su : rs);
        v[13] = fmaT(w2, D, E); v[14] = fmaT(w2, D, -E);
    }
    {
        const T su = uy + uz, rs = ruy + ruz;
        const T D = fmaT((T)4.5 * rs, su, pyz + ayz), E = w2x3 * rs;
        v[15] = fmaT(w2, D, E); v[16] = fmaT(w2, D, -E);
    }
    {
        const T su = uy - uz, rs = ruy - ruz;
        const T D = fmaT((T)4.5 * rs, su, pyz - ayz), E = w2x3 * rs;
        v[17] = fmaT(w2, D, E); v[18] = fmaT(w2, D, -E);
    }
    oux = ux; ouy = uy; ouz = uz; orho = rho;
}

// collision dispatch: FAST selects the moment-space form, on deviations for shifted storage
template <class S, class T>
__device__ __forceinline__ ShiftK<T> shiftk(const StepArgs<S, T>& a) {
    return ShiftK<T>{a.su, a.suu, a.s45, a.s15};
}
template <class S, class T>
__device__ __forceinline__ ShiftK<F2> shiftk2(const StepArgs<S, T>& a) {
    return ShiftK<F2>{F2(a.su), F2(a.suu), F2(a.s45), F2(a.s15)};
}

template <class P, bool FAST>
__device__ __forceinline__ void collide_any(typename P::T (&f)[Q], int32_t x, int32_t nx, typename P::T tau,
                                            typename P::T csmag, const ShiftK<typename P::T>& sk,
                                            typename P::T& ux, typename P::T& uy, typename P::T& uz,
                                            typename P::T& rho) {
    if constexpr (FAST) collide_fast<typename P::T, P::shifted>(f, x, nx, tau, csmag, sk, ux, uy, uz, rho);
    else collide<typename P::T>(f, x, nx, tau, csmag, ux, uy, uz, rho);
}

// population value as the collision of mode FAST takes it: f_i (+ w_i undone for shifted
// storage in the exact form), or the stored deviation itself in the fast form
template <class P, bool FAST, int I, class A>
__device__ __forceinline__ typename P::T ld_in(const A& a, const typename P::S* p) {
    if constexpr (FAST) return P::to(*p);
    else return ld_pop<P, I>(p, a.e[I]);
}

template <class P, bool FAST, int I, class A>
__device__ __forceinline__ void st_out(const A& a, typename P::S* p, typename P::T v) {
    if constexpr (FAST) *p = P::from(v);
    else st_pop<P, I>(p, v, a.e[I]);
}

// Pull of one cell with bounce-back and moving belt where a source is non-fluid
// (server/lbm.py:110-124).
template <class P, bool FAST>
__device__ __forceinline__ void pull_generic(const StepArgs<typename P::S, typename P::T>& a, int32_t idx,
                                             bool near, typename P::T (&f)[Q]) {
    using T = typename P::T;
    f[0] = ld_in<P, FAST, 0>(a, a.src[0] + idx);
    unroll<1, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if (!near) {
            f[i] = ld_in<P, FAST, i>(a, a.src[i] + idx);
        } else {
            const int32_t off = cx(i) + cy(i) * a.nx + cz(i) * a.nxy;
            const int t = a.solid[idx - off];
            if (t == 0) {
                f[i] = ld_in<P, FAST, i>(a, a.src[i] + idx);
            } else {
                // bounce-back; in deviation form the shift difference e_opp(i) - e_i is added
                f[i] = ld_in<P, FAST, opp(i)>(a, a.fin + (int64_t)opp(i) * a.n + idx);
                if constexpr (FAST && P::shifted) f[i] = f[i] + a.bb[i];
                if constexpr (cx(i) != 0) {
                    if (t == 2) f[i] = f[i] + (T)(6.0 * wd(i) * cx(i)) * a.uin;
                }
            }
        }
    });
}

template <class P, bool FAST>
__device__ __forceinline__ void store_cell(const StepArgs<typename P::S, typename P::T>& a, int32_t idx,
                                           const typename P::T (&f)[Q]) {
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        st_out<P, FAST, i>(a, a.dst[i] + idx, f[i]);
    });
}

// One cell outside the vector fast path: inlet, "previous-read" faces, solids and fluid
// cells next to non-fluid cells. Cells of k_step_faces (z = nz-1 plane, y = ny-1 rows of
// interior z) are skipped, and so is the outlet x = nx-1 of an interior row: the caller
// handles it with outlet_cell once its x = nx-2 neighbour's values are known. The cell's
// macro values (what it writes to mac) are returned in m*.
template <class P, bool FAST>
__device__ __forceinline__ void general_cell(const StepArgs<typename P::S, typename P::T>& a, int32_t idx, int32_t x,
                                             int32_t y, int32_t z, uint32_t code, bool face_row, bool row_shell,
                                             typename P::T& mx, typename P::T& my, typename P::T& mz,
                                             typename P::T& mr) {
    using T = typename P::T;
    const int32_t nx = a.nx, ny = a.ny, nz = a.nz;
    mx = (T)0.0; my = (T)0.0; mz = (T)0.0; mr = (T)1.0;
    const bool later = x > 0 && (face_row ? (z == nz - 1 || (y == ny - 1 && z > 0)) : x == nx - 1);
    if (later) return;
    bool write = a.mac_all;
    if (code & CODE_SOLID) {
        write = write || (row_shell || (!face_row && (x == 1 || x == nx - 2)));
    } else if (x == 0) {
        mx = a.uin;
        face_eq<P>(a, idx, (T)1.0, a.uin, (T)0.0, (T)0.0);
    } else if (face_row) {
        const int32_t cxi = min(max(x, 1), nx - 2), cyi = min(max(y, 1), ny - 2), czi = min(max(z, 1), nz - 2);
        T px, py, pz, pr;
        load_mac(a.mac_prev, cxi + nx * (cyi + ny * czi), px, py, pz, pr);
        face_values<T>(x, y, z, nx, ny, nz, a.uin, px, py, pz, pr, mr, mx, my, mz);
        face_eq<P>(a, idx, mr, mx, my, mz);
    } else {
        T f[Q];
        pull_generic<P, FAST>(a, idx, (code & CODE_NEAR) != 0, f);
        collide_any<P, FAST>(f, x, nx, a.tau, a.csmag, shiftk(a), mx, my, mz, mr);
        store_cell<P, FAST>(a, idx, f);
        write = write || row_shell || x == 1 || x == nx - 2;
    }
    if (write) store_mac(a.mac_cur, idx, mx, my, mz, mr);
}

// Outlet x = nx-1 of an interior row (server/lbm.py:101-103): equilibrium at rho = 1 from the
// current values of its x = nx-2 neighbour (the neighbour has the smaller index, so in the
// reference's serial order it is already updated).
template <class P>
__device__ __forceinline__ void outlet_cell(const StepArgs<typename P::S, typename P::T>& a, int32_t idx, int32_t y,
                                            int32_t z, uint32_t code, typename P::T qx, typename P::T qy,
                                            typename P::T qz, typename P::T qr) {
    using T = typename P::T;
    if (code & CODE_SOLID) {
        if (a.mac_all) store_mac(a.mac_cur, idx, (T)0.0, (T)0.0, (T)0.0, (T)1.0);
        return;
    }
    T br, bux, buy, buz;
    face_values<T>(a.nx - 1, y, z, a.nx, a.ny, a.nz, a.uin, qx, qy, qz, qr, br, bux, buy, buz);
    face_eq<P>(a, idx, br, bux, buy, buz);
    if (a.mac_all) store_mac(a.mac_cur, idx, bux, buy, buz, br);
}

// V consecutive cells starting at idx0 (a multiple of V, and idx0 % 32 is the lane's
// multiple of V, so for V == 1 the previous cell is the previous lane). All 32 lanes of a
// warp must call this together (the V == 1 outlet exchanges values by shuffle).
// Collision of V consecutive plain fluid cells of one row, with their mac stores in cell
// order; the fast float form takes the cells two at a time on F2 (bit-identical per cell).
// mx..mr end as the last cell's macro values.
template <class P, bool FAST, int V>
__device__ __forceinline__ void collide_cells(const StepArgs<typename P::S, typename P::T>& a,
                                              typename P::T (&f)[V][Q], int32_t idx0, int32_t x0, bool row_shell,
                                              typename P::T& mx, typename P::T& my, typename P::T& mz,
                                              typename P::T& mr) {
    using T = typename P::T;
    const int32_t nx = a.nx;
    if constexpr (FAST && V % 2 == 0 && std::is_same<T, float>::value) {
#pragma unroll
        for (int k = 0; k < V; k += 2) {
            F2 g[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) g[i] = F2(f[k][i], f[k + 1][i]);
            F2 ux, uy, uz, rho;
            collide_fast<F2, P::shifted>(g, x0 + k, nx, F2(a.tau), F2(a.csmag), shiftk2(a), ux, uy, uz, rho);
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                f[k][i] = g[i].v.x;
                f[k + 1][i] = g[i].v.y;
            }
            if (a.mac_all || row_shell || x0 + k == 1 || x0 + k == nx - 2)
                store_mac(a.mac_cur, idx0 + k, ux.v.x, uy.v.x, uz.v.x, rho.v.x);
            mx = ux.v.y; my = uy.v.y; mz = uz.v.y; mr = rho.v.y;
            if (a.mac_all || row_shell || x0 + k + 1 == 1 || x0 + k + 1 == nx - 2)
                store_mac(a.mac_cur, idx0 + k + 1, mx, my, mz, mr);
        }
    } else {
#pragma unroll
        for (int k = 0; k < V; ++k) {
            collide_any<P, FAST>(f[k], x0 + k, nx, a.tau, a.csmag, shiftk(a), mx, my, mz, mr);
            if (a.mac_all || row_shell || x0 + k == 1 || x0 + k == nx - 2) store_mac(a.mac_cur, idx0 + k, mx, my, mz, mr);
        }
    }
}

// Face equilibrium populations from (br, bux, buy, buz), the values face_eq stores, in the form
// store_cells takes them: deviations f - w for the fast form of shifted storage, else f.
template <class P, bool FAST, class A>
__device__ __forceinline__ void eq_values(const A& a, typename P::T br, typename P::T bux, typename P::T buy,
                                          typename P::T buz, typename P::T (&out)[Q]) {
    using T = typename P::T;
    const T bsq = (T)1.5 * (bux * bux + buy * buy + buz * buz);
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        T s = (T)0.0;
        if constexpr (cx(i) > 0) s = s + bux;
        if constexpr (cx(i) < 0) s = s - bux;
        if constexpr (cy(i) > 0) s = s + buy;
        if constexpr (cy(i) < 0) s = s - buy;
        if constexpr (cz(i) > 0) s = s + buz;
        if constexpr (cz(i) < 0) s = s - buz;
        const T bc = (T)3.0 * s;
        const T v = (T)wd(i) * br * ((T)1.0 + bc + (T)0.5 * bc * bc - bsq);
        if constexpr (P::shifted && FAST) out[i] = v - a.e[i];
        else out[i] = v;
    });
}

// Collision of two cells of one row (pair form for the fast float collision); m[k] gets
// cell k's macro values (ux, uy, uz, rho). No mac stores.
template <class P, bool FAST>
__device__ __forceinline__ void collide_two(const StepArgs<typename P::S, typename P::T>& a, typename P::T (&f)[2][Q],
                                            int32_t x0, typename P::T (&m)[2][4]) {
    using T = typename P::T;
    if constexpr (FAST && std::is_same<T, float>::value) {
        F2 g[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i] = F2(f[0][i], f[1][i]);
        F2 ux, uy, uz, rho;
        collide_fast<F2, P::shifted>(g, x0, a.nx, F2(a.tau), F2(a.csmag), shiftk2(a), ux, uy, uz, rho);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            f[0][i] = g[i].v.x;
            f[1][i] = g[i].v.y;
        }
        m[0][0] = ux.v.x; m[0][1] = uy.v.x; m[0][2] = uz.v.x; m[0][3] = rho.v.x;
        m[1][0] = ux.v.y; m[1][1] = uy.v.y; m[1][2] = uz.v.y; m[1][3] = rho.v.y;
    } else {
#pragma unroll
        for (int k = 0; k < 2; ++k) collide_any<P, FAST>(f[k], x0 + k, a.nx, a.tau, a.csmag, shiftk(a), m[k][0], m[k][1], m[k][2], m[k][3]);
    }
}

// Population I of V consecutive cells to p (aligned to V elements); half-width storage
// rounds two values per conversion (each to nearest, as one at a time).
template <class P, bool FAST, int V, int I, class A>
__device__ __forceinline__ void store_cells(const A& a, typename P::S* p, const typename P::T (&f)[V][Q]) {
    using S = typename P::S;
    using T = typename P::T;
    if constexpr (V == 1) {
        st_out<P, FAST, I>(a, p, f[0][I]);
    } else {
        SVec<S, V> v;
#pragma unroll
        for (int k = 0; k < V; k += 2) {
            T lo = f[k][I], hi = f[k + 1][I];
            if constexpr (P::shifted && !FAST) {
                lo = lo - a.e[I];
                hi = hi - a.e[I];
            }
            if constexpr (std::is_same<S, __half>::value) {
                const __half2 h = __floats2half2_rn(lo, hi);
                memcpy(&v.v[k], &h, 4);
            } else if constexpr (std::is_same<S, __nv_bfloat16>::value) {
                const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
                memcpy(&v.v[k], &h, 4);
            } else {
                v.v[k] = P::from(lo);
                v.v[k + 1] = P::from(hi);
            }
        }
        vstore<S, V>(p, v);
    }
}

// Raw stored values of the pull of one pair of cells (x0 even) of an interior row: for each
// population the aligned two-element vector at p + cx(i) and, where cx(i) != 0, the one
// element outside it; plus the pair's code bytes.
template <class S>
struct PairRaw {
    SVec<S, 2> v[Q];
    S e[Q];
    uint32_t codes;
};

// every source of an interior row lies inside the lattice
template <int PREC>
__device__ __forceinline__ void pair_load(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                          int32_t idx0, PairRaw<typename Prec<PREC>::S>& r) {
    using S = typename Prec<PREC>::S;
    // float and double: each population from its own pull base (a kernel parameter) plus the
    // cell index; half width: one per-thread base plus offsets that are the same for every
    // thread (the faster form for each, measured)
    const S* fb = a.fin + idx0;
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        const S* p = sizeof(S) >= 4
                         ? a.src[i] + idx0
                         : fb + ((int64_t)i * a.n - (cx(i) + cy(i) * (int64_t)a.nx + cz(i) * (int64_t)a.nxy));
        r.v[i] = vload<S, 2>(p + cx(i));  // aligned: the shift cancels
        if constexpr (cx(i) > 0) r.e[i] = p[0];
        if constexpr (cx(i) < 0) r.e[i] = p[1];
    });
    r.codes = *reinterpret_cast<const uint16_t*>(a.code + idx0);
}

template <class P, bool FAST, class A>
__device__ __forceinline__ void pair_unpack(const A& a, const PairRaw<typename P::S>& r, typename P::T (&f)[2][Q]) {
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (cx(i) == 0) {
            f[0][i] = ld_in<P, FAST, i>(a, &r.v[i].v[0]);
            f[1][i] = ld_in<P, FAST, i>(a, &r.v[i].v[1]);
        } else if constexpr (cx(i) > 0) {
            f[0][i] = ld_in<P, FAST, i>(a, &r.e[i]);
            f[1][i] = ld_in<P, FAST, i>(a, &r.v[i].v[0]);
        } else {
            f[0][i] = ld_in<P, FAST, i>(a, &r.v[i].v[1]);
            f[1][i] = ld_in<P, FAST, i>(a, &r.e[i]);
        }
    });
}

// Two cells (x0 even) of an interior row, whatever their kind, in one lane-uniform sequence:
// vector pull of both, bounce-back at links into non-fluid cells (server/lbm.py:110-124),
// one pair collision, then the inlet (x = 0) and outlet (x = nx-1, from its x = nx-2
// neighbour's values of this step, server/lbm.py:87-107) take face equilibria; a solid cell's
// populations are not written. The results and mac writes are those of general_cell and
// outlet_cell, but a warp no longer splits into per-cell branches at walls and row ends.
// pair_finish takes the pulled populations; interior_pair loads them itself.
// Bounce-back and moving belt (server/lbm.py:110-124) as overrides of a pair's pulled values:
// for each cell of the pair next to a non-fluid cell (CODE_NEAR in c0 / c1), every population
// whose source is non-fluid takes the cell's own opposite population instead.
template <int PREC, bool FAST>
__device__ __forceinline__ void pair_walls(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                           int32_t idx0, uint32_t c0, uint32_t c1, typename Prec<PREC>::T (&f)[2][Q]) {
    using P = Prec<PREC>;
    using T = typename P::T;
    unroll<1, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        const int32_t off = cx(i) + cy(i) * a.nx + cz(i) * a.nxy;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (((k ? c1 : c0) & CODE_NEAR) == 0) continue;
            const int t = a.solid[idx0 + k - off];
            if (t != 0) {
                // bounce-back; in deviation form the shift difference e_opp(i) - e_i is added
                T b = ld_in<P, FAST, opp(i)>(a, a.fin + (int64_t)opp(i) * a.n + idx0 + k);
                if constexpr (FAST && P::shifted) b = b + a.bb[i];
                if constexpr (cx(i) != 0) {
                    if (t == 2) b = b + (T)(6.0 * wd(i) * cx(i)) * a.uin;
                }
                f[k][i] = b;
            }
        }
    });
}

// the macro values (ux, uy, uz, rho) of a solid cell
template <class T>
__device__ __forceinline__ void solid_macro(T (&m)[4]) {
    m[0] = (T)0.0; m[1] = (T)0.0; m[2] = (T)0.0; m[3] = (T)1.0;
}

// pair_finish hands the pair's macro values (what it writes to mac) back in mo.
template <int PREC, bool FAST>
__device__ __forceinline__ void pair_finish(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                            int32_t idx0, int32_t x0, int32_t y, int32_t z, uint32_t codes,
                                            bool row_shell, typename Prec<PREC>::T (&f)[2][Q],
                                            typename Prec<PREC>::T (&mo)[2][4]) {
    using P = Prec<PREC>;
    using T = typename P::T;
    const int32_t nx = a.nx;
    const uint32_t c0 = codes & 0xffu, c1 = (codes >> 8) & 0xffu;
    const bool sol0 = (c0 & CODE_SOLID) != 0, sol1 = (c1 & CODE_SOLID) != 0;
    const bool inlet = x0 == 0, outlet = x0 + 1 == nx - 1;
    const bool wsol0 = a.mac_all || row_shell || x0 == 1 || x0 == nx - 2;
    const bool wsol1 = outlet ? a.mac_all : (a.mac_all || row_shell || x0 + 1 == 1 || x0 + 1 == nx - 2);
    if (sol0 && sol1) {
        if (wsol0) store_mac(a.mac_cur, idx0, (T)0.0, (T)0.0, (T)0.0, (T)1.0);
        if (wsol1) store_mac(a.mac_cur, idx0 + 1, (T)0.0, (T)0.0, (T)0.0, (T)1.0);
        solid_macro(mo[0]);
        solid_macro(mo[1]);
        return;
    }
    if ((c0 | c1) & CODE_NEAR) pair_walls<PREC, FAST>(a, idx0, c0, c1, f);
    T m[2][4];
    collide_two<P, FAST>(a, f, x0, m);
    if (sol0) {  // a solid cell's macro values are (0, 0, 0, 1); the outlet may read them
        m[0][0] = (T)0.0; m[0][1] = (T)0.0; m[0][2] = (T)0.0; m[0][3] = (T)1.0;
    }
    if (inlet && !sol0) {
        eq_values<P, FAST>(a, (T)1.0, a.uin, (T)0.0, (T)0.0, f[0]);
        m[0][0] = a.uin; m[0][1] = (T)0.0; m[0][2] = (T)0.0; m[0][3] = (T)1.0;
    }
    if (outlet && !sol1) {
        T br, bux, buy, buz;
        face_values<T>(nx - 1, y, z, nx, a.ny, a.nz, a.uin, m[0][0], m[0][1], m[0][2], m[0][3], br, bux, buy, buz);
        eq_values<P, FAST>(a, br, bux, buy, buz, f[1]);
        m[1][0] = bux; m[1][1] = buy; m[1][2] = buz; m[1][3] = br;
    }
    typename P::S* ob = a.dst[0] + idx0;  // population i of the output is at ob + i n
    if (!sol0 && !sol1) {
        unroll<0, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            store_cells<P, FAST, 2, i>(a, sizeof(typename P::S) >= 4 ? a.dst[i] + idx0 : ob + (int64_t)i * a.n, f);
        });
    } else {
        const int32_t k = sol0 ? 1 : 0;  // the one fluid cell of the pair (selects, no indexing)
        unroll<0, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            st_out<P, FAST, i>(a, ob + (int64_t)i * a.n + k, sol0 ? f[1][i] : f[0][i]);
        });
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const bool sol = k ? sol1 : sol0;
        const int32_t x = x0 + k;
        bool w;
        if (sol) w = k ? wsol1 : wsol0;
        else if (x == 0 || x == nx - 1) w = a.mac_all;  // inlet / outlet
        else w = a.mac_all || row_shell || x == 1 || x == nx - 2;
        if (w) {
            if (sol) store_mac(a.mac_cur, idx0 + k, (T)0.0, (T)0.0, (T)0.0, (T)1.0);
            else store_mac(a.mac_cur, idx0 + k, m[k][0], m[k][1], m[k][2], m[k][3]);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) mo[k][c] = sol ? (c == 3 ? (T)1.0 : (T)0.0) : m[k][c];
    }
}
template <int PREC, bool FAST>
__device__ __forceinline__ void pair_finish(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                            int32_t idx0, int32_t x0, int32_t y, int32_t z, uint32_t codes,
                                            bool row_shell, typename Prec<PREC>::T (&f)[2][Q]) {
    typename Prec<PREC>::T mo[2][4];
    pair_finish<PREC, FAST>(a, idx0, x0, y, z, codes, row_shell, f, mo);
}

template <int PREC, bool FAST>
__device__ __forceinline__ void interior_pair(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                              int32_t idx0, int32_t x0, int32_t y, int32_t z, uint32_t codes,
                                              bool row_shell, typename Prec<PREC>::T (&mo)[2][4]) {
    using P = Prec<PREC>;
    using T = typename P::T;
    const bool sol0 = (codes & CODE_SOLID) != 0, sol1 = ((codes >> 8) & CODE_SOLID) != 0;
    T f[2][Q];
    if (!(sol0 && sol1)) {  // an all-solid pair pulls nothing
        PairRaw<typename P::S> r;
        pair_load<PREC>(a, idx0, r);
        pair_unpack<P, FAST>(a, r, f);
    }
    pair_finish<PREC, FAST>(a, idx0, x0, y, z, codes, row_shell, f, mo);
}
template <int PREC, bool FAST>
__device__ __forceinline__ void interior_pair(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                              int32_t idx0, int32_t x0, int32_t y, int32_t z, uint32_t codes,
                                              bool row_shell) {
    typename Prec<PREC>::T mo[2][4];
    interior_pair<PREC, FAST>(a, idx0, x0, y, z, codes, row_shell, mo);
}

// interior_pair with the pull issued together with the code bytes instead of after them, so
// the two loads' latencies overlap; an all-solid pair pulls too (and discards it)
template <int PREC, bool FAST>
__device__ __forceinline__ void interior_pair_early(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                                    int32_t idx0, int32_t x0, int32_t y, int32_t z, bool row_shell) {
    using P = Prec<PREC>;
    typename P::T f[2][Q], mo[2][4];
    PairRaw<typename P::S> r;
    pair_load<PREC>(a, idx0, r);
    pair_unpack<P, FAST>(a, r, f);
    pair_finish<PREC, FAST>(a, idx0, x0, y, z, r.codes, row_shell, f, mo);
}

template <int PREC, bool FAST, int V, bool EARLY = false>
__device__ __forceinline__ void bulk_cells(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                           int32_t idx0, bool valid) {
    using P = Prec<PREC>;
    using T = typename P::T;
    using S = typename P::S;
    const int32_t nx = a.nx, ny = a.ny, nz = a.nz;
    const int32_t row = (int32_t)a.dnx.div((uint32_t)(valid ? idx0 : 0));
    const int32_t x0 = (valid ? idx0 : 0) - row * nx;
    const int32_t z = (int32_t)a.dny.div((uint32_t)row);
    const int32_t y = row - z * ny;
    const bool face_row = y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
    const bool row_shell = !face_row && (y == 1 || y == ny - 2 || z == 1 || z == nz - 2);
    if constexpr (V == 2 && EARLY) {
        if (valid && !face_row) {
            interior_pair_early<PREC, FAST>(a, idx0, x0, y, z, row_shell);
            return;
        }
    }
    T mx = (T)0.0, my = (T)0.0, mz = (T)0.0, mr = (T)1.0;  // macro values of the latest cell
    uint32_t codes = 0;
    if (valid) {
        if constexpr (V == 4) codes = *reinterpret_cast<const uint32_t*>(a.code + idx0);
        else if constexpr (V == 2) codes = *reinterpret_cast<const uint16_t*>(a.code + idx0);
        else codes = a.code[idx0];
    }
    if constexpr (V == 2) {
        if (valid && !face_row) {
            interior_pair<PREC, FAST>(a, idx0, x0, y, z, codes, row_shell);
            return;
        }
    }
    if (valid && !face_row && x0 > 0 && x0 + V <= nx - 2 + (V == 1) && codes == 0) {
        // ---- fast path: V plain interior fluid cells, vector loads and stores ----
        T f[V][Q];
        unroll<0, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            const S* p = a.src[i] + idx0;
            if constexpr (V == 1) {
                f[0][i] = ld_in<P, FAST, i>(a, p);
            } else {
                const SVec<S, V> v = vload<S, V>(p + cx(i));  // aligned: the shift cancels
                if constexpr (cx(i) == 0) {
#pragma unroll
                    for (int k = 0; k < V; ++k) f[k][i] = ld_in<P, FAST, i>(a, &v.v[k]);
                } else if constexpr (cx(i) > 0) {
                    f[0][i] = ld_in<P, FAST, i>(a, p);
#pragma unroll
                    for (int k = 1; k < V; ++k) f[k][i] = ld_in<P, FAST, i>(a, &v.v[k - 1]);
                } else {
#pragma unroll
                    for (int k = 0; k < V - 1; ++k) f[k][i] = ld_in<P, FAST, i>(a, &v.v[k + 1]);
                    f[V - 1][i] = ld_in<P, FAST, i>(a, p + V - 1);
                }
            }
        });
        collide_cells<P, FAST, V>(a, f, idx0, x0, row_shell, mx, my, mz, mr);
        unroll<0, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            store_cells<P, FAST, V, i>(a, a.dst[i] + idx0, f);
        });
    } else if (valid) {
        // ---- general path: cell by cell (faces, inlet, outlet, solids, cells next to solids) ----
#pragma unroll 1
        for (int k = 0; k < V; ++k) {
            const uint32_t code = (codes >> (8 * k)) & 0xffu;
            if (V > 1 && !face_row && x0 + k == nx - 1) {
                // its x = nx-2 neighbour is this thread's previous cell
                outlet_cell<P>(a, idx0 + k, y, z, code, mx, my, mz, mr);
            } else {
                general_cell<P, FAST>(a, idx0 + k, x0 + k, y, z, code, face_row, row_shell, mx, my, mz, mr);
            }
        }
    }
    if constexpr (V == 1) {
        // outlet with one cell per thread: nx is even, so the outlet index is odd and never
        // starts a warp; its x = nx-2 neighbour is the previous lane
        const T qx = __shfl_up_sync(0xffffffffu, mx, 1);
        const T qy = __shfl_up_sync(0xffffffffu, my, 1);
        const T qz = __shfl_up_sync(0xffffffffu, mz, 1);
        const T qr = __shfl_up_sync(0xffffffffu, mr, 1);
        if (valid && !face_row && x0 == nx - 1) outlet_cell<P>(a, idx0, y, z, codes, qx, qy, qz, qr);
    }
}

template <int PREC, bool FAST, int V, int BLOCK, int MINB, bool EARLY = false>
__global__ void __launch_bounds__(BLOCK, MINB) k_step_bulk(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T> a) {
    const int32_t idx0 = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x) * V;
    bulk_cells<PREC, FAST, V, EARLY>(a, idx0, idx0 < a.n);
}

// Face cell number t of the tunnel's k_step_faces set (z = nz-1 plane, then the y = ny-1
// rows of interior z).
template <int PREC>
__device__ __forceinline__ void face_cell(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                          int32_t t) {
    using P = Prec<PREC>;
    using T = typename P::T;
    const int32_t nx = a.nx, ny = a.ny, nz = a.nz;
    const int32_t nplane = a.nxy, nrows = nx * (nz - 2);
    if (t >= nplane + nrows) return;
    int32_t x, y, z;
    if (t < nplane) {  // z = nz-1 plane
        z = nz - 1;
        y = (int32_t)a.dnx.div((uint32_t)t);
        x = t - y * nx;
    } else {  // y = ny-1 rows of interior z
        const int32_t t2 = t - nplane;
        const int32_t r = (int32_t)a.dnx.div((uint32_t)t2);
        z = 1 + r;
        y = ny - 1;
        x = t2 - r * nx;
    }
    if (x == 0) return;
    const int32_t idx = x + nx * (y + ny * z);
    if (a.code[idx] & CODE_SOLID) {
        if (a.mac_all) store_mac(a.mac_cur, idx, (T)0.0, (T)0.0, (T)0.0, (T)1.0);
        return;
    }
    const int32_t cxi = min(max(x, 1), nx - 2), cyi = min(max(y, 1), ny - 2), czi = min(max(z, 1), nz - 2);
    T px, py, pz, pr, br, bux, buy, buz;
    load_mac(a.mac_cur, cxi + nx * (cyi + ny * czi), px, py, pz, pr);
    face_values<T>(x, y, z, nx, ny, nz, a.uin, px, py, pz, pr, br, bux, buy, buz);
    face_eq<P>(a, idx, br, bux, buy, buz);
    if (a.mac_all) store_mac(a.mac_cur, idx, bux, buy, buz, br);
}

template <int PREC>
__global__ void __launch_bounds__(256) k_step_faces(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T> a) {
    face_cell<PREC>(a, (int32_t)(blockIdx.x * blockDim.x + threadIdx.x));
}

// ---------------------------------------------------------------------------------
// Row-grid form of the two-cell tile. The grid is (x-runs, ny, nz): a block covers 2 * BLOCK
// consecutive cells of one lattice row, so the row's y and z come from the block index (no
// division) and the face-row and shell-row tests are uniform over the block. A warp of an
// interior row whose 64 cells are all fluid takes a lean path: pull, pair collision and stores,
// with the few lanes next to a wall, at the inlet or at the outlet applying their boundary
// rule as a per-lane override (pair_walls, eq_values), as pair_finish does. A warp holding a
// solid cell runs interior_pair, and face rows run bulk_cells, so the results are bit for bit
// those of the one-dimensional two-cell tiles.
//
// Addressing (ADDR): 0 -- population i is pulled from src[i] + idx0 and stored to
// dst[i] + idx0, one wide multiply-add of a kernel-parameter base per population; 1 -- from one
// per-thread base fin + idx0 plus a per-population byte offset computed on the host
// (RowArgs::loff, soff), one 64-bit add per population.
// ---------------------------------------------------------------------------------
template <class S, class T>
struct RowArgs {
    StepArgs<S, T> a;
    int64_t loff[Q];  // bytes from fin + idx0 to the aligned pull pair of population i
    int64_t soff[Q];  // bytes from fout + idx0 to population i of the output
};

template <int PREC, bool FAST>
__device__ __forceinline__ void pair_lean_finish(const RowArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& r,
                                                 typename Prec<PREC>::T (&f)[2][Q], int32_t idx0, int32_t x0,
                                                 int32_t y, int32_t z, uint32_t codes, bool row_shell, bool offs,
                                                 typename Prec<PREC>::T (&mo)[2][4]);

template <int PREC, bool FAST, int ADDR>
__device__ __forceinline__ void pair_lean(const RowArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& r,
                                          int32_t idx0, int32_t x0, int32_t y, int32_t z, uint32_t codes,
                                          bool row_shell, typename Prec<PREC>::T (&mo)[2][4]) {
    using P = Prec<PREC>;
    using S = typename P::S;
    using T = typename P::T;
    const auto& a = r.a;
    const char* fb = reinterpret_cast<const char*>(a.fin) + (int64_t)idx0 * (int64_t)sizeof(S);
    T f[2][Q];
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        // the aligned pair holding the pull sources of both cells but for the x-shifted one; the
        // shifted one lies just outside it, inside the row: x0 - 1 >= 0 when cx > 0 pulls into
        // x0 > 0, and the inlet cell x0 = 0 has a source at x = -1 only in its own (discarded)
        // pull, which reads the previous row's last cell, still inside the buffer
        const S* p = ADDR == 0 ? a.src[i] + idx0 + cx(i) : reinterpret_cast<const S*>(fb + r.loff[i]);
        const SVec<S, 2> v = vload<S, 2>(p);
        if constexpr (cx(i) == 0) {
            f[0][i] = ld_in<P, FAST, i>(a, &v.v[0]);
            f[1][i] = ld_in<P, FAST, i>(a, &v.v[1]);
        } else if constexpr (cx(i) > 0) {
            f[0][i] = ld_in<P, FAST, i>(a, p - 1);
            f[1][i] = ld_in<P, FAST, i>(a, &v.v[0]);
        } else {
            f[0][i] = ld_in<P, FAST, i>(a, &v.v[1]);
            f[1][i] = ld_in<P, FAST, i>(a, p + 2);
        }
    });
    pair_lean_finish<PREC, FAST>(r, f, idx0, x0, y, z, codes, row_shell, ADDR == 1, mo);
}

// The lean path after the pull: walls, collision, inlet / outlet, stores and mac (see k_step_rows).
template <int PREC, bool FAST>
__device__ __forceinline__ void pair_lean_finish(const RowArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& r,
                                                 typename Prec<PREC>::T (&f)[2][Q], int32_t idx0, int32_t x0,
                                                 int32_t y, int32_t z, uint32_t codes, bool row_shell, bool offs,
                                                 typename Prec<PREC>::T (&mo)[2][4]) {
    using P = Prec<PREC>;
    using S = typename P::S;
    using T = typename P::T;
    const auto& a = r.a;
    const int32_t nx = a.nx;
    const uint32_t c0 = codes & 0xffu, c1 = codes >> 8;
    if ((c0 | c1) & CODE_NEAR) pair_walls<PREC, FAST>(a, idx0, c0, c1, f);  // lanes next to a wall
    T m[2][4];
    collide_two<P, FAST>(a, f, x0, m);
    const bool inlet = x0 == 0, outlet = x0 + 2 == nx;
    if (inlet) {  // x = 0: the inlet equilibrium replaces the collision (server/lbm.py:96-99)
        eq_values<P, FAST>(a, (T)1.0, a.uin, (T)0.0, (T)0.0, f[0]);
        m[0][0] = a.uin; m[0][1] = (T)0.0; m[0][2] = (T)0.0; m[0][3] = (T)1.0;
    } else if (outlet) {  // x = nx-1: the outlet from its x = nx-2 neighbour (server/lbm.py:100-103)
        T br, bux, buy, buz;
        face_values<T>(nx - 1, y, z, nx, a.ny, a.nz, a.uin, m[0][0], m[0][1], m[0][2], m[0][3], br, bux, buy, buz);
        eq_values<P, FAST>(a, br, bux, buy, buz, f[1]);
        m[1][0] = bux; m[1][1] = buy; m[1][2] = buz; m[1][3] = br;
    }
    char* ob = reinterpret_cast<char*>(a.dst[0]) + (int64_t)idx0 * (int64_t)sizeof(S);
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        store_cells<P, FAST, 2, i>(a, offs ? reinterpret_cast<S*>(ob + r.soff[i]) : a.dst[i] + idx0, f);
    });
    // mac where faces read it (coordinates 1 and n-2), and everywhere when mac_all
    const bool w0 = a.mac_all || (!inlet && (row_shell || x0 == nx - 2));
    const bool w1 = a.mac_all || (!outlet && (row_shell || inlet));
    if (w0) store_mac(a.mac_cur, idx0, m[0][0], m[0][1], m[0][2], m[0][3]);
    if (w1) store_mac(a.mac_cur, idx0 + 1, m[1][0], m[1][1], m[1][2], m[1][3]);
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int c = 0; c < 4; ++c) mo[k][c] = m[k][c];
}

// The face cells that read this step's mac (k_step_faces: the y = ny-1 rows of interior z and the
// z = nz-1 plane, x > 0) take it from one interior row each: a face cell at (x, y, z) reads the
// cell (clamp(x), clamp(y), clamp(z)) clamped to the interior, and for these rows that is the row
// (ny-2, z), (y, nz-2), (1, nz-2) or (ny-2, nz-2). With FUSE, the block of that interior row
// computes them from its pair's own macro values right after the pair, so no separate kernel
// (nor its launch and tail) is needed; the arithmetic is face_cell's, so the bits are too.
// Face row (fy, fz), pair x0 (both cells of the row x0, x0 + 1), from the interior pair's values m.
template <int PREC, bool FAST>
__device__ __forceinline__ void fused_face_pair(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                                int32_t x0, int32_t fy, int32_t fz,
                                                const typename Prec<PREC>::T (&m)[2][4]) {
    using P = Prec<PREC>;
    using T = typename P::T;
    const int32_t nx = a.nx;
    const int32_t fidx = x0 + nx * (fy + a.ny * fz);
    const uint32_t codes = *reinterpret_cast<const uint16_t*>(a.code + fidx);
    T fv[2][Q], fm[2][4];
    bool fluid[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int32_t x = x0 + k;
        const int j = x <= nx - 2 ? k : 0;  // clamp(x) to nx - 2: the pair's cell x0 (x = nx - 1)
        fluid[k] = x > 0 && ((codes >> (8 * k)) & CODE_SOLID) == 0;  // x = 0: the face row's own block
        face_values<T>(x, fy, fz, nx, a.ny, a.nz, a.uin, m[j][0], m[j][1], m[j][2], m[j][3], fm[k][3], fm[k][0],
                       fm[k][1], fm[k][2]);
        if (fluid[k]) eq_values<P, FAST>(a, fm[k][3], fm[k][0], fm[k][1], fm[k][2], fv[k]);
    }
    typename P::S* ob = a.dst[0] + fidx;
    if (fluid[0] && fluid[1]) {
        unroll<0, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            store_cells<P, FAST, 2, i>(a, ob + (int64_t)i * a.n, fv);
        });
    } else if (fluid[0] || fluid[1]) {
        const int32_t k = fluid[0] ? 0 : 1;
        unroll<0, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            st_out<P, FAST, i>(a, ob + (int64_t)i * a.n + k, fluid[0] ? fv[0][i] : fv[1][i]);
        });
    }
    if (a.mac_all) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (x0 + k == 0) continue;
            if (fluid[k]) store_mac(a.mac_cur, fidx + k, fm[k][0], fm[k][1], fm[k][2], fm[k][3]);
            else store_mac(a.mac_cur, fidx + k, (T)0.0, (T)0.0, (T)0.0, (T)1.0);
        }
    }
}

// The pull of a pair of an interior row in the lean path's addressing (ADDR), with the pair's
// code bytes: the same values as pair_load.
template <int PREC, int ADDR>
__device__ __forceinline__ void pair_load_rows(const RowArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& r,
                                               int32_t idx0, PairRaw<typename Prec<PREC>::S>& o) {
    using S = typename Prec<PREC>::S;
    const auto& a = r.a;
    o.codes = *reinterpret_cast<const uint16_t*>(a.code + idx0);
    const char* fb = reinterpret_cast<const char*>(a.fin) + (int64_t)idx0 * (int64_t)sizeof(S);
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        const S* p = ADDR == 0 ? a.src[i] + idx0 + cx(i) : reinterpret_cast<const S*>(fb + r.loff[i]);
        o.v[i] = vload<S, 2>(p);
        if constexpr (cx(i) > 0) o.e[i] = p[-1];
        if constexpr (cx(i) < 0) o.e[i] = p[2];
    });
}

// One block of the row grid: x-run bx of lattice row (y, z).
template <int PREC, bool FAST, int BLOCK, int ADDR, bool FUSE, bool EARLY>
__device__ __forceinline__ void row_tile(const RowArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& r,
                                         int32_t bx, int32_t y, int32_t z) {
    using T = typename Prec<PREC>::T;
    const auto& a = r.a;
    const int32_t nx = a.nx, ny = a.ny, nz = a.nz;
    const int32_t x0 = (bx * BLOCK + (int32_t)threadIdx.x) * 2;
    const bool valid = x0 < nx;
    const int32_t idx0 = x0 + nx * (y + ny * z);
    if (y == 0 || y == ny - 1 || z == 0 || z == nz - 1) {  // a face row (uniform over the block)
        bulk_cells<PREC, FAST, 2>(a, idx0, valid);
        return;
    }
    const bool row_shell = y == 1 || y == ny - 2 || z == 1 || z == nz - 2;
    T m[2][4];
    if constexpr (EARLY) {
        // the pull goes out with the code bytes, not after the vote on them, so the two loads'
        // latencies overlap; both paths take the same pulled values
        PairRaw<typename Prec<PREC>::S> pr;
        uint32_t codes = 0xffffu;
        if (valid) {
            pair_load_rows<PREC, ADDR>(r, idx0, pr);
            codes = pr.codes;
        }
        if (__all_sync(0xffffffffu, (codes & (CODE_SOLID * 0x0101u)) == 0)) {
            T f[2][Q];
            pair_unpack<Prec<PREC>, FAST>(a, pr, f);
            pair_lean_finish<PREC, FAST>(r, f, idx0, x0, y, z, codes, row_shell, ADDR == 1, m);
        } else if (valid) {
            T f[2][Q];
            pair_unpack<Prec<PREC>, FAST>(a, pr, f);  // an all-solid pair's values go unused
            pair_finish<PREC, FAST>(a, idx0, x0, y, z, codes, row_shell, f, m);
        }
    } else {
        const uint32_t codes = valid ? *reinterpret_cast<const uint16_t*>(a.code + idx0) : 0xffffu;
        // lean unless a cell of the warp is solid (or past the row's end)
        if (__all_sync(0xffffffffu, (codes & (CODE_SOLID * 0x0101u)) == 0)) {
            pair_lean<PREC, FAST, ADDR>(r, idx0, x0, y, z, codes, row_shell, m);
        } else if (valid) {
            interior_pair<PREC, FAST>(a, idx0, x0, y, z, codes, row_shell, m);
        }
    }
    if constexpr (FUSE) {
        if (valid && (y == ny - 2 || z == nz - 2)) {  // uniform over the block
            if (y == ny - 2) fused_face_pair<PREC, FAST>(a, x0, ny - 1, z, m);
            if (z == nz - 2) {
                fused_face_pair<PREC, FAST>(a, x0, y, nz - 1, m);
                if (y == 1) fused_face_pair<PREC, FAST>(a, x0, 0, nz - 1, m);
                if (y == ny - 2) fused_face_pair<PREC, FAST>(a, x0, ny - 1, nz - 1, m);
            }
        }
    }
}

template <int PREC, bool FAST, int BLOCK, int MINB, int ADDR, bool FUSE = false, bool EARLY = false>
__global__ void __launch_bounds__(BLOCK, MINB) k_step_rows(const RowArgs<typename Prec<PREC>::S, typename Prec<PREC>::T> r) {
    row_tile<PREC, FAST, BLOCK, ADDR, FUSE, EARLY>(r, (int32_t)blockIdx.x, (int32_t)blockIdx.y, (int32_t)blockIdx.z);
}

// ---------------------------------------------------------------------------------
// Streaming form of the bulk kernel: shared-memory staging through bulk async copies.
//
// With pull streaming, the destination cells [c0, c0 + L) read population i from the
// contiguous source range src[i][c0 .. c0 + L): every population of a chunk of cells is
// one 1-D bulk copy (cp.async.bulk, no tensor map, no multicast). The copy starts at the
// 16-byte boundary at or below the range (chunk_src[i] = src[i] - chunk_r[i]) and is one
// vector longer, so the cell at chunk offset c is stage[i][chunk_r[i] + c].
//
// Warp-specialised pipeline of NS stages per CTA: warp 0 is the producer (one lane issues
// the 19 population copies and the chunk's code bytes into a free stage and arms the
// stage's "full" mbarrier with the byte count); the other warps consume (wait on "full",
// update their cells from shared memory, store to global memory, then arrive on the
// stage's "empty" mbarrier). There is no CTA-wide barrier in the loop, so a consumer warp
// slowed by boundary cells does not hold the others back. Persistent CTAs walk chunks
// blockIdx.x + j*gridDim.x. Every wait is bounded; a wait that gives up sets the tunnel's
// status word to WT_ERR_TIMEOUT and the warp leaves.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// try_wait suspends the thread until the phase completes or ~SUSPEND_NS elapse
constexpr uint32_t SUSPEND_NS = 1000;
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "n"(SUSPEND_NS)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded waits. The suspend hint of try_wait is only an upper bound (a try may return early),
// so the limit is time on the GPU's global nanosecond timer: a wait gives up WAIT_NS after its
// first unsuccessful try. WAIT_TRIES also caps the tries (about a second at 30 ns a try), so a
// wait ends even if the timer were to stand still. DRAIN_NS is the longer limit for copies
// that were already issued and are only being waited out before the CTA exits.
constexpr uint64_t WAIT_NS = 1000000000ull;
constexpr uint64_t DRAIN_NS = 10000000000ull;
constexpr uint32_t WAIT_TRIES = 1u << 25;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = WAIT_NS) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    const uint32_t tries = limit_ns > WAIT_NS ? WAIT_TRIES * (uint32_t)(limit_ns / WAIT_NS > 16 ? 16 : limit_ns / WAIT_NS)
                                              : WAIT_TRIES;
    for (uint32_t it = 0; it < tries; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
    return false;
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

template <class S>
__device__ __forceinline__ S lds(const S* p) {
    static_assert(sizeof(S) == 1 || sizeof(S) == 2 || sizeof(S) == 4 || sizeof(S) == 8, "lds width");
    const uint32_t a = smem_u32(p);
    if constexpr (sizeof(S) == 1) {
        unsigned short v;
        asm volatile("ld.shared.u8 %0, [%1];" : "=h"(v) : "r"(a));
        return (S)v;
    } else if constexpr (sizeof(S) == 4) {
        float v;
        asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
        return *reinterpret_cast<S*>(&v);
    } else if constexpr (sizeof(S) == 2) {
        unsigned short v;
        asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(a));
        return *reinterpret_cast<S*>(&v);
    } else {
        double v;
        asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
        return *reinterpret_cast<S*>(&v);
    }
}
template <class S>
__device__ __forceinline__ void sts(S* p, S v) {
    static_assert(sizeof(S) == 2 || sizeof(S) == 4 || sizeof(S) == 8, "sts width");
    const uint32_t a = smem_u32(p);
    if constexpr (sizeof(S) == 4) {
        asm volatile("st.shared.b32 [%0], %1;" ::"r"(a), "r"(*reinterpret_cast<uint32_t*>(&v)) : "memory");
    } else if constexpr (sizeof(S) == 2) {
        asm volatile("st.shared.b16 [%0], %1;" ::"r"(a), "h"(*reinterpret_cast<unsigned short*>(&v)) : "memory");
    } else {
        asm volatile("st.shared.b64 [%0], %1;" ::"r"(a), "l"(*reinterpret_cast<unsigned long long*>(&v)) : "memory");
    }
}

template <class S>
__device__ __forceinline__ SVec<S, 2> lds_pair(const S* p) {  // p aligned to 2 elements
    SVec<S, 2> r;
    const uint32_t a = smem_u32(p);
    if constexpr (sizeof(S) == 2) {
        uint32_t v;
        asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(a));
        memcpy(&r, &v, 4);
    } else if constexpr (sizeof(S) == 4) {
        uint2 v;
        asm volatile("ld.shared.v2.b32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(a));
        memcpy(&r, &v, 8);
    } else {
        uint4 v;
        asm volatile("ld.shared.v4.b32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
        memcpy(&r, &v, 16);
    }
    return r;
}
// the same from a shared-memory stage
template <class P, bool FAST, int I, class A>
__device__ __forceinline__ typename P::T ld_in_smem(const A& a, const typename P::S* p) {
    const typename P::S v = lds(p);
    return ld_in<P, FAST, I>(a, &v);
}

template <class S, int L>
struct StreamLayout {
    static constexpr int VEC = 16 / (int)sizeof(S);
    static constexpr int LP = L + VEC;                        // elements per population buffer
    static constexpr int POP_BYTES = LP * (int)sizeof(S);     // multiple of 16
    static constexpr int STAGE_BYTES = Q * POP_BYTES + L;     // populations + code bytes
    static_assert(L % 16 == 0, "chunk length");
};

template <int PREC, int L>
__device__ __forceinline__ bool stream_issue(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>& a,
                                             unsigned char* stage, uint64_t* full, int32_t chunk) {
    using S = typename Prec<PREC>::S;
    using LY = StreamLayout<S, L>;
    if (chunk + 1 == a.test_skip_chunk) return false;  // test hook: leave the stage empty
    const int32_t c0 = chunk * L;
    const int32_t len = min(L, a.n - c0);
    const int32_t len16 = (len + LY::VEC - 1) / LY::VEC * LY::VEC;
    const uint32_t pop_bytes = (uint32_t)((len16 + LY::VEC) * (int)sizeof(S));
    const uint32_t code_bytes = (uint32_t)((len + 15) / 16 * 16);
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(full, Q * pop_bytes + code_bytes);
#pragma unroll 1
    for (int i = 0; i < Q; ++i) bulk_g2s(stage + i * LY::POP_BYTES, a.chunk_src[i] + c0, pop_bytes, full);
    bulk_g2s(stage + Q * LY::POP_BYTES, a.code + c0, code_bytes, full);
    return true;
}

template <int PREC, bool FAST, int L, int NS, int THREADS, int MINB, int CPT>
__global__ void __launch_bounds__(THREADS, MINB) k_step_stream(const StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T> a) {
    using P = Prec<PREC>;
    using T = typename P::T;
    using S = typename P::S;
    using LY = StreamLayout<S, L>;
    constexpr int CONSUMERS = THREADS / 32 - 1;  // consumer warps
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + NS * LY::STAGE_BYTES);
    uint64_t* empty = full + NS;
    const int32_t nchunks = (a.n + L - 1) / L;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int st = 0; st < NS; ++st) {
            mbar_init(&full[st], 1);
            mbar_init(&empty[st], CONSUMERS);
        }
        mbar_fence_init();
    }
    __syncthreads();  // the only CTA-wide barrier: barriers initialised

    if (warp == 0) {
        // ---- producer ----
        if (lane != 0) return;
        int32_t issued_lo = 0, j = 0;  // chunks [issued_lo, j) issued and possibly unconsumed
        for (;; ++j) {
            const int32_t k = blockIdx.x + j * gridDim.x;
            if (k >= nchunks) break;
            const int st = j % NS;
            if (j >= NS) {
                if (!mbar_wait(&empty[st], (uint32_t)(((j / NS) - 1) & 1))) {
                    if (a.status) atomicExch(a.status, WT_ERR_TIMEOUT);
                    break;
                }
                issued_lo = j - NS + 1;
            }
            if (!stream_issue<PREC, L>(a, smem + (size_t)st * LY::STAGE_BYTES, &full[st], k)) continue;
        }
        // Keep the CTA's shared memory alive until every issued copy has landed. Issued copies
        // always complete, so this waits DRAIN_NS (ten times the pipeline's limit) before it
        // gives up; if it ever does, the tunnel is marked failed, because a copy could then
        // still land in shared memory the CTA no longer owns.
        for (int32_t q = issued_lo; q < j; ++q) {
            const int32_t k = blockIdx.x + q * gridDim.x;
            if (k + 1 == a.test_skip_chunk) continue;
            if (!mbar_wait(&full[q % NS], (uint32_t)((q / NS) & 1), DRAIN_NS) && a.status)
                atomicExch(a.status, WT_ERR_TIMEOUT);
        }
        return;
    }

    // ---- consumers ----
    // Consumer thread ct owns CPT consecutive cells of each chunk (L = 32 * CONSUMERS * CPT),
    // so a warp reads and writes contiguous runs; with CPT = 2 loads and stores are pairs.
    static_assert(L == 32 * CONSUMERS * CPT, "chunk = consumer threads x cells per thread");
    static_assert(L % 32 == 0, "chunk starts at a warp boundary (outlet shuffle)");
    const int ct = threadIdx.x - 32;
    const int32_t nx = a.nx, ny = a.ny, nz = a.nz;
#pragma unroll 1
    for (int32_t j = 0;; ++j) {
        const int32_t k = blockIdx.x + j * gridDim.x;
        if (k >= nchunks) break;
        const int st = j % NS;
        if (!__all_sync(0xffffffffu, mbar_wait(&full[st], (uint32_t)((j / NS) & 1)))) {
            // the stage never filled: report and leave (the tunnel is invalid until reset)
            if (a.status && lane == 0) atomicExch(a.status, WT_ERR_TIMEOUT);
            return;
        }
        const unsigned char* stage = smem + (size_t)st * LY::STAGE_BYTES;
        const uint8_t* codes = stage + Q * LY::POP_BYTES;
        const int32_t c0 = k * L;
        const int32_t len = min(L, a.n - c0);
        const int32_t c = ct * CPT;
        const bool valid = c < len;  // len is a multiple of 16, so all CPT cells are in range
        T mx = (T)0.0, my = (T)0.0, mz = (T)0.0, mr = (T)1.0;  // macro values of the latest cell
        int32_t idx = 0, x = 0, y = 0, z = 0;
        bool face_row = true;
        uint32_t code = 0;
        if (valid) {
            idx = c0 + c;
            const int32_t row = (int32_t)a.dnx.div((uint32_t)idx);
            x = idx - row * nx;  // nx is a multiple of CPT: the cells share the row
            z = (int32_t)a.dny.div((uint32_t)row);
            y = row - z * ny;
            face_row = y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
            const bool row_shell = !face_row && (y == 1 || y == ny - 2 || z == 1 || z == nz - 2);
            if constexpr (CPT == 1) code = lds(codes + c);
            else code = lds(reinterpret_cast<const uint16_t*>(codes + c));
            if (CPT == 2 && !face_row) {
                // every cell kind of an interior row: the pair path (see pair_finish)
                T f[2][Q];
                unroll<0, Q>([&](auto ic) {
                    constexpr int i = decltype(ic)::value;
                    const S* sp = reinterpret_cast<const S*>(stage + i * LY::POP_BYTES) + a.chunk_r[i] + c;
                    if constexpr (cx(i) == 0) {  // chunk_r[i] == 0: an aligned pair
                        const SVec<S, 2> v = lds_pair(sp);
                        f[0][i] = ld_in<P, FAST, i>(a, &v.v[0]);
                        f[1][i] = ld_in<P, FAST, i>(a, &v.v[1]);
                    } else {
                        f[0][i] = ld_in_smem<P, FAST, i>(a, sp);
                        f[1][i] = ld_in_smem<P, FAST, i>(a, sp + 1);
                    }
                });
                if constexpr (CPT == 2) pair_finish<PREC, FAST>(a, idx, x, y, z, code, row_shell, f);
            } else if (!face_row && x > 0 && x + CPT < nx && code == 0) {
                T f[CPT][Q];
                unroll<0, Q>([&](auto ic) {
                    constexpr int i = decltype(ic)::value;
                    const S* sp = reinterpret_cast<const S*>(stage + i * LY::POP_BYTES) + a.chunk_r[i] + c;
                    if constexpr (CPT == 1) {
                        f[0][i] = ld_in_smem<P, FAST, i>(a, sp);
                    } else if constexpr (cx(i) == 0) {  // chunk_r[i] == 0: an aligned pair
                        const SVec<S, 2> v = lds_pair(sp);
                        f[0][i] = ld_in<P, FAST, i>(a, &v.v[0]);
                        f[1][i] = ld_in<P, FAST, i>(a, &v.v[1]);
                    } else {
                        f[0][i] = ld_in_smem<P, FAST, i>(a, sp);
                        f[1][i] = ld_in_smem<P, FAST, i>(a, sp + 1);
                    }
                });
                collide_cells<P, FAST, CPT>(a, f, idx, x, row_shell, mx, my, mz, mr);
                unroll<0, Q>([&](auto ic) {
                    constexpr int i = decltype(ic)::value;
                    store_cells<P, FAST, CPT, i>(a, a.dst[i] + idx, f);
                });
            } else {
#pragma unroll 1
                for (int q = 0; q < CPT; ++q) {
                    const uint32_t cq = (code >> (8 * q)) & 0xffu;
                    if (CPT > 1 && !face_row && x + q == nx - 1)
                        outlet_cell<P>(a, idx + q, y, z, cq, mx, my, mz, mr);  // neighbour: cell q-1
                    else
                        general_cell<P, FAST>(a, idx + q, x + q, y, z, cq, face_row, row_shell, mx, my, mz, mr);
                }
            }
        }
        if constexpr (CPT == 1) {
            // outlet: chunk starts are multiples of 32 and the outlet index is odd, so its
            // x = nx-2 neighbour is the previous lane
            const T qx = __shfl_up_sync(0xffffffffu, mx, 1);
            const T qy = __shfl_up_sync(0xffffffffu, my, 1);
            const T qz = __shfl_up_sync(0xffffffffu, mz, 1);
            const T qr = __shfl_up_sync(0xffffffffu, mr, 1);
            if (valid && !face_row && x == nx - 1) outlet_cell<P>(a, idx, y, z, code, qx, qy, qz, qr);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[st]);  // this warp is done with the stage
    }
}

// SM count of the current device (the persistent kernels size their grids from it)
inline int num_sms() {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    return sms;
}

}  // namespace wt
