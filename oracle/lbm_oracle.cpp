// CPU restatement of the wind-tunnel LBM hot path -- TEST INFRASTRUCTURE ONLY.
//
// This is the oracle: the parity checker for the CUDA kernels and the timed CPU
// baseline. It is never part of the product path. Only tests/, the smoke check and
// bench.py's CPU-baseline/reference legs load it.
//
// It restates, operation for operation, the kernels of RICKxxROLLING/wind-tunnel
// server/lbm.py (NVIDIA Warp 1.17 kernels, written here in plain C++):
//   oracle_init_*     <- init_kernel      (generated, server/lbm.py:64-69)
//   oracle_step_*     <- step_kernel      (generated, server/lbm.py:72-166)
//   oracle_force_*    <- force_kernel     (generated, server/lbm.py:169-197)
//   oracle_advect_*   <- advect_kernel    (server/lbm.py:233-263, with cidx/sample_mac :201-230)
//   oracle_pack_*     <- pack_particles   (server/lbm.py:266-275)
//   oracle_slice_*    <- slice_kernel     (server/lbm.py:278-318, with vort)
//   oracle_cp_*       <- cp_kernel        (server/lbm.py:321-368, with rho_fluid)
// Every floating-point expression keeps the reference's association order (the
// generator's lin()/cu_expr() left-to-right sums, server/lbm.py:37-53) and the file is
// compiled with -ffp-contract=off, so the float instantiation is bit-identical to the
// reference kernels run serially (pinned against golden vectors made by
// oracle/warp_shim.py from the reference's own source).
//
// Face cells read mac[] of an interior neighbour that the same launch writes
// (server/lbm.py:87 vs :166). Warp's CPU backend runs tids in order, so a neighbour with a
// smaller linear index is already updated. oracle_step_serial_* reproduces that with a
// literal in-order loop; oracle_step_* computes the same result in parallel: it snapshots
// mac, updates every cell that does not need a current-step value, then the face cells
// whose neighbour index is smaller than their own.
//
// Storage variants (not in the reference): populations stored as fp16/bf16 shifted values
// f_i - w_i (rounded to nearest even on store), collision in float; and fp64 throughout.
//
// Particle respawn uses this project's counter-based RNG (PCG-RXS-M-XS output hash,
// Jarzynski & Olano, "Hash Functions for GPU Rendering", JCGT 2020), not Warp's
// wp.rand_init/randf, whose source is not part of the reference.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int Q = 19;
// D3Q19 velocity set in the reference's order (server/lbm.py:15-17)
constexpr int CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
constexpr int CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
constexpr int CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
constexpr int OPP[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};

// weights as the reference computes them in double (server/lbm.py:18)
inline double w_d(int i) {
    int s = std::abs(CX[i]) + std::abs(CY[i]) + std::abs(CZ[i]);
    return i == 0 ? 1.0 / 3.0 : (s == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
}

template <class T>
struct Consts {
    T w[Q], belt[Q], c45w[Q], a3[Q], b45[Q];
    Consts() {
        for (int i = 0; i < Q; ++i) {
            w[i] = (T)w_d(i);
            belt[i] = (T)(6.0 * w_d(i) * CX[i]);       // F(6 * W[i] * cx), :124
            c45w[i] = (T)(4.5 * w_d(i));               // F(4.5 * W[i]), :165
            a3[i] = (T)(3.0 * CX[i]);                  // F(3 * c[0]), :68
            b45[i] = (T)(4.5 * CX[i] * CX[i]);         // F(4.5 * c[0] ** 2), :68
        }
    }
};

// ---------------- storage conversions ----------------
// Tag types select the population storage; Real is the arithmetic type.
struct StF32 { using Store = float; using Real = float; static constexpr bool shifted = false; };
struct StF64 { using Store = double; using Real = double; static constexpr bool shifted = false; };
struct StF16 { using Store = _Float16; using Real = float; static constexpr bool shifted = true; };
struct StBF16 { using Store = __bf16; using Real = float; static constexpr bool shifted = true; };

// Shift of the fp16/bf16 storage (the library's wt_grid.shift_u, restated): populations are
// stored as f_i - e_i, e_i = w_i (1 + 3 c_xi U + 4.5 c_xi^2 U^2 - 1.5 U^2) in double rounded to
// float; bb_i = e_opp(i) - e_i; dw_i = e_i - w_i; su, suu, s45, s15 = U, U^2, 4.5 U^2, 1.5 U^2.
// U = 0 gives e_i = w_i. Set by oracle_set_shift; applies to every later call.
struct ShiftState {
    float e[Q], bb[Q], dw[Q];
    float su, suu, s45, s15;
};
static ShiftState g_shift = [] {
    ShiftState t{};
    for (int i = 0; i < Q; ++i) t.e[i] = (float)w_d(i);
    return t;
}();

template <class St>
inline typename St::Real ld(const typename St::Store* f, int64_t n, int i, int64_t idx, const Consts<typename St::Real>& K) {
    using T = typename St::Real;
    if constexpr (St::shifted) return (T)f[(int64_t)i * n + idx] + (T)g_shift.e[i];
    else return (T)f[(int64_t)i * n + idx];
}
template <class St>
inline void st(typename St::Store* f, int64_t n, int i, int64_t idx, typename St::Real v, const Consts<typename St::Real>& K) {
    using S = typename St::Store;
    if constexpr (St::shifted) f[(int64_t)i * n + idx] = (S)(v - (typename St::Real)g_shift.e[i]);
    else f[(int64_t)i * n + idx] = (S)v;
}

// raw stored value (the fast collision works on deviations directly for shifted storage)
template <class St>
inline typename St::Real ldv(const typename St::Store* f, int64_t n, int i, int64_t idx) {
    return (typename St::Real)f[(int64_t)i * n + idx];
}
template <class St>
inline void stv(typename St::Store* f, int64_t n, int i, int64_t idx, typename St::Real v) {
    f[(int64_t)i * n + idx] = (typename St::Store)v;
}

template <class T>
inline T clampT(T x, T a, T b) { return std::min(std::max(x, a), b); }

template <class T>
inline T fmaT(T a, T b, T c) { return std::fma(a, b, c); }

// Moment-space form of the regularized Smagorinsky collision: the same operation
// sequence as collide_fast in the CUDA library (wt_step.cu), so results are bit-identical.
// Mathematically equal to the reference collision; see the CUDA source for the derivation.
template <class T, bool SHIFT>
void collide_fast(T (&v)[Q], int x, int nx, T tau, T csmag, T& oux, T& ouy, T& ouz, T& orho) {
    const double wd0 = w_d(0), wd1 = w_d(1), wd7 = w_d(7);
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
    // shifted storage: the shift's own moments (+ U^2 in xx, + U in jx) restored
    const T xxx0 = (s1 + d7) + d11, xyy = (s3 + d7) + d15, xzz = (s5 + d11) + d15;
    const T xxx = SHIFT ? xxx0 + (T)g_shift.suu : xxx0;
    const T xxy = s7 - s9, xxz = s11 - s13, xyz = s15 - s17;
    const T S = ((v[0] + s1) + (s3 + s5)) + ((d7 + d11) + d15);
    const T jx0 = ((a1 + a7) + (a9 + a11)) + a13;
    const T jx = SHIFT ? jx0 + (T)g_shift.su : jx0;
    const T jy = ((a3 + a7) - (a9 - a15)) + a17;
    const T jz = ((a5 + a11) - (a13 - a15)) - a17;
    const T rho = SHIFT ? S + (T)1.0 : S;
    const T ir = (T)1.0 / rho;
    T ux = jx * ir, uy = jy * ir, uz = jz * ir;
    T usq = fmaT(uz, uz, fmaT(uy, uy, ux * ux));
    if (usq > (T)0.1225) {
        const T sc = (T)0.35 / std::sqrt(usq);
        ux = ux * sc; uy = uy * sc; uz = uz * sc;
        usq = fmaT(uz, uz, fmaT(uy, uy, ux * ux));
    }
    const T rux = rho * ux, ruy = rho * uy, ruz = rho * uz;
    const T t3 = (SHIFT ? S : rho) * ((T)1.0 / (T)3.0);
    const T nxx = fmaT(-rux, ux, xxx - t3), nyy = fmaT(-ruy, uy, xyy - t3), nzz = fmaT(-ruz, uz, xzz - t3);
    const T nxy = fmaT(-rux, uy, xxy), nxz = fmaT(-rux, uz, xxz), nyz = fmaT(-ruy, uz, xyz);
    const T q1 = fmaT(nzz, nzz, fmaT(nyy, nyy, nxx * nxx));
    const T q2 = fmaT(nyz, nyz, fmaT(nxz, nxz, nxy * nxy));
    const T qn = std::sqrt(fmaT((T)2.0, q2, q1));
    T tau0 = tau;
    const T sp = (T)x - (T)(nx - 24);
    if (sp > (T)0.0) tau0 = fmaT(sp, (T)0.015, tau);
    const T tau_e = (T)0.5 * (tau0 + std::sqrt(fmaT(tau0, tau0, csmag * qn * ir)));
    const T keep = (T)1.0 - (T)1.0 / tau_e;
    const T k45 = (T)4.5 * keep, k9 = (T)9.0 * keep;
    const T axx = k45 * nxx, ayy = k45 * nyy, azz = k45 * nzz;
    const T axy = k9 * nxy, axz = k9 * nxz, ayz = k9 * nyz;
    const T tra3 = ((axx + ayy) + azz) * ((T)1.0 / (T)3.0);
    const T B0 = fmaT(-rho, (T)1.5 * usq, SHIFT ? S : rho) - tra3;
    const T B = SHIFT ? B0 + (T)g_shift.s15 : B0;
    // shifted storage: directions with c_x != 0 lose the shift's 3 c_x U and 4.5 U^2 terms
    const T s45 = (T)g_shift.s45, su_ = (T)g_shift.su;
    auto dsh = [&](T D) { return SHIFT ? D - s45 : D; };
    auto rsh = [&](T r) { return SHIFT ? r - su_ : r; };
    const T w0 = (T)wd0, w1 = (T)wd1, w2 = (T)wd7;
    const T w1x3 = (T)(3.0 * wd1), w2x3 = (T)(3.0 * wd7);
    v[0] = w0 * B;
    const T bxx = B + axx, byy = B + ayy;
    auto pair = [&](int i, T w, T wx3, T D, T rs) {
        const T E = wx3 * rs;
        v[i] = fmaT(w, D, E);
        v[i + 1] = fmaT(w, D, -E);
    };
    pair(1, w1, w1x3, dsh(fmaT((T)4.5 * rux, ux, bxx)), rsh(rux));
    pair(3, w1, w1x3, fmaT((T)4.5 * ruy, uy, byy), ruy);
    pair(5, w1, w1x3, fmaT((T)4.5 * ruz, uz, B + azz), ruz);
    const T pxy = bxx + ayy, pxz = bxx + azz, pyz = byy + azz;
    {
        const T su = ux + uy, rs = rux + ruy;
        pair(7, w2, w2x3, dsh(fmaT((T)4.5 * rs, su, pxy + axy)), rsh(rs));
    }
    {
        const T su = ux - uy, rs = rux - ruy;
        pair(9, w2, w2x3, dsh(fmaT((T)4.5 * rs, su, pxy - axy)), rsh(rs));
    }
    {
        const T su = ux + uz, rs = rux + ruz;
        pair(11, w2, w2x3, dsh(fmaT((T)4.5 * rs, su, pxz + axz)), rsh(rs));
    }
    {
        const T su = ux - uz, rs = rux - ruz;
        pair(13, w2, w2x3, dsh(fmaT((T)4.5 * rs, su, pxz - axz)), rsh(rs));
    }
    {
        const T su = uy + uz, rs = ruy + ruz;
        pair(15, w2, w2x3, fmaT((T)4.5 * rs, su, pyz + ayz), rs);
    }
    {
        const T su = uy - uz, rs = ruy - ruz;
        pair(17, w2, w2x3, fmaT((T)4.5 * rs, su, pyz - ayz), rs);
    }
    oux = ux; ouy = uy; ouz = uz; orho = rho;
}
inline int clampI(int x, int a, int b) { return std::min(std::max(x, a), b); }

// ---------------- init (server/lbm.py:64-69) ----------------
template <class St>
void init_impl(typename St::Store* f, typename St::Real* mac, int64_t n, typename St::Real uin) {
    using T = typename St::Real;
    static const Consts<T> K;
    T v[Q];
    for (int i = 0; i < Q; ++i)
        v[i] = K.w[i] * ((T)1.0 + K.a3[i] * uin + K.b45[i] * uin * uin - (T)1.5 * uin * uin);
#pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < n; ++idx) {
        for (int i = 0; i < Q; ++i) st<St>(f, n, i, idx, v[i], K);
        mac[4 * idx + 0] = uin; mac[4 * idx + 1] = 0; mac[4 * idx + 2] = 0; mac[4 * idx + 3] = 1;
    }
}

// ---------------- step (server/lbm.py:72-166) ----------------
template <class St>
struct StepArgs {
    using T = typename St::Real;
    const typename St::Store* fin;
    typename St::Store* fout;
    const uint8_t* solid;
    T* mac;            // written; in serial mode also read
    const T* mac_rd;   // values a face cell reads for a not-yet-updated neighbour
    int nx, ny, nz;
    int64_t n;
    T uin, tau, smag;
    int fast;  // 1: moment-space collision (collide_fast)
};

// One cell of step_kernel. `cur_mac` is where a face cell reads its neighbour's mac.
template <class St>
void step_cell(const StepArgs<St>& a, int64_t idx, int x, int y, int z, const typename St::Real* rd_mac) {
    using T = typename St::Real;
    static const Consts<T> K;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int64_t n = a.n;
    T* mac = a.mac;
    if (a.solid[idx] != 0) {
        mac[4 * idx + 0] = 0; mac[4 * idx + 1] = 0; mac[4 * idx + 2] = 0; mac[4 * idx + 3] = 1;
        return;
    }
    if (x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1) {
        int64_t j = clampI(x, 1, nx - 2) + (int64_t)nx * (clampI(y, 1, ny - 2) + (int64_t)ny * clampI(z, 1, nz - 2));
        const T* m = rd_mac + 4 * j;
        T br = clampT(m[3], (T)0.9, (T)1.1);
        T bux = m[0], buy = m[1], buz = m[2];
        if (y == 0 || y == ny - 1) buy = 0;
        if (z == 0 || z == nz - 1) buz = 0;
        if (x == 0) {
            br = 1; bux = a.uin; buy = 0; buz = 0;
        } else if (x == nx - 1) {
            br = 1; bux = std::max(bux, (T)0.0);
        }
        T bsq = (T)1.5 * (bux * bux + buy * buy + buz * buz);
        for (int i = 0; i < Q; ++i) {
            T s = 0;
            if (CX[i]) s = CX[i] > 0 ? s + bux : s - bux;
            if (CY[i]) s = CY[i] > 0 ? s + buy : s - buy;
            if (CZ[i]) s = CZ[i] > 0 ? s + buz : s - buz;
            T bc = (T)3.0 * s;
            st<St>(a.fout, n, i, idx, K.w[i] * br * ((T)1.0 + bc + (T)0.5 * bc * bc - bsq), K);
        }
        mac[4 * idx + 0] = bux; mac[4 * idx + 1] = buy; mac[4 * idx + 2] = buz; mac[4 * idx + 3] = br;
        return;
    }
    if (a.fast) {
        T v[Q];
        v[0] = ldv<St>(a.fin, n, 0, idx);
        const int64_t sy = nx, sz = (int64_t)nx * ny;
        for (int i = 1; i < Q; ++i) {
            int64_t s = idx - CX[i] - CY[i] * sy - CZ[i] * sz;
            int t = a.solid[s];
            if (t == 0) {
                v[i] = ldv<St>(a.fin, n, i, s);
            } else {
                v[i] = ldv<St>(a.fin, n, OPP[i], idx);
                if constexpr (St::shifted) v[i] = v[i] + (T)g_shift.bb[i];  // deviation: + e_opp - e_i
                if (CX[i] != 0 && t == 2) v[i] = v[i] + K.belt[i] * a.uin;
            }
        }
        T ux, uy, uz, rho;
        const T csmag = (T)25.4558441 * a.smag * a.smag;
        collide_fast<T, St::shifted>(v, x, nx, a.tau, csmag, ux, uy, uz, rho);
        for (int i = 0; i < Q; ++i) stv<St>(a.fout, n, i, idx, v[i]);
        mac[4 * idx + 0] = ux; mac[4 * idx + 1] = uy; mac[4 * idx + 2] = uz; mac[4 * idx + 3] = rho;
        return;
    }
    T f[Q];
    f[0] = ld<St>(a.fin, n, 0, idx, K);
    const int64_t sy = nx, sz = (int64_t)nx * ny;
    for (int i = 1; i < Q; ++i) {
        int64_t s = idx - CX[i] - CY[i] * sy - CZ[i] * sz;
        int t = a.solid[s];
        if (t == 0) {
            f[i] = ld<St>(a.fin, n, i, s, K);
        } else {
            f[i] = ld<St>(a.fin, n, OPP[i], idx, K);
            if (CX[i] != 0 && t == 2) f[i] = f[i] + K.belt[i] * a.uin;
        }
    }
    T rho = 0, jx = 0, jy = 0, jz = 0;
    for (int i = 0; i < Q; ++i) rho = rho + f[i];
    for (int i = 0; i < Q; ++i) if (CX[i]) jx = CX[i] > 0 ? jx + f[i] : jx - f[i];
    for (int i = 0; i < Q; ++i) if (CY[i]) jy = CY[i] > 0 ? jy + f[i] : jy - f[i];
    for (int i = 0; i < Q; ++i) if (CZ[i]) jz = CZ[i] > 0 ? jz + f[i] : jz - f[i];
    T ir = (T)1.0 / rho;
    T ux = jx * ir, uy = jy * ir, uz = jz * ir;
    T um = std::sqrt(ux * ux + uy * uy + uz * uz);
    if (um > (T)0.35) {
        T sc = (T)0.35 / um;
        ux = ux * sc; uy = uy * sc; uz = uz * sc;
    }
    T usq = (T)1.5 * (ux * ux + uy * uy + uz * uz);
    T e[Q], d[Q];
    for (int i = 0; i < Q; ++i) {
        T s = 0;
        if (CX[i]) s = CX[i] > 0 ? s + ux : s - ux;
        if (CY[i]) s = CY[i] > 0 ? s + uy : s - uy;
        if (CZ[i]) s = CZ[i] > 0 ? s + uz : s - uz;
        T cu = (T)3.0 * s;
        e[i] = K.w[i] * rho * ((T)1.0 + cu + (T)0.5 * cu * cu - usq);
        d[i] = f[i] - e[i];
    }
    T pxx = 0, pyy = 0, pzz = 0, pxy = 0, pxz = 0, pyz = 0;
    for (int i = 0; i < Q; ++i) {
        if (CX[i]) pxx = pxx + d[i];
        if (CY[i]) pyy = pyy + d[i];
        if (CZ[i]) pzz = pzz + d[i];
        int kxy = CX[i] * CY[i], kxz = CX[i] * CZ[i], kyz = CY[i] * CZ[i];
        if (kxy) pxy = kxy > 0 ? pxy + d[i] : pxy - d[i];
        if (kxz) pxz = kxz > 0 ? pxz + d[i] : pxz - d[i];
        if (kyz) pyz = kyz > 0 ? pyz + d[i] : pyz - d[i];
    }
    T qn = std::sqrt(pxx * pxx + pyy * pyy + pzz * pzz + (T)2.0 * (pxy * pxy + pxz * pxz + pyz * pyz));
    T tau0 = a.tau;
    T sp = (T)x - (T)nx + (T)24.0;
    if (sp > (T)0.0) tau0 = tau0 + sp * (T)0.015;
    T tau_e = (T)0.5 * (tau0 + std::sqrt(tau0 * tau0 + (T)25.4558441 * a.smag * a.smag * qn * ir));
    T keep = (T)1.0 - (T)1.0 / tau_e;
    T tr3 = (pxx + pyy + pzz) * ((T)1.0 / (T)3.0);
    for (int i = 0; i < Q; ++i) {
        // qp: the generator's ' + '.join(terms) + ' - tr3' (server/lbm.py:157-164)
        T qp;
        bool any = false;
        T acc = 0;
        auto add = [&](T v) { acc = any ? acc + v : v; any = true; };
        if (CX[i]) add(pxx);
        if (CY[i]) add(pyy);
        if (CZ[i]) add(pzz);
        if (CX[i] && CY[i]) add((T)(2 * CX[i] * CY[i]) * pxy);
        if (CX[i] && CZ[i]) add((T)(2 * CX[i] * CZ[i]) * pxz);
        if (CY[i] && CZ[i]) add((T)(2 * CY[i] * CZ[i]) * pyz);
        qp = (any ? acc : (T)0.0) - tr3;
        st<St>(a.fout, n, i, idx, e[i] + K.c45w[i] * keep * qp, K);
    }
    mac[4 * idx + 0] = ux; mac[4 * idx + 1] = uy; mac[4 * idx + 2] = uz; mac[4 * idx + 3] = rho;
}

// The reference's launch executed literally in tid order (Warp CPU order).
template <class St>
void step_serial_impl(const StepArgs<St>& a) {
    for (int z = 0; z < a.nz; ++z)
        for (int y = 0; y < a.ny; ++y)
            for (int x = 0; x < a.nx; ++x) {
                int64_t idx = x + (int64_t)a.nx * (y + (int64_t)a.ny * z);
                step_cell<St>(a, idx, x, y, z, a.mac);
            }
}

// Same result, parallel: cells that read a not-yet-updated neighbour use a snapshot.
template <class St>
void step_parallel_impl(StepArgs<St> a, std::vector<typename St::Real>& snap) {
    using T = typename St::Real;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    snap.assign(a.mac, a.mac + 4 * a.n);
    const T* prev = snap.data();
    auto needs_current = [&](int x, int y, int z) {
        if (x == 0) return false;
        bool face = x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
        if (!face) return false;
        int cx = clampI(x, 1, nx - 2), cy = clampI(y, 1, ny - 2), cz = clampI(z, 1, nz - 2);
        if (cz != z) return cz < z;
        if (cy != y) return cy < y;
        return cx < x;
    };
#pragma omp parallel for schedule(static) collapse(2)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                if (needs_current(x, y, z)) continue;
                int64_t idx = x + (int64_t)nx * (y + (int64_t)ny * z);
                step_cell<St>(a, idx, x, y, z, prev);
            }
#pragma omp parallel for schedule(static) collapse(2)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                if (!needs_current(x, y, z)) continue;
                int64_t idx = x + (int64_t)nx * (y + (int64_t)ny * z);
                step_cell<St>(a, idx, x, y, z, a.mac);
            }
}

// ---------------- force (server/lbm.py:169-197) ----------------
// out_ref: the reference's float accumulation (per-cell sums added in tid order, the
// order Warp's CPU backend applies its atomic_adds). out_f64: the same per-cell sums
// accumulated in double. out_body_f64: as out_f64 but without links whose solid cell
// lies on the y = 0 plane (a no-slip floor tagged 1 would otherwise add its shear).
template <class St>
void force_impl(const typename St::Store* f, const uint8_t* solid, int nx, int ny, int nz,
                typename St::Real* out_ref, double* out_f64, double* out_body_f64) {
    using T = typename St::Real;
    static const Consts<T> K;
    const int64_t n = (int64_t)nx * ny * nz;
    T acc[3] = {0, 0, 0};
    double accd[3] = {0, 0, 0}, accb[3] = {0, 0, 0};
    for (int z = 1; z < nz - 1; ++z)
        for (int y = 1; y < ny - 1; ++y)
            for (int x = 1; x < nx - 1; ++x) {
                int64_t idx = x + (int64_t)nx * (y + (int64_t)ny * z);
                if (solid[idx] != 0) continue;
                T fx = 0, fy = 0, fz = 0;
                T bx = 0, by = 0, bz = 0;
                bool hit = false;
                for (int i = 1; i < Q; ++i) {
                    int64_t s = (x + CX[i]) + (int64_t)nx * ((y + CY[i]) + (int64_t)ny * (z + CZ[i]));
                    if (solid[s] != 1) continue;
                    T v;
                    if constexpr (St::shifted) v = (T)2.0 * ((T)f[(int64_t)i * n + idx] + (T)g_shift.dw[i]);
                    else v = (T)2.0 * (ld<St>(f, n, i, idx, K) - K.w[i]);
                    if (CX[i]) fx = CX[i] > 0 ? fx + v : fx - v;
                    if (CY[i]) fy = CY[i] > 0 ? fy + v : fy - v;
                    if (CZ[i]) fz = CZ[i] > 0 ? fz + v : fz - v;
                    if (y + CY[i] != 0) {
                        if (CX[i]) bx = CX[i] > 0 ? bx + v : bx - v;
                        if (CY[i]) by = CY[i] > 0 ? by + v : by - v;
                        if (CZ[i]) bz = CZ[i] > 0 ? bz + v : bz - v;
                    }
                    hit = true;
                }
                if (hit) {
                    acc[0] = acc[0] + fx; acc[1] = acc[1] + fy; acc[2] = acc[2] + fz;
                    accd[0] += (double)fx; accd[1] += (double)fy; accd[2] += (double)fz;
                    accb[0] += (double)bx; accb[1] += (double)by; accb[2] += (double)bz;
                }
            }
    for (int k = 0; k < 3; ++k) {
        if (out_ref) out_ref[k] = acc[k];
        if (out_f64) out_f64[k] = accd[k];
        if (out_body_f64) out_body_f64[k] = accb[k];
    }
}

template <class St>
double mass_impl(const typename St::Store* f, const uint8_t* solid, int64_t n) {
    double tot = 0;
#pragma omp parallel for schedule(static) reduction(+ : tot)
    for (int64_t idx = 0; idx < n; ++idx) {
        if (solid[idx] != 0) continue;
        double c = 0;
        for (int i = 0; i < Q; ++i) {
            double v = (double)f[(int64_t)i * n + idx];
            if constexpr (St::shifted) v += (double)g_shift.e[i];
            c += v;
        }
        tot += c;
    }
    return tot;
}

// ---------------- particles / slices / surface pressure ----------------
inline int64_t cidx(int x, int y, int z, int nx, int ny, int nz) {
    return clampI(x, 0, nx - 1) + (int64_t)nx * (clampI(y, 0, ny - 1) + (int64_t)ny * clampI(z, 0, nz - 1));
}

template <class T>
inline void lerp4(const T* a, const T* b, T t, T* o) {
    for (int k = 0; k < 4; ++k) o[k] = a[k] * ((T)1.0 - t) + b[k] * t;
}

template <class T>
void sample_mac(const T* mac, const T* p, int nx, int ny, int nz, T* out) {
    T qx = clampT(p[0], (T)0.0, (T)nx - (T)1.001);
    T qy = clampT(p[1], (T)0.0, (T)ny - (T)1.001);
    T qz = clampT(p[2], (T)0.0, (T)nz - (T)1.001);
    T bx = std::floor(qx), by = std::floor(qy), bz = std::floor(qz);
    T tx = qx - bx, ty = qy - by, tz = qz - bz;
    int ix = (int)bx, iy = (int)by, iz = (int)bz;
    const T* c000 = mac + 4 * cidx(ix, iy, iz, nx, ny, nz);
    const T* c100 = mac + 4 * cidx(ix + 1, iy, iz, nx, ny, nz);
    const T* c010 = mac + 4 * cidx(ix, iy + 1, iz, nx, ny, nz);
    const T* c110 = mac + 4 * cidx(ix + 1, iy + 1, iz, nx, ny, nz);
    const T* c001 = mac + 4 * cidx(ix, iy, iz + 1, nx, ny, nz);
    const T* c101 = mac + 4 * cidx(ix + 1, iy, iz + 1, nx, ny, nz);
    const T* c011 = mac + 4 * cidx(ix, iy + 1, iz + 1, nx, ny, nz);
    const T* c111 = mac + 4 * cidx(ix + 1, iy + 1, iz + 1, nx, ny, nz);
    T l0[4], l1[4], l2[4], l3[4], a[4], b[4];
    lerp4(c000, c100, tx, l0); lerp4(c010, c110, tx, l1); lerp4(l0, l1, ty, a);
    lerp4(c001, c101, tx, l2); lerp4(c011, c111, tx, l3); lerp4(l2, l3, ty, b);
    lerp4(a, b, tz, out);
}

inline uint32_t pcg_hash(uint32_t v) {
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
inline uint32_t rng_init(uint32_t seed, uint32_t i) { return pcg_hash(pcg_hash(seed) + i); }
inline float rng_f(uint32_t& s) {
    s = pcg_hash(s);
    return (float)(s >> 8) * (1.0f / 16777216.0f);
}

template <class T>
void advect_impl(T* pos, T* spd, const T* mac, const uint8_t* solid, int nx, int ny, int nz, int64_t np_,
                 T dt, T uin, T max_age, int seed, T sx, T scy, T scz, T shy, T shz) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < np_; ++i) {
        T* p = pos + 4 * i;
        T q[3] = {p[0], p[1], p[2]};
        T m1[4], m2[4];
        sample_mac(mac, q, nx, ny, nz, m1);
        T hd = (T)0.5 * dt;
        T qm[3] = {q[0] + hd * m1[0], q[1] + hd * m1[1], q[2] + hd * m1[2]};
        sample_mac(mac, qm, nx, ny, nz, m2);
        q[0] = q[0] + dt * m2[0]; q[1] = q[1] + dt * m2[1]; q[2] = q[2] + dt * m2[2];
        T age = p[3] + (T)1.0;
        T s = std::sqrt(m2[0] * m2[0] + m2[1] * m2[1] + m2[2] * m2[2]) / uin;
        bool dead = age > max_age || q[0] < (T)0.5 || q[1] < (T)0.5 || q[2] < (T)0.5;
        if (q[0] > (T)nx - (T)3.0 || q[1] > (T)ny - (T)1.5 || q[2] > (T)nz - (T)1.5 || !(s < (T)100.0)) dead = true;
        if (!dead) {
            int64_t c = cidx((int)std::round(q[0]), (int)std::round(q[1]), (int)std::round(q[2]), nx, ny, nz);
            if (solid[c] != 0) dead = true;
        }
        if (dead) {
            uint32_t r = rng_init((uint32_t)seed, (uint32_t)i);
            T r0 = (T)rng_f(r), r1 = (T)rng_f(r), r2 = (T)rng_f(r);
            q[0] = sx + r0 * (T)2.0;
            q[1] = scy + (r1 * (T)2.0 - (T)1.0) * shy;
            q[2] = scz + (r2 * (T)2.0 - (T)1.0) * shz;
            age = 0;
            s = 1;
        }
        p[0] = q[0]; p[1] = q[1]; p[2] = q[2]; p[3] = age;
        spd[i] = s;
    }
}

template <class T>
void pack_impl(const T* pos, const T* spd, uint16_t* q16, uint8_t* q8, int nx, int ny, int nz, int64_t np_) {
    for (int64_t i = 0; i < np_; ++i) {
        const T* p = pos + 4 * i;
        q16[4 * i + 0] = (uint16_t)(int)(clampT(p[0] / (T)nx, (T)0.0, (T)1.0) * (T)65535.0 + (T)0.5);
        q16[4 * i + 1] = (uint16_t)(int)(clampT(p[1] / (T)ny, (T)0.0, (T)1.0) * (T)65535.0 + (T)0.5);
        q16[4 * i + 2] = (uint16_t)(int)(clampT(p[2] / (T)nz, (T)0.0, (T)1.0) * (T)65535.0 + (T)0.5);
        q16[4 * i + 3] = (uint16_t)(int)(clampT(p[3], (T)0.0, (T)65535.0));
        q8[i] = (uint8_t)(int)(clampT(spd[i] / (T)2.0, (T)0.0, (T)1.0) * (T)255.0 + (T)0.5);
    }
}

template <class T>
T vort(const T* mac, int x, int y, int z, int nx, int ny, int nz) {
    const T* xp = mac + 4 * cidx(x + 1, y, z, nx, ny, nz);
    const T* xm = mac + 4 * cidx(x - 1, y, z, nx, ny, nz);
    const T* yp = mac + 4 * cidx(x, y + 1, z, nx, ny, nz);
    const T* ym = mac + 4 * cidx(x, y - 1, z, nx, ny, nz);
    const T* zp = mac + 4 * cidx(x, y, z + 1, nx, ny, nz);
    const T* zm = mac + 4 * cidx(x, y, z - 1, nx, ny, nz);
    T dx[4], dy[4], dz[4];
    for (int k = 0; k < 4; ++k) {
        dx[k] = (xp[k] - xm[k]) * (T)0.5;
        dy[k] = (yp[k] - ym[k]) * (T)0.5;
        dz[k] = (zp[k] - zm[k]) * (T)0.5;
    }
    T a = dy[2] - dz[1], b = dz[0] - dx[2], c = dx[1] - dy[0];
    return std::sqrt(a * a + b * b + c * c);
}

template <class T>
void slice_impl(const T* mac, const uint8_t* solid, uint8_t* out, int nx, int ny, int nz, int axis, int index,
                int field, int w, int h, T uin, T lref, T vmin, T vmax) {
    for (int64_t k = 0; k < (int64_t)w * h; ++k) {
        int a = (int)(k % w), b = (int)(k / w);
        int cx = index, cy = b, cz = a;
        if (axis == 2) { cx = a; cy = b; cz = index; }
        else if (axis == 1) { cx = a; cy = index; cz = b; }
        int64_t idx = cx + (int64_t)nx * (cy + (int64_t)ny * cz);
        const T* m = mac + 4 * idx;
        T v = m[0] / uin;
        if (field == 0) v = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]) / uin;
        else if (field == 1) v = (m[3] - (T)1.0) / ((T)1.5 * uin * uin);
        else if (field == 2) v = vort(mac, cx, cy, cz, nx, ny, nz) * lref / uin;
        T t = clampT((v - vmin) / (vmax - vmin), (T)0.0, (T)1.0);
        out[2 * k] = (uint8_t)(int)(t * (T)255.0 + (T)0.5);
        out[2 * k + 1] = solid[idx] != 0 ? 0 : 255;
    }
}

template <class T>
void rho_fluid(const T* mac, const uint8_t* solid, const T* p, int nx, int ny, int nz, T* acc) {
    T qx = clampT(p[0], (T)0.0, (T)nx - (T)1.001);
    T qy = clampT(p[1], (T)0.0, (T)ny - (T)1.001);
    T qz = clampT(p[2], (T)0.0, (T)nz - (T)1.001);
    int ix = (int)std::floor(qx), iy = (int)std::floor(qy), iz = (int)std::floor(qz);
    T tx = qx - (T)ix, ty = qy - (T)iy, tz = qz - (T)iz;
    acc[0] = 0; acc[1] = 0;
    for (int c = 0; c < 8; ++c) {
        int ox = c & 1, oy = (c >> 1) & 1, oz = (c >> 2) & 1;
        int64_t ci = cidx(ix + ox, iy + oy, iz + oz, nx, ny, nz);
        T wx = ox ? tx : (T)1.0 - tx;
        T wy = oy ? ty : (T)1.0 - ty;
        T wz = oz ? tz : (T)1.0 - tz;
        T wt = wx * wy * wz;
        if (solid[ci] == 0) {
            acc[0] = acc[0] + wt * mac[4 * ci + 3];
            acc[1] = acc[1] + wt;
        }
    }
}

template <class T>
void cp_impl(const T* mac, const uint8_t* solid, const T* verts, const T* norms, int8_t* out, int nx, int ny, int nz,
             int64_t nv, T uin, T cp_range) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nv; ++i) {
        const T* p = verts + 3 * i;
        const T* nr = norms + 3 * i;
        T pa[3], pb[3], a[2], b[2];
        for (int k = 0; k < 3; ++k) { pa[k] = p[k] + nr[k] * (T)1.25; pb[k] = p[k] - nr[k] * (T)1.25; }
        rho_fluid(mac, solid, pa, nx, ny, nz, a);
        rho_fluid(mac, solid, pb, nx, ny, nz, b);
        const T* s = b;
        if (a[1] >= b[1]) s = a;
        T cp = 0;
        if (s[1] > (T)0.05) cp = (s[0] / s[1] - (T)1.0) / ((T)1.5 * uin * uin);
        out[i] = (int8_t)(int)std::round(clampT(cp / cp_range, (T)-1.0, (T)1.0) * (T)127.0);
    }
}

template <class St>
void step_dispatch(const typename St::Store* fin, typename St::Store* fout, const uint8_t* solid,
                   typename St::Real* mac, int nx, int ny, int nz, typename St::Real uin,
                   typename St::Real tau, typename St::Real smag, int serial, int fast) {
    StepArgs<St> a{fin, fout, solid, mac, mac, nx, ny, nz, (int64_t)nx * ny * nz, uin, tau, smag, fast};
    if (serial) {
        step_serial_impl<St>(a);
    } else {
        std::vector<typename St::Real> snap;
        step_parallel_impl<St>(a, snap);
    }
}

}  // namespace

extern "C" {

int oracle_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

// precision codes: 0 f32, 1 f16-shifted, 2 bf16-shifted, 3 f64 (same as the product ABI)
#define WT_DISPATCH(prec, CALL_F32, CALL_F16, CALL_BF16, CALL_F64) \
    switch (prec) {                                                \
        case 0: CALL_F32; return 0;                                \
        case 1: CALL_F16; return 0;                                \
        case 2: CALL_BF16; return 0;                               \
        case 3: CALL_F64; return 0;                                \
        default: return -1;                                        \
    }

int oracle_init(int prec, void* f, void* mac, int64_t n, double uin) {
    WT_DISPATCH(prec,
                init_impl<StF32>((float*)f, (float*)mac, n, (float)uin),
                init_impl<StF16>((_Float16*)f, (float*)mac, n, (float)uin),
                init_impl<StBF16>((__bf16*)f, (float*)mac, n, (float)uin),
                init_impl<StF64>((double*)f, (double*)mac, n, uin))
}

// collision: 0 = the reference's expressions in the reference's order, 1 = moment-space form
int oracle_step(int prec, const void* fin, void* fout, const uint8_t* solid, void* mac, int nx, int ny, int nz,
                double uin, double tau, double smag, int serial, int collision) {
    if (nx < 3 || ny < 3 || nz < 3) return -2;
    if (collision != 0 && collision != 1) return -1;
    WT_DISPATCH(prec,
                step_dispatch<StF32>((const float*)fin, (float*)fout, solid, (float*)mac, nx, ny, nz, (float)uin, (float)tau, (float)smag, serial, collision),
                step_dispatch<StF16>((const _Float16*)fin, (_Float16*)fout, solid, (float*)mac, nx, ny, nz, (float)uin, (float)tau, (float)smag, serial, collision),
                step_dispatch<StBF16>((const __bf16*)fin, (__bf16*)fout, solid, (float*)mac, nx, ny, nz, (float)uin, (float)tau, (float)smag, serial, collision),
                step_dispatch<StF64>((const double*)fin, (double*)fout, solid, (double*)mac, nx, ny, nz, uin, tau, smag, serial, collision))
}

// out_ref is float* for prec 0-2 and double* for prec 3
int oracle_force(int prec, const void* f, const uint8_t* solid, int nx, int ny, int nz, void* out_ref,
                 double* out_f64, double* out_body_f64) {
    WT_DISPATCH(prec,
                force_impl<StF32>((const float*)f, solid, nx, ny, nz, (float*)out_ref, out_f64, out_body_f64),
                force_impl<StF16>((const _Float16*)f, solid, nx, ny, nz, (float*)out_ref, out_f64, out_body_f64),
                force_impl<StBF16>((const __bf16*)f, solid, nx, ny, nz, (float*)out_ref, out_f64, out_body_f64),
                force_impl<StF64>((const double*)f, solid, nx, ny, nz, (double*)out_ref, out_f64, out_body_f64))
}

int oracle_mass(int prec, const void* f, const uint8_t* solid, int64_t n, double* out) {
    WT_DISPATCH(prec,
                *out = mass_impl<StF32>((const float*)f, solid, n),
                *out = mass_impl<StF16>((const _Float16*)f, solid, n),
                *out = mass_impl<StBF16>((const __bf16*)f, solid, n),
                *out = mass_impl<StF64>((const double*)f, solid, n))
}

int oracle_advect_f32(float* pos, float* spd, const float* mac, const uint8_t* solid, int nx, int ny, int nz,
                      int64_t np_, float dt, float uin, float max_age, int seed, float sx, float scy, float scz,
                      float shy, float shz) {
    advect_impl<float>(pos, spd, mac, solid, nx, ny, nz, np_, dt, uin, max_age, seed, sx, scy, scz, shy, shz);
    return 0;
}

int oracle_pack_f32(const float* pos, const float* spd, uint16_t* q16, uint8_t* q8, int nx, int ny, int nz,
                    int64_t np_) {
    pack_impl<float>(pos, spd, q16, q8, nx, ny, nz, np_);
    return 0;
}

int oracle_slice_f32(const float* mac, const uint8_t* solid, uint8_t* out, int nx, int ny, int nz, int axis,
                     int index, int field, int w, int h, float uin, float lref, float vmin, float vmax) {
    slice_impl<float>(mac, solid, out, nx, ny, nz, axis, index, field, w, h, uin, lref, vmin, vmax);
    return 0;
}

int oracle_cp_f32(const float* mac, const uint8_t* solid, const float* verts, const float* norms, int8_t* out,
                  int nx, int ny, int nz, int64_t nv, float uin, float cp_range) {
    cp_impl<float>(mac, solid, verts, norms, out, nx, ny, nz, nv, uin, cp_range);
    return 0;
}

uint32_t oracle_rng_hash(uint32_t v) { return pcg_hash(v); }

void oracle_set_shift(double U) {
    double e[Q];
    for (int i = 0; i < Q; ++i) {
        const double cu = 3.0 * CX[i] * U;
        e[i] = w_d(i) * (1.0 + cu + 0.5 * cu * cu - 1.5 * U * U);
    }
    for (int i = 0; i < Q; ++i) {
        g_shift.e[i] = (float)(U != 0.0 ? e[i] : w_d(i));
        g_shift.bb[i] = (float)(e[OPP[i]] - e[i]);
        g_shift.dw[i] = (float)(e[i] - w_d(i));
    }
    g_shift.su = (float)U;
    g_shift.suu = (float)(U * U);
    g_shift.s45 = (float)(4.5 * U * U);
    g_shift.s15 = (float)(1.5 * U * U);
}

}  // extern "C"
