// Fused D3Q19 step: pull streaming + bounce-back / moving belt + equilibrium faces +
// regularized collision with Smagorinsky eddy viscosity and outlet sponge.
// Semantics: step_kernel of RICKxxROLLING/wind-tunnel server/lbm.py:72-166.
//
// One step = two launches:
//   k_step_bulk  -- every cell except the "current-read" faces below. Interior cells pull
//                   and collide; x = 0 inlet cells; face cells whose interior neighbour has
//                   a LARGER linear index read that neighbour's mac from the previous step
//                   (mac_prev); outlet cells x = nx-1 with interior y, z take the current
//                   value of their x = nx-2 neighbour from the adjacent lane by shuffle.
//   k_step_faces -- the z = nz-1 plane and the y = ny-1 rows of interior z (x > 0): their
//                   neighbour has a SMALLER linear index, so they read the mac that
//                   k_step_bulk just wrote (mac_cur).
// This is exactly the value each face cell sees when the reference launch runs in tid
// order (Warp's CPU backend), and it is deterministic, unlike the single-launch race of
// server/lbm.py:87 vs :166 on a GPU.
//
// mac is double-buffered: the step that writes f[b] writes mac[b]. Every step writes mac
// for the shell of interior cells that faces read (coordinates 1 or n-2); with
// mac_all set (the last step before a frame) every cell writes it, as the reference does.
#include "wt_common.cuh"

namespace wt {

template <class T>
struct StepArgs {
    const void* fin;
    void* fout;
    const T* mac_prev;
    T* mac_cur;
    const uint8_t* solid;
    const uint8_t* code;
    int32_t nx, ny, nz, n, nxy;
    FastDiv dnx, dnxy;
    T uin, tau, smag;
    int32_t mac_all;
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
        float4 v = reinterpret_cast<const float4*>(mac)[idx];
        a = v.x; b = v.y; c = v.z; d = v.w;
    } else {
        double2 v0 = reinterpret_cast<const double2*>(mac)[2 * idx];
        double2 v1 = reinterpret_cast<const double2*>(mac)[2 * idx + 1];
        a = v0.x; b = v0.y; c = v1.x; d = v1.y;
    }
}

template <class T>
__device__ __forceinline__ T clampv(T x, T lo, T hi) { return x < lo ? lo : (x > hi ? hi : x); }

// Equilibrium face populations from (br, bux, buy, buz) (server/lbm.py:104-107).
template <class P>
__device__ __forceinline__ void face_eq(typename P::S* fout, int64_t n, int32_t idx, typename P::T br,
                                        typename P::T bux, typename P::T buy, typename P::T buz) {
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
        st_pop<P, i>(fout + (int64_t)i * n + idx, (T)wd(i) * br * ((T)1.0 + bc + (T)0.5 * bc * bc - bsq));
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

// Interior cell: pull, bounce-back, moments, regularized Smagorinsky collision
// (server/lbm.py:110-166). Returns the macroscopic values written to mac.
template <class P>
__device__ __forceinline__ void interior(const StepArgs<typename P::T>& a, int32_t idx, int32_t x, uint8_t code,
                                         typename P::T& oux, typename P::T& ouy, typename P::T& ouz,
                                         typename P::T& orho) {
    using T = typename P::T;
    using S = typename P::S;
    const S* __restrict__ fin = static_cast<const S*>(a.fin);
    S* __restrict__ fout = static_cast<S*>(a.fout);
    const int64_t n = a.n;
    const int32_t sy = a.nx, sz = a.nxy;
    T f[Q];
    f[0] = ld_pop<P, 0>(fin + idx);
    if (!(code & CODE_NEAR)) {
        unroll<1, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            const int32_t off = cx(i) + cy(i) * sy + cz(i) * sz;
            f[i] = ld_pop<P, i>(fin + (int64_t)i * n + (idx - off));
        });
    } else {
        unroll<1, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            const int32_t off = cx(i) + cy(i) * sy + cz(i) * sz;
            const int t = a.solid[idx - off];
            if (t == 0) {
                f[i] = ld_pop<P, i>(fin + (int64_t)i * n + (idx - off));
            } else {
                f[i] = ld_pop<P, opp(i)>(fin + (int64_t)opp(i) * n + idx);
                if constexpr (cx(i) != 0) {
                    if (t == 2) f[i] = f[i] + (T)(6.0 * wd(i) * cx(i)) * a.uin;
                }
            }
        });
    }
    T rho = (T)0.0, jx = (T)0.0, jy = (T)0.0, jz = (T)0.0;
    unroll<0, Q>([&](auto ic) { constexpr int i = decltype(ic)::value; rho = rho + f[i]; });
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (cx(i) > 0) jx = jx + f[i];
        if constexpr (cx(i) < 0) jx = jx - f[i];
    });
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (cy(i) > 0) jy = jy + f[i];
        if constexpr (cy(i) < 0) jy = jy - f[i];
    });
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (cz(i) > 0) jz = jz + f[i];
        if constexpr (cz(i) < 0) jz = jz - f[i];
    });
    const T ir = (T)1.0 / rho;
    T ux = jx * ir, uy = jy * ir, uz = jz * ir;
    const T um = sqrt(ux * ux + uy * uy + uz * uz);
    if (um > (T)0.35) {
        const T sc = (T)0.35 / um;
        ux = ux * sc; uy = uy * sc; uz = uz * sc;
    }
    const T usq = (T)1.5 * (ux * ux + uy * uy + uz * uz);
    // f[] now holds the non-equilibrium parts d_i = f_i - e_i; e[] the equilibria
    T e[Q];
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        T s = (T)0.0;
        if constexpr (cx(i) > 0) s = s + ux;
        if constexpr (cx(i) < 0) s = s - ux;
        if constexpr (cy(i) > 0) s = s + uy;
        if constexpr (cy(i) < 0) s = s - uy;
        if constexpr (cz(i) > 0) s = s + uz;
        if constexpr (cz(i) < 0) s = s - uz;
        const T cu = (T)3.0 * s;
        e[i] = (T)wd(i) * rho * ((T)1.0 + cu + (T)0.5 * cu * cu - usq);
        f[i] = f[i] - e[i];
    });
    T pxx = (T)0.0, pyy = (T)0.0, pzz = (T)0.0, pxy = (T)0.0, pxz = (T)0.0, pyz = (T)0.0;
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (cx(i) != 0) pxx = pxx + f[i];
    });
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (cy(i) != 0) pyy = pyy + f[i];
    });
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (cz(i) != 0) pzz = pzz + f[i];
    });
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (cx(i) * cy(i) > 0) pxy = pxy + f[i];
        if constexpr (cx(i) * cy(i) < 0) pxy = pxy - f[i];
    });
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (cx(i) * cz(i) > 0) pxz = pxz + f[i];
        if constexpr (cx(i) * cz(i) < 0) pxz = pxz - f[i];
    });
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (cy(i) * cz(i) > 0) pyz = pyz + f[i];
        if constexpr (cy(i) * cz(i) < 0) pyz = pyz - f[i];
    });
    const T qn = sqrt(pxx * pxx + pyy * pyy + pzz * pzz + (T)2.0 * (pxy * pxy + pxz * pxz + pyz * pyz));
    T tau0 = a.tau;
    const T sp = (T)x - (T)a.nx + (T)24.0;
    if (sp > (T)0.0) tau0 = tau0 + sp * (T)0.015;
    const T tau_e = (T)0.5 * (tau0 + sqrt(tau0 * tau0 + (T)25.4558441 * a.smag * a.smag * qn * ir));
    const T keep = (T)1.0 - (T)1.0 / tau_e;
    const T tr3 = (pxx + pyy + pzz) * ((T)1.0 / (T)3.0);
    unroll<0, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        // the generator's ' + '.join(terms) + ' - tr3' (server/lbm.py:157-164)
        T qp;
        if constexpr (i == 0) {
            qp = (T)0.0 - tr3;
        } else {
            constexpr bool hx = cx(i) != 0, hy = cy(i) != 0, hz = cz(i) != 0;
            T acc = hx ? pxx : (hy ? pyy : pzz);  // first present term
            if constexpr (hx && hy) acc = acc + pyy;
            if constexpr ((hx || hy) && hz) acc = acc + pzz;
            if constexpr (cx(i) != 0 && cy(i) != 0) acc = acc + (T)(2 * cx(i) * cy(i)) * pxy;
            if constexpr (cx(i) != 0 && cz(i) != 0) acc = acc + (T)(2 * cx(i) * cz(i)) * pxz;
            if constexpr (cy(i) != 0 && cz(i) != 0) acc = acc + (T)(2 * cy(i) * cz(i)) * pyz;
            qp = acc - tr3;
        }
        st_pop<P, i>(fout + (int64_t)i * n + idx, e[i] + (T)(4.5 * wd(i)) * keep * qp);
    });
    oux = ux; ouy = uy; ouz = uz; orho = rho;
}

enum Kind { K_NONE = 0, K_SOLID, K_INLET, K_FACE, K_OUTLET, K_INTERIOR, K_LATER };

template <int PREC>
__global__ void __launch_bounds__(256) k_step_bulk(const StepArgs<typename Prec<PREC>::T> a) {
    using P = Prec<PREC>;
    using T = typename P::T;
    using S = typename P::S;
    const int32_t idx = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    const bool valid = idx < a.n;
    const int32_t nx = a.nx, ny = a.ny, nz = a.nz;
    const int32_t z = valid ? (int32_t)a.dnxy.div((uint32_t)idx) : 0;
    const int32_t r = idx - z * a.nxy;
    const int32_t y = (int32_t)a.dnx.div((uint32_t)r);
    const int32_t x = r - y * nx;
    T mx = (T)0.0, my = (T)0.0, mz = (T)0.0, mr = (T)1.0;
    int kind = K_NONE;
    if (valid) {
        const uint8_t code = a.code[idx];
        const bool face = x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1;
        if (code & CODE_SOLID) {
            kind = K_SOLID;
        } else if (x == 0) {
            kind = K_INLET;
            mx = a.uin;
            face_eq<P>(static_cast<S*>(a.fout), a.n, idx, (T)1.0, a.uin, (T)0.0, (T)0.0);
        } else if (face) {
            if (z == nz - 1 || (y == ny - 1 && z > 0)) {
                kind = K_LATER;
            } else if (x == nx - 1 && y > 0 && y < ny - 1 && z > 0 && z < nz - 1) {
                kind = K_OUTLET;
            } else {
                kind = K_FACE;
                const int32_t cxi = min(max(x, 1), nx - 2), cyi = min(max(y, 1), ny - 2), czi = min(max(z, 1), nz - 2);
                T px, py, pz, pr;
                load_mac(a.mac_prev, cxi + nx * (cyi + ny * czi), px, py, pz, pr);
                face_values<T>(x, y, z, nx, ny, nz, a.uin, px, py, pz, pr, mr, mx, my, mz);
                face_eq<P>(static_cast<S*>(a.fout), a.n, idx, mr, mx, my, mz);
            }
        } else {
            kind = K_INTERIOR;
            interior<P>(a, idx, x, code, mx, my, mz, mr);
        }
    }
    // outlet x = nx-1 (interior y, z): its neighbour x = nx-2 is the previous lane. nx is
    // even, so idx of x = nx-1 is odd and never lane 0.
    const T qx = __shfl_up_sync(0xffffffffu, mx, 1);
    const T qy = __shfl_up_sync(0xffffffffu, my, 1);
    const T qz = __shfl_up_sync(0xffffffffu, mz, 1);
    const T qr = __shfl_up_sync(0xffffffffu, mr, 1);
    if (kind == K_OUTLET) {
        face_values<T>(x, y, z, nx, ny, nz, a.uin, qx, qy, qz, qr, mr, mx, my, mz);
        face_eq<P>(static_cast<S*>(a.fout), a.n, idx, mr, mx, my, mz);
    }
    if (kind == K_SOLID) { mx = (T)0.0; my = (T)0.0; mz = (T)0.0; mr = (T)1.0; }
    if (kind != K_NONE && kind != K_LATER) {
        const bool shell = !(x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || z == 0 || z == nz - 1) &&
                           (x == 1 || x == nx - 2 || y == 1 || y == ny - 2 || z == 1 || z == nz - 2);
        if (a.mac_all || shell) store_mac(a.mac_cur, idx, mx, my, mz, mr);
    }
}

template <int PREC>
__global__ void __launch_bounds__(256) k_step_faces(const StepArgs<typename Prec<PREC>::T> a) {
    using P = Prec<PREC>;
    using T = typename P::T;
    using S = typename P::S;
    const int32_t t = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    const int32_t nx = a.nx, ny = a.ny, nz = a.nz;
    const int32_t nplane = a.nxy;
    if (t >= nplane + nx * (nz - 2)) return;
    int32_t x, y, z;
    if (t < nplane) {
        z = nz - 1;
        y = (int32_t)a.dnx.div((uint32_t)t);
        x = t - y * nx;
    } else {
        const int32_t t2 = t - nplane;
        const int32_t row = (int32_t)a.dnx.div((uint32_t)t2);
        z = 1 + row;
        y = ny - 1;
        x = t2 - row * nx;
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
    face_eq<P>(static_cast<S*>(a.fout), a.n, idx, br, bux, buy, buz);
    if (a.mac_all) store_mac(a.mac_cur, idx, bux, buy, buz, br);
}

template <int PREC>
int step_impl(const wt_grid* g, int32_t cur, int32_t steps, double uin, double tau, double smag, int32_t flags,
              cudaStream_t stream) {
    using T = typename Prec<PREC>::T;
    StepArgs<T> a;
    a.solid = g->solid;
    a.code = g->code;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    a.nxy = g->nx * g->ny;
    a.n = a.nxy * g->nz;
    a.dnx = FastDiv((uint32_t)g->nx);
    a.dnxy = FastDiv((uint32_t)a.nxy);
    a.uin = (T)uin; a.tau = (T)tau; a.smag = (T)smag;
    const unsigned nb_bulk = (unsigned)((a.n + 255) / 256);
    const int32_t nface = a.nxy + a.nx * (a.nz - 2);
    const unsigned nb_face = (unsigned)((nface + 255) / 256);
    for (int32_t s = 0; s < steps; ++s) {
        a.fin = g->f[cur];
        a.fout = g->f[cur ^ 1];
        a.mac_prev = static_cast<const T*>(g->mac[cur]);
        a.mac_cur = static_cast<T*>(g->mac[cur ^ 1]);
        a.mac_all = (flags & WT_STEP_MAC_ALL_LAST) && s == steps - 1;
        k_step_bulk<PREC><<<nb_bulk, 256, 0, stream>>>(a);
        k_step_faces<PREC><<<nb_face, 256, 0, stream>>>(a);
        cur ^= 1;
    }
    return wt_cuda_check("wt_step launch");
}

}  // namespace wt

extern "C" int wt_step(const wt_grid* g, int32_t cur, int32_t steps, double uin, double tau, double smag,
                       int32_t flags, void* stream) {
    if (!g || !g->f[0] || !g->f[1] || !g->mac[0] || !g->mac[1] || !g->solid || !g->code)
        return wt_set_error(WT_ERR_ARG, "wt_step: null buffer in grid");
    if (int rc = wt_check_dims(g->nx, g->ny, g->nz)) return rc;
    if (cur != 0 && cur != 1) return wt_set_error(WT_ERR_ARG, "wt_step: cur must be 0 or 1");
    if (steps < 0) return wt_set_error(WT_ERR_ARG, "wt_step: steps < 0");
    if (steps == 0) return WT_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (g->precision) {
        case WT_F32: return wt::step_impl<WT_F32>(g, cur, steps, uin, tau, smag, flags, st);
        case WT_F16: return wt::step_impl<WT_F16>(g, cur, steps, uin, tau, smag, flags, st);
        case WT_BF16: return wt::step_impl<WT_BF16>(g, cur, steps, uin, tau, smag, flags, st);
        case WT_F64: return wt::step_impl<WT_F64>(g, cur, steps, uin, tau, smag, flags, st);
        default: return wt_set_error(WT_ERR_ARG, "wt_step: unknown precision %d", g->precision);
    }
}
