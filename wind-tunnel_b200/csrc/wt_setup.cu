// Set-up kernels: equilibrium init (server/lbm.py:64-69), per-cell codes, and the compacted
// momentum-exchange link list (the cells force_kernel visits, server/lbm.py:177-193).
#include "wt_common.cuh"

namespace wt {

template <class T>
struct InitVals {
    T v[Q];
};

template <int PREC>
__global__ void __launch_bounds__(256) k_init(typename Prec<PREC>::S* __restrict__ f, typename Prec<PREC>::T* __restrict__ mac,
                                              int64_t n, typename Prec<PREC>::T uin, InitVals<typename Prec<PREC>::T> e) {
    using P = Prec<PREC>;
    using T = typename P::T;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n; idx += (int64_t)gridDim.x * blockDim.x) {
        unroll<0, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            // W * (1 + 3 c_x u + 4.5 c_x^2 u u - 1.5 u u), left to right as generated (:68)
            const T v = (T)wd(i) * ((T)1.0 + (T)(3.0 * cx(i)) * uin + (T)(4.5 * cx(i) * cx(i)) * uin * uin -
                                    (T)1.5 * uin * uin);
            st_pop<P, i>(f + i * n + idx, v, e.v[i]);
        });
        mac[4 * idx + 0] = uin;
        mac[4 * idx + 1] = (T)0.0;
        mac[4 * idx + 2] = (T)0.0;
        mac[4 * idx + 3] = (T)1.0;
    }
}

struct Geo {
    int32_t nx, ny, nz, n, nxy;
    FastDiv dnx, dnxy;
    __device__ __forceinline__ void coords(int32_t idx, int32_t& x, int32_t& y, int32_t& z) const {
        z = (int32_t)dnxy.div((uint32_t)idx);
        const int32_t r = idx - z * nxy;
        y = (int32_t)dnx.div((uint32_t)r);
        x = r - y * nx;
    }
    __device__ __forceinline__ bool interior(int32_t x, int32_t y, int32_t z) const {
        return x > 0 && x < nx - 1 && y > 0 && y < ny - 1 && z > 0 && z < nz - 1;
    }
};

static Geo make_geo(const wt_grid* g) {
    Geo G;
    G.nx = g->nx; G.ny = g->ny; G.nz = g->nz;
    G.nxy = g->nx * g->ny;
    G.n = G.nxy * g->nz;
    G.dnx = FastDiv((uint32_t)G.nx);
    G.dnxy = FastDiv((uint32_t)G.nxy);
    return G;
}

__global__ void __launch_bounds__(256) k_codes(const uint8_t* __restrict__ solid, uint8_t* __restrict__ code, Geo G) {
    const int32_t idx = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (idx >= G.n) return;
    int32_t x, y, z;
    G.coords(idx, x, y, z);
    uint8_t c = 0;
    if (solid[idx] != 0) {
        c = CODE_SOLID;
    } else if (G.interior(x, y, z)) {
        bool near = false;
        unroll<1, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            near |= solid[idx - (cx(i) + cy(i) * G.nx + cz(i) * G.nxy)] != 0;
        });
        if (near) c = CODE_NEAR;
    }
    code[idx] = c;
}

// link mask of one cell: bit i-1 set when solid[x + c_i] == 1 (server/lbm.py:188)
__device__ __forceinline__ uint32_t link_mask(const uint8_t* __restrict__ solid, const Geo& G, int32_t idx) {
    if (idx >= G.n) return 0;
    int32_t x, y, z;
    G.coords(idx, x, y, z);
    if (!G.interior(x, y, z) || solid[idx] != 0) return 0;
    uint32_t m = 0;
    unroll<1, Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if (solid[idx + cx(i) + cy(i) * G.nx + cz(i) * G.nxy] == 1) m |= 1u << (i - 1);
    });
    return m;
}

constexpr int LINK_THREADS = 256;
constexpr int LINK_CELLS = 4;  // consecutive cells per thread
constexpr int LINK_TILE = LINK_THREADS * LINK_CELLS;

__global__ void __launch_bounds__(LINK_THREADS) k_links_count(const uint8_t* __restrict__ solid, Geo G,
                                                              int64_t* __restrict__ counts) {
    __shared__ int warp_sums[LINK_THREADS / 32];
    const int32_t base = blockIdx.x * LINK_TILE + threadIdx.x * LINK_CELLS;
    int c = 0;
#pragma unroll
    for (int k = 0; k < LINK_CELLS; ++k) c += link_mask(solid, G, base + k) != 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < LINK_THREADS / 32; ++w) s += warp_sums[w];
        counts[blockIdx.x] = s;
    }
}

// exclusive scan of counts[0..nb) in place; counts[nb] = total; *total_out = total
__global__ void __launch_bounds__(1024) k_scan(int64_t* __restrict__ counts, int64_t nb, int64_t* __restrict__ total_out) {
    __shared__ int64_t sh[1024];
    const int t = threadIdx.x;
    const int64_t per = (nb + 1023) / 1024;
    const int64_t b0 = t * per, b1 = min(nb, b0 + per);
    int64_t s = 0;
    for (int64_t b = b0; b < b1; ++b) s += counts[b];
    sh[t] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {  // Hillis-Steele inclusive scan
        int64_t v = t >= o ? sh[t - o] : 0;
        __syncthreads();
        sh[t] += v;
        __syncthreads();
    }
    int64_t run = t > 0 ? sh[t - 1] : 0;
    for (int64_t b = b0; b < b1; ++b) {
        int64_t c = counts[b];
        counts[b] = run;
        run += c;
    }
    if (t == 1023) {
        counts[nb] = sh[1023];
        if (total_out) *total_out = sh[1023];
    }
}

__global__ void __launch_bounds__(LINK_THREADS) k_links_fill(const uint8_t* __restrict__ solid, Geo G,
                                                             const int64_t* __restrict__ offsets,
                                                             int32_t* __restrict__ cells, uint32_t* __restrict__ masks,
                                                             int64_t capacity) {
    __shared__ int warp_sums[LINK_THREADS / 32];
    const int32_t base = blockIdx.x * LINK_TILE + threadIdx.x * LINK_CELLS;
    uint32_t m[LINK_CELLS];
    int c = 0;
#pragma unroll
    for (int k = 0; k < LINK_CELLS; ++k) {
        m[k] = link_mask(solid, G, base + k);
        c += m[k] != 0;
    }
    // block-wide exclusive prefix of c in thread order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    int wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += warp_sums[w];
    int64_t pos = offsets[blockIdx.x] + wbase + (incl - c);
#pragma unroll
    for (int k = 0; k < LINK_CELLS; ++k) {
        if (m[k]) {
            if (pos < capacity) {
                cells[pos] = base + k;
                masks[pos] = m[k];
            }
            ++pos;
        }
    }
}

template <int PREC>
int init_impl(void* f, void* mac, int64_t n, double uin, double shift_u, cudaStream_t st) {
    using P = Prec<PREC>;
    using T = typename P::T;
    const ShiftTables t = shift_tables(P::shifted ? shift_u : 0.0);
    InitVals<T> e;
    for (int i = 0; i < Q; ++i) e.v[i] = (T)t.e[i];
    const int64_t nb = std::min<int64_t>((n + 255) / 256, 148 * 64);
    k_init<PREC><<<(unsigned)nb, 256, 0, st>>>(static_cast<typename P::S*>(f), static_cast<T*>(mac), n, (T)uin, e);
    return wt_cuda_check("wt_init_eq launch");
}

}  // namespace wt

using namespace wt;

extern "C" int wt_init_eq(int32_t precision, void* f, void* mac, int64_t n, double uin, double shift_u,
                          void* stream) {
    if (!f || !mac || n <= 0) return wt_set_error(WT_ERR_ARG, "wt_init_eq: null buffer or n <= 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (precision) {
        case WT_F32: return init_impl<WT_F32>(f, mac, n, uin, shift_u, st);
        case WT_F16: return init_impl<WT_F16>(f, mac, n, uin, shift_u, st);
        case WT_BF16: return init_impl<WT_BF16>(f, mac, n, uin, shift_u, st);
        case WT_F64: return init_impl<WT_F64>(f, mac, n, uin, shift_u, st);
        default: return wt_set_error(WT_ERR_ARG, "wt_init_eq: unknown precision %d", precision);
    }
}

extern "C" int wt_build_codes(const wt_grid* g, void* stream) {
    if (!g || !g->solid || !g->code) return wt_set_error(WT_ERR_ARG, "wt_build_codes: null buffer");
    if (int rc = wt_check_dims(g->nx, g->ny, g->nz)) return rc;
    Geo G = make_geo(g);
    k_codes<<<(unsigned)((G.n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(g->solid, g->code, G);
    return wt_cuda_check("wt_build_codes launch");
}

extern "C" int64_t wt_links_scratch_len(int64_t n) { return (n + LINK_TILE - 1) / LINK_TILE + 1; }

extern "C" int wt_links_scan(const wt_grid* g, int64_t* scratch, int64_t* count_dev, void* stream) {
    if (!g || !g->solid || !scratch) return wt_set_error(WT_ERR_ARG, "wt_links_scan: null buffer");
    if (int rc = wt_check_dims(g->nx, g->ny, g->nz)) return rc;
    Geo G = make_geo(g);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t nb = (G.n + LINK_TILE - 1) / LINK_TILE;
    k_links_count<<<(unsigned)nb, LINK_THREADS, 0, st>>>(g->solid, G, scratch);
    k_scan<<<1, 1024, 0, st>>>(scratch, nb, count_dev);
    return wt_cuda_check("wt_links_scan launch");
}

extern "C" int wt_links_fill(const wt_grid* g, const int64_t* scratch, int32_t* cells, uint32_t* masks,
                             int64_t capacity, void* stream) {
    if (!g || !g->solid || !scratch) return wt_set_error(WT_ERR_ARG, "wt_links_fill: null buffer");
    if (capacity > 0 && (!cells || !masks)) return wt_set_error(WT_ERR_ARG, "wt_links_fill: null output");
    if (int rc = wt_check_dims(g->nx, g->ny, g->nz)) return rc;
    Geo G = make_geo(g);
    const int64_t nb = (G.n + LINK_TILE - 1) / LINK_TILE;
    k_links_fill<<<(unsigned)nb, LINK_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(g->solid, G, scratch, cells,
                                                                                       masks, capacity);
    return wt_cuda_check("wt_links_fill launch");
}
