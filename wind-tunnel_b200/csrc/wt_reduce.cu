// Deterministic fp64 reductions: momentum-exchange force over the compacted link list
// (force_kernel, server/lbm.py:169-197) and the total mass.
//
// The reference adds per-cell float sums into three global floats with atomics
// (server/lbm.py:194-197): the result depends on scheduling and all threads contend on
// three addresses. Here each cell's sum is formed exactly as the reference forms it, then
// cells are accumulated in double: a fixed grid of RED_BLOCKS blocks, each thread walking a
// fixed stride of the list, a fixed shuffle tree per warp and block, and a second one-block
// pass over the block partials. The order never depends on scheduling, so repeated runs
// are bit-identical.
#include <mutex>

#include "wt_common.cuh"

namespace wt {

constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 148 * 4;
constexpr int FORCE_VALS = 6;

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* __restrict__ out) {
    __shared__ double sh[RED_THREADS / 32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[warp][k] = v[k];
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int w = 0; w < RED_THREADS / 32; ++w) s += sh[w][threadIdx.x];
        out[threadIdx.x] = s;
    }
}

// per-population constants of the shifted storage passed by value
template <class T>
struct PopVals {
    T v[Q];
};

template <int PREC>
__global__ void __launch_bounds__(RED_THREADS) k_force_partial(const typename Prec<PREC>::S* __restrict__ f,
                                                               const int32_t* __restrict__ cells,
                                                               const uint32_t* __restrict__ masks, int64_t count,
                                                               int64_t n, int32_t nx, int32_t nxy, FastDiv dnx,
                                                               FastDiv dnxy, PopVals<typename Prec<PREC>::T> dw,
                                                               double* __restrict__ partials) {
    using P = Prec<PREC>;
    using T = typename P::T;
    double acc[FORCE_VALS] = {0, 0, 0, 0, 0, 0};
    for (int64_t k = blockIdx.x * (int64_t)RED_THREADS + threadIdx.x; k < count; k += (int64_t)gridDim.x * RED_THREADS) {
        const int32_t idx = cells[k];
        const uint32_t m = masks[k];
        const int32_t z = (int32_t)dnxy.div((uint32_t)idx);
        const int32_t y = (int32_t)dnx.div((uint32_t)(idx - z * nxy));
        T fx = (T)0.0, fy = (T)0.0, fz = (T)0.0, bx = (T)0.0, by = (T)0.0, bz = (T)0.0;
        unroll<1, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            if (m & (1u << (i - 1))) {
                // 2 (f_i - w_i) per link (server/lbm.py:189); shifted storage holds f_i - e_i,
                // so f_i - w_i = stored + (e_i - w_i)
                T v;
                if constexpr (P::shifted) v = (T)2.0 * (P::to(f[(int64_t)i * n + idx]) + dw.v[i]);
                else v = (T)2.0 * (P::to(f[(int64_t)i * n + idx]) - (T)wd(i));
                if constexpr (cx(i) > 0) fx = fx + v;
                if constexpr (cx(i) < 0) fx = fx - v;
                if constexpr (cy(i) > 0) fy = fy + v;
                if constexpr (cy(i) < 0) fy = fy - v;
                if constexpr (cz(i) > 0) fz = fz + v;
                if constexpr (cz(i) < 0) fz = fz - v;
                if (y + cy(i) != 0) {  // links into the y = 0 plane are left out of the body force
                    if constexpr (cx(i) > 0) bx = bx + v;
                    if constexpr (cx(i) < 0) bx = bx - v;
                    if constexpr (cy(i) > 0) by = by + v;
                    if constexpr (cy(i) < 0) by = by - v;
                    if constexpr (cz(i) > 0) bz = bz + v;
                    if constexpr (cz(i) < 0) bz = bz - v;
                }
            }
        });
        acc[0] += (double)fx; acc[1] += (double)fy; acc[2] += (double)fz;
        acc[3] += (double)bx; acc[4] += (double)by; acc[5] += (double)bz;
    }
    block_reduce_store<FORCE_VALS>(acc, partials + (int64_t)blockIdx.x * FORCE_VALS);
}

template <int NV>
__global__ void __launch_bounds__(RED_THREADS) k_final(const double* __restrict__ partials, int nblocks,
                                                       double* __restrict__ out) {
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += RED_THREADS) {
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += partials[(int64_t)b * NV + k];
    }
    block_reduce_store<NV>(acc, out);
}

template <int PREC>
__global__ void __launch_bounds__(RED_THREADS) k_mass_partial(const typename Prec<PREC>::S* __restrict__ f,
                                                              const uint8_t* __restrict__ solid, int64_t n,
                                                              PopVals<typename Prec<PREC>::T> e,
                                                              double* __restrict__ partials) {
    using P = Prec<PREC>;
    double acc[1] = {0.0};
    for (int64_t idx = blockIdx.x * (int64_t)RED_THREADS + threadIdx.x; idx < n; idx += (int64_t)RED_BLOCKS * RED_THREADS) {
        if (solid[idx] != 0) continue;
        double c = 0.0;
        unroll<0, Q>([&](auto ic) {
            constexpr int i = decltype(ic)::value;
            double v = (double)P::to(f[(int64_t)i * n + idx]);
            if constexpr (P::shifted) v += (double)e.v[i];  // the shift as the kernels apply it
            c += v;
        });
        acc[0] += c;
    }
    block_reduce_store<1>(acc, partials + blockIdx.x);
}

template <int PREC>
PopVals<typename Prec<PREC>::T> shift_vals(const wt_grid* g, bool dw) {
    using T = typename Prec<PREC>::T;
    const ShiftTables t = shift_tables(Prec<PREC>::shifted ? (double)g->shift_u : 0.0);
    PopVals<T> r;
    for (int i = 0; i < Q; ++i) r.v[i] = (T)(dw ? t.dw[i] : t.e[i]);
    return r;
}

template <int PREC>
int forces_impl(const wt_grid* g, int32_t cur, const int32_t* cells, const uint32_t* masks, int64_t count,
                double* partials, double* out6, cudaStream_t st) {
    using S = typename Prec<PREC>::S;
    const int32_t nxy = g->nx * g->ny;
    const int64_t n = (int64_t)nxy * g->nz;
    k_force_partial<PREC><<<RED_BLOCKS, RED_THREADS, 0, st>>>(static_cast<const S*>(g->f[cur]), cells, masks, count,
                                                              n, g->nx, nxy, FastDiv((uint32_t)g->nx),
                                                              FastDiv((uint32_t)nxy), shift_vals<PREC>(g, true),
                                                              partials);
    k_final<FORCE_VALS><<<1, RED_THREADS, 0, st>>>(partials, RED_BLOCKS, out6);
    return wt_cuda_check("wt_forces launch");
}

template <int PREC>
int mass_impl(const wt_grid* g, int32_t cur, double* partials, double* out1, cudaStream_t st) {
    using S = typename Prec<PREC>::S;
    const int64_t n = (int64_t)g->nx * g->ny * g->nz;
    k_mass_partial<PREC><<<RED_BLOCKS, RED_THREADS, 0, st>>>(static_cast<const S*>(g->f[cur]), g->solid, n,
                                                             shift_vals<PREC>(g, false), partials);
    k_final<1><<<1, RED_THREADS, 0, st>>>(partials, RED_BLOCKS, out1);
    return wt_cuda_check("wt_mass launch");
}

}  // namespace wt

using namespace wt;

extern "C" int64_t wt_reduce_scratch_len(int64_t count) {
    (void)count;
    return (int64_t)RED_BLOCKS * FORCE_VALS;
}

extern "C" int wt_forces(const wt_grid* g, int32_t cur, const int32_t* cells, const uint32_t* masks, int64_t n_links,
                         double* partials, double* out6, void* stream) {
    if (!g || !g->f[0] || !g->f[1] || !partials || !out6) return wt_set_error(WT_ERR_ARG, "wt_forces: null buffer");
    if (n_links < 0 || (n_links > 0 && (!cells || !masks))) return wt_set_error(WT_ERR_ARG, "wt_forces: bad link list");
    if (cur != 0 && cur != 1) return wt_set_error(WT_ERR_ARG, "wt_forces: cur must be 0 or 1");
    if (int rc = wt_check_dims(g->nx, g->ny, g->nz)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (g->precision) {
        case WT_F32: return forces_impl<WT_F32>(g, cur, cells, masks, n_links, partials, out6, st);
        case WT_F16: return forces_impl<WT_F16>(g, cur, cells, masks, n_links, partials, out6, st);
        case WT_BF16: return forces_impl<WT_BF16>(g, cur, cells, masks, n_links, partials, out6, st);
        case WT_F64: return forces_impl<WT_F64>(g, cur, cells, masks, n_links, partials, out6, st);
        default: return wt_set_error(WT_ERR_ARG, "wt_forces: unknown precision %d", g->precision);
    }
}

extern "C" int wt_mass(const wt_grid* g, int32_t cur, double* partials, double* out1, void* stream) {
    if (!g || !g->f[0] || !g->f[1] || !g->solid || !partials || !out1)
        return wt_set_error(WT_ERR_ARG, "wt_mass: null buffer");
    if (cur != 0 && cur != 1) return wt_set_error(WT_ERR_ARG, "wt_mass: cur must be 0 or 1");
    if (int rc = wt_check_dims(g->nx, g->ny, g->nz)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (g->precision) {
        case WT_F32: return mass_impl<WT_F32>(g, cur, partials, out1, st);
        case WT_F16: return mass_impl<WT_F16>(g, cur, partials, out1, st);
        case WT_BF16: return mass_impl<WT_BF16>(g, cur, partials, out1, st);
        case WT_F64: return mass_impl<WT_F64>(g, cur, partials, out1, st);
        default: return wt_set_error(WT_ERR_ARG, "wt_mass: unknown precision %d", g->precision);
    }
}

// ---------------------------------------------------------------------------------------
// Forces without caller-provided scratch.
//
// Some callers cannot allocate device memory on the call path: a host framework that owns
// the device's memory pool and hands this library only its input and output buffers
// (a plugin), or a per-frame serving loop where a cudaMalloc/cudaFree pair would
// synchronise the device and stall every tunnel sharing the GPU. For them the block
// partials of the force reduction live in the array below, compiled into the library:
// every GPU that loads libwt.so holds these 192 KB until the process exits.
//
// Limits and sharing: one block of RED_THREADS threads per RED_THREADS link cells, so at
// most NOALLOC_MAX_BLOCKS * RED_THREADS = 1,048,576 link cells per call; longer lists are
// rejected with WT_ERR_CAPACITY. Every call on a device uses the same array and it keeps
// the last call's contents. Nothing has to start at zero: each call writes every partial
// it then reads. Calls whose kernels overlap on the GPU (different streams, no ordering
// between them) race on the array and must not be issued.
// ---------------------------------------------------------------------------------------
constexpr int NOALLOC_MAX_BLOCKS = 4096;
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_BLOCKS * FORCE_VALS];

// The current thread's CUDA context as a process-unique id (driver cuCtxGetCurrent +
// cuCtxGetId, fetched through the runtime so the library needs no link to libcuda); 0 when
// no context is current or the driver lacks the entry points.
static unsigned long long current_context_id() {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        return cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
                       q == cudaDriverEntryPointSuccess
                   ? reinterpret_cast<GetCurrent>(fn)
                   : nullptr;
    }();
    static GetId get_id = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        return cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
                       q == cudaDriverEntryPointSuccess
                   ? reinterpret_cast<GetId>(fn)
                   : nullptr;
    }();
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of g_noalloc_partials in the current device's context, looked up on the
// first call on each device and again whenever that device's context has been re-created
// (after cudaDeviceReset, say): the host-side symbol is only a stand-in and must never be
// passed to a kernel, and an address from a destroyed context must not be reused.
static int noalloc_scratch(double** out) {
    struct Entry {
        unsigned long long ctx;
        double* addr;
    };
    static std::mutex mu;
    static Entry cache[128] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
        return wt_set_error(WT_ERR_CUDA, "wt_forces_noalloc: no current CUDA device");
    std::lock_guard<std::mutex> lock(mu);
    const unsigned long long ctx = current_context_id();
    if (!cache[dev].addr || ctx == 0 || cache[dev].ctx != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);  // makes the context current
        if (e != cudaSuccess || !p)
            return wt_set_error(WT_ERR_CUDA, "wt_forces_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        cache[dev].addr = static_cast<double*>(p);
        cache[dev].ctx = current_context_id();
    }
    *out = cache[dev].addr;
    return WT_OK;
}

template <int PREC>
static int forces_noalloc_impl(const wt_grid* g, int32_t cur, const int32_t* cells, const uint32_t* masks,
                               int64_t count, double* partials, double* out6, cudaStream_t st) {
    using S = typename Prec<PREC>::S;
    const int32_t nxy = g->nx * g->ny;
    const int64_t n = (int64_t)nxy * g->nz;
    const int nb = (int)((count + RED_THREADS - 1) / RED_THREADS);
    if (nb > 0)
        k_force_partial<PREC><<<nb, RED_THREADS, 0, st>>>(static_cast<const S*>(g->f[cur]), cells, masks, count, n,
                                                           g->nx, nxy, FastDiv((uint32_t)g->nx), FastDiv((uint32_t)nxy),
                                                           shift_vals<PREC>(g, true), partials);
    k_final<FORCE_VALS><<<1, RED_THREADS, 0, st>>>(partials, nb, out6);
    return wt_cuda_check("wt_forces_noalloc launch");
}

extern "C" int wt_forces_noalloc(const wt_grid* g, int32_t cur, const int32_t* cells, const uint32_t* masks,
                                 int64_t n_links, double* out6, void* stream) {
    if (n_links > (int64_t)NOALLOC_MAX_BLOCKS * RED_THREADS)
        return wt_set_error(WT_ERR_CAPACITY,
                            "wt_forces_noalloc: %lld link cells exceed the built-in scratch limit of %d; "
                            "use wt_forces with caller scratch",
                            (long long)n_links, NOALLOC_MAX_BLOCKS * RED_THREADS);
    if (!g || !g->f[0] || !g->f[1] || !out6) return wt_set_error(WT_ERR_ARG, "wt_forces_noalloc: null buffer");
    if (n_links < 0 || (n_links > 0 && (!cells || !masks)))
        return wt_set_error(WT_ERR_ARG, "wt_forces_noalloc: bad link list");
    if (cur != 0 && cur != 1) return wt_set_error(WT_ERR_ARG, "wt_forces_noalloc: cur must be 0 or 1");
    if (int rc = wt_check_dims(g->nx, g->ny, g->nz)) return rc;
    double* partials = nullptr;
    if (int rc = noalloc_scratch(&partials)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (g->precision) {
        case WT_F32: return forces_noalloc_impl<WT_F32>(g, cur, cells, masks, n_links, partials, out6, st);
        case WT_F16: return forces_noalloc_impl<WT_F16>(g, cur, cells, masks, n_links, partials, out6, st);
        case WT_BF16: return forces_noalloc_impl<WT_BF16>(g, cur, cells, masks, n_links, partials, out6, st);
        case WT_F64: return forces_noalloc_impl<WT_F64>(g, cur, cells, masks, n_links, partials, out6, st);
        default: return wt_set_error(WT_ERR_ARG, "wt_forces_noalloc: unknown precision %d", g->precision);
    }
}
