// Definitions behind wt_variants.cuh: the tile-variant tables and launchers of the
// single-tunnel step kernels and of the batched kernels, templated on the storage precision.
// Each wt_kernels_<prec>.cu includes this once and instantiates one precision
// (WT_INSTANTIATE), so the four precisions compile in parallel.
#pragma once

#include "wt_step_impl.cuh"
#include "wt_variants.cuh"

namespace wt {

// ---- single tunnel ----

template <int PREC, bool FAST, int V, int BLOCK, int MINB, bool EARLY = false>
static int launch_bulk(const void* args, int32_t n, cudaStream_t st) {
    using P = Prec<PREC>;
    const auto& a = *static_cast<const StepArgs<typename P::S, typename P::T>*>(args);
    const int32_t nthreads = n / V;
    k_step_bulk<PREC, FAST, V, BLOCK, MINB, EARLY><<<(unsigned)((nthreads + BLOCK - 1) / BLOCK), BLOCK, 0, st>>>(a);
    return WT_OK;
}

template <int PREC, bool FAST, int L, int NS, int THREADS, int MINB, int CPT>
static int launch_stream(const void* args, int32_t n, cudaStream_t st) {
    using P = Prec<PREC>;
    using LY = StreamLayout<typename P::S, L>;
    constexpr int SMEM = NS * LY::STAGE_BYTES + 2 * NS * 8;
    if (SMEM > 227 * 1024) return wt_set_error(WT_ERR_ARG, "streaming tile needs %d bytes of shared memory", SMEM);
    static bool configured = false;
    if (!configured) {
        if (cudaFuncSetAttribute(k_step_stream<PREC, FAST, L, NS, THREADS, MINB, CPT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM) != cudaSuccess)
            return wt_cuda_check("wt_step: shared-memory carve-out");
        configured = true;
    }
    const auto& a = *static_cast<const StepArgs<typename P::S, typename P::T>*>(args);
    const int32_t nchunks = (n + L - 1) / L;
    const int32_t grid = std::min(nchunks, num_sms() * MINB);
    k_step_stream<PREC, FAST, L, NS, THREADS, MINB, CPT><<<grid, THREADS, SMEM, st>>>(a);
    return WT_OK;
}

// the row-grid arguments of one tunnel's step: its StepArgs plus the per-population byte offsets
// of the pull and store
template <class S, class T>
static void fill_rows(RowArgs<S, T>& r, const StepArgs<S, T>& a) {
    r.a = a;
    for (int i = 0; i < Q; ++i) {
        // the pair of population i is pulled from cells idx - (cy, cz) (the x shift cancels
        // against the pair's alignment)
        r.loff[i] = ((int64_t)i * a.n - (int64_t)cy(i) * a.nx - (int64_t)cz(i) * a.nxy) * (int64_t)sizeof(S);
        r.soff[i] = (int64_t)i * a.n * (int64_t)sizeof(S);
    }
}

template <int PREC, bool FAST, int BLOCK, int MINB, int ADDR, bool FUSE = false, bool EARLY = false>
static int launch_rows(const void* args, int32_t n, cudaStream_t st) {
    using P = Prec<PREC>;
    using S = typename P::S;
    using T = typename P::T;
    (void)n;
    RowArgs<S, T> r;
    fill_rows<S, T>(r, *static_cast<const StepArgs<S, T>*>(args));
    const StepArgs<S, T>& a = r.a;
    const dim3 grid((unsigned)((a.nx / 2 + BLOCK - 1) / BLOCK), (unsigned)a.ny, (unsigned)a.nz);
    k_step_rows<PREC, FAST, BLOCK, MINB, ADDR, FUSE, EARLY><<<grid, BLOCK, 0, st>>>(r);
    return WT_OK;
}

// Tile variants. Direct-load forms (kind 0): cells per thread (V), threads per block, minimum
// resident blocks per SM. Streaming forms (kind 1): chunk length L, pipeline stages NS,
// threads per block, blocks per SM. Row-grid forms (kind 2, k_step_rows): two cells per
// thread, threads per block, minimum resident blocks per SM, and in the last field the
// addressing form (0: per-population bases, 1: one base plus byte offsets); kind 4 is the row
// grid with the face cells of k_step_faces computed by the blocks of the rows they read
// (k_step_rows with FUSE), so the step is one kernel. Tiles 29-32 issue each pair's pull
// together with its code bytes instead of after them (EARLY): 29 is tile 18 so, 30-32 are
// tiles 19, 21 and 22, and 33-35 the same rows at 32 threads x 32 blocks and 64 threads x 14
// or 12 blocks per SM. wt_grid.tile
// selects one (0 = the default for the precision and collision form); autotune.py times them.
#define WT_VARIANTS(PREC, FAST)                                                          \
    {1, 0, 1, 256, 4, 0, 0, launch_bulk<PREC, FAST, 1, 256, 4>},                         \
    {2, 0, 1, 128, 8, 0, 0, launch_bulk<PREC, FAST, 1, 128, 8>},                         \
    {3, 0, 2, 128, 6, 0, 0, launch_bulk<PREC, FAST, 2, 128, 6>},                         \
    {4, 0, 2, 128, 4, 0, 0, launch_bulk<PREC, FAST, 2, 128, 4>},                         \
    {5, 0, 4, 128, 4, 0, 0, launch_bulk<PREC, FAST, 4, 128, 4>},                         \
    {6, 0, 4, 128, 3, 0, 0, launch_bulk<PREC, FAST, 4, 128, 3>},                         \
    {7, 0, 2, 256, 3, 0, 0, launch_bulk<PREC, FAST, 2, 256, 3>},                         \
    {8, 1, 1, 512, 2, 480, 3, launch_stream<PREC, FAST, 480, 3, 512, 2, 1>},             \
    {9, 1, 1, 512, 2, 480, 2, launch_stream<PREC, FAST, 480, 2, 512, 2, 1>},             \
    {10, 1, 1, 1024, 1, 992, 2, launch_stream<PREC, FAST, 992, 2, 1024, 1, 1>},          \
    {11, 1, 2, 512, 1, 960, 2, launch_stream<PREC, FAST, 960, 2, 512, 1, 2>},            \
    {12, 1, 1, 512, 2, 480, 4, launch_stream<PREC, FAST, 480, 4, 512, 2, 1>},            \
    {13, 1, 2, 512, 2, 960, 2, launch_stream<PREC, FAST, 960, 2, 512, 2, 2>},            \
    {14, 1, 2, 512, 1, 960, 3, launch_stream<PREC, FAST, 960, 3, 512, 1, 2>},            \
    {15, 1, 2, 512, 1, 960, 4, launch_stream<PREC, FAST, 960, 4, 512, 1, 2>},            \
    {16, 1, 2, 256, 2, 448, 4, launch_stream<PREC, FAST, 448, 4, 256, 2, 2>},            \
    {17, 1, 2, 384, 1, 704, 4, launch_stream<PREC, FAST, 704, 4, 384, 1, 2>},            \
    {18, 0, 2, 128, 8, 0, 0, launch_bulk<PREC, FAST, 2, 128, 8>},                        \
    {19, 2, 2, 128, 8, 0, 0, launch_rows<PREC, FAST, 128, 8, 0>},                        \
    {20, 2, 2, 128, 8, 0, 1, launch_rows<PREC, FAST, 128, 8, 1>},                        \
    {21, 2, 2, 64, 16, 0, 0, launch_rows<PREC, FAST, 64, 16, 0>},                        \
    {22, 2, 2, 64, 16, 0, 1, launch_rows<PREC, FAST, 64, 16, 1>},                        \
    {23, 2, 2, 256, 4, 0, 1, launch_rows<PREC, FAST, 256, 4, 1>},                        \
    {24, 2, 2, 128, 4, 0, 0, launch_rows<PREC, FAST, 128, 4, 0>},                        \
    {25, 2, 2, 128, 9, 0, 0, launch_rows<PREC, FAST, 128, 9, 0>},                        \
    {26, 2, 2, 128, 10, 0, 0, launch_rows<PREC, FAST, 128, 10, 0>},                      \
    {27, 4, 2, 128, 8, 0, 0, launch_rows<PREC, FAST, 128, 8, 0, true>},                  \
    {28, 4, 2, 64, 16, 0, 0, launch_rows<PREC, FAST, 64, 16, 0, true>},                 \
    {29, 0, 2, 128, 8, 0, 0, launch_bulk<PREC, FAST, 2, 128, 8, true>},                  \
    {30, 2, 2, 128, 8, 0, 0, launch_rows<PREC, FAST, 128, 8, 0, false, true>},           \
    {31, 2, 2, 64, 16, 0, 0, launch_rows<PREC, FAST, 64, 16, 0, false, true>},           \
    {32, 2, 2, 64, 16, 0, 1, launch_rows<PREC, FAST, 64, 16, 1, false, true>},           \
    {33, 2, 2, 32, 32, 0, 0, launch_rows<PREC, FAST, 32, 32, 0, false, true>},           \
    {34, 2, 2, 64, 14, 0, 0, launch_rows<PREC, FAST, 64, 14, 0, false, true>},           \
    {35, 2, 2, 64, 12, 0, 0, launch_rows<PREC, FAST, 64, 12, 0, false, true>}

template <int PREC, bool FAST>
const StepVariant* variants_of(int* count) {
    static const StepVariant table[] = {WT_VARIANTS(PREC, FAST)};
    *count = (int)(sizeof(table) / sizeof(table[0]));
    return table;
}

template <int PREC>
const StepVariant* step_variants(bool fast, int* count) {
    return fast ? variants_of<PREC, true>(count) : variants_of<PREC, false>(count);
}

// defaults until the autotuner has measured the tunnel, chosen from timings of the benchmark body
// at nx = 512, 320, 200 and 144: the row-grid tiles win where a lattice row splits into whole
// blocks of pairs (each row's last block otherwise runs part-empty, and its partial warp takes
// the general pair path), the one-dimensional two-cell tiles elsewhere. fp32 and the
// reference-order collision: tile 34 (rows, 64 threads x 14 blocks, early pulls) when nx is a
// multiple of 128, else tile 18. fp16 / bf16 with the moment-space collision: tile 31 (rows, 64
// x 16, early pulls) when nx is a multiple of 128, tile 33 (rows, 32 x 32) when of 64, else tile
// 29 (one-dimensional, early pulls). fp32 with the moment-space collision: tile 27 (rows, 128 x
// 8, fused faces) when nx is a multiple of 256, else 18. Rows need nx >= 256 here: below that
// the grid is too small to have been timed. fp64 needs 128 registers to avoid spills, so it
// keeps two cells per thread at 128 registers (tile 4).
template <int PREC>
const StepVariant* pick_variant(const wt_grid* g) {
    int count;
    const bool fast = g->collision == WT_COLLIDE_FAST;
    const StepVariant* t = step_variants<PREC>(fast, &count);
    const bool half = PREC == WT_F16 || PREC == WT_BF16;
    const bool big = g->nx >= 256;
    int dflt = 18;
    if (PREC == WT_F64) dflt = 4;
    else if (fast && half) dflt = big && g->nx % 128 == 0 ? 31 : (big && g->nx % 64 == 0 ? 33 : 29);
    else if (fast) dflt = big && g->nx % 256 == 0 ? 27 : 18;
    else if (big && g->nx % 128 == 0) dflt = 34;
    const int want = g->tile > 0 ? g->tile : dflt;
    for (int k = 0; k < count; ++k) {
        if (t[k].id != want) continue;
        if (g->nx % t[k].v != 0) return nullptr;
        if (PREC == WT_F64 && t[k].v == 4) return nullptr;
        if (t[k].kind == 1 && g->nx % 16 != 0) return nullptr;  // 16-byte copies of rows and code bytes
        return &t[k];
    }
    return nullptr;
}

template <int PREC>
int step_prec(const wt_grid* g, int32_t cur, int32_t steps, double uin, double tau, double smag, int32_t flags,
              int32_t skip_chunk, cudaStream_t stream) {
    using P = Prec<PREC>;
    using T = typename P::T;
    using S = typename P::S;
    StepArgs<S, T> a;
    a.solid = g->solid;
    a.code = g->code;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    a.nxy = g->nx * g->ny;
    a.n = a.nxy * g->nz;
    a.dnx = FastDiv((uint32_t)g->nx);
    a.dny = FastDiv((uint32_t)g->ny);
    a.uin = (T)uin; a.tau = (T)tau;
    const T sm = (T)smag;
    a.csmag = (T)25.4558441 * sm * sm;  // same left-to-right product as server/lbm.py:152
    const StepVariant* var = pick_variant<PREC>(g);
    if (!var) return wt_set_error(WT_ERR_ARG, "wt_step: no kernel variant for tile %d (nx=%d)", g->tile, g->nx);
    for (int b = 0; b < 2; ++b) {
        const uintptr_t al = reinterpret_cast<uintptr_t>(g->f[b]);
        if (al % 16 != 0) return wt_set_error(WT_ERR_ARG, "wt_step: population buffer %d not 16-byte aligned", b);
    }
    if (reinterpret_cast<uintptr_t>(g->code) % 16 != 0)
        return wt_set_error(WT_ERR_ARG, "wt_step: code buffer not 16-byte aligned");
    a.status = g->status;
    a.test_skip_chunk = skip_chunk;
    set_shift(a, P::shifted ? (double)g->shift_u : 0.0);
    constexpr int VEC = 16 / (int)sizeof(S);
    const int32_t nface = a.nxy + a.nx * (a.nz - 2);
    const unsigned nb_face = (unsigned)((nface + 255) / 256);
    for (int32_t s = 0; s < steps; ++s) {
        const S* fin = static_cast<const S*>(g->f[cur]);
        S* fout = static_cast<S*>(g->f[cur ^ 1]);
        for (int i = 0; i < Q; ++i) {
            const int64_t off = cx(i) + (int64_t)cy(i) * a.nx + (int64_t)cz(i) * a.nxy;
            a.src[i] = fin + (int64_t)i * a.n - off;
            a.dst[i] = fout + (int64_t)i * a.n;
            const int32_t r = (int32_t)(((-off) % VEC + VEC) % VEC);  // n and chunk starts are multiples of VEC
            a.chunk_r[i] = r;
            a.chunk_src[i] = a.src[i] - r;
        }
        a.fin = fin;
        a.mac_prev = static_cast<const T*>(g->mac[cur]);
        a.mac_cur = static_cast<T*>(g->mac[cur ^ 1]);
        a.mac_all = (flags & WT_STEP_MAC_ALL_LAST) && s == steps - 1;
        if (int rc = var->launch(&a, a.n, stream)) return rc;
        if (var->kind != 4) k_step_faces<PREC><<<nb_face, 256, 0, stream>>>(a);
        cur ^= 1;
    }
    return wt_cuda_check("wt_step launch");
}

// ---- many tunnels: one persistent bulk kernel over a work list, then one face kernel ----

// one descriptor into shared memory (all threads; two barriers around the use)
template <class A>
__device__ __forceinline__ void copy_desc(A* dst, const A* src) {
    static_assert(sizeof(A) % 4 == 0, "descriptor size");
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(dst);
    for (int k = threadIdx.x; k < (int)(sizeof(A) / 4); k += blockDim.x) d[k] = s[k];
}

template <int PREC, bool FAST, int V, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_batch_bulk(const BatchArgs b) {
    using A = StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>;
    __shared__ __align__(16) A a;
#pragma unroll 1
    for (int32_t w = blockIdx.x; w < b.n_bulk; w += gridDim.x) {
        const int2 item = b.bulk[w];
        copy_desc(&a, static_cast<const A*>(b.desc) + item.x * 4 + b.parity * 2 + b.mac_all);
        __syncthreads();
        // SUB consecutive sub-tiles of BLOCK * V cells, no barrier between them
#pragma unroll 1
        for (int sub = 0; sub < ITEM_SUB; ++sub) {
            const int32_t idx0 = item.y + (sub * BLOCK + (int32_t)threadIdx.x) * V;
            bulk_cells<PREC, FAST, V>(a, idx0, idx0 < a.n);
        }
        __syncthreads();
    }
}

template <int PREC>
__global__ void __launch_bounds__(FACE_BLOCK) k_batch_faces(const BatchArgs b) {
    using A = StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>;
    __shared__ __align__(16) A a;
#pragma unroll 1
    for (int32_t w = blockIdx.x; w < b.n_faces; w += gridDim.x) {
        const int2 item = b.faces[w];
        copy_desc(&a, static_cast<const A*>(b.desc) + item.x * 4 + b.parity * 2 + b.mac_all);
        __syncthreads();
#pragma unroll 1
        for (int sub = 0; sub < ITEM_SUB; ++sub) face_cell<PREC>(a, item.y + sub * FACE_BLOCK + (int32_t)threadIdx.x);
        __syncthreads();
    }
}

// Grid forms of the same two kernels: one block per sub-tile of the work list (block b: item
// b / ITEM_SUB, sub-tile b % ITEM_SUB), the descriptor read in place from the workspace. With no
// loop over items the compiler keeps no descriptor field in a register across tiles, so the
// two-cell tile fits the 64 registers of the single-tunnel tile 18 (the persistent loop above
// needs 80, or spills).
template <int PREC, bool FAST, int V, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_batch_bulk_grid(const BatchArgs b) {
    using A = StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>;
    const int32_t w = (int32_t)blockIdx.x / ITEM_SUB, sub = (int32_t)blockIdx.x % ITEM_SUB;
    const int2 item = b.bulk[w];
    const A* __restrict__ a = static_cast<const A*>(b.desc) + item.x * 4 + b.parity * 2 + b.mac_all;
    const int32_t idx0 = item.y + (sub * BLOCK + (int32_t)threadIdx.x) * V;
    bulk_cells<PREC, FAST, V>(*a, idx0, idx0 < a->n);
}

template <int PREC>
__global__ void __launch_bounds__(FACE_BLOCK) k_batch_faces_grid(const BatchArgs b) {
    using A = StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>;
    const int32_t w = (int32_t)blockIdx.x / ITEM_SUB, sub = (int32_t)blockIdx.x % ITEM_SUB;
    const int2 item = b.faces[w];
    const A* __restrict__ a = static_cast<const A*>(b.desc) + item.x * 4 + b.parity * 2 + b.mac_all;
    face_cell<PREC>(*a, item.y + sub * FACE_BLOCK + (int32_t)threadIdx.x);
}

template <int PREC, bool FAST, int V, int BLOCK, int MINB>
static void launch_batch_bulk_grid(const void* args, int grid, cudaStream_t st) {
    k_batch_bulk_grid<PREC, FAST, V, BLOCK, MINB><<<grid, BLOCK, 0, st>>>(*static_cast<const BatchArgs*>(args));
}
template <int PREC>
static void launch_batch_faces_grid(const void* args, int grid, cudaStream_t st) {
    k_batch_faces_grid<PREC><<<grid, FACE_BLOCK, 0, st>>>(*static_cast<const BatchArgs*>(args));
}

template <int PREC, bool FAST, int V, int BLOCK, int MINB>
static void launch_batch_bulk(const void* args, int grid, cudaStream_t st) {
    k_batch_bulk<PREC, FAST, V, BLOCK, MINB><<<grid, BLOCK, 0, st>>>(*static_cast<const BatchArgs*>(args));
}
template <int PREC>
static void launch_batch_faces(const void* args, int grid, cudaStream_t st) {
    k_batch_faces<PREC><<<grid, FACE_BLOCK, 0, st>>>(*static_cast<const BatchArgs*>(args));
}

// Parameter-space forms: the descriptors of up to MAXT tunnels and each tunnel's first block
// (prefix sums of its block counts) are the kernel's argument, read through the constant bank;
// block b belongs to the last tunnel t with first[t] <= b. No load of a work item or a
// descriptor stands between a block's start and its pull.
template <class S, class T>
struct BatchParams {
    static constexpr int MAXT = (32764 - 16) / (int)(sizeof(StepArgs<S, T>) + 4);
    int32_t count;
    int32_t first[MAXT + 1];
    StepArgs<S, T> args[MAXT];
};

template <class BP>
__device__ __forceinline__ int32_t param_tunnel(const BP& bp, int32_t b) {
    int32_t lo = 0, hi = bp.count - 1;
    while (lo < hi) {
        const int32_t mid = (lo + hi + 1) >> 1;
        if (bp.first[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int PREC, bool FAST, int V, int BLOCK, int MINB, bool EARLY>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_batch_bulk_params(const __grid_constant__ BatchParams<typename Prec<PREC>::S, typename Prec<PREC>::T> bp) {
    const int32_t b = (int32_t)blockIdx.x;
    const int32_t t = param_tunnel(bp, b);
    const auto& a = bp.args[t];
    const int32_t idx0 = ((b - bp.first[t]) * BLOCK + (int32_t)threadIdx.x) * V;
    bulk_cells<PREC, FAST, V, EARLY>(a, idx0, idx0 < a.n);
}

template <int PREC>
__global__ void __launch_bounds__(FACE_BLOCK)
    k_batch_faces_params(const __grid_constant__ BatchParams<typename Prec<PREC>::S, typename Prec<PREC>::T> bp) {
    const int32_t b = (int32_t)blockIdx.x;
    const int32_t t = param_tunnel(bp, b);
    face_cell<PREC>(bp.args[t], (b - bp.first[t]) * FACE_BLOCK + (int32_t)threadIdx.x);
}

// FACES: the face kernel (FACE_BLOCK face cells per block) instead of the bulk one
template <int PREC, bool FAST, int V, int BLOCK, int MINB, bool EARLY, bool FACES>
static int launch_batch_params(const void* descs, int32_t count, cudaStream_t st) {
    using S = typename Prec<PREC>::S;
    using T = typename Prec<PREC>::T;
    using BP = BatchParams<S, T>;
    static_assert(sizeof(BP) <= 32764, "kernel parameters are limited to 32764 bytes");
    const StepArgs<S, T>* d = static_cast<const StepArgs<S, T>*>(descs);
    BP bp;
    for (int32_t g0 = 0; g0 < count; g0 += BP::MAXT) {
        const int32_t gc = std::min<int32_t>(count - g0, BP::MAXT);
        bp.count = gc;
        bp.first[0] = 0;
        for (int32_t t = 0; t < gc; ++t) {
            const StepArgs<S, T>& a = d[g0 + t];
            bp.args[t] = a;
            const int64_t cells = FACES ? (int64_t)a.nxy + (int64_t)a.nx * (a.nz - 2) : (int64_t)a.n;
            const int64_t per = FACES ? FACE_BLOCK : (int64_t)BLOCK * V;
            bp.first[t + 1] = bp.first[t] + (int32_t)((cells + per - 1) / per);
        }
        if constexpr (FACES) k_batch_faces_params<PREC><<<(unsigned)bp.first[gc], FACE_BLOCK, 0, st>>>(bp);
        else k_batch_bulk_params<PREC, FAST, V, BLOCK, MINB, EARLY><<<(unsigned)bp.first[gc], BLOCK, 0, st>>>(bp);
    }
    return WT_OK;
}

// the direct-load tile shapes of wt_step, same ids, as persistent kernels; ids 100 + k are
// the grid forms of tile k, ids 200 + k the parameter-space forms (229: tile 18 with the pull
// issued with the code bytes, as single-tunnel tile 29)
#define WT_BATCH_P(PREC, FAST, V, BLOCK, MINB, EARLY)                                                        \
    nullptr, nullptr, launch_batch_params<PREC, FAST, V, BLOCK, MINB, EARLY, false>,                          \
        launch_batch_params<PREC, FAST, V, BLOCK, MINB, EARLY, true>
#define WT_BATCH_VARIANTS(PREC, FAST)                                                                        \
    {1, 1, 256, 4, BATCH_PERSISTENT, launch_batch_bulk<PREC, FAST, 1, 256, 4>, launch_batch_faces<PREC>},    \
    {2, 1, 128, 8, BATCH_PERSISTENT, launch_batch_bulk<PREC, FAST, 1, 128, 8>, launch_batch_faces<PREC>},    \
    {3, 2, 128, 6, BATCH_PERSISTENT, launch_batch_bulk<PREC, FAST, 2, 128, 6>, launch_batch_faces<PREC>},    \
    {4, 2, 128, 4, BATCH_PERSISTENT, launch_batch_bulk<PREC, FAST, 2, 128, 4>, launch_batch_faces<PREC>},    \
    {5, 4, 128, 4, BATCH_PERSISTENT, launch_batch_bulk<PREC, FAST, 4, 128, 4>, launch_batch_faces<PREC>},    \
    {7, 2, 256, 3, BATCH_PERSISTENT, launch_batch_bulk<PREC, FAST, 2, 256, 3>, launch_batch_faces<PREC>},    \
    {18, 2, 128, 8, BATCH_PERSISTENT, launch_batch_bulk<PREC, FAST, 2, 128, 8>, launch_batch_faces<PREC>},   \
    {102, 1, 128, 8, BATCH_GRID, launch_batch_bulk_grid<PREC, FAST, 1, 128, 8>, launch_batch_faces_grid<PREC>}, \
    {103, 2, 128, 6, BATCH_GRID, launch_batch_bulk_grid<PREC, FAST, 2, 128, 6>, launch_batch_faces_grid<PREC>}, \
    {104, 2, 128, 4, BATCH_GRID, launch_batch_bulk_grid<PREC, FAST, 2, 128, 4>, launch_batch_faces_grid<PREC>}, \
    {118, 2, 128, 8, BATCH_GRID, launch_batch_bulk_grid<PREC, FAST, 2, 128, 8>, launch_batch_faces_grid<PREC>}, \
    {203, 2, 128, 6, BATCH_PARAMS, WT_BATCH_P(PREC, FAST, 2, 128, 6, false)},                                \
    {204, 2, 128, 4, BATCH_PARAMS, WT_BATCH_P(PREC, FAST, 2, 128, 4, false)},                                \
    {218, 2, 128, 8, BATCH_PARAMS, WT_BATCH_P(PREC, FAST, 2, 128, 8, false)},                                \
    {229, 2, 128, 8, BATCH_PARAMS, WT_BATCH_P(PREC, FAST, 2, 128, 8, true)}

template <int PREC, bool FAST>
const BatchVariant* batch_variant_of(int id) {
    static const BatchVariant table[] = {WT_BATCH_VARIANTS(PREC, FAST)};
    for (const auto& v : table)
        if (v.id == id) return &v;
    return nullptr;
}

template <int PREC>
const BatchVariant* batch_variant(bool fast, int id) {
    return fast ? batch_variant_of<PREC, true>(id) : batch_variant_of<PREC, false>(id);
}

}  // namespace wt

#define WT_INSTANTIATE(PREC)                                                                                       \
    namespace wt {                                                                                                 \
    template const StepVariant* step_variants<PREC>(bool, int*);                                                   \
    template int step_prec<PREC>(const wt_grid*, int32_t, int32_t, double, double, double, int32_t, int32_t, cudaStream_t); \
    template const BatchVariant* batch_variant<PREC>(bool, int);                                                   \
    }
