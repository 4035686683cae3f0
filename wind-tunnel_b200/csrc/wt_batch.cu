// Many tunnels of uneven sizes advanced together: one bulk kernel over a tile work-list
// spanning every tunnel, then one face kernel over all tunnels' face cells, per step; optionally
// captured as a CUDA graph of an even number of steps and replayed. The kernels come in three
// forms (wt_kernels.cuh): persistent (one wave of blocks looping over the lists), grid (one
// block per sub-tile of the lists, tile ids 100 + k), which fits the 64 registers of the
// single-tunnel two-cell tile, and parameter-space (tile ids 200 + k: the descriptors travel in
// the kernel arguments, groups of up to BatchParams::MAXT tunnels per launch, and the device
// workspace is unused).
//
// Device workspace of the first two forms (caller-allocated, wt_batch_workspace_bytes):
//   desc  -- 4 StepArgs per tunnel, indexed [tunnel][parity][mac_all]: parity p holds the
//            tunnel's buffers for cur = cur0 ^ p, so all tunnels flip together;
//   bulk  -- work items {tunnel, first cell} of BLOCK * V * ITEM_SUB cells each;
//   faces -- work items {tunnel, first face index} of FACE_BLOCK * ITEM_SUB face cells each.
// A persistent block copies the descriptor of its current item into shared memory; a grid-form
// block reads it in place. Either way the kernel body is the single-tunnel one (bulk_cells /
// face_cell of wt_step_impl.cuh) and every tunnel gives bit-identical results alone or in a
// batch. The kernels (k_batch_bulk, k_batch_faces)
// are instantiated per precision in wt_kernels_<prec>.cu; this file is the host side.
#include <cstring>
#include <vector>

#include "wt_step_impl.cuh"
#include "wt_variants.cuh"

using namespace wt;

struct wt_batch {
    int32_t precision, collision, count;
    int32_t base;  // parity offset: tunnel t's current buffer is cur0[t] ^ base
    std::vector<int32_t> cur0;
    const BatchVariant* var;
    void* desc;
    int2* bulk;
    int2* faces;
    int32_t n_bulk, n_faces;
    int grid_bulk, grid_faces;
    std::vector<unsigned char> pdesc;  // parameter-space form: descriptors [parity][mac_all][tunnel]
    std::vector<int32_t> par;          // parameter-space form: tunnel t's current buffer is cur0[t] ^ par[t]
    std::vector<unsigned char> group;  // parameter-space form: one step's descriptors, gathered
    size_t desc_bytes;
    cudaGraphExec_t graph;
    int32_t graph_steps;
};

namespace {

template <int PREC>
size_t desc_size() {
    return sizeof(StepArgs<typename Prec<PREC>::S, typename Prec<PREC>::T>);
}

size_t desc_bytes_for(int32_t precision) {
    switch (precision) {
        case WT_F32: return desc_size<WT_F32>();
        case WT_F16: return desc_size<WT_F16>();
        case WT_BF16: return desc_size<WT_BF16>();
        case WT_F64: return desc_size<WT_F64>();
        default: return 0;
    }
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// tile shape of a batch (direct-load variants only; 100 + k is the grid form of tile k, 200 + k
// its parameter-space form); 0 picks the parameter-space two-cell tile with early pulls (229),
// or at 128 registers (204) for fp64
int tile_shape(int32_t tile, int32_t precision, int* v, int* block) {
    static const int ids[][3] = {{1, 1, 256},   {2, 1, 128},   {3, 2, 128},   {4, 2, 128},   {5, 4, 128},
                                 {7, 2, 256},   {18, 2, 128},  {102, 1, 128}, {103, 2, 128}, {104, 2, 128},
                                 {118, 2, 128}, {203, 2, 128}, {204, 2, 128}, {218, 2, 128}, {229, 2, 128}};
    const int want = tile > 0 ? tile : (precision == WT_F64 ? 204 : 229);
    for (const auto& r : ids)
        if (r[0] == want) {
            *v = r[1];
            *block = r[2];
            return want;
        }
    return 0;
}

void work_counts(const wt_grid* grids, int32_t count, int tile_cells, int64_t* nb, int64_t* nf) {
    *nb = 0;
    *nf = 0;
    for (int32_t t = 0; t < count; ++t) {
        const int64_t n = (int64_t)grids[t].nx * grids[t].ny * grids[t].nz;
        const int64_t nface = (int64_t)grids[t].nx * grids[t].ny + (int64_t)grids[t].nx * (grids[t].nz - 2);
        *nb += (n + tile_cells - 1) / tile_cells;
        *nf += (nface + FACE_BLOCK * ITEM_SUB - 1) / (FACE_BLOCK * ITEM_SUB);
    }
}

template <int PREC>
void fill_desc(const wt_grid& g, int32_t cur0, double uin, double tau, double smag, int parity, int mac_all,
               void* out) {
    using P = Prec<PREC>;
    using T = typename P::T;
    using S = typename P::S;
    StepArgs<S, T> a;
    std::memset(&a, 0, sizeof(a));
    const int cur = cur0 ^ parity;
    a.solid = g.solid;
    a.code = g.code;
    a.nx = g.nx; a.ny = g.ny; a.nz = g.nz;
    a.nxy = g.nx * g.ny;
    a.n = a.nxy * g.nz;
    a.dnx = FastDiv((uint32_t)g.nx);
    a.dny = FastDiv((uint32_t)g.ny);
    a.uin = (T)uin; a.tau = (T)tau;
    const T sm = (T)smag;
    a.csmag = (T)25.4558441 * sm * sm;  // left-to-right, as server/lbm.py:152
    const S* fin = static_cast<const S*>(g.f[cur]);
    S* fout = static_cast<S*>(g.f[cur ^ 1]);
    constexpr int VEC = 16 / (int)sizeof(S);
    for (int i = 0; i < Q; ++i) {
        const int64_t off = cx(i) + (int64_t)cy(i) * a.nx + (int64_t)cz(i) * a.nxy;
        a.src[i] = fin + (int64_t)i * a.n - off;
        a.dst[i] = fout + (int64_t)i * a.n;
        const int32_t r = (int32_t)(((-off) % VEC + VEC) % VEC);
        a.chunk_r[i] = r;
        a.chunk_src[i] = a.src[i] - r;
    }
    a.fin = fin;
    a.mac_prev = static_cast<const T*>(g.mac[cur]);
    a.mac_cur = static_cast<T*>(g.mac[cur ^ 1]);
    a.mac_all = mac_all;
    a.status = g.status;
    a.test_skip_chunk = 0;
    set_shift(a, Prec<PREC>::shifted ? (double)g.shift_u : 0.0);
    std::memcpy(out, &a, sizeof(a));
}

// Parameter-space form: tunnel t advances each[t] steps (all `steps` when each is null). Step s
// launches the tunnels with more than s steps to go, each with the descriptor of its own
// parity, so tunnels with different counts keep their own buffer parity.
int launch_params(wt_batch* b, const int32_t* each, int32_t steps, int32_t flags, cudaStream_t st) {
    int32_t smax = steps;
    if (each) {
        smax = 0;
        for (int32_t t = 0; t < b->count; ++t) smax = std::max(smax, each[t]);
    }
    const size_t ds = b->desc_bytes;
    b->group.resize((size_t)b->count * ds);
    for (int32_t s = 0; s < smax; ++s) {
        int32_t m = 0;
        for (int32_t t = 0; t < b->count; ++t) {
            const int32_t k = each ? each[t] : steps;
            if (s >= k) continue;
            const int parity = (b->par[t] + s) & 1;
            const int mac_all = (flags & WT_STEP_MAC_ALL_LAST) && s == k - 1;
            std::memcpy(b->group.data() + (size_t)m * ds,
                        b->pdesc.data() + ((size_t)(parity * 2 + mac_all) * b->count + t) * ds, ds);
            ++m;
        }
        if (int rc = b->var->bulk_p(b->group.data(), m, st)) return rc;
        if (int rc = b->var->faces_p(b->group.data(), m, st)) return rc;
    }
    if (int rc = wt_cuda_check("wt_batch step launch")) return rc;
    for (int32_t t = 0; t < b->count; ++t) b->par[t] ^= (each ? each[t] : steps) & 1;
    return WT_OK;
}

int launch_steps(wt_batch* b, int32_t steps, int32_t flags, cudaStream_t st) {
    if (b->var->form == BATCH_PARAMS) return launch_params(b, nullptr, steps, flags, st);
    for (int32_t s = 0; s < steps; ++s) {
        const int parity = (b->base + s) & 1;
        const int mac_all = (flags & WT_STEP_MAC_ALL_LAST) && s == steps - 1;
        BatchArgs args{b->desc, b->bulk, b->faces, b->n_bulk, b->n_faces, parity, mac_all};
        b->var->bulk(&args, b->grid_bulk, st);
        b->var->faces(&args, b->grid_faces, st);
    }
    if (int rc = wt_cuda_check("wt_batch step launch")) return rc;
    b->base ^= steps & 1;
    return WT_OK;
}

}  // namespace

extern "C" int64_t wt_batch_workspace_bytes(const wt_grid* grids, int32_t count, int32_t tile) {
    if (!grids || count <= 0) return wt_set_error(WT_ERR_ARG, "wt_batch_workspace_bytes: no tunnels");
    int v, block;
    const int id = tile_shape(tile, grids[0].precision, &v, &block);
    if (!id) return wt_set_error(WT_ERR_ARG, "wt_batch: tile %d has no batched form", tile);
    const size_t ds = desc_bytes_for(grids[0].precision);
    if (!ds) return wt_set_error(WT_ERR_ARG, "wt_batch: unknown precision %d", grids[0].precision);
    if (id / 100 == 2) return 256;  // parameter-space form: nothing on the device
    int64_t nb, nf;
    work_counts(grids, count, v * block * ITEM_SUB, &nb, &nf);
    return (int64_t)(align256(4 * ds * count) + align256(8 * nb) + align256(8 * nf));
}

extern "C" int wt_batch_create(const wt_grid* grids, int32_t count, const double* uin, const double* tau,
                               const double* smag, const int32_t* cur, int32_t tile, void* workspace,
                               int64_t workspace_bytes, void* stream, wt_batch** out) {
    if (!grids || count <= 0 || !uin || !tau || !smag || !cur || !workspace || !out)
        return wt_set_error(WT_ERR_ARG, "wt_batch_create: null argument");
    const int32_t prec = grids[0].precision, coll = grids[0].collision;
    for (int32_t t = 0; t < count; ++t) {
        const wt_grid& g = grids[t];
        if (g.precision != prec || g.collision != coll)
            return wt_set_error(WT_ERR_ARG, "wt_batch_create: tunnel %d differs in precision or collision form", t);
        if (!g.f[0] || !g.f[1] || !g.mac[0] || !g.mac[1] || !g.solid || !g.code)
            return wt_set_error(WT_ERR_ARG, "wt_batch_create: tunnel %d has a null buffer", t);
        if (int rc = wt_check_dims(g.nx, g.ny, g.nz)) return rc;
        if (cur[t] != 0 && cur[t] != 1) return wt_set_error(WT_ERR_ARG, "wt_batch_create: cur of tunnel %d", t);
    }
    int v, block;
    const int id = tile_shape(tile, prec, &v, &block);
    if (!id) return wt_set_error(WT_ERR_ARG, "wt_batch: tile %d has no batched form", tile);
    const BatchVariant* var = nullptr;
    switch (prec) {
        case WT_F32: var = batch_variant<WT_F32>(coll == WT_COLLIDE_FAST, id); break;
        case WT_F16: var = batch_variant<WT_F16>(coll == WT_COLLIDE_FAST, id); break;
        case WT_BF16: var = batch_variant<WT_BF16>(coll == WT_COLLIDE_FAST, id); break;
        case WT_F64: var = batch_variant<WT_F64>(coll == WT_COLLIDE_FAST, id); break;
        default: return wt_set_error(WT_ERR_ARG, "wt_batch_create: unknown precision %d", prec);
    }
    if (!var) return wt_set_error(WT_ERR_ARG, "wt_batch_create: no batched kernel for tile %d", id);
    for (int32_t t = 0; t < count; ++t)
        if (grids[t].nx % v) return wt_set_error(WT_ERR_DIMS, "wt_batch_create: nx of tunnel %d not a multiple of %d", t, v);
    const int64_t need = wt_batch_workspace_bytes(grids, count, id);
    if (need < 0) return (int)need;
    if (workspace_bytes < need)
        return wt_set_error(WT_ERR_CAPACITY, "wt_batch_create: workspace %lld < %lld bytes", (long long)workspace_bytes,
                            (long long)need);
    if (reinterpret_cast<uintptr_t>(workspace) % 256)
        return wt_set_error(WT_ERR_ARG, "wt_batch_create: workspace not 256-byte aligned");

    const size_t ds = desc_bytes_for(prec);
    if (var->form == BATCH_PARAMS) {
        wt_batch* b = new wt_batch();
        b->precision = prec;
        b->collision = coll;
        b->count = count;
        b->base = 0;
        b->cur0.assign(cur, cur + count);
        b->var = var;
        b->desc = nullptr;
        b->bulk = b->faces = nullptr;
        b->n_bulk = b->n_faces = 0;
        b->grid_bulk = b->grid_faces = 0;
        b->desc_bytes = ds;
        b->par.assign(count, 0);
        b->pdesc.assign((size_t)4 * count * ds, 0);
        for (int32_t t = 0; t < count; ++t)
            for (int p = 0; p < 2; ++p)
                for (int m = 0; m < 2; ++m) {
                    void* dst = b->pdesc.data() + ((size_t)(p * 2 + m) * count + t) * ds;
                    switch (prec) {
                        case WT_F32: fill_desc<WT_F32>(grids[t], cur[t], uin[t], tau[t], smag[t], p, m, dst); break;
                        case WT_F16: fill_desc<WT_F16>(grids[t], cur[t], uin[t], tau[t], smag[t], p, m, dst); break;
                        case WT_BF16: fill_desc<WT_BF16>(grids[t], cur[t], uin[t], tau[t], smag[t], p, m, dst); break;
                        case WT_F64: fill_desc<WT_F64>(grids[t], cur[t], uin[t], tau[t], smag[t], p, m, dst); break;
                    }
                }
        b->graph = nullptr;
        b->graph_steps = 0;
        *out = b;
        return WT_OK;
    }
    int64_t nb, nf;
    work_counts(grids, count, v * block * ITEM_SUB, &nb, &nf);
    std::vector<unsigned char> host(need, 0);
    unsigned char* hd = host.data();
    int2* hb = reinterpret_cast<int2*>(hd + align256(4 * ds * count));
    int2* hf = reinterpret_cast<int2*>(hd + align256(4 * ds * count) + align256(8 * nb));
    int64_t kb = 0, kf = 0;
    for (int32_t t = 0; t < count; ++t) {
        const wt_grid& g = grids[t];
        for (int p = 0; p < 2; ++p)
            for (int m = 0; m < 2; ++m) {
                void* dst = hd + (size_t)(t * 4 + p * 2 + m) * ds;
                switch (prec) {
                    case WT_F32: fill_desc<WT_F32>(g, cur[t], uin[t], tau[t], smag[t], p, m, dst); break;
                    case WT_F16: fill_desc<WT_F16>(g, cur[t], uin[t], tau[t], smag[t], p, m, dst); break;
                    case WT_BF16: fill_desc<WT_BF16>(g, cur[t], uin[t], tau[t], smag[t], p, m, dst); break;
                    case WT_F64: fill_desc<WT_F64>(g, cur[t], uin[t], tau[t], smag[t], p, m, dst); break;
                }
            }
        const int64_t n = (int64_t)g.nx * g.ny * g.nz;
        for (int64_t c0 = 0; c0 < n; c0 += (int64_t)v * block * ITEM_SUB) hb[kb++] = make_int2(t, (int32_t)c0);
        const int64_t nface = (int64_t)g.nx * g.ny + (int64_t)g.nx * (g.nz - 2);
        for (int64_t f0 = 0; f0 < nface; f0 += FACE_BLOCK * ITEM_SUB) hf[kf++] = make_int2(t, (int32_t)f0);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemcpyAsync(workspace, host.data(), (size_t)need, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return wt_cuda_check("wt_batch_create upload");
    wt_batch* b = new wt_batch();
    b->precision = prec;
    b->collision = coll;
    b->count = count;
    b->base = 0;
    b->cur0.assign(cur, cur + count);
    b->var = var;
    b->desc = workspace;
    b->bulk = reinterpret_cast<int2*>(static_cast<unsigned char*>(workspace) + align256(4 * ds * count));
    b->faces = reinterpret_cast<int2*>(static_cast<unsigned char*>(workspace) + align256(4 * ds * count) + align256(8 * nb));
    b->n_bulk = (int32_t)nb;
    b->n_faces = (int32_t)nf;
    if (var->form == BATCH_PERSISTENT) {  // one wave of blocks looping over the lists
        b->grid_bulk = (int)std::min<int64_t>(nb, (int64_t)num_sms() * var->minb);
        b->grid_faces = (int)std::min<int64_t>(nf, (int64_t)num_sms() * 8);
    } else {  // one block per sub-tile
        b->grid_bulk = (int)(nb * ITEM_SUB);
        b->grid_faces = (int)(nf * ITEM_SUB);
    }
    b->desc_bytes = ds;
    b->graph = nullptr;
    b->graph_steps = 0;
    *out = b;
    return WT_OK;
}

extern "C" int wt_batch_step(wt_batch* b, int32_t steps, int32_t flags, void* stream) {
    if (!b) return wt_set_error(WT_ERR_ARG, "wt_batch_step: null batch");
    if (steps < 0) return wt_set_error(WT_ERR_ARG, "wt_batch_step: steps < 0");
    return launch_steps(b, steps, flags, static_cast<cudaStream_t>(stream));
}

extern "C" int wt_batch_step_each(wt_batch* b, const int32_t* steps, int32_t flags, void* stream) {
    if (!b || !steps) return wt_set_error(WT_ERR_ARG, "wt_batch_step_each: null argument");
    bool uniform = true;
    for (int32_t t = 0; t < b->count; ++t) {
        if (steps[t] < 0) return wt_set_error(WT_ERR_ARG, "wt_batch_step_each: steps of tunnel %d < 0", t);
        uniform = uniform && steps[t] == steps[0];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (b->var->form == BATCH_PARAMS) return launch_params(b, steps, 0, flags, st);
    if (!uniform)
        return wt_set_error(WT_ERR_ARG, "wt_batch_step_each: tile %d steps every tunnel alike (use a 200 + k tile)",
                            b->var->id);
    return launch_steps(b, steps[0], flags, st);
}

extern "C" int wt_batch_capture(wt_batch* b, int32_t steps, int32_t flags, void* stream) {
    if (!b) return wt_set_error(WT_ERR_ARG, "wt_batch_capture: null batch");
    if (steps <= 0 || (steps & 1))
        return wt_set_error(WT_ERR_ARG, "wt_batch_capture: steps must be even and positive (got %d)", steps);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!st) return wt_set_error(WT_ERR_ARG, "wt_batch_capture: needs a non-default stream");
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return wt_cuda_check("wt_batch_capture begin");
    const int rc = launch_steps(b, steps, flags, st);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return wt_set_error(WT_ERR_CUDA, "wt_batch_capture end: %s", cudaGetErrorString(e));
    const cudaError_t e2 = cudaGraphInstantiate(&b->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
        b->graph = nullptr;
        return wt_set_error(WT_ERR_CUDA, "wt_batch_capture instantiate: %s", cudaGetErrorString(e2));
    }
    b->graph_steps = steps;
    return WT_OK;
}

extern "C" int wt_batch_replay(wt_batch* b, void* stream) {
    if (!b || !b->graph) return wt_set_error(WT_ERR_ARG, "wt_batch_replay: no captured graph");
    if (cudaGraphLaunch(b->graph, static_cast<cudaStream_t>(stream)) != cudaSuccess)
        return wt_cuda_check("wt_batch_replay");
    return WT_OK;  // an even number of steps leaves every tunnel's current buffer unchanged
}

extern "C" int wt_batch_cur(const wt_batch* b, int32_t* cur_out) {
    if (!b || !cur_out) return wt_set_error(WT_ERR_ARG, "wt_batch_cur: null argument");
    for (int32_t t = 0; t < b->count; ++t)
        cur_out[t] = b->cur0[t] ^ (b->var->form == BATCH_PARAMS ? b->par[t] : b->base);
    return WT_OK;
}

extern "C" int wt_batch_destroy(wt_batch* b) {
    if (!b) return WT_OK;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    delete b;
    return WT_OK;
}
