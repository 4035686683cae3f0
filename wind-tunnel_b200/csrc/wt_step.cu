// Single-tunnel step entry points (wt_step, wt_step_tiles). The kernels and their tile-variant
// tables are instantiated per storage precision in wt_kernels_<prec>.cu (see wt_kernels.cuh).
#include "wt_variants.cuh"

static int step_any(const wt_grid* g, int32_t cur, int32_t steps, double uin, double tau, double smag,
                    int32_t flags, int32_t skip_chunk, void* stream) {
    if (!g || !g->f[0] || !g->f[1] || !g->mac[0] || !g->mac[1] || !g->solid || !g->code)
        return wt_set_error(WT_ERR_ARG, "wt_step: null buffer in grid");
    if (int rc = wt_check_dims(g->nx, g->ny, g->nz)) return rc;
    if (cur != 0 && cur != 1) return wt_set_error(WT_ERR_ARG, "wt_step: cur must be 0 or 1");
    if (steps < 0) return wt_set_error(WT_ERR_ARG, "wt_step: steps < 0");
    if (steps == 0) return WT_OK;
    if (g->collision != WT_COLLIDE_EXACT && g->collision != WT_COLLIDE_FAST)
        return wt_set_error(WT_ERR_ARG, "wt_step: unknown collision form %d", g->collision);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (g->precision) {
        case WT_F32: return wt::step_prec<WT_F32>(g, cur, steps, uin, tau, smag, flags, skip_chunk, st);
        case WT_F16: return wt::step_prec<WT_F16>(g, cur, steps, uin, tau, smag, flags, skip_chunk, st);
        case WT_BF16: return wt::step_prec<WT_BF16>(g, cur, steps, uin, tau, smag, flags, skip_chunk, st);
        case WT_F64: return wt::step_prec<WT_F64>(g, cur, steps, uin, tau, smag, flags, skip_chunk, st);
        default: return wt_set_error(WT_ERR_ARG, "wt_step: unknown precision %d", g->precision);
    }
}

extern "C" int wt_step(const wt_grid* g, int32_t cur, int32_t steps, double uin, double tau, double smag,
                       int32_t flags, void* stream) {
    return step_any(g, cur, steps, uin, tau, smag, flags, 0, stream);
}

extern "C" int wt_step_test_skip_chunk(const wt_grid* g, int32_t cur, int32_t steps, double uin, double tau,
                                       double smag, int32_t flags, int32_t skip_chunk, void* stream) {
    if (skip_chunk < 0) return wt_set_error(WT_ERR_ARG, "wt_step_test_skip_chunk: skip_chunk < 0");
    return step_any(g, cur, steps, uin, tau, smag, flags, skip_chunk, stream);
}

extern "C" int wt_step_tiles(int32_t precision, int32_t collision, int32_t* out, int32_t cap) {
    if (collision != WT_COLLIDE_EXACT && collision != WT_COLLIDE_FAST)
        return wt_set_error(WT_ERR_ARG, "wt_step_tiles: unknown collision form %d", collision);
    const bool fast = collision == WT_COLLIDE_FAST;
    int count = 0;
    const wt::StepVariant* t = nullptr;
    switch (precision) {
        case WT_F32: t = wt::step_variants<WT_F32>(fast, &count); break;
        case WT_F16: t = wt::step_variants<WT_F16>(fast, &count); break;
        case WT_BF16: t = wt::step_variants<WT_BF16>(fast, &count); break;
        case WT_F64: t = wt::step_variants<WT_F64>(fast, &count); break;
        default: return wt_set_error(WT_ERR_ARG, "wt_step_tiles: unknown precision %d", precision);
    }
    for (int k = 0; k < count && k < cap; ++k) {
        if (!out) break;
        out[4 * k + 0] = t[k].id;
        out[4 * k + 1] = t[k].kind == 1 ? -t[k].chunk : t[k].v;  // negative: streaming chunk length
        out[4 * k + 2] = t[k].block;
        out[4 * k + 3] = t[k].kind == 1 ? t[k].stages : t[k].minb;
    }
    return count;
}
