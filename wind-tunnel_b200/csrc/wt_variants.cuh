// Kernel-variant tables of the step and batch kernels. The kernels are instantiated once per
// storage precision, each precision in its own translation unit (wt_kernels_<prec>.cu), so the
// build compiles them in parallel; wt_step.cu and wt_batch.cu hold the host code and reach the
// kernels only through the functions declared here.
#pragma once

#include "wt_common.cuh"

namespace wt {

// One tile shape of the single-tunnel step kernel. kind 0: direct loads over a 1-D grid of
// cells (v cells per thread, block threads, minb resident blocks per SM, which bounds
// registers); kind 1: streaming through shared memory (chunk cells per stage, stages
// pipeline stages); kind 2: direct loads over a grid of lattice rows (one block row per
// x-run of a lattice row, v = 2 cells per thread); kind 4: kind 2 with the later face cells
// fused in (no separate face kernel).
struct StepVariant {
    int id, kind, v, block, minb, chunk, stages;
    int (*launch)(const void* args, int32_t n, cudaStream_t st);
};

// One tile shape of the batched bulk kernel and its face kernel, in one of three forms:
// BATCH_PERSISTENT -- a grid of one wave whose blocks loop over the device work list;
// BATCH_GRID -- one block per sub-tile of the device work list;
// BATCH_PARAMS -- no device work list: the tunnels' descriptors and block counts travel in the
// kernel's parameter space (up to 32 KB), each block finds its tunnel there, and a batch larger
// than one parameter block is launched in groups (bulk_p / faces_p take the host copies of the
// count descriptors of this step's parity).
enum BatchForm { BATCH_PERSISTENT = 0, BATCH_GRID = 1, BATCH_PARAMS = 2 };
struct BatchVariant {
    int id, v, block, minb;
    int form;
    void (*bulk)(const void* args, int grid, cudaStream_t st);
    void (*faces)(const void* args, int grid, cudaStream_t st);
    int (*bulk_p)(const void* descs, int32_t count, cudaStream_t st);
    int (*faces_p)(const void* descs, int32_t count, cudaStream_t st);
};

// A batch work item is ITEM_SUB sub-tiles: BLOCK * V * ITEM_SUB cells of one tunnel (bulk) or
// FACE_BLOCK * ITEM_SUB face cells (faces).
constexpr int ITEM_SUB = 16;
constexpr int FACE_BLOCK = 256;

struct BatchArgs {
    const void* desc;  // StepArgs<S, T>[count][2][2] of the batch's precision
    const int2* bulk;
    const int2* faces;
    int32_t n_bulk, n_faces;
    int32_t parity, mac_all;
};

// the step variants of precision PREC for one collision form (fast = WT_COLLIDE_FAST)
template <int PREC>
const StepVariant* step_variants(bool fast, int* count);
// `steps` steps of one tunnel (wt_step after argument checks; skip_chunk is the failure-path
// test hook of wt_step_test_skip_chunk, 0 = off)
template <int PREC>
int step_prec(const wt_grid* g, int32_t cur, int32_t steps, double uin, double tau, double smag, int32_t flags,
              int32_t skip_chunk, cudaStream_t stream);
// the batched kernels of tile id `id`, or null
template <int PREC>
const BatchVariant* batch_variant(bool fast, int id);

}  // namespace wt
