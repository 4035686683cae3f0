/* wt.h -- C ABI of libwt.so, the B200 (sm_100a) kernels of the wind-tunnel LBM hot path.
 *
 * Drop-in boundary: these entry points replace the NVIDIA Warp launches that the
 * reference Solver (RICKxxROLLING/wind-tunnel, server/lbm.py:398-482) makes. A host
 * binding (ctypes here; cgo/JNI would bind the same symbols) owns the device buffers
 * and calls these with raw device pointers, sizes and a cudaStream_t passed as void*.
 *
 * Conventions
 *   - Every function returns 0 (WT_OK) or a negative WT_ERR_* code; wt_last_error()
 *     gives a message for the calling thread's last failure.
 *   - Layout is the reference's: cell index idx = x + nx*(y + ny*z), x fastest
 *     (server/lbm.py:78-80); populations are SoA, population i of cell idx at f[i*n + idx]
 *     (server/lbm.py:404); mac is 4 reals per cell (ux, uy, uz, rho) (server/lbm.py:406);
 *     solid is one byte per cell: 0 fluid, 1 static solid, 2 moving belt, any other
 *     non-zero value a static solid that force sums ignore (server/lbm.py:81, 115-124, 188).
 *   - Kernels are asynchronous on `stream` (NULL = legacy default stream). Nothing here
 *     allocates device memory in a hot call; scratch is passed in by the caller.
 *   - Scalar parameters are passed as double and rounded once to the kernel's arithmetic
 *     type (float, as Warp rounds the reference's Python floats; double for WT_F64).
 *   - Storage precision: WT_F32 stores populations as float (the reference's form);
 *     WT_F16 / WT_BF16 store f_i - w_i as half / bfloat16 (rounded to nearest even) with
 *     all collision arithmetic in float; WT_F64 stores and computes in double (the
 *     oracle run). mac is float for WT_F32/F16/BF16 and double for WT_F64.
 */
#ifndef WT_H
#define WT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WT_ABI_VERSION 4

enum {
    WT_OK = 0,
    WT_ERR_ARG = -1,      /* bad pointer, size or enum */
    WT_ERR_DIMS = -2,     /* grid shape not supported (see wt_check_dims) */
    WT_ERR_CUDA = -3,     /* a CUDA runtime call failed */
    WT_ERR_CAPACITY = -4, /* a caller buffer is too small */
    WT_ERR_TIMEOUT = -5   /* a bounded device wait gave up */
};

/* population storage. WT_F16 / WT_BF16 store deviations d_i = f_i - e_i in half width,
 * e_i = w_i (1 + 3 c_xi U + 4.5 c_xi^2 U^2 - 1.5 U^2), the equilibrium at rho = 1,
 * u = (U, 0, 0) with U = wt_grid.shift_u (evaluated in double, rounded to float once); near
 * the free stream the deviations are small, where half precision resolves them finely.
 * U = 0 gives e_i = w_i. Arithmetic is float in every case. */
enum { WT_F32 = 0, WT_F16 = 1, WT_BF16 = 2, WT_F64 = 3 };

/* collision forms. EXACT evaluates the reference's expressions in the reference's order
 * (bit-identical to server/lbm.py run serially). FAST evaluates the same regularized
 * Smagorinsky collision in moment space with fused multiply-adds (about 40% fewer
 * operations; equal to EXACT up to rounding); with fp16/bf16 storage it works on the
 * stored deviations f_i - e_i directly. */
enum { WT_COLLIDE_EXACT = 0, WT_COLLIDE_FAST = 1 };

/* wt_step flags */
#define WT_STEP_MAC_ALL_LAST 1 /* write mac for every cell on the last step (needed before frames) */

/* One tunnel's device state. Mirrors the buffers the reference Solver allocates
 * (server/lbm.py:404-407) plus the derived per-cell code byte. */
typedef struct wt_grid {
    int32_t nx, ny, nz;    /* lattice size */
    int32_t precision;     /* WT_F32 / WT_F16 / WT_BF16 / WT_F64 */
    void* f[2];            /* two population buffers, 19*n elements each */
    void* mac[2];          /* two macroscopic buffers, 4*n reals each (double-buffered) */
    const uint8_t* solid;  /* n bytes, reference mask semantics */
    uint8_t* code;         /* n bytes, filled by wt_build_codes from solid */
    int32_t tile;          /* step kernel tile variant (wt_step_tiles); 0 = library default, by
                              precision, collision form and nx */
    int32_t collision;     /* WT_COLLIDE_EXACT (reference operation order) or WT_COLLIDE_FAST */
    int32_t* status;       /* optional device int: set to WT_ERR_TIMEOUT if a bounded wait gives up */
    float shift_u;         /* fp16/bf16 storage shift velocity U (see WT_F16); ignored otherwise.
                              Must equal the shift_u the buffers were initialised with. */
} wt_grid;

/* ---- library ---- */
const char* wt_last_error(void);
int wt_abi_version(void);
/* 0 if (nx, ny, nz) is supported: nx even and >= 4, ny and nz >= 3, n < 2^31. */
int wt_check_dims(int32_t nx, int32_t ny, int32_t nz);
/* Bytes of device memory one population buffer needs at this precision. */
int64_t wt_population_bytes(int32_t precision, int64_t n);

/* ---- set-up ---- */
/* init_kernel (server/lbm.py:64-69), launched by Solver.reset (:415-417): equilibrium at
 * rho = 1, u = (uin, 0, 0) into population buffer f, and mac = (uin, 0, 0, 1). fp16/bf16
 * buffers are written relative to the shift at velocity shift_u (wt_grid.shift_u of the
 * tunnel; uin itself keeps the free stream's deviations near zero). */
int wt_init_eq(int32_t precision, void* f, void* mac, int64_t n, double uin, double shift_u, void* stream);
/* Derive the per-cell code byte from solid (after Solver.set_solid, server/lbm.py:419-421). */
int wt_build_codes(const wt_grid* g, void* stream);
/* Compacted momentum-exchange link list: every interior fluid cell with at least one
 * neighbour x + c_i whose solid byte is 1 (the cells force_kernel visits,
 * server/lbm.py:177-193), in increasing idx order, with an 18-bit mask of those links.
 * Two calls: wt_links_scan fills scratch (>= wt_links_scratch_len(n) int64) and writes
 * the link count to *count_dev (device); wt_links_fill then writes cells/masks
 * (capacity >= count). */
int64_t wt_links_scratch_len(int64_t n);
int wt_links_scan(const wt_grid* g, int64_t* scratch, int64_t* count_dev, void* stream);
int wt_links_fill(const wt_grid* g, const int64_t* scratch, int32_t* cells, uint32_t* masks, int64_t capacity,
                  void* stream);

/* Tile variants of the step kernel for a storage precision and collision form (WT_COLLIDE_*):
 * writes up to `cap` rows of 4 ints into out and returns the count. Direct-load and row-grid
 * tiles: {id, cells_per_thread, threads_per_block, min_blocks_per_sm}; streaming tiles
 * (shared-memory staging through bulk async copies): {id, -chunk_cells, threads_per_block,
 * pipeline_stages}. Select one with wt_grid.tile. */
int wt_step_tiles(int32_t precision, int32_t collision, int32_t* out, int32_t cap);

/* ---- hot path ---- */
/* `steps` launches of step_kernel (server/lbm.py:72-166), issued by Solver.step
 * (:442-447): fused pull-streaming, bounce-back / moving belt, equilibrium faces,
 * regularized collision with Smagorinsky eddy viscosity and the outlet sponge. Reads
 * f[cur], writes f[cur ^ 1], alternating; the final populations are in f[cur ^ (steps & 1)].
 * Face cells see exactly the neighbour values the reference's serial (Warp CPU) order
 * gives. Each step is two kernels (one with the fused-face row tiles). */
int wt_step(const wt_grid* g, int32_t cur, int32_t steps, double uin, double tau, double smag, int32_t flags,
            void* stream);
/* Test entry point for the failure path; no counterpart in the reference. wt_step with chunk
 * skip_chunk - 1 (skip_chunk > 0) of a streaming tile never loaded, so the kernel's bounded
 * wait for it runs out: the kernel sets *wt_grid.status to WT_ERR_TIMEOUT and returns, the
 * context stays usable and the tunnel's populations are invalid until the next reset. Only
 * streaming tiles (a negative second field in wt_step_tiles) wait; other tiles ignore it. */
int wt_step_test_skip_chunk(const wt_grid* g, int32_t cur, int32_t steps, double uin, double tau, double smag,
                            int32_t flags, int32_t skip_chunk, void* stream);

/* Momentum-exchange force (force_kernel, server/lbm.py:169-197, run by Solver.frame
 * :479-481) on f[cur] over the compacted link list. out6 (device, 6 doubles):
 * [Fx, Fy, Fz] over all solid==1 links, then the same without links into the y = 0 plane.
 * Per-cell sums are formed as the reference forms them; cells are accumulated in double
 * in a fixed order (deterministic). partials: scratch of >= wt_reduce_scratch_len(n_links)
 * doubles. */
int64_t wt_reduce_scratch_len(int64_t count);
int wt_forces(const wt_grid* g, int32_t cur, const int32_t* cells, const uint32_t* masks, int64_t n_links,
              double* partials, double* out6, void* stream);
/* wt_forces without caller scratch. No counterpart in the reference: it exists for callers
 * that cannot allocate device memory on the call path (a host framework that owns the
 * device memory pool and passes only inputs and outputs, or a per-frame loop where an
 * allocation would synchronise the device). The block partials live in a 192 KB array
 * compiled into libwt.so, held by every GPU that loads the library until exit. At most
 * WT_NOALLOC_MAX_LINKS link cells per call (WT_ERR_CAPACITY beyond). The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress), and so does the first
 * call after that device's context was re-created (cudaDeviceReset); make such a call
 * before any stream capture. All calls share the array: calls whose kernels overlap on the
 * GPU race and must not be issued. Results equal wt_forces to fp64 rounding (the blocks
 * partition the list differently). */
#define WT_NOALLOC_MAX_LINKS 1048576
int wt_forces_noalloc(const wt_grid* g, int32_t cur, const int32_t* cells, const uint32_t* masks, int64_t n_links,
                      double* out6, void* stream);
/* Total mass sum_{fluid cells} sum_i f_i of f[cur] in double, deterministic. */
int wt_mass(const wt_grid* g, int32_t cur, double* partials, double* out1, void* stream);

/* ---- many tunnels at once ----
 * A batch advances `count` tunnels of uneven sizes together: per step one bulk kernel over all
 * tunnels' cells, then one kernel over all tunnels' face cells. No
 * counterpart in the reference, which runs one tunnel (server/app.py:116); each tunnel's
 * results are bit-identical to stepping it alone with wt_step. All tunnels share precision and
 * collision form. tile selects the shape: a direct-load tile id k of wt_step_tiles (1-5, 7, 18)
 * runs as a persistent kernel (one wave of blocks looping over the work list); 100 + k (102,
 * 103, 104, 118) as one block per work-list tile; 200 + k (203, 204, 218, and 229, which is
 * tile 18 with each pair's pull issued with its code bytes) with the tunnels' descriptors in the
 * kernel parameters, one block per tile of BLOCK * V cells, groups of tunnels that fit the 32 KB
 * parameter space per launch, and no device work list. The caller allocates
 * a 256-byte aligned device workspace of wt_batch_workspace_bytes (descriptor table and work
 * lists; 256 bytes, unused, for the 200 + k forms). Tile 0 is 229 (204 for fp64). cur gives each tunnel's
 * current population buffer at creation; wt_batch_cur reports it later. A batch must be
 * re-created after any of its tunnels is stepped on its own. */
typedef struct wt_batch wt_batch;
int64_t wt_batch_workspace_bytes(const wt_grid* grids, int32_t count, int32_t tile);
int wt_batch_create(const wt_grid* grids, int32_t count, const double* uin, const double* tau, const double* smag,
                    const int32_t* cur, int32_t tile, void* workspace, int64_t workspace_bytes, void* stream,
                    wt_batch** out);
int wt_batch_step(wt_batch* b, int32_t steps, int32_t flags, void* stream);
/* Tunnel t advances steps[t] steps (0 leaves it as it is); WT_STEP_MAC_ALL_LAST applies to
 * each tunnel's own last step. Uneven counts need a parameter-space tile (200 + k); the other
 * forms accept equal counts only. */
int wt_batch_step_each(wt_batch* b, const int32_t* steps, int32_t flags, void* stream);
/* Capture `steps` (even) steps as a CUDA graph on a non-default stream; replay it with
 * wt_batch_replay (each replay advances every tunnel by `steps` steps). */
int wt_batch_capture(wt_batch* b, int32_t steps, int32_t flags, void* stream);
int wt_batch_replay(wt_batch* b, void* stream);
int wt_batch_cur(const wt_batch* b, int32_t* cur_out);
int wt_batch_destroy(wt_batch* b);

/* ---- server-side voxeliser (web/js/voxelize.js:5-115) ---- */
/* voxelize(): a triangle soup in lattice coordinates (tris: num_tris x 9 floats, device) to a
 * mask (solid: n bytes, device): ray parity along +x, surface shell, flood fill of fluid from
 * the boundary, then the y = 0 layer tagged 2 when ground != 0. Arithmetic in double in the
 * reference's order; triangles with a non-finite coordinate are skipped. out4 (host) receives
 * frontal area, planform area, solid cell count (before the ground layer) and the number of
 * ray crossings. The workspace (device, 256-byte aligned) holds up to max_crossings crossings;
 * with fewer, the call returns WT_ERR_CAPACITY with the needed number in out4[3]. The call
 * synchronises `stream` (a set-up step). */
int64_t wt_voxelize_workspace_bytes(int32_t nx, int32_t ny, int32_t nz, int64_t max_crossings);
int wt_voxelize(const float* tris, int64_t num_tris, int32_t nx, int32_t ny, int32_t nz, int32_t ground,
                uint8_t* solid, void* workspace, int64_t workspace_bytes, int64_t* out4, void* stream);

/* ---- frame outputs (Solver.frame, server/lbm.py:458-482) ---- */
/* advect_kernel (server/lbm.py:233-263): RK2 streamline particles through mac.
 * Respawn uses this library's counter-based RNG (not Warp's). mac: float (4*n). */
int wt_advect(float* pos, float* spd, const float* mac, const uint8_t* solid, int32_t nx, int32_t ny, int32_t nz,
              int64_t num_p, float dt, float uin, float max_age, uint32_t seed, float seed_x, float seed_cy,
              float seed_cz, float seed_hy, float seed_hz, void* stream);
/* pack_particles (server/lbm.py:266-275). */
int wt_pack_particles(const float* pos, const float* spd, uint16_t* q16, uint8_t* q8, int32_t nx, int32_t ny,
                      int32_t nz, int64_t num_p, void* stream);
/* slice_kernel + vort (server/lbm.py:278-318); out has 2*w*h bytes, (w, h) per
 * Solver.slice_dims (server/lbm.py:455-456). */
int wt_slice(const float* mac, const uint8_t* solid, uint8_t* out, int32_t nx, int32_t ny, int32_t nz,
             int32_t axis, int32_t index, int32_t field, float uin, float lref, float vmin, float vmax,
             void* stream);
/* cp_kernel + rho_fluid (server/lbm.py:321-368). verts/norms: 3 floats per vertex. */
int wt_cp(const float* mac, const uint8_t* solid, const float* verts, const float* norms, int8_t* out, int32_t nx,
          int32_t ny, int32_t nz, int64_t num_verts, float uin, float cp_range, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WT_H */
