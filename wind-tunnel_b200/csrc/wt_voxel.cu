// Server-side voxeliser: the browser's voxelize.js (web/js/voxelize.js:5-115) on the GPU, so
// a triangle soup in lattice coordinates becomes a solid mask without a browser round trip.
// Same stages and the same double-precision arithmetic in the same order (the library is
// built without FMA contraction):
//   1. ray parity along +x for every (y, z) column, rays jittered off edges and vertices by
//      (OY, OZ); crossings are counted per column, the columns' offsets scanned, the crossings
//      stored, then each column sorted and filled between consecutive pairs of crossings;
//   2. a rasterised surface shell (every triangle sampled at s <= 256 steps per edge, points
//      rounded as Math.round does), so thin or leaky geometry still blocks flow;
//   3. a flood fill of fluid from the domain boundary: line sweeps along x, y and z, repeated
//      until nothing changes; every fluid cell 6-connected to a boundary fluid cell is reached,
//      as by the reference's depth-first fill, and unreached cells become solid;
//   4. the frontal and planform areas of the solid, then the ground layer y = 0 tagged 2.
// The atomic appends of stage 1 land in any order; sorting each column makes the result exact.
#include <algorithm>

#include "wt_common.cuh"

namespace wt {

constexpr double VOX_OY = 0.01373, VOX_OZ = 0.00717;  // voxelize.js:9

struct VoxGeo {
    int32_t nx, ny, nz;
    int64_t n;
};

// A triangle with a non-finite coordinate adds nothing (the reference's loops then run zero
// times for NaN); skipping it keeps every index computed below inside the lattice.
__device__ __forceinline__ bool tri_finite(const float* p) {
    bool ok = true;
#pragma unroll
    for (int q = 0; q < 9; ++q) ok = ok && isfinite(p[q]);
    return ok;
}

// Stage 1: crossings of triangle t with the jittered rays of its y-z footprint (voxelize.js:12-37).
// COUNT: count per column; else append at offsets[c] + cursor[c].
template <bool COUNT>
__global__ void __launch_bounds__(256) k_vox_cross(const float* __restrict__ tris, int64_t num_tris, VoxGeo g,
                                                   int32_t* __restrict__ counts, const int64_t* __restrict__ offsets,
                                                   int32_t* __restrict__ cursor, double* __restrict__ xs) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < num_tris; t += (int64_t)gridDim.x * blockDim.x) {
        const float* p = tris + 9 * t;
        if (!tri_finite(p)) continue;
        const double ax = p[0], ay = p[1], az = p[2], bx = p[3], by = p[4], bz = p[5], cx_ = p[6], cy_ = p[7], cz_ = p[8];
        const double y0 = fmax(1.0, ceil(fmin(fmin(ay, by), cy_) - VOX_OY));
        const double y1 = fmin((double)(g.ny - 2), floor(fmax(fmax(ay, by), cy_) - VOX_OY));
        const double z0 = fmax(1.0, ceil(fmin(fmin(az, bz), cz_) - VOX_OZ));
        const double z1 = fmin((double)(g.nz - 2), floor(fmax(fmax(az, bz), cz_) - VOX_OZ));
        if (y0 > y1 || z0 > z1) continue;
        const double e1y = by - ay, e1z = bz - az, e2y = cy_ - ay, e2z = cz_ - az;
        const double det = e1y * e2z - e2y * e1z;
        if (det == 0.0) continue;
        const double id = 1.0 / det;
        for (int32_t k = (int32_t)z0; k <= (int32_t)z1; ++k) {
            const double pz = ((double)k + VOX_OZ) - az;
            for (int32_t j = (int32_t)y0; j <= (int32_t)y1; ++j) {
                const double py = ((double)j + VOX_OY) - ay;
                const double w1 = (py * e2z - e2y * pz) * id;
                if (w1 < 0.0) continue;
                const double w2 = (e1y * pz - py * e1z) * id;
                if (w2 < 0.0 || w1 + w2 > 1.0) continue;
                const int64_t c = j + (int64_t)g.ny * k;
                if constexpr (COUNT) {
                    atomicAdd(&counts[c], 1);
                } else {
                    const double x = (ax + w1 * (bx - ax)) + w2 * (cx_ - ax);
                    const int64_t q = offsets[c] + atomicAdd(&cursor[c], 1);
                    if (q < offsets[c + 1]) xs[q] = x;  // the count pass found the same crossings
                }
            }
        }
    }
}

// Exclusive scan of the column counts into offsets[0..m] (one block; m = ny * nz columns).
constexpr int VOX_SCAN = 1024;
__global__ void __launch_bounds__(VOX_SCAN) k_vox_scan(const int32_t* __restrict__ counts, int64_t m,
                                                       int64_t* __restrict__ offsets) {
    __shared__ int64_t part[VOX_SCAN];
    const int64_t per = (m + VOX_SCAN - 1) / VOX_SCAN;
    const int64_t lo = threadIdx.x * per, hi = min(m, lo + per);
    int64_t s = 0;
    for (int64_t c = lo; c < hi; ++c) s += counts[c];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {  // VOX_SCAN partial sums, serially: a set-up step
        int64_t acc = 0;
        for (int i = 0; i < VOX_SCAN; ++i) {
            const int64_t v = part[i];
            part[i] = acc;
            acc += v;
        }
        offsets[m] = acc;
    }
    __syncthreads();
    int64_t acc = part[threadIdx.x];
    for (int64_t c = lo; c < hi; ++c) {
        offsets[c] = acc;
        acc += counts[c];
    }
}

// Sort each column's crossings and fill between consecutive pairs (voxelize.js:39-49).
__global__ void __launch_bounds__(256) k_vox_spans(double* __restrict__ xs, const int64_t* __restrict__ offsets,
                                                   VoxGeo g, uint8_t* __restrict__ vox) {
    const int64_t m = (int64_t)g.ny * g.nz;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < m; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b0 = offsets[c], len = offsets[c + 1] - b0;
        if (len < 2) continue;
        double* l = xs + b0;
        for (int64_t i = 1; i < len; ++i) {  // insertion sort: columns hold a handful of crossings
            const double v = l[i];
            int64_t j = i - 1;
            while (j >= 0 && l[j] > v) {
                l[j + 1] = l[j];
                --j;
            }
            l[j + 1] = v;
        }
        const int64_t j = c % g.ny, k = c / g.ny;
        uint8_t* row = vox + g.nx * (j + (int64_t)g.ny * k);
        for (int64_t i = 0; i + 1 < len; i += 2) {
            const double a = fmax(1.0, ceil(l[i]));
            const double b = fmin((double)(g.nx - 2), floor(l[i + 1]));
            if (!(a <= b)) continue;  // then 1 <= a <= b <= nx-2: both fit the row
            for (int32_t x = (int32_t)a; x <= (int32_t)b; ++x) row[x] = 1;
        }
    }
}

// Math.round: the nearest integer, halves towards +infinity (x - floor(x) is exact in double)
__device__ __forceinline__ double js_round(double x) {
    const double f = floor(x);
    return x - f >= 0.5 ? f + 1.0 : f;
}

// Stage 2: surface shell (voxelize.js:51-71); one block per triangle, a thread per row a.
__global__ void __launch_bounds__(256) k_vox_shell(const float* __restrict__ tris, int64_t num_tris, VoxGeo g,
                                                   uint8_t* __restrict__ vox) {
    for (int64_t t = blockIdx.x; t < num_tris; t += gridDim.x) {
        const float* p = tris + 9 * t;
        if (!tri_finite(p)) continue;
        const double ax = p[0], ay = p[1], az = p[2];
        const double ux = (double)p[3] - ax, uy = (double)p[4] - ay, uz = (double)p[5] - az;
        const double vx = (double)p[6] - ax, vy = (double)p[7] - ay, vz = (double)p[8] - az;
        const double dx = ux - vx, dy = uy - vy, dz = uz - vz;
        const double L = sqrt(fmax(fmax(ux * ux + uy * uy + uz * uz, vx * vx + vy * vy + vz * vz),
                                   dx * dx + dy * dy + dz * dz));
        const int32_t s = (int32_t)fmax(1.0, fmin(256.0, ceil(L / 0.5)));
        for (int32_t a = threadIdx.x; a <= s; a += blockDim.x) {
            const double fa = (double)a / (double)s;
            for (int32_t b = 0; a + b <= s; ++b) {
                const double fb = (double)b / (double)s;
                const double x = js_round((ax + ux * fa) + vx * fb);
                const double y = js_round((ay + uy * fa) + vy * fb);
                const double z = js_round((az + uz * fa) + vz * fb);
                if (!(x >= 1.0 && y >= 1.0 && z >= 1.0 && x <= g.nx - 2 && y <= g.ny - 2 && z <= g.nz - 2)) continue;
                vox[(int64_t)x + g.nx * ((int64_t)y + (int64_t)g.ny * (int64_t)z)] = 1;
            }
        }
    }
}

// Stage 3: flood fill. seen starts as the boundary cells that are not vox.
__global__ void __launch_bounds__(256) k_vox_seed(const uint8_t* __restrict__ vox, VoxGeo g, uint8_t* __restrict__ seen) {
    const int64_t nxy = (int64_t)g.nx * g.ny;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t z = i / nxy, r = i - z * nxy, y = r / g.nx, x = r - y * g.nx;
        const bool edge = x == 0 || y == 0 || z == 0 || x == g.nx - 1 || y == g.ny - 1 || z == g.nz - 1;
        seen[i] = edge && !vox[i];
    }
}

// One line of `len` cells at stride `st` from `base`: fluid carries `seen` both ways until a
// vox cell stops it. Sets *changed when a cell is newly reached.
__device__ __forceinline__ void flood_line(const uint8_t* __restrict__ vox, uint8_t* __restrict__ seen, int64_t base,
                                           int64_t st, int32_t len, int32_t* changed) {
    bool carry = false, any = false;
    for (int32_t q = 0; q < len; ++q) {
        const int64_t i = base + q * st;
        if (vox[i]) { carry = false; continue; }
        if (seen[i]) carry = true;
        else if (carry) { seen[i] = 1; any = true; }
    }
    carry = false;
    for (int32_t q = len - 1; q >= 0; --q) {
        const int64_t i = base + q * st;
        if (vox[i]) { carry = false; continue; }
        if (seen[i]) carry = true;
        else if (carry) { seen[i] = 1; any = true; }
    }
    if (any) atomicExch(changed, 1);
}

// AXIS 0: lines along x (thread per (y, z)); 1: along y (thread per (x, z)); 2: along z (per (x, y)).
template <int AXIS>
__global__ void __launch_bounds__(256) k_vox_sweep(const uint8_t* __restrict__ vox, VoxGeo g, uint8_t* __restrict__ seen,
                                                   int32_t* changed) {
    const int64_t nxy = (int64_t)g.nx * g.ny;
    const int64_t lines = AXIS == 0 ? (int64_t)g.ny * g.nz : (AXIS == 1 ? (int64_t)g.nx * g.nz : nxy);
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < lines; l += (int64_t)gridDim.x * blockDim.x) {
        if constexpr (AXIS == 0) {
            flood_line(vox, seen, l * g.nx, 1, g.nx, changed);
        } else if constexpr (AXIS == 1) {
            const int64_t z = l / g.nx, x = l - z * g.nx;
            flood_line(vox, seen, x + z * nxy, g.nx, g.ny, changed);
        } else {
            flood_line(vox, seen, l, nxy, g.nz, changed);
        }
    }
}

// Stage 4: solid = not reached (written over vox), counts, areas (voxelize.js:94-113).
__global__ void __launch_bounds__(256) k_vox_solid(const uint8_t* __restrict__ seen, VoxGeo g, uint8_t* __restrict__ solid,
                                                   unsigned long long* __restrict__ stats) {
    unsigned long long cnt = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t s = seen[i] ? 0 : 1;
        solid[i] = s;
        cnt += s;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&stats[2], cnt);
}

__global__ void __launch_bounds__(256) k_vox_areas(const uint8_t* __restrict__ solid, VoxGeo g,
                                                   unsigned long long* __restrict__ stats) {
    const int64_t rows = (int64_t)g.ny * g.nz, cols = (int64_t)g.nx * g.nz;
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < rows + cols; l += (int64_t)gridDim.x * blockDim.x) {
        if (l < rows) {  // frontal: (y, z) rows holding any solid cell
            const uint8_t* r = solid + l * g.nx;
            for (int32_t x = 0; x < g.nx; ++x)
                if (r[x]) { atomicAdd(&stats[0], 1ull); break; }
        } else {  // planform: (x, z) columns holding any solid cell
            const int64_t q = l - rows, z = q / g.nx, x = q - z * g.nx;
            const uint8_t* c = solid + x + z * (int64_t)g.nx * g.ny;
            for (int32_t y = 0; y < g.ny; ++y)
                if (c[(int64_t)y * g.nx]) { atomicAdd(&stats[1], 1ull); break; }
        }
    }
}

__global__ void __launch_bounds__(256) k_vox_ground(VoxGeo g, uint8_t* __restrict__ solid) {
    const int64_t m = (int64_t)g.nx * g.nz;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < m; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t z = q / g.nx, x = q - z * g.nx;
        solid[x + z * (int64_t)g.nx * g.ny] = 2;
    }
}

// workspace carve-up
struct VoxWork {
    int32_t* counts;
    int32_t* cursor;
    int64_t* offsets;
    uint8_t* seen;
    int32_t* changed;
    unsigned long long* stats;
    double* xs;
    int64_t max_xs;
};

inline size_t vox_align(size_t b) { return (b + 255) / 256 * 256; }

inline int64_t vox_fixed_bytes(int64_t m, int64_t n) {
    return (int64_t)(vox_align(4 * m) * 2 + vox_align(8 * (m + 1)) + vox_align(n) + vox_align(4) + vox_align(8 * 3));
}

inline VoxWork vox_carve(void* ws, int64_t bytes, int64_t m, int64_t n) {
    VoxWork w;
    char* p = static_cast<char*>(ws);
    w.counts = reinterpret_cast<int32_t*>(p); p += vox_align(4 * m);
    w.cursor = reinterpret_cast<int32_t*>(p); p += vox_align(4 * m);
    w.offsets = reinterpret_cast<int64_t*>(p); p += vox_align(8 * (m + 1));
    w.seen = reinterpret_cast<uint8_t*>(p); p += vox_align(n);
    w.changed = reinterpret_cast<int32_t*>(p); p += vox_align(4);
    w.stats = reinterpret_cast<unsigned long long*>(p); p += vox_align(8 * 3);
    w.xs = reinterpret_cast<double*>(p);
    w.max_xs = (bytes - vox_fixed_bytes(m, n)) / 8;
    return w;
}

}  // namespace wt

using namespace wt;

extern "C" int64_t wt_voxelize_workspace_bytes(int32_t nx, int32_t ny, int32_t nz, int64_t max_crossings) {
    if (int rc = wt_check_dims(nx, ny, nz)) return rc;
    if (max_crossings < 0) return wt_set_error(WT_ERR_ARG, "wt_voxelize_workspace_bytes: max_crossings < 0");
    const int64_t m = (int64_t)ny * nz, n = (int64_t)nx * ny * nz;
    return vox_fixed_bytes(m, n) + 8 * max_crossings;
}

extern "C" int wt_voxelize(const float* tris, int64_t num_tris, int32_t nx, int32_t ny, int32_t nz, int32_t ground,
                           uint8_t* solid, void* workspace, int64_t workspace_bytes, int64_t* out4, void* stream) {
    if (int rc = wt_check_dims(nx, ny, nz)) return rc;
    if (!solid || !workspace || !out4 || num_tris < 0 || (num_tris > 0 && !tris))
        return wt_set_error(WT_ERR_ARG, "wt_voxelize: null buffer or negative triangle count");
    if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
        return wt_set_error(WT_ERR_ARG, "wt_voxelize: workspace not 256-byte aligned");
    const VoxGeo g{nx, ny, nz, (int64_t)nx * ny * nz};
    const int64_t m = (int64_t)ny * nz;
    if (workspace_bytes < vox_fixed_bytes(m, g.n))
        return wt_set_error(WT_ERR_CAPACITY, "wt_voxelize: workspace below wt_voxelize_workspace_bytes(..., 0)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const VoxWork w = vox_carve(workspace, workspace_bytes, m, g.n);
    const int sms = 148;
    const unsigned gt = (unsigned)std::max<int64_t>(1, std::min<int64_t>((num_tris + 255) / 256, 64 * sms));
    const unsigned gn = (unsigned)std::max<int64_t>(1, std::min<int64_t>((g.n + 255) / 256, 64 * sms));
    // stage 1: count, scan, check capacity, fill, sort and fill spans
    cudaMemsetAsync(w.counts, 0, 4 * m, st);
    cudaMemsetAsync(w.cursor, 0, 4 * m, st);
    cudaMemsetAsync(solid, 0, g.n, st);
    cudaMemsetAsync(w.stats, 0, 24, st);
    if (num_tris > 0) k_vox_cross<true><<<gt, 256, 0, st>>>(tris, num_tris, g, w.counts, nullptr, nullptr, nullptr);
    k_vox_scan<<<1, VOX_SCAN, 0, st>>>(w.counts, m, w.offsets);
    int64_t total = 0;
    if (cudaMemcpyAsync(&total, w.offsets + m, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return wt_cuda_check("wt_voxelize: crossing count");
    out4[3] = total;
    if (total > w.max_xs)
        return wt_set_error(WT_ERR_CAPACITY, "wt_voxelize: %lld ray crossings, workspace holds %lld",
                            (long long)total, (long long)w.max_xs);
    if (num_tris > 0) {
        k_vox_cross<false><<<gt, 256, 0, st>>>(tris, num_tris, g, nullptr, w.offsets, w.cursor, w.xs);
        k_vox_spans<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((m + 255) / 256, 16 * sms)), 256, 0, st>>>(
            w.xs, w.offsets, g, solid);
        // stage 2
        k_vox_shell<<<(unsigned)std::min<int64_t>(num_tris, 64 * sms), 256, 0, st>>>(tris, num_tris, g, solid);
    }
    // stage 3: sweeps until a full round reaches nothing new (each round at least one line
    // further, so the loop ends; the bound below is the lattice's cell count)
    k_vox_seed<<<gn, 256, 0, st>>>(solid, g, w.seen);
    const unsigned gl = (unsigned)std::max<int64_t>(1, std::min<int64_t>(((int64_t)nx * std::max(ny, nz) + 255) / 256, 16 * sms));
    for (int64_t round = 0; round < g.n; ++round) {
        int32_t changed = 0;
        cudaMemsetAsync(w.changed, 0, 4, st);
        k_vox_sweep<0><<<gl, 256, 0, st>>>(solid, g, w.seen, w.changed);
        k_vox_sweep<1><<<gl, 256, 0, st>>>(solid, g, w.seen, w.changed);
        k_vox_sweep<2><<<gl, 256, 0, st>>>(solid, g, w.seen, w.changed);
        if (cudaMemcpyAsync(&changed, w.changed, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return wt_cuda_check("wt_voxelize: flood fill");
        if (!changed) break;
    }
    // stage 4
    k_vox_solid<<<gn, 256, 0, st>>>(w.seen, g, solid, w.stats);
    k_vox_areas<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((m + (int64_t)nx * nz + 255) / 256, 16 * sms)), 256, 0,
                  st>>>(solid, g, w.stats);
    if (ground) k_vox_ground<<<(unsigned)std::max<int64_t>(1, ((int64_t)nx * nz + 255) / 256), 256, 0, st>>>(g, solid);
    unsigned long long stats[3] = {0, 0, 0};
    if (cudaMemcpyAsync(stats, w.stats, 24, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return wt_cuda_check("wt_voxelize: statistics");
    out4[0] = (int64_t)stats[0];
    out4[1] = (int64_t)stats[1];
    out4[2] = (int64_t)stats[2];
    return wt_cuda_check("wt_voxelize launch");
}
