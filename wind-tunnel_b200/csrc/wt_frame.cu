// Frame-output kernels run by Solver.step / Solver.frame (server/lbm.py:448-482):
// streamline particle advection, particle packing, slice extraction, surface pressure.
// Each follows the reference kernel's arithmetic in the same order (the library is built
// without FMA contraction), so results are bit-identical to the reference run serially.
#include "wt_common.cuh"

namespace wt {

__device__ __forceinline__ int32_t cidx(int32_t x, int32_t y, int32_t z, int32_t nx, int32_t ny, int32_t nz) {
    return min(max(x, 0), nx - 1) + nx * (min(max(y, 0), ny - 1) + ny * min(max(z, 0), nz - 1));
}
__device__ __forceinline__ float clampf_(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }
__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
    // Warp's lerp: a * (1 - t) + b * t
    const float s = 1.0f - t;
    return make_float4(a.x * s + b.x * t, a.y * s + b.y * t, a.z * s + b.z * t, a.w * s + b.w * t);
}

// cidx + sample_mac (server/lbm.py:201-230)
__device__ __forceinline__ float4 sample_mac(const float4* __restrict__ mac, float px, float py, float pz, int32_t nx,
                                             int32_t ny, int32_t nz) {
    const float qx = clampf_(px, 0.0f, (float)nx - 1.001f);
    const float qy = clampf_(py, 0.0f, (float)ny - 1.001f);
    const float qz = clampf_(pz, 0.0f, (float)nz - 1.001f);
    const float bx = floorf(qx), by = floorf(qy), bz = floorf(qz);
    const float tx = qx - bx, ty = qy - by, tz = qz - bz;
    const int32_t ix = (int32_t)bx, iy = (int32_t)by, iz = (int32_t)bz;
    const float4 c000 = mac[cidx(ix, iy, iz, nx, ny, nz)];
    const float4 c100 = mac[cidx(ix + 1, iy, iz, nx, ny, nz)];
    const float4 c010 = mac[cidx(ix, iy + 1, iz, nx, ny, nz)];
    const float4 c110 = mac[cidx(ix + 1, iy + 1, iz, nx, ny, nz)];
    const float4 c001 = mac[cidx(ix, iy, iz + 1, nx, ny, nz)];
    const float4 c101 = mac[cidx(ix + 1, iy, iz + 1, nx, ny, nz)];
    const float4 c011 = mac[cidx(ix, iy + 1, iz + 1, nx, ny, nz)];
    const float4 c111 = mac[cidx(ix + 1, iy + 1, iz + 1, nx, ny, nz)];
    const float4 a = lerp4(lerp4(c000, c100, tx), lerp4(c010, c110, tx), ty);
    const float4 b = lerp4(lerp4(c001, c101, tx), lerp4(c011, c111, tx), ty);
    return lerp4(a, b, tz);
}

// Counter-based RNG for particle respawn: PCG-RXS-M-XS 32-bit output hash
// (Jarzynski & Olano, "Hash Functions for GPU Rendering", JCGT 2020) applied to a
// per-particle counter. Stands in for Warp's wp.rand_init/randf (server/lbm.py:256-259).
__host__ __device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
__device__ __forceinline__ float rng_f(uint32_t& s) {
    s = pcg_hash(s);
    return (float)(s >> 8) * (1.0f / 16777216.0f);
}

struct AdvectArgs {
    float4* pos;
    float* spd;
    const float4* mac;
    const uint8_t* solid;
    int32_t nx, ny, nz;
    int64_t num_p;
    float dt, uin, max_age;
    uint32_t seed;
    float sx, scy, scz, shy, shz;
};

// advect_kernel (server/lbm.py:233-263)
__global__ void __launch_bounds__(256) k_advect(const AdvectArgs a) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= a.num_p) return;
    const float4 p = a.pos[i];
    const float4 m1 = sample_mac(a.mac, p.x, p.y, p.z, a.nx, a.ny, a.nz);
    const float hd = 0.5f * a.dt;
    const float4 m2 = sample_mac(a.mac, p.x + hd * m1.x, p.y + hd * m1.y, p.z + hd * m1.z, a.nx, a.ny, a.nz);
    float qx = p.x + a.dt * m2.x, qy = p.y + a.dt * m2.y, qz = p.z + a.dt * m2.z;
    float age = p.w + 1.0f;
    float s = sqrtf(m2.x * m2.x + m2.y * m2.y + m2.z * m2.z) / a.uin;
    bool dead = age > a.max_age || qx < 0.5f || qy < 0.5f || qz < 0.5f;
    if (qx > (float)a.nx - 3.0f || qy > (float)a.ny - 1.5f || qz > (float)a.nz - 1.5f || !(s < 100.0f)) dead = true;
    if (!dead) {
        const int32_t c = cidx((int32_t)roundf(qx), (int32_t)roundf(qy), (int32_t)roundf(qz), a.nx, a.ny, a.nz);
        if (a.solid[c] != 0) dead = true;
    }
    if (dead) {
        uint32_t r = pcg_hash(pcg_hash(a.seed) + (uint32_t)i);
        const float r0 = rng_f(r), r1 = rng_f(r), r2 = rng_f(r);
        qx = a.sx + r0 * 2.0f;
        qy = a.scy + (r1 * 2.0f - 1.0f) * a.shy;
        qz = a.scz + (r2 * 2.0f - 1.0f) * a.shz;
        age = 0.0f;
        s = 1.0f;
    }
    a.pos[i] = make_float4(qx, qy, qz, age);
    a.spd[i] = s;
}

// pack_particles (server/lbm.py:266-275)
__global__ void __launch_bounds__(256) k_pack(const float4* __restrict__ pos, const float* __restrict__ spd,
                                              ushort4* __restrict__ q16, uint8_t* __restrict__ q8, int32_t nx,
                                              int32_t ny, int32_t nz, int64_t num_p) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= num_p) return;
    const float4 p = pos[i];
    ushort4 o;
    o.x = (uint16_t)(int32_t)(clampf_(p.x / (float)nx, 0.0f, 1.0f) * 65535.0f + 0.5f);
    o.y = (uint16_t)(int32_t)(clampf_(p.y / (float)ny, 0.0f, 1.0f) * 65535.0f + 0.5f);
    o.z = (uint16_t)(int32_t)(clampf_(p.z / (float)nz, 0.0f, 1.0f) * 65535.0f + 0.5f);
    o.w = (uint16_t)(int32_t)clampf_(p.w, 0.0f, 65535.0f);
    q16[i] = o;
    q8[i] = (uint8_t)(int32_t)(clampf_(spd[i] / 2.0f, 0.0f, 1.0f) * 255.0f + 0.5f);
}

// vort (server/lbm.py:278-283)
__device__ __forceinline__ float vort(const float4* __restrict__ mac, int32_t x, int32_t y, int32_t z, int32_t nx,
                                      int32_t ny, int32_t nz) {
    const float4 xp = mac[cidx(x + 1, y, z, nx, ny, nz)], xm = mac[cidx(x - 1, y, z, nx, ny, nz)];
    const float4 yp = mac[cidx(x, y + 1, z, nx, ny, nz)], ym = mac[cidx(x, y - 1, z, nx, ny, nz)];
    const float4 zp = mac[cidx(x, y, z + 1, nx, ny, nz)], zm = mac[cidx(x, y, z - 1, nx, ny, nz)];
    const float dx1 = (xp.y - xm.y) * 0.5f, dx2 = (xp.z - xm.z) * 0.5f;
    const float dy0 = (yp.x - ym.x) * 0.5f, dy2 = (yp.z - ym.z) * 0.5f;
    const float dz0 = (zp.x - zm.x) * 0.5f, dz1 = (zp.y - zm.y) * 0.5f;
    const float a = dy2 - dz1, b = dz0 - dx2, c = dx1 - dy0;
    return sqrtf(a * a + b * b + c * c);
}

// slice_kernel (server/lbm.py:286-318)
__global__ void __launch_bounds__(256) k_slice(const float4* __restrict__ mac, const uint8_t* __restrict__ solid,
                                               uchar2* __restrict__ out, int32_t nx, int32_t ny, int32_t nz,
                                               int32_t axis, int32_t index, int32_t field, int32_t w, int32_t h,
                                               float uin, float lref, float vmin, float vmax) {
    const int32_t k = (int32_t)(blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= w * h) return;
    const int32_t a = k % w, b = k / w;
    int32_t cxv = index, cyv = b, czv = a;
    if (axis == 2) { cxv = a; cyv = b; czv = index; }
    else if (axis == 1) { cxv = a; cyv = index; czv = b; }
    const int32_t idx = cxv + nx * (cyv + ny * czv);
    const float4 m = mac[idx];
    float v = m.x / uin;
    if (field == 0) v = sqrtf(m.x * m.x + m.y * m.y + m.z * m.z) / uin;
    else if (field == 1) v = (m.w - 1.0f) / (1.5f * uin * uin);
    else if (field == 2) v = vort(mac, cxv, cyv, czv, nx, ny, nz) * lref / uin;
    const float t = clampf_((v - vmin) / (vmax - vmin), 0.0f, 1.0f);
    out[k] = make_uchar2((uint8_t)(int32_t)(t * 255.0f + 0.5f), solid[idx] != 0 ? 0 : 255);
}

// rho_fluid (server/lbm.py:321-350)
__device__ __forceinline__ float2 rho_fluid(const float4* __restrict__ mac, const uint8_t* __restrict__ solid, float px,
                                            float py, float pz, int32_t nx, int32_t ny, int32_t nz) {
    const float qx = clampf_(px, 0.0f, (float)nx - 1.001f);
    const float qy = clampf_(py, 0.0f, (float)ny - 1.001f);
    const float qz = clampf_(pz, 0.0f, (float)nz - 1.001f);
    const int32_t ix = (int32_t)floorf(qx), iy = (int32_t)floorf(qy), iz = (int32_t)floorf(qz);
    const float tx = qx - (float)ix, ty = qy - (float)iy, tz = qz - (float)iz;
    float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int ox = c & 1, oy = (c >> 1) & 1, oz = (c >> 2) & 1;
        const int32_t ci = cidx(ix + ox, iy + oy, iz + oz, nx, ny, nz);
        const float wx = ox ? tx : 1.0f - tx;
        const float wy = oy ? ty : 1.0f - ty;
        const float wz = oz ? tz : 1.0f - tz;
        const float wt = wx * wy * wz;
        if (solid[ci] == 0) {
            a0 = a0 + wt * mac[ci].w;
            a1 = a1 + wt;
        }
    }
    return make_float2(a0, a1);
}

// cp_kernel (server/lbm.py:353-368)
__global__ void __launch_bounds__(256) k_cp(const float4* __restrict__ mac, const uint8_t* __restrict__ solid,
                                            const float* __restrict__ verts, const float* __restrict__ norms,
                                            int8_t* __restrict__ out, int32_t nx, int32_t ny, int32_t nz, int64_t nv,
                                            float uin, float cp_range) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const float px = verts[3 * i], py = verts[3 * i + 1], pz = verts[3 * i + 2];
    const float nx_ = norms[3 * i], ny_ = norms[3 * i + 1], nz_ = norms[3 * i + 2];
    const float2 a = rho_fluid(mac, solid, px + nx_ * 1.25f, py + ny_ * 1.25f, pz + nz_ * 1.25f, nx, ny, nz);
    const float2 b = rho_fluid(mac, solid, px - nx_ * 1.25f, py - ny_ * 1.25f, pz - nz_ * 1.25f, nx, ny, nz);
    const float2 s = a.y >= b.y ? a : b;
    float cp = 0.0f;
    if (s.y > 0.05f) cp = (s.x / s.y - 1.0f) / (1.5f * uin * uin);
    out[i] = (int8_t)(int32_t)roundf(clampf_(cp / cp_range, -1.0f, 1.0f) * 127.0f);
}

}  // namespace wt

using namespace wt;

static int grid_check(int32_t nx, int32_t ny, int32_t nz) {
    if (nx < 1 || ny < 1 || nz < 1 || (int64_t)nx * ny * nz >= (1ll << 31))
        return wt_set_error(WT_ERR_DIMS, "grid %dx%dx%d out of range", nx, ny, nz);
    return WT_OK;
}

extern "C" int wt_advect(float* pos, float* spd, const float* mac, const uint8_t* solid, int32_t nx, int32_t ny,
                         int32_t nz, int64_t num_p, float dt, float uin, float max_age, uint32_t seed, float seed_x,
                         float seed_cy, float seed_cz, float seed_hy, float seed_hz, void* stream) {
    if (num_p == 0) return WT_OK;
    if (!pos || !spd || !mac || !solid || num_p < 0) return wt_set_error(WT_ERR_ARG, "wt_advect: bad arguments");
    if (int rc = grid_check(nx, ny, nz)) return rc;
    AdvectArgs a{reinterpret_cast<float4*>(pos), spd, reinterpret_cast<const float4*>(mac), solid, nx, ny, nz, num_p,
                 dt, uin, max_age, seed, seed_x, seed_cy, seed_cz, seed_hy, seed_hz};
    k_advect<<<(unsigned)((num_p + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
    return wt_cuda_check("wt_advect launch");
}

extern "C" int wt_pack_particles(const float* pos, const float* spd, uint16_t* q16, uint8_t* q8, int32_t nx,
                                 int32_t ny, int32_t nz, int64_t num_p, void* stream) {
    if (num_p == 0) return WT_OK;
    if (!pos || !spd || !q16 || !q8 || num_p < 0) return wt_set_error(WT_ERR_ARG, "wt_pack_particles: bad arguments");
    k_pack<<<(unsigned)((num_p + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float4*>(pos), spd, reinterpret_cast<ushort4*>(q16), q8, nx, ny, nz, num_p);
    return wt_cuda_check("wt_pack_particles launch");
}

extern "C" int wt_slice(const float* mac, const uint8_t* solid, uint8_t* out, int32_t nx, int32_t ny, int32_t nz,
                        int32_t axis, int32_t index, int32_t field, float uin, float lref, float vmin, float vmax,
                        void* stream) {
    if (!mac || !solid || !out) return wt_set_error(WT_ERR_ARG, "wt_slice: null buffer");
    if (int rc = grid_check(nx, ny, nz)) return rc;
    int32_t w, h, dim;
    if (axis == 2) { w = nx; h = ny; dim = nz; }
    else if (axis == 1) { w = nx; h = nz; dim = ny; }
    else if (axis == 0) { w = nz; h = ny; dim = nx; }
    else return wt_set_error(WT_ERR_ARG, "wt_slice: axis %d not in {0,1,2}", axis);
    if (index < 0 || index >= dim) return wt_set_error(WT_ERR_ARG, "wt_slice: index %d outside [0,%d)", index, dim);
    k_slice<<<(unsigned)((w * h + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float4*>(mac), solid, reinterpret_cast<uchar2*>(out), nx, ny, nz, axis, index, field,
        w, h, uin, lref, vmin, vmax);
    return wt_cuda_check("wt_slice launch");
}

extern "C" int wt_cp(const float* mac, const uint8_t* solid, const float* verts, const float* norms, int8_t* out,
                     int32_t nx, int32_t ny, int32_t nz, int64_t num_verts, float uin, float cp_range, void* stream) {
    if (num_verts == 0) return WT_OK;
    if (!mac || !solid || !verts || !norms || !out || num_verts < 0)
        return wt_set_error(WT_ERR_ARG, "wt_cp: bad arguments");
    if (int rc = grid_check(nx, ny, nz)) return rc;
    k_cp<<<(unsigned)((num_verts + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float4*>(mac), solid, verts, norms, out, nx, ny, nz, num_verts, uin, cp_range);
    return wt_cuda_check("wt_cp launch");
}
