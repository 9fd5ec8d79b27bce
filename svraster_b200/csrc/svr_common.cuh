// Shared device-side definitions of the sm_100a sparse-voxel rasterizer.
//
// The arithmetic helpers restate the reference's device math (cuda/src/auxiliary.h) with
// the same expression shapes, so nvcc contracts them into the same FMAs and the integer
// stages (bbox rounding, octant bits, sort keys) come out bit-identical.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/svraster_b200.h"

namespace svr {

constexpr int TILE = SVR_TILE;             // 16x16 pixel tiles (cuda/src/config.h:14-15)
constexpr int BLOCK = TILE * TILE;         // one thread per pixel
constexpr int MAX_LEVELS = 16;             // config.h:16
constexpr int RANK_BITS = 3 * MAX_LEVELS;  // config.h:38
constexpr float MIN_ALPHA = 0.00001f;      // config.h:19
constexpr float EARLY_STOP_T = 0.0001f;    // config.h:20

// Device status word bits (no __trap on a shared GPU: kernels record and return).
constexpr unsigned ERR_WAIT_TIMEOUT = 1u;
constexpr unsigned ERR_BAD_INDEX = 2u;
constexpr unsigned ERR_COUNT_MISMATCH = 4u;
constexpr unsigned ERR_CAPACITY = 8u;      // more records than the binning buffer holds
constexpr unsigned ERR_KEY_FORMAT = 16u;   // a rendered path has bits the trimmed key drops
constexpr unsigned ERR_DRAIN = 64u;        // a timed-out CTA exited with a bulk copy not seen to land

struct Views {
    int n;
    svr_view_t v[SVR_MAX_VIEWS];
};

// One sorted (tile, voxel, octant) record as staged into shared memory: 80 bytes,
// 16-byte aligned so a run of records moves with one cp.async.bulk.
struct __align__(16) Rec {
    float cx, cy, cz, len;      // voxel centre, edge length
    float g[8];                 // corner SDF values (corner = x<<2 | y<<1 | z)
    float r, gr, b;             // colour
    uint32_t bbox0, bbox1;      // projected bbox (x<<16 | y) min / max
    uint32_t val;               // octant << 29 | voxel id
    float sdf_lo, sdf_hi;       // corner SDF bounds widened by the rounding margin (record_dead)
};
static_assert(sizeof(Rec) == 80, "record must stay 80 bytes");

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float b) { return f3(a.x - b, a.y - b, a.z - b); }
__device__ __forceinline__ float3 operator+(float3 a, float b) { return f3(a.x + b, a.y + b, a.z + b); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator*(float b, float3 a) { return f3(a.x * b, a.y * b, a.z * b); }
__device__ __forceinline__ float3 operator*(float3 a, float b) { return f3(a.x * b, a.y * b, a.z * b); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// auxiliary.h:212-243.  Rounded product by product and sum by sum, no fused multiply-add:
// the projection feeds integer bboxes, so its rounding is spelled out (the C oracle does the
// same) instead of left to the compiler's contraction.  Measured against the reference's
// compiled extension on the benchmark workloads' 20 views, this form gives the fewest bbox
// differences of every pairing of these products into FMAs (31 of ~58M rendered voxel views,
// each a projected coordinate within an ulp of a pixel rounding boundary).
__device__ __forceinline__ float row34(const float* m, float3 p) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], p.x), __fmul_rn(m[1], p.y)), __fmul_rn(m[2], p.z)), m[3]);
}
__device__ __forceinline__ float3 xform34(const float* m, float3 p) {
    return f3(row34(m, p), row34(m + 4, p), row34(m + 8, p));
}
__device__ __forceinline__ float3 rot34(const float* m, float3 p) {
    return f3(m[0] * p.x + m[1] * p.y + m[2] * p.z,
              m[4] * p.x + m[5] * p.y + m[6] * p.z,
              m[8] * p.x + m[9] * p.y + m[10] * p.z);
}

// auxiliary.h:251-264: slab test of the ray against the voxel box.
__device__ __forceinline__ float2 ray_box(float3 c, float l, float3 ro, float3 rd_inv) {
    const float r = 0.5f * l;
    const float3 dir = c - ro;
    const float3 c0_ = (dir - r) * rd_inv;
    const float3 c1_ = (dir + r) * rd_inv;
    const float3 lo = f3(fminf(c0_.x, c1_.x), fminf(c0_.y, c1_.y), fminf(c0_.z, c1_.z));
    const float3 hi = f3(fmaxf(c0_.x, c1_.x), fmaxf(c0_.y, c1_.y), fmaxf(c0_.z, c1_.z));
    return make_float2(fmaxf(fmaxf(lo.x, lo.y), lo.z), fminf(fminf(hi.x, hi.y), hi.z));
}

// auxiliary.h:319-333: trilinear weights, corner index x<<2 | y<<1 | z.
__device__ __forceinline__ void tri_weights(const float3 q, float w[8]) {
    const float wx0 = 1.f - q.x, wx1 = q.x, wy0 = 1.f - q.y, wy1 = q.y, wz0 = 1.f - q.z, wz1 = q.z;
    w[0] = wx0 * wy0 * wz0; w[1] = wx0 * wy0 * wz1; w[2] = wx0 * wy1 * wz0; w[3] = wx0 * wy1 * wz1;
    w[4] = wx1 * wy0 * wz0; w[5] = wx1 * wy0 * wz1; w[6] = wx1 * wy1 * wz0; w[7] = wx1 * wy1 * wz1;
}
__device__ __forceinline__ float interp8(const float* g, const float* w) {
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += g[i] * w[i];
    return s;
}
// The logistic CDF of the NeuS density (forward.cu:270).
__device__ __forceinline__ float phi_of(float s_val, float sdf) { return 1.f / (1.f + expf(-s_val * sdf)); }
__device__ __forceinline__ float safe_rnorm(float x, float y, float z) { return rsqrtf(x * x + y * y + z * z + 1e-15f); }

__device__ __forceinline__ uint32_t ray_octant(float3 rd) {
    return ((rd.x < 0) << 2) | ((rd.y < 0) << 1) | (rd.z < 0);
}
__device__ __forceinline__ bool pix_in_bbox(uint32_t px, uint32_t py, uint32_t b0, uint32_t b1) {
    return px >= (b0 >> 16) && py >= (b0 << 16 >> 16) && px <= (b1 >> 16) && py <= (b1 << 16 >> 16);
}

// Camera ray of pixel (px, py), auxiliary.h:128-136 + forward.cu:124-133.
struct Ray {
    float3 ro, rd, rd_inv;
    float rd_norm_inv;
};
__device__ __forceinline__ Ray pixel_ray(const svr_view_t& v, int px, int py) {
    const float pfx = (float)px, pfy = (float)py;
    const float3 cam_rd = f3((pfx + 0.5f - v.cx) * 2.f * v.tanfovx / (float)v.width,
                             (pfy + 0.5f - v.cy) * 2.f * v.tanfovy / (float)v.height, 1.f);
    const float rd_norm = sqrtf(dot3(cam_rd, cam_rd));
    const float* m = v.c2w;
    const float3 raw = rot34(m, cam_rd);
    Ray r;
    r.rd_norm_inv = 1.f / rd_norm;
    r.ro = f3(m[3], m[7], m[11]);
    r.rd = raw * r.rd_norm_inv;
    r.rd_inv = f3(1.f / r.rd.x, 1.f / r.rd.y, 1.f / r.rd.z);
    return r;
}

// Pixel of thread t in a 16x16 tile: warps cover 8x4 blocks (forward.cu:87-102).
__device__ __forceinline__ void tile_pixel(int t, int& dx, int& dy) {
    const int warp = t >> 5, lane = t & 31;
    dx = (warp & 1) * 8 + (lane & 7);
    dy = (warp >> 1) * 4 + (lane >> 3);
}

__device__ __forceinline__ int view_of_tile(const Views& V, int tile) {
    int lo = 0, hi = V.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (V.v[mid].tile_offset <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------------------ mbarrier + bulk copy
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bounded wait for phase `parity` of `bar`.  Returns false after ~`limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = (1u << 22)) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n"
            " mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok) : "r"(a), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}
// One bulk global->shared copy completing on `bar` (size and addresses 16-byte aligned).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

}  // namespace svr
