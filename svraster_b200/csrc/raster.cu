// sm_100a sparse-voxel SDF rasterizer: preprocess, binning, forward and adjoint render.
//
// Behaviour follows the reference's SDF path (cuda/src/preprocess.cu, forward.cu,
// backward.cu); the organisation is ours:
//  * all stages take a batch of views (one launch per stage for the whole batch);
//  * binning sorts a key trimmed to the octree levels in use (order-equivalent to the
//    reference's 64-bit [tile | rank] key), then gathers each sorted record into an
//    80-byte AoS stream so a tile's records reach shared memory with one bulk copy;
//  * the render kernels double-buffer those copies on mbarriers, pre-filter records per
//    warp (8x4 pixel footprint + octant set) once per record instead of once per pixel,
//    and the adjoint accumulates per-record gradients in shared memory so each record
//    reaches global memory with one vector atomic per CTA instead of one per pixel.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "svr_common.cuh"

using namespace svr;

// ------------------------------------------------------------------ error plumbing
static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};
extern "C" const char* svr_last_error(void) { return g_last_error.c_str(); }
extern "C" int svr_version(void) { return 1; }
extern "C" long long svr_kernel_launches(void) { return g_launches.load(); }
void svr_note_launch(int n) { g_launches += n; }

int svr_fail(int code, const char* what) {
    g_last_error = what;
    return code;
}
#define CUDA_TRY(x)                                                                      \
    do {                                                                                 \
        cudaError_t e_ = (x);                                                            \
        if (e_ != cudaSuccess) {                                                         \
            return svr_fail(SVR_ERR_CUDA, (std::string(#x) + ": " + cudaGetErrorString(e_)).c_str()); \
        }                                                                                \
    } while (0)
#define LAUNCH_CHECK() do { svr_note_launch(1); CUDA_TRY(cudaGetLastError()); } while (0)

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// ------------------------------------------------------------------ buffer layouts
// geom buffer: meta | n_dup u32[M] | scan u32[M] | bbox uint2[M] | bits u32[M] | scan tmp
struct GeomMeta {
    unsigned long long path_or;   // OR of octree paths of rendered voxels
    unsigned long long total;     // sum of n_dup (64-bit, detects u32 scan overflow)
    unsigned int status;
    unsigned int pad[59];
};
static_assert(sizeof(GeomMeta) == 256, "meta block");

struct GeomLayout {
    size_t ndup, scan, bbox, bits, tmp, tmp_bytes, total;
};
static GeomLayout geom_layout(int64_t M) {
    GeomLayout L{};
    size_t off = sizeof(GeomMeta);
    L.ndup = off; off = align_up(off + 4 * (size_t)M, 256);
    L.scan = off; off = align_up(off + 4 * (size_t)M, 256);
    L.bbox = off; off = align_up(off + 8 * (size_t)M, 256);
    L.bits = off; off = align_up(off + 4 * (size_t)M, 256);
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)(M > 0 ? M : 1));
    L.tmp = off; L.tmp_bytes = tb; off = align_up(off + tb, 256);
    L.total = off;
    return L;
}

// binning buffer: meta | keys_in | keys_out | vals_in | vals_out | sort tmp | records
struct BinMeta {
    int rank_bits;   // rank bits kept in the sort key (tile id sits above them)
    int key64;       // 1 when keys are 64-bit
    int pad[62];
};
static_assert(sizeof(BinMeta) == 256, "bin meta block");
struct BinLayout {
    size_t keys_in, keys_out, vals_in, vals_out, tmp, tmp_bytes, recs, total;
};
static BinLayout bin_layout(int64_t R) {
    BinLayout L{};
    const int n = (int)(R > 0 ? R : 1);
    size_t t64 = 0, t32 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t64, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, n);
    cub::DeviceRadixSort::SortPairs(nullptr, t32, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, n);
    size_t off = sizeof(BinMeta);
    L.keys_in = off; off = align_up(off + 8 * (size_t)n, 256);
    L.keys_out = off; off = align_up(off + 8 * (size_t)n, 256);
    L.vals_in = off; off = align_up(off + 4 * (size_t)n, 256);
    L.vals_out = off; off = align_up(off + 4 * (size_t)n, 256);
    L.tmp = off; L.tmp_bytes = t64 > t32 ? t64 : t32; off = align_up(off + L.tmp_bytes, 256);
    L.recs = off; off = align_up(off + sizeof(Rec) * (size_t)n, 256);
    L.total = off;
    return L;
}

// image buffer: ranges uint2[T] | tile_last u32[T] | n_contrib u32[P] | status
struct ImgLayout {
    size_t ranges, tile_last, n_contrib, status, total;
};
static ImgLayout img_layout(int64_t P, int T) {
    ImgLayout L{};
    size_t off = 0;
    L.ranges = off; off = align_up(off + 8 * (size_t)T, 256);
    L.tile_last = off; off = align_up(off + 4 * (size_t)T, 256);
    L.n_contrib = off; off = align_up(off + 4 * (size_t)P, 256);
    L.status = off; off = align_up(off + 256, 256);
    L.total = off;
    return L;
}

extern "C" size_t svr_geom_buffer_bytes(int64_t n_items) { return geom_layout(n_items).total; }
extern "C" size_t svr_binning_buffer_bytes(int64_t R, int total_tiles) { (void)total_tiles; return bin_layout(R).total; }
extern "C" size_t svr_image_buffer_bytes(int64_t P, int T) { return img_layout(P, T).total; }

static int build_views(const svr_view_t* vh, int n, Views& V, int& total_tiles, int64_t& total_pix) {
    if (n <= 0 || n > SVR_MAX_VIEWS || vh == nullptr) return svr_fail(SVR_ERR_ARG, "bad view count");
    memset(&V, 0, sizeof(V));
    V.n = n;
    total_tiles = 0; total_pix = 0;
    for (int i = 0; i < n; ++i) {
        V.v[i] = vh[i];
        svr_view_t& v = V.v[i];
        if (v.width <= 0 || v.height <= 0 || v.width > 65535 || v.height > 65535)
            return svr_fail(SVR_ERR_ARG, "image size out of range");
        if (!v.w2c || !v.c2w) return svr_fail(SVR_ERR_ARG, "null camera matrix");
        v.tiles_x = (v.width + TILE - 1) / TILE;
        v.tiles_y = (v.height + TILE - 1) / TILE;
        v.tile_offset = total_tiles;
        v.pix_offset = total_pix;
        total_tiles += v.tiles_x * v.tiles_y;
        total_pix += (int64_t)v.width * v.height;
    }
    return SVR_OK;
}

// ------------------------------------------------------------------ preprocess
// Per (view, voxel): cull, projected bbox, octant bitset, duplicate count
// (preprocess.cu:36-154).  Also ORs the octree paths and sums the counts in 64 bits.
__global__ void __launch_bounds__(256) preprocess_kernel(
    const __grid_constant__ Views V, int N, const float3* __restrict__ centers,
    const float* __restrict__ lengths, const uint8_t* __restrict__ is_leaf,
    const int64_t* __restrict__ octpaths, int32_t* __restrict__ out_ndup,
    uint32_t* __restrict__ ndup, uint2* __restrict__ bboxes, uint32_t* __restrict__ bitsets,
    GeomMeta* __restrict__ meta)
{
    const int vi = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const svr_view_t& view = V.v[vi];
    uint32_t cnt = 0;
    unsigned long long path = 0;
    if (i < N) {
        const size_t item = (size_t)vi * N + i;
        uint2 bbox = make_uint2(0, 0);
        uint32_t qbits = 0;
        if (is_leaf[i] != 0) {
            const float3 vox_c = centers[i];
            const float vox_r = 0.5f * lengths[i];
            const float* c2w = view.c2w;
            const float3 ro = f3(c2w[3], c2w[7], c2w[11]);
            float w2c[12];
#pragma unroll
            for (int k = 0; k < 12; ++k) w2c[k] = view.w2c[k];
            const float3 rel = vox_c - ro;
            const float near = view.near_plane;
            if (!(dot3(rel, rel) < near * near)) {
                const float focal_x = 0.5f * view.width / view.tanfovx;
                const float focal_y = 0.5f * view.height / view.tanfovy;
                float2 cmin = make_float2(1e9f, 1e9f), cmax = make_float2(-1e9f, -1e9f);
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const float3 shift = f3((float)(((k & 4) >> 2) * 2 - 1), (float)(((k & 2) >> 1) * 2 - 1),
                                            (float)(((k & 1)) * 2 - 1));
                    const float3 wc = vox_c + vox_r * shift;
                    const float3 cc = xform34(w2c, wc);
                    if (cc.z < near) continue;
                    const float inv_z = 1.0f / cc.z;
                    const float u = cc.x * inv_z, v = cc.y * inv_z;
                    const uint32_t q = ((wc.x < ro.x) << 2) | ((wc.y < ro.y) << 1) | (wc.z < ro.z);
                    cmin = make_float2(fminf(cmin.x, u), fminf(cmin.y, v));
                    cmax = make_float2(fmaxf(cmax.x, u), fmaxf(cmax.y, v));
                    qbits |= (1u << q);
                }
                const float cx_h = view.cx - 0.5f, cy_h = view.cy - 0.5f;
                const float bminx = fmaxf(focal_x * cmin.x + cx_h, 0.0f);
                const float bminy = fmaxf(focal_y * cmin.y + cy_h, 0.0f);
                const float bmaxx = fminf(focal_x * cmax.x + cx_h, (float)view.width);
                const float bmaxy = fminf(focal_y * cmax.y + cy_h, (float)view.height);
                if (!(bminx > bmaxx || bminy > bmaxy)) {
                    bbox = make_uint2((((uint32_t)lrintf(bminx)) << 16) | ((uint32_t)lrintf(bminy)),
                                      (((uint32_t)lrintf(bmaxx)) << 16) | ((uint32_t)lrintf(bmaxy)));
                    // auxiliary.h:138-152
                    const int gx = view.tiles_x, gy = view.tiles_y;
                    const int tx0 = max(0, min(gx - 1, (int)((bbox.x >> 16) / TILE)));
                    const int ty0 = max(0, min(gy - 1, (int)((bbox.x << 16 >> 16) / TILE)));
                    const int tx1 = max(0, min(gx - 1, (int)((bbox.y >> 16) / TILE)));
                    const int ty1 = max(0, min(gy - 1, (int)((bbox.y << 16 >> 16) / TILE)));
                    cnt = (uint32_t)((1 + ty1 - ty0) * (1 + tx1 - tx0)) * __popc(qbits);
                    path = (unsigned long long)octpaths[i];
                } else {
                    qbits = 0;
                    bbox = make_uint2(0, 0);
                }
            } else {
                qbits = 0;
            }
        }
        if (cnt == 0) { qbits = 0; bbox = make_uint2(0, 0); }
        out_ndup[item] = (int32_t)cnt;
        ndup[item] = cnt;
        bboxes[item] = bbox;
        bitsets[item] = qbits;
    }
    // warp-aggregated 64-bit total and path OR: one atomic per warp
    unsigned long long tot = cnt;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        tot += __shfl_xor_sync(0xffffffffu, tot, o);
        path |= __shfl_xor_sync(0xffffffffu, path, o);
    }
    if ((threadIdx.x & 31) == 0 && tot) {
        atomicAdd(&meta->total, tot);
        atomicOr(&meta->path_or, path);
    }
}

extern "C" int svr_preprocess(const svr_view_t* views_host, int n_views, int N, const float* centers,
                              const float* lengths, const uint8_t* is_leaf, const int64_t* octpaths,
                              int32_t* out_n_dup, void* geom_buffer, void* stream)
{
    Views V;
    int T; int64_t P;
    int rc = build_views(views_host, n_views, V, T, P);
    if (rc) return rc;
    if (N < 0 || (N > 0 && (!centers || !lengths || !is_leaf || !octpaths || !out_n_dup || !geom_buffer)))
        return svr_fail(SVR_ERR_ARG, "preprocess: null argument");
    if ((int64_t)N >= (1ll << 29)) return svr_fail(SVR_ERR_ARG, "voxel ids need 29 bits");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t M = (int64_t)N * n_views;
    GeomLayout L = geom_layout(M);
    char* g = (char*)geom_buffer;
    CUDA_TRY(cudaMemsetAsync(g, 0, sizeof(GeomMeta), st));
    if (N == 0) return SVR_OK;
    dim3 grid((N + 255) / 256, n_views);
    preprocess_kernel<<<grid, 256, 0, st>>>(V, N, (const float3*)centers, lengths, is_leaf, octpaths, out_n_dup,
                                            (uint32_t*)(g + L.ndup), (uint2*)(g + L.bbox), (uint32_t*)(g + L.bits),
                                            (GeomMeta*)g);
    LAUNCH_CHECK();
    return SVR_OK;
}

extern "C" int svr_unpack_geom(const void* geom_buffer, int64_t M, uint32_t* ndup, uint32_t* bboxes,
                               uint32_t* bits, void* stream)
{
    GeomLayout L = geom_layout(M);
    const char* g = (const char*)geom_buffer;
    cudaStream_t st = (cudaStream_t)stream;
    if (M == 0) return SVR_OK;
    if (ndup) CUDA_TRY(cudaMemcpyAsync(ndup, g + L.ndup, 4 * M, cudaMemcpyDeviceToDevice, st));
    if (bboxes) CUDA_TRY(cudaMemcpyAsync(bboxes, g + L.bbox, 8 * M, cudaMemcpyDeviceToDevice, st));
    if (bits) CUDA_TRY(cudaMemcpyAsync(bits, g + L.bits, 4 * M, cudaMemcpyDeviceToDevice, st));
    return SVR_OK;
}

extern "C" int svr_count_rendered(int64_t M, void* geom_buffer, int64_t* num_rendered_host,
                                  uint64_t* path_or_host, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    char* g = (char*)geom_buffer;
    GeomLayout L = geom_layout(M);
    if (M > 0) {
        size_t tb = L.tmp_bytes;
        CUDA_TRY(cub::DeviceScan::InclusiveSum(g + L.tmp, tb, (const uint32_t*)(g + L.ndup),
                                               (uint32_t*)(g + L.scan), (int)M, st));
    }
    GeomMeta meta;
    CUDA_TRY(cudaMemcpyAsync(&meta, g, 16, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (meta.total >= (1ull << 32)) return svr_fail(SVR_ERR_CAPACITY, "more than 2^32 duplicated records");
    if (num_rendered_host) *num_rendered_host = (int64_t)meta.total;
    if (path_or_host) *path_or_host = meta.path_or;
    return SVR_OK;
}

// ------------------------------------------------------------------ binning
struct KeyFmt {
    int rank_shift;   // low rank bits dropped (all equal to the octant pattern)
    int rank_bits;    // rank bits kept
    int key_bits;     // tile bits + rank bits
};
static KeyFmt key_format(uint64_t path_or, int total_tiles) {
    KeyFmt f;
    // Lowest 3-bit level group that is non-zero in any rendered path; every group below it
    // is zero in all paths, so after the XOR with the octant pattern it equals the octant
    // id.  Keeping one such group preserves the octant tie-break; the rest is redundant.
    int g = 0;
    if (path_or == 0) g = MAX_LEVELS;
    else g = (__builtin_ctzll(path_or)) / 3;
    f.rank_shift = g > 0 ? 3 * (g - 1) : 0;
    f.rank_bits = RANK_BITS - f.rank_shift;
    int tb = 0;
    while ((1ll << tb) < (long long)total_tiles) ++tb;
    f.key_bits = tb + f.rank_bits;
    return f;
}

__device__ __forceinline__ uint64_t rep3(uint32_t q) {
    uint64_t v = 0;
#pragma unroll
    for (int l = 0; l < MAX_LEVELS; ++l) v = (v << 3) | q;
    return v;
}

// forward.cu:749-802: emit one (key, value) per (octant, tile) of every rendered voxel,
// in voxel-major, octant, row, column order (the order the stable sort preserves on ties).
template <typename KeyT>
__global__ void __launch_bounds__(256) duplicate_kernel(
    const __grid_constant__ Views V, int N, const int64_t* __restrict__ octpaths,
    const uint32_t* __restrict__ ndup, const uint32_t* __restrict__ scan, const uint2* __restrict__ bboxes,
    const uint32_t* __restrict__ bitsets, KeyT* __restrict__ keys, uint32_t* __restrict__ vals,
    int rank_shift, int rank_bits, BinMeta* __restrict__ meta, unsigned* status)
{
    const int64_t item = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (item == 0) { meta->rank_bits = rank_bits; meta->key64 = sizeof(KeyT) == 8; }
    const int64_t M = (int64_t)N * V.n;
    if (item >= M) return;
    const uint32_t cnt = ndup[item];
    if (cnt == 0) return;
    const int vi = (int)(item / N);
    const int i = (int)(item - (int64_t)vi * N);
    const svr_view_t& view = V.v[vi];
    uint32_t off = scan[item] - cnt;
    const uint32_t end = scan[item];
    const uint2 bb = bboxes[item];
    const int gx = view.tiles_x, gy = view.tiles_y;
    const int tx0 = max(0, min(gx - 1, (int)((bb.x >> 16) / TILE)));
    const int ty0 = max(0, min(gy - 1, (int)((bb.x << 16 >> 16) / TILE)));
    const int tx1 = max(0, min(gx - 1, (int)((bb.y >> 16) / TILE)));
    const int ty1 = max(0, min(gy - 1, (int)((bb.y << 16 >> 16) / TILE)));
    const uint64_t path = (uint64_t)octpaths[i];
    const uint32_t qb = bitsets[item];
    for (uint32_t q = 0; q < 8; ++q) {
        if (!(qb & (1u << q))) continue;
        const uint64_t rank = (path ^ rep3(q)) >> rank_shift;
        for (int y = ty0; y <= ty1; ++y)
            for (int x = tx0; x <= tx1; ++x) {
                if (off >= end) { atomicOr(status, ERR_COUNT_MISMATCH); return; }
                const uint64_t tile = (uint64_t)(view.tile_offset + y * gx + x);
                keys[off] = (KeyT)((tile << rank_bits) | rank);
                vals[off] = (q << 29) | (uint32_t)i;
                ++off;
            }
    }
    if (off != end) atomicOr(status, ERR_COUNT_MISMATCH);
}

// forward.cu:807-829
template <typename KeyT>
__global__ void tile_ranges_kernel(int64_t R, const KeyT* __restrict__ keys, int rank_bits, int T,
                                   uint2* __restrict__ ranges, unsigned* status)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R) return;
    const uint32_t t = (uint32_t)((uint64_t)keys[k] >> rank_bits);
    if (t >= (uint32_t)T) { atomicOr(status, ERR_BAD_INDEX); return; }
    if (k == 0) ranges[t].x = 0;
    else {
        const uint32_t p = (uint32_t)((uint64_t)keys[k - 1] >> rank_bits);
        if (p != t) { ranges[p].y = (uint32_t)k; ranges[t].x = (uint32_t)k; }
    }
    if (k == R - 1) ranges[t].y = (uint32_t)R;
}

extern "C" int svr_bin_and_sort(const svr_view_t* views_host, int n_views, int N, int64_t R, uint64_t path_or,
                                const int64_t* octpaths, void* geom_buffer, void* binning_buffer,
                                size_t binning_bytes, void* image_buffer, void* stream)
{
    Views V;
    int T; int64_t P;
    int rc = build_views(views_host, n_views, V, T, P);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t M = (int64_t)N * n_views;
    GeomLayout GL = geom_layout(M);
    BinLayout BL = bin_layout(R);
    ImgLayout IL = img_layout(P, T);
    if (binning_bytes < BL.total) return svr_fail(SVR_ERR_CAPACITY, "binning buffer too small");
    char* g = (char*)geom_buffer;
    char* b = (char*)binning_buffer;
    char* im = (char*)image_buffer;
    unsigned* status = (unsigned*)(im + IL.status);
    CUDA_TRY(cudaMemsetAsync(im + IL.ranges, 0, 8 * (size_t)T, st));
    CUDA_TRY(cudaMemsetAsync(status, 0, 4, st));
    if (R == 0) return SVR_OK;
    const KeyFmt kf = key_format(path_or, T);
    const int nb = (int)((M + 255) / 256);
    const int rb = (int)((R + 255) / 256);
    if (kf.key_bits <= 32) {
        duplicate_kernel<uint32_t><<<nb, 256, 0, st>>>(V, N, octpaths, (const uint32_t*)(g + GL.ndup),
            (const uint32_t*)(g + GL.scan), (const uint2*)(g + GL.bbox), (const uint32_t*)(g + GL.bits),
            (uint32_t*)(b + BL.keys_in), (uint32_t*)(b + BL.vals_in), kf.rank_shift, kf.rank_bits, (BinMeta*)b, status);
        LAUNCH_CHECK();
        size_t tb = BL.tmp_bytes;
        CUDA_TRY(cub::DeviceRadixSort::SortPairs(b + BL.tmp, tb, (const uint32_t*)(b + BL.keys_in),
                                                 (uint32_t*)(b + BL.keys_out), (const uint32_t*)(b + BL.vals_in),
                                                 (uint32_t*)(b + BL.vals_out), (int)R, 0, kf.key_bits, st));
        tile_ranges_kernel<uint32_t><<<rb, 256, 0, st>>>(R, (const uint32_t*)(b + BL.keys_out), kf.rank_bits, T,
                                                          (uint2*)(im + IL.ranges), status);
        LAUNCH_CHECK();
    } else {
        if (kf.key_bits > 64) return svr_fail(SVR_ERR_UNSUPPORTED, "sort key wider than 64 bits");
        duplicate_kernel<uint64_t><<<nb, 256, 0, st>>>(V, N, octpaths, (const uint32_t*)(g + GL.ndup),
            (const uint32_t*)(g + GL.scan), (const uint2*)(g + GL.bbox), (const uint32_t*)(g + GL.bits),
            (uint64_t*)(b + BL.keys_in), (uint32_t*)(b + BL.vals_in), kf.rank_shift, kf.rank_bits, (BinMeta*)b, status);
        LAUNCH_CHECK();
        size_t tb = BL.tmp_bytes;
        CUDA_TRY(cub::DeviceRadixSort::SortPairs(b + BL.tmp, tb, (const uint64_t*)(b + BL.keys_in),
                                                 (uint64_t*)(b + BL.keys_out), (const uint32_t*)(b + BL.vals_in),
                                                 (uint32_t*)(b + BL.vals_out), (int)R, 0, kf.key_bits, st));
        tile_ranges_kernel<uint64_t><<<rb, 256, 0, st>>>(R, (const uint64_t*)(b + BL.keys_out), kf.rank_bits, T,
                                                          (uint2*)(im + IL.ranges), status);
        LAUNCH_CHECK();
    }
    return SVR_OK;
}

extern "C" int svr_unpack_binning(const void* binning_buffer, int64_t R, int T, const void* image_buffer,
                                  int64_t P, uint32_t* vals, uint32_t* ranges, uint32_t* tile_last,
                                  uint32_t* n_contrib, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    BinLayout BL = bin_layout(R);
    ImgLayout IL = img_layout(P, T);
    const char* b = (const char*)binning_buffer;
    const char* im = (const char*)image_buffer;
    if (vals && R > 0) CUDA_TRY(cudaMemcpyAsync(vals, b + BL.vals_out, 4 * R, cudaMemcpyDeviceToDevice, st));
    if (ranges) CUDA_TRY(cudaMemcpyAsync(ranges, im + IL.ranges, 8 * (size_t)T, cudaMemcpyDeviceToDevice, st));
    if (tile_last) CUDA_TRY(cudaMemcpyAsync(tile_last, im + IL.tile_last, 4 * (size_t)T, cudaMemcpyDeviceToDevice, st));
    if (n_contrib) CUDA_TRY(cudaMemcpyAsync(n_contrib, im + IL.n_contrib, 4 * (size_t)P, cudaMemcpyDeviceToDevice, st));
    return SVR_OK;
}

// ------------------------------------------------------------------ record packing
// Gather each sorted record's voxel data into one 80-byte record.  The record's view is
// the view of its tile, read from the sorted key.
__global__ void __launch_bounds__(256) pack_records_kernel(
    const __grid_constant__ Views V, int N, int64_t R, const BinMeta* __restrict__ meta,
    const void* __restrict__ keys, const uint32_t* __restrict__ vals, const uint2* __restrict__ bboxes,
    const float* __restrict__ centers, const float* __restrict__ lengths, const float4* __restrict__ geos,
    const float* __restrict__ rgbs, int rgb_per_view, Rec* __restrict__ recs, unsigned* status)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R) return;
    const int rank_bits = meta->rank_bits;
    const uint64_t key = meta->key64 ? ((const uint64_t*)keys)[k] : (uint64_t)((const uint32_t*)keys)[k];
    const int vi = V.n == 1 ? 0 : view_of_tile(V, (int)(key >> rank_bits));
    const uint32_t val = vals[k];
    const uint32_t vid = val & 0x1FFFFFFFu;
    if (vid >= (uint32_t)N) { atomicOr(status, ERR_BAD_INDEX); return; }
    Rec r;
    r.cx = centers[3 * (size_t)vid]; r.cy = centers[3 * (size_t)vid + 1]; r.cz = centers[3 * (size_t)vid + 2];
    r.len = lengths[vid];
    const float4 g0 = geos[2 * (size_t)vid], g1 = geos[2 * (size_t)vid + 1];
    r.g[0] = g0.x; r.g[1] = g0.y; r.g[2] = g0.z; r.g[3] = g0.w;
    r.g[4] = g1.x; r.g[5] = g1.y; r.g[6] = g1.z; r.g[7] = g1.w;
    const size_t cb = 3 * ((rgb_per_view ? (size_t)vi * N : 0) + vid);
    r.r = rgbs[cb]; r.gr = rgbs[cb + 1]; r.b = rgbs[cb + 2];
    const uint2 bb = bboxes[(size_t)vi * N + vid];
    r.bbox0 = bb.x; r.bbox1 = bb.y;
    r.val = val;
    r.view = (uint32_t)vi;
    r.pad = 0;
    const float4* src = reinterpret_cast<const float4*>(&r);
    float4* dst = reinterpret_cast<float4*>(recs + k);
#pragma unroll
    for (int q = 0; q < 5; ++q) dst[q] = src[q];
}

// ------------------------------------------------------------------ forward render
struct alignas(16) FwdSmem {
    Rec buf[2][BLOCK];
    uint8_t wmask[BLOCK];
    uint64_t bar[2];
    uint32_t warp_quads[8];
    uint32_t red[8];
};

template <int NS, bool DEPTH, bool NORMAL, bool MAXW>
__global__ void __launch_bounds__(BLOCK) render_fwd_kernel(
    const __grid_constant__ Views V, const uint2* __restrict__ ranges, const Rec* __restrict__ recs,
    const float* __restrict__ s_ptr, uint32_t* __restrict__ tile_last, uint32_t* __restrict__ n_contrib,
    float* __restrict__ out_color, float* __restrict__ out_depth, float* __restrict__ out_normal,
    float* __restrict__ out_T, float* __restrict__ max_w, unsigned* __restrict__ status)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    FwdSmem& S = *reinterpret_cast<FwdSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = blockIdx.x;
    const int vi = view_of_tile(V, tile);
    const svr_view_t& view = V.v[vi];
    const int W = view.width, H = view.height;
    const int lt = tile - view.tile_offset;
    const int tx = lt % view.tiles_x, ty = lt / view.tiles_x;
    int dx, dy;
    tile_pixel(tid, dx, dy);
    const uint32_t px = tx * TILE + dx, py = ty * TILE + dy;
    const bool inside = (px < (uint32_t)W) && (py < (uint32_t)H);
    const Ray ray = pixel_ray(view, px, py);
    const uint32_t pq = ray_octant(ray.rd);
    const float s_val = *s_ptr;

    // octants present in each warp (only inside pixels can match a record)
    const uint32_t wq = __reduce_or_sync(0xffffffffu, inside ? (1u << pq) : 0u);
    if (lane == 0) S.warp_quads[warp] = wq;
    if (tid == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        fence_mbar_init();
    }
    const uint2 range = ranges[tile];
    const int n = (int)(range.y - range.x);
    const int nbatch = (n + BLOCK - 1) / BLOCK;
    __syncthreads();
    if (tid == 0 && nbatch > 0) {
        const uint32_t bytes = (uint32_t)min(BLOCK, n) * sizeof(Rec);
        mbar_arrive_tx(&S.bar[0], bytes);
        bulk_g2s(S.buf[0], recs + range.x, bytes, &S.bar[0]);
    }

    float T = 1.f, D = 0.f;
    float3 C = f3(0.f, 0.f, 0.f), Nn = f3(0.f, 0.f, 0.f);
    int64_t med_rec = -1;
    float med_T = 0.f;
    uint32_t last = 0;
    bool done = !inside;
    uint32_t parity = 0;   // bit b: parity of the next wait on bar[b]
    int b = 0;
    bool failed = false;
    for (; b < nbatch; ++b) {
        const int ndone = __syncthreads_count(done);
        if (ndone == BLOCK) break;
        if (tid == 0 && b + 1 < nbatch) {
            const int nb1 = min(BLOCK, n - (b + 1) * BLOCK);
            const uint32_t bytes = (uint32_t)nb1 * sizeof(Rec);
            mbar_arrive_tx(&S.bar[(b + 1) & 1], bytes);
            bulk_g2s(S.buf[(b + 1) & 1], recs + range.x + (size_t)(b + 1) * BLOCK, bytes, &S.bar[(b + 1) & 1]);
        }
        const int sb = b & 1;
        if (!mbar_wait(&S.bar[sb], (parity >> sb) & 1)) { failed = true; break; }
        parity ^= (1u << sb);
        const int cnt = min(BLOCK, n - b * BLOCK);
        const Rec* buf = S.buf[sb];
        // per-record warp footprint mask: bbox overlap with each warp's 8x4 block and the
        // record's octant present in that warp
        if (tid < cnt) {
            const Rec& r = buf[tid];
            const uint32_t x0 = r.bbox0 >> 16, y0 = r.bbox0 & 0xFFFF, x1 = r.bbox1 >> 16, y1 = r.bbox1 & 0xFFFF;
            const uint32_t q = r.val >> 29;
            uint32_t m = 0;
#pragma unroll
            for (int w = 0; w < 8; ++w) {
                const uint32_t wx0 = tx * TILE + (w & 1) * 8, wy0 = ty * TILE + (w >> 1) * 4;
                const bool hit = x0 <= wx0 + 7 && x1 >= wx0 && y0 <= wy0 + 3 && y1 >= wy0 &&
                                 ((S.warp_quads[w] >> q) & 1);
                m |= (uint32_t)hit << w;
            }
            S.wmask[tid] = (uint8_t)m;
        }
        __syncthreads();
        const int nchunk = (cnt + 31) >> 5;
        for (int c = 0; c < nchunk; ++c) {
            const int j = c * 32 + lane;
            const uint32_t rel = __ballot_sync(0xffffffffu, j < cnt && ((S.wmask[j] >> warp) & 1));
            if (rel == 0) continue;
            uint32_t cand = 0;
            if (!done) {
                uint32_t rr = rel;
                while (rr) {
                    const int k = __ffs(rr) - 1;
                    rr &= rr - 1;
                    const Rec& r = buf[c * 32 + k];
                    if (!pix_in_bbox(px, py, r.bbox0, r.bbox1) || pq != (r.val >> 29)) continue;
                    const float2 ab = ray_box(f3(r.cx, r.cy, r.cz), r.len, ray.ro, ray.rd_inv);
                    if (ab.x > ab.y) continue;
                    cand |= 1u << k;
                }
            }
            while (cand && !done) {
                const int k = __ffs(cand) - 1;
                cand &= cand - 1;
                const int j2 = c * 32 + k;
                const Rec& r = buf[j2];
                const float3 vox_c = f3(r.cx, r.cy, r.cz);
                const float vox_l = r.len;
                const float2 ab = ray_box(vox_c, vox_l, ray.ro, ray.rd_inv);
                const float a = ab.x, bb = ab.y;
                float g[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) g[q] = r.g[q];
                // forward.cu:255-306: NeuS alpha from the logistic CDF at entry and exit
                float w8[8];
                float local_a[NS > 1 ? NS : 1];
                const float vox_l_inv = 1.f / vox_l;
                const float3 p_entry = ray.ro + a * ray.rd;
                const float3 P_step = (bb - a) * ray.rd / (float)NS;
                const float3 qt_entry = (p_entry - (vox_c - 0.5f * vox_l)) * vox_l_inv;
                const float3 qt_step = P_step * vox_l_inv;
                tri_weights(qt_entry, w8);
                float sdf_former = interp8(g, w8);
                float phi_former = 1.f / (1.f + expf(-s_val * sdf_former));
                const float phi_entry = phi_former;
#pragma unroll
                for (int s = 0; s < NS; ++s) {
                    const float3 qt_curr = qt_entry + qt_step * (float)(s + 1);
                    tri_weights(qt_curr, w8);
                    const float sdf_curr = interp8(g, w8);
                    const float phi_curr = 1.f / (1.f + expf(-s_val * sdf_curr));
                    if (DEPTH && NS > 1) local_a[s] = fmaxf((phi_former - phi_curr) / (phi_former + 1e-6f), 0.f);
                    phi_former = phi_curr;
                    sdf_former = sdf_curr;
                }
                const float alpha = fmaxf((phi_entry - phi_former) / (phi_entry + 1e-6f), 0.f);
                if (alpha < MIN_ALPHA) continue;
                const float pt_w = T * alpha;
                C = C + pt_w * f3(r.r, r.gr, r.b);
                if (DEPTH) {
                    float dval;
                    if (NS == 3) {
                        const float step_sz = 0.3333333f * (bb - a);
                        const float a0 = local_a[0], a1 = local_a[NS > 1 ? 1 : 0], a2 = local_a[NS > 2 ? 2 : 0];
                        const float t0 = a + 0.5f * step_sz, t1 = a + 1.5f * step_sz, t2 = a + 2.5f * step_sz;
                        dval = a0 * t0 + (1.f - a0) * a1 * t1 + (1.f - a0) * (1.f - a1) * a2 * t2;
                    } else if (NS == 2) {
                        const float step_sz = 0.5f * (bb - a);
                        const float a0 = local_a[0], a1 = local_a[NS > 1 ? 1 : 0];
                        const float t0 = a + 0.5f * step_sz, t1 = a + 1.5f * step_sz;
                        dval = a0 * t0 + (1.f - a0) * a1 * t1;
                    } else {
                        dval = alpha * 0.5f * (a + bb);
                    }
                    D = D + T * dval;
                    if (T > 0.5f) { med_rec = (int64_t)range.x + b * BLOCK + j2; med_T = T; }
                }
                if (NORMAL) {
                    const float lin_nx = (g[4] + g[5] + g[6] + g[7]) - (g[0] + g[1] + g[2] + g[3]);
                    const float lin_ny = (g[2] + g[3] + g[6] + g[7]) - (g[0] + g[1] + g[4] + g[5]);
                    const float lin_nz = (g[1] + g[3] + g[5] + g[7]) - (g[0] + g[2] + g[4] + g[6]);
                    const float r_lin = safe_rnorm(lin_nx, lin_ny, lin_nz);
                    Nn = Nn + pt_w * r_lin * f3(lin_nx, lin_ny, lin_nz);
                }
                T *= (1.f - alpha);
                done |= (T < EARLY_STOP_T);
                last = (uint32_t)(b * BLOCK + j2 + 1);
                if (MAXW) atomicMax(((int*)max_w) + (r.val & 0x1FFFFFFFu), __float_as_int(pt_w));
            }
        }
    }
    // drain a copy still in flight when the loop left early
    if (!failed && b < nbatch) {
        const int sb = b & 1;
        if (!mbar_wait(&S.bar[sb], (parity >> sb) & 1)) failed = true;
    }
    if (failed && tid == 0) atomicOr(status, ERR_WAIT_TIMEOUT);

    float D_med = 0.f;
    if (DEPTH && inside && med_rec >= 0) {
        // forward.cu:450-521: 16-step refinement of the median-depth crossing
        const Rec& r = recs[med_rec];
        const float3 vox_c = f3(r.cx, r.cy, r.cz);
        const float vox_l = r.len;
        float g[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) g[q] = r.g[q];
        const float2 ab = ray_box(vox_c, vox_l, ray.ro, ray.rd_inv);
        const float a = ab.x, bb = ab.y;
        const float vox_l_inv = 1.f / vox_l;
        const float step_sz = (bb - a) * (1.f / 16);
        const float3 step = step_sz * ray.rd;
        D_med = a - 0.5f * step_sz;
        float3 q_edge = ((ray.ro + a * ray.rd) - (vox_c - 0.5f * vox_l)) * vox_l_inv;
        const float3 q_edge_step = step * vox_l_inv;
        float w8[8];
        tri_weights(q_edge, w8);
        float phi_prev = 1.f / (1.f + expf(-s_val * interp8(g, w8)));
        for (int k = 0; k < 16 && med_T > 0.5f; ++k) {
            D_med += step_sz;
            q_edge = q_edge + q_edge_step;
            tri_weights(q_edge, w8);
            const float phi_curr = 1.f / (1.f + expf(-s_val * interp8(g, w8)));
            const float alpha_k = (phi_prev - phi_curr) / (phi_prev + 1e-6f);
            med_T *= (1.f - alpha_k);
            phi_prev = phi_curr;
        }
    }

    uint32_t my_last = 0;
    if (inside) {
        const int64_t HW = (int64_t)W * H;
        const int64_t pix = (int64_t)py * W + px;
        const float* bg = view.bg;
        n_contrib[view.pix_offset + pix] = last;
        float* oc = out_color + 3 * view.pix_offset;
        oc[pix] = C.x + T * bg[0];
        oc[HW + pix] = C.y + T * bg[1];
        oc[2 * HW + pix] = C.z + T * bg[2];
        out_T[view.pix_offset + pix] = T;
        if (DEPTH) {
            float* od = out_depth + 4 * view.pix_offset;
            od[pix] = D * ray.rd_norm_inv;
            od[HW + pix] = 0.f;
            od[2 * HW + pix] = D_med * ray.rd_norm_inv;
            od[3 * HW + pix] = 0.f;
        }
        if (NORMAL) {
            float* on = out_normal + 3 * view.pix_offset;
            on[pix] = Nn.x; on[HW + pix] = Nn.y; on[2 * HW + pix] = Nn.z;
        }
        my_last = last;
    }
    const uint32_t wl = __reduce_max_sync(0xffffffffu, my_last);
    if (lane == 0) S.red[warp] = wl;
    __syncthreads();
    if (tid == 0) {
        uint32_t m = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) m = max(m, S.red[w]);
        tile_last[tile] = range.x + m;
        mbar_inval(&S.bar[0]);
        mbar_inval(&S.bar[1]);
    }
}

template <int NS, bool DEPTH, bool NORMAL, bool MAXW>
static int launch_fwd(int T, cudaStream_t st, const Views& V, const uint2* ranges, const Rec* recs,
                      const float* s_val, uint32_t* tile_last, uint32_t* n_contrib, float* color, float* depth,
                      float* normal, float* outT, float* max_w, unsigned* status)
{
    auto k = render_fwd_kernel<NS, DEPTH, NORMAL, MAXW>;
    const int smem = (int)sizeof(FwdSmem);
    CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k<<<T, BLOCK, smem, st>>>(V, ranges, recs, s_val, tile_last, n_contrib, color, depth, normal, outT, max_w, status);
    LAUNCH_CHECK();
    return SVR_OK;
}

extern "C" int svr_render_fwd(const svr_view_t* views_host, int n_views, int N, int64_t R, int n_samp,
                              int need_depth, int need_normal, const float* centers, const float* lengths,
                              const float* geos, const float* rgbs, int n_rgb_views, const float* s_val,
                              void* geom_buffer, void* binning_buffer, void* image_buffer, float* out_color,
                              float* out_depth, float* out_normal, float* out_T, float* max_w, void* stream)
{
    Views V;
    int T; int64_t P;
    int rc = build_views(views_host, n_views, V, T, P);
    if (rc) return rc;
    if (n_samp < 1 || n_samp > 3) return svr_fail(SVR_ERR_UNSUPPORTED, "n_samp must be 1, 2 or 3");
    if (!out_color || !out_T || !s_val || (need_depth && !out_depth) || (need_normal && !out_normal))
        return svr_fail(SVR_ERR_ARG, "render_fwd: null output");
    if (n_rgb_views != 1 && n_rgb_views != n_views) return svr_fail(SVR_ERR_ARG, "n_rgb_views");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t M = (int64_t)N * n_views;
    GeomLayout GL = geom_layout(M);
    BinLayout BL = bin_layout(R);
    ImgLayout IL = img_layout(P, T);
    char* g = (char*)geom_buffer;
    char* b = (char*)binning_buffer;
    char* im = (char*)image_buffer;
    unsigned* status = (unsigned*)(im + IL.status);
    const uint2* ranges = (const uint2*)(im + IL.ranges);
    Rec* recs = (Rec*)(b + BL.recs);
    if (R > 0) {
        pack_records_kernel<<<(unsigned)((R + 255) / 256), 256, 0, st>>>(
            V, N, R, (const BinMeta*)b, b + BL.keys_out, (const uint32_t*)(b + BL.vals_out),
            (const uint2*)(g + GL.bbox), centers, lengths, (const float4*)geos, rgbs, n_rgb_views > 1, recs, status);
        LAUNCH_CHECK();
    }
    uint32_t* tl = (uint32_t*)(im + IL.tile_last);
    uint32_t* nc = (uint32_t*)(im + IL.n_contrib);
    const bool D = need_depth != 0, Nm = need_normal != 0, MW = max_w != nullptr;
#define FWD_CASE(NS_)                                                                                   \
    if (n_samp == NS_) {                                                                                \
        if (D && Nm && !MW) return launch_fwd<NS_, true, true, false>(T, st, V, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, status); \
        if (D && Nm && MW) return launch_fwd<NS_, true, true, true>(T, st, V, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, status); \
        if (D && !Nm && !MW) return launch_fwd<NS_, true, false, false>(T, st, V, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, status); \
        if (D && !Nm && MW) return launch_fwd<NS_, true, false, true>(T, st, V, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, status); \
        if (!D && Nm && !MW) return launch_fwd<NS_, false, true, false>(T, st, V, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, status); \
        if (!D && Nm && MW) return launch_fwd<NS_, false, true, true>(T, st, V, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, status); \
        if (!D && !Nm && !MW) return launch_fwd<NS_, false, false, false>(T, st, V, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, status); \
        return launch_fwd<NS_, false, false, true>(T, st, V, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, status); \
    }
    FWD_CASE(1)
    FWD_CASE(2)
    FWD_CASE(3)
#undef FWD_CASE
    return svr_fail(SVR_ERR_UNSUPPORTED, "n_samp");
}

// ------------------------------------------------------------------ adjoint render
struct alignas(16) BwdSmem {
    Rec buf[2][BLOCK];
    float acc[BLOCK][12];
    uint8_t wmask[BLOCK];
    uint8_t touched[BLOCK];
    uint64_t bar[2];
    uint32_t warp_quads[8];
    float red[8];
};

template <bool DEPTH, bool NORMAL, bool RCONC>
__global__ void __launch_bounds__(BLOCK) render_bwd_kernel(
    const __grid_constant__ Views V, int N, const uint2* __restrict__ ranges, const uint32_t* __restrict__ tile_last,
    const uint32_t* __restrict__ n_contrib, const Rec* __restrict__ recs, const float* __restrict__ s_ptr,
    const float* __restrict__ out_T, const float* __restrict__ dL_dcolor, const float* __restrict__ dL_ddepth,
    const float* __restrict__ dL_dnormal, const float* __restrict__ dL_dT, float lambda_R, const float* __restrict__ gt_color,
    float* __restrict__ dL_dvox, float* __restrict__ drgbs, float* __restrict__ dL_ds, unsigned* __restrict__ status)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    BwdSmem& S = *reinterpret_cast<BwdSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = blockIdx.x;
    const int vi = view_of_tile(V, tile);
    const svr_view_t& view = V.v[vi];
    const int W = view.width, H = view.height;
    const int lt = tile - view.tile_offset;
    const int tx = lt % view.tiles_x, ty = lt / view.tiles_x;
    int dx, dy;
    tile_pixel(tid, dx, dy);
    const uint32_t px = tx * TILE + dx, py = ty * TILE + dy;
    const bool inside = (px < (uint32_t)W) && (py < (uint32_t)H);
    const Ray ray = pixel_ray(view, px, py);
    const uint32_t pq = ray_octant(ray.rd);
    const float s_val = *s_ptr;

    const uint32_t wq = __reduce_or_sync(0xffffffffu, inside ? (1u << pq) : 0u);
    if (lane == 0) S.warp_quads[warp] = wq;
    if (tid == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        fence_mbar_init();
    }
#pragma unroll
    for (int k = 0; k < 12; ++k) S.acc[tid][k] = 0.f;
    S.touched[tid] = 0;

    const uint32_t r0 = ranges[tile].x;
    const uint32_t r1 = tile_last[tile];
    const int n = r1 > r0 ? (int)(r1 - r0) : 0;
    const int nbatch = (n + BLOCK - 1) / BLOCK;

    // per-pixel adjoint state (backward.cu:156-216)
    const int64_t HW = (int64_t)W * H;
    const int64_t pix = (int64_t)py * W + px;
    float T = 0.f;
    uint32_t last_c = 0;
    float3 dpix = f3(0.f, 0.f, 0.f), dN = f3(0.f, 0.f, 0.f), gt = f3(0.f, 0.f, 0.f);
    float last_dT = 0.f, dD = 0.f;
    if (inside) {
        T = out_T[view.pix_offset + pix];
        last_c = n_contrib[view.pix_offset + pix];
        const float* dc = dL_dcolor + 3 * view.pix_offset;
        dpix = f3(dc[pix], dc[HW + pix], dc[2 * HW + pix]);
        const float* bg = view.bg;
        last_dT = dL_dT[view.pix_offset + pix] + dot3(f3(bg[0], bg[1], bg[2]), dpix);
        if (DEPTH) dD = dL_ddepth[4 * view.pix_offset + pix] * ray.rd_norm_inv;
        if (NORMAL) {
            const float* dn = dL_dnormal + 3 * view.pix_offset;
            dN = f3(dn[pix], dn[HW + pix], dn[2 * HW + pix]);
        }
        if (RCONC) {
            const float* gc = gt_color + 3 * view.pix_offset;
            gt = f3(gc[pix], gc[HW + pix], gc[2 * HW + pix]);
        }
    }
    const float WH_inv = 1.f / ((float)(W * H));
    const float weight_R = lambda_R * WH_inv;
    float ds_acc = 0.f;
    const bool active = inside && last_c > 0;

    __syncthreads();
    if (tid == 0 && nbatch > 0) {
        const int c0 = min(BLOCK, n);
        const uint32_t bytes = (uint32_t)c0 * sizeof(Rec);
        mbar_arrive_tx(&S.bar[0], bytes);
        bulk_g2s(S.buf[0], recs + (r1 - c0), bytes, &S.bar[0]);
    }
    uint32_t parity = 0;
    bool failed = false;
    int b = 0;
    for (; b < nbatch; ++b) {
        __syncthreads();   // batch b-1 processed and flushed: its buffer may be refilled
        if (tid == 0 && b + 1 < nbatch) {
            const int hi1 = n - (b + 1) * BLOCK;           // exclusive end (relative)
            const int c1 = min(BLOCK, hi1);
            const uint32_t bytes = (uint32_t)c1 * sizeof(Rec);
            mbar_arrive_tx(&S.bar[(b + 1) & 1], bytes);
            bulk_g2s(S.buf[(b + 1) & 1], recs + r0 + (hi1 - c1), bytes, &S.bar[(b + 1) & 1]);
        }
        const int sb = b & 1;
        if (!mbar_wait(&S.bar[sb], (parity >> sb) & 1)) { failed = true; break; }
        parity ^= (1u << sb);
        const int hi = n - b * BLOCK;
        const int cnt = min(BLOCK, hi);
        const int lo = hi - cnt;                    // relative index of slot 0
        const Rec* buf = S.buf[sb];
        if (tid < cnt) {
            const Rec& r = buf[tid];
            const uint32_t x0 = r.bbox0 >> 16, y0 = r.bbox0 & 0xFFFF, x1 = r.bbox1 >> 16, y1 = r.bbox1 & 0xFFFF;
            const uint32_t q = r.val >> 29;
            uint32_t m = 0;
#pragma unroll
            for (int w = 0; w < 8; ++w) {
                const uint32_t wx0 = tx * TILE + (w & 1) * 8, wy0 = ty * TILE + (w >> 1) * 4;
                const bool hit = x0 <= wx0 + 7 && x1 >= wx0 && y0 <= wy0 + 3 && y1 >= wy0 &&
                                 ((S.warp_quads[w] >> q) & 1);
                m |= (uint32_t)hit << w;
            }
            S.wmask[tid] = (uint8_t)m;
        }
        __syncthreads();
        const int nchunk = (cnt + 31) >> 5;
        for (int c = nchunk - 1; c >= 0; --c) {
            const int j = c * 32 + lane;
            const uint32_t rel = __ballot_sync(0xffffffffu, j < cnt && ((S.wmask[j] >> warp) & 1));
            if (rel == 0) continue;
            uint32_t cand = 0;
            if (active) {
                uint32_t rr = rel;
                while (rr) {
                    const int k = __ffs(rr) - 1;
                    rr &= rr - 1;
                    const int jj = c * 32 + k;
                    if ((uint32_t)(lo + jj) >= last_c) continue;
                    const Rec& r = buf[jj];
                    if (!pix_in_bbox(px, py, r.bbox0, r.bbox1) || pq != (r.val >> 29)) continue;
                    const float2 ab = ray_box(f3(r.cx, r.cy, r.cz), r.len, ray.ro, ray.rd_inv);
                    if (ab.x > ab.y) continue;
                    cand |= 1u << k;
                }
            }
            while (cand) {
                const int k = 31 - __clz(cand);           // back to front
                cand &= ~(1u << k);
                const int jj = c * 32 + k;
                const Rec& r = buf[jj];
                const float3 vox_c = f3(r.cx, r.cy, r.cz);
                const float vox_l = r.len;
                const float2 ab = ray_box(vox_c, vox_l, ray.ro, ray.rd_inv);
                const float a = ab.x, bb = ab.y;
                float g[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) g[q] = r.g[q];
                const float vox_l_inv = 1.f / vox_l;
                // backward.cu:313-388: entry / exit from ro + t rd, three sub-segment alphas
                const float3 p_entry = ray.ro + a * ray.rd;
                const float3 p_exit = ray.ro + bb * ray.rd;
                const float3 qt_entry = (p_entry - (vox_c - 0.5f * vox_l)) * vox_l_inv;
                const float3 qt_exit = (p_exit - (vox_c - 0.5f * vox_l)) * vox_l_inv;
                float we[8], wx[8];
                tri_weights(qt_entry, we);
                tri_weights(qt_exit, wx);
                float sdf_entry = 0.f, sdf_exit = 0.f;
#pragma unroll
                for (int i = 0; i < 8; ++i) { sdf_entry += g[i] * we[i]; sdf_exit += g[i] * wx[i]; }
                const float phi_entry = 1.f / (1.f + expf(-s_val * sdf_entry));
                const float phi_exit = 1.f / (1.f + expf(-s_val * sdf_exit));
                const float denom = phi_entry + 1e-6f;
                const float alpha = fmaxf((phi_entry - phi_exit) / denom, 0.f);
                if (alpha < MIN_ALPHA) continue;   // lambda_ascending == 0
                float dg[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) dg[i] = 0.f;
                float la[3] = {0.f, 0.f, 0.f};
                float eg[3][8];
                if (DEPTH) {
                    const float3 qt0 = ((ray.ro + a * ray.rd) - (vox_c - 0.5f * vox_l)) * vox_l_inv;
                    const float3 qt_step = ((bb - a) * ray.rd / 3.0f) * vox_l_inv;
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk) {
                        const float3 qk = qt0 + qt_step * (float)kk;
                        const float3 qk1 = qt0 + qt_step * (float)(kk + 1);
                        float wk[8], wk1[8];
                        tri_weights(qk, wk);
                        tri_weights(qk1, wk1);
                        float sdf_k = 0.f, sdf_k1 = 0.f;
#pragma unroll
                        for (int i = 0; i < 8; ++i) { sdf_k += g[i] * wk[i]; sdf_k1 += g[i] * wk1[i]; }
                        const float phi_k = 1.f / (1.f + expf(-s_val * sdf_k));
                        const float phi_k1 = 1.f / (1.f + expf(-s_val * sdf_k1));
                        const float denom_k = phi_k + 1e-6f;
                        const float raw_k = (phi_k - phi_k1) / denom_k;
                        const float allow = raw_k > 0.f ? 1.f : 0.f;
                        la[kk] = fmaxf(raw_k, 0.f);
                        const float d_ad_phi_k = allow * ((phi_k1) / (denom_k * denom_k));
                        const float d_ad_phi_k1 = allow * (-1.f / denom_k);
                        const float dphi_k = s_val * phi_k * (1.f - phi_k);
                        const float dphi_k1 = s_val * phi_k1 * (1.f - phi_k1);
#pragma unroll
                        for (int i = 0; i < 8; ++i) eg[kk][i] = d_ad_phi_k * dphi_k * wk[i] + d_ad_phi_k1 * dphi_k1 * wk1[i];
                    }
                }
                T = T / (1.f - alpha);
                const float pt_w = alpha * T;
                const float3 c3 = f3(r.r, r.gr, r.b);
                float dL_dpt_w = dot3(dpix, c3);
                if (NORMAL) {
                    // backward.cu:604-639
                    const float lin_nx = (g[4] + g[5] + g[6] + g[7]) - (g[0] + g[1] + g[2] + g[3]);
                    const float lin_ny = (g[2] + g[3] + g[6] + g[7]) - (g[0] + g[1] + g[4] + g[5]);
                    const float lin_nz = (g[1] + g[3] + g[5] + g[7]) - (g[0] + g[2] + g[4] + g[6]);
                    const float3 lin_n = f3(lin_nx, lin_ny, lin_nz);
                    const float r_lin = safe_rnorm(lin_nx, lin_ny, lin_nz);
                    const float3 surf_n = r_lin * lin_n;
                    dL_dpt_w += dot3(dN, surf_n);
                    const float3 dL_dsurf_n = pt_w * dN;
                    const float3 d = r_lin * (dL_dsurf_n - dot3(dL_dsurf_n, lin_n) * r_lin * surf_n);
                    dg[0] += -d.x - d.y - d.z; dg[1] += -d.x - d.y + d.z;
                    dg[2] += -d.x + d.y - d.z; dg[3] += -d.x + d.y + d.z;
                    dg[4] += +d.x - d.y - d.z; dg[5] += +d.x - d.y + d.z;
                    dg[6] += +d.x + d.y - d.z; dg[7] += +d.x + d.y + d.z;
                }
                const float dL_dalpha = T * (dL_dpt_w - last_dT);
                last_dT += alpha * (dL_dpt_w - last_dT);
                {
                    // backward.cu:650-671
                    const float pe = s_val * phi_entry * (1.f - phi_entry);
                    const float px_ = s_val * phi_exit * (1.f - phi_exit);
                    const float d_alpha_d_entry = (pe * (1.f - alpha)) / denom;
                    const float d_alpha_d_exit = -px_ / denom;
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        dg[i] += d_alpha_d_entry * we[i] * dL_dalpha;
                        dg[i] += d_alpha_d_exit * wx[i] * dL_dalpha;
                    }
                    const float d_phi_entry_ds = phi_entry * (1.f - phi_entry) * sdf_entry;
                    const float d_phi_exit_ds = phi_exit * (1.f - phi_exit) * sdf_exit;
                    const float d_alpha_ds = ((d_phi_entry_ds * (1.f - alpha)) + (-d_phi_exit_ds)) / denom;
                    ds_acc += dL_dalpha * d_alpha_ds;
                }
                if (DEPTH) {
                    // backward.cu:682-768 (n_samp 3, SDF)
                    const float step_sz = 0.3333333f * (bb - a);
                    const float a0 = la[0], a1 = la[1], a2 = la[2];
                    const float t0 = a + 0.5f * step_sz, t1 = a + 1.5f * step_sz, t2 = a + 2.5f * step_sz;
                    const float dval = a0 * t0 + (1.f - a0) * a1 * t1 + (1.f - a0) * (1.f - a1) * a2 * t2;
                    const float d0 = dD * T * (t0 + a1 * a2 * t2 - a1 * t1 - a2 * t2);
                    const float d1 = dD * T * (t1 + a0 * a2 * t2 - a0 * t1 - a2 * t2);
                    const float d2 = dD * T * (t2 + a0 * a1 * t2 - a0 * t2 - a1 * t2);
                    last_dT += dD * dval;
#pragma unroll
                    for (int i = 0; i < 8; ++i) dg[i] += d0 * eg[0][i] + d1 * eg[1][i] + d2 * eg[2][i];
                }
                float drgb0 = pt_w * dpix.x, drgb1 = pt_w * dpix.y, drgb2 = pt_w * dpix.z;
                if (RCONC) {
                    const float3 gr = weight_R * pt_w * 2.0f * (c3 - gt);
                    drgb0 += gr.x; drgb1 += gr.y; drgb2 += gr.z;
                }
                float* acc = S.acc[jj];
#pragma unroll
                for (int i = 0; i < 8; ++i) atomicAdd(acc + i, dg[i]);
                atomicAdd(acc + 8, drgb0);
                atomicAdd(acc + 9, drgb1);
                atomicAdd(acc + 10, drgb2);
                atomicAdd(acc + 11, fabsf(dL_dalpha * alpha));
                S.touched[jj] = 1;
            }
        }
        __syncthreads();
        // one vector atomic per touched record per CTA
        if (tid < cnt && S.touched[tid]) {
            const uint32_t vid = buf[tid].val & 0x1FFFFFFFu;
            float* a = S.acc[tid];
            if (vid < (uint32_t)N) {
                float4* dst = reinterpret_cast<float4*>(dL_dvox + 12 * (size_t)vid);
                atomicAdd(dst, make_float4(a[0], a[1], a[2], a[3]));
                atomicAdd(dst + 1, make_float4(a[4], a[5], a[6], a[7]));
                if (drgbs) {
                    float* cr = drgbs + 3 * ((size_t)vi * N + vid);
                    atomicAdd(cr, a[8]); atomicAdd(cr + 1, a[9]); atomicAdd(cr + 2, a[10]);
                    atomicAdd(dL_dvox + 12 * (size_t)vid + 11, a[11]);
                } else {
                    atomicAdd(dst + 2, make_float4(a[8], a[9], a[10], a[11]));
                }
            } else {
                atomicOr(status, ERR_BAD_INDEX);
            }
#pragma unroll
            for (int k = 0; k < 12; ++k) a[k] = 0.f;
            S.touched[tid] = 0;
        }
    }
    if (!failed && b < nbatch) {
        const int sb = b & 1;
        if (!mbar_wait(&S.bar[sb], (parity >> sb) & 1)) failed = true;
    }
    if (failed && tid == 0) atomicOr(status, ERR_WAIT_TIMEOUT);
    // one dL/ds atomic per CTA
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ds_acc += __shfl_xor_sync(0xffffffffu, ds_acc, o);
    if (lane == 0) S.red[warp] = ds_acc;
    __syncthreads();
    if (tid == 0) {
        float s = 0.f;
#pragma unroll
        for (int w = 0; w < 8; ++w) s += S.red[w];
        if (s != 0.f) atomicAdd(dL_ds, s);
        mbar_inval(&S.bar[0]);
        mbar_inval(&S.bar[1]);
    }
}

template <bool DEPTH, bool NORMAL, bool RCONC>
static int launch_bwd(int T, int N, cudaStream_t st, const Views& V, const uint2* ranges, const uint32_t* tl,
                      const uint32_t* nc, const Rec* recs, const float* s_val, const float* out_T,
                      const float* dc, const float* dd, const float* dn, const float* dT, float lam,
                      const float* gt, float* dvox, float* drgbs, float* ds, unsigned* status)
{
    auto k = render_bwd_kernel<DEPTH, NORMAL, RCONC>;
    const int smem = (int)sizeof(BwdSmem);
    CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k<<<T, BLOCK, smem, st>>>(V, N, ranges, tl, nc, recs, s_val, out_T, dc, dd, dn, dT, lam, gt, dvox, drgbs, ds,
                               status);
    LAUNCH_CHECK();
    return SVR_OK;
}

extern "C" int svr_render_bwd(const svr_view_t* views_host, int n_views, int N, int64_t R, int need_depth,
                              int need_normal, float lambda_R_concen, const float* gt_color, const float* s_val,
                              void* binning_buffer, void* image_buffer, const float* out_T,
                              const float* dL_dcolor, const float* dL_ddepth, const float* dL_dnormal,
                              const float* dL_dT, float* dL_dvox, float* drgbs, float* dL_ds, void* stream)
{
    Views V;
    int T; int64_t P;
    int rc = build_views(views_host, n_views, V, T, P);
    if (rc) return rc;
    if (!dL_dvox || !dL_ds || !dL_dcolor || !dL_dT || !out_T || (need_depth && !dL_ddepth) ||
        (need_normal && !dL_dnormal) || (lambda_R_concen > 0 && !gt_color))
        return svr_fail(SVR_ERR_ARG, "render_bwd: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    BinLayout BL = bin_layout(R);
    ImgLayout IL = img_layout(P, T);
    char* b = (char*)binning_buffer;
    char* im = (char*)image_buffer;
    unsigned* status = (unsigned*)(im + IL.status);
    const uint2* ranges = (const uint2*)(im + IL.ranges);
    const uint32_t* tl = (const uint32_t*)(im + IL.tile_last);
    const uint32_t* nc = (const uint32_t*)(im + IL.n_contrib);
    const Rec* recs = (const Rec*)(b + BL.recs);
    const bool D = need_depth != 0, Nm = need_normal != 0, RC = lambda_R_concen > 0;
#define BWD_ARGS T, N, st, V, ranges, tl, nc, recs, s_val, out_T, dL_dcolor, dL_ddepth, dL_dnormal, dL_dT, lambda_R_concen, gt_color, dL_dvox, drgbs, dL_ds, status
    if (D && Nm && RC) return launch_bwd<true, true, true>(BWD_ARGS);
    if (D && Nm && !RC) return launch_bwd<true, true, false>(BWD_ARGS);
    if (D && !Nm && RC) return launch_bwd<true, false, true>(BWD_ARGS);
    if (D && !Nm && !RC) return launch_bwd<true, false, false>(BWD_ARGS);
    if (!D && Nm && RC) return launch_bwd<false, true, true>(BWD_ARGS);
    if (!D && Nm && !RC) return launch_bwd<false, true, false>(BWD_ARGS);
    if (!D && !Nm && RC) return launch_bwd<false, false, true>(BWD_ARGS);
    return launch_bwd<false, false, false>(BWD_ARGS);
#undef BWD_ARGS
}

// Device status of the last raster launches on this image buffer (0 = clean).
extern "C" int svr_read_status(const void* image_buffer, int64_t P, int T, uint32_t* status_host, void* stream)
{
    ImgLayout IL = img_layout(P, T);
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(cudaMemcpyAsync(status_host, (const char*)image_buffer + IL.status, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return SVR_OK;
}
