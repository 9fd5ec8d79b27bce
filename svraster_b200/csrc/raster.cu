// sm_100a sparse-voxel SDF rasterizer: preprocess, binning, forward and adjoint render.
//
// Behaviour follows the reference's SDF path (cuda/src/preprocess.cu, forward.cu,
// backward.cu); the organisation is ours:
//  * all stages take a batch of views (one launch per stage for the whole batch);
//  * binning gives the reference's record order either by a radix sort of a key trimmed to
//    the octree levels in use (order-equivalent to its 64-bit [tile | rank] key) or, in the
//    training step, by per-tile counting, scatter and a one-CTA-per-tile sort over a
//    pair-order table (tile_sort.cuh); each sorted record is then packed into an 80-byte
//    AoS stream so a tile's records reach shared memory with one bulk copy per slot;
//  * the render kernels (render_pairs.cuh) stream 128-record slots through an mbarrier
//    ring, filter each slot's records once for the whole tile, and evaluate the candidate
//    (pixel, record) pairs on full warps; the forward stores each slot's candidate masks,
//    which the adjoint reads back instead of filtering again, and the adjoint sends each
//    pair's gradients with vector reductions.
#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "svr_common.cuh"
#include "tile_sort.cuh"

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

// Raise a kernel's dynamic shared-memory limit once per device (kept out of the launch
// path so that launches can be captured into a graph without extra API calls).
template <typename K>
static int ensure_smem(K k, int smem, std::atomic<unsigned long long>& done)
{
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return SVR_OK;
    CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    done.fetch_or(bit, std::memory_order_acq_rel);
    return SVR_OK;
}


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
    int rank_bits;     // rank bits kept in the sort key (tile id sits above them)
    int key64;         // 1 when keys are 64-bit
    long long count;   // records binned: min(total from preprocess, capacity)
    int cand_ok;       // 1 when the candidate rows hold the masks of the last forward over these records
    int pad[59];
};
static_assert(sizeof(BinMeta) == 256, "bin meta block");
struct BinLayout {
    size_t keys_in, keys_out, vals_in, vals_out, tmp, tmp_bytes, recs, pairs_b, cand, total;
    int64_t cand_slots;
};
// Candidate rows: the forward's per-pixel candidate masks of every slot it streams (SVR_BATCH
// records of a tile), one uint4 per pixel of the tile, 4 KB per slot; the adjoint reads them
// instead of filtering again.  Slot s of the tile with records [r0, r1) is row block
// r0 / SVR_BATCH + tile + s: distinct for every (tile, slot), below R / SVR_BATCH + T + 1.
#ifndef SVR_BATCH
#define SVR_BATCH 128
#endif
static int64_t cand_slot_count(int64_t R, int T) { return (R > 0 ? R : 0) / SVR_BATCH + (T > 0 ? T : 0) + 1; }
static BinLayout bin_layout(int64_t R, int T) {
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
    L.pairs_b = off; off = align_up(off + 8 * (size_t)n, 256);   // per-tile sort: second (key, value) array
    L.cand_slots = cand_slot_count(R, T);
    L.cand = off; off = align_up(off + (size_t)L.cand_slots * BLOCK * sizeof(uint4), 256);
    L.total = off;
    return L;
}

// image buffer: ranges uint2[T] | tile_last u32[T] | n_contrib u32[P] | status |
//               launch order u32[T] | order sort keys / values / scratch
struct ImgLayout {
    size_t ranges, tile_last, n_contrib, status, order, okeys_in, okeys_out, ovals_in, otmp, otmp_bytes;
    size_t tile_cnt, cursor, blk_sum, blk_hist, total;   // tile binning (svr_bin_tiles)
};
static ImgLayout img_layout(int64_t P, int T) {
    ImgLayout L{};
    size_t off = 0;
    const int nt = T > 0 ? T : 1;
    L.ranges = off; off = align_up(off + 8 * (size_t)T, 256);
    L.tile_last = off; off = align_up(off + 4 * (size_t)T, 256);
    L.n_contrib = off; off = align_up(off + 4 * (size_t)P, 256);
    L.status = off; off = align_up(off + 256, 256);
    L.order = off; off = align_up(off + 4 * (size_t)nt, 256);
    L.okeys_in = off; off = align_up(off + 4 * (size_t)nt, 256);
    L.okeys_out = off; off = align_up(off + 4 * (size_t)nt, 256);
    L.ovals_in = off; off = align_up(off + 4 * (size_t)nt, 256);
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, nt);
    L.otmp = off; L.otmp_bytes = tb; off = align_up(off + tb, 256);
    const size_t nblk = (size_t)(nt + TS_BLK - 1) / TS_BLK;
    L.tile_cnt = off; off = align_up(off + 4 * (size_t)nt, 256);
    L.cursor = off; off = align_up(off + 4 * (size_t)nt, 256);
    L.blk_sum = off; off = align_up(off + 4 * nblk, 256);
    L.blk_hist = off; off = align_up(off + 4 * 256 * nblk, 256);
    L.total = off;
    return L;
}

extern "C" size_t svr_geom_buffer_bytes(int64_t n_items) { return geom_layout(n_items).total; }
extern "C" size_t svr_binning_buffer_bytes(int64_t R, int total_tiles) { return bin_layout(R, total_tiles).total; }
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
// Grid-stride over the voxels of view blockIdx.y with a bounded grid: the running total and
// path OR are reduced over the block and leave with one atomic each (one per warp put tens
// of millions of same-address atomics on one L2 slice for a 64-view batch).
__global__ void __launch_bounds__(256, 4) preprocess_kernel(
    const __grid_constant__ Views V, int N, const float3* __restrict__ centers,
    const float* __restrict__ lengths, const uint8_t* __restrict__ is_leaf,
    const int64_t* __restrict__ octpaths, int32_t* __restrict__ out_ndup,
    uint32_t* __restrict__ ndup, uint2* __restrict__ bboxes, uint32_t* __restrict__ bitsets,
    GeomMeta* __restrict__ meta)
{
    __shared__ unsigned long long s_tot[8], s_path[8];
    const int vi = blockIdx.y;
    const svr_view_t& view = V.v[vi];
    const float* c2w = view.c2w;
    const float3 ro = f3(c2w[3], c2w[7], c2w[11]);
    float w2c[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) w2c[k] = view.w2c[k];
    const float near = view.near_plane;
    const float focal_x = 0.5f * view.width / view.tanfovx;
    const float focal_y = 0.5f * view.height / view.tanfovy;
    const float cx_h = view.cx - 0.5f, cy_h = view.cy - 0.5f;
    const int gx = view.tiles_x, gy = view.tiles_y;
    unsigned long long tot = 0, path = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const size_t item = (size_t)vi * N + i;
        uint32_t cnt = 0;
        uint2 bbox = make_uint2(0, 0);
        uint32_t qbits = 0;
        if (is_leaf[i] != 0) {
            const float3 vox_c = centers[i];
            const float vox_r = 0.5f * lengths[i];
            const float3 rel = vox_c - ro;
            const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(rel.x, rel.x), __fmul_rn(rel.y, rel.y)),
                                       __fmul_rn(rel.z, rel.z));
            if (!(d2 < near * near)) {
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
                // fused (one rounding), as the C oracle spells it
                const float bminx = fmaxf(fmaf(focal_x, cmin.x, cx_h), 0.0f);
                const float bminy = fmaxf(fmaf(focal_y, cmin.y, cy_h), 0.0f);
                const float bmaxx = fminf(fmaf(focal_x, cmax.x, cx_h), (float)view.width);
                const float bmaxy = fminf(fmaf(focal_y, cmax.y, cy_h), (float)view.height);
                if (!(bminx > bmaxx || bminy > bmaxy)) {
                    bbox = make_uint2((((uint32_t)lrintf(bminx)) << 16) | ((uint32_t)lrintf(bminy)),
                                      (((uint32_t)lrintf(bmaxx)) << 16) | ((uint32_t)lrintf(bmaxy)));
                    // auxiliary.h:138-152
                    const int tx0 = max(0, min(gx - 1, (int)((bbox.x >> 16) / TILE)));
                    const int ty0 = max(0, min(gy - 1, (int)((bbox.x << 16 >> 16) / TILE)));
                    const int tx1 = max(0, min(gx - 1, (int)((bbox.y >> 16) / TILE)));
                    const int ty1 = max(0, min(gy - 1, (int)((bbox.y << 16 >> 16) / TILE)));
                    cnt = (uint32_t)((1 + ty1 - ty0) * (1 + tx1 - tx0)) * __popc(qbits);
                    if (cnt) path |= (unsigned long long)octpaths[i];
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
        tot += cnt;
    }
    // block reduction, then one atomic per block for each of the total and the path OR
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        tot += __shfl_xor_sync(0xffffffffu, tot, o);
        path |= __shfl_xor_sync(0xffffffffu, path, o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { s_tot[warp] = tot; s_path[warp] = path; }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0, pth = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) { t += s_tot[w]; pth |= s_path[w]; }
        if (t) {
            atomicAdd(&meta->total, t);
            atomicOr(&meta->path_or, pth);
        }
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
    // about 8 blocks per SM in total, split over the views
    const int per_view = std::max(1, std::min((N + 255) / 256, (8 * 148 + n_views - 1) / n_views));
    dim3 grid(per_view, n_views);
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

extern "C" int svr_scan_rendered(int64_t M, void* geom_buffer, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    char* g = (char*)geom_buffer;
    GeomLayout L = geom_layout(M);
    if (M > 0) {
        size_t tb = L.tmp_bytes;
        CUDA_TRY(cub::DeviceScan::InclusiveSum(g + L.tmp, tb, (const uint32_t*)(g + L.ndup),
                                               (uint32_t*)(g + L.scan), (int)M, st));
    }
    return SVR_OK;
}

extern "C" int svr_count_rendered(int64_t M, void* geom_buffer, int64_t* num_rendered_host,
                                  uint64_t* path_or_host, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    char* g = (char*)geom_buffer;
    int rc = svr_scan_rendered(M, geom_buffer, stream);
    if (rc) return rc;
    GeomMeta meta;
    CUDA_TRY(cudaMemcpyAsync(&meta, g, 16, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (meta.total >= (1ull << 32)) return svr_fail(SVR_ERR_CAPACITY, "more than 2^32 duplicated records");
    if (num_rendered_host) *num_rendered_host = (int64_t)meta.total;
    if (path_or_host) *path_or_host = meta.path_or;
    return SVR_OK;
}

// Record total and path OR of a preprocessed batch, read without the scan that
// svr_count_rendered runs for the radix-sort binning (svr_bin_tiles needs no scan).
extern "C" int svr_rendered_total(const void* geom_buffer, int64_t* num_rendered_host, uint64_t* path_or_host,
                                  void* stream)
{
    if (!geom_buffer) return svr_fail(SVR_ERR_ARG, "rendered_total: null buffer");
    cudaStream_t st = (cudaStream_t)stream;
    GeomMeta meta;
    CUDA_TRY(cudaMemcpyAsync(&meta, geom_buffer, 16, cudaMemcpyDeviceToHost, st));
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
// Records past the capacity `cap` of the binning buffer are dropped and flagged
// (ERR_CAPACITY); the record count read by the later stages is min(total, cap), taken
// from the device, so the host need not know the total (graph capture).
template <typename KeyT>
__global__ void __launch_bounds__(256) duplicate_kernel(
    const __grid_constant__ Views V, int N, const int64_t* __restrict__ octpaths,
    const uint32_t* __restrict__ ndup, const uint32_t* __restrict__ scan, const uint2* __restrict__ bboxes,
    const uint32_t* __restrict__ bitsets, KeyT* __restrict__ keys, uint32_t* __restrict__ vals,
    int rank_shift, int rank_bits, const GeomMeta* __restrict__ gmeta, int64_t cap, BinMeta* __restrict__ meta,
    unsigned* status, const uint32_t* __restrict__ rank_table)
{
    const int64_t item = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (item == 0) {
        const unsigned long long total = gmeta->total;
        meta->rank_bits = rank_bits;
        meta->key64 = sizeof(KeyT) == 8;
        meta->count = total < (unsigned long long)cap ? (long long)total : (long long)cap;
        if (total > (unsigned long long)cap) atomicOr(status, ERR_CAPACITY);
    }
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
    if (rank_shift > 0 && (path & ((1ull << rank_shift) - 1ull))) atomicOr(status, ERR_KEY_FORMAT);
    const uint32_t qb = bitsets[item];
    for (uint32_t q = 0; q < 8; ++q) {
        if (!(qb & (1u << q))) continue;
        // the dense rank of (voxel, octant) when a table is given: same order, fewer bits
        const uint64_t rank = rank_table ? (uint64_t)rank_table[8 * (size_t)i + q] : (path ^ rep3(q)) >> rank_shift;
        for (int y = ty0; y <= ty1; ++y)
            for (int x = tx0; x <= tx1; ++x) {
                if (off >= end) { atomicOr(status, ERR_COUNT_MISMATCH); return; }
                if ((int64_t)off >= cap) return;   // flagged above
                const uint64_t tile = (uint64_t)(view.tile_offset + y * gx + x);
                keys[off] = (KeyT)((tile << rank_bits) | rank);
                vals[off] = (q << 29) | (uint32_t)i;
                ++off;
            }
    }
    if (off != end) atomicOr(status, ERR_COUNT_MISMATCH);
}

// Slots [count, cap) of the key array get the largest key of the format, so the stable
// sort leaves them after every real record.
template <typename KeyT>
__global__ void pad_keys_kernel(const BinMeta* __restrict__ meta, int64_t cap, KeyT sentinel,
                                KeyT* __restrict__ keys, uint32_t* __restrict__ vals)
{
    const int64_t count = meta->count;
    for (int64_t k = count + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < cap;
         k += (int64_t)gridDim.x * blockDim.x) {
        keys[k] = sentinel;
        vals[k] = 0u;
    }
}

// forward.cu:807-829
template <typename KeyT>
__global__ void tile_ranges_kernel(const BinMeta* __restrict__ meta, const KeyT* __restrict__ keys, int rank_bits,
                                   int T, uint2* __restrict__ ranges, unsigned* status)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t R = meta->count;
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

template <typename KeyT>
static int bin_sort_typed(const Views& V, int N, int64_t R, const KeyFmt& kf, int T, const int64_t* octpaths,
                          char* g, const GeomLayout& GL, char* b, const BinLayout& BL, char* im, const ImgLayout& IL,
                          unsigned* status, cudaStream_t st, const uint32_t* rank_table = nullptr)
{
    const int64_t M = (int64_t)N * V.n;
    const int nb = (int)((M + 255) / 256);
    const int rb = (int)((R + 255) / 256);
    BinMeta* meta = (BinMeta*)b;
    KeyT* keys_in = (KeyT*)(b + BL.keys_in);
    uint32_t* vals_in = (uint32_t*)(b + BL.vals_in);
    duplicate_kernel<KeyT><<<nb, 256, 0, st>>>(V, N, octpaths, (const uint32_t*)(g + GL.ndup),
        (const uint32_t*)(g + GL.scan), (const uint2*)(g + GL.bbox), (const uint32_t*)(g + GL.bits),
        keys_in, vals_in, kf.rank_shift, kf.rank_bits, (const GeomMeta*)g, R, meta, status, rank_table);
    LAUNCH_CHECK();
    const KeyT sentinel = kf.key_bits >= (int)(8 * sizeof(KeyT)) ? (KeyT)~(KeyT)0
                                                                    : (KeyT)((((KeyT)1) << kf.key_bits) - 1);
    pad_keys_kernel<KeyT><<<2 * 148, 256, 0, st>>>(meta, R, sentinel, keys_in, vals_in);
    LAUNCH_CHECK();
    size_t tb = BL.tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(b + BL.tmp, tb, (const KeyT*)keys_in, (KeyT*)(b + BL.keys_out),
                                             (const uint32_t*)vals_in, (uint32_t*)(b + BL.vals_out), (int)R, 0,
                                             kf.key_bits, st));
    tile_ranges_kernel<KeyT><<<rb, 256, 0, st>>>(meta, (const KeyT*)(b + BL.keys_out), kf.rank_bits, T,
                                                 (uint2*)(im + IL.ranges), status);
    LAUNCH_CHECK();
    return SVR_OK;
}

// Launch order of the tiles: most records first (stable, so equal counts keep tile order).
// CTAs start roughly in blockIdx order, so the long tiles no longer start in the last wave
// and leave the GPU waiting on a few of them.
__global__ void tile_order_keys_kernel(int T, const uint2* __restrict__ ranges, uint32_t* __restrict__ keys,
                                       uint32_t* __restrict__ vals)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const uint2 r = ranges[t];
    keys[t] = 0xFFFFFFFFu - (r.y > r.x ? r.y - r.x : 0u);
    vals[t] = (uint32_t)t;
}

static int tile_launch_order(int T, char* im, const ImgLayout& IL, cudaStream_t st)
{
    if (T <= 0) return SVR_OK;
    tile_order_keys_kernel<<<(T + 255) / 256, 256, 0, st>>>(T, (const uint2*)(im + IL.ranges),
                                                            (uint32_t*)(im + IL.okeys_in),
                                                            (uint32_t*)(im + IL.ovals_in));
    LAUNCH_CHECK();
    size_t tb = IL.otmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(im + IL.otmp, tb, (const uint32_t*)(im + IL.okeys_in),
                                             (uint32_t*)(im + IL.okeys_out), (const uint32_t*)(im + IL.ovals_in),
                                             (uint32_t*)(im + IL.order), T, 0, 32, st));
    return SVR_OK;
}

extern "C" int svr_binning_count(const void* binning_buffer, int64_t* count_host, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    long long c = 0;
    CUDA_TRY(cudaMemcpyAsync(&c, (const char*)binning_buffer + offsetof(BinMeta, count), 8, cudaMemcpyDeviceToHost,
                             st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *count_host = c;
    return SVR_OK;
}

extern "C" int svr_binning_candidates_valid(const void* binning_buffer, int* valid_host, void* stream)
{
    if (!binning_buffer || !valid_host) return svr_fail(SVR_ERR_ARG, "candidates valid: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    int v = 0;
    CUDA_TRY(cudaMemcpyAsync(&v, (const char*)binning_buffer + offsetof(BinMeta, cand_ok), sizeof(int),
                             cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *valid_host = v;
    return SVR_OK;
}

extern "C" int svr_workspace_query(int n_views, int N, int64_t capacity, int64_t total_pixels, int total_tiles,
                                   size_t* sizes_host)
{
    if (!sizes_host || n_views <= 0 || N < 0 || capacity < 0) return svr_fail(SVR_ERR_ARG, "workspace query");
    sizes_host[0] = geom_layout((int64_t)N * n_views).total;
    sizes_host[1] = bin_layout(capacity, total_tiles).total;
    sizes_host[2] = img_layout(total_pixels, total_tiles).total;
    return SVR_OK;
}

static int bin_and_sort_impl(const svr_view_t* views_host, int n_views, int N, int64_t R, uint64_t path_or,
                             const int64_t* octpaths, const uint32_t* rank_table, int rank_table_bits,
                             void* geom_buffer, void* binning_buffer, size_t binning_bytes, void* image_buffer,
                             void* stream)
{
    Views V;
    int T; int64_t P;
    int rc = build_views(views_host, n_views, V, T, P);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t M = (int64_t)N * n_views;
    GeomLayout GL = geom_layout(M);
    BinLayout BL = bin_layout(R, T);
    ImgLayout IL = img_layout(P, T);
    if (binning_bytes < BL.total) return svr_fail(SVR_ERR_CAPACITY, "binning buffer too small");
    char* g = (char*)geom_buffer;
    char* b = (char*)binning_buffer;
    char* im = (char*)image_buffer;
    unsigned* status = (unsigned*)(im + IL.status);
    CUDA_TRY(cudaMemsetAsync(im + IL.ranges, 0, 8 * (size_t)T, st));
    CUDA_TRY(cudaMemsetAsync(status, 0, 4, st));
    // new records: no forward has written their candidate rows yet
    CUDA_TRY(cudaMemsetAsync(b + offsetof(BinMeta, cand_ok), 0, sizeof(int), st));
    if (R == 0) return tile_launch_order(T, im, IL, st);
    KeyFmt kf = key_format(path_or, T);
    if (rank_table) {
        if (rank_table_bits < 1 || rank_table_bits > 32) return svr_fail(SVR_ERR_ARG, "rank table bits");
        kf.key_bits = kf.key_bits - kf.rank_bits + rank_table_bits;
        kf.rank_bits = rank_table_bits;
    }
    if (kf.key_bits > 64) return svr_fail(SVR_ERR_UNSUPPORTED, "sort key wider than 64 bits");
    rc = kf.key_bits <= 32
             ? bin_sort_typed<uint32_t>(V, N, R, kf, T, octpaths, g, GL, b, BL, im, IL, status, st, rank_table)
             : bin_sort_typed<uint64_t>(V, N, R, kf, T, octpaths, g, GL, b, BL, im, IL, status, st, rank_table);
    if (rc) return rc;
    return tile_launch_order(T, im, IL, st);
}

extern "C" int svr_bin_and_sort(const svr_view_t* views_host, int n_views, int N, int64_t R, uint64_t path_or,
                                const int64_t* octpaths, void* geom_buffer, void* binning_buffer,
                                size_t binning_bytes, void* image_buffer, void* stream)
{
    return bin_and_sort_impl(views_host, n_views, N, R, path_or, octpaths, nullptr, 0, geom_buffer, binning_buffer,
                             binning_bytes, image_buffer, stream);
}

extern "C" int svr_bin_and_sort_ranked(const svr_view_t* views_host, int n_views, int N, int64_t R,
                                       uint64_t path_or, const int64_t* octpaths, const uint32_t* rank_table,
                                       int rank_table_bits, void* geom_buffer, void* binning_buffer,
                                       size_t binning_bytes, void* image_buffer, void* stream)
{
    if (!rank_table) return svr_fail(SVR_ERR_ARG, "rank table");
    return bin_and_sort_impl(views_host, n_views, N, R, path_or, octpaths, rank_table, rank_table_bits, geom_buffer,
                             binning_buffer, binning_bytes, image_buffer, stream);
}

// ------------------------------------------------------------------ tile binning
// Per step: count, scan, scatter and per-tile sort of the batch's records (tile_sort.cuh).
// R is the record capacity of the binning buffer; the device bins min(total, R) records.
extern "C" int svr_bin_tiles(const svr_view_t* views_host, int n_views, int N, int64_t R, const uint32_t* pair_pos,
                             int key_bits, void* geom_buffer, void* binning_buffer, size_t binning_bytes,
                             void* image_buffer, void* stream)
{
    Views V;
    int T; int64_t P;
    int rc = build_views(views_host, n_views, V, T, P);
    if (rc) return rc;
    if (N < 0 || (N > 0 && (!pair_pos || !geom_buffer || !binning_buffer || !image_buffer)))
        return svr_fail(SVR_ERR_ARG, "bin_tiles: null argument");
    if (key_bits < 1 || key_bits > 32) return svr_fail(SVR_ERR_ARG, "bin_tiles: key bits");
    if (R >= (1ll << 32)) return svr_fail(SVR_ERR_CAPACITY, "bin_tiles: capacity above 2^32 records");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t M = (int64_t)N * n_views;
    GeomLayout GL = geom_layout(M);
    BinLayout BL = bin_layout(R, T);
    ImgLayout IL = img_layout(P, T);
    if (binning_bytes < BL.total) return svr_fail(SVR_ERR_CAPACITY, "binning buffer too small");
    char* g = (char*)geom_buffer;
    char* b = (char*)binning_buffer;
    char* im = (char*)image_buffer;
    unsigned* status = (unsigned*)(im + IL.status);
    BinMeta* meta = (BinMeta*)b;
    uint32_t* tile_cnt = (uint32_t*)(im + IL.tile_cnt);
    uint32_t* cursor = (uint32_t*)(im + IL.cursor);
    CUDA_TRY(cudaMemsetAsync(status, 0, 4, st));
    CUDA_TRY(cudaMemsetAsync(b + offsetof(BinMeta, cand_ok), 0, sizeof(int), st));   // new records
    CUDA_TRY(cudaMemsetAsync(tile_cnt, 0, 4 * (size_t)T, st));
    const uint32_t* ndup = (const uint32_t*)(g + GL.ndup);
    const uint2* bbox = (const uint2*)(g + GL.bbox);
    const uint32_t* bits = (const uint32_t*)(g + GL.bits);
    // per-view histograms in shared memory when the largest view's tiles fit in 96 KB
    int max_nt = 0;
    for (int v = 0; v < n_views; ++v) max_nt = std::max(max_nt, V.v[v].tiles_x * V.v[v].tiles_y);
    constexpr int MAX_HIST_TILES = 24576;     // 96 KB of shared memory
    const bool smem_hist = max_nt <= MAX_HIST_TILES;
    const int hist_bytes = smem_hist ? 4 * max_nt : 0;
    // about 8 CTAs per SM in all, split over the views (as preprocess)
    const int per_view = std::max(1, std::min((N + 255) / 256, (8 * 148 + n_views - 1) / n_views));
    dim3 grid(per_view, n_views);
    // the count kernel's per-CTA histograms [per_view, T] go to the radix path's unsorted values
    // (4R bytes, unused here) when they fit, and the scatter reads them instead of recounting
    uint32_t* chist = (smem_hist && R > 0 && (int64_t)per_view * T <= R) ? (uint32_t*)(b + BL.vals_in) : nullptr;
    if (N > 0) {
        if (smem_hist) {
            static std::atomic<unsigned long long> d1{0}, d2{0};
            // the limit is raised once per device, to the largest histogram this path uses
            if ((rc = ensure_smem(tile_count_kernel<true>, 4 * MAX_HIST_TILES, d1))) return rc;
            if ((rc = ensure_smem(tile_scatter_kernel<true>, 4 * MAX_HIST_TILES, d2))) return rc;
            tile_count_kernel<true><<<grid, 256, hist_bytes, st>>>(V, N, ndup, bbox, bits, tile_cnt, chist, T);
        } else {
            tile_count_kernel<false><<<grid, 256, 0, st>>>(V, N, ndup, bbox, bits, tile_cnt, nullptr, T);
        }
        LAUNCH_CHECK();
    }
    const int nblk = (T + TS_BLK - 1) / TS_BLK;
    tile_sum_kernel<<<nblk, 256, 0, st>>>(T, tile_cnt, (uint32_t*)(im + IL.blk_sum), (uint32_t*)(im + IL.blk_hist));
    LAUNCH_CHECK();
    tile_offsets_kernel<<<nblk, 256, 0, st>>>(T, nblk, tile_cnt, (const uint32_t*)(im + IL.blk_sum),
                                              (const uint32_t*)(im + IL.blk_hist), R, (uint2*)(im + IL.ranges), cursor,
                                              (uint32_t*)(im + IL.order), &meta->count, &meta->rank_bits, status);
    LAUNCH_CHECK();
    if (N == 0 || R == 0) return SVR_OK;
    // (key, value) pairs: A in keys_in, B (large tiles' passes) in pairs_b; results: vals_out
    // and the tile id of every record in keys_out (read by the record packing)
    uint2* pa = (uint2*)(b + BL.keys_in);
    uint2* pb = (uint2*)(b + BL.pairs_b);
    uint32_t* tile_out = (uint32_t*)(b + BL.keys_out);
    if (smem_hist)
        tile_scatter_kernel<true><<<grid, 256, hist_bytes, st>>>(V, N, ndup, bbox, bits, pair_pos, cursor, R, pa,
                                                                 chist, T, status);
    else
        tile_scatter_kernel<false><<<grid, 256, 0, st>>>(V, N, ndup, bbox, bits, pair_pos, cursor, R, pa, nullptr,
                                                         T, status);
    LAUNCH_CHECK();
    static std::atomic<unsigned long long> d3{0};
    const int ts_smem = (int)sizeof(TileSortSmem);
    if ((rc = ensure_smem(tile_sort_kernel, ts_smem, d3))) return rc;
    tile_sort_kernel<<<T, TS_THREADS, ts_smem, st>>>(T, (const uint32_t*)(im + IL.order),
                                                      (const uint2*)(im + IL.ranges), key_bits, pa, pb,
                                                      (uint32_t*)(b + BL.vals_out), tile_out, status);
    LAUNCH_CHECK();
    return SVR_OK;
}

// ------------------------------------------------------------------ dense rank table
// Once per octree and trimming: the trimmed rank (path ^ rep3(q)) >> shift of every (voxel,
// octant) pair, sorted; equal ranks share one dense index, so the dense index orders and ties
// exactly as the rank does and the binning key narrows from 3 * MAX_LEVELS - shift bits to
// the bits of the number of distinct ranks.
struct RankWs { size_t keys_in, keys_out, vals_in, vals_out, flags, tmp, tmp_bytes, total; };
static int rank_ws(int64_t n8, RankWs& w)
{
    const int n = (int)(n8 > 0 ? n8 : 1);
    size_t ts = 0, tc = 0;
    if (cub::DeviceRadixSort::SortPairs(nullptr, ts, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                        (const uint32_t*)nullptr, (uint32_t*)nullptr, n) != cudaSuccess ||
        cub::DeviceScan::InclusiveSum(nullptr, tc, (const uint32_t*)nullptr, (uint32_t*)nullptr, n) != cudaSuccess)
        return svr_fail(SVR_ERR_CUDA, "rank table: size query");
    size_t off = 0;
    w.keys_in = off; off = align_up(off + 8 * (size_t)n, 256);
    w.keys_out = off; off = align_up(off + 8 * (size_t)n, 256);
    w.vals_in = off; off = align_up(off + 4 * (size_t)n, 256);
    w.vals_out = off; off = align_up(off + 4 * (size_t)n, 256);
    w.flags = off; off = align_up(off + 4 * (size_t)n, 256);
    w.tmp = off; w.tmp_bytes = ts > tc ? ts : tc; off = align_up(off + w.tmp_bytes, 256);
    w.total = off;
    return SVR_OK;
}

extern "C" int svr_rank_table_workspace_bytes(int64_t N, size_t* bytes)
{
    if (!bytes || N < 0 || 8 * N >= (1ll << 31)) return svr_fail(SVR_ERR_ARG, "rank table: N");
    RankWs w;
    if (int rc = rank_ws(8 * N, w)) return rc;
    *bytes = w.total;
    return SVR_OK;
}

__global__ void rank_key_kernel(int64_t N, const int64_t* __restrict__ octpaths, int shift, uint64_t* __restrict__ keys,
                                uint32_t* __restrict__ vals)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 8 * N) return;
    const uint32_t q = (uint32_t)(s & 7);
    keys[s] = ((uint64_t)octpaths[s >> 3] ^ rep3(q)) >> shift;
    vals[s] = (uint32_t)s;
}

__global__ void rank_flag_kernel(int64_t n, const uint64_t* __restrict__ keys, uint32_t* __restrict__ flags)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void rank_scatter_kernel(int64_t n, const uint32_t* __restrict__ vals, const uint32_t* __restrict__ incl,
                                    uint32_t* __restrict__ table)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    table[vals[i]] = incl[i] - 1u;
}

extern "C" int svr_rank_table_build(int64_t N, const int64_t* octpaths, uint64_t path_or, uint32_t* table,
                                    int* rank_bits_host, void* ws, size_t ws_bytes, void* stream)
{
    size_t need = 0;
    if (int rc = svr_rank_table_workspace_bytes(N, &need)) return rc;
    if (N <= 0 || !octpaths || !table || !rank_bits_host || !ws || ws_bytes < need)
        return svr_fail(SVR_ERR_ARG, "rank table: bad argument or workspace too small");
    RankWs w;
    if (int rc = rank_ws(8 * N, w)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    char* base = (char*)ws;
    uint64_t* kin = (uint64_t*)(base + w.keys_in);
    uint64_t* kout = (uint64_t*)(base + w.keys_out);
    uint32_t* vin = (uint32_t*)(base + w.vals_in);
    uint32_t* vout = (uint32_t*)(base + w.vals_out);
    uint32_t* flags = (uint32_t*)(base + w.flags);
    const KeyFmt kf = key_format(path_or, 1);
    const int64_t n = 8 * N;
    const unsigned nb = (unsigned)((n + 255) / 256);
    rank_key_kernel<<<nb, 256, 0, st>>>(N, octpaths, kf.rank_shift, kin, vin);
    LAUNCH_CHECK();
    size_t tb = w.tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(base + w.tmp, tb, kin, kout, vin, vout, (int)n, 0, kf.rank_bits, st));
    rank_flag_kernel<<<nb, 256, 0, st>>>(n, kout, flags);
    LAUNCH_CHECK();
    tb = w.tmp_bytes;
    CUDA_TRY(cub::DeviceScan::InclusiveSum(base + w.tmp, tb, flags, flags, (int)n, st));
    rank_scatter_kernel<<<nb, 256, 0, st>>>(n, vout, flags, table);
    LAUNCH_CHECK();
    uint32_t n_unique = 0;
    CUDA_TRY(cudaMemcpyAsync(&n_unique, flags + (n - 1), 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    int bits = 1;
    while (bits < 32 && (1ull << bits) < (unsigned long long)n_unique) ++bits;
    *rank_bits_host = bits;
    return SVR_OK;
}

extern "C" int svr_pair_order_build(int64_t N, const int64_t* octpaths, uint32_t* pair_pos, int* key_bits_host,
                                    void* ws, size_t ws_bytes, void* stream)
{
    size_t need = 0;
    if (int rc = svr_rank_table_workspace_bytes(N, &need)) return rc;
    if (N <= 0 || !octpaths || !pair_pos || !key_bits_host || !ws || ws_bytes < need)
        return svr_fail(SVR_ERR_ARG, "pair order: bad argument or workspace too small");
    RankWs w;
    if (int rc = rank_ws(8 * N, w)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    char* base = (char*)ws;
    uint64_t* kin = (uint64_t*)(base + w.keys_in);
    uint64_t* kout = (uint64_t*)(base + w.keys_out);
    uint32_t* vin = (uint32_t*)(base + w.vals_in);
    uint32_t* vout = (uint32_t*)(base + w.vals_out);
    const int64_t n = 8 * N;
    const unsigned nb = (unsigned)((n + 255) / 256);
    pair_rank_kernel<<<nb, 256, 0, st>>>(N, octpaths, kin, vin);
    LAUNCH_CHECK();
    size_t tb = w.tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(base + w.tmp, tb, kin, kout, vin, vout, (int)n, 0, RANK_BITS, st));
    pair_pos_kernel<<<nb, 256, 0, st>>>(N, vout, pair_pos);
    LAUNCH_CHECK();
    int bits = 1;
    while (bits < 32 && (1ll << bits) < n) ++bits;
    *key_bits_host = bits;
    return SVR_OK;
}

extern "C" int svr_unpack_binning(const void* binning_buffer, int64_t R, int T, const void* image_buffer,
                                  int64_t P, uint32_t* vals, uint32_t* ranges, uint32_t* tile_last,
                                  uint32_t* n_contrib, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    BinLayout BL = bin_layout(R, T);
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
// Centre and edge length of every voxel as one float4 (x, y, z, length): record packing
// then gathers one 16-byte piece per record instead of four scalars from two arrays (the
// gathers miss L2 on large batches, so this is one DRAM sector per record instead of two
// or three).  Written into the unsorted-key region of the binning buffer, which is dead
// once the records are sorted.
__global__ void center_len_kernel(int N, const float* __restrict__ centers, const float* __restrict__ lengths,
                                  float4* __restrict__ center_len)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) center_len[i] = make_float4(centers[3 * (size_t)i], centers[3 * (size_t)i + 1],
                                           centers[3 * (size_t)i + 2], lengths[i]);
}

// Per-voxel block of the record packing's gathers: centre and size, then the 8 corner SDF
// values, in one 64-byte-aligned block (one DRAM burst per gathered voxel instead of two).
struct __align__(64) VoxBlock {
    float4 cl, g0, g1, pad;
};
__global__ void vox_block_kernel(int N, const float* __restrict__ centers, const float* __restrict__ lengths,
                                 const float4* __restrict__ geos, VoxBlock* __restrict__ blocks)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    VoxBlock v;
    v.cl = make_float4(centers[3 * (size_t)i], centers[3 * (size_t)i + 1], centers[3 * (size_t)i + 2], lengths[i]);
    v.g0 = geos[2 * (size_t)i];
    v.g1 = geos[2 * (size_t)i + 1];
    v.pad = make_float4(0.f, 0.f, 0.f, 0.f);
    blocks[i] = v;
}

// Gather each sorted record's voxel data into one 80-byte record.  The record's view is
// the view of its tile, read from the sorted key.  The voxel's centre, size and corner values
// come from `blocks` when given, else from center_len (when given) or the plain arrays and
// geos.
__global__ void __launch_bounds__(256) pack_records_kernel(
    const __grid_constant__ Views V, int N, int64_t R, const BinMeta* __restrict__ meta,
    const void* __restrict__ keys, const uint32_t* __restrict__ vals, const uint2* __restrict__ bboxes,
    const float* __restrict__ centers, const float* __restrict__ lengths, const float4* __restrict__ geos,
    const float* __restrict__ rgbs, int rgb_per_view, const float4* __restrict__ center_len,
    const VoxBlock* __restrict__ blocks, Rec* __restrict__ recs, unsigned* status)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= R || k >= meta->count) return;
    const int rank_bits = meta->rank_bits;
    const uint64_t key = meta->key64 ? ((const uint64_t*)keys)[k] : (uint64_t)((const uint32_t*)keys)[k];
    const int vi = V.n == 1 ? 0 : view_of_tile(V, (int)(key >> rank_bits));
    const uint32_t val = vals[k];
    const uint32_t vid = val & 0x1FFFFFFFu;
    if (vid >= (uint32_t)N) { atomicOr(status, ERR_BAD_INDEX); return; }
    Rec r;
    float4 g0, g1;
    if (blocks) {
        const float4 c = blocks[vid].cl;
        r.cx = c.x; r.cy = c.y; r.cz = c.z; r.len = c.w;
        g0 = blocks[vid].g0;
        g1 = blocks[vid].g1;
    } else {
        if (center_len) {
            const float4 c = center_len[vid];
            r.cx = c.x; r.cy = c.y; r.cz = c.z; r.len = c.w;
        } else {
            r.cx = centers[3 * (size_t)vid]; r.cy = centers[3 * (size_t)vid + 1];
            r.cz = centers[3 * (size_t)vid + 2];
            r.len = lengths[vid];
        }
        g0 = geos[2 * (size_t)vid];
        g1 = geos[2 * (size_t)vid + 1];
    }
    r.g[0] = g0.x; r.g[1] = g0.y; r.g[2] = g0.z; r.g[3] = g0.w;
    r.g[4] = g1.x; r.g[5] = g1.y; r.g[6] = g1.z; r.g[7] = g1.w;
    const size_t cb = 3 * ((rgb_per_view ? (size_t)vi * N : 0) + vid);
    r.r = rgbs[cb]; r.gr = rgbs[cb + 1]; r.b = rgbs[cb + 2];
    const uint2 bb = bboxes[(size_t)vi * N + vid];
    r.bbox0 = bb.x; r.bbox1 = bb.y;
    r.val = val;
    // corner bounds for the render filter's dead-record test (record_dead, render_pairs.cuh):
    // min / max corner widened by 5% of the spread plus 1e-4 of the largest magnitude
    {
        const float lo = fminf(fminf(fminf(g0.x, g0.y), fminf(g0.z, g0.w)), fminf(fminf(g1.x, g1.y), fminf(g1.z, g1.w)));
        const float hi = fmaxf(fmaxf(fmaxf(g0.x, g0.y), fmaxf(g0.z, g0.w)), fmaxf(fmaxf(g1.x, g1.y), fmaxf(g1.z, g1.w)));
        const float margin = __fadd_rn(__fmul_rn(0.05f, __fsub_rn(hi, lo)), __fmul_rn(1e-4f, fmaxf(fabsf(lo), fabsf(hi))));
        r.sdf_lo = __fsub_rn(lo, margin);
        r.sdf_hi = __fadd_rn(hi, margin);
    }
    const float4* src = reinterpret_cast<const float4*>(&r);
    float4* dst = reinterpret_cast<float4*>(recs + k);
#pragma unroll
    for (int q = 0; q < 5; ++q) dst[q] = src[q];
}

// ------------------------------------------------------------------ render kernels
#include "render_kernels.cuh"
#include "render_pairs.cuh"

// Which render kernels the launches use: 0 = the warp-filter kernels (render_fwd_kernel /
// render_bwd_kernel), 1 = record-parallel filter with dense pair evaluation
// (render_fwd_pairs_kernel / render_bwd_pairs_kernel) with warps on 8x4 pixel blocks, 2 = the
// same with every warp on a lattice spread over the tile, 3 (the default) = the same with the
// pairs of a slot numbered and evaluated over the whole CTA.  All give the same forward outputs
// bit for bit and the same gradients up to the order of their float atomics.
static std::atomic<int> g_fwd_impl{3}, g_bwd_impl{3};
static std::atomic<int> g_fwd_cfg{0}, g_bwd_cfg{0};   // launch variant (kFwdCfgs / kBwdCfgs)
extern "C" int svr_render_set_impl(int fwd_impl, int bwd_impl)
{
    if (fwd_impl < 0 || fwd_impl > 3 || bwd_impl < 0 || bwd_impl > 3) return svr_fail(SVR_ERR_ARG, "render impl");
    g_fwd_impl.store(fwd_impl);
    g_bwd_impl.store(bwd_impl);
    g_fwd_cfg.store(0);            // the family's default configuration
    g_bwd_cfg.store(0);
    return SVR_OK;
}
extern "C" int svr_render_get_impl(int* fwd_impl, int* bwd_impl)
{
    if (fwd_impl) *fwd_impl = g_fwd_impl.load();
    if (bwd_impl) *bwd_impl = g_bwd_impl.load();
    return SVR_OK;
}

// Stage timing: an event recorded by svr_render_fwd on its stream between the record packing
// launch and the render launch (null = none).
static std::atomic<cudaEvent_t> g_pack_event{nullptr};
extern "C" int svr_set_pack_event(void* event)
{
    g_pack_event.store((cudaEvent_t)event);
    return SVR_OK;
}

#ifndef SVR_PBWD_RING
#define SVR_PBWD_RING 3
#endif
#ifndef SVR_PBWD_MINB
#define SVR_PBWD_MINB 3
#endif
template <bool DEPTH, bool NORMAL, bool RCONC, bool LATTICE = true, bool CTAW = false, int RING = SVR_PBWD_RING,
          int MINB = SVR_PBWD_MINB>
static int launch_bwd_pairs(int T, int N, cudaStream_t st, const Views& V, const uint32_t* order, const uint2* ranges,
                            const uint32_t* tl, const uint32_t* nc, const Rec* recs, const float* s_val,
                            const float* out_T, const float* dc, const float* dd, const float* dn, const float* dT,
                            float lam, const float* gt, float* dvox, float* drgbs, float* ds, unsigned* status,
                            const uint4* cand, const int* cand_ok)
{
    auto k = render_bwd_pairs_kernel<DEPTH, NORMAL, RCONC, RING, MINB, LATTICE, CTAW>;
    const int smem = (int)sizeof(PairBwdSmem<RING>);
    static std::atomic<unsigned long long> done{0};
    int rc = ensure_smem(k, smem, done);
    if (rc) return rc;
    k<<<T, BLOCK, smem, st>>>(V, N, order, ranges, tl, nc, recs, s_val, out_T, dc, dd, dn, dT, lam, gt, dvox, drgbs, ds,
                               status, CTAW ? cand : nullptr, cand_ok);
    LAUNCH_CHECK();
    return SVR_OK;
}

// Set by the forward launchers: whether the kernel just launched writes the candidate rows.
static thread_local bool t_cand_written = false;

#ifndef SVR_PFWD_RING
#define SVR_PFWD_RING 3
#endif
#ifndef SVR_PFWD_MINB
#define SVR_PFWD_MINB 4
#endif
template <int NS, bool DEPTH, bool NORMAL, bool MAXW, bool COUNT, bool LATTICE = true, bool CTAW = false,
          int RING = SVR_PFWD_RING, int MINB = SVR_PFWD_MINB>
static int launch_fwd_pairs(int T, cudaStream_t st, const Views& V, const uint32_t* order, const uint2* ranges,
                            const Rec* recs, const float* s_val, uint32_t* tile_last, uint32_t* n_contrib,
                            float* color, float* depth, float* normal, float* outT, float* max_w, int64_t mw_stride,
                            unsigned* status, unsigned long long* pair_count, uint4* cand)
{
    auto k = render_fwd_pairs_kernel<NS, DEPTH, NORMAL, MAXW, RING, MINB, COUNT, LATTICE, CTAW>;
    const int smem = (int)sizeof(PairFwdSmem<RING>);
    static std::atomic<unsigned long long> done{0};
    int rc = ensure_smem(k, smem, done);
    if (rc) return rc;
    if (!CTAW) cand = nullptr;
    k<<<T, BLOCK, smem, st>>>(V, order, ranges, recs, s_val, tile_last, n_contrib, color, depth, normal, outT, max_w,
                              mw_stride, status, pair_count, cand);
    LAUNCH_CHECK();
    t_cand_written = cand != nullptr;
    return SVR_OK;
}

// Launch variants (kernel family, ring slots, CTAs per SM) the tuner chooses between for the
// common flag sets (three sub-samples, depth and normal on; with or without the
// R-concentration term).  Index 0 = the family selected by svr_render_set_impl (default 3) in
// its default configuration; the others name their family.  The choice is process-wide and
// read when a launch is issued (so a captured graph keeps the one in force then).
struct RenderCfg { int impl, ring, minb; };
static const RenderCfg kFwdCfgs[] = {{3, SVR_PFWD_RING, SVR_PFWD_MINB}, {3, 3, 3}, {3, 4, 3},
                                     {2, SVR_PFWD_RING, SVR_PFWD_MINB}, {0, SVR_NSLOT, SVR_FWD_MINB}, {0, 4, 3}};
static const RenderCfg kBwdCfgs[] = {{3, SVR_PBWD_RING, SVR_PBWD_MINB}, {3, 3, 2}, {3, 4, 2},
                                     {2, SVR_PBWD_RING, SVR_PBWD_MINB}, {0, SVR_BWD_NSLOT, SVR_BWD_MINB}, {0, 4, 2}};
constexpr int N_FWD_CFGS = 6, N_BWD_CFGS = 6;
// The per-warp filter kernels' default configuration follows the launch size.  Launches of a
// few thousand tiles are bound by their heaviest tiles and run best with more registers per
// thread; measured with the tuner on the mid-size scene (800x800 views, 2500 tiles each):
//   1 view  : forward 4x3 0.954 ms (4x4 1.006); adjoint 4x2 1.085 ms (4x3 1.185, 3x4 1.30)
//   2 views : forward 4x3 1.089 ms (4x4 1.163); adjoint 4x2 1.139 ms (4x3 1.287)
//   4 views : forward 4x4 1.382 ms;             adjoint 4x3 1.466 ms (3x4 1.664)
//   8 views : forward 4x4 2.47 ms;              adjoint 3x4 3.02 ms (4x3 3.12)
constexpr int SMALL_LAUNCH_TILES = 8192;    // below: forward 4x3, adjoint 4x2
constexpr int MEDIUM_LAUNCH_TILES = 16384;  // below: adjoint 4x3

extern "C" int svr_render_config_count(int* n_fwd, int* n_bwd)
{
    if (n_fwd) *n_fwd = N_FWD_CFGS;
    if (n_bwd) *n_bwd = N_BWD_CFGS;
    return SVR_OK;
}

extern "C" int svr_render_config_describe(int pass, int index, int* impl, int* ring, int* ctas_per_sm)
{
    const int n = pass == 0 ? N_FWD_CFGS : N_BWD_CFGS;
    if (index < 0 || index >= n) return svr_fail(SVR_ERR_ARG, "render config index");
    const RenderCfg c = pass == 0 ? kFwdCfgs[index] : kBwdCfgs[index];
    if (impl) *impl = c.impl;
    if (ring) *ring = c.ring;
    if (ctas_per_sm) *ctas_per_sm = c.minb;
    return SVR_OK;
}

extern "C" int svr_render_set_config(int fwd_index, int bwd_index)
{
    if (fwd_index < 0 || fwd_index >= N_FWD_CFGS || bwd_index < 0 || bwd_index >= N_BWD_CFGS)
        return svr_fail(SVR_ERR_ARG, "render config index");
    g_fwd_cfg.store(fwd_index);
    g_bwd_cfg.store(bwd_index);
    return SVR_OK;
}

extern "C" int svr_render_get_config(int* fwd_index, int* bwd_index)
{
    if (fwd_index) *fwd_index = g_fwd_cfg.load();
    if (bwd_index) *bwd_index = g_bwd_cfg.load();
    return SVR_OK;
}

template <int NS, bool DEPTH, bool NORMAL, bool MAXW, int RING, int MINB>
static int launch_fwd_cfg(int T, cudaStream_t st, const Views& V, const uint32_t* order, const uint2* ranges,
                          const Rec* recs, const float* s_val, uint32_t* tile_last, uint32_t* n_contrib,
                          float* color, float* depth, float* normal, float* outT, float* max_w, int64_t mw_stride,
                          unsigned* status)
{
    auto k = render_fwd_kernel<NS, DEPTH, NORMAL, MAXW, RING, MINB>;
    const int smem = (int)sizeof(FwdSmem<RING>);
    static std::atomic<unsigned long long> done{0};
    int rc = ensure_smem(k, smem, done);
    if (rc) return rc;
    k<<<T, BLOCK, smem, st>>>(V, order, ranges, recs, s_val, tile_last, n_contrib, color,
                              depth, normal, outT, max_w, mw_stride, status, nullptr);
    LAUNCH_CHECK();
    t_cand_written = false;
    return SVR_OK;
}

template <int NS, bool DEPTH, bool NORMAL, bool MAXW>
static int launch_fwd(int T, cudaStream_t st, const Views& V, const uint32_t* order, const uint2* ranges,
                      const Rec* recs,
                      const float* s_val, uint32_t* tile_last, uint32_t* n_contrib, float* color, float* depth,
                      float* normal, float* outT, float* max_w, int64_t mw_stride, unsigned* status, uint4* cand)
{
#define FWD_PAIR_ARGS T, st, V, order, ranges, recs, s_val, tile_last, n_contrib, color, depth, normal, outT, max_w, mw_stride, status, nullptr, cand
#define FWD_CFG_ARGS T, st, V, order, ranges, recs, s_val, tile_last, n_contrib, color, depth, normal, outT, max_w, mw_stride, status
    if constexpr (NS == 3 && DEPTH && NORMAL && !MAXW) {
        switch (g_fwd_cfg.load()) {       // kFwdCfgs
            case 1: return launch_fwd_pairs<NS, DEPTH, NORMAL, MAXW, false, true, true, 3, 3>(FWD_PAIR_ARGS);
            case 2: return launch_fwd_pairs<NS, DEPTH, NORMAL, MAXW, false, true, true, 4, 3>(FWD_PAIR_ARGS);
            case 3: return launch_fwd_pairs<NS, DEPTH, NORMAL, MAXW, false, true, false>(FWD_PAIR_ARGS);
            case 4: return launch_fwd_cfg<NS, DEPTH, NORMAL, MAXW, SVR_NSLOT, SVR_FWD_MINB>(FWD_CFG_ARGS);
            case 5: return launch_fwd_cfg<NS, DEPTH, NORMAL, MAXW, 4, 3>(FWD_CFG_ARGS);
            default: break;
        }
    }
    const int impl = g_fwd_impl.load();
    if (impl == 1) return launch_fwd_pairs<NS, DEPTH, NORMAL, MAXW, false, false>(FWD_PAIR_ARGS);
    if (impl == 2) return launch_fwd_pairs<NS, DEPTH, NORMAL, MAXW, false, true>(FWD_PAIR_ARGS);
    if (impl == 3) return launch_fwd_pairs<NS, DEPTH, NORMAL, MAXW, false, true, true>(FWD_PAIR_ARGS);
    if constexpr (NS == 3 && DEPTH && NORMAL && !MAXW) {
        if (T < SMALL_LAUNCH_TILES) return launch_fwd_cfg<NS, DEPTH, NORMAL, MAXW, 4, 3>(FWD_CFG_ARGS);
    }
    return launch_fwd_cfg<NS, DEPTH, NORMAL, MAXW, SVR_NSLOT, SVR_FWD_MINB>(FWD_CFG_ARGS);
#undef FWD_CFG_ARGS
#undef FWD_PAIR_ARGS
}

static int render_fwd_impl(const svr_view_t* views_host, int n_views, int N, int64_t R, int n_samp,
                           int need_depth, int need_normal, const float* centers, const float* lengths,
                           const float* geos, const float* rgbs, int n_rgb_views, const float* s_val,
                           void* geom_buffer, void* binning_buffer, void* image_buffer, float* out_color,
                           float* out_depth, float* out_normal, float* out_T, float* max_w, int64_t mw_stride,
                           void* stream);

extern "C" int svr_render_fwd(const svr_view_t* views_host, int n_views, int N, int64_t R, int n_samp,
                              int need_depth, int need_normal, const float* centers, const float* lengths,
                              const float* geos, const float* rgbs, int n_rgb_views, const float* s_val,
                              void* geom_buffer, void* binning_buffer, void* image_buffer, float* out_color,
                              float* out_depth, float* out_normal, float* out_T, float* max_w, void* stream)
{
    return render_fwd_impl(views_host, n_views, N, R, n_samp, need_depth, need_normal, centers, lengths, geos, rgbs,
                           n_rgb_views, s_val, geom_buffer, binning_buffer, image_buffer, out_color, out_depth,
                           out_normal, out_T, max_w, 0, stream);
}

extern "C" int svr_render_fwd_max_w_views(const svr_view_t* views_host, int n_views, int N, int64_t R, int n_samp,
                                          int need_depth, int need_normal, const float* centers,
                                          const float* lengths, const float* geos, const float* rgbs,
                                          int n_rgb_views, const float* s_val, void* geom_buffer,
                                          void* binning_buffer, void* image_buffer, float* out_color,
                                          float* out_depth, float* out_normal, float* out_T,
                                          float* max_w_views, void* stream)
{
    if (!max_w_views) return svr_fail(SVR_ERR_ARG, "render_fwd_max_w_views: null max_w");
    return render_fwd_impl(views_host, n_views, N, R, n_samp, need_depth, need_normal, centers, lengths, geos, rgbs,
                           n_rgb_views, s_val, geom_buffer, binning_buffer, image_buffer, out_color, out_depth,
                           out_normal, out_T, max_w_views, (int64_t)N, stream);
}

static int render_fwd_impl(const svr_view_t* views_host, int n_views, int N, int64_t R, int n_samp,
                           int need_depth, int need_normal, const float* centers, const float* lengths,
                           const float* geos, const float* rgbs, int n_rgb_views, const float* s_val,
                           void* geom_buffer, void* binning_buffer, void* image_buffer, float* out_color,
                           float* out_depth, float* out_normal, float* out_T, float* max_w, int64_t mw_stride,
                           void* stream)
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
    BinLayout BL = bin_layout(R, T);
    ImgLayout IL = img_layout(P, T);
    char* g = (char*)geom_buffer;
    char* b = (char*)binning_buffer;
    char* im = (char*)image_buffer;
    unsigned* status = (unsigned*)(im + IL.status);
    const uint2* ranges = (const uint2*)(im + IL.ranges);
    const uint32_t* order = (const uint32_t*)(im + IL.order);
    Rec* recs = (Rec*)(b + BL.recs);
    if (R > 0) {
        // the sort's scratch pairs (8 bytes per record slot, free once sorted) hold the N
        // 64-byte voxel blocks when R >= 8N, else the unsorted keys hold N float4 of centre and
        // size when R >= 2N
        float4* cl = nullptr;
        VoxBlock* vb = nullptr;
        if (N > 0 && R >= 8 * (int64_t)N) {
            vb = (VoxBlock*)(b + BL.pairs_b);
            vox_block_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(N, centers, lengths, (const float4*)geos,
                                                                          vb);
            LAUNCH_CHECK();
        } else if (N > 0 && R >= 2 * (int64_t)N) {
            cl = (float4*)(b + BL.keys_in);
            center_len_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(N, centers, lengths, cl);
            LAUNCH_CHECK();
        }
        pack_records_kernel<<<(unsigned)((R + 255) / 256), 256, 0, st>>>(
            V, N, R, (const BinMeta*)b, b + BL.keys_out, (const uint32_t*)(b + BL.vals_out),
            (const uint2*)(g + GL.bbox), centers, lengths, (const float4*)geos, rgbs, n_rgb_views > 1, cl, vb, recs,
            status);
        LAUNCH_CHECK();
    }
    if (cudaEvent_t ev = g_pack_event.load()) {
        const cudaError_t e = cudaEventRecord(ev, st);
        if (e != cudaSuccess) return svr_fail(SVR_ERR_CUDA, cudaGetErrorString(e));
    }
    uint32_t* tl = (uint32_t*)(im + IL.tile_last);
    uint32_t* nc = (uint32_t*)(im + IL.n_contrib);
    const bool D = need_depth != 0, Nm = need_normal != 0, MW = max_w != nullptr;
#define FWD_CASE(NS_)                                                                                   \
    if (n_samp == NS_) {                                                                                \
        if (D && Nm && !MW) return launch_fwd<NS_, true, true, false>(T, st, V, order, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, mw_stride, status, cand); \
        if (D && Nm && MW) return launch_fwd<NS_, true, true, true>(T, st, V, order, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, mw_stride, status, cand); \
        if (D && !Nm && !MW) return launch_fwd<NS_, true, false, false>(T, st, V, order, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, mw_stride, status, cand); \
        if (D && !Nm && MW) return launch_fwd<NS_, true, false, true>(T, st, V, order, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, mw_stride, status, cand); \
        if (!D && Nm && !MW) return launch_fwd<NS_, false, true, false>(T, st, V, order, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, mw_stride, status, cand); \
        if (!D && Nm && MW) return launch_fwd<NS_, false, true, true>(T, st, V, order, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, mw_stride, status, cand); \
        if (!D && !Nm && !MW) return launch_fwd<NS_, false, false, false>(T, st, V, order, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, mw_stride, status, cand); \
        return launch_fwd<NS_, false, false, true>(T, st, V, order, ranges, recs, s_val, tl, nc, out_color, out_depth, out_normal, out_T, max_w, mw_stride, status, cand); \
    }
    uint4* cand = (uint4*)(b + BL.cand);
    t_cand_written = false;
    auto dispatch = [&]() -> int {
        FWD_CASE(1)
        FWD_CASE(2)
        FWD_CASE(3)
        return svr_fail(SVR_ERR_UNSUPPORTED, "n_samp");
    };
#undef FWD_CASE
    rc = dispatch();
    if (rc) return rc;
    // the adjoint may read the candidate rows only when this forward wrote them: it packed the
    // records they refer to
    CUDA_TRY(cudaMemsetAsync(b + offsetof(BinMeta, cand_ok), t_cand_written ? 1 : 0, 1, st));
    return SVR_OK;
}

// The pair-counting instance of the forward (three sub-samples, depth and normal on, the
// default launch configuration): the same outputs as svr_render_fwd plus the pair counts.
extern "C" int svr_render_fwd_count_pairs(const svr_view_t* views_host, int n_views, int N, int64_t R,
                                          const float* s_val, void* binning_buffer, void* image_buffer,
                                          float* out_color, float* out_depth, float* out_normal, float* out_T,
                                          unsigned long long* pair_count, void* stream)
{
    Views V;
    int T; int64_t P;
    int rc = build_views(views_host, n_views, V, T, P);
    if (rc) return rc;
    if (!out_color || !out_depth || !out_normal || !out_T || !s_val || !pair_count)
        return svr_fail(SVR_ERR_ARG, "render_fwd_count_pairs: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    BinLayout BL = bin_layout(R, T);
    ImgLayout IL = img_layout(P, T);
    char* b = (char*)binning_buffer;
    char* im = (char*)image_buffer;
    CUDA_TRY(cudaMemsetAsync(pair_count, 0, 3 * sizeof(unsigned long long), st));
    if (g_fwd_impl.load() >= 1)
        return launch_fwd_pairs<3, true, true, false, true>(T, st, V, (const uint32_t*)(im + IL.order),
                                                            (const uint2*)(im + IL.ranges), (const Rec*)(b + BL.recs),
                                                            s_val, (uint32_t*)(im + IL.tile_last),
                                                            (uint32_t*)(im + IL.n_contrib), out_color, out_depth,
                                                            out_normal, out_T, nullptr, 0,
                                                            (unsigned*)(im + IL.status), pair_count, nullptr);
    auto k = render_fwd_kernel<3, true, true, false, SVR_NSLOT, SVR_FWD_MINB, true>;
    const int smem = (int)sizeof(FwdSmem<SVR_NSLOT>);
    static std::atomic<unsigned long long> done{0};
    rc = ensure_smem(k, smem, done);
    if (rc) return rc;
    k<<<T, BLOCK, smem, st>>>(V, (const uint32_t*)(im + IL.order), (const uint2*)(im + IL.ranges),
                              (const Rec*)(b + BL.recs), s_val, (uint32_t*)(im + IL.tile_last),
                              (uint32_t*)(im + IL.n_contrib), out_color, out_depth, out_normal, out_T, nullptr, 0,
                              (unsigned*)(im + IL.status), pair_count);
    LAUNCH_CHECK();
    return SVR_OK;
}

template <bool DEPTH, bool NORMAL, bool RCONC, int RING, int MINB>
static int launch_bwd_cfg(int T, int N, cudaStream_t st, const Views& V, const uint32_t* order, const uint2* ranges,
                          const uint32_t* tl, const uint32_t* nc, const Rec* recs, const float* s_val,
                          const float* out_T, const float* dc, const float* dd, const float* dn, const float* dT,
                          float lam, const float* gt, float* dvox, float* drgbs, float* ds, unsigned* status,
                          const uint4*, const int*)
{
    auto k = render_bwd_kernel<DEPTH, NORMAL, RCONC, RING, MINB>;
    const int smem = (int)sizeof(BwdSmem<RING>);
    static std::atomic<unsigned long long> done{0};
    int rc = ensure_smem(k, smem, done);
    if (rc) return rc;
    k<<<T, BLOCK, smem, st>>>(V, N, order, ranges, tl, nc, recs, s_val, out_T, dc, dd, dn, dT, lam, gt, dvox, drgbs, ds,
                               status);
    LAUNCH_CHECK();
    return SVR_OK;
}

template <bool DEPTH, bool NORMAL, bool RCONC>
static int launch_bwd(int T, int N, cudaStream_t st, const Views& V, const uint32_t* order, const uint2* ranges,
                      const uint32_t* tl,
                      const uint32_t* nc, const Rec* recs, const float* s_val, const float* out_T,
                      const float* dc, const float* dd, const float* dn, const float* dT, float lam,
                      const float* gt, float* dvox, float* drgbs, float* ds, unsigned* status, const uint4* cand,
                      const int* cand_ok)
{
#define BWD_CFG_ARGS T, N, st, V, order, ranges, tl, nc, recs, s_val, out_T, dc, dd, dn, dT, lam, gt, dvox, drgbs, ds, status, cand, cand_ok
    if constexpr (DEPTH && NORMAL) {
        switch (g_bwd_cfg.load()) {       // kBwdCfgs
            case 1: return launch_bwd_pairs<DEPTH, NORMAL, RCONC, true, true, 3, 2>(BWD_CFG_ARGS);
            case 2: return launch_bwd_pairs<DEPTH, NORMAL, RCONC, true, true, 4, 2>(BWD_CFG_ARGS);
            case 3: return launch_bwd_pairs<DEPTH, NORMAL, RCONC, true, false>(BWD_CFG_ARGS);
            case 4: return launch_bwd_cfg<DEPTH, NORMAL, RCONC, SVR_BWD_NSLOT, SVR_BWD_MINB>(BWD_CFG_ARGS);
            case 5: return launch_bwd_cfg<DEPTH, NORMAL, RCONC, 4, 2>(BWD_CFG_ARGS);
            default: break;
        }
    }
    const int impl = g_bwd_impl.load();
    if (impl == 1) return launch_bwd_pairs<DEPTH, NORMAL, RCONC, false>(BWD_CFG_ARGS);
    if (impl == 2) return launch_bwd_pairs<DEPTH, NORMAL, RCONC, true>(BWD_CFG_ARGS);
    if (impl == 3) return launch_bwd_pairs<DEPTH, NORMAL, RCONC, true, true>(BWD_CFG_ARGS);
    if constexpr (DEPTH && NORMAL) {
        if (T < SMALL_LAUNCH_TILES) return launch_bwd_cfg<DEPTH, NORMAL, RCONC, 4, 2>(BWD_CFG_ARGS);
        if (T < MEDIUM_LAUNCH_TILES) return launch_bwd_cfg<DEPTH, NORMAL, RCONC, 4, 3>(BWD_CFG_ARGS);
    }
    return launch_bwd_cfg<DEPTH, NORMAL, RCONC, SVR_BWD_NSLOT, SVR_BWD_MINB>(BWD_CFG_ARGS);
#undef BWD_CFG_ARGS
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
    BinLayout BL = bin_layout(R, T);
    ImgLayout IL = img_layout(P, T);
    char* b = (char*)binning_buffer;
    char* im = (char*)image_buffer;
    unsigned* status = (unsigned*)(im + IL.status);
    const uint2* ranges = (const uint2*)(im + IL.ranges);
    const uint32_t* tl = (const uint32_t*)(im + IL.tile_last);
    const uint32_t* nc = (const uint32_t*)(im + IL.n_contrib);
    const Rec* recs = (const Rec*)(b + BL.recs);
    const bool D = need_depth != 0, Nm = need_normal != 0, RC = lambda_R_concen > 0;
    const uint4* cand = (const uint4*)(b + BL.cand);
    const int* cand_ok = (const int*)(b + offsetof(BinMeta, cand_ok));
#define BWD_ARGS T, N, st, V, (const uint32_t*)(im + IL.order), ranges, tl, nc, recs, s_val, out_T, dL_dcolor, dL_ddepth, dL_dnormal, dL_dT, lambda_R_concen, gt_color, dL_dvox, drgbs, dL_ds, status, cand, cand_ok
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
