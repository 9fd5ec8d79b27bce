// Dense-grid registration and the parent-child / sibling smoothness adjoints.
//
// valid table: cuda/src/utils.cu:190-252 registers every voxel's cells of the virtual dense
// grid through an atomic slot counter and sorts afterwards (src/utils/octree_utils.py:
// 293-314).  Here the slots come from a prefix sum of per-voxel cell counts (deterministic,
// no N*64 over-allocation) and a stable radix sort orders the (key, voxel) pairs.
// Laplacian / grid-Eikonal adjoints: cuda/src/ls_compute.cu:14-109, ge_compute.cu:14-117
// with the sample helpers of auxiliary.h:392-471.  The jitter seed is an argument.
#include <mutex>
#include <string>

#include <cuda.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "svr_common.cuh"

using namespace svr;

int svr_fail(int code, const char* what);
void svr_note_launch(int n);
#define CUDA_TRY(x)                                                                      \
    do {                                                                                 \
        cudaError_t e_ = (x);                                                            \
        if (e_ != cudaSuccess) return svr_fail(SVR_ERR_CUDA, cudaGetErrorString(e_));    \
    } while (0)

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

__device__ __forceinline__ bool voxel_cells(const float* center, float size, const float* scene_center, float ext,
                                            int res, bool leaf, int lo[3], int hi[3]) {
    const float cells = (size / ext) * res;
    if ((!leaf) && ((cells > 1.5f) || (cells < 0.9f))) return false;
    if ((leaf) && (cells < 0.9f)) return false;
    float mn[3], mx[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) { mn[d] = scene_center[d] - 0.5f * ext; mx[d] = scene_center[d] + 0.5f * ext; }
#pragma unroll
    for (int d = 0; d < 3; ++d) if (center[d] < mn[d] || center[d] > mx[d]) return false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float a = center[d] - 0.5f * size, b = center[d] + 0.5f * size;
        lo[d] = int(roundf((a - mn[d]) / (mx[d] - mn[d]) * res));
        hi[d] = int(roundf((b - mn[d]) / (mx[d] - mn[d]) * res));
        // stay inside the dense grid (a voxel straddling the inside bound would otherwise
        // register cells past the end of grid_mask)
        lo[d] = max(0, min(res, lo[d]));
        hi[d] = max(0, min(res, hi[d]));
    }
    return true;
}

__global__ void cell_count_kernel(int N, const float* __restrict__ centers, const float* __restrict__ sizes,
                                  const float* __restrict__ sc, float ext, int res, const uint8_t* __restrict__ leaf,
                                  uint32_t* __restrict__ counts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int lo[3], hi[3];
    uint32_t c = 0;
    if (voxel_cells(centers + 3 * (size_t)i, sizes[i], sc, ext, res, leaf[i] != 0, lo, hi)) {
        const int a = hi[0] - lo[0], b = hi[1] - lo[1], d = hi[2] - lo[2];
        if (a > 0 && b > 0 && d > 0) c = (uint32_t)a * b * d;
    }
    counts[i] = c;
}

__global__ void cell_fill_kernel(int N, const float* __restrict__ centers, const float* __restrict__ sizes,
                                 const float* __restrict__ sc, float ext, int res, const uint8_t* __restrict__ leaf,
                                 const uint32_t* __restrict__ counts, const uint32_t* __restrict__ scan,
                                 uint8_t* __restrict__ mask, int32_t* __restrict__ keys, int32_t* __restrict__ vox)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || counts[i] == 0) return;
    int lo[3], hi[3];
    voxel_cells(centers + 3 * (size_t)i, sizes[i], sc, ext, res, leaf[i] != 0, lo, hi);
    uint32_t off = scan[i] - counts[i];
    for (int x = lo[0]; x < hi[0]; ++x)
        for (int y = lo[1]; y < hi[1]; ++y)
            for (int z = lo[2]; z < hi[2]; ++z) {
                const int f = x + res * (y + res * z);
                mask[f] = 1;
                keys[off] = f;
                vox[off] = i;
                ++off;
            }
}

struct TableWs {
    size_t counts, scan, scan_tmp, scan_tmp_bytes, keys_in, vox_in, sort_tmp, sort_tmp_bytes, total;
};
static TableWs table_ws(int N, int64_t G) {
    TableWs L{};
    const int n = N > 0 ? N : 1;
    const int g = G > 0 ? (int)G : 1;
    size_t st = 0, rt = 0;
    cub::DeviceScan::InclusiveSum(nullptr, st, (const uint32_t*)nullptr, (uint32_t*)nullptr, n);
    cub::DeviceRadixSort::SortPairs(nullptr, rt, (const int32_t*)nullptr, (int32_t*)nullptr,
                                    (const int32_t*)nullptr, (int32_t*)nullptr, g);
    size_t off = 0;
    L.counts = off; off = align_up(off + 4 * (size_t)n, 256);
    L.scan = off; off = align_up(off + 4 * (size_t)n, 256);
    L.scan_tmp = off; L.scan_tmp_bytes = st; off = align_up(off + st, 256);
    L.keys_in = off; off = align_up(off + 4 * (size_t)g, 256);
    L.vox_in = off; off = align_up(off + 4 * (size_t)g, 256);
    L.sort_tmp = off; L.sort_tmp_bytes = rt; off = align_up(off + rt, 256);
    L.total = off;
    return L;
}

extern "C" size_t svr_valid_table_workspace_bytes(int N, int64_t count) { return table_ws(N, count).total; }

extern "C" int svr_valid_table_count(int N, const float* centers, const float* sizes, const float* scene_center,
                                     float inside_extent, int res_pow2, const uint8_t* is_leaf, void* workspace,
                                     int64_t* count_host, void* stream)
{
    if (res_pow2 < 1 || res_pow2 > 10) return svr_fail(SVR_ERR_ARG, "grid resolution must be 2^1..2^10");
    cudaStream_t st = (cudaStream_t)stream;
    if (N <= 0) { *count_host = 0; return SVR_OK; }
    TableWs L = table_ws(N, 0);
    char* w = (char*)workspace;
    const int res = 1 << res_pow2;
    cell_count_kernel<<<(N + 255) / 256, 256, 0, st>>>(N, centers, sizes, scene_center, inside_extent, res, is_leaf,
                                                      (uint32_t*)(w + L.counts));
    svr_note_launch(1);
    CUDA_TRY(cudaGetLastError());
    size_t tb = L.scan_tmp_bytes;
    CUDA_TRY(cub::DeviceScan::InclusiveSum(w + L.scan_tmp, tb, (const uint32_t*)(w + L.counts),
                                           (uint32_t*)(w + L.scan), N, st));
    uint32_t total = 0;
    CUDA_TRY(cudaMemcpyAsync(&total, w + L.scan + 4 * (size_t)(N - 1), 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *count_host = total;
    return SVR_OK;
}

extern "C" int svr_valid_table_fill(int N, const float* centers, const float* sizes, const float* scene_center,
                                    float inside_extent, int res_pow2, const uint8_t* is_leaf, int64_t count,
                                    void* workspace, uint8_t* grid_mask, int32_t* grid_keys, int32_t* grid2voxel,
                                    void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const int res = 1 << res_pow2;
    CUDA_TRY(cudaMemsetAsync(grid_mask, 0, (size_t)res * res * res, st));
    if (N <= 0 || count <= 0) return SVR_OK;
    // counts / scan live at the same offsets for any G, so the count pass's results stay valid
    TableWs L = table_ws(N, count);
    char* w = (char*)workspace;
    cell_fill_kernel<<<(N + 255) / 256, 256, 0, st>>>(N, centers, sizes, scene_center, inside_extent, res, is_leaf,
                                                     (const uint32_t*)(w + L.counts), (const uint32_t*)(w + L.scan),
                                                     grid_mask, (int32_t*)(w + L.keys_in), (int32_t*)(w + L.vox_in));
    svr_note_launch(1);
    CUDA_TRY(cudaGetLastError());
    int bits = 1;
    while ((1ll << bits) < (long long)res * res * res) ++bits;
    size_t tb = L.sort_tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(w + L.sort_tmp, tb, (const int32_t*)(w + L.keys_in), grid_keys,
                                             (const int32_t*)(w + L.vox_in), grid2voxel, (int)count, 0, bits, st));
    return SVR_OK;
}

// ------------------------------------------------------------------ direct-mapped key index
// dense[key] = row of `key` in the sorted table, -1 elsewhere (first row when a key repeats).
// One 4-byte read replaces each 20+-step binary search of the smoothness adjoints; the
// table costs 4 * res^3 bytes (512 MB at res 512) and is rebuilt with the grid table.
__global__ void grid_index_kernel(int G, const int32_t* __restrict__ keys, int cells, int32_t* __restrict__ dense,
                                  unsigned* status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G) return;
    const int k = keys[i];
    if (k < 0 || k >= cells) { atomicOr(status, ERR_BAD_INDEX); return; }
    if (i == 0 || keys[i - 1] != k) dense[k] = i;
}

extern "C" int svr_grid_index_build(int G, const int32_t* grid_keys, int grid_res, int32_t* dense_index,
                                    uint32_t* status, void* stream)
{
    if (grid_res <= 0 || grid_res > 1024) return svr_fail(SVR_ERR_ARG, "grid index: resolution");
    if (!dense_index || (G > 0 && (!grid_keys || !status)))
        return svr_fail(SVR_ERR_ARG, "grid index: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int cells = grid_res * grid_res * grid_res;
    CUDA_TRY(cudaMemsetAsync(dense_index, 0xFF, 4 * (size_t)cells, st));
    if (G <= 0) return SVR_OK;
    grid_index_kernel<<<(G + 255) / 256, 256, 0, st>>>(G, grid_keys, cells, dense_index, status);
    svr_note_launch(1);
    CUDA_TRY(cudaGetLastError());
    return SVR_OK;
}

// ------------------------------------------------------------------ smoothness adjoints
__device__ __forceinline__ float hash_to_float(uint32_t x) {
    x ^= x >> 17; x *= 0xed5ad4bbu; x ^= x >> 11; x *= 0xac4c1b51u; x ^= x >> 15; x *= 0x31848babu; x ^= x >> 14;
    return (x & 0xFFFFFF) / float(0x1000000);
}
__device__ __forceinline__ float3 rand_vec(int tid, int seed) {
    return f3(hash_to_float((uint32_t)(seed * 73856093 ^ tid * 3 + 0)),
              hash_to_float((uint32_t)(seed * 19349663 ^ tid * 3 + 1)),
              hash_to_float((uint32_t)(seed * 83492791 ^ tid * 3 + 2)));
}
__device__ __forceinline__ int find_key(const int32_t* keys, int n, int key) {
    int l = 0, r = n - 1;
    while (l <= r) {
        const int m = (l + r) / 2;
        const int k = keys[m];
        if (k == key) return m;
        if (k < key) l = m + 1; else r = m - 1;
    }
    return -1;
}
__device__ __forceinline__ bool neighbours_ok(int x, int y, int z, int res, const uint8_t* mask) {
    if (x <= 0 || x >= res - 1 || y <= 0 || y >= res - 1 || z <= 0 || z >= res - 1) return false;
    const int rr = res * res;
    const int c = x + y * res + z * rr;
    return mask[c + 1] && mask[c - 1] && mask[c + res] && mask[c - res] && mask[c + rr] && mask[c - rr];
}

// Cell index -> (x, y, z).  The dense grid's side is a power of two in every caller of the
// reference (2^level), which takes shifts; any other side takes the divisions.
__device__ __forceinline__ void cell_xyz(int gk, int res, int& x, int& y, int& z) {
    if ((res & (res - 1)) == 0) {
        const int lg = __ffs(res) - 1;
        x = gk & (res - 1); y = (gk >> lg) & (res - 1); z = gk >> (2 * lg);
    } else {
        x = gk % res; y = (gk / res) % res; z = gk / (res * res);
    }
}

// (p - base) / size as the reference divides, per component.  Grid-unit voxel sizes are
// powers of two, for which multiplying by the reciprocal (itself exact) gives the same bits
// as the division; any other size divides.
__device__ __forceinline__ float3 local_coord(float3 p, float3 base, float size) {
    const float3 d = p - base;
    const uint32_t b = __float_as_uint(size);
    if ((b & 0x007FFFFFu) == 0u && ((b >> 23) & 0xFFu) - 1u < 0xFDu) {   // normal power of two
        const float r = __uint_as_float(((254u - ((b >> 23) & 0xFFu)) << 23) | (b & 0x80000000u));
        return f3(d.x * r, d.y * r, d.z * r);
    }
    return d / size;
}

struct SampleCtx {
    int G, N, M, res;
    const int32_t* dense;   // optional direct-mapped key -> table row (-1 when absent)
    const int32_t* keys;
    const int32_t* g2v;
    const float* coords;
    const float* vsizes;
    const int64_t* vox_key;
    const float* grid;
};

// auxiliary.h:433-482: owner voxel of grid cell (x,y,z), clamped trilinear weights at the
// jittered point, SDF value.  Returns the owner id or -1.
__device__ __forceinline__ int sample_cell(const SampleCtx& c, int x, int y, int z, float3 rv, float w[8], float& sdf,
                                           unsigned* status) {
    sdf = 0.f;
    const int key = x + y * c.res + z * c.res * c.res;
    const int id = c.dense ? c.dense[key] : find_key(c.keys, c.G, key);
    if (id < 0) return -1;
    const int v = c.g2v[id];
    if (v < 0 || v >= c.N) { atomicOr(status, ERR_BAD_INDEX); return -1; }
    const float3 pt = f3(x + rv.x, y + rv.y, z + rv.z);
    const float3 base = f3(c.coords[3 * v], c.coords[3 * v + 1], c.coords[3 * v + 2]);
    const float size = c.vsizes[v];
    tri_weights(local_coord(pt, base, size), w);
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (w[i] < 0) w[i] = 0;
        if (w[i] > 1) w[i] = 1;
        const int64_t p = c.vox_key[8 * (int64_t)v + i];
        if (p < 0 || p >= c.M) { atomicOr(status, ERR_BAD_INDEX); return -1; }
        s += c.grid[p] * w[i];
    }
    sdf = s;
    return v;
}
__device__ __forceinline__ void scatter8(const SampleCtx& c, int v, const float* w, float d, float* grad) {
    if (v < 0) return;
#pragma unroll
    for (int i = 0; i < 8; ++i) atomicAdd(grad + c.vox_key[8 * (int64_t)v + i], d * w[i]);
}

// Sums acc[0:8] over each run of lanes [head, next head) of a warp into the run's head
// lane (a segmented shuffle reduction).  The rounds stop at the warp's longest run: a
// further round would add nothing to any head, so each head's sum, and its order, is the
// one all five rounds give.  Warps whose runs are all single lanes skip the shuffles.
__device__ __forceinline__ void run_sum8(float acc[8], unsigned heads, bool head, int lane) {
    const unsigned FULL = 0xffffffffu;
    const unsigned upto = FULL >> (31 - lane);            // lanes 0..lane
    const int my_head = 31 - __clz(heads & upto);
    const unsigned later = heads & ~upto;                 // heads after this lane
    const unsigned run = head ? (unsigned)((later ? __ffs(later) - 1 : 32) - lane) : 0u;
    const int longest = (int)__reduce_max_sync(FULL, run);
    for (int off = 1; off < longest; off <<= 1) {
        const int other_head = __shfl_down_sync(FULL, my_head, off);
        const bool same = (lane + off < 32) && other_head == my_head;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float v = __shfl_down_sync(FULL, acc[i], off);
            if (same) acc[i] += v;
        }
    }
}

// Gradient scatter of one key's samples with two levels of aggregation before the atomics:
// samples whose owner voxel equals the primary sample's are merged in registers, then lanes
// of a warp holding the same primary voxel in a contiguous run (consecutive keys inside one
// coarse voxel) are summed by a segmented shuffle reduction, and only the run head issues
// the 8 atomics.  Inside a level-6 voxel this turns 56 atomics per key into 8 per warp.
template <int S>
__device__ __forceinline__ void scatter_samples(const SampleCtx& c, bool valid, const int* vid, float (*w)[8],
                                                const float* d, float* grad) {
    const int primary = valid ? vid[0] : -1;
    float acc[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i] = 0.f;
    if (valid) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            if (vid[s] == primary) {
#pragma unroll
                for (int i = 0; i < 8; ++i) acc[i] += d[s] * w[s][i];
            } else {
                scatter8(c, vid[s], w[s], d[s], grad);
            }
        }
    }
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int prev = __shfl_up_sync(FULL, primary, 1);
    const bool head = lane == 0 || prev != primary;
    const unsigned heads = __ballot_sync(FULL, head);
    run_sum8(acc, heads, head, lane);
    if (head && primary >= 0) {
#pragma unroll
        for (int i = 0; i < 8; ++i) atomicAdd(grad + c.vox_key[8 * (int64_t)primary + i], acc[i]);
    }
}

__global__ void __launch_bounds__(256) laplacian_kernel(SampleCtx c, int A, const int32_t* __restrict__ active,
                                                        const uint8_t* __restrict__ mask, float weight,
                                                        float vox_size_inv, int seed,
                                                        const int64_t* __restrict__ seed_step,
                                                        float* __restrict__ grad, unsigned* status)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = tid < A;
    int x = 0, y = 0, z = 0, gk = 0;
    const int res = c.res;
    if (valid) {
        const int a = active[tid];
        if (a < 0 || a >= c.G) { atomicOr(status, ERR_BAD_INDEX); valid = false; }
        else {
            gk = c.keys[a];
            if (gk < 0 || gk >= res * res * res) { atomicOr(status, ERR_BAD_INDEX); valid = false; }
            else {
                cell_xyz(gk, res, x, y, z);
                valid = mask[gk] && neighbours_ok(x, y, z, res, mask);
            }
        }
    }
    float w[7][8];
    int vid[7];
    float dd[7];
    if (valid) {
        const float3 rv = rand_vec(tid, seed_step ? seed + (int)*seed_step : seed);
        const int dx[6] = {+1, -1, 0, 0, 0, 0}, dy[6] = {0, 0, +1, -1, 0, 0}, dz[6] = {0, 0, 0, 0, +1, -1};
        float nb[6], center;
        vid[0] = sample_cell(c, x, y, z, rv, w[0], center, status);
#pragma unroll
        for (int i = 0; i < 6; ++i) vid[i + 1] = sample_cell(c, x + dx[i], y + dy[i], z + dz[i], rv, w[i + 1], nb[i], status);
        const float lx = nb[0] + nb[1] - 2.0f * center;
        const float ly = nb[2] + nb[3] - 2.0f * center;
        const float lz = nb[4] + nb[5] - 2.0f * center;
        const float lr = sqrtf(lx * lx + ly * ly + lz * lz + 1e-10f);
        // ls_compute.cu:79-83 evaluates these in double (0.5 is a double literal there)
        const float size = weight * 0.5 * vox_size_inv * vox_size_inv;
        const float gx = 0.5 / lr * 2 * lx * size;
        const float gy = 0.5 / lr * 2 * ly * size;
        const float gz = 0.5 / lr * 2 * lz * size;
        dd[0] = -2.0f * (gx + gy + gz);
        dd[1] = gx; dd[2] = gx; dd[3] = gy; dd[4] = gy; dd[5] = gz; dd[6] = gz;
    }
    scatter_samples<7>(c, valid, vid, w, dd, grad);
}

__global__ void __launch_bounds__(256) eikonal_kernel(SampleCtx c, int A, const int32_t* __restrict__ active,
                                                      const uint8_t* __restrict__ mask, float weight,
                                                      float vox_size_inv, int seed,
                                                      const int64_t* __restrict__ seed_step,
                                                      float* __restrict__ grad, unsigned* status)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = tid < A;
    int x = 0, y = 0, z = 0, gk = 0;
    const int res = c.res;
    if (valid) {
        const int a = active[tid];
        if (a < 0 || a >= c.G) { atomicOr(status, ERR_BAD_INDEX); valid = false; }
        else {
            gk = c.keys[a];
            if (gk < 0 || gk >= res * res * res) { atomicOr(status, ERR_BAD_INDEX); valid = false; }
            else {
                cell_xyz(gk, res, x, y, z);
                valid = mask[gk] && neighbours_ok(x, y, z, res, mask);
            }
        }
    }
    float w[6][8];
    int vid[6];
    float dd[6];
    if (valid) {
        const float3 rv = rand_vec(tid, seed_step ? seed + (int)*seed_step : seed);
        const int dx[6] = {+1, -1, 0, 0, 0, 0}, dy[6] = {0, 0, +1, -1, 0, 0}, dz[6] = {0, 0, 0, 0, +1, -1};
        float s[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) vid[i] = sample_cell(c, x + dx[i], y + dy[i], z + dz[i], rv, w[i], s[i], status);
        const float dxv = (s[0] - s[1]) * 0.5f, dyv = (s[2] - s[3]) * 0.5f, dzv = (s[4] - s[5]) * 0.5f;
        const float gn = sqrtf(dxv * dxv + dyv * dyv + dzv * dzv + 1e-6f);
        const float gw = gn * 0.5 * vox_size_inv;   // ge_compute.cu:93, double literal
        const float dg = 2.0f * (gw - 1.0f) * weight;
        const float ddx = dg * dxv / gn * 0.5f * vox_size_inv;
        const float ddy = dg * dyv / gn * 0.5f * vox_size_inv;
        const float ddz = dg * dzv / gn * 0.5f * vox_size_inv;
        dd[0] = ddx; dd[1] = -ddx; dd[2] = ddy; dd[3] = -ddy; dd[4] = ddz; dd[5] = -ddz;
    }
    scatter_samples<6>(c, valid, vid, w, dd, grad);
}

static int grid_loss(bool lap, int G, int A, const int32_t* active, const int32_t* keys, const int32_t* g2v, int res,
                     const uint8_t* mask, const int32_t* dense, const float* coords, const float* vsizes, int N, const int64_t* vox_key,
                     const float* grid, int M, float weight, float vox_size_inv, int seed, float* grad,
                     unsigned* status, void* stream, const int64_t* seed_step = nullptr)
{
    if (A <= 0) return SVR_OK;
    if (!active || !keys || !g2v || !mask || !coords || !vsizes || !vox_key || !grid || !grad || !status)
        return svr_fail(SVR_ERR_ARG, "grid loss: null argument");
    SampleCtx c{G, N, M, res, dense, keys, g2v, coords, vsizes, vox_key, grid};
    cudaStream_t st = (cudaStream_t)stream;
    if (lap) laplacian_kernel<<<(A + 255) / 256, 256, 0, st>>>(c, A, active, mask, weight, vox_size_inv, seed, seed_step,
                                                                 grad, status);
    else eikonal_kernel<<<(A + 255) / 256, 256, 0, st>>>(c, A, active, mask, weight, vox_size_inv, seed, seed_step, grad,
                                                         status);
    svr_note_launch(1);
    CUDA_TRY(cudaGetLastError());
    return SVR_OK;
}

extern "C" int svr_laplacian_bw(int G, int A, const int32_t* active, const int32_t* grid_keys, const int32_t* grid2voxel,
                                int grid_res, const uint8_t* grid_mask, const int32_t* dense_index, const float* voxel_coords,
                                const float* voxel_sizes, int N, const int64_t* vox_key, const float* grid_pts, int M,
                                float weight, float vox_size_inv, int seed, float* grid_grad, uint32_t* status,
                                void* stream)
{
    return grid_loss(true, G, A, active, grid_keys, grid2voxel, grid_res, grid_mask, dense_index, voxel_coords, voxel_sizes, N,
                     vox_key, grid_pts, M, weight, vox_size_inv, seed, grid_grad, status, stream);
}

extern "C" int svr_eikonal_bw(int G, int A, const int32_t* active, const int32_t* grid_keys, const int32_t* grid2voxel,
                                int grid_res, const uint8_t* grid_mask, const int32_t* dense_index, const float* voxel_coords,
                              const float* voxel_sizes, int N, const int64_t* vox_key, const float* grid_pts, int M,
                              float weight, float vox_size_inv, int seed, float* grid_grad, uint32_t* status,
                              void* stream)
{
    return grid_loss(false, G, A, active, grid_keys, grid2voxel, grid_res, grid_mask, dense_index, voxel_coords, voxel_sizes, N,
                     vox_key, grid_pts, M, weight, vox_size_inv, seed, grid_grad, status, stream);
}

// Graph-replayable variants: the jitter seed is seed_base + *step (a device counter), so a
// captured step draws fresh jitter on every replay like the per-call seed does.
extern "C" int svr_laplacian_bw_at_step(int G, int A, const int32_t* active, const int32_t* grid_keys,
                                        const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                                        const int32_t* dense_index, const float* voxel_coords,
                                        const float* voxel_sizes, int N, const int64_t* vox_key,
                                        const float* grid_pts, int M, float weight, float vox_size_inv,
                                        int seed_base, const int64_t* step, float* grid_grad, uint32_t* status,
                                        void* stream)
{
    if (!step) return svr_fail(SVR_ERR_ARG, "grid loss: null step counter");
    return grid_loss(true, G, A, active, grid_keys, grid2voxel, grid_res, grid_mask, dense_index, voxel_coords,
                     voxel_sizes, N, vox_key, grid_pts, M, weight, vox_size_inv, seed_base, grid_grad, status, stream,
                     step);
}

extern "C" int svr_eikonal_bw_at_step(int G, int A, const int32_t* active, const int32_t* grid_keys,
                                      const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                                      const int32_t* dense_index, const float* voxel_coords,
                                      const float* voxel_sizes, int N, const int64_t* vox_key,
                                      const float* grid_pts, int M, float weight, float vox_size_inv,
                                      int seed_base, const int64_t* step, float* grid_grad, uint32_t* status,
                                      void* stream)
{
    if (!step) return svr_fail(SVR_ERR_ARG, "grid loss: null step counter");
    return grid_loss(false, G, A, active, grid_keys, grid2voxel, grid_res, grid_mask, dense_index, voxel_coords,
                     voxel_sizes, N, vox_key, grid_pts, M, weight, vox_size_inv, seed_base, grid_grad, status, stream,
                     step);
}

// ------------------------------------------------------------------ fused per-voxel form
// Laplacian and grid-Eikonal adjoints in one pass, accumulated per voxel corner.  With one
// seed both losses sample the same six neighbour cells at the same jittered offset, so each
// neighbour is sampled once and its two gradient terms are added before the scatter.  The
// corner SDF values come from geos[v] (= grid[vox_key[v]], the gather at the start of the
// step) and the corner gradients accumulate into dvox[v, 0:8] with vector atomics; the
// per-voxel gradient scatter (svr_scatter_vox_grads) then moves them to the grid points with
// the render adjoint's.  Sample values and per-sample gradient terms are computed exactly
// as in laplacian_kernel / eikonal_kernel; only the summation order of the atomics differs.
struct VoxCtx {
    int G, N, res;
    const int32_t* dense;
    const int32_t* keys;
    const int32_t* g2v;
    const float* coords;
    const float* vsizes;
    const float4* geos;   // [N][2] float4 = 8 corner values
};

// Weight clamp to [0, 1] in two NaN-propagating min/max instructions.  It equals
// `w < 0 ? 0 : (w > 1 ? 1 : w)` for every input but -0.0, which becomes +0.0 (a zero
// weight either way).
__device__ __forceinline__ float clamp01(float w) {
    float r;
    asm("max.NaN.f32 %0, %1, 0f00000000;" : "=f"(r) : "f"(w));
    asm("min.NaN.f32 %0, %1, 0f3F800000;" : "=f"(r) : "f"(r));
    return r;
}

// Owner voxel of table row `id` and the sample at cell (x,y,z) + rv: returns the SDF value,
// writes the owner (-1 if absent) and the local coordinate q used for the weights.
__device__ __forceinline__ float sample_vox(const VoxCtx& c, int id, int x, int y, int z, float3 rv, int& v,
                                            float3& q, unsigned* status) {
    v = -1;
    q = f3(0.f, 0.f, 0.f);
    if (id < 0) return 0.f;
    const int vv = c.g2v[id];
    if (vv < 0 || vv >= c.N) { atomicOr(status, ERR_BAD_INDEX); return 0.f; }
    const float3 pt = f3(x + rv.x, y + rv.y, z + rv.z);
    const float3 base = f3(c.coords[3 * vv], c.coords[3 * vv + 1], c.coords[3 * vv + 2]);
    const float size = c.vsizes[vv];
    q = local_coord(pt, base, size);
    const float4 g0 = c.geos[2 * (size_t)vv], g1 = c.geos[2 * (size_t)vv + 1];
    const float g[8] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
    float w[8];
    tri_weights(q, w);
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        w[i] = clamp01(w[i]);
        s += g[i] * w[i];
    }
    v = vv;
    return s;
}

__device__ __forceinline__ void clamped_weights(float3 q, float w[8]) {
    tri_weights(q, w);
#pragma unroll
    for (int i = 0; i < 8; ++i) w[i] = clamp01(w[i]);
}

__device__ __forceinline__ void add8(float* dvox, int ld, bool vec4, int v, const float* a) {
    float* row = dvox + (size_t)v * ld;
    if (vec4) {
        atomicAdd(reinterpret_cast<float4*>(row), make_float4(a[0], a[1], a[2], a[3]));
        atomicAdd(reinterpret_cast<float4*>(row + 4), make_float4(a[4], a[5], a[6], a[7]));
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) atomicAdd(row + i, a[i]);
    }
}

template <bool LS, bool GE>
__global__ void __launch_bounds__(256, 5) smooth_vox_kernel(VoxCtx c, int A, const int32_t* __restrict__ active,
                                                         const uint8_t* __restrict__ mask, float w_ls, float w_ge,
                                                         float vox_size_inv, int seed,
                                                         const int64_t* __restrict__ seed_step,
                                                         float* __restrict__ dvox, int ld, bool vec4,
                                                         unsigned* status)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = tid < A;
    int a = 0, x = 0, y = 0, z = 0;
    const int res = c.res;
    if (valid) {
        a = active ? active[tid] : tid;
        if (a < 0 || a >= c.G) { atomicOr(status, ERR_BAD_INDEX); valid = false; }
        else {
            const int gk = c.keys[a];
            if (gk < 0 || gk >= res * res * res) { atomicOr(status, ERR_BAD_INDEX); valid = false; }
            else {
                cell_xyz(gk, res, x, y, z);
                valid = mask[gk] && neighbours_ok(x, y, z, res, mask);
            }
        }
    }
    constexpr int S = 7;
    int vid[S];
    float3 q[S];
    float d[S];
#pragma unroll
    for (int s = 0; s < S; ++s) { vid[s] = -1; d[s] = 0.f; q[s] = f3(0.f, 0.f, 0.f); }
    if (valid) {
        const float3 rv = rand_vec(tid, seed_step ? seed + (int)*seed_step : seed);
        const int rr = res * res;
        const int cell = x + y * res + z * rr;
        const int dx[6] = {+1, -1, 0, 0, 0, 0}, dy[6] = {0, 0, +1, -1, 0, 0}, dz[6] = {0, 0, 0, 0, +1, -1};
        const int step[6] = {1, -1, res, -res, rr, -rr};
        int id[S];
        id[0] = LS ? c.dense[cell] : -1;
#pragma unroll
        for (int i = 0; i < 6; ++i) id[i + 1] = c.dense[cell + step[i]];
        float f[S];
        f[0] = LS ? sample_vox(c, id[0], x, y, z, rv, vid[0], q[0], status) : 0.f;
#pragma unroll
        for (int i = 0; i < 6; ++i)
            f[i + 1] = sample_vox(c, id[i + 1], x + dx[i], y + dy[i], z + dz[i], rv, vid[i + 1], q[i + 1], status);
        if (LS) {
            const float center = f[0];
            const float lx = f[1] + f[2] - 2.0f * center;
            const float ly = f[3] + f[4] - 2.0f * center;
            const float lz = f[5] + f[6] - 2.0f * center;
            const float lr = sqrtf(lx * lx + ly * ly + lz * lz + 1e-10f);
            const float size = w_ls * 0.5 * vox_size_inv * vox_size_inv;
            const float gx = 0.5 / lr * 2 * lx * size;
            const float gy = 0.5 / lr * 2 * ly * size;
            const float gz = 0.5 / lr * 2 * lz * size;
            d[0] = -2.0f * (gx + gy + gz);
            d[1] = gx; d[2] = gx; d[3] = gy; d[4] = gy; d[5] = gz; d[6] = gz;
        }
        if (GE) {
            const float dxv = (f[1] - f[2]) * 0.5f, dyv = (f[3] - f[4]) * 0.5f, dzv = (f[5] - f[6]) * 0.5f;
            const float gn = sqrtf(dxv * dxv + dyv * dyv + dzv * dzv + 1e-6f);
            const float gw = gn * 0.5 * vox_size_inv;
            const float dg = 2.0f * (gw - 1.0f) * w_ge;
            const float ddx = dg * dxv / gn * 0.5f * vox_size_inv;
            const float ddy = dg * dyv / gn * 0.5f * vox_size_inv;
            const float ddz = dg * dzv / gn * 0.5f * vox_size_inv;
            d[1] += ddx; d[2] += -ddx; d[3] += ddy; d[4] += -ddy; d[5] += ddz; d[6] += -ddz;
        }
    }
    // merge samples owned by the primary voxel in registers, atomics for the others
    int primary = -1;
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (primary < 0 && vid[s] >= 0) primary = vid[s];
    float acc[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i] = 0.f;
    if (valid) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            if (vid[s] < 0) continue;
            float w[8];
            clamped_weights(q[s], w);
            if (vid[s] == primary) {
#pragma unroll
                for (int i = 0; i < 8; ++i) acc[i] += d[s] * w[i];
            } else {
                float t[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) t[i] = d[s] * w[i];
                add8(dvox, ld, vec4, vid[s], t);
            }
        }
    }
    // lanes holding the same primary voxel in a contiguous run are summed by a segmented
    // shuffle reduction; the run head issues the atomics
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    if (!valid) primary = -1;
    const int prev = __shfl_up_sync(FULL, primary, 1);
    const bool head = lane == 0 || prev != primary;
    const unsigned heads = __ballot_sync(FULL, head);
    run_sum8(acc, heads, head, lane);
    if (head && primary >= 0) add8(dvox, ld, vec4, primary, acc);
}

extern "C" int svr_smoothness_bw_vox(int G, int A, const int32_t* active, const int32_t* grid_keys,
                                     const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                                     const int32_t* dense_index, const float* voxel_coords,
                                     const float* voxel_sizes, int N, const float* geos, float w_ls,
                                     float w_ge, float vox_size_inv, int seed, const int64_t* seed_step,
                                     float* dvox, int ld, uint32_t* status, void* stream)
{
    if (A <= 0 || (w_ls == 0.f && w_ge == 0.f)) return SVR_OK;
    if (!grid_keys || !grid2voxel || !grid_mask || !dense_index || !voxel_coords || !voxel_sizes || !geos || !dvox ||
        !status || ld < 8)
        return svr_fail(SVR_ERR_ARG, "smoothness: null argument or ld < 8");
    if (!active && A > G) return svr_fail(SVR_ERR_ARG, "smoothness: A > G without an active list");
    if (((uintptr_t)geos & 15) != 0) return svr_fail(SVR_ERR_ARG, "smoothness: geos must be 16-byte aligned");
    const bool vec4 = (ld % 4 == 0) && (((uintptr_t)dvox & 15) == 0);
    VoxCtx c{G, N, grid_res, dense_index, grid_keys, grid2voxel, voxel_coords, voxel_sizes, (const float4*)geos};
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned nb = (unsigned)((A + 255) / 256);
    if (w_ls != 0.f && w_ge != 0.f)
        smooth_vox_kernel<true, true><<<nb, 256, 0, st>>>(c, A, active, grid_mask, w_ls, w_ge, vox_size_inv, seed,
                                                          seed_step, dvox, ld, vec4, status);
    else if (w_ls != 0.f)
        smooth_vox_kernel<true, false><<<nb, 256, 0, st>>>(c, A, active, grid_mask, w_ls, w_ge, vox_size_inv, seed,
                                                           seed_step, dvox, ld, vec4, status);
    else
        smooth_vox_kernel<false, true><<<nb, 256, 0, st>>>(c, A, active, grid_mask, w_ls, w_ge, vox_size_inv, seed,
                                                           seed_step, dvox, ld, vec4, status);
    svr_note_launch(1);
    CUDA_TRY(cudaGetLastError());
    return SVR_OK;
}

// ------------------------------------------------------------------ other grid regularisers
// vg_compute.cu:23-77 (voxel Eikonal): per active voxel, the centre gradient from the 8 corner
// SDFs by averaged central differences, loss gradient 4 (|g|^2 - 2) w g, chained back to the
// corners with the factor 0.25 (the reference's constants, kept).
__global__ void __launch_bounds__(256) voxel_gradient_kernel(int A, const int32_t* __restrict__ active, int N,
                                                             const int64_t* __restrict__ vox_key,
                                                             const float* __restrict__ grid, int64_t M,
                                                             const float* __restrict__ vox_size_inv, float weight,
                                                             float* __restrict__ grad, unsigned* status)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= A) return;
    const int v = active[tid];
    if (v < 0 || v >= N) { atomicOr(status, ERR_BAD_INDEX); return; }
    const float inv4h = 0.25f * vox_size_inv[v];
    // all keys, then one range test, then all corner loads: the loads issue together
    const longlong2* kp = reinterpret_cast<const longlong2*>(vox_key + 8 * (int64_t)v);
    const longlong2 k0 = kp[0], k1 = kp[1], k2 = kp[2], k3 = kp[3];
    const int64_t key[8] = {k0.x, k0.y, k1.x, k1.y, k2.x, k2.y, k3.x, k3.y};
    float S[8];
    bool bad = false;
#pragma unroll
    for (int i = 0; i < 8; ++i) bad |= key[i] < 0 || key[i] >= M;
    if (bad) { atomicOr(status, ERR_BAD_INDEX); return; }
#pragma unroll
    for (int i = 0; i < 8; ++i) S[i] = grid[key[i]];
    float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float sx = (i & 4) ? 1.f : -1.f, sy = (i & 2) ? 1.f : -1.f, sz = (i & 1) ? 1.f : -1.f;
        gx += sx * S[i];
        gy += sy * S[i];
        gz += sz * S[i];
    }
    gx *= inv4h; gy *= inv4h; gz *= inv4h;
    const float g2 = gx * gx + gy * gy + gz * gz;
    const float scale = 4.f * (g2 - 2.f) * weight;
    const float dx = scale * gx, dy = scale * gy, dz = scale * gz;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float sx = (i & 4) ? 1.f : -1.f, sy = (i & 2) ? 1.f : -1.f, sz = (i & 1) ? 1.f : -1.f;
        atomicAdd(grad + key[i], (dx * sx + dy * sy + dz * sz) * 0.25f);
    }
}

extern "C" int svr_voxel_gradient_bw(int N, int A, const int32_t* active, const int64_t* vox_key,
                                     const float* grid_pts, int64_t M, const float* vox_size_inv, float weight,
                                     float* grid_grad, uint32_t* status, void* stream)
{
    if (A <= 0) return SVR_OK;
    if (!active || !vox_key || !grid_pts || !vox_size_inv || !grid_grad || !status)
        return svr_fail(SVR_ERR_ARG, "voxel gradient: null argument");
    if (((uintptr_t)vox_key & 15) != 0) return svr_fail(SVR_ERR_ARG, "voxel gradient: vox_key not 16-byte aligned");
    voxel_gradient_kernel<<<(A + 255) / 256, 256, 0, (cudaStream_t)stream>>>(A, active, N, vox_key, grid_pts, M,
                                                                             vox_size_inv, weight, grid_grad,
                                                                             status);
    svr_note_launch(1);
    CUDA_TRY(cudaGetLastError());
    return SVR_OK;
}

// svr_total_variation_bw lives in voxel_order.cu beside its spatially ordered form.

// pl_compute.cu:14-63 (points on the surface): each point (grid units) is located in its
// cell (truncating casts, as there), the owner voxel's trilinear SDF (weights not clamped) is
// driven to 0 with loss sdf^2 * weight.  A masked cell missing from the table is skipped
// (the reference would index grid2voxel[-1]).
__global__ void __launch_bounds__(256) points_loss_kernel(int P, const float* __restrict__ pts, SampleCtx c,
                                                          const uint8_t* __restrict__ mask, float weight,
                                                          float* __restrict__ grad, unsigned* status)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= P) return;
    const float px = pts[3 * (int64_t)tid], py = pts[3 * (int64_t)tid + 1], pz = pts[3 * (int64_t)tid + 2];
    const int ix = (int)px, iy = (int)py, iz = (int)pz;
    const int res = c.res;
    if (ix < 0 || ix >= res || iy < 0 || iy >= res || iz < 0 || iz >= res) return;
    const int key = ix + iy * res + iz * res * res;
    if (!mask[key]) return;
    const int id = c.dense ? c.dense[key] : find_key(c.keys, c.G, key);
    if (id < 0) return;
    const int v = c.g2v[id];
    if (v < 0 || v >= c.N) { atomicOr(status, ERR_BAD_INDEX); return; }
    const float size = c.vsizes[v];
    const float3 q = local_coord(f3(px, py, pz), f3(c.coords[3 * v], c.coords[3 * v + 1], c.coords[3 * v + 2]),
                                 size);
    float w[8];
    tri_weights(q, w);
    int64_t k[8];
    float sdf = 0.f;
    bool bad = false;
#pragma unroll
    for (int i = 0; i < 8; ++i) k[i] = c.vox_key[8 * (int64_t)v + i];
#pragma unroll
    for (int i = 0; i < 8; ++i) bad |= k[i] < 0 || k[i] >= c.M;
    if (bad) { atomicOr(status, ERR_BAD_INDEX); return; }
#pragma unroll
    for (int i = 0; i < 8; ++i) sdf += w[i] * c.grid[k[i]];
    const float dL = 2.0f * (sdf - 0.0f) * weight;
#pragma unroll
    for (int i = 0; i < 8; ++i) atomicAdd(grad + k[i], dL * w[i]);
}

extern "C" int svr_points_loss_bw(int P, const float* points_in_grid, int G, const int32_t* grid_keys,
                                  const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                                  const int32_t* dense_index, const float* voxel_coords, const float* voxel_sizes,
                                  int N, const int64_t* vox_key, const float* grid_pts, int M, float weight,
                                  float* grid_grad, uint32_t* status, void* stream)
{
    if (P <= 0) return SVR_OK;
    if (!points_in_grid || !grid_keys || !grid2voxel || !grid_mask || !voxel_coords || !voxel_sizes || !vox_key ||
        !grid_pts || !grid_grad || !status)
        return svr_fail(SVR_ERR_ARG, "points loss: null argument");
    SampleCtx c{G, N, M, grid_res, dense_index, grid_keys, grid2voxel, voxel_coords, voxel_sizes, vox_key, grid_pts};
    points_loss_kernel<<<(P + 255) / 256, 256, 0, (cudaStream_t)stream>>>(P, points_in_grid, c, grid_mask, weight,
                                                                          grid_grad, status);
    svr_note_launch(1);
    CUDA_TRY(cudaGetLastError());
    return SVR_OK;
}

// ------------------------------------------------------------------ allocation-free variant
// For callers that cannot allocate device memory themselves (for example a host framework
// that hands out all device memory from a fixed arena reserved at start-up and forbids any
// later cudaMalloc): the direct-mapped key index of the Laplacian adjoint lives in this
// file-scope device array instead of caller memory.  Every GPU that loads the library holds
// it (8 MiB) until the process exits.
#define SVR_NOALLOC_MAX_RES 128
static __device__ __align__(256) int32_t g_noalloc_grid_index[SVR_NOALLOC_MAX_RES * SVR_NOALLOC_MAX_RES *
                                                                SVR_NOALLOC_MAX_RES];

// Device address of g_noalloc_grid_index per device.  The host-side name of the array is a
// stand-in, not a device address, so the address comes from cudaGetSymbolAddress, resolved
// once per device with that device current.  The cached address belongs to the context that
// was current when it was resolved: after cudaDeviceReset (or any teardown of the primary
// context) the module is loaded again, possibly elsewhere, so the cache is keyed on the
// context as well and resolved again when the context changes.
static int32_t* g_noalloc_index_ptr[64];
static CUcontext g_noalloc_index_ctx[64];
static std::mutex g_noalloc_mutex;

// cuCtxGetCurrent through the runtime's driver entry point (the library links only cudart)
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
static CUcontext current_context() {
    static CtxGetCurrentFn fn = []() -> CtxGetCurrentFn {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return (CtxGetCurrentFn)f;
    }();
    CUcontext ctx = nullptr;
    if (!fn || fn(&ctx) != CUDA_SUCCESS) return nullptr;
    return ctx;
}

static int noalloc_index_ptr(int32_t** out) {
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return svr_fail(SVR_ERR_UNSUPPORTED, "noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    CUcontext ctx = current_context();
    if (!g_noalloc_index_ptr[dev] || ctx == nullptr || g_noalloc_index_ctx[dev] != ctx) {
        void* p = nullptr;
        CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_grid_index));   // makes the primary context current
        g_noalloc_index_ptr[dev] = (int32_t*)p;
        g_noalloc_index_ctx[dev] = current_context();
    }
    *out = g_noalloc_index_ptr[dev];
    return SVR_OK;
}

extern "C" int svr_laplacian_bw_noalloc(int G, int A, const int32_t* active, const int32_t* grid_keys,
                                        const int32_t* grid2voxel, int grid_res, const uint8_t* grid_mask,
                                        const float* voxel_coords, const float* voxel_sizes, int N,
                                        const int64_t* vox_key, const float* grid_pts, int M, float weight,
                                        float vox_size_inv, int seed, float* grid_grad, uint32_t* status,
                                        void* stream)
{
    if (grid_res <= 0) return svr_fail(SVR_ERR_ARG, "svr_laplacian_bw_noalloc: grid_res must be positive");
    if (grid_res > SVR_NOALLOC_MAX_RES)
        return svr_fail(SVR_ERR_CAPACITY, "svr_laplacian_bw_noalloc: grid_res exceeds the static index capacity "
                                          "(maximum 128)");
    if (A <= 0) return SVR_OK;
    // every pointer the adjoint reads is checked before the index build launches anything
    if (!active || !grid_keys || !grid2voxel || !grid_mask || !voxel_coords || !voxel_sizes || !vox_key ||
        !grid_pts || !grid_grad || !status)
        return svr_fail(SVR_ERR_ARG, "svr_laplacian_bw_noalloc: null argument");
    int32_t* index = nullptr;
    int rc = noalloc_index_ptr(&index);
    if (rc) return rc;
    // the array keeps the previous call's index: rebuild it (the build clears it to -1 first)
    rc = svr_grid_index_build(G, grid_keys, grid_res, index, status, stream);
    if (rc) return rc;
    return grid_loss(true, G, A, active, grid_keys, grid2voxel, grid_res, grid_mask, index, voxel_coords,
                     voxel_sizes, N, vox_key, grid_pts, M, weight, vox_size_inv, seed, grid_grad, status, stream);
}
