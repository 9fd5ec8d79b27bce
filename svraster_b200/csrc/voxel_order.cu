// Spatially ordered forms of the voxel Eikonal and the sign total variation adjoints.
//
// The reference runs one thread per voxel in storage order (cuda/src/vg_compute.cu:23-77,
// cuda/src/tv_compute.cu:22-158).  Voxels are stored in no spatial order, so the 8 corner
// reads and 8 atomic adds of a warp land on 32 different 32-byte sectors each: every voxel
// costs 16 scattered L2 requests, and that request count, not DRAM, bounds those kernels.
// Here the voxels are visited in the order of their first corner's grid-point index (a
// permutation sorted once per octree and cached by the caller).  Grid points are stored in
// lexicographic (x, y, z) order, so consecutive voxels in that order have neighbouring corner
// indices and a warp's corner reads and adds fall on about a third as many sectors.
#include <cstdint>
#include <string>

#include <cub/device/device_radix_sort.cuh>

#include "svr_common.cuh"

using namespace svr;

int svr_fail(int code, const char* what);
void svr_note_launch(int n);

#define CUDA_TRY(x)                                                                      \
    do {                                                                                 \
        cudaError_t e_ = (x);                                                            \
        if (e_ != cudaSuccess) {                                                         \
            return svr_fail(SVR_ERR_CUDA, (std::string(#x) + ": " + cudaGetErrorString(e_)).c_str()); \
        }                                                                                \
    } while (0)
#define LAUNCHED() do { svr_note_launch(1); CUDA_TRY(cudaGetLastError()); } while (0)

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
static inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }
static inline int bits_for(int64_t m) { int b = 1; while (b < 31 && (1ll << b) < m) ++b; return b; }

// ------------------------------------------------------------------ the visit order
// order[i] = the voxel with the i-th smallest vox_key[v, 0] (ties by voxel id), rank = its
// inverse.
struct OrderWs {
    size_t keys_in, keys_out, vals_in, tmp, tmp_bytes, total;
};
static int order_ws(int64_t N, OrderWs& w) {
    w.keys_in = 0;
    w.keys_out = align_up(4 * (size_t)N, 256);
    w.vals_in = w.keys_out + align_up(4 * (size_t)N, 256);
    w.tmp = w.vals_in + align_up(4 * (size_t)N, 256);
    w.tmp_bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, w.tmp_bytes, (const uint32_t*)nullptr,
                                                    (uint32_t*)nullptr, (const int32_t*)nullptr, (int32_t*)nullptr,
                                                    (int)N);
    if (e != cudaSuccess) return svr_fail(SVR_ERR_CUDA, "voxel order: sort size query");
    w.total = align_up(w.tmp + w.tmp_bytes, 256);
    return SVR_OK;
}

extern "C" int svr_voxel_order_workspace_bytes(int64_t N, size_t* bytes)
{
    if (!bytes || N < 0 || N >= (1ll << 31)) return svr_fail(SVR_ERR_ARG, "voxel order: N");
    OrderWs w;
    if (int rc = order_ws(N, w)) return rc;
    *bytes = w.total;
    return SVR_OK;
}

__global__ void order_key_kernel(int64_t N, const int64_t* __restrict__ vox_key, int64_t M,
                                 uint32_t* __restrict__ keys, int32_t* __restrict__ vals, unsigned* status)
{
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const int64_t k = vox_key[8 * v];
    if (k < 0 || k >= M) atomicOr(status, ERR_BAD_INDEX);
    keys[v] = (k < 0 || k >= M) ? 0u : (uint32_t)k;
    vals[v] = (int32_t)v;
}

__global__ void order_rank_kernel(int64_t N, const int32_t* __restrict__ order, int32_t* __restrict__ rank)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    rank[order[i]] = (int32_t)i;
}

extern "C" int svr_voxel_order(int64_t N, const int64_t* vox_key, int64_t M, int32_t* order, int32_t* rank,
                               void* ws, size_t ws_bytes, uint32_t* status, void* stream)
{
    size_t need = 0;
    if (int rc = svr_voxel_order_workspace_bytes(N, &need)) return rc;
    if (N == 0) return SVR_OK;
    if (!vox_key || !order || !rank || !status || !ws || ws_bytes < need || M <= 0 || M >= (1ll << 31))
        return svr_fail(SVR_ERR_ARG, "voxel order: bad argument or workspace too small");
    OrderWs w;
    if (int rc = order_ws(N, w)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    char* base = (char*)ws;
    uint32_t* kin = (uint32_t*)(base + w.keys_in);
    uint32_t* kout = (uint32_t*)(base + w.keys_out);
    int32_t* vin = (int32_t*)(base + w.vals_in);
    order_key_kernel<<<nblk(N, 256), 256, 0, st>>>(N, vox_key, M, kin, vin, status);
    LAUNCHED();
    size_t tb = w.tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(base + w.tmp, tb, kin, kout, vin, order, (int)N, 0, bits_for(M), st));
    order_rank_kernel<<<nblk(N, 256), 256, 0, st>>>(N, order, rank);
    LAUNCHED();
    return SVR_OK;
}

// ------------------------------------------------------------------ sign total variation
// tv_compute.cu:22-158 (per (voxel, channel), each corner gets w * the sum over its 3 edge
// neighbours of +1 if it is larger, else -1; w = weight, times 0.01 / size unless no_tv_s),
// thread t on (order[t / C], t % C), or (t / C, t % C) in storage order when order is null.
// With tv_sparse only voxels with a nonzero gradient at one of their corners take part; the
// reference reads that gradient while other threads add to it, here a first pass decides
// from the gradient as it was on entry (no race).
__global__ void tv_ord_valid_kernel(int64_t NC, int C, const int32_t* __restrict__ order,
                                    const int64_t* __restrict__ vox_key, const float* __restrict__ grad, int64_t M,
                                    uint8_t* __restrict__ valid)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= NC) return;
    const uint32_t row = C == 1 ? (uint32_t)t : (uint32_t)t / (uint32_t)C;
    const int64_t n = order ? order[row] : row;
    const int c = C == 1 ? 0 : (int)((uint32_t)t - row * (uint32_t)C);
    bool v = false;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int64_t k = vox_key[8 * n + i];
        if (k >= 0 && k < M) v |= grad[k * C + c] != 0.f;
    }
    valid[t] = v;
}

template <bool NO_TV_S, bool SPARSE>
__global__ void __launch_bounds__(256) tv_ord_kernel(int64_t NC, int C, const int32_t* __restrict__ order,
                                                     const int64_t* __restrict__ vox_key,
                                                     const float* __restrict__ grid, int64_t M, float weight,
                                                     const float* __restrict__ vox_size_inv,
                                                     const uint8_t* __restrict__ valid, float* __restrict__ grad,
                                                     unsigned* status)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= NC) return;
    if (SPARSE && !valid[t]) return;
    const uint32_t row = C == 1 ? (uint32_t)t : (uint32_t)t / (uint32_t)C;
    const int64_t n = order ? order[row] : row;
    const int c = C == 1 ? 0 : (int)((uint32_t)t - row * (uint32_t)C);
    const longlong2* kp = reinterpret_cast<const longlong2*>(vox_key + 8 * n);
    const longlong2 k0 = kp[0], k1 = kp[1], k2 = kp[2], k3 = kp[3];
    const int64_t key[8] = {k0.x, k0.y, k1.x, k1.y, k2.x, k2.y, k3.x, k3.y};
    float v[8];
    bool bad = false;
#pragma unroll
    for (int i = 0; i < 8; ++i) bad |= key[i] < 0 || key[i] >= M;
    if (bad) { atomicOr(status, ERR_BAD_INDEX); return; }
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = grid[key[i] * C + c];
    float w = weight;
    if (!NO_TV_S) w *= 0.01f * vox_size_inv[n];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int s = ((v[i] > v[i ^ 1]) * 2 - 1) + ((v[i] > v[i ^ 2]) * 2 - 1) + ((v[i] > v[i ^ 4]) * 2 - 1);
        atomicAdd(grad + key[i] * C + c, w * (float)s);
    }
}

static int tv_launch(int64_t N, int C, const int32_t* order, const int64_t* vox_key, const float* grid_pts,
                     int64_t M, float weight, const float* vox_size_inv, int no_tv_s, int tv_sparse,
                     uint8_t* valid_ws, float* grid_grad, uint32_t* status, void* stream)
{
    if (N <= 0) return SVR_OK;
    if (C <= 0 || !vox_key || !grid_pts || !grid_grad || !status || (!no_tv_s && !vox_size_inv) ||
        (tv_sparse && !valid_ws) || N * C >= (1ll << 32))
        return svr_fail(SVR_ERR_ARG, "total variation: bad argument");
    if (((uintptr_t)vox_key & 15) != 0) return svr_fail(SVR_ERR_ARG, "total variation: vox_key not 16-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t NC = N * C;
    const unsigned nb = nblk(NC, 256);
    if (tv_sparse) {
        tv_ord_valid_kernel<<<nb, 256, 0, st>>>(NC, C, order, vox_key, grid_grad, M, valid_ws);
        LAUNCHED();
    }
#define TV_ORD(A, B) tv_ord_kernel<A, B><<<nb, 256, 0, st>>>(NC, C, order, vox_key, grid_pts, M, weight, \
                                                               vox_size_inv, valid_ws, grid_grad, status)
    if (no_tv_s && tv_sparse) TV_ORD(true, true);
    else if (no_tv_s) TV_ORD(true, false);
    else if (tv_sparse) TV_ORD(false, true);
    else TV_ORD(false, false);
#undef TV_ORD
    LAUNCHED();
    return SVR_OK;
}

extern "C" int svr_total_variation_bw(int64_t N, int C, const int64_t* vox_key, const float* grid_pts, int64_t M,
                                      float weight, const float* vox_size_inv, int no_tv_s, int tv_sparse,
                                      uint8_t* valid_ws, float* grid_grad, uint32_t* status, void* stream)
{
    return tv_launch(N, C, nullptr, vox_key, grid_pts, M, weight, vox_size_inv, no_tv_s, tv_sparse, valid_ws,
                     grid_grad, status, stream);
}

extern "C" int svr_total_variation_bw_ordered(int64_t N, int C, const int32_t* order, const int64_t* vox_key,
                                              const float* grid_pts, int64_t M, float weight,
                                              const float* vox_size_inv, int no_tv_s, int tv_sparse,
                                              uint8_t* valid_ws, float* grid_grad, uint32_t* status, void* stream)
{
    if (N > 0 && !order) return svr_fail(SVR_ERR_ARG, "total variation (ordered): null order");
    return tv_launch(N, C, order, vox_key, grid_pts, M, weight, vox_size_inv, no_tv_s, tv_sparse, valid_ws,
                     grid_grad, status, stream);
}

// ------------------------------------------------------------------ voxel Eikonal
// vg_compute.cu:23-77 for the voxels listed in active: the list is turned into a listing
// count per visit position (cnt[rank[v]] += 1), then thread i visits voxel order[i] and adds
// its corner contributions cnt times (a voxel listed twice adds twice, as in the reference).
__global__ void vg_count_kernel(int A, const int32_t* __restrict__ active, int N, const int32_t* __restrict__ rank,
                                int32_t* __restrict__ cnt, unsigned* status)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A) return;
    const int v = active[t];
    if (v < 0 || v >= N) { atomicOr(status, ERR_BAD_INDEX); return; }
    atomicAdd(cnt + rank[v], 1);
}

__global__ void __launch_bounds__(256) vg_ord_kernel(int N, const int32_t* __restrict__ order,
                                                     const int32_t* __restrict__ cnt,
                                                     const int64_t* __restrict__ vox_key,
                                                     const float* __restrict__ grid, int64_t M,
                                                     const float* __restrict__ vox_size_inv, float weight,
                                                     float* __restrict__ grad, unsigned* status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int m = cnt[i];
    if (m == 0) return;
    const int64_t v = order[i];
    const longlong2* kp = reinterpret_cast<const longlong2*>(vox_key + 8 * v);
    const longlong2 k0 = kp[0], k1 = kp[1], k2 = kp[2], k3 = kp[3];
    const int64_t key[8] = {k0.x, k0.y, k1.x, k1.y, k2.x, k2.y, k3.x, k3.y};
    float S[8];
    bool bad = false;
#pragma unroll
    for (int c = 0; c < 8; ++c) bad |= key[c] < 0 || key[c] >= M;
    if (bad) { atomicOr(status, ERR_BAD_INDEX); return; }
#pragma unroll
    for (int c = 0; c < 8; ++c) S[c] = grid[key[c]];
    const float inv4h = 0.25f * vox_size_inv[v];
    float gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const float sx = (c & 4) ? 1.f : -1.f, sy = (c & 2) ? 1.f : -1.f, sz = (c & 1) ? 1.f : -1.f;
        gx += sx * S[c];
        gy += sy * S[c];
        gz += sz * S[c];
    }
    gx *= inv4h; gy *= inv4h; gz *= inv4h;
    const float g2 = gx * gx + gy * gy + gz * gz;
    const float scale = 4.f * (g2 - 2.f) * weight;
    const float dx = scale * gx, dy = scale * gy, dz = scale * gz;
    for (int r = 0; r < m; ++r) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float sx = (c & 4) ? 1.f : -1.f, sy = (c & 2) ? 1.f : -1.f, sz = (c & 1) ? 1.f : -1.f;
            atomicAdd(grad + key[c], (dx * sx + dy * sy + dz * sz) * 0.25f);
        }
    }
}

extern "C" int svr_voxel_gradient_bw_ordered(int N, int A, const int32_t* active, const int32_t* order,
                                             const int32_t* rank, const int64_t* vox_key, const float* grid_pts,
                                             int64_t M, const float* vox_size_inv, float weight, int32_t* count_ws,
                                             float* grid_grad, uint32_t* status, void* stream)
{
    if (A <= 0 || N <= 0) return SVR_OK;
    if (!active || !order || !rank || !vox_key || !grid_pts || !vox_size_inv || !count_ws || !grid_grad || !status)
        return svr_fail(SVR_ERR_ARG, "voxel gradient (ordered): null argument");
    if (((uintptr_t)vox_key & 15) != 0)
        return svr_fail(SVR_ERR_ARG, "voxel gradient (ordered): vox_key not 16-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_TRY(cudaMemsetAsync(count_ws, 0, 4 * (size_t)N, st));
    vg_count_kernel<<<nblk(A, 256), 256, 0, st>>>(A, active, N, rank, count_ws, status);
    LAUNCHED();
    vg_ord_kernel<<<nblk(N, 256), 256, 0, st>>>(N, order, count_ws, vox_key, grid_pts, M, vox_size_inv, weight,
                                                grid_grad, status);
    LAUNCHED();
    return SVR_OK;
}
