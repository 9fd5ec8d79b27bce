// Adaptive pruning / subdivision support and training statistics.
//
// Behaviour of src/utils/octree_utils.py:129-222 (build_grid_pts_link: the corner grid points
// shared between voxels, unique(dim=0) with inverse), src/sparse_voxel_gears/adaptive.py:
// 349-411 (agg_voxel_into_grid_pts: index_reduce_ mean; subdivide_by_interp: trilinear child
// corner values) and adaptive.py:80-113 (compute_training_stat: max blending weight, minimum
// sampling interval and visible-view count per voxel).  Organisation (ours): one packed 51-bit
// key per corner (x << 34 | y << 17 | z at the finest level, the lexicographic order of
// unique(dim=0)), a stable radix sort, a flag + scan for the unique rows and the inverse; the
// statistics reduce per-view maxima that one batched forward over all views records.
#include <cstdint>
#include <string>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

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

// ------------------------------------------------------------------ grid-point link
struct LinkWs {
    size_t keys_in, keys_out, vals_in, vals_out, flags, pos, tmp, tmp_bytes, total;
};
static LinkWs link_ws(int64_t N)
{
    LinkWs L{};
    const int n = (int)(8 * (N > 0 ? N : 1));
    size_t ts = 0, tc = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, ts, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, n);
    cub::DeviceScan::InclusiveSum(nullptr, tc, (const uint32_t*)nullptr, (uint32_t*)nullptr, n);
    size_t off = 0;
    L.keys_in = off; off = align_up(off + 8 * (size_t)n, 256);
    L.keys_out = off; off = align_up(off + 8 * (size_t)n, 256);
    L.vals_in = off; off = align_up(off + 4 * (size_t)n, 256);
    L.vals_out = off; off = align_up(off + 4 * (size_t)n, 256);
    L.flags = off; off = align_up(off + 4 * (size_t)n, 256);
    L.pos = off; off = align_up(off + 4 * (size_t)n, 256);
    L.tmp = off; L.tmp_bytes = ts > tc ? ts : tc; off = align_up(off + L.tmp_bytes, 256);
    L.total = off;
    return L;
}

// octree_utils.py:129-144 gen_gridpoints_coordinate: corner k of voxel v at the finest level,
// (ijk + shift_k) << (16 - level) with shift_k = (k >> 2 & 1, k >> 1 & 1, k & 1).
__global__ void corner_key_kernel(int64_t N, const int64_t* __restrict__ octpath, const int8_t* __restrict__ level,
                                  uint64_t* __restrict__ keys, uint32_t* __restrict__ vals, unsigned* status)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 8 * N) return;
    const int64_t v = t >> 3;
    const int k = (int)(t & 7);
    const int lv = level[v];
    if (lv < 0 || lv > MAX_LEVELS) { atomicOr(status, ERR_BAD_INDEX); keys[t] = 0; vals[t] = (uint32_t)t; return; }
    uint64_t p = (uint64_t)octpath[v] >> (3 * (MAX_LEVELS - lv));
    uint64_t i = 0, j = 0, l = 0;
    for (int b = 0; b < lv; ++b) {          // utils.cu:160-189 octpath_2_ijk
        const uint64_t d = p & 7;
        i |= ((d >> 2) & 1) << b;
        j |= ((d >> 1) & 1) << b;
        l |= (d & 1) << b;
        p >>= 3;
    }
    const int s = MAX_LEVELS - lv;
    const uint64_t x = (i + ((k >> 2) & 1)) << s, y = (j + ((k >> 1) & 1)) << s, z = (l + (k & 1)) << s;
    keys[t] = (x << 34) | (y << 17) | z;
    vals[t] = (uint32_t)t;
}

__global__ void unique_flag_kernel(int64_t n, const uint64_t* __restrict__ keys, uint32_t* __restrict__ flags)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void link_write_kernel(int64_t n, const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                                  const uint32_t* __restrict__ flags, const uint32_t* __restrict__ pos,
                                  int64_t* __restrict__ grid_pts_key, int64_t* __restrict__ vox_key)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t row = (int64_t)pos[i] - 1;
    if (flags[i]) {
        const uint64_t k = keys[i];
        const uint64_t m17 = (1ull << 17) - 1;
        grid_pts_key[3 * row] = (int64_t)(k >> 34);
        grid_pts_key[3 * row + 1] = (int64_t)((k >> 17) & m17);
        grid_pts_key[3 * row + 2] = (int64_t)(k & m17);
    }
    vox_key[vals[i]] = row;
}

extern "C" size_t svr_grid_link_workspace_bytes(int64_t N) { return link_ws(N).total; }

extern "C" int svr_grid_link(int64_t N, const int64_t* octpath, const int8_t* octlevel, void* workspace,
                             size_t workspace_bytes, int64_t* grid_pts_key, int64_t* vox_key, int64_t* M_host,
                             uint32_t* status, void* stream)
{
    if (N < 0 || 8 * N >= (1ll << 31)) return svr_fail(SVR_ERR_ARG, "grid link: voxel count out of range");
    if (M_host) *M_host = 0;
    if (N == 0) return SVR_OK;
    if (!octpath || !octlevel || !workspace || !grid_pts_key || !vox_key || !status)
        return svr_fail(SVR_ERR_ARG, "grid link: null argument");
    const LinkWs L = link_ws(N);
    if (workspace_bytes < L.total) return svr_fail(SVR_ERR_CAPACITY, "grid link: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    char* w = (char*)workspace;
    const int64_t n = 8 * N;
    auto ki = (uint64_t*)(w + L.keys_in), ko = (uint64_t*)(w + L.keys_out);
    auto vi = (uint32_t*)(w + L.vals_in), vo = (uint32_t*)(w + L.vals_out);
    auto fl = (uint32_t*)(w + L.flags), ps = (uint32_t*)(w + L.pos);
    corner_key_kernel<<<nblk(n, 256), 256, 0, st>>>(N, octpath, octlevel, ki, vi, status);
    LAUNCHED();
    size_t tb = L.tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(w + L.tmp, tb, (const uint64_t*)ki, ko, (const uint32_t*)vi, vo, (int)n,
                                             0, 51, st));
    unique_flag_kernel<<<nblk(n, 256), 256, 0, st>>>(n, ko, fl);
    LAUNCHED();
    tb = L.tmp_bytes;
    CUDA_TRY(cub::DeviceScan::InclusiveSum(w + L.tmp, tb, (const uint32_t*)fl, ps, (int)n, st));
    link_write_kernel<<<nblk(n, 256), 256, 0, st>>>(n, ko, vo, fl, ps, grid_pts_key, vox_key);
    LAUNCHED();
    if (M_host) {
        uint32_t m = 0;
        CUDA_TRY(cudaMemcpyAsync(&m, ps + (n - 1), 4, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        *M_host = m;
    }
    return SVR_OK;
}

// ------------------------------------------------------------------ subdivision by interpolation
// adaptive.py:374-411: child m of a subdivided voxel takes at its corner m ^ x the parent's
// corner m (x = 0), the mean of an edge's two corners (x = 1, 2, 4), of a face's four corners
// (x = 3, 5, 6, summed in the reference's order) or of all eight (x = 7).
__global__ void subdivide_interp_kernel(int64_t n, int C, const float* __restrict__ v, float* __restrict__ out)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;   // (parent, child, x, channel)
    if (t >= n * 64 * C) return;
    const int c = (int)(t % C);
    const int64_t r = t / C;
    const int x = (int)(r & 7), m = (int)((r >> 3) & 7);
    const int64_t p = r >> 6;
    const float* pv = v + p * 8 * C;
    auto at = [&](int corner) { return pv[corner * C + c]; };
    float val;
    switch (x) {
        case 0: val = at(m); break;
        case 1: case 2: case 4: val = 0.5f * (at(m) + at(m ^ x)); break;
        case 3: val = 0.25f * (((at(m) + at(m ^ 1)) + at(m ^ 2)) + at(m ^ 3)); break;
        case 5: val = 0.25f * (((at(m) + at(m ^ 1)) + at(m ^ 4)) + at(m ^ 5)); break;
        case 6: val = 0.25f * (((at(m) + at(m ^ 2)) + at(m ^ 4)) + at(m ^ 6)); break;
        default: {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < 8; ++k) s += at(k);
            val = s / 8.0f;
        }
    }
    out[((p * 8 + m) * 8 + (m ^ x)) * C + c] = val;
}

extern "C" int svr_subdivide_interp(int64_t n, int C, const float* vox_val, float* out, void* stream)
{
    if (n < 0 || C <= 0) return svr_fail(SVR_ERR_ARG, "subdivide: bad size");
    if (n == 0) return SVR_OK;
    if (!vox_val || !out) return svr_fail(SVR_ERR_ARG, "subdivide: null argument");
    subdivide_interp_kernel<<<nblk(n * 64 * C, 256), 256, 0, (cudaStream_t)stream>>>(n, C, vox_val, out);
    LAUNCHED();
    return SVR_OK;
}

// ------------------------------------------------------------------ aggregation into grid points
// adaptive.py:349-372: index_reduce_(mean, include_self=False) into zeros: each grid point gets
// the mean of the corner values of every voxel that has it as a corner; others stay 0.
__global__ void agg_sum_kernel(int64_t n8, int C, int64_t M, const int64_t* __restrict__ vox_key,
                               const float* __restrict__ vox_val, float* __restrict__ out, float* __restrict__ cnt,
                               unsigned* status)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;   // (voxel corner, channel)
    if (t >= n8 * C) return;
    const int64_t e = t / C;
    const int c = (int)(t % C);
    const int64_t k = vox_key[e];
    if (k < 0 || k >= M) { atomicOr(status, ERR_BAD_INDEX); return; }
    atomicAdd(out + k * C + c, vox_val[t]);
    if (c == 0) atomicAdd(cnt + k, 1.0f);
}

__global__ void agg_div_kernel(int64_t M, int C, float* __restrict__ out, const float* __restrict__ cnt)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M * C) return;
    const float n = cnt[t / C];
    if (n > 0.f) out[t] = out[t] / n;
}

extern "C" int svr_agg_voxel_into_grid_pts(int64_t N, int C, const int64_t* vox_key, const float* vox_val, int64_t M,
                                           float* out, float* count_ws, uint32_t* status, void* stream)
{
    if (N < 0 || M < 0 || C <= 0) return svr_fail(SVR_ERR_ARG, "aggregate: bad size");
    cudaStream_t st = (cudaStream_t)stream;
    if (M > 0) {
        if (!out || !count_ws) return svr_fail(SVR_ERR_ARG, "aggregate: null output");
        CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)M * C, st));
        CUDA_TRY(cudaMemsetAsync(count_ws, 0, sizeof(float) * (size_t)M, st));
    }
    if (N == 0 || M == 0) return SVR_OK;
    if (!vox_key || !vox_val || !status) return svr_fail(SVR_ERR_ARG, "aggregate: null argument");
    agg_sum_kernel<<<nblk(8 * N * C, 256), 256, 0, st>>>(8 * N, C, M, vox_key, vox_val, out, count_ws, status);
    LAUNCHED();
    agg_div_kernel<<<nblk(M * C, 256), 256, 0, st>>>(M, C, out, count_ws);
    LAUNCHED();
    return SVR_OK;
}

// ------------------------------------------------------------------ training statistics
// adaptive.py:80-113 over the views of a batch: max_w = max over views; a voxel is visible in a
// view when its max weight there is > 0, and then min_samp_interval = min over those views of
// ((centre - camera position) . lookat) * pix_size and view_cnt counts them.
__global__ void training_stat_kernel(int V, int64_t N, const float* __restrict__ mw, const float3* __restrict__ centers,
                                     const float3* __restrict__ pos, const float3* __restrict__ lookat,
                                     const float* __restrict__ pix_size, float* __restrict__ max_w,
                                     float* __restrict__ min_samp, float* __restrict__ view_cnt)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float m = max_w[i], s = min_samp[i], cnt = view_cnt[i];
    const float3 c = centers[i];
    for (int v = 0; v < V; ++v) {
        const float w = mw[(int64_t)v * N + i];
        m = fmaxf(m, w);
        if (w > 0.f) {
            const float3 d = c - pos[v];
            const float3 l = lookat[v];
            const float zdist = __fadd_rn(__fadd_rn(__fmul_rn(d.x, l.x), __fmul_rn(d.y, l.y)), __fmul_rn(d.z, l.z));
            s = fminf(s, __fmul_rn(zdist, pix_size[v]));
            cnt += 1.0f;
        }
    }
    max_w[i] = m;
    min_samp[i] = s;
    view_cnt[i] = cnt;
}

extern "C" int svr_training_stat_reduce(int n_views, int64_t N, const float* max_w_views, const float* centers,
                                        const float* cam_pos, const float* cam_lookat, const float* pix_size,
                                        float* max_w, float* min_samp_interval, float* view_cnt, void* stream)
{
    if (n_views <= 0 || N < 0) return svr_fail(SVR_ERR_ARG, "training stat: bad size");
    if (N == 0) return SVR_OK;
    if (!max_w_views || !centers || !cam_pos || !cam_lookat || !pix_size || !max_w || !min_samp_interval || !view_cnt)
        return svr_fail(SVR_ERR_ARG, "training stat: null argument");
    training_stat_kernel<<<nblk(N, 256), 256, 0, (cudaStream_t)stream>>>(
        n_views, N, max_w_views, (const float3*)centers, (const float3*)cam_pos, (const float3*)cam_lookat, pix_size,
        max_w, min_samp_interval, view_cnt);
    LAUNCHED();
    return SVR_OK;
}
