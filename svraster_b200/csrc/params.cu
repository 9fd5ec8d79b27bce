// Per-voxel parameter kernels: corner-SDF gather (+ adjoint), SH colour (+ adjoint), Adam.
// Behaviour of cuda/src/geo_params_gather.cu, sh_compute.cu and adam_step.cu; all are
// HBM-bound elementwise/gather work, mapped one thread per (voxel, corner) or per element
// with 16-byte accesses where the layout allows.
#include <cmath>
#include <cuda_bf16.h>
#include <string>

#include "svr_common.cuh"

using namespace svr;

int svr_fail(int code, const char* what);
void svr_note_launch(int n);
#define CUDA_TRY(x)                                                                      \
    do {                                                                                 \
        cudaError_t e_ = (x);                                                            \
        if (e_ != cudaSuccess) return svr_fail(SVR_ERR_CUDA, cudaGetErrorString(e_));    \
    } while (0)
#define LAUNCHED() do { svr_note_launch(1); CUDA_TRY(cudaGetLastError()); } while (0)

static inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// ------------------------------------------------------------------ gather
// geo_params_gather.cu:22-46: geos[i, k] = grid[vox_key[i, k]] for i in care_idx.
// Eight threads per voxel: the key reads and the geos writes are fully coalesced.
__global__ void gather_geo_kernel(int64_t n_care, const int64_t* __restrict__ care_idx,
                                  const int64_t* __restrict__ vox_key, const float* __restrict__ grid,
                                  float* __restrict__ geos)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_care * 8) return;
    const int64_t i = care_idx[t >> 3];
    const int k = (int)(t & 7);
    geos[8 * i + k] = __ldg(grid + vox_key[8 * i + k]);
}

// geo_params_gather.cu:48-72
__global__ void gather_geo_bw_kernel(int64_t n_care, const int64_t* __restrict__ care_idx,
                                     const int64_t* __restrict__ vox_key, const float* __restrict__ dgeos,
                                     float* __restrict__ dgrid)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_care * 8) return;
    const int64_t i = care_idx[t >> 3];
    const int k = (int)(t & 7);
    const float d = dgeos[8 * i + k];
    if (d != 0.f) atomicAdd(dgrid + vox_key[8 * i + k], d);
}

extern "C" int svr_gather_geo(int64_t n_care, const int64_t* care_idx, const int64_t* vox_key,
                              const float* grid_pts, float* geos, void* stream)
{
    if (n_care <= 0) return SVR_OK;
    if (!care_idx || !vox_key || !grid_pts || !geos) return svr_fail(SVR_ERR_ARG, "gather: null argument");
    gather_geo_kernel<<<nblk(n_care * 8, 256), 256, 0, (cudaStream_t)stream>>>(n_care, care_idx, vox_key, grid_pts, geos);
    LAUNCHED();
    return SVR_OK;
}

extern "C" int svr_gather_geo_bw(int64_t n_care, const int64_t* care_idx, const int64_t* vox_key,
                                 const float* dgeos, float* dgrid, void* stream)
{
    if (n_care <= 0) return SVR_OK;
    if (!care_idx || !vox_key || !dgeos || !dgrid) return svr_fail(SVR_ERR_ARG, "gather_bw: null argument");
    gather_geo_bw_kernel<<<nblk(n_care * 8, 256), 256, 0, (cudaStream_t)stream>>>(n_care, care_idx, vox_key, dgeos, dgrid);
    LAUNCHED();
    return SVR_OK;
}

// Scatter per-voxel corner gradients (row stride `ld`, e.g. the 12-wide render adjoint
// output) into the grid-point gradient for all N voxels; rows of zeros cost no atomics.
__global__ void scatter_vox_grads_kernel(int64_t N, int ld, const int64_t* __restrict__ vox_key,
                                         const float* __restrict__ dvox, float* __restrict__ dgrid)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * 8) return;
    const int64_t i = t >> 3;
    const int k = (int)(t & 7);
    const float d = dvox[i * ld + k];
    if (d != 0.f) atomicAdd(dgrid + vox_key[8 * i + k], d);
}

extern "C" int svr_scatter_vox_grads(int64_t N, int ld, const int64_t* vox_key, const float* dvox, float* dgrid,
                                     void* stream)
{
    if (N <= 0) return SVR_OK;
    if (ld < 8 || !vox_key || !dvox || !dgrid) return svr_fail(SVR_ERR_ARG, "scatter_vox_grads: bad argument");
    scatter_vox_grads_kernel<<<nblk(N * 8, 256), 256, 0, (cudaStream_t)stream>>>(N, ld, vox_key, dvox, dgrid);
    LAUNCHED();
    return SVR_OK;
}

// ------------------------------------------------------------------ SH
// sh_compute.cu:33-106 (forward) and :111-176 (adjoint; the clamp is not differentiated,
// as in the reference).
__constant__ float kSH_C2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                                -1.0925484305920792f, 0.5462742152960396f};
__constant__ float kSH_C3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                                0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                                -0.5900435899266435f};
constexpr float SH_C0 = 0.28209479177387814f;
constexpr float SH_C1 = 0.4886025119029199f;

template <int DEG>
__device__ __forceinline__ void sh_basis(float3 dir, float* B) {
    const float x = dir.x, y = dir.y, z = dir.z;
    B[0] = SH_C0;
    if (DEG > 0) { B[1] = -SH_C1 * y; B[2] = SH_C1 * z; B[3] = -SH_C1 * x; }
    if (DEG > 1) {
        const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
        B[4] = kSH_C2[0] * xy; B[5] = kSH_C2[1] * yz; B[6] = kSH_C2[2] * (2.0f * zz - xx - yy);
        B[7] = kSH_C2[3] * xz; B[8] = kSH_C2[4] * (xx - yy);
        if (DEG > 2) {
            B[9] = kSH_C3[0] * y * (3.0f * xx - yy);
            B[10] = kSH_C3[1] * xy * z;
            B[11] = kSH_C3[2] * y * (4.0f * zz - xx - yy);
            B[12] = kSH_C3[3] * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
            B[13] = kSH_C3[4] * x * (4.0f * zz - xx - yy);
            B[14] = kSH_C3[5] * z * (xx - yy);
            B[15] = kSH_C3[6] * x * (xx - 3.0f * yy);
        }
    }
}

template <int DEG>
__global__ void sh_eval_kernel(int N, int64_t n_idx, const int64_t* __restrict__ idx, int M,
                               const float3* __restrict__ centers, const float3* __restrict__ cam_pos,
                               const float3* __restrict__ sh0, const float3* __restrict__ shs,
                               float3* __restrict__ rgbs)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = n_idx > 0 ? n_idx : N;
    if (t >= n) return;
    const int64_t i = n_idx > 0 ? idx[t] : t;
    const float3 ro = *cam_pos;
    float3 dir = centers[i] - ro;
    dir = dir * rnorm3df(dir.x, dir.y, dir.z);
    float B[16];
    sh_basis<DEG>(dir, B);
    const float3* sh = shs + i * (M - 1);
    float3 res = B[0] * sh0[i];
    constexpr int NB = (DEG + 1) * (DEG + 1);
#pragma unroll
    for (int k = 1; k < NB; ++k) res = res + B[k] * sh[k - 1];
    res = res + 0.5f;
    res.x *= (res.x > 0.0f);
    res.y *= (res.y > 0.0f);
    res.z *= (res.z > 0.0f);
    rgbs[i] = res;
}

// Same evaluation with coalesced row loads when every coefficient row is full (NB == M): each
// warp loads its 32 voxels' 180-byte rows one row at a time with consecutive lanes into
// shared memory, then every thread evaluates its voxel from there (same arithmetic and order).
template <int DEG>
__global__ void __launch_bounds__(128) sh_eval_rows_kernel(int N, int64_t n_idx, const int64_t* __restrict__ idx,
                                                           const float3* __restrict__ centers,
                                                           const float3* __restrict__ cam_pos,
                                                           const float3* __restrict__ sh0, const float* __restrict__ shs,
                                                           float3* __restrict__ rgbs)
{
    constexpr int NB = (DEG + 1) * (DEG + 1);
    constexpr int ROW = 3 * (NB - 1);
    __shared__ float rows[128 * ROW + 1];
    __shared__ int64_t vox[128];
    const int64_t n = n_idx > 0 ? n_idx : N;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t tt = (int64_t)blockIdx.x * 128 + t;
    const int64_t i = tt < n ? (n_idx > 0 ? idx[tt] : tt) : -1;
    vox[t] = i;
    __syncwarp();
    // all 32 rows' loads issue before any store (a row is at most 45 floats: two per lane)
    static_assert(ROW <= 64, "row wider than two loads per lane");
    float a[32], b[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) {
        const int64_t v = vox[warp * 32 + r];
        a[r] = (v >= 0 && lane < ROW) ? shs[ROW * v + lane] : 0.f;
        b[r] = (v >= 0 && lane + 32 < ROW) ? shs[ROW * v + lane + 32] : 0.f;
    }
#pragma unroll
    for (int r = 0; r < 32; ++r) {
        float* row = rows + (warp * 32 + r) * ROW;
        if (lane < ROW) row[lane] = a[r];
        if (lane + 32 < ROW) row[lane + 32] = b[r];
    }
    __syncwarp();
    if (i < 0) return;
    const float3 ro = *cam_pos;
    float3 dir = centers[i] - ro;
    dir = dir * rnorm3df(dir.x, dir.y, dir.z);
    float B[16];
    sh_basis<DEG>(dir, B);
    const float* sh = rows + t * ROW;
    float3 res = B[0] * sh0[i];
#pragma unroll
    for (int k = 1; k < NB; ++k) res = res + B[k] * f3(sh[3 * (k - 1)], sh[3 * (k - 1) + 1], sh[3 * (k - 1) + 2]);
    res = res + 0.5f;
    res.x *= (res.x > 0.0f);
    res.y *= (res.y > 0.0f);
    res.z *= (res.z > 0.0f);
    rgbs[i] = res;
}

template <int DEG>
__global__ void sh_eval_bw_kernel(int N, int64_t n_idx, const int64_t* __restrict__ idx, int M,
                                  const float3* __restrict__ centers, const float3* __restrict__ cam_pos,
                                  const float3* __restrict__ drgbs, float3* __restrict__ dsh0,
                                  float3* __restrict__ dshs)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = n_idx > 0 ? n_idx : N;
    if (t >= n) return;
    const int64_t i = n_idx > 0 ? idx[t] : t;
    const float3 ro = *cam_pos;
    float3 dir = centers[i] - ro;
    dir = dir * rnorm3df(dir.x, dir.y, dir.z);
    float B[16];
    sh_basis<DEG>(dir, B);
    const float3 d = drgbs[i];
    dsh0[i] = B[0] * d;
    float3* o = dshs + i * (M - 1);
    constexpr int NB = (DEG + 1) * (DEG + 1);
#pragma unroll
    for (int k = 1; k < NB; ++k) o[k - 1] = B[k] * d;
}

extern "C" int svr_sh_eval(int N, int64_t n_idx, const int64_t* idx, int degree, int M, const float* centers,
                           const float* cam_pos, const float* sh0, const float* shs, float* rgbs, void* stream)
{
    if (degree < 0 || degree > 3 || M < (degree + 1) * (degree + 1)) return svr_fail(SVR_ERR_ARG, "sh degree");
    const int64_t n = n_idx > 0 ? n_idx : N;
    if (n <= 0) return SVR_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned g = nblk(n, 256);
    const auto c = (const float3*)centers; const auto cp = (const float3*)cam_pos;
    const auto s0 = (const float3*)sh0; const auto ss = (const float3*)shs; auto o = (float3*)rgbs;
    if (degree == 3 && M == 16) {
        sh_eval_rows_kernel<3><<<nblk(n, 128), 128, 0, st>>>(N, n_idx, idx, c, cp, s0, shs, o);
        LAUNCHED();
        return SVR_OK;
    }
    switch (degree) {
        case 0: sh_eval_kernel<0><<<g, 256, 0, st>>>(N, n_idx, idx, M, c, cp, s0, ss, o); break;
        case 1: sh_eval_kernel<1><<<g, 256, 0, st>>>(N, n_idx, idx, M, c, cp, s0, ss, o); break;
        case 2: sh_eval_kernel<2><<<g, 256, 0, st>>>(N, n_idx, idx, M, c, cp, s0, ss, o); break;
        default: sh_eval_kernel<3><<<g, 256, 0, st>>>(N, n_idx, idx, M, c, cp, s0, ss, o); break;
    }
    LAUNCHED();
    return SVR_OK;
}

// Same adjoint with coalesced row stores when every coefficient row is full (NB == M): each
// thread stages its voxel's 3 + 3(NB-1) gradient values in shared memory, then each warp
// writes its 32 voxels' rows one row at a time with consecutive lanes (a 180-byte row is 6
// sectors; one thread per row left 32 scattered sectors per warp store).
template <int DEG>
__global__ void __launch_bounds__(128) sh_eval_bw_rows_kernel(int N, int64_t n_idx, const int64_t* __restrict__ idx,
                                                              const float3* __restrict__ centers,
                                                              const float3* __restrict__ cam_pos,
                                                              const float3* __restrict__ drgbs,
                                                              float* __restrict__ dsh0, float* __restrict__ dshs)
{
    constexpr int NB = (DEG + 1) * (DEG + 1);
    constexpr int ROW = 3 * (NB - 1);
    __shared__ float rows[128 * ROW + 1];
    __shared__ float dc[128 * 3];
    __shared__ int64_t vox[128];
    const int64_t n = n_idx > 0 ? n_idx : N;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t tt = (int64_t)blockIdx.x * 128 + t;
    int64_t i = -1;
    if (tt < n) {
        i = n_idx > 0 ? idx[tt] : tt;
        const float3 ro = *cam_pos;
        float3 dir = centers[i] - ro;
        dir = dir * rnorm3df(dir.x, dir.y, dir.z);
        float B[16];
        sh_basis<DEG>(dir, B);
        const float3 d = drgbs[i];
        dc[3 * t] = B[0] * d.x; dc[3 * t + 1] = B[0] * d.y; dc[3 * t + 2] = B[0] * d.z;
#pragma unroll
        for (int k = 1; k < NB; ++k) {
            rows[t * ROW + 3 * (k - 1)] = B[k] * d.x;
            rows[t * ROW + 3 * (k - 1) + 1] = B[k] * d.y;
            rows[t * ROW + 3 * (k - 1) + 2] = B[k] * d.z;
        }
    }
    vox[t] = i;
    __syncwarp();
    for (int r = warp * 32; r < warp * 32 + 32; ++r) {
        const int64_t v = vox[r];
        if (v < 0) break;                                  // the warp's remaining slots are empty too
        if (lane < 3) dsh0[3 * v + lane] = dc[3 * r + lane];
        for (int j = lane; j < ROW; j += 32) dshs[ROW * v + j] = rows[r * ROW + j];
    }
}

extern "C" int svr_sh_eval_bw(int N, int64_t n_idx, const int64_t* idx, int degree, int M, const float* centers,
                              const float* cam_pos, const float* drgbs, float* dsh0, float* dshs, void* stream)
{
    if (degree < 0 || degree > 3 || M < (degree + 1) * (degree + 1)) return svr_fail(SVR_ERR_ARG, "sh degree");
    const int64_t n = n_idx > 0 ? n_idx : N;
    if (n <= 0) return SVR_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned g = nblk(n, 256);
    const auto c = (const float3*)centers; const auto cp = (const float3*)cam_pos;
    const auto d = (const float3*)drgbs; auto o0 = (float3*)dsh0; auto o1 = (float3*)dshs;
    if (degree == 3 && M == 16) {
        sh_eval_bw_rows_kernel<3><<<nblk(n, 128), 128, 0, st>>>(N, n_idx, idx, c, cp, d, dsh0, dshs);
        LAUNCHED();
        return SVR_OK;
    }
    switch (degree) {
        case 0: sh_eval_bw_kernel<0><<<g, 256, 0, st>>>(N, n_idx, idx, M, c, cp, d, o0, o1); break;
        case 1: sh_eval_bw_kernel<1><<<g, 256, 0, st>>>(N, n_idx, idx, M, c, cp, d, o0, o1); break;
        case 2: sh_eval_bw_kernel<2><<<g, 256, 0, st>>>(N, n_idx, idx, M, c, cp, d, o0, o1); break;
        default: sh_eval_bw_kernel<3><<<g, 256, 0, st>>>(N, n_idx, idx, M, c, cp, d, o0, o1); break;
    }
    LAUNCHED();
    return SVR_OK;
}

// Multi-view SH: one thread per voxel reads its coefficients once and serves every view
// (forward writes rgbs[v, i]; the adjoint sums the views' colour gradients into one
// coefficient gradient).  Same per-view arithmetic as sh_compute.cu:55-176.
// Coefficient storage: float3, or bf16 triples (converted exactly to f32 on load; all SH
// arithmetic, compositing and gradient accumulation stay f32).
struct ShF32 {
    const float3* sh0;
    const float3* shs;
    __device__ __forceinline__ float3 dc(int64_t i) const { return sh0[i]; }
    __device__ __forceinline__ float3 rest(int64_t j) const { return shs[j]; }
};
struct ShBF16 {
    const __nv_bfloat16* sh0;
    const __nv_bfloat16* shs;
    __device__ __forceinline__ static float3 get(const __nv_bfloat16* p, int64_t j) {
        return f3(__bfloat162float(p[3 * j]), __bfloat162float(p[3 * j + 1]), __bfloat162float(p[3 * j + 2]));
    }
    __device__ __forceinline__ float3 dc(int64_t i) const { return get(sh0, i); }
    __device__ __forceinline__ float3 rest(int64_t j) const { return get(shs, j); }
};

template <int DEG, typename Coef>
__global__ void sh_views_kernel(int N, int V, int M, const float3* __restrict__ centers,
                                const float3* __restrict__ cam_pos, Coef sh, float3* __restrict__ rgbs)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    constexpr int NB = (DEG + 1) * (DEG + 1);
    float3 c[NB];
    c[0] = sh.dc(i);
#pragma unroll
    for (int k = 1; k < NB; ++k) c[k] = sh.rest(i * (M - 1) + k - 1);
    const float3 ctr = centers[i];
    for (int v = 0; v < V; ++v) {
        float3 dir = ctr - cam_pos[v];
        dir = dir * rnorm3df(dir.x, dir.y, dir.z);
        float B[16];
        sh_basis<DEG>(dir, B);
        float3 res = B[0] * c[0];
#pragma unroll
        for (int k = 1; k < NB; ++k) res = res + B[k] * c[k];
        res = res + 0.5f;
        res.x *= (res.x > 0.0f);
        res.y *= (res.y > 0.0f);
        res.z *= (res.z > 0.0f);
        rgbs[(int64_t)v * N + i] = res;
    }
}

template <int DEG, bool ADD = false>
__global__ void sh_views_bw_kernel(int N, int V, int M, const float3* __restrict__ centers,
                                   const float3* __restrict__ cam_pos, const float3* __restrict__ drgbs,
                                   float3* __restrict__ dsh0, float3* __restrict__ dshs)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    constexpr int NB = (DEG + 1) * (DEG + 1);
    float3 acc[NB];
#pragma unroll
    for (int k = 0; k < NB; ++k) acc[k] = f3(0.f, 0.f, 0.f);
    const float3 ctr = centers[i];
    for (int v = 0; v < V; ++v) {
        const float3 d = drgbs[(int64_t)v * N + i];
        if (d.x == 0.f && d.y == 0.f && d.z == 0.f) continue;
        float3 dir = ctr - cam_pos[v];
        dir = dir * rnorm3df(dir.x, dir.y, dir.z);
        float B[16];
        sh_basis<DEG>(dir, B);
#pragma unroll
        for (int k = 0; k < NB; ++k) acc[k] = acc[k] + B[k] * d;
    }
    dsh0[i] = ADD ? dsh0[i] + acc[0] : acc[0];
#pragma unroll
    for (int k = 1; k < NB; ++k) {
        float3& o = dshs[i * (M - 1) + k - 1];
        o = ADD ? o + acc[k] : acc[k];
    }
}

// Same adjoint with coalesced stores when every coefficient row is full (NB == M): the block's
// rows are staged in shared memory and written back as one contiguous range (one thread per
// voxel writing its 180-byte row left 32 scattered sectors per warp store).
template <int DEG, bool ADD = false>
__global__ void __launch_bounds__(128) sh_views_bw_full_kernel(int N, int V, const float3* __restrict__ centers,
                                                               const float3* __restrict__ cam_pos,
                                                               const float3* __restrict__ drgbs,
                                                               float* __restrict__ dsh0, float* __restrict__ dshs)
{
    constexpr int NB = (DEG + 1) * (DEG + 1);
    constexpr int ROW = 3 * (NB - 1);
    __shared__ float rows[128 * ROW + 1];
    __shared__ float dc[128 * 3];
    const int64_t base = (int64_t)blockIdx.x * 128;
    const int t = threadIdx.x;
    const int64_t i = base + t;
    float3 acc[NB];
#pragma unroll
    for (int k = 0; k < NB; ++k) acc[k] = f3(0.f, 0.f, 0.f);
    if (i < N) {
        const float3 ctr = centers[i];
        for (int v = 0; v < V; ++v) {
            const float3 d = drgbs[(int64_t)v * N + i];
            if (d.x == 0.f && d.y == 0.f && d.z == 0.f) continue;
            float3 dir = ctr - cam_pos[v];
            dir = dir * rnorm3df(dir.x, dir.y, dir.z);
            float B[16];
            sh_basis<DEG>(dir, B);
#pragma unroll
            for (int k = 0; k < NB; ++k) acc[k] = acc[k] + B[k] * d;
        }
    }
    dc[3 * t] = acc[0].x; dc[3 * t + 1] = acc[0].y; dc[3 * t + 2] = acc[0].z;
#pragma unroll
    for (int k = 1; k < NB; ++k) {
        rows[t * ROW + 3 * (k - 1)] = acc[k].x;
        rows[t * ROW + 3 * (k - 1) + 1] = acc[k].y;
        rows[t * ROW + 3 * (k - 1) + 2] = acc[k].z;
    }
    __syncthreads();
    const int nv = (int)min((int64_t)128, (int64_t)N - base);
    float* o0 = dsh0 + 3 * base;
    for (int j = t; j < 3 * nv; j += 128) o0[j] = ADD ? o0[j] + dc[j] : dc[j];
    float* o1 = dshs + (int64_t)ROW * base;
    for (int j = t; j < ROW * nv; j += 128) o1[j] = ADD ? o1[j] + rows[j] : rows[j];
}

template <typename Coef>
static int sh_views_launch(int degree, int N, int V, int M, const float3* c, const float3* cp, Coef sh, float3* o,
                           void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned g = nblk(N, 128);
    switch (degree) {
        case 0: sh_views_kernel<0, Coef><<<g, 128, 0, st>>>(N, V, M, c, cp, sh, o); break;
        case 1: sh_views_kernel<1, Coef><<<g, 128, 0, st>>>(N, V, M, c, cp, sh, o); break;
        case 2: sh_views_kernel<2, Coef><<<g, 128, 0, st>>>(N, V, M, c, cp, sh, o); break;
        default: sh_views_kernel<3, Coef><<<g, 128, 0, st>>>(N, V, M, c, cp, sh, o); break;
    }
    LAUNCHED();
    return SVR_OK;
}

extern "C" int svr_sh_eval_views(int N, int n_views, int degree, int M, const float* centers, const float* cam_pos,
                                 const float* sh0, const float* shs, float* rgbs, void* stream)
{
    if (degree < 0 || degree > 3 || M < (degree + 1) * (degree + 1) || n_views <= 0)
        return svr_fail(SVR_ERR_ARG, "sh views: bad degree / view count");
    if (N <= 0) return SVR_OK;
    auto c = (const float3*)centers; auto cp = (const float3*)cam_pos; auto o = (float3*)rgbs;
    return sh_views_launch(degree, N, n_views, M, c, cp, ShF32{(const float3*)sh0, (const float3*)shs}, o, stream);
}

extern "C" int svr_sh_eval_views_bf16(int N, int n_views, int degree, int M, const float* centers,
                                      const float* cam_pos, const uint16_t* sh0, const uint16_t* shs, float* rgbs,
                                      void* stream)
{
    if (degree < 0 || degree > 3 || M < (degree + 1) * (degree + 1) || n_views <= 0)
        return svr_fail(SVR_ERR_ARG, "sh views: bad degree / view count");
    if (N <= 0) return SVR_OK;
    auto c = (const float3*)centers; auto cp = (const float3*)cam_pos; auto o = (float3*)rgbs;
    return sh_views_launch(degree, N, n_views, M, c, cp,
                           ShBF16{(const __nv_bfloat16*)sh0, (const __nv_bfloat16*)shs}, o, stream);
}

template <bool ADD>
static int sh_views_bw_impl(int N, int n_views, int degree, int M, const float* centers, const float* cam_pos,
                            const float* drgbs, float* dsh0, float* dshs, void* stream);

extern "C" int svr_sh_eval_views_bw(int N, int n_views, int degree, int M, const float* centers,
                                    const float* cam_pos, const float* drgbs, float* dsh0, float* dshs, void* stream)
{
    return sh_views_bw_impl<false>(N, n_views, degree, M, centers, cam_pos, drgbs, dsh0, dshs, stream);
}

extern "C" int svr_sh_eval_views_bw_add(int N, int n_views, int degree, int M, const float* centers,
                                        const float* cam_pos, const float* drgbs, float* dsh0, float* dshs,
                                        void* stream)
{
    return sh_views_bw_impl<true>(N, n_views, degree, M, centers, cam_pos, drgbs, dsh0, dshs, stream);
}

template <bool ADD>
static int sh_views_bw_impl(int N, int n_views, int degree, int M, const float* centers, const float* cam_pos,
                            const float* drgbs, float* dsh0, float* dshs, void* stream)
{
    if (degree < 0 || degree > 3 || M < (degree + 1) * (degree + 1) || n_views <= 0)
        return svr_fail(SVR_ERR_ARG, "sh views bw: bad degree / view count");
    if (N <= 0) return SVR_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (degree == 3 && M == 16) {
        sh_views_bw_full_kernel<3, ADD><<<nblk(N, 128), 128, 0, st>>>(N, n_views, (const float3*)centers,
                                                                 (const float3*)cam_pos, (const float3*)drgbs,
                                                                 dsh0, dshs);
        LAUNCHED();
        return SVR_OK;
    }
    const unsigned g = nblk(N, 128);
    auto c = (const float3*)centers; auto cp = (const float3*)cam_pos; auto d = (const float3*)drgbs;
    auto o0 = (float3*)dsh0; auto o1 = (float3*)dshs;
    switch (degree) {
        case 0: sh_views_bw_kernel<0, ADD><<<g, 128, 0, st>>>(N, n_views, M, c, cp, d, o0, o1); break;
        case 1: sh_views_bw_kernel<1, ADD><<<g, 128, 0, st>>>(N, n_views, M, c, cp, d, o0, o1); break;
        case 2: sh_views_bw_kernel<2, ADD><<<g, 128, 0, st>>>(N, n_views, M, c, cp, d, o0, o1); break;
        default: sh_views_bw_kernel<3, ADD><<<g, 128, 0, st>>>(N, n_views, M, c, cp, d, o0, o1); break;
    }
    LAUNCHED();
    return SVR_OK;
}

// ------------------------------------------------------------------ Adam
// adam_step.cu:21-104: lerp via two FMAs, bias corrections from the host in double.
__device__ __forceinline__ float lerp_fma(float v0, float v1, float t) { return fmaf(t, v1, fmaf(-t, v0, v0)); }

template <bool SPARSE, bool BIASED>
__device__ __forceinline__ void adam_one(float& p, float g, float& m, float& v, float step_size, float b1, float b2,
                                         float rbc2, float eps) {
    if (SPARSE && g == 0.0f) return;
    m = lerp_fma(g, m, b1);
    v = lerp_fma(g * g, v, b2);
    const float denom = BIASED ? sqrtf(v) + eps : fmaf(sqrtf(v), rbc2, eps);
    p -= step_size * (m / denom);
}

// Coefficients of one update: from the launch arguments, or (graph replay) from row *step
// of a host-computed table [rows][2] = {lr / bc1, 1 / sqrt(bc2)}.
struct AdamCoef {
    float step_size, rbc2;
    const float* table;
    const int64_t* step;
    int64_t rows;
    unsigned* status;
};

__device__ __forceinline__ bool adam_coef(const AdamCoef& c, float& step_size, float& rbc2) {
    step_size = c.step_size; rbc2 = c.rbc2;
    if (!c.table) return true;
    const int64_t t = *c.step;
    if (t < 0 || t >= c.rows) {
        if (threadIdx.x == 0 && blockIdx.x == 0 && c.status) atomicOr(c.status, ERR_BAD_INDEX);
        return false;
    }
    step_size = c.table[2 * t];
    rbc2 = c.table[2 * t + 1];
    return true;
}

template <bool SPARSE, bool BIASED>
__global__ void adam_scalar_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ g,
                                   float* __restrict__ m, float* __restrict__ v, AdamCoef co, float b1, float b2,
                                   float eps)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float step_size, rbc2;
    if (!adam_coef(co, step_size, rbc2)) return;
    float P = p[i], Mv = m[i], Vv = v[i];
    adam_one<SPARSE, BIASED>(P, g[i], Mv, Vv, step_size, b1, b2, rbc2, eps);
    p[i] = P; m[i] = Mv; v[i] = Vv;
}

template <bool SPARSE, bool BIASED>
__global__ void adam_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, AdamCoef co, float b1, float b2, float eps)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t i4 = t * 4;
    if (i4 >= n) return;
    float step_size, rbc2;
    if (!adam_coef(co, step_size, rbc2)) return;
    if (i4 + 3 < n) {
        float4 P = reinterpret_cast<float4*>(p)[t];
        const float4 G = reinterpret_cast<const float4*>(g)[t];
        float4 Mv = reinterpret_cast<float4*>(m)[t];
        float4 Vv = reinterpret_cast<float4*>(v)[t];
        adam_one<SPARSE, BIASED>(P.x, G.x, Mv.x, Vv.x, step_size, b1, b2, rbc2, eps);
        adam_one<SPARSE, BIASED>(P.y, G.y, Mv.y, Vv.y, step_size, b1, b2, rbc2, eps);
        adam_one<SPARSE, BIASED>(P.z, G.z, Mv.z, Vv.z, step_size, b1, b2, rbc2, eps);
        adam_one<SPARSE, BIASED>(P.w, G.w, Mv.w, Vv.w, step_size, b1, b2, rbc2, eps);
        reinterpret_cast<float4*>(p)[t] = P;
        reinterpret_cast<float4*>(m)[t] = Mv;
        reinterpret_cast<float4*>(v)[t] = Vv;
    } else {
        for (int64_t i = i4; i < n; ++i) {
            float P = p[i], Mv = m[i], Vv = v[i];
            adam_one<SPARSE, BIASED>(P, g[i], Mv, Vv, step_size, b1, b2, rbc2, eps);
            p[i] = P; m[i] = Mv; v[i] = Vv;
        }
    }
}

static void adam_host_coefs(int biased, double step, double lr, double beta1, double beta2, float& step_size,
                            float& rbc2)
{
    if (biased) { step_size = (float)lr; rbc2 = 1.f; return; }
    const double bc1 = 1.0 - std::pow(beta1, step);
    const double bc2 = 1.0 - std::pow(beta2, step);
    step_size = (float)(lr / bc1);
    rbc2 = (float)(1.0 / std::sqrt(bc2));
}

static int adam_launch(int64_t numel, int biased, int sparse, float* param, const float* grad, float* exp_avg,
                       float* exp_avg_sq, const AdamCoef& co, double beta1, double beta2, float eps, void* stream)
{
    if (numel <= 0) return SVR_OK;
    if (!param || !grad || !exp_avg || !exp_avg_sq) return svr_fail(SVR_ERR_ARG, "adam: null argument");
    const bool aligned = (((uintptr_t)param | (uintptr_t)grad | (uintptr_t)exp_avg | (uintptr_t)exp_avg_sq) & 15) == 0;
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned g = nblk((numel + 3) / 4, 256);
    const float b1 = (float)beta1, b2 = (float)beta2;
    if (!aligned) {
        const unsigned gs = nblk(numel, 256);
        if (biased && sparse) adam_scalar_kernel<true, true><<<gs, 256, 0, st>>>(numel, param, grad, exp_avg, exp_avg_sq, co, b1, b2, eps);
        else if (biased) adam_scalar_kernel<false, true><<<gs, 256, 0, st>>>(numel, param, grad, exp_avg, exp_avg_sq, co, b1, b2, eps);
        else if (sparse) adam_scalar_kernel<true, false><<<gs, 256, 0, st>>>(numel, param, grad, exp_avg, exp_avg_sq, co, b1, b2, eps);
        else adam_scalar_kernel<false, false><<<gs, 256, 0, st>>>(numel, param, grad, exp_avg, exp_avg_sq, co, b1, b2, eps);
        LAUNCHED();
        return SVR_OK;
    }
    if (biased) {
        if (sparse) adam_kernel<true, true><<<g, 256, 0, st>>>(numel, param, grad, exp_avg, exp_avg_sq, co, b1, b2, eps);
        else adam_kernel<false, true><<<g, 256, 0, st>>>(numel, param, grad, exp_avg, exp_avg_sq, co, b1, b2, eps);
    } else {
        if (sparse) adam_kernel<true, false><<<g, 256, 0, st>>>(numel, param, grad, exp_avg, exp_avg_sq, co, b1, b2, eps);
        else adam_kernel<false, false><<<g, 256, 0, st>>>(numel, param, grad, exp_avg, exp_avg_sq, co, b1, b2, eps);
    }
    LAUNCHED();
    return SVR_OK;
}

extern "C" int svr_adam_step(int64_t numel, int biased, int sparse, float* param, const float* grad, float* exp_avg,
                             float* exp_avg_sq, double step, double lr, double beta1, double beta2, float eps,
                             void* stream)
{
    AdamCoef co{};
    adam_host_coefs(biased, step, lr, beta1, beta2, co.step_size, co.rbc2);
    return adam_launch(numel, biased, sparse, param, grad, exp_avg, exp_avg_sq, co, beta1, beta2, eps, stream);
}

extern "C" int svr_adam_coef_table(int biased, double lr, double beta1, double beta2, int64_t rows, float* table_host)
{
    if (rows <= 0 || !table_host) return svr_fail(SVR_ERR_ARG, "adam coefficient table");
    table_host[0] = 0.f;   // row 0: no step has that number
    table_host[1] = 1.f;
    for (int64_t t = 1; t < rows; ++t)
        adam_host_coefs(biased, (double)t, lr, beta1, beta2, table_host[2 * t], table_host[2 * t + 1]);
    return SVR_OK;
}

extern "C" int svr_adam_step_at(int64_t numel, int biased, int sparse, float* param, const float* grad,
                                float* exp_avg, float* exp_avg_sq, const float* coef_table, int64_t rows,
                                const int64_t* step, double beta1, double beta2, float eps, uint32_t* status,
                                void* stream)
{
    if (!coef_table || !step || rows <= 0) return svr_fail(SVR_ERR_ARG, "adam: null coefficient table or step");
    AdamCoef co{0.f, 1.f, coef_table, step, rows, status};
    return adam_launch(numel, biased, sparse, param, grad, exp_avg, exp_avg_sq, co, beta1, beta2, eps, stream);
}

// Parameters stored in bf16 (SH coefficients in the precision configuration): moments stay
// f32, the update is computed in f32 from the stored value and rounded to nearest.
template <bool SPARSE, bool BIASED>
__global__ void adam_bf16_kernel(int64_t n, __nv_bfloat16* __restrict__ p, const float* __restrict__ g,
                                 float* __restrict__ m, float* __restrict__ v, AdamCoef co, float b1, float b2,
                                 float eps)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float step_size, rbc2;
    if (!adam_coef(co, step_size, rbc2)) return;
    float P = __bfloat162float(p[i]), Mv = m[i], Vv = v[i];
    const float G = g[i];
    if (SPARSE && G == 0.0f) return;
    adam_one<SPARSE, BIASED>(P, G, Mv, Vv, step_size, b1, b2, rbc2, eps);
    p[i] = __float2bfloat16_rn(P);
    m[i] = Mv; v[i] = Vv;
}

static int adam_bf16_launch(int64_t numel, int biased, int sparse, uint16_t* param, const float* grad, float* m,
                            float* v, const AdamCoef& co, double beta1, double beta2, float eps, void* stream)
{
    if (numel <= 0) return SVR_OK;
    if (!param || !grad || !m || !v) return svr_fail(SVR_ERR_ARG, "adam bf16: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned gs = nblk(numel, 256);
    auto P = (__nv_bfloat16*)param;
    const float b1 = (float)beta1, b2 = (float)beta2;
    if (biased && sparse) adam_bf16_kernel<true, true><<<gs, 256, 0, st>>>(numel, P, grad, m, v, co, b1, b2, eps);
    else if (biased) adam_bf16_kernel<false, true><<<gs, 256, 0, st>>>(numel, P, grad, m, v, co, b1, b2, eps);
    else if (sparse) adam_bf16_kernel<true, false><<<gs, 256, 0, st>>>(numel, P, grad, m, v, co, b1, b2, eps);
    else adam_bf16_kernel<false, false><<<gs, 256, 0, st>>>(numel, P, grad, m, v, co, b1, b2, eps);
    LAUNCHED();
    return SVR_OK;
}

extern "C" int svr_adam_step_bf16(int64_t numel, int biased, int sparse, uint16_t* param, const float* grad,
                                  float* exp_avg, float* exp_avg_sq, double step, double lr, double beta1,
                                  double beta2, float eps, void* stream)
{
    AdamCoef co{};
    adam_host_coefs(biased, step, lr, beta1, beta2, co.step_size, co.rbc2);
    return adam_bf16_launch(numel, biased, sparse, param, grad, exp_avg, exp_avg_sq, co, beta1, beta2, eps, stream);
}

extern "C" int svr_adam_step_bf16_at(int64_t numel, int biased, int sparse, uint16_t* param, const float* grad,
                                     float* exp_avg, float* exp_avg_sq, const float* coef_table, int64_t rows,
                                     const int64_t* step, double beta1, double beta2, float eps, uint32_t* status,
                                     void* stream)
{
    if (!coef_table || !step || rows <= 0) return svr_fail(SVR_ERR_ARG, "adam: null coefficient table or step");
    AdamCoef co{0.f, 1.f, coef_table, step, rows, status};
    return adam_bf16_launch(numel, biased, sparse, param, grad, exp_avg, exp_avg_sq, co, beta1, beta2, eps, stream);
}

__global__ void counter_add_kernel(int64_t* c, int64_t d) { *c += d; }

extern "C" int svr_counter_add(int64_t* counter, int64_t delta, void* stream)
{
    if (!counter) return svr_fail(SVR_ERR_ARG, "counter: null");
    counter_add_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(counter, delta);
    LAUNCHED();
    return SVR_OK;
}
