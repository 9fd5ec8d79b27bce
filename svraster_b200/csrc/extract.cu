// Surface extraction on sm_100a: TSDF fusion of rendered depth maps into grid points and
// sparse marching cubes over the octree's voxels.
//
// TSDF: behaviour of src/utils/fuser_utils.py:54-156 (Fuser.integrate / tsdf).  The
// reference integrates one view at a time with a chain of tensor ops that gathers and
// scatters the accumulators per view; here one thread owns a grid point and folds every
// view of the batch into register accumulators, reading the point once and writing it once.
// Element-wise steps use round-to-nearest intrinsics where the reference rounds each tensor
// op separately, so fp32 results follow the reference's rounding; a float64-accumulator
// mode keeps the weighted running sums in double.
//
// Marching cubes: behaviour of cuda/svraster_cuda/marching_cubes.py:271-380.  Classify
// (case index, triangle count) -> scan -> emit face vertices in voxel order -> lexicographic
// unique of the vertex rows (three stable 32-bit radix passes) -> face indices.  Vertex
// interpolation uses uncontracted IEEE operations, so vertices and topology are bit-exact
// against the reference given the same SDF values.
#include <cmath>
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
        if (e_ != cudaSuccess) return svr_fail(SVR_ERR_CUDA, cudaGetErrorString(e_));    \
    } while (0)
#define LAUNCHED() do { svr_note_launch(1); CUDA_TRY(cudaGetLastError()); } while (0)

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
static inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// ============================================================================ TSDF
struct TsdfParams {
    const float* depth;      // packed per view: plane (view, depth_sel) of depth_ch channels
    int depth_ch, depth_sel;
    const float* alpha;      // may be NULL
    int alpha_ch, alpha_sel, alpha_is_T;
    const float* inv_trunc_pts;   // per point 1/trunc (may be NULL)
    float inv_trunc;              // scalar 1/trunc
    float keep;                   // |uv| <= 1 - crop_border
    float alpha_thres;
    int use_trunc, depth_weight, border_weight;
    float max_norm_dist;
    float border_c;               // 9 / sqrt(2)
    float proj[SVR_MAX_VIEWS][4]; // per view: 1/tanfovx, 1/tanfovy, 2 cx/W - 1, 2 cy/H - 1
};

// torch grid_sample, bilinear, zeros padding, align_corners=False (normalised uv in [-1, 1]).
__device__ __forceinline__ float sample_bilinear(const float* plane, int W, int H, float u, float v, bool from_T) {
    const float ix = ((u + 1.f) * W - 1) / 2;
    const float iy = ((v + 1.f) * H - 1) / 2;
    const int ix_nw = (int)floorf(ix), iy_nw = (int)floorf(iy);
    const int ix_ne = ix_nw + 1, iy_ne = iy_nw;
    const int ix_sw = ix_nw, iy_sw = iy_nw + 1;
    const int ix_se = ix_nw + 1, iy_se = iy_nw + 1;
    const float nw = (ix_se - ix) * (iy_se - iy);
    const float ne = (ix - ix_sw) * (iy_sw - iy);
    const float sw = (ix_ne - ix) * (iy - iy_ne);
    const float se = (ix - ix_nw) * (iy - iy_nw);
    auto at = [&](int y, int x) {
        const float t = plane[(int64_t)y * W + x];
        return from_T ? __fsub_rn(1.f, t) : t;
    };
    float out = 0.f;
    if (iy_nw >= 0 && iy_nw < H && ix_nw >= 0 && ix_nw < W) out += at(iy_nw, ix_nw) * nw;
    if (iy_ne >= 0 && iy_ne < H && ix_ne >= 0 && ix_ne < W) out += at(iy_ne, ix_ne) * ne;
    if (iy_sw >= 0 && iy_sw < H && ix_sw >= 0 && ix_sw < W) out += at(iy_sw, ix_sw) * sw;
    if (iy_se >= 0 && iy_se < H && ix_se >= 0 && ix_se < W) out += at(iy_se, ix_se) * se;
    return out;
}

template <typename Acc>
__global__ void __launch_bounds__(256) tsdf_kernel(const __grid_constant__ Views V, int64_t M,
                                                   const float3* __restrict__ xyz, const __grid_constant__ TsdfParams P,
                                                   Acc* __restrict__ wacc, Acc* __restrict__ sacc)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    const float3 p = xyz[i];
    const float inv_trunc = P.inv_trunc_pts ? P.inv_trunc_pts[i] : P.inv_trunc;
    Acc aw = wacc[i], as = sacc[i];
    for (int vi = 0; vi < V.n; ++vi) {
        const svr_view_t& view = V.v[vi];
        const float* m = view.w2c;
        // src/cameras.py:89-103 project(): pts @ R^T + t, uv = xy / z, scale and shift
        const float cx_ = fmaf(p.z, m[2], fmaf(p.y, m[1], p.x * m[0])) + m[3];
        const float cy_ = fmaf(p.z, m[6], fmaf(p.y, m[5], p.x * m[4])) + m[7];
        const float cz_ = fmaf(p.z, m[10], fmaf(p.y, m[9], p.x * m[8])) + m[11];
        const float sx = P.proj[vi][0], sy = P.proj[vi][1], shx = P.proj[vi][2], shy = P.proj[vi][3];
        const float u = __fadd_rn(__fmul_rn(__fdiv_rn(cx_, cz_), sx), shx);
        const float v = __fadd_rn(__fmul_rn(__fdiv_rn(cy_, cz_), sy), shy);
        if (!(fabsf(u) <= P.keep && fabsf(v) <= P.keep)) continue;
        const int W = view.width, H = view.height;
        const float* dplane = P.depth + (int64_t)P.depth_ch * view.pix_offset + (int64_t)P.depth_sel * W * H;
        const float frame_depth = sample_bilinear(dplane, W, H, u, v, false);
        const float* c2w = view.c2w;
        const float dx = __fsub_rn(p.x, c2w[3]), dy = __fsub_rn(p.y, c2w[7]), dz = __fsub_rn(p.z, c2w[11]);
        const float xyz_depth = fmaf(dz, c2w[10], fmaf(dy, c2w[6], dx * c2w[2]));
        float sdf = __fmul_rn(__fsub_rn(frame_depth, xyz_depth), inv_trunc);
        float w;
        if (P.use_trunc) {
            if (!(sdf >= -1.f)) continue;
            sdf = fminf(fmaxf(sdf, -1.f), 1.f);
            w = 1.f;
        } else {
            w = expf(-fminf(fabsf(sdf), P.max_norm_dist));
        }
        if (P.alpha) {
            const float* aplane = P.alpha + (int64_t)P.alpha_ch * view.pix_offset + (int64_t)P.alpha_sel * W * H;
            const float a = sample_bilinear(aplane, W, H, u, v, P.alpha_is_T != 0);
            w = __fmul_rn(w, a);
            if (!(a >= P.alpha_thres)) continue;
        }
        if (P.depth_weight) w = __fmul_rn(w, __frcp_rn(fmaxf(frame_depth, 0.1f)));
        if (P.border_weight) {
            const float r = __fsqrt_rn(__fadd_rn(__fmul_rn(u, u), __fmul_rn(v, v)));
            w = __fmul_rn(w, __frcp_rn(__fadd_rn(1.f, __fmul_rn(P.border_c, r))));
        }
        if (sizeof(Acc) == 8) {
            aw += (Acc)w;
            as += (Acc)w * (Acc)sdf;
        } else {
            aw = __fadd_rn(aw, w);
            as = __fadd_rn(as, __fmul_rn(w, sdf));
        }
    }
    wacc[i] = aw;
    sacc[i] = as;
}

extern "C" int svr_tsdf_integrate(const svr_view_t* views_host, const double* proj_host, int n_views, int64_t M,
                                  const float* xyz, const float* depth, int depth_ch, int depth_sel, const float* alpha,
                                  int alpha_ch, int alpha_sel, int alpha_is_T, const float* inv_trunc_pts, double trunc,
                                  double crop_border, float alpha_thres, int use_trunc, int depth_weight,
                                  int border_weight, float max_norm_dist, int fp64, void* weight_acc, void* sdf_acc,
                                  void* stream)
{
    if (n_views <= 0 || n_views > SVR_MAX_VIEWS) return svr_fail(SVR_ERR_ARG, "tsdf: view count");
    if (M <= 0) return SVR_OK;
    if (!xyz || !depth || !weight_acc || !sdf_acc) return svr_fail(SVR_ERR_ARG, "tsdf: null argument");
    if (depth_sel < 0 || depth_sel >= depth_ch || (alpha && (alpha_sel < 0 || alpha_sel >= alpha_ch)))
        return svr_fail(SVR_ERR_ARG, "tsdf: channel selection");
    Views V;
    memset(&V, 0, sizeof(V));
    V.n = n_views;
    int64_t pix = 0;
    for (int i = 0; i < n_views; ++i) {
        V.v[i] = views_host[i];
        if (V.v[i].width <= 0 || V.v[i].height <= 0 || !V.v[i].w2c || !V.v[i].c2w)
            return svr_fail(SVR_ERR_ARG, "tsdf: bad view");
        V.v[i].pix_offset = pix;
        pix += (int64_t)V.v[i].width * V.v[i].height;
    }
    TsdfParams P;
    P.depth = depth; P.depth_ch = depth_ch; P.depth_sel = depth_sel;
    P.alpha = alpha; P.alpha_ch = alpha_ch; P.alpha_sel = alpha_sel; P.alpha_is_T = alpha_is_T;
    P.inv_trunc_pts = inv_trunc_pts;
    P.inv_trunc = (float)(1.0 / (double)trunc);
    P.keep = (float)(1.0 - (double)crop_border);
    P.alpha_thres = alpha_thres;
    P.use_trunc = use_trunc; P.depth_weight = depth_weight; P.border_weight = border_weight;
    P.max_norm_dist = max_norm_dist;
    P.border_c = (float)(9.0 / std::sqrt(2.0));
    for (int i = 0; i < n_views; ++i) {
        // src/cameras.py:95-99: scale = 1 / tanfov, shift = 2 c_p - 1, evaluated in double and
        // applied in float32 (proj_host carries the double camera values when given)
        const double tx = proj_host ? proj_host[4 * i + 0] : (double)V.v[i].tanfovx;
        const double ty = proj_host ? proj_host[4 * i + 1] : (double)V.v[i].tanfovy;
        const double cxp = proj_host ? proj_host[4 * i + 2] : (double)V.v[i].cx / V.v[i].width;
        const double cyp = proj_host ? proj_host[4 * i + 3] : (double)V.v[i].cy / V.v[i].height;
        P.proj[i][0] = (float)(1.0 / tx);
        P.proj[i][1] = (float)(1.0 / ty);
        P.proj[i][2] = (float)(2.0 * cxp - 1.0);
        P.proj[i][3] = (float)(2.0 * cyp - 1.0);
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (fp64)
        tsdf_kernel<double><<<nblk(M, 256), 256, 0, st>>>(V, M, (const float3*)xyz, P, (double*)weight_acc,
                                                          (double*)sdf_acc);
    else
        tsdf_kernel<float><<<nblk(M, 256), 256, 0, st>>>(V, M, (const float3*)xyz, P, (float*)weight_acc,
                                                         (float*)sdf_acc);
    LAUNCHED();
    return SVR_OK;
}

// ============================================================================ marching cubes
__constant__ unsigned long long kMcCases[256] = {
#include "mc_table.inc"
};
// voxel edges as pairs of corner ids (corner = x<<2 | y<<1 | z), marching_cubes.py:336-349
__constant__ unsigned char kMcEdge[12][2] = {{0, 1}, {1, 5}, {5, 4}, {4, 0}, {2, 3}, {3, 7},
                                            {7, 6}, {6, 2}, {0, 2}, {1, 3}, {5, 7}, {4, 6}};

__device__ __forceinline__ int mc_case_tris(unsigned long long w) {
    int n = 0;
#pragma unroll
    for (int k = 0; k < 15; ++k) n += ((w >> (4 * k)) & 15ull) != 15ull;
    return n / 3;
}

// marching_cubes.py:324-328 (filter) and :352-354 (case index)
__global__ void mc_classify_kernel(int64_t n_vox, const int64_t* __restrict__ vox_key, int64_t M,
                                   const float* __restrict__ val, float iso, uint32_t* __restrict__ ntri,
                                   uint8_t* __restrict__ cube, unsigned* __restrict__ err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_vox) return;
    bool gt = false, lt = false, nan = false;
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int64_t g = vox_key[8 * i + k];
        if (g < 0 || g >= M) { atomicAdd(err, 1u); ntri[i] = 0; cube[i] = 0; return; }
        const float f = val[g];
        gt |= f > iso;
        lt |= f < iso;
        nan |= isnan(f);
        c |= (uint32_t)(f < iso) << k;
    }
    const bool keep = gt && lt && !nan;
    cube[i] = (uint8_t)c;
    ntri[i] = keep ? (uint32_t)mc_case_tris(kMcCases[c]) : 0u;
}

// marching_cubes.py:271-275 vert_interp with separately rounded ops (no FMA contraction)
template <bool FP64>
__device__ __forceinline__ float3 mc_interp(float iso, float3 p1, float3 p2, float v1, float v2) {
    if (FP64) {
        double r = ((double)iso - (double)v1) / ((double)v2 - (double)v1);
        if (fabsf(__fsub_rn(v1, v2)) < 1e-9f) r = 0.5;
        return f3((float)((double)p1.x + r * ((double)p2.x - (double)p1.x)),
                  (float)((double)p1.y + r * ((double)p2.y - (double)p1.y)),
                  (float)((double)p1.z + r * ((double)p2.z - (double)p1.z)));
    }
    float r = __fdiv_rn(__fsub_rn(iso, v1), __fsub_rn(v2, v1));
    if (fabsf(__fsub_rn(v1, v2)) < 1e-9f) r = 0.5f;
    return f3(__fadd_rn(p1.x, __fmul_rn(r, __fsub_rn(p2.x, p1.x))),
              __fadd_rn(p1.y, __fmul_rn(r, __fsub_rn(p2.y, p1.y))),
              __fadd_rn(p1.z, __fmul_rn(r, __fsub_rn(p2.z, p1.z))));
}

__device__ __forceinline__ uint32_t float_order_key(float f) {
    if (f == 0.f) f = 0.f;   // -0 and +0 compare equal in the reference's unique
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// marching_cubes.py:355-370: triangles of each voxel's case, vertices in table order
template <bool FP64>
__global__ void mc_emit_kernel(int64_t n_vox, const int64_t* __restrict__ vox_key, const float* __restrict__ val,
                               const float3* __restrict__ xyz, float iso, const uint32_t* __restrict__ ntri,
                               const uint32_t* __restrict__ scan, const uint8_t* __restrict__ cube,
                               float3* __restrict__ fverts, uint32_t* __restrict__ kz, uint32_t* __restrict__ idx)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_vox) return;
    const uint32_t nt = ntri[i];
    if (nt == 0) return;
    const uint64_t w = kMcCases[cube[i]];
    float v[8];
    float3 p[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int64_t g = vox_key[8 * i + k];
        v[k] = val[g];
        p[k] = xyz[g];
    }
    uint32_t out = 3u * (scan[i] - nt);
    for (uint32_t t = 0; t < 3 * nt; ++t) {
        const int e = (int)((w >> (4 * t)) & 15ull);
        const int a = kMcEdge[e][0], b = kMcEdge[e][1];
        const float3 q = mc_interp<FP64>(iso, p[a], p[b], v[a], v[b]);
        fverts[out] = q;
        kz[out] = float_order_key(q.z);
        idx[out] = out;
        ++out;
    }
}

__global__ void mc_gather_key_kernel(int64_t n, const uint32_t* __restrict__ idx, const float3* __restrict__ fverts,
                                     int axis, uint32_t* __restrict__ key)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 q = fverts[idx[i]];
    key[i] = float_order_key(axis == 0 ? q.x : (axis == 1 ? q.y : q.z));
}

__global__ void mc_flag_kernel(int64_t n, const uint32_t* __restrict__ idx, const float3* __restrict__ fverts,
                               uint32_t* __restrict__ flag)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i == 0) { flag[0] = 1; return; }
    const float3 a = fverts[idx[i]], b = fverts[idx[i - 1]];
    flag[i] = (a.x != b.x || a.y != b.y || a.z != b.z) ? 1u : 0u;
}

__global__ void mc_write_kernel(int64_t n, const uint32_t* __restrict__ idx, const float3* __restrict__ fverts,
                                const uint32_t* __restrict__ flag, const uint32_t* __restrict__ uid,
                                float3* __restrict__ verts, int64_t* __restrict__ faces)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t u = uid[i] - 1;      // inclusive scan of the flags
    const uint32_t src = idx[i];
    if (flag[i]) verts[u] = fverts[src];
    faces[src] = (int64_t)u;
}

struct McWs {
    size_t err, ntri, scan, cube, scan_tmp, scan_tmp_bytes, fverts, k0, k1, i0, i1, flag, uid, sort_tmp, sort_tmp_bytes,
        total;
};
static McWs mc_ws(int64_t n_vox, int64_t n_tri) {
    McWs L{};
    const int64_t nv = n_vox > 0 ? n_vox : 1;
    const int64_t nf = n_tri > 0 ? 3 * n_tri : 1;
    size_t st = 0, rt = 0;
    cub::DeviceScan::InclusiveSum(nullptr, st, (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)nv);
    size_t st2 = 0;
    cub::DeviceScan::InclusiveSum(nullptr, st2, (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)nf);
    st = st > st2 ? st : st2;
    cub::DeviceRadixSort::SortPairs(nullptr, rt, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)nf);
    size_t off = 0;
    L.err = off; off += 256;
    L.ntri = off; off = align_up(off + 4 * (size_t)nv, 256);
    L.scan = off; off = align_up(off + 4 * (size_t)nv, 256);
    L.cube = off; off = align_up(off + (size_t)nv, 256);
    L.scan_tmp = off; L.scan_tmp_bytes = st; off = align_up(off + st, 256);
    L.fverts = off; off = align_up(off + 12 * (size_t)nf, 256);
    L.k0 = off; off = align_up(off + 4 * (size_t)nf, 256);
    L.k1 = off; off = align_up(off + 4 * (size_t)nf, 256);
    L.i0 = off; off = align_up(off + 4 * (size_t)nf, 256);
    L.i1 = off; off = align_up(off + 4 * (size_t)nf, 256);
    L.flag = off; off = align_up(off + 4 * (size_t)nf, 256);
    L.uid = off; off = align_up(off + 4 * (size_t)nf, 256);
    L.sort_tmp = off; L.sort_tmp_bytes = rt; off = align_up(off + rt, 256);
    L.total = off;
    return L;
}

extern "C" size_t svr_mc_workspace_bytes(int64_t n_vox, int64_t n_tri) { return mc_ws(n_vox, n_tri).total; }

extern "C" int svr_mc_count(int64_t n_vox, const int64_t* vox_key, int64_t M, const float* grid_val, float iso,
                            void* workspace, int64_t* n_tri_host, void* stream)
{
    *n_tri_host = 0;
    if (n_vox <= 0) return SVR_OK;
    if (n_vox >= (1ll << 31)) return svr_fail(SVR_ERR_ARG, "mc: too many voxels for one call");
    cudaStream_t st = (cudaStream_t)stream;
    McWs L = mc_ws(n_vox, 0);
    char* w = (char*)workspace;
    CUDA_TRY(cudaMemsetAsync(w + L.err, 0, 4, st));
    mc_classify_kernel<<<nblk(n_vox, 256), 256, 0, st>>>(n_vox, vox_key, M, grid_val, iso, (uint32_t*)(w + L.ntri),
                                                         (uint8_t*)(w + L.cube), (unsigned*)(w + L.err));
    LAUNCHED();
    size_t tb = L.scan_tmp_bytes;
    CUDA_TRY(cub::DeviceScan::InclusiveSum(w + L.scan_tmp, tb, (const uint32_t*)(w + L.ntri), (uint32_t*)(w + L.scan),
                                           (int)n_vox, st));
    uint32_t total = 0, bad = 0;
    CUDA_TRY(cudaMemcpyAsync(&total, w + L.scan + 4 * (size_t)(n_vox - 1), 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(&bad, w + L.err, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (bad) return svr_fail(SVR_ERR_ARG, "mc: vox_key holds grid indices outside [0, M)");
    *n_tri_host = total;
    return SVR_OK;
}

extern "C" int svr_mc_emit(int64_t n_vox, const int64_t* vox_key, const float* grid_val, const float* grid_xyz,
                           float iso, int64_t n_tri, int fp64, void* workspace, float* verts, int64_t* faces,
                           int64_t* n_verts_host, void* stream)
{
    *n_verts_host = 0;
    if (n_vox <= 0 || n_tri <= 0) return SVR_OK;
    if (3 * n_tri >= (1ll << 31)) return svr_fail(SVR_ERR_ARG, "mc: too many triangles for one call");
    cudaStream_t st = (cudaStream_t)stream;
    McWs L = mc_ws(n_vox, n_tri);
    // count-pass arrays sit at the same offsets whatever n_tri is
    char* w = (char*)workspace;
    const int64_t nf = 3 * n_tri;
    float3* fv = (float3*)(w + L.fverts);
    uint32_t *k0 = (uint32_t*)(w + L.k0), *k1 = (uint32_t*)(w + L.k1);
    uint32_t *i0 = (uint32_t*)(w + L.i0), *i1 = (uint32_t*)(w + L.i1);
    if (fp64)
        mc_emit_kernel<true><<<nblk(n_vox, 128), 128, 0, st>>>(n_vox, vox_key, grid_val, (const float3*)grid_xyz, iso,
            (const uint32_t*)(w + L.ntri), (const uint32_t*)(w + L.scan), (const uint8_t*)(w + L.cube), fv, k0, i0);
    else
        mc_emit_kernel<false><<<nblk(n_vox, 128), 128, 0, st>>>(n_vox, vox_key, grid_val, (const float3*)grid_xyz, iso,
            (const uint32_t*)(w + L.ntri), (const uint32_t*)(w + L.scan), (const uint8_t*)(w + L.cube), fv, k0, i0);
    LAUNCHED();
    // lexicographic (x, y, z) order by three stable LSD passes: z, then y, then x
    size_t tb = L.sort_tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(w + L.sort_tmp, tb, k0, k1, i0, i1, (int)nf, 0, 32, st));
    mc_gather_key_kernel<<<nblk(nf, 256), 256, 0, st>>>(nf, i1, fv, 1, k0);
    LAUNCHED();
    tb = L.sort_tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(w + L.sort_tmp, tb, k0, k1, i1, i0, (int)nf, 0, 32, st));
    mc_gather_key_kernel<<<nblk(nf, 256), 256, 0, st>>>(nf, i0, fv, 0, k0);
    LAUNCHED();
    tb = L.sort_tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(w + L.sort_tmp, tb, k0, k1, i0, i1, (int)nf, 0, 32, st));
    uint32_t* flag = (uint32_t*)(w + L.flag);
    uint32_t* uid = (uint32_t*)(w + L.uid);
    mc_flag_kernel<<<nblk(nf, 256), 256, 0, st>>>(nf, i1, fv, flag);
    LAUNCHED();
    tb = L.scan_tmp_bytes;
    CUDA_TRY(cub::DeviceScan::InclusiveSum(w + L.scan_tmp, tb, flag, uid, (int)nf, st));
    mc_write_kernel<<<nblk(nf, 256), 256, 0, st>>>(nf, i1, fv, flag, uid, (float3*)verts, faces);
    LAUNCHED();
    uint32_t nu = 0;
    CUDA_TRY(cudaMemcpyAsync(&nu, uid + nf - 1, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *n_verts_host = nu;
    return SVR_OK;
}
