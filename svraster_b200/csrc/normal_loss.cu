// Normal-from-depth consistency losses with their gradients, all views in one launch.
//
// Behaviour of src/cameras.py:104-127 (depth2pts, depth2normal) and
// src/utils/loss_utils.py:345-407 (NormalDepthConsistencyLoss: rendered normal against the
// alpha-weighted negated normal of the mean-depth surface, tolerance mask on the angle to the
// viewing ray; NormalMedianConsistencyLoss: against the negated normal of the median-depth
// surface).  The reference builds the point map, the finite differences, the cross product
// and the loss as separate torch ops and differentiates them with autograd.  Here one CTA
// owns a 32x8 pixel tile: it stages the back-projected points of the tile plus a 2*pad halo
// in shared memory, computes for the tile plus a pad halo each pixel's pseudo-normal, loss
// term and the gradients with respect to its two difference vectors, then gathers every
// tile pixel's depth gradient from the (up to) four neighbours whose differences used it.
// The loss (per view, float64) and both gradients come out of the same pass; the gradients
// are added into the caller's upstream planes (depth plane 0 or 2, normal planes), so the
// pass can run between the render forward and the render adjoint.
#include <cstdint>
#include <string>

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

namespace {

constexpr int NTW = 32, NTH = 8, MAXPAD = 4;

__device__ __forceinline__ float3 cross3(float3 a, float3 b)
{
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// PAD = ks / 2 fixes the halo, so shared memory holds exactly the tile's stencil
template <int PAD, bool ALPHA>
__global__ void __launch_bounds__(NTW * NTH, 4) normal_loss_kernel(Views V, int dplane, float tol_cos, float weight,
                                                                   const float* __restrict__ depth,
                                                                   const float* __restrict__ normal,
                                                                   const float* __restrict__ Tm,
                                                                   double* __restrict__ loss_out,
                                                                   float* __restrict__ grad_depth,
                                                                   float* __restrict__ grad_normal)
{
    constexpr int AW = NTW + 4 * PAD, AH = NTH + 4 * PAD;     // staged points
    constexpr int BW = NTW + 2 * PAD, BH = NTH + 2 * PAD;     // per-pixel difference gradients
    __shared__ float sP[3][AH * AW];
    __shared__ float sGx[3][BH * BW];
    __shared__ float sGy[3][BH * BW];
    __shared__ float sU[AW], sV[AH];                          // camera-space ray x / y per column / row
    __shared__ float sM[12];
    __shared__ double sLoss[NTW * NTH / 32];
    const svr_view_t& view = V.v[blockIdx.z];
    const int W = view.width, H = view.height;
    const int x0 = blockIdx.x * NTW, y0 = blockIdx.y * NTH;
    if (x0 >= W || y0 >= H) return;                       // the whole CTA leaves together
    const int tid = threadIdx.x;
    if (tid < 12) sM[tid] = view.c2w[tid];
    // cuda/src/utils.cu:47-72 (compute_rd): camera-space x depends on the column only, y on
    // the row only; the same expressions, once per column / row of the staged region
    if (tid < AW) sU[tid] = ((float)(x0 - 2 * PAD + tid) + 0.5f - view.cx) * 2.f * view.tanfovx / (float)W;
    if (tid >= 64 && tid < 64 + AH)
        sV[tid - 64] = ((float)(y0 - 2 * PAD + tid - 64) + 0.5f - view.cy) * 2.f * view.tanfovy / (float)H;
    __syncthreads();
    auto ray = [&](int ax, int ay) {
        const float u = sU[ax], w = sV[ay];
        return f3(sM[0] * u + sM[1] * w + sM[2], sM[4] * u + sM[5] * w + sM[6], sM[8] * u + sM[9] * w + sM[10]);
    };
    const int64_t HW = (int64_t)W * H;
    const float* dp = depth + 4 * view.pix_offset + dplane * HW;
    const float* np_ = normal + 3 * view.pix_offset;
    const float* tp = ALPHA ? Tm + view.pix_offset : nullptr;
    const float inv_hw = 1.f / (float)HW;
    const float3 cam = f3(sM[3], sM[7], sM[11]);

    // points of the tile and a 2*PAD halo
    for (int i = tid; i < AW * AH; i += blockDim.x) {
        const int ax = i % AW, ay = i / AW;
        const int x = x0 - 2 * PAD + ax, y = y0 - 2 * PAD + ay;
        float3 p = f3(0.f, 0.f, 0.f);
        if (x >= 0 && x < W && y >= 0 && y < H) {
            const float3 r = ray(ax, ay);
            const float d = dp[(int64_t)y * W + x];
            p = f3(cam.x + r.x * d, cam.y + r.y * d, cam.z + r.z * d);
        }
        sP[0][i] = p.x; sP[1][i] = p.y; sP[2][i] = p.z;
    }
    __syncthreads();

    // per pixel of the tile and a PAD halo: pseudo-normal, loss term, difference gradients
    float loss = 0.f;
    for (int i = tid; i < BW * BH; i += blockDim.x) {
        const int bx = i % BW, by = i / BW;
        const int x = x0 - PAD + bx, y = y0 - PAD + by;
        float3 gx = f3(0.f, 0.f, 0.f), gy = f3(0.f, 0.f, 0.f);
        if (x >= PAD && x < W - PAD && y >= PAD && y < H - PAD) {
            const int ac = (by + PAD) * AW + bx + PAD;            // this pixel in the staged points
            auto P = [&](int a) { return f3(sP[0][a], sP[1][a], sP[2][a]); };
            const float3 dx = P(ac + PAD) - P(ac - PAD);
            const float3 dy = P(ac + PAD * AW) - P(ac - PAD * AW);
            const float3 c = cross3(dx, dy);
            const float cn = sqrtf(c.x * c.x + c.y * c.y + c.z * c.z);
            const float rden = __frcp_rn(cn > 1e-12f ? cn : 1e-12f);
            const float3 n = f3(c.x * rden, c.y * rden, c.z * rden);
            float s = 1.f;
            if (tol_cos > 0.f) {
                const float3 pd = P(ac) - cam;
                const float pn = sqrtf(pd.x * pd.x + pd.y * pd.y + pd.z * pd.z);
                const float rpn = __frcp_rn(pn > 1e-12f ? pn : 1e-12f);
                const float dot = n.x * (pd.x * rpn) + n.y * (pd.y * rpn) + n.z * (pd.z * rpn);
                if (!(dot > tol_cos)) s = 0.f;
            }
            const int64_t q = (int64_t)y * W + x;
            const float alpha = ALPHA ? 1.f - tp[q] : 1.f;
            if (ALPHA) s *= alpha;
            const float3 N = f3(-n.x * s, -n.y * s, -n.z * s);
            if (N.x != 0.f || N.y != 0.f || N.z != 0.f) {
                const float3 nr = f3(np_[q], np_[HW + q], np_[2 * HW + q]);
                const bool own = bx >= PAD && bx < PAD + NTW && by >= PAD && by < PAD + NTH;
                if (own) {
                    const float target = ALPHA ? alpha * alpha : 1.f;
                    loss += target - (nr.x * N.x + nr.y * N.y + nr.z * N.z);
                    const float gw = weight * inv_hw;
                    grad_normal[3 * view.pix_offset + q] += -N.x * gw;
                    grad_normal[3 * view.pix_offset + HW + q] += -N.y * gw;
                    grad_normal[3 * view.pix_offset + 2 * HW + q] += -N.z * gw;
                }
                const float k = s * weight * inv_hw;
                const float3 g = f3(k * nr.x, k * nr.y, k * nr.z);
                // through the clamped normalisation (the clamp passes no gradient to the norm)
                float3 gc;
                if (cn > 1e-12f) {
                    const float ng = n.x * g.x + n.y * g.y + n.z * g.z;
                    gc = f3((g.x - n.x * ng) * rden, (g.y - n.y * ng) * rden, (g.z - n.z * ng) * rden);
                } else {
                    gc = f3(g.x * 1e12f, g.y * 1e12f, g.z * 1e12f);
                }
                gx = cross3(dy, gc);        // dL/d dx
                gy = cross3(gc, dx);        // dL/d dy
            }
        }
        sGx[0][i] = gx.x; sGx[1][i] = gx.y; sGx[2][i] = gx.z;
        sGy[0][i] = gy.x; sGy[1][i] = gy.y; sGy[2][i] = gy.z;
    }
    __syncthreads();

    // each tile pixel's depth gradient from the neighbours whose differences used its point
    {
        const int tx = tid % NTW, ty = tid / NTW;
        const int x = x0 + tx, y = y0 + ty;
        if (x < W && y < H) {
            const int bc = (ty + PAD) * BW + tx + PAD;
            float3 gp;
            gp.x = sGx[0][bc - PAD] - sGx[0][bc + PAD] + sGy[0][bc - PAD * BW] - sGy[0][bc + PAD * BW];
            gp.y = sGx[1][bc - PAD] - sGx[1][bc + PAD] + sGy[1][bc - PAD * BW] - sGy[1][bc + PAD * BW];
            gp.z = sGx[2][bc - PAD] - sGx[2][bc + PAD] + sGy[2][bc - PAD * BW] - sGy[2][bc + PAD * BW];
            const float3 r = ray(tx + 2 * PAD, ty + 2 * PAD);
            const int64_t q = (int64_t)y * W + x;
            grad_depth[4 * view.pix_offset + dplane * HW + q] += r.x * gp.x + r.y * gp.y + r.z * gp.z;
        }
    }
    double l = (double)loss;
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((tid & 31) == 0) sLoss[tid >> 5] = l;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < NTW * NTH / 32; ++w) t += sLoss[w];
        if (t != 0.0) atomicAdd(loss_out + blockIdx.z, t * (double)weight / (double)HW);
    }
}

template <int PAD>
void launch_pad(dim3 grid, cudaStream_t st, const Views& V, int mode, float tol_cos, float weight,
                const float* depth, const float* normal, const float* T, double* loss_out, float* grad_depth,
                float* grad_normal)
{
    if (mode == 0)
        normal_loss_kernel<PAD, true><<<grid, NTW * NTH, 0, st>>>(V, 0, tol_cos, weight, depth, normal, T, loss_out,
                                                                  grad_depth, grad_normal);
    else
        normal_loss_kernel<PAD, false><<<grid, NTW * NTH, 0, st>>>(V, 2, -1.f, weight, depth, normal, nullptr,
                                                                   loss_out, grad_depth, grad_normal);
}

}  // namespace

extern "C" int svr_normal_depth_loss(const svr_view_t* views_host, int n_views, int mode, int ks, float tol_cos,
                                     float weight, const float* depth, const float* normal, const float* T,
                                     double* loss_out, float* grad_depth, float* grad_normal, void* stream)
{
    if (n_views <= 0) return SVR_OK;
    if (!views_host || n_views > SVR_MAX_VIEWS || (mode != 0 && mode != 1) || ks < 1 || ks % 2 == 0 ||
        ks / 2 > MAXPAD)
        return svr_fail(SVR_ERR_ARG, "normal-depth loss: views, mode (0 mean, 1 median) or ks (odd, <= 9)");
    if (!depth || !normal || !loss_out || !grad_depth || !grad_normal || (mode == 0 && !T))
        return svr_fail(SVR_ERR_ARG, "normal-depth loss: null argument");
    Views V;
    V.n = n_views;
    int mw = 0, mh = 0;
    for (int i = 0; i < n_views; ++i) {
        V.v[i] = views_host[i];
        if (!V.v[i].c2w || V.v[i].width <= 0 || V.v[i].height <= 0)
            return svr_fail(SVR_ERR_ARG, "normal-depth loss: a view without c2w or with an empty image");
        mw = V.v[i].width > mw ? V.v[i].width : mw;
        mh = V.v[i].height > mh ? V.v[i].height : mh;
    }
    const dim3 grid((mw + NTW - 1) / NTW, (mh + NTH - 1) / NTH, n_views);
    cudaStream_t st = (cudaStream_t)stream;
    switch (ks / 2) {
    case 0: launch_pad<0>(grid, st, V, mode, tol_cos, weight, depth, normal, T, loss_out, grad_depth, grad_normal); break;
    case 1: launch_pad<1>(grid, st, V, mode, tol_cos, weight, depth, normal, T, loss_out, grad_depth, grad_normal); break;
    case 2: launch_pad<2>(grid, st, V, mode, tol_cos, weight, depth, normal, T, loss_out, grad_depth, grad_normal); break;
    case 3: launch_pad<3>(grid, st, V, mode, tol_cos, weight, depth, normal, T, loss_out, grad_depth, grad_normal); break;
    default: launch_pad<4>(grid, st, V, mode, tol_cos, weight, depth, normal, T, loss_out, grad_depth, grad_normal); break;
    }
    svr_note_launch(1);
    CUDA_TRY(cudaGetLastError());
    return SVR_OK;
}
