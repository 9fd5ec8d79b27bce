// Forward tile render with a record-parallel filter and dense pair evaluation.
//
// Same behaviour and per-pair arithmetic as render_fwd_kernel (cuda/src/forward.cu:41-564,
// SDF branch); the work is distributed differently.  The records of a tile still stream
// through a ring of bulk-copied shared-memory slots, but every slot is consumed by the whole
// CTA in three phases:
//  * F (filter, one record per two threads): the record's pixel rectangle inside the tile,
//    the octant and liveness of each pixel and the slab test give the record's candidate
//    pixels, set in per-pixel 128-bit candidate masks with shared-memory atomics; records
//    with a large rectangle are enumerated by a whole warp.  A record costs a handful of
//    instructions unless it has candidates, where the warp-wide filter cost every warp of
//    the tile a 32x32 bit transpose per 32 records;
//  * P (pairs): the candidate pairs are numbered (pixel-major, record order) and evaluated
//    one pair per lane -- per warp, 32 at a time, or (CTAW, the default) over the whole CTA,
//    a window of 256 pairs at a time -- so the SDF / logistic-CDF arithmetic runs on full
//    warps however unevenly the pixels' candidates are spread;
//  * C (compositing, per pixel): each pixel folds its own pairs in record order with the
//    forward's expressions, so every output is bit-identical to render_fwd_kernel's.
// Per-warp variant: a CTA barrier when the slot has arrived (every warp is then through the
// previous slot, which is refilled) and one after F.  CTA-wide variant: no barrier at the slot's
// start -- the candidate masks alternate between two buffers by slot parity, the record normals
// are computed where a pair uses them, and the refill of the previous slot waits for the
// barrier after F -- so a warp filters slot b + 1 while others still composite slot b; then the
// barrier of the pair numbering and one per window.  The CTA-wide variant also stores each
// slot's masks (one 16-byte row per pixel, the candidate rows) for the adjoint.
#pragma once

#include <climits>

#include "render_kernels.cuh"
#include "svr_common.cuh"

namespace svr {

constexpr uint32_t PIX_LIVE = 8u;           // pixel flag in the filter's ray table: still compositing
constexpr int SMALL_RECT = 16;              // rectangles above this many pixels: warp-wide filter

template <int RING>
struct alignas(128) PairFwdSmem {
    Rec buf[RING][BATCH];
    uint64_t full[RING];
    uint32_t armed[RING];
    float4 pray[BLOCK];          // per tile pixel slot: rd_inv, octant | PIX_LIVE
    float4 pdir[BLOCK];          // rd, 1 / |camera ray|
    // candidate records of a slot, per pixel; the CTA-wide kernel alternates the two buffers
    // by slot parity, so that a warp can filter slot b + 1 while others still composite b
    alignas(16) uint32_t mask[2][BLOCK][4];
    union {
        float2 res[NWARP][32];   // per-warp windows: alpha and depth value of a warp's pairs
        float2 cres[2][BLOCK];   // CTA-wide windows: the pairs of a window (two buffers)
    };
    uint32_t red[NWARP];
    int ppre[BLOCK];             // CTA-wide windows: each thread's pair offset within its warp
    int wcnt[NWARP];             // and the warps' pair counts
    int fail;                    // a wait of this CTA timed out
};

// Position of the k-th (from 0) set bit of w (k < popc(w)).
__device__ __forceinline__ int kth_set_bit(uint32_t w, int k) {
    int pos = 0;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const int c = __popc(w & ((1u << s) - 1u));
        if (k >= c) { k -= c; w >>= s; pos += s; }
    }
    return pos;
}

// A pixel's 128-bit candidate mask as one 16-byte shared-memory access.
__device__ __forceinline__ uint4 load_row(const uint32_t (&m)[4]) { return *reinterpret_cast<const uint4*>(m); }
__device__ __forceinline__ void store_row(uint32_t (&m)[4], uint4 v) { *reinterpret_cast<uint4*>(m) = v; }

// Shared-memory slot of tile pixel p = dy * 16 + dx in the per-pixel arrays (rays, masks,
// upstream gradients): bits 3 and 5 of p are folded into its low bits, so that the 8 lanes of a
// quarter-warp reading their own pixels' 16-byte rows (lattice or 8x4 blocks) hit 8 different
// bank groups.  An involution, hence a bijection of [0, 256).
__device__ __forceinline__ int pix_slot(int p) { return p ^ ((((p >> 3) & 1) << 1) | ((p >> 5) & 1)); }

// Pixel (dx, dy) of lane `lane` of warp `warp` in a 16x16 tile.  LATTICE: every warp owns a
// stride-4 x stride-2 lattice spread over the whole tile, so the warps' pair counts are alike
// and the CTA barriers wait less on the warp holding the silhouette; else 8x4 blocks.
template <bool LATTICE>
__device__ __forceinline__ void pair_pixel(int warp, int lane, int& dx, int& dy) {
    if (LATTICE) {
        dx = (warp & 3) + 4 * (lane & 3);
        dy = (warp >> 2) + 2 * (lane >> 2);
    } else {
        dx = (warp & 1) * 8 + (lane & 7);
        dy = (warp >> 1) * 4 + (lane >> 3);
    }
}

// Corner-difference normal of a record's SDF corners (forward.cu:422-432, backward.cu:
// 607-618), with its reciprocal norm in .w.
__device__ __forceinline__ float4 record_normal(const Rec& rec) {
    const float* g = rec.g;
    const float lin_nx = (g[4] + g[5] + g[6] + g[7]) - (g[0] + g[1] + g[2] + g[3]);
    const float lin_ny = (g[2] + g[3] + g[6] + g[7]) - (g[0] + g[1] + g[4] + g[5]);
    const float lin_nz = (g[1] + g[3] + g[5] + g[7]) - (g[0] + g[2] + g[4] + g[6]);
    return make_float4(lin_nx, lin_ny, lin_nz, safe_rnorm(lin_nx, lin_ny, lin_nz));
}

// A record none of whose (pixel, record) pairs can reach MIN_ALPHA, by its SDF corners alone.
// The packing stores the min / max corner widened by 5% of the corner spread plus 1e-4 of the
// largest corner (points rounded just outside the voxel); if every point of the voxel then has
// s * sdf >= 16, the logistic CDF at entry and exit is within 1.2e-7 of 1 and alpha <= 1.2e-7,
// and if s * sdf <= -30 the CDF at entry is below 1e-13 and alpha < 1e-7 (its denominator
// keeps 1e-6).  The forward and the adjoint skip a pair with alpha < MIN_ALPHA (1e-5)
// entirely (forward.cu:304, backward.cu:428), so such a record is given no candidate pixels:
// the outputs are the same bit for bit.  A NaN corner makes every evaluation NaN (alpha 0),
// so dropping such a record is exact too; infinite corners give an infinite margin and keep
// the record.
__device__ __forceinline__ bool record_dead(const Rec& rec, float s_val) {
    // rec.sdf_lo / sdf_hi: the min / max corner widened by the margin, set by the packing
    return s_val > 0.f && (s_val * rec.sdf_lo >= 16.f || s_val * rec.sdf_hi <= -30.f);
}

// Filter test of one (record, pixel): live pixel, matching octant, slab test passed.
__device__ __forceinline__ bool filter_hit(const float4 pr, uint32_t q, float3 c, float l, float3 ro) {
    const uint32_t f = __float_as_uint(pr.w);
    if (!(f & PIX_LIVE) || (f & 7u) != q) return false;
    const float2 ab = ray_box(c, l, ro, f3(pr.x, pr.y, pr.z));
    return !(ab.x > ab.y);
}

// Owner of pair i (< the CTA's pair total) of a CTA-wide numbering (thread-major, each
// thread's pairs in record order): the thread t and i's rank k among t's pairs, from the
// warps' pair counts and the per-thread offsets within the warp.
__device__ __forceinline__ void cta_pair_owner(const int* wcnt, const int* ppre, int i, int& t, int& k) {
    int acc = 0, ow = 0, oacc = 0;
#pragma unroll
    for (int q = 0; q < NWARP; ++q) {
        if (acc <= i) { ow = q; oacc = acc; }
        acc += wcnt[q];
    }
    const int x = i - oacc;
    const int* pp = ppre + ow * 32;
    int l = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1)
        if (pp[l + step] <= x) l += step;
    t = ow * 32 + l;
    k = x - pp[l];
}

// The evaluation of one (pixel, record) pair of the forward (forward.cu:255-306, as
// render_fwd_kernel): alpha and the depth value.
template <int NS, bool DEPTH>
__device__ __forceinline__ float2 fwd_pair_eval(const Rec& r, float3 ro, float3 rd, float3 rd_inv, float s_val) {
    const float3 vox_c = f3(r.cx, r.cy, r.cz);
    const float vox_l = r.len;
    const float2 ab = ray_box(vox_c, vox_l, ro, rd_inv);
    const float a = ab.x, bb = ab.y;
    float g[8];
#pragma unroll
    for (int qq = 0; qq < 8; ++qq) g[qq] = r.g[qq];
    float w8[8];
    float local_a[NS > 1 ? NS : 1];
    const float vox_l_inv = 1.f / vox_l;
    const float3 p_entry = ro + a * rd;
    const float3 P_step = (bb - a) * rd / (float)NS;
    const float3 qt_entry = (p_entry - (vox_c - 0.5f * vox_l)) * vox_l_inv;
    const float3 qt_step = P_step * vox_l_inv;
    tri_weights(qt_entry, w8);
    float phi_former = 1.f / (1.f + expf(-s_val * interp8(g, w8)));
    const float phi_entry = phi_former;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        const float3 qt_curr = qt_entry + qt_step * (float)(s + 1);
        tri_weights(qt_curr, w8);
        const float phi_curr = 1.f / (1.f + expf(-s_val * interp8(g, w8)));
        if (DEPTH && NS > 1) local_a[s] = fmaxf((phi_former - phi_curr) / (phi_former + 1e-6f), 0.f);
        phi_former = phi_curr;
    }
    const float alpha = fmaxf((phi_entry - phi_former) / (phi_entry + 1e-6f), 0.f);
    float dval = 0.f;
    if (DEPTH && !(alpha < MIN_ALPHA)) {
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
    }
    return make_float2(alpha, dval);
}

template <int NS, bool DEPTH, bool NORMAL, bool MAXW, int RING = 3, int MINB = 4, bool COUNT = false,
          bool LATTICE = true, bool CTAW = false>
__global__ void __launch_bounds__(BLOCK, MINB) render_fwd_pairs_kernel(
    const __grid_constant__ Views V, const uint32_t* __restrict__ order, const uint2* __restrict__ ranges,
    const Rec* __restrict__ recs, const float* __restrict__ s_ptr, uint32_t* __restrict__ tile_last,
    uint32_t* __restrict__ n_contrib,
    float* __restrict__ out_color, float* __restrict__ out_depth, float* __restrict__ out_normal,
    float* __restrict__ out_T, float* __restrict__ max_w, int64_t max_w_stride, unsigned* __restrict__ status,
    unsigned long long* __restrict__ pair_count, uint4* __restrict__ cand)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    PairFwdSmem<RING>& S = *reinterpret_cast<PairFwdSmem<RING>*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = order ? (int)order[blockIdx.x] : (int)blockIdx.x;   // heavy tiles first
    const int vi = view_of_tile(V, tile);
    const svr_view_t& view = V.v[vi];
    const int W = view.width, H = view.height;
    const int lt = tile - view.tile_offset;
    const int tx = lt % view.tiles_x, ty = lt / view.tiles_x;
    int dx, dy;
    pair_pixel<LATTICE>(warp, lane, dx, dy);
    const uint32_t px = tx * TILE + dx, py = ty * TILE + dy;
    const bool inside = (px < (uint32_t)W) && (py < (uint32_t)H);
    const Ray ray = pixel_ray(view, px, py);
    const uint32_t pq = ray_octant(ray.rd);
    const float s_val = *s_ptr;
    const int p_own = pix_slot(dy * TILE + dx);             // the pixel's shared-memory slot
    S.pray[p_own] = make_float4(ray.rd_inv.x, ray.rd_inv.y, ray.rd_inv.z,
                                __uint_as_float(pq | (inside ? PIX_LIVE : 0u)));
    S.pdir[p_own] = make_float4(ray.rd.x, ray.rd.y, ray.rd.z, ray.rd_norm_inv);
    store_row(S.mask[0][p_own], make_uint4(0u, 0u, 0u, 0u));
    store_row(S.mask[1][p_own], make_uint4(0u, 0u, 0u, 0u));

    const uint2 range = ranges[tile];
    const int n = (int)(range.y - range.x);
    const int nbatch = (n + BATCH - 1) / BATCH;
    if (tid == 0) {
#pragma unroll
        for (int k = 0; k < RING; ++k) { mbar_init(&S.full[k], 1); S.armed[k] = 0; }
        S.fail = 0;
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int b) {
        const int slot = b % RING;
        const uint32_t bytes = (uint32_t)min(BATCH, n - b * BATCH) * (uint32_t)sizeof(Rec);
        ++S.armed[slot];
        mbar_arrive_tx(&S.full[slot], bytes);
        bulk_g2s(S.buf[slot], recs + range.x + (size_t)b * BATCH, bytes, &S.full[slot]);
    };
    if (tid == 0)
        for (int b = 0; b < min(RING, nbatch); ++b) issue(b);

    const float3 ro = ray.ro;
    float T = 1.f, D = 0.f;
    float3 C = f3(0.f, 0.f, 0.f), Nn = f3(0.f, 0.f, 0.f);
    int64_t med_rec = -1;
    float med_T = 0.f;
    uint32_t last = 0;
    bool done = !inside;
    uint32_t parity = 0;
    bool failed = false;
    uint32_t n_eval = 0, n_acc = 0, n_eval_last = 0;   // COUNT only
    const int tx0 = tx * TILE, ty0 = ty * TILE;

    for (int b = 0; b < nbatch; ++b) {
        const int slot = b % RING;
        // the slot's candidate masks: the CTA-wide kernel alternates two buffers by parity
        uint32_t (*M)[4] = S.mask[CTAW ? (b & 1) : 0];
        if (CTAW) {
            // no CTA barrier here: a warp starts filtering this slot as soon as its records
            // have arrived, while other warps may still composite the previous one.  A timed-
            // out wait is flagged in shared memory and agreed on at the filter's barrier (the
            // filter only indexes inside the slot and the tile).
            if (!mbar_wait(&S.full[slot], (parity >> slot) & 1)) { failed = true; S.fail = 1; }
            parity ^= 1u << slot;
        } else {
            if (!mbar_wait(&S.full[slot], (parity >> slot) & 1)) failed = true;
            // every thread must reach the barriers below: a timed-out wait is agreed on by all
            if (__syncthreads_or(failed)) { failed = true; break; }
            parity ^= 1u << slot;
            // every warp is through the previous slot: refill it with the batch RING ahead
            if (tid == 0 && b >= 1 && b - 1 + RING < nbatch) {
                fence_proxy_async_smem();
                issue(b - 1 + RING);
            }
        }
        const int cnt = min(BATCH, n - b * BATCH);
        const Rec* buf = S.buf[slot];
        // ---------------------------------------------------------------- F: filter
        {
            const int r = tid >> 1, h = tid & 1;
            bool big = false;
            int c0 = 0, c1 = -1, r0 = 0, r1 = -1;
            uint32_t q = 0;
            float3 vc = f3(0.f, 0.f, 0.f);
            float vl = 0.f;
            if (r < cnt) {
                const Rec& rec = buf[r];
                c0 = max((int)(rec.bbox0 >> 16) - tx0, 0);
                c1 = record_dead(rec, s_val) ? -1 : min((int)(rec.bbox1 >> 16) - tx0, TILE - 1);
                r0 = max((int)(rec.bbox0 & 0xFFFFu) - ty0, 0);
                r1 = min((int)(rec.bbox1 & 0xFFFFu) - ty0, TILE - 1);
                q = rec.val >> 29;
                vc = f3(rec.cx, rec.cy, rec.cz);
                vl = rec.len;
                const int area = (c1 >= c0 && r1 >= r0) ? (c1 - c0 + 1) * (r1 - r0 + 1) : 0;
                big = area > SMALL_RECT;
                if (!big) {
                    for (int y = r0 + h; y <= r1; y += 2)
                        for (int x = c0; x <= c1; ++x) {
                            const int p = pix_slot(y * TILE + x);
                            if (filter_hit(S.pray[p], q, vc, vl, ro)) atomicOr(&M[p][r >> 5], 1u << (r & 31));
                        }
                }
            }
            // records with a large rectangle: the whole warp walks its pixels
            uint32_t bigm = __ballot_sync(0xffffffffu, big && h == 0);
            while (bigm) {
                const int src = __ffs(bigm) - 1;
                bigm &= bigm - 1;
                const int rr = __shfl_sync(0xffffffffu, r, src);
                const int bc0 = __shfl_sync(0xffffffffu, c0, src), bc1 = __shfl_sync(0xffffffffu, c1, src);
                const int br0 = __shfl_sync(0xffffffffu, r0, src), br1 = __shfl_sync(0xffffffffu, r1, src);
                const Rec& rec = buf[rr];
                const uint32_t bq = rec.val >> 29;
                const float3 bc = f3(rec.cx, rec.cy, rec.cz);
                const float bl = rec.len;
                const int wdt = bc1 - bc0 + 1, area = wdt * (br1 - br0 + 1);
                for (int k = lane; k < area; k += 32) {
                    const int p = pix_slot((br0 + k / wdt) * TILE + bc0 + k % wdt);
                    if (filter_hit(S.pray[p], bq, bc, bl, ro)) atomicOr(&M[p][rr >> 5], 1u << (rr & 31));
                }
            }
        }
        // the masks are complete; stop streaming once every pixel is done (as of the last slot)
        if constexpr (CTAW) {
            const int n_done = __syncthreads_count(done);
            if (S.fail) { failed = true; break; }
            if (n_done == BLOCK) break;
            // every warp is through the previous slot (its compositing ended before this
            // barrier): refill it with the batch RING ahead
            if (tid == 0 && b >= 1 && b - 1 + RING < nbatch) {
                fence_proxy_async_smem();
                issue(b - 1 + RING);
            }
            // the slot's candidate row of this thread's pixel, for the adjoint (row block
            // range.x / BATCH + tile + b; thread tid owns the same pixel there)
            if (cand) cand[((size_t)(range.x / BATCH) + (size_t)tile + (size_t)b) * BLOCK + tid] = load_row(M[p_own]);
        } else {
            if (__syncthreads_and(done)) break;
        }
        if constexpr (CTAW) {
            // ------------------------------------------------------------ P + C, CTA-wide
            // pairs numbered over the whole CTA (thread-major); each window of BLOCK pairs is
            // evaluated one pair per thread, then every pixel folds its pairs of the window
            uint32_t mc[4];
            {
                const uint4 mv = load_row(M[p_own]);
                mc[0] = mv.x; mc[1] = mv.y; mc[2] = mv.z; mc[3] = mv.w;
            }
            const int cnt_own = __popc(mc[0]) + __popc(mc[1]) + __popc(mc[2]) + __popc(mc[3]);
            int incl = cnt_own;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            S.ppre[tid] = incl - cnt_own;
            if (lane == 31) S.wcnt[warp] = incl;
            __syncthreads();
            int pre = incl - cnt_own, total = 0;
#pragma unroll
            for (int q = 0; q < NWARP; ++q) {
                const int c = S.wcnt[q];
                if (q < warp) pre += c;
                total += c;
            }
            int wi = 0;
            for (int base = 0; base < total; base += BLOCK, wi ^= 1) {
                const int i = base + tid;
                if (i < total) {
                    int t, k;
                    cta_pair_owner(S.wcnt, S.ppre, i, t, k);
                    int odx, ody;
                    pair_pixel<LATTICE>(t >> 5, t & 31, odx, ody);
                    const int p = pix_slot(ody * TILE + odx);
                    const uint4 omv = load_row(M[p]);
                    const uint32_t om0 = omv.x, om1 = omv.y, om2 = omv.z, om3 = omv.w;
                    int jb = 0;
                    uint32_t wsel = om0;
                    int c = __popc(om0);
                    if (k >= c) {
                        k -= c; wsel = om1; jb = 32; c = __popc(om1);
                        if (k >= c) {
                            k -= c; wsel = om2; jb = 64; c = __popc(om2);
                            if (k >= c) { k -= c; wsel = om3; jb = 96; }
                        }
                    }
                    const int j = jb + kth_set_bit(wsel, k);
                    const float4 pr = S.pray[p], pd = S.pdir[p];
                    S.cres[wi][tid] = fwd_pair_eval<NS, DEPTH>(buf[j], ro, f3(pd.x, pd.y, pd.z),
                                                               f3(pr.x, pr.y, pr.z), s_val);
                }
                __syncthreads();
                // C: this pixel's pairs of the window, in record order
                const int e = min(base + BLOCK, pre + cnt_own);
                for (int ii = max(base, pre); ii < e && !done; ++ii) {
                    int j2;
                    if (mc[0]) { j2 = __ffs(mc[0]) - 1; mc[0] &= mc[0] - 1; }
                    else if (mc[1]) { j2 = __ffs(mc[1]) + 31; mc[1] &= mc[1] - 1; }
                    else if (mc[2]) { j2 = __ffs(mc[2]) + 63; mc[2] &= mc[2] - 1; }
                    else { j2 = __ffs(mc[3]) + 95; mc[3] &= mc[3] - 1; }
                    const float2 rv = S.cres[wi][ii - base];
                    const float alpha = rv.x;
                    if (COUNT) ++n_eval;
                    if (alpha < MIN_ALPHA) continue;
                    if (COUNT) { ++n_acc; n_eval_last = n_eval; }
                    const Rec& r = buf[j2];
                    const float pt_w = T * alpha;
                    C = C + pt_w * f3(r.r, r.gr, r.b);
                    if (DEPTH) {
                        D = D + T * rv.y;
                        if (T > 0.5f) { med_rec = (int64_t)range.x + (int64_t)b * BATCH + j2; med_T = T; }
                    }
                    if (NORMAL) {
                        const float4 nv = record_normal(buf[j2]);
                        Nn = Nn + pt_w * nv.w * f3(nv.x, nv.y, nv.z);
                    }
                    T *= (1.f - alpha);
                    done |= (T < EARLY_STOP_T);
                    last = (uint32_t)(b * BATCH + j2 + 1);
                    if (MAXW)
                        atomicMax(((int*)max_w) + (size_t)vi * max_w_stride + (r.val & 0x1FFFFFFFu),
                                  __float_as_int(pt_w));
                }
            }
            // every owner lookup of the slot is behind the last window's barrier
            store_row(M[p_own], make_uint4(0u, 0u, 0u, 0u));
        } else {
            // ---------------------------------------------------------------- P + C, per warp
            uint32_t m[4], mc[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) { m[k] = mc[k] = M[p_own][k]; M[p_own][k] = 0u; }
            const int cnt_own = __popc(m[0]) + __popc(m[1]) + __popc(m[2]) + __popc(m[3]);
            int incl = cnt_own;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int pre = incl - cnt_own;
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            for (int base = 0; base < total; base += 32) {
                // P: pair base + lane
                const int i = base + lane;
                int ol = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const int cand = ol + step;
                    const int pv = __shfl_sync(0xffffffffu, pre, cand);
                    if (pv <= i) ol = cand;
                }
                const int opre = __shfl_sync(0xffffffffu, pre, ol);
                uint32_t om[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) om[k] = __shfl_sync(0xffffffffu, m[k], ol);
                if (i < total) {
                    int k = i - opre, jb = 0;
                    uint32_t wsel = om[0];
                    int c = __popc(om[0]);
                    if (k >= c) {
                        k -= c; wsel = om[1]; jb = 32; c = __popc(om[1]);
                        if (k >= c) {
                            k -= c; wsel = om[2]; jb = 64; c = __popc(om[2]);
                            if (k >= c) { k -= c; wsel = om[3]; jb = 96; }
                        }
                    }
                    const int j = jb + kth_set_bit(wsel, k);
                    int odx, ody;
                    pair_pixel<LATTICE>(warp, ol, odx, ody);
                    const int p = pix_slot(ody * TILE + odx);
                    const float4 pr = S.pray[p], pd = S.pdir[p];
                    S.res[warp][lane] = fwd_pair_eval<NS, DEPTH>(buf[j], ro, f3(pd.x, pd.y, pd.z),
                                                                 f3(pr.x, pr.y, pr.z), s_val);
                }
                __syncwarp();
                // C: this pixel's pairs of the window, in record order (popped from a copy: the
                // pair numbering above reads every lane's whole mask in each window)
                const int e = min(base + 32, pre + cnt_own);
                for (int ii = max(base, pre); ii < e && !done; ++ii) {
                    int j2;
                    if (mc[0]) { j2 = __ffs(mc[0]) - 1; mc[0] &= mc[0] - 1; }
                    else if (mc[1]) { j2 = __ffs(mc[1]) + 31; mc[1] &= mc[1] - 1; }
                    else if (mc[2]) { j2 = __ffs(mc[2]) + 63; mc[2] &= mc[2] - 1; }
                    else { j2 = __ffs(mc[3]) + 95; mc[3] &= mc[3] - 1; }
                    const float2 rv = S.res[warp][ii - base];
                    const float alpha = rv.x;
                    if (COUNT) ++n_eval;
                    if (alpha < MIN_ALPHA) continue;
                    if (COUNT) { ++n_acc; n_eval_last = n_eval; }
                    const Rec& r = buf[j2];
                    const float pt_w = T * alpha;
                    C = C + pt_w * f3(r.r, r.gr, r.b);
                    if (DEPTH) {
                        D = D + T * rv.y;
                        if (T > 0.5f) { med_rec = (int64_t)range.x + (int64_t)b * BATCH + j2; med_T = T; }
                    }
                    if (NORMAL) {
                        const float4 nv = record_normal(buf[j2]);
                        Nn = Nn + pt_w * nv.w * f3(nv.x, nv.y, nv.z);
                    }
                    T *= (1.f - alpha);
                    done |= (T < EARLY_STOP_T);
                    last = (uint32_t)(b * BATCH + j2 + 1);
                    if (MAXW)
                        atomicMax(((int*)max_w) + (size_t)vi * max_w_stride + (r.val & 0x1FFFFFFFu),
                                  __float_as_int(pt_w));
                }
                __syncwarp();
            }
        }
        if (done && inside) {
            const float4 pr = S.pray[p_own];
            S.pray[p_own].w = __uint_as_float(__float_as_uint(pr.w) & ~PIX_LIVE);
        }
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
        for (int qq = 0; qq < 8; ++qq) g[qq] = r.g[qq];
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
    if (COUNT) {
        const unsigned long long e = __reduce_add_sync(0xffffffffu, n_eval);
        const unsigned long long a = __reduce_add_sync(0xffffffffu, n_acc);
        const unsigned long long l = __reduce_add_sync(0xffffffffu, n_eval_last);
        if (lane == 0) {
            atomicAdd(pair_count, e);
            atomicAdd(pair_count + 1, a);
            atomicAdd(pair_count + 2, l);
        }
    }
    const uint32_t wl = __reduce_max_sync(0xffffffffu, my_last);
    if (lane == 0) S.red[warp] = wl;
    __syncthreads();
    if (tid == 0) {
        uint32_t mx = 0;
#pragma unroll
        for (int w = 0; w < NWARP; ++w) mx = max(mx, S.red[w]);
        tile_last[tile] = range.x + mx;
        drain_ring<RING>(S.full, S.armed, status);
    }
}

}  // namespace svr

namespace svr {

// ============================================================================ adjoint
// The adjoint of render_bwd_kernel (cuda/src/backward.cu:41-851, SDF, three sub-samples) with
// the same per-pair expressions, split so that the expensive per-pair arithmetic runs on full
// warps.  Per ring slot (records back to front):
//  * F: as the forward's filter, with each pixel's limit of its last contributor -- or, when
//    the last forward over these records was the CTA-wide one, that forward's candidate row of
//    the pixel read back (one 16-byte load, issued a slot ahead) and cut at the same limit,
//    which gives the same masks without testing a record again.  Slots are the forward's:
//    records [s * BATCH, (s + 1) * BATCH) of the tile, taken from the last one down;
//  * per warp, pairs numbered pixel-major and, within a pixel, in descending record order;
//    for every window of 32 pairs:
//    A (one pair per lane): alpha, dL/d(point weight) and the alpha, logistic-CDF and depth
//      derivative factors that do not depend on the transmittance;
//    B (per pixel, back to front): transmittance recovery, dL/dalpha, the suffix terms and
//      the depth-term scales, dL/ds;
//    C (one pair per lane): the eight corner gradients, colour and |dL/dalpha * alpha|, sent
//      with vector reductions.
// Per pair of a warp's window.  B overwrites what it consumed: dpw becomes dL/dalpha, dval
// the point weight and part[] the scaled depth terms, which C reads.
struct PairBwdRes {
    float alpha;                     // A -> B, C
    float dpw;                       // A -> B: dL/d(point weight); B -> C: dL/dalpha
    float dval;                      // A -> B: depth value; B -> C: point weight
    float das;                       // A -> B: dalpha/ds factor
    float part[3];                   // A -> B: depth-term factors (backward.cu:682-768); B -> C: scaled
    float dae, dax;                  // A -> C: alpha derivatives at entry / exit
    float c_lo[3], c_hi[3];          // A -> C: sub-segment alpha derivatives
};

template <int RING>
struct alignas(128) PairBwdSmem {
    Rec buf[RING][BATCH];
    uint64_t full[RING];
    uint32_t armed[RING];
    float4 pray[BLOCK];          // rd_inv, octant | PIX_LIVE
    float4 pdir[BLOCK];          // rd, d(depth) upstream / |camera ray|
    float4 pdc[BLOCK];           // dL/dcolor, last contributor (as bits)
    float4 pdn[BLOCK];           // dL/dnormal
    float4 pgt[BLOCK];           // target colour (R-concentration term)
    // candidate records of a slot, per pixel; the CTA-wide kernel alternates the two buffers
    // by slot parity (a warp can filter slot b + 1 while others still finish slot b)
    alignas(16) uint32_t mask[2][BLOCK][4];
    PairBwdRes res[NWARP][32];   // a warp's window, or (CTA-wide) the CTA's window in thread order
    float red[NWARP];
    int ppre[BLOCK];             // CTA-wide windows: each thread's pair offset within its warp
    int wcnt[NWARP];             // and the warps' pair counts
    int fail;                    // a wait of this CTA timed out
};

// Position of the k-th (from 0) highest set bit of the 128-bit mask m[0..3].
__device__ __forceinline__ int kth_highest_bit(const uint32_t (&m)[4], int k) {
    uint32_t wsel = m[3];
    int jb = 96;
    int c = __popc(m[3]);
    if (k >= c) {
        k -= c; wsel = m[2]; jb = 64; c = __popc(m[2]);
        if (k >= c) {
            k -= c; wsel = m[1]; jb = 32; c = __popc(m[1]);
            if (k >= c) { k -= c; wsel = m[0]; jb = 0; }
        }
    }
    return jb + 31 - kth_set_bit(__brev(wsel), k);
}

// Adjoint phase A of one (pixel p, record j) pair (backward.cu:313-388, 650-671, 682-768):
// alpha, dL/d(point weight) and the factors that do not depend on the transmittance, into R.
template <bool DEPTH, bool NORMAL, class SM>
__device__ __forceinline__ void bwd_pair_A(PairBwdRes& R, const SM& S, const Rec* buf, int j, int p, float3 ro,
                                           float s_val)
{
    const Rec& r = buf[j];
    const float4 pr = S.pray[p], pd = S.pdir[p], pc = S.pdc[p];
    const float3 rd = f3(pd.x, pd.y, pd.z);
    const float3 vox_c = f3(r.cx, r.cy, r.cz);
    const float vox_l = r.len;
    const float2 ab = ray_box(vox_c, vox_l, ro, f3(pr.x, pr.y, pr.z));
    const float a = ab.x, bb = ab.y;
    float g[8];
#pragma unroll
    for (int qq = 0; qq < 8; ++qq) g[qq] = r.g[qq];
    const float vox_l_inv = 1.f / vox_l;
    const float3 lo3 = vox_c - 0.5f * vox_l;
    // backward.cu:313-337: entry / exit from ro + t rd
    const float3 qt_entry = ((ro + a * rd) - lo3) * vox_l_inv;
    const float3 qt_exit = ((ro + bb * rd) - lo3) * vox_l_inv;
    float we[8], wx[8];
    tri_weights(qt_entry, we);
    tri_weights(qt_exit, wx);
    float sdf_entry = 0.f, sdf_exit = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) { sdf_entry += g[q] * we[q]; sdf_exit += g[q] * wx[q]; }
    const float phi_entry = 1.f / (1.f + expf(-s_val * sdf_entry));
    const float phi_exit = 1.f / (1.f + expf(-s_val * sdf_exit));
    const float denom = phi_entry + 1e-6f;
    const float alpha = fmaxf((phi_entry - phi_exit) / denom, 0.f);
    R.alpha = alpha;
    if (!(alpha < MIN_ALPHA)) {
        const float3 c3 = f3(r.r, r.gr, r.b);
        float dL_dpt_w = dot3(f3(pc.x, pc.y, pc.z), c3);
        if (NORMAL) {
            const float4 nv = record_normal(buf[j]);
            const float3 surf_n = nv.w * f3(nv.x, nv.y, nv.z);
            const float4 pn = S.pdn[p];
            dL_dpt_w += dot3(f3(pn.x, pn.y, pn.z), surf_n);
        }
        R.dpw = dL_dpt_w;
        const float pe = s_val * phi_entry * (1.f - phi_entry);
        {
            // backward.cu:650-671
            const float pxv = s_val * phi_exit * (1.f - phi_exit);
            R.dae = (pe * (1.f - alpha)) / denom;
            R.dax = -pxv / denom;
            const float dpe = phi_entry * (1.f - phi_entry) * sdf_entry;
            const float dpx = phi_exit * (1.f - phi_exit) * sdf_exit;
            R.das = ((dpe * (1.f - alpha)) + (-dpx)) / denom;
        }
        if (DEPTH) {
            // backward.cu:338-388 and :682-768 (three sub-segments); the first end
            // point is the entry point (same phi and phi', bit for bit)
            const float3 qt_step = ((bb - a) * rd / 3.0f) * vox_l_inv;
            float ph[4], dph[4];
            ph[0] = phi_entry;
            dph[0] = pe;
#pragma unroll
            for (int k2 = 1; k2 < 4; ++k2) {
                const float3 qk = qt_entry + qt_step * (float)k2;
                float wk[8];
                tri_weights(qk, wk);
                ph[k2] = 1.f / (1.f + expf(-s_val * interp8(g, wk)));
                dph[k2] = s_val * ph[k2] * (1.f - ph[k2]);
            }
            float la[3];
#pragma unroll
            for (int k2 = 0; k2 < 3; ++k2) {
                const float dk = ph[k2] + 1e-6f;
                const float raw = (ph[k2] - ph[k2 + 1]) / dk;
                const float allow = raw > 0.f ? 1.f : 0.f;
                la[k2] = fmaxf(raw, 0.f);
                R.c_lo[k2] = allow * (ph[k2 + 1] / (dk * dk)) * dph[k2];
                R.c_hi[k2] = allow * (-1.f / dk) * dph[k2 + 1];
            }
            const float step_sz = 0.3333333f * (bb - a);
            const float a0 = la[0], a1 = la[1], a2 = la[2];
            const float t0 = a + 0.5f * step_sz, t1 = a + 1.5f * step_sz, t2 = a + 2.5f * step_sz;
            R.dval = a0 * t0 + (1.f - a0) * a1 * t1 + (1.f - a0) * (1.f - a1) * a2 * t2;
            R.part[0] = t0 + a1 * a2 * t2 - a1 * t1 - a2 * t2;
            R.part[1] = t1 + a0 * a2 * t2 - a0 * t1 - a2 * t2;
            R.part[2] = t2 + a0 * a1 * t2 - a0 * t2 - a1 * t2;
        }
    }
}

// Adjoint phase B of one pair, in a pixel's back-to-front walk (backward.cu:640-680):
// transmittance recovery, dL/dalpha, the suffix term and dL/ds; R's dpw becomes dL/dalpha, its
// dval the point weight and its part[] the depth-term scales.
template <bool DEPTH>
__device__ __forceinline__ void bwd_pair_B(PairBwdRes& Q, float& T, float& last_dT, float& ds_acc, float dD) {
    const float alpha = Q.alpha;
    if (alpha < MIN_ALPHA) return;          // lambda_ascending == 0
    T = T / (1.f - alpha);
    const float pt_w = alpha * T;
    const float dL_dpt_w = Q.dpw;
    const float dL_dalpha = T * (dL_dpt_w - last_dT);
    last_dT += alpha * (dL_dpt_w - last_dT);
    ds_acc += dL_dalpha * Q.das;
    if (DEPTH) {
        const float dval = Q.dval;
        Q.part[0] = dD * T * Q.part[0];
        Q.part[1] = dD * T * Q.part[1];
        Q.part[2] = dD * T * Q.part[2];
        last_dT += dD * dval;
    }
    Q.dpw = dL_dalpha;
    Q.dval = pt_w;
}

// Adjoint phase C of one pair with alpha >= MIN_ALPHA (backward.cu:585-639, 650-768, 824-848,
// the lambda_ascending term off as in the forward's defaults): the eight corner
// gradients, colour and |dL/dalpha * alpha| from the factors of A and the scales of B, sent
// with vector reductions.
template <bool DEPTH, bool NORMAL, bool RCONC, class SM>
__device__ __forceinline__ void bwd_pair_C(const PairBwdRes& R, const SM& S, const Rec* buf, int j, int p, float3 ro,
                                           float weight_R, int vi, int N, float* __restrict__ dL_dvox,
                                           float* __restrict__ drgbs, unsigned* __restrict__ status)
{
    const Rec& r = buf[j];
    const float4 pr = S.pray[p], pd = S.pdir[p], pc = S.pdc[p];
    const float3 rd = f3(pd.x, pd.y, pd.z);
    const float3 vox_c = f3(r.cx, r.cy, r.cz);
    const float vox_l = r.len;
    const float2 ab = ray_box(vox_c, vox_l, ro, f3(pr.x, pr.y, pr.z));
    const float a = ab.x, bb = ab.y;
    const float vox_l_inv = 1.f / vox_l;
    const float3 lo3 = vox_c - 0.5f * vox_l;
    const float3 qt_entry = ((ro + a * rd) - lo3) * vox_l_inv;
    const float3 qt_exit = ((ro + bb * rd) - lo3) * vox_l_inv;
    const float dL_dalpha = R.dpw, pt_w = R.dval, alpha = R.alpha;
    float dg[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) dg[q] = 0.f;
    if (NORMAL) {
        // backward.cu:604-639
        const float4 nv = record_normal(buf[j]);
        const float3 lin_n = f3(nv.x, nv.y, nv.z);
        const float r_lin = nv.w;
        const float3 surf_n = r_lin * lin_n;
        const float4 pn = S.pdn[p];
        const float3 dsn = pt_w * f3(pn.x, pn.y, pn.z);
        const float3 d = r_lin * (dsn - dot3(dsn, lin_n) * r_lin * surf_n);
        dg[0] += -d.x - d.y - d.z; dg[1] += -d.x - d.y + d.z;
        dg[2] += -d.x + d.y - d.z; dg[3] += -d.x + d.y + d.z;
        dg[4] += +d.x - d.y - d.z; dg[5] += +d.x - d.y + d.z;
        dg[6] += +d.x + d.y - d.z; dg[7] += +d.x + d.y + d.z;
    }
    {
        float we[8], wx[8];
        tri_weights(qt_entry, we);
        tri_weights(qt_exit, wx);
        const float dae = R.dae, dax = R.dax;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            dg[q] += dae * we[q] * dL_dalpha;
            dg[q] += dax * wx[q] * dL_dalpha;
        }
    }
    if (DEPTH) {
        const float3 qt_step = ((bb - a) * rd / 3.0f) * vox_l_inv;
        const float d0 = R.part[0], d1 = R.part[1], d2 = R.part[2];
        const float cp[4] = {d0 * R.c_lo[0], d0 * R.c_hi[0] + d1 * R.c_lo[1],
                             d1 * R.c_hi[1] + d2 * R.c_lo[2], d2 * R.c_hi[2]};
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) {
            const float3 qk = qt_entry + qt_step * (float)k2;
            float wk[8];
            tri_weights(qk, wk);
#pragma unroll
            for (int q = 0; q < 8; ++q) dg[q] += cp[k2] * wk[q];
        }
    }
    float drgb0 = pt_w * pc.x, drgb1 = pt_w * pc.y, drgb2 = pt_w * pc.z;
    if (RCONC) {
        const float4 pg = S.pgt[p];
        const float3 gr = weight_R * pt_w * 2.0f * (f3(r.r, r.gr, r.b) - f3(pg.x, pg.y, pg.z));
        drgb0 += gr.x; drgb1 += gr.y; drgb2 += gr.z;
    }
    const uint32_t vid = r.val & 0x1FFFFFFFu;
    if (vid < (uint32_t)N) {
        float4* dst = reinterpret_cast<float4*>(dL_dvox + 12 * (size_t)vid);
        atomicAdd(dst, make_float4(dg[0], dg[1], dg[2], dg[3]));
        atomicAdd(dst + 1, make_float4(dg[4], dg[5], dg[6], dg[7]));
        if (drgbs) {
            float* cr = drgbs + 3 * ((size_t)vi * N + vid);
            atomicAdd(cr, drgb0); atomicAdd(cr + 1, drgb1); atomicAdd(cr + 2, drgb2);
            atomicAdd(dL_dvox + 12 * (size_t)vid + 11, fabsf(dL_dalpha * alpha));
        } else {
            atomicAdd(dst + 2, make_float4(drgb0, drgb1, drgb2, fabsf(dL_dalpha * alpha)));
        }
    } else {
        atomicOr(status, ERR_BAD_INDEX);
    }
}

template <bool DEPTH, bool NORMAL, bool RCONC, int RING = 3, int MINB = 3, bool LATTICE = true, bool CTAW = false>
__global__ void __launch_bounds__(BLOCK, MINB) render_bwd_pairs_kernel(
    const __grid_constant__ Views V, int N, const uint32_t* __restrict__ order, const uint2* __restrict__ ranges,
    const uint32_t* __restrict__ tile_last,
    const uint32_t* __restrict__ n_contrib, const Rec* __restrict__ recs, const float* __restrict__ s_ptr,
    const float* __restrict__ out_T, const float* __restrict__ dL_dcolor, const float* __restrict__ dL_ddepth,
    const float* __restrict__ dL_dnormal, const float* __restrict__ dL_dT, float lambda_R,
    const float* __restrict__ gt_color, float* __restrict__ dL_dvox, float* __restrict__ drgbs,
    float* __restrict__ dL_ds, unsigned* __restrict__ status, const uint4* __restrict__ cand,
    const int* __restrict__ cand_ok)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    PairBwdSmem<RING>& S = *reinterpret_cast<PairBwdSmem<RING>*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = order ? (int)order[blockIdx.x] : (int)blockIdx.x;   // heavy tiles first
    const int vi = view_of_tile(V, tile);
    const svr_view_t& view = V.v[vi];
    const int W = view.width, H = view.height;
    const int lt = tile - view.tile_offset;
    const int tx = lt % view.tiles_x, ty = lt / view.tiles_x;
    int dx, dy;
    pair_pixel<LATTICE>(warp, lane, dx, dy);
    const uint32_t px = tx * TILE + dx, py = ty * TILE + dy;
    const bool inside = (px < (uint32_t)W) && (py < (uint32_t)H);
    const Ray ray = pixel_ray(view, px, py);
    const uint32_t pq = ray_octant(ray.rd);
    const float s_val = *s_ptr;
    const int p_own = pix_slot(dy * TILE + dx);

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
    const bool active = inside && last_c > 0;
    S.pray[p_own] = make_float4(ray.rd_inv.x, ray.rd_inv.y, ray.rd_inv.z,
                                __uint_as_float(pq | (active ? PIX_LIVE : 0u)));
    S.pdir[p_own] = make_float4(ray.rd.x, ray.rd.y, ray.rd.z, dD);
    S.pdc[p_own] = make_float4(dpix.x, dpix.y, dpix.z, __uint_as_float(last_c));
    S.pdn[p_own] = make_float4(dN.x, dN.y, dN.z, 0.f);
    if (RCONC) S.pgt[p_own] = make_float4(gt.x, gt.y, gt.z, 0.f);
    store_row(S.mask[0][p_own], make_uint4(0u, 0u, 0u, 0u));
    store_row(S.mask[1][p_own], make_uint4(0u, 0u, 0u, 0u));

    const uint32_t rg0 = ranges[tile].x;
    const uint32_t rg1 = tile_last[tile];
    const int n = rg1 > rg0 ? (int)(rg1 - rg0) : 0;
    const int nbatch = (n + BATCH - 1) / BATCH;
    if (tid == 0) {
#pragma unroll
        for (int k = 0; k < RING; ++k) { mbar_init(&S.full[k], 1); S.armed[k] = 0; }
        S.fail = 0;
        fence_mbar_init();
    }
    __syncthreads();
    // batch b (back to front) is the forward's slot nbatch - 1 - b: relative records
    // [lo, lo + c) with lo = (nbatch - 1 - b) * BATCH, c = min(BATCH, n - lo)
    auto issue = [&](int b) {
        const int slot = b % RING;
        const int lo = (nbatch - 1 - b) * BATCH;
        const int c = min(BATCH, n - lo);
        const uint32_t bytes = (uint32_t)c * (uint32_t)sizeof(Rec);
        ++S.armed[slot];
        mbar_arrive_tx(&S.full[slot], bytes);
        bulk_g2s(S.buf[slot], recs + rg0 + lo, bytes, &S.full[slot]);
    };
    if (tid == 0)
        for (int b = 0; b < min(RING, nbatch); ++b) issue(b);

    const float3 ro = ray.ro;
    const float WH_inv = 1.f / ((float)(W * H));
    const float weight_R = lambda_R * WH_inv;
    float ds_acc = 0.f;
    uint32_t parity = 0;
    bool failed = false;
    const int tx0 = tx * TILE, ty0 = ty * TILE;
    // the forward's candidate rows of this tile, when the last forward over these records wrote
    // them: the filter is then one row read per slot (prefetched a slot ahead), limited to the
    // pixel's last contributor -- the same masks the filter below computes
    const bool use_cand = CTAW && cand != nullptr && *cand_ok != 0;
    const size_t cand0 = (size_t)(rg0 / BATCH) + (size_t)tile;
    uint4 crow = make_uint4(0u, 0u, 0u, 0u);
    if (use_cand && nbatch > 0) crow = cand[(cand0 + (size_t)(nbatch - 1)) * BLOCK + tid];

    for (int b = 0; b < nbatch; ++b) {
        const int slot = b % RING;
        uint32_t (*M)[4] = S.mask[CTAW ? (b & 1) : 0];   // the slot's candidate masks
        if (CTAW) {
            // no CTA barrier here (see render_fwd_pairs_kernel): a timed-out wait is flagged in
            // shared memory and agreed on at the filter's barrier
            if (!mbar_wait(&S.full[slot], (parity >> slot) & 1)) { failed = true; S.fail = 1; }
            parity ^= 1u << slot;
        } else {
            if (!mbar_wait(&S.full[slot], (parity >> slot) & 1)) failed = true;
            if (__syncthreads_or(failed)) { failed = true; break; }
            parity ^= 1u << slot;
            // every warp is through the previous slot: refill it with the batch RING ahead
            if (tid == 0 && b >= 1 && b - 1 + RING < nbatch) {
                fence_proxy_async_smem();
                issue(b - 1 + RING);
            }
        }
        const int lo = (nbatch - 1 - b) * BATCH;      // relative index of slot entry 0
        const int cnt = min(BATCH, n - lo);
        const Rec* buf = S.buf[slot];
        // ---------------------------------------------------------------- F: filter
        if (use_cand) {
            // bits r of the forward's row with lo + r below the pixel's last contributor count
            const uint4 row = crow;
            if (b + 1 < nbatch) crow = cand[(cand0 + (size_t)(nbatch - 2 - b)) * BLOCK + tid];
            const int k = min(max((int)last_c - lo, 0), BATCH);
            const uint32_t k0 = (uint32_t)min(k, 32), k1 = (uint32_t)min(max(k - 32, 0), 32);
            const uint32_t k2 = (uint32_t)min(max(k - 64, 0), 32), k3 = (uint32_t)min(max(k - 96, 0), 32);
            auto low = [](uint32_t c) { return c >= 32u ? 0xffffffffu : (1u << c) - 1u; };
            store_row(M[p_own], make_uint4(row.x & low(k0), row.y & low(k1), row.z & low(k2), row.w & low(k3)));
        } else {
            const int r = tid >> 1, h = tid & 1;
            bool big = false;
            int c0 = 0, c1 = -1, r0 = 0, r1 = -1;
            if (r < cnt) {
                const Rec& rec = buf[r];
                c0 = max((int)(rec.bbox0 >> 16) - tx0, 0);
                c1 = record_dead(rec, s_val) ? -1 : min((int)(rec.bbox1 >> 16) - tx0, TILE - 1);
                r0 = max((int)(rec.bbox0 & 0xFFFFu) - ty0, 0);
                r1 = min((int)(rec.bbox1 & 0xFFFFu) - ty0, TILE - 1);
                const uint32_t q = rec.val >> 29;
                const float3 vc = f3(rec.cx, rec.cy, rec.cz);
                const float vl = rec.len;
                const uint32_t rel = (uint32_t)(lo + r);
                const int area = (c1 >= c0 && r1 >= r0) ? (c1 - c0 + 1) * (r1 - r0 + 1) : 0;
                big = area > SMALL_RECT;
                if (!big) {
                    for (int y = r0 + h; y <= r1; y += 2)
                        for (int x = c0; x <= c1; ++x) {
                            const int p = pix_slot(y * TILE + x);
                            if (rel < __float_as_uint(S.pdc[p].w) && filter_hit(S.pray[p], q, vc, vl, ro))
                                atomicOr(&M[p][r >> 5], 1u << (r & 31));
                        }
                }
            }
            uint32_t bigm = __ballot_sync(0xffffffffu, big && h == 0);
            while (bigm) {
                const int src = __ffs(bigm) - 1;
                bigm &= bigm - 1;
                const int rr = __shfl_sync(0xffffffffu, r, src);
                const int bc0 = __shfl_sync(0xffffffffu, c0, src), bc1 = __shfl_sync(0xffffffffu, c1, src);
                const int br0 = __shfl_sync(0xffffffffu, r0, src), br1 = __shfl_sync(0xffffffffu, r1, src);
                const Rec& rec = buf[rr];
                const uint32_t bq = rec.val >> 29;
                const float3 bc = f3(rec.cx, rec.cy, rec.cz);
                const float bl = rec.len;
                const uint32_t rel = (uint32_t)(lo + rr);
                const int wdt = bc1 - bc0 + 1, area = wdt * (br1 - br0 + 1);
                for (int k = lane; k < area; k += 32) {
                    const int p = pix_slot((br0 + k / wdt) * TILE + bc0 + k % wdt);
                    if (rel < __float_as_uint(S.pdc[p].w) && filter_hit(S.pray[p], bq, bc, bl, ro))
                        atomicOr(&M[p][rr >> 5], 1u << (rr & 31));
                }
            }
        }
        // with candidate rows each thread has written only its own row: the numbering barrier
        // below is the slot's first, and the timeout check and the refill follow it there
        if (!use_cand) __syncthreads();
        if constexpr (CTAW) {
            if (!use_cand) {
                if (S.fail) { failed = true; break; }
                // every warp is through the previous slot: refill it with the batch RING ahead
                if (tid == 0 && b >= 1 && b - 1 + RING < nbatch) {
                    fence_proxy_async_smem();
                    issue(b - 1 + RING);
                }
            }
        }
        if constexpr (CTAW) {
            // ------------------------------------------------------------ CTA-wide windows
            // pairs numbered over the whole CTA (thread-major, each pixel's pairs back to
            // front); per window of BLOCK pairs: A one pair per thread, B per pixel, C one pair
            // per thread
            uint32_t m[4];
            {
                const uint4 mv = load_row(M[p_own]);
                m[0] = mv.x; m[1] = mv.y; m[2] = mv.z; m[3] = mv.w;
            }
            const int cnt_own = __popc(m[0]) + __popc(m[1]) + __popc(m[2]) + __popc(m[3]);
            int incl = cnt_own;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            S.ppre[tid] = incl - cnt_own;
            if (lane == 31) S.wcnt[warp] = incl;
            __syncthreads();
            if (use_cand) {
                if (S.fail) { failed = true; break; }
                // every warp is through the previous slot: refill it with the batch RING ahead
                if (tid == 0 && b >= 1 && b - 1 + RING < nbatch) {
                    fence_proxy_async_smem();
                    issue(b - 1 + RING);
                }
            }
            int pre = incl - cnt_own, total = 0;
#pragma unroll
            for (int q = 0; q < NWARP; ++q) {
                const int c = S.wcnt[q];
                if (q < warp) pre += c;
                total += c;
            }
            PairBwdRes* RF = &S.res[0][0];
            for (int base = 0; base < total; base += BLOCK) {
                const int i = base + tid;
                const bool has = i < total;
                int j = 0, p = 0;
                if (has) {
                    int t, k;
                    cta_pair_owner(S.wcnt, S.ppre, i, t, k);
                    int odx, ody;
                    pair_pixel<LATTICE>(t >> 5, t & 31, odx, ody);
                    p = pix_slot(ody * TILE + odx);
                    const uint4 omv = load_row(M[p]);
                    const uint32_t om[4] = {omv.x, omv.y, omv.z, omv.w};
                    j = kth_highest_bit(om, k);
                }
                PairBwdRes& R = RF[tid];
                if (has) bwd_pair_A<DEPTH, NORMAL>(R, S, buf, j, p, ro, s_val);
                __syncthreads();
                const int e = min(base + BLOCK, pre + cnt_own);
                for (int ii = max(base, pre); ii < e; ++ii) bwd_pair_B<DEPTH>(RF[ii - base], T, last_dT, ds_acc, dD);
                __syncthreads();
                if (has && !(R.alpha < MIN_ALPHA))
                    bwd_pair_C<DEPTH, NORMAL, RCONC>(R, S, buf, j, p, ro, weight_R, vi, N, dL_dvox, drgbs, status);
                __syncthreads();   // the next window overwrites RF
            }
            // every owner lookup of the slot is behind the last window's barriers
            store_row(M[p_own], make_uint4(0u, 0u, 0u, 0u));
        } else {
            // ---------------------------------------------------------------- per warp
            uint32_t m[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) { m[k] = M[p_own][k]; M[p_own][k] = 0u; }
            const int cnt_own = __popc(m[0]) + __popc(m[1]) + __popc(m[2]) + __popc(m[3]);
            int incl = cnt_own;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int pre = incl - cnt_own;
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            for (int base = 0; base < total; base += 32) {
                // which pair this lane evaluates in A and C: its pixel (lane ol) and record j
                const int i = base + lane;
                int ol = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const int cand = ol + step;
                    const int pv = __shfl_sync(0xffffffffu, pre, cand);
                    if (pv <= i) ol = cand;
                }
                const int opre = __shfl_sync(0xffffffffu, pre, ol);
                uint32_t om[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) om[k] = __shfl_sync(0xffffffffu, m[k], ol);
                const bool has = i < total;
                const int j = has ? kth_highest_bit(om, i - opre) : 0;
                int odx, ody;
                pair_pixel<LATTICE>(warp, ol, odx, ody);
                const int p = pix_slot(ody * TILE + odx);
                PairBwdRes& R = S.res[warp][lane];
                // ---------------------------------------------------------- A
                if (has) bwd_pair_A<DEPTH, NORMAL>(R, S, buf, j, p, ro, s_val);
                __syncwarp();
                // ---------------------------------------------------------- B: this pixel, back to front
                {
                    const int e = min(base + 32, pre + cnt_own);
                    for (int ii = max(base, pre); ii < e; ++ii)
                        bwd_pair_B<DEPTH>(S.res[warp][ii - base], T, last_dT, ds_acc, dD);
                }
                __syncwarp();
                // ---------------------------------------------------------- C
                if (has && !(R.alpha < MIN_ALPHA))
                    bwd_pair_C<DEPTH, NORMAL, RCONC>(R, S, buf, j, p, ro, weight_R, vi, N, dL_dvox, drgbs, status);
                __syncwarp();
            }
        }
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
        for (int w = 0; w < NWARP; ++w) s += S.red[w];
        if (s != 0.f) atomicAdd(dL_ds, s);
        drain_ring<RING>(S.full, S.armed, status);
    }
}

}  // namespace svr
