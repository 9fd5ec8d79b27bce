// Forward and adjoint tile-render kernels (SDF density).
//
// Behaviour: cuda/src/forward.cu:41-564 and cuda/src/backward.cu:41-851 of the reference,
// SDF branch, with the same per-pair arithmetic.  Organisation (ours):
//  * one CTA per 16x16 tile, 8 warps each owning an 8x4 pixel block;
//  * the tile's sorted 80-byte records stream through a ring of NSLOT shared-memory slots,
//    BATCH records each, every slot filled by ONE cp.async.bulk completing on a per-slot
//    mbarrier; warps consume slots independently (no CTA barrier per batch); the last warp
//    to finish a slot refills it with the batch NSLOT ahead;
//  * each warp pre-filters a slot's records against its 8x4 footprint and octant set with
//    one ballot per 32 records, then every lane collects its candidate pairs for the whole
//    slot and processes them in record order;
//  * the adjoint sends each pair's 12 gradient terms to dL_dvox / drgbs with vector
//    reductions (two or three float4 red per pair).  A shared-memory accumulator per slot,
//    flushed by the slot's last warp, measured 5.40 ms against 3.58 ms for the direct
//    reductions on 8 views 800x800: while one warp flushed, the others waited for the slot.
#pragma once

#include <climits>

#include "svr_common.cuh"

namespace svr {

#ifndef SVR_BATCH
#define SVR_BATCH 128
#endif
#ifndef SVR_NSLOT
#define SVR_NSLOT 4
#endif
// Minimum resident CTAs per SM requested from the register allocator.  Left to itself the
// allocator gives the adjoint 127-133 registers: 2 CTAs per SM at best, 1 when it crosses 128.
// Defaults are the autotuner's choices on both bench workloads (mid-size 8 x 800x800 and
// 64 mixed-resolution views): forward 4 ring slots x 4 CTAs (64 registers); adjoint 3 ring
// slots x 4 CTAs (64 registers, 248 B spilled to L1), 3.02 ms vs 3.12 ms for 4 x 3 (80
// registers) and 3.68 ms for 4 x 2 on the mid-size batch.
#ifndef SVR_FWD_MINB
#define SVR_FWD_MINB 4
#endif
#ifndef SVR_BWD_MINB
#define SVR_BWD_MINB 4
#endif
#ifndef SVR_BWD_NSLOT
#define SVR_BWD_NSLOT 3
#endif
constexpr int BATCH = SVR_BATCH;   // records per slot (80 B each)
constexpr int NSLOT = SVR_NSLOT;   // ring depth
constexpr int NWARP = BLOCK / 32;
static_assert(BATCH % 32 == 0 && BATCH <= 128, "slot holds at most 128 records (two 64-bit masks)");

// Candidate set of one lane over a slot: bit j = record j of the slot (j < 128).
struct CandMask {
    unsigned long long lo, hi;
    __device__ __forceinline__ void set(int j) {
        if (j < 64) lo |= 1ull << j; else hi |= 1ull << (j - 64);
    }
    __device__ __forceinline__ bool any() const { return (lo | hi) != 0ull; }
    // lowest / highest set record, removed from the set
    __device__ __forceinline__ int pop_first() {
        if (lo) { const int j = __ffsll(lo) - 1; lo &= lo - 1; return j; }
        const int j = __ffsll(hi) - 1; hi &= hi - 1; return j + 64;
    }
    __device__ __forceinline__ int pop_last() {
        if (hi) { const int j = 63 - __clzll(hi); hi &= ~(1ull << j); return j + 64; }
        const int j = 63 - __clzll(lo); lo &= ~(1ull << j); return j;
    }
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

template <int RING>
struct alignas(128) FwdSmem {
    Rec buf[RING][BATCH];
    uint64_t full[RING];
    uint32_t arrived[RING];
    uint32_t armed[RING];      // phases armed on each slot (bulk copies and end-of-stream arrivals)
    uint32_t octl[NWARP][8];
    uint32_t warps_done;
    int32_t stop;              // first batch not issued once every warp is done (INT_MAX before)
    uint32_t red[NWARP];
};

template <int RING>
struct alignas(128) BwdSmem {
    Rec buf[RING][BATCH];
    uint64_t full[RING];
    uint32_t arrived[RING];
    uint32_t armed[RING];      // phases armed on each slot (bulk copies)
    uint32_t octl[NWARP][8];
    float red[NWARP];
};

// Candidates of chunk c (records 32c .. 32c+31 of the slot) for every lane of the warp.
// Lane j takes record 32c+j and forms the set of the warp's pixels (lane = row * 8 + col of
// its 8x4 block) inside the record's pixel bbox (pix_in_bbox, inclusive) whose ray octant
// equals the record's (octl[q] = lanes with octant q) and that are still live; a 32x32 bit
// transpose then hands each lane the records of the chunk that pass for its own pixel
// (bit j = record 32c+j).  Same predicate as testing every record in every lane, at one
// record per lane.
__device__ __forceinline__ uint32_t chunk_candidates(const Rec* buf, int c, int cnt, int lane, int wx0, int wy0,
                                                     const uint32_t* octl, uint32_t live) {
    const int j = c * 32 + lane;
    uint32_t m = 0u;
    if (j < cnt) {
        const Rec& r = buf[j];
        const int c0 = max((int)(r.bbox0 >> 16) - wx0, 0), c1 = min((int)(r.bbox1 >> 16) - wx0, 7);
        const int r0 = max((int)(r.bbox0 & 0xFFFFu) - wy0, 0), r1 = min((int)(r.bbox1 & 0xFFFFu) - wy0, 3);
        if (c0 <= c1 && r0 <= r1) {
            const uint32_t cm = (0xFFu >> (7 - c1)) & (0xFFu << c0);
            const uint32_t rm = (0xFFFFFFFFu >> (8 * (3 - r1))) & (0xFFFFFFFFu << (8 * r0));
            m = (cm * 0x01010101u) & rm & octl[r.val >> 29] & live;
        }
    }
    // bit transpose: afterwards lane i holds bit j = (row j had bit i)
#pragma unroll
    for (int k = 16; k >= 1; k >>= 1) {
        const uint32_t M = k == 16 ? 0x0000FFFFu : k == 8 ? 0x00FF00FFu : k == 4 ? 0x0F0F0F0Fu
                         : k == 2 ? 0x33333333u : 0x55555555u;
        const uint32_t y = __shfl_xor_sync(0xffffffffu, m, k);
        m = (lane & k) ? ((m & ~M) | ((y >> k) & M)) : ((m & M) | ((y & M) << k));
    }
    return m;
}

// octl[q] = lanes of this warp whose pixel is in the image and whose ray octant is q
__device__ __forceinline__ void warp_octant_lanes(uint32_t* octl, bool inside, uint32_t pq, int lane) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const uint32_t b = __ballot_sync(0xffffffffu, inside && pq == (uint32_t)q);
        if (lane == q) octl[q] = b;
    }
    __syncwarp();
}

// Before a CTA exits: wait (bounded) for the last phase armed on every ring slot, so no bulk
// copy is still writing this CTA's shared memory when the next CTA on the SM takes it over.
// On the normal path every armed phase has been consumed and each wait returns at once; it
// matters after a timed-out wait, when warps left the stream with copies in flight.  A slot
// whose phase does not complete within the bound keeps its mbarrier and flags ERR_DRAIN:
// that path is bounded, not provably drained.
template <int RING>
__device__ __forceinline__ void drain_ring(uint64_t* full, const uint32_t* armed, unsigned* status) {
#pragma unroll
    for (int k = 0; k < RING; ++k) {
        const uint32_t a = armed[k];
        if (a == 0u || mbar_wait(&full[k], (a - 1u) & 1u)) mbar_inval(&full[k]);
        else atomicOr(status, ERR_DRAIN | ERR_WAIT_TIMEOUT);
    }
}

// ============================================================================ forward
// RING (ring slots) and MINB (CTAs per SM asked of the register allocator) change only the
// schedule, never the arithmetic: every (RING, MINB) instance produces the same outputs.
// COUNT (a separate instance, used only to measure the work) also adds to pair_count[0..2]
// the (pixel, record) pairs that reached the SDF evaluation, those accepted (alpha >=
// MIN_ALPHA), and those evaluated up to the pixel's last contributor (the pairs the adjoint
// evaluates).
template <int NS, bool DEPTH, bool NORMAL, bool MAXW, int RING = NSLOT, int MINB = SVR_FWD_MINB, bool COUNT = false>
__global__ void __launch_bounds__(BLOCK, MINB) render_fwd_kernel(
    const __grid_constant__ Views V, const uint32_t* __restrict__ order, const uint2* __restrict__ ranges,
    const Rec* __restrict__ recs, const float* __restrict__ s_ptr, uint32_t* __restrict__ tile_last,
    uint32_t* __restrict__ n_contrib,
    float* __restrict__ out_color, float* __restrict__ out_depth, float* __restrict__ out_normal,
    float* __restrict__ out_T, float* __restrict__ max_w, int64_t max_w_stride, unsigned* __restrict__ status,
    unsigned long long* __restrict__ pair_count = nullptr)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    FwdSmem<RING>& S = *reinterpret_cast<FwdSmem<RING>*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = order ? (int)order[blockIdx.x] : (int)blockIdx.x;   // heavy tiles first
    const int vi = view_of_tile(V, tile);
    const svr_view_t& view = V.v[vi];
    const int W = view.width, H = view.height;
    const int lt = tile - view.tile_offset;
    const int tx = lt % view.tiles_x, ty = lt / view.tiles_x;
    int dx, dy;
    tile_pixel(tid, dx, dy);
    const uint32_t px = tx * TILE + dx, py = ty * TILE + dy;
    const int wx0 = tx * TILE + (warp & 1) * 8, wy0 = ty * TILE + (warp >> 1) * 4;
    const bool inside = (px < (uint32_t)W) && (py < (uint32_t)H);
    const Ray ray = pixel_ray(view, px, py);
    const uint32_t pq = ray_octant(ray.rd);
    const float s_val = *s_ptr;
    warp_octant_lanes(S.octl[warp], inside, pq, lane);

    const uint2 range = ranges[tile];
    const int n = (int)(range.y - range.x);
    const int nbatch = (n + BATCH - 1) / BATCH;
    if (tid == 0) {
#pragma unroll
        for (int k = 0; k < RING; ++k) { mbar_init(&S.full[k], 1); S.arrived[k] = 0; S.armed[k] = 0; }
        S.warps_done = 0;
        S.stop = INT_MAX;
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

    float T = 1.f, D = 0.f;
    float3 C = f3(0.f, 0.f, 0.f), Nn = f3(0.f, 0.f, 0.f);
    int64_t med_rec = -1;
    float med_T = 0.f;
    uint32_t last = 0;
    bool done = !inside;
    bool reported = false;
    uint32_t parity = 0;
    bool failed = false;
    uint32_t n_eval = 0, n_acc = 0, n_eval_last = 0;   // COUNT only

    for (int b = 0; b < nbatch; ++b) {
        const int slot = b % RING;
        if (!mbar_wait(&S.full[slot], (parity >> slot) & 1)) { failed = true; break; }
        parity ^= 1u << slot;
        if (b >= *(volatile int32_t*)&S.stop) break;
        const int cnt = min(BATCH, n - b * BATCH);
        const Rec* buf = S.buf[slot];
        if (!__all_sync(0xffffffffu, done)) {
            // candidate pairs of this lane over the whole slot, in record order
            CandMask cand{0ull, 0ull};
            const uint32_t live = __ballot_sync(0xffffffffu, !done);
            for (int c = 0; c * 32 < cnt; ++c) {
                uint32_t bits = chunk_candidates(buf, c, cnt, lane, wx0, wy0, S.octl[warp], live);
                while (bits) {
                    const int k = __ffs(bits) - 1;
                    bits &= bits - 1;
                    const Rec& r = buf[c * 32 + k];
                    const float2 ab = ray_box(f3(r.cx, r.cy, r.cz), r.len, ray.ro, ray.rd_inv);
                    if (ab.x > ab.y) continue;
                    cand.set(c * 32 + k);
                }
            }
            {
                while (cand.any() && !done) {
                    const int j2 = cand.pop_first();
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
                    if (COUNT) ++n_eval;
                    if (alpha < MIN_ALPHA) continue;
                    if (COUNT) { ++n_acc; n_eval_last = n_eval; }
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
                        if (T > 0.5f) { med_rec = (int64_t)range.x + (int64_t)b * BATCH + j2; med_T = T; }
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
                    last = (uint32_t)(b * BATCH + j2 + 1);
                    if (MAXW)   // max_w_stride 0: one row for all views; N: a row per view
                        atomicMax(((int*)max_w) + (size_t)vi * max_w_stride + (r.val & 0x1FFFFFFFu),
                                  __float_as_int(pt_w));
                }
            }
        }
        // release the slot; the last warp refills it (or ends the stream once all are done)
        const bool wdone = __all_sync(0xffffffffu, done);
        if (lane == 0) {
            if (wdone && !reported) { atomicAdd(&S.warps_done, 1u); reported = true; }
            __threadfence_block();
            const uint32_t prev = atomicAdd(&S.arrived[slot], 1u);
            if (prev == NWARP - 1) {
                __threadfence_block();
                S.arrived[slot] = 0;
                const int nb2 = b + RING;
                if (nb2 < nbatch) {
                    if (*(volatile uint32_t*)&S.warps_done == NWARP) {
                        atomicMin(&S.stop, nb2);
                        ++S.armed[slot];
                        __threadfence_block();
                        mbar_arrive(&S.full[slot]);          // wakes waiters without data
                    } else {
                        fence_proxy_async_smem();
                        issue(nb2);
                    }
                }
            }
        }
        __syncwarp();
    }
    if (failed && lane == 0) atomicOr(status, ERR_WAIT_TIMEOUT);

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
        uint32_t m = 0;
#pragma unroll
        for (int w = 0; w < NWARP; ++w) m = max(m, S.red[w]);
        tile_last[tile] = range.x + m;
        drain_ring<RING>(S.full, S.armed, status);
    }
}

// ============================================================================ adjoint
template <bool DEPTH, bool NORMAL, bool RCONC, int RING = SVR_BWD_NSLOT, int MINB = SVR_BWD_MINB>
__global__ void __launch_bounds__(BLOCK, MINB) render_bwd_kernel(
    const __grid_constant__ Views V, int N, const uint32_t* __restrict__ order, const uint2* __restrict__ ranges,
    const uint32_t* __restrict__ tile_last,
    const uint32_t* __restrict__ n_contrib, const Rec* __restrict__ recs, const float* __restrict__ s_ptr,
    const float* __restrict__ out_T, const float* __restrict__ dL_dcolor, const float* __restrict__ dL_ddepth,
    const float* __restrict__ dL_dnormal, const float* __restrict__ dL_dT, float lambda_R,
    const float* __restrict__ gt_color, float* __restrict__ dL_dvox, float* __restrict__ drgbs,
    float* __restrict__ dL_ds, unsigned* __restrict__ status)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    BwdSmem<RING>& S = *reinterpret_cast<BwdSmem<RING>*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tile = order ? (int)order[blockIdx.x] : (int)blockIdx.x;   // heavy tiles first
    const int vi = view_of_tile(V, tile);
    const svr_view_t& view = V.v[vi];
    const int W = view.width, H = view.height;
    const int lt = tile - view.tile_offset;
    const int tx = lt % view.tiles_x, ty = lt / view.tiles_x;
    int dx, dy;
    tile_pixel(tid, dx, dy);
    const uint32_t px = tx * TILE + dx, py = ty * TILE + dy;
    const int wx0 = tx * TILE + (warp & 1) * 8, wy0 = ty * TILE + (warp >> 1) * 4;
    const bool inside = (px < (uint32_t)W) && (py < (uint32_t)H);
    const Ray ray = pixel_ray(view, px, py);
    const uint32_t pq = ray_octant(ray.rd);
    const float s_val = *s_ptr;
    warp_octant_lanes(S.octl[warp], inside, pq, lane);

    const uint32_t r0 = ranges[tile].x;
    const uint32_t r1 = tile_last[tile];
    const int n = r1 > r0 ? (int)(r1 - r0) : 0;
    const int nbatch = (n + BATCH - 1) / BATCH;
    if (tid == 0) {
#pragma unroll
        for (int k = 0; k < RING; ++k) { mbar_init(&S.full[k], 1); S.arrived[k] = 0; S.armed[k] = 0; }
        fence_mbar_init();
    }
    __syncthreads();
    // batch b covers relative records [lo, hi) with hi = n - b*BATCH (back to front)
    auto issue = [&](int b) {
        const int slot = b % RING;
        const int hi = n - b * BATCH;
        const int c = min(BATCH, hi);
        const uint32_t bytes = (uint32_t)c * (uint32_t)sizeof(Rec);
        ++S.armed[slot];
        mbar_arrive_tx(&S.full[slot], bytes);
        bulk_g2s(S.buf[slot], recs + r0 + (hi - c), bytes, &S.full[slot]);
    };
    if (tid == 0)
        for (int b = 0; b < min(RING, nbatch); ++b) issue(b);

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
    const uint32_t live = __ballot_sync(0xffffffffu, active);
    const bool warp_active = live != 0u;
    uint32_t parity = 0;
    bool failed = false;

    for (int b = 0; b < nbatch; ++b) {
        const int slot = b % RING;
        if (!mbar_wait(&S.full[slot], (parity >> slot) & 1)) { failed = true; break; }
        parity ^= 1u << slot;
        const int hi = n - b * BATCH;
        const int cnt = min(BATCH, hi);
        const int lo = hi - cnt;                      // relative index of slot entry 0
        const Rec* buf = S.buf[slot];
        if (warp_active) {
            CandMask cand{0ull, 0ull};
            for (int c = 0; c * 32 < cnt; ++c) {
                uint32_t bits = chunk_candidates(buf, c, cnt, lane, wx0, wy0, S.octl[warp], live);
                // only records before this pixel's last contributor
                const int lim = (int)last_c - lo - c * 32;
                bits &= lim >= 32 ? 0xFFFFFFFFu : (lim <= 0 ? 0u : ((1u << lim) - 1u));
                while (bits) {
                    const int k = __ffs(bits) - 1;
                    bits &= bits - 1;
                    const int jj = c * 32 + k;
                    const Rec& r = buf[jj];
                    const float2 ab = ray_box(f3(r.cx, r.cy, r.cz), r.len, ray.ro, ray.rd_inv);
                    if (ab.x > ab.y) continue;
                    cand.set(jj);
                }
            }
            {
                while (cand.any()) {
                    const int jj = cand.pop_last();           // back to front
                    const Rec& r = buf[jj];
                    const float3 vox_c = f3(r.cx, r.cy, r.cz);
                    const float vox_l = r.len;
                    const float2 ab = ray_box(vox_c, vox_l, ray.ro, ray.rd_inv);
                    const float a = ab.x, bb = ab.y;
                    float g[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) g[q] = r.g[q];
                    const float vox_l_inv = 1.f / vox_l;
                    const float3 lo3 = vox_c - 0.5f * vox_l;
                    // backward.cu:313-337: entry / exit from ro + t rd
                    const float3 qt_entry = ((ray.ro + a * ray.rd) - lo3) * vox_l_inv;
                    const float3 qt_exit = ((ray.ro + bb * ray.rd) - lo3) * vox_l_inv;
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
                    if (alpha < MIN_ALPHA) continue;          // lambda_ascending == 0
                    float dg[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) dg[i] = 0.f;
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
                        const float3 dsn = pt_w * dN;
                        const float3 d = r_lin * (dsn - dot3(dsn, lin_n) * r_lin * surf_n);
                        dg[0] += -d.x - d.y - d.z; dg[1] += -d.x - d.y + d.z;
                        dg[2] += -d.x + d.y - d.z; dg[3] += -d.x + d.y + d.z;
                        dg[4] += +d.x - d.y - d.z; dg[5] += +d.x - d.y + d.z;
                        dg[6] += +d.x + d.y - d.z; dg[7] += +d.x + d.y + d.z;
                    }
                    const float dL_dalpha = T * (dL_dpt_w - last_dT);
                    last_dT += alpha * (dL_dpt_w - last_dT);
                    const float pe = s_val * phi_entry * (1.f - phi_entry);
                    {
                        // backward.cu:650-671
                        const float pxv = s_val * phi_exit * (1.f - phi_exit);
                        const float dae = (pe * (1.f - alpha)) / denom;
                        const float dax = -pxv / denom;
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            dg[i] += dae * we[i] * dL_dalpha;
                            dg[i] += dax * wx[i] * dL_dalpha;
                        }
                        const float dpe = phi_entry * (1.f - phi_entry) * sdf_entry;
                        const float dpx = phi_exit * (1.f - phi_exit) * sdf_exit;
                        ds_acc += dL_dalpha * (((dpe * (1.f - alpha)) + (-dpx)) / denom);
                    }
                    if (DEPTH) {
                        // backward.cu:338-388 and :682-768 (three sub-segments): the 4
                        // sub-segment end points are evaluated once; each point's weight
                        // gradient collects both segments it bounds
                        const float3 qt_step = ((bb - a) * ray.rd / 3.0f) * vox_l_inv;
                        // the first end point is the entry point: its phi and phi' are
                        // phi_entry and pe, bit for bit (same weights, same summation order)
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
                        float la[3], c_lo[3], c_hi[3];
#pragma unroll
                        for (int k2 = 0; k2 < 3; ++k2) {
                            const float dk = ph[k2] + 1e-6f;
                            const float raw = (ph[k2] - ph[k2 + 1]) / dk;
                            const float allow = raw > 0.f ? 1.f : 0.f;
                            la[k2] = fmaxf(raw, 0.f);
                            c_lo[k2] = allow * (ph[k2 + 1] / (dk * dk)) * dph[k2];
                            c_hi[k2] = allow * (-1.f / dk) * dph[k2 + 1];
                        }
                        const float step_sz = 0.3333333f * (bb - a);
                        const float a0 = la[0], a1 = la[1], a2 = la[2];
                        const float t0 = a + 0.5f * step_sz, t1 = a + 1.5f * step_sz, t2 = a + 2.5f * step_sz;
                        const float dval = a0 * t0 + (1.f - a0) * a1 * t1 + (1.f - a0) * (1.f - a1) * a2 * t2;
                        const float d0 = dD * T * (t0 + a1 * a2 * t2 - a1 * t1 - a2 * t2);
                        const float d1 = dD * T * (t1 + a0 * a2 * t2 - a0 * t1 - a2 * t2);
                        const float d2 = dD * T * (t2 + a0 * a1 * t2 - a0 * t2 - a1 * t2);
                        last_dT += dD * dval;
                        const float cp[4] = {d0 * c_lo[0], d0 * c_hi[0] + d1 * c_lo[1], d1 * c_hi[1] + d2 * c_lo[2],
                                             d2 * c_hi[2]};
#pragma unroll
                        for (int k2 = 0; k2 < 4; ++k2) {
                            const float3 qk = qt_entry + qt_step * (float)k2;
                            float wk[8];
                            tri_weights(qk, wk);
#pragma unroll
                            for (int i = 0; i < 8; ++i) dg[i] += cp[k2] * wk[i];
                        }
                    }
                    float drgb0 = pt_w * dpix.x, drgb1 = pt_w * dpix.y, drgb2 = pt_w * dpix.z;
                    if (RCONC) {
                        const float3 gr = weight_R * pt_w * 2.0f * (c3 - gt);
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
            }
        }
        // release the slot; the last warp to release it refills it
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            const uint32_t prev = atomicAdd(&S.arrived[slot], 1u);
            if (prev == NWARP - 1) {
                __threadfence_block();
                S.arrived[slot] = 0;
                const int nb2 = b + RING;
                if (nb2 < nbatch) {
                    fence_proxy_async_smem();
                    issue(nb2);
                }
            }
        }
        __syncwarp();
    }
    if (failed && lane == 0) atomicOr(status, ERR_WAIT_TIMEOUT);
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
