"""ctypes front-end of the C oracle (``svr_oracle.c``) -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module, and only as a checker or a timed CPU baseline.  Everything takes and returns
numpy arrays in the reference's layouts (see ``svr_oracle.c`` for the file:line map).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = {32: os.path.join(_HERE, "_build", "libsvr_oracle.so"), 64: os.path.join(_HERE, "_build", "libsvr_oracle64.so")}
_libs = {}


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(bits=32):
    """The single-precision checker (bits=32) or the FP64 per-ray oracle (bits=64)."""
    if bits not in _libs:
        if not os.path.exists(_SO[bits]):
            build()
        L = C.CDLL(_SO[bits])
        L.svo_num_rendered.restype = C.c_int64
        L.svo_valid_table_count.restype = C.c_int64
        _libs[bits] = L
    return _libs[bits]


def set_threads(n: int):
    """Host threads for the render loops of both builds (1 = deterministic)."""
    for b in (32, 64):
        lib(b).svo_set_threads(C.c_int(int(n)))


def _r(x, bits):
    return C.c_double(float(x)) if bits == 64 else C.c_float(float(x))


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _f(x):
    return C.c_float(float(x))


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def preprocess(cam, centers, lengths, is_leaf):
    """cuda/src/preprocess.cu:36-154 -> (n_dup int32[N], bboxes uint32[N,2], bits uint32[N])."""
    centers = _c(centers, np.float32); lengths = _c(lengths, np.float32).reshape(-1)
    is_leaf = _c(is_leaf, np.uint8).reshape(-1)
    N = len(lengths)
    ndup = np.zeros(N, np.int32); bb = np.zeros((N, 2), np.uint32); bits = np.zeros(N, np.uint32)
    lib().svo_preprocess(C.c_int(N), C.c_int(cam.width), C.c_int(cam.height), _f(cam.tanfovx), _f(cam.tanfovy),
                         _f(cam.cx), _f(cam.cy), _p(_c(cam.w2c, np.float32)), _p(_c(cam.c2w, np.float32)),
                         _f(cam.near), _p(centers), _p(lengths), _p(is_leaf), _p(ndup), _p(bb), _p(bits))
    return ndup, bb, bits


def binning(cam, octpath, ndup, bboxes, bits):
    """forward.cu:749-829 + stable sort -> (keys uint64[R], vals uint32[R], ranges uint32[T,2])."""
    ndup = _c(ndup, np.int32)
    R = lib().svo_num_rendered(C.c_int(len(ndup)), _p(ndup))
    gx, gy = (cam.width + 15) // 16, (cam.height + 15) // 16
    keys = np.zeros(max(R, 1), np.uint64); vals = np.zeros(max(R, 1), np.uint32)
    ranges = np.zeros((gx * gy, 2), np.uint32)
    lib().svo_binning(C.c_int(len(ndup)), C.c_int(cam.width), C.c_int(cam.height), _p(_c(octpath, np.int64)),
                      _p(ndup), _p(_c(bboxes, np.uint32)), _p(_c(bits, np.uint32)), _p(keys), _p(vals), _p(ranges))
    return keys[:R], vals[:R], ranges


def set_pixel_mask(mask, bits=32):
    """Render only the pixels where ``mask`` (uint8[H*W]) is nonzero in later render_fwd /
    render_bwd calls of that build; None renders every pixel.  The array is kept alive here."""
    global _mask_keep
    if mask is None:
        _mask_keep = None
        lib(bits).svo_set_pixel_mask(None)
        return
    _mask_keep = np.ascontiguousarray(mask, dtype=np.uint8)
    lib(bits).svo_set_pixel_mask(_p(_mask_keep))


_mask_keep = None
_trace_keep = None


def set_trace(pixel_trace, voxel_trace=None, bits=32):
    """Record decision flags in later render_fwd / render_bwd calls of that build:
    ``pixel_trace`` uint8[H*W] (flags ORed in: 1 alpha near MIN_ALPHA, 2 transmittance near the
    early stop, 4 a median-depth decision near T = 0.5, 8 an adjoint alpha or depth-derivative
    switch near its threshold), ``voxel_trace`` uint8[N] (set for voxels that a pixel with a
    forward flag sends gradient to).  None stops recording.  The arrays are written in place."""
    global _trace_keep
    if pixel_trace is None:
        _trace_keep = None
        lib(bits).svo_set_trace(None, None)
        return
    assert pixel_trace.dtype == np.uint8 and pixel_trace.flags.c_contiguous
    assert voxel_trace is None or (voxel_trace.dtype == np.uint8 and voxel_trace.flags.c_contiguous)
    _trace_keep = (pixel_trace, voxel_trace)
    lib(bits).svo_set_trace(_p(pixel_trace), _p(voxel_trace))


_abs_keep = None


def set_abs_sum(abs_sum, bits=32):
    """Accumulate |term| of every adjoint pair term into ``abs_sum`` ([N,12], the build's float
    type) in later render_bwd calls; None stops."""
    global _abs_keep
    if abs_sum is None:
        _abs_keep = None
        lib(bits).svo_set_abs_sum(None)
        return
    assert abs_sum.dtype == (np.float64 if bits == 64 else np.float32) and abs_sum.flags.c_contiguous
    _abs_keep = abs_sum
    lib(bits).svo_set_abs_sum(_p(abs_sum))


def render_fwd(cam, bg, n_samp, need_depth, need_normal, ranges, vals, bboxes, centers, lengths, geos, rgbs,
               s_val, track_max_w=False, bits=32):
    """forward.cu:41-564 (SDF) -> dict of outputs in the reference layouts.  ``bits=64``
    evaluates the same per-ray algorithm in double precision."""
    W, H = cam.width, cam.height
    dt = np.float64 if bits == 64 else np.float32
    N = len(lengths.reshape(-1))
    T_t = ((W + 15) // 16) * ((H + 15) // 16)
    o = dict(color=np.zeros((3, H, W), dt), depth=np.zeros((4, H, W), dt),
             normal=np.zeros((3, H, W), dt), T=np.zeros((1, H, W), dt),
             max_w=np.zeros((N, 1), dt) if track_max_w else None,
             tile_last=np.zeros(T_t, np.uint32), n_contrib=np.zeros(H * W, np.uint32))
    vals = _c(vals, np.uint32)
    lib(bits).svo_render_fwd(C.c_int(W), C.c_int(H), _f(cam.tanfovx), _f(cam.tanfovy), _f(cam.cx), _f(cam.cy),
                             _p(_c(cam.c2w, np.float32)), _p(_c(bg, np.float32)), C.c_int(n_samp),
                             C.c_int(int(need_depth)), C.c_int(int(need_normal)), _p(_c(ranges, np.uint32)),
                             _p(vals if len(vals) else np.zeros(1, np.uint32)), _p(_c(bboxes, np.uint32)),
                             _p(_c(centers, dt)), _p(_c(lengths, dt)), _p(_c(geos, dt)),
                             _p(_c(rgbs, dt)), _r(s_val, bits), _p(o["color"]), _p(o["depth"]), _p(o["normal"]),
                             _p(o["T"]), _p(o["max_w"]), _p(o["tile_last"]), _p(o["n_contrib"]))
    return o


def render_bwd(cam, bg, need_depth, need_normal, ranges, tile_last, vals, bboxes, centers, lengths, geos, rgbs,
               s_val, out_T, n_contrib, dcolor, ddepth, dnormal, dT, lambda_R_concen=0.0, gt_color=None, bits=32):
    """backward.cu:41-851 (SDF, n_samp=3) -> (dL_dvox [N,12], dL_ds float)."""
    W, H = cam.width, cam.height
    dt = np.float64 if bits == 64 else np.float32
    N = len(lengths.reshape(-1))
    dvox = np.zeros((N, 12), dt)
    ds = np.zeros(1, dt)
    vals = _c(vals, np.uint32)
    gt = _c(gt_color, dt) if gt_color is not None else np.zeros(3 * H * W, dt)
    lib(bits).svo_render_bwd(C.c_int(W), C.c_int(H), _f(cam.tanfovx), _f(cam.tanfovy), _f(cam.cx), _f(cam.cy),
                             _p(_c(cam.c2w, np.float32)), _p(_c(bg, np.float32)), C.c_int(int(need_depth)),
                             C.c_int(int(need_normal)), _p(_c(ranges, np.uint32)), _p(_c(tile_last, np.uint32)),
                             _p(vals if len(vals) else np.zeros(1, np.uint32)), _p(_c(bboxes, np.uint32)),
                             _p(_c(centers, dt)), _p(_c(lengths, dt)), _p(_c(geos, dt)),
                             _p(_c(rgbs, dt)), _r(s_val, bits), _p(_c(out_T, dt)),
                             _p(_c(n_contrib, np.uint32)), _p(_c(dcolor, dt)), _p(_c(ddepth, dt)),
                             _p(_c(dnormal, dt)), _p(_c(dT, dt)), _r(lambda_R_concen, bits), _p(gt),
                             _p(dvox), _p(ds))
    return dvox, float(ds[0])


def gather_geo(care_idx, vox_key, grid, n_vox):
    geos = np.zeros((n_vox, 8), np.float32)
    care_idx = _c(care_idx, np.int64)
    lib().svo_gather_geo(C.c_int(len(care_idx)), _p(care_idx), _p(_c(vox_key, np.int64)),
                         _p(_c(grid, np.float32)), _p(geos))
    return geos


def gather_geo_bw(care_idx, vox_key, dgeos, n_grid):
    dgrid = np.zeros((n_grid, 1), np.float32)
    care_idx = _c(care_idx, np.int64)
    lib().svo_gather_geo_bw(C.c_int(len(care_idx)), _p(care_idx), _p(_c(vox_key, np.int64)),
                            _p(_c(dgeos, np.float32)), _p(dgrid))
    return dgrid


def sh_eval(deg, idx, centers, cam_pos, sh0, shs):
    N = len(centers); M = 1 + shs.shape[1]
    idx = _c(idx if idx is not None else np.zeros(0, np.int64), np.int64)
    rgbs = np.zeros((N, 3), np.float32)
    lib().svo_sh_eval(C.c_int(N), C.c_int(len(idx)), _p(idx if len(idx) else np.zeros(1, np.int64)), C.c_int(deg),
                      C.c_int(M), _p(_c(centers, np.float32)), _p(_c(cam_pos, np.float32)),
                      _p(_c(sh0, np.float32)), _p(_c(shs, np.float32)), _p(rgbs))
    return rgbs


def sh_eval_bw(deg, idx, centers, cam_pos, drgbs, M):
    N = len(centers)
    idx = _c(idx if idx is not None else np.zeros(0, np.int64), np.int64)
    dsh0 = np.zeros((N, 3), np.float32); dshs = np.zeros((N, M - 1, 3), np.float32)
    lib().svo_sh_eval_bw(C.c_int(N), C.c_int(len(idx)), _p(idx if len(idx) else np.zeros(1, np.int64)),
                         C.c_int(deg), C.c_int(M), _p(_c(centers, np.float32)), _p(_c(cam_pos, np.float32)),
                         _p(_c(drgbs, np.float32)), _p(dsh0), _p(dshs))
    return dsh0, dshs


def valid_table(centers, sizes, scene_center, inside_extent, res_pow2, is_leaf):
    centers = _c(centers, np.float32); sizes = _c(sizes, np.float32).reshape(-1)
    sc = _c(scene_center, np.float32); leaf = _c(is_leaf, np.uint8).reshape(-1)
    N = len(sizes)
    G = lib().svo_valid_table_count(C.c_int(N), _p(centers), _p(sizes), _p(sc), _f(inside_extent),
                                    C.c_int(res_pow2), _p(leaf))
    res = 1 << res_pow2
    mask = np.zeros(res ** 3, np.uint8)
    keys = np.zeros(max(G, 1), np.int32); g2v = np.zeros(max(G, 1), np.int32)
    lib().svo_valid_table(C.c_int(N), _p(centers), _p(sizes), _p(sc), _f(inside_extent), C.c_int(res_pow2),
                          _p(leaf), _p(mask), _p(keys), _p(g2v))
    return mask.astype(bool), keys[:G], g2v[:G]


def _grid_loss(fn, grid, vox_key, coords, vsizes, res, mask, keys, g2v, active, weight, vox_size_inv, seed, grad):
    grad = _c(grad, np.float32).copy()
    active = _c(active, np.int32)
    fn(C.c_int(len(keys)), C.c_int(len(active)), _p(active), _p(_c(keys, np.int32)), _p(_c(g2v, np.int32)),
       C.c_int(res), _p(_c(mask, np.uint8)), _p(_c(coords, np.float32)), _p(_c(vsizes, np.float32)),
       _p(_c(vox_key, np.int64)), _p(_c(grid, np.float32)), _f(weight), _f(vox_size_inv), C.c_int(seed), _p(grad))
    return grad


def laplacian_bw(*a, **k):
    """ls_compute.cu:14-109 with an explicit seed."""
    return _grid_loss(lib().svo_laplacian_bw, *a, **k)


def eikonal_bw(*a, **k):
    """ge_compute.cu:14-117 with an explicit seed."""
    return _grid_loss(lib().svo_eikonal_bw, *a, **k)


def voxel_gradient_bw(grid, vox_key, vox_size_inv, active, weight, grad):
    """vg_compute.cu:23-77 (voxel Eikonal); grid holds one channel."""
    grad = _c(grad, np.float32).copy()
    active = _c(active, np.int32)
    lib().svo_voxel_gradient_bw(C.c_int(len(active)), _p(active), _p(_c(vox_key, np.int64)),
                                _p(_c(grid, np.float32)), _p(_c(vox_size_inv, np.float32)), _f(weight), _p(grad))
    return grad


def total_variation_bw(grid, vox_key, weight, vox_size_inv, no_tv_s, tv_sparse, grad):
    """tv_compute.cu:22-158; the tv_sparse test reads the gradient as it was on entry."""
    grid = _c(grid, np.float32)
    M = grid.shape[0]
    Cc = grid.shape[1] if grid.ndim > 1 else 1
    grad = _c(grad, np.float32).copy()
    vox_key = _c(vox_key, np.int64)
    lib().svo_total_variation_bw(C.c_int64(vox_key.shape[0]), C.c_int(Cc), _p(vox_key), _p(grid), _f(weight),
                                 _p(_c(vox_size_inv, np.float32)), C.c_int(int(no_tv_s)), C.c_int(int(tv_sparse)),
                                 _p(grad), C.c_int64(M))
    return grad


def points_loss_bw(points, grid, vox_key, coords, vsizes, res, mask, keys, g2v, weight, grad):
    """pl_compute.cu:14-63; points in grid units [P, 3]."""
    grad = _c(grad, np.float32).copy()
    points = _c(points, np.float32)
    lib().svo_points_loss_bw(C.c_int(points.shape[0]), _p(points), C.c_int(len(keys)), _p(_c(keys, np.int32)),
                             _p(_c(g2v, np.int32)), C.c_int(res), _p(_c(mask, np.uint8)), _p(_c(coords, np.float32)),
                             _p(_c(vsizes, np.float32)), _p(_c(vox_key, np.int64)), _p(_c(grid, np.float32)),
                             _f(weight), _p(grad))
    return grad


def quantize(values, max_iter=10):
    """io.py:123-167: (index u8 shaped like values, codebook f32[256], rounds that moved values)."""
    v = _c(values, np.float32)
    idx = np.empty(v.shape, np.uint8)
    book = np.empty(256, np.float32)
    rounds = lib().svo_quantize(C.c_int64(v.size), _p(v), C.c_int(max_iter), _p(idx), _p(book))
    return idx, book, rounds


def normal_depth_loss(W, H, cx, cy, tanfovx, tanfovy, c2w, depth, normal, T, ks, tol_cos):
    """cameras.py:104-127 + loss_utils.py:345-407 for one view: (loss, dL/ddepth f32[H,W],
    dL/dnormal f32[3,H,W]).  T given: NormalDepthConsistencyLoss on ``depth``; T None:
    NormalMedianConsistencyLoss.  tol_cos <= 0 turns the tolerance mask off."""
    L = lib()
    L.svo_normal_depth_loss.restype = C.c_double
    d = _c(depth, np.float32).reshape(H, W)
    n = _c(normal, np.float32).reshape(3, H, W)
    t = None if T is None else _c(T, np.float32).reshape(H, W)
    gd = np.zeros((H, W), np.float32)
    gn = np.zeros((3, H, W), np.float32)
    m = _c(np.asarray(c2w, np.float32)[:3, :4], np.float32)
    loss = L.svo_normal_depth_loss(C.c_int(W), C.c_int(H), _f(cx), _f(cy), _f(tanfovx), _f(tanfovy), _p(m), _p(d),
                                   _p(n), _p(t), C.c_int(ks), _f(tol_cos), _p(gd), _p(gn))
    return loss, gd, gn


def adam(param, grad, m, v, step, lr, beta1, beta2, eps, biased=False, sparse=False):
    p = _c(param, np.float32).copy(); m = _c(m, np.float32).copy(); v = _c(v, np.float32).copy()
    lib().svo_adam(C.c_int(p.size), C.c_int(int(biased)), C.c_int(int(sparse)), _p(p), _p(_c(grad, np.float32)),
                   _p(m), _p(v), C.c_double(step), C.c_double(lr), C.c_double(beta1), C.c_double(beta2), _f(eps))
    return p, m, v
