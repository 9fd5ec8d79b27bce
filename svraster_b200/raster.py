"""Host orchestration of the sm_100a rasterizer: buffers, stream, C-ABI calls.

One object per render batch.  Views are described by dicts (see ``_lib.make_views``);
a single view reproduces the reference's per-view ``_C.rasterize_preprocess`` /
``_C.rasterize_voxels`` / ``_C.rasterize_voxels_backward`` (cuda/src/preprocess.cu:158-228,
forward.cu:986-1096, backward.cu:986-1109) and several views run batched: one launch per
stage for the whole batch, one sort over every view's records.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check, ptr, stream_ptr

_u8 = torch.uint8


def _empty_bytes(n, device):
    return torch.empty(max(int(n), 16), dtype=_u8, device=device)


class RasterState:
    """Geometry / binning / image buffers of one batch of views (opaque byte tensors, like
    the reference's geomBuffer / binningBuffer / imgBuffer)."""

    def __init__(self, cams, n_vox, device):
        self.cams = cams
        self.views, self.total_tiles, self.total_pix = _lib.make_views(cams)
        self.n_views = len(cams)
        self.N = int(n_vox)
        self.device = device
        self.geom = None
        self.binning = None
        self.image = None
        self.num_rendered = 0
        self.path_or = 0

    # -------------------------------------------------------------- preprocess
    def preprocess(self, octpaths, centers, lengths, is_leaf):
        L = _lib.load()
        M = self.N * self.n_views
        n_dup = torch.empty(M, dtype=torch.int32, device=self.device)
        self.geom = _empty_bytes(L.svr_geom_buffer_bytes(M), self.device)
        check(L.svr_preprocess(self.views, self.n_views, self.N, ptr(centers), ptr(lengths), ptr(is_leaf),
                               ptr(octpaths), ptr(n_dup), ptr(self.geom), stream_ptr(self.device)),
              "svr_preprocess")
        return n_dup

    # -------------------------------------------------------------- binning
    def bin(self, octpaths, capacity=None, path_or=None, rank_table=None, pair_order=None):
        """Duplicate, sort and range the records.  By default the record total is read back
        (one host synchronisation, as the reference does).  With ``capacity`` (and ``path_or``,
        the OR of every voxel's octree path) nothing is read back: the buffers hold
        ``capacity`` records and the device bins min(total, capacity) of them (status bit 8
        if any were dropped), which lets the call be captured into a CUDA graph.
        ``rank_table`` (a ``RankTable``) narrows the sort key to dense ranks when it was built
        for the same trimming as this call's path_or (same order, fewer radix passes).
        ``pair_order`` (a ``PairOrder`` of the same octree) bins with the per-tile sort
        (svr_bin_tiles: count, scan, scatter, one CTA per tile) instead of the global radix
        sort; the record order is the same."""
        L = _lib.load()
        M = self.N * self.n_views
        if capacity is None:
            R, por = C.c_int64(0), C.c_uint64(0)
            if pair_order is not None:     # the per-tile sort needs the total only, no scan
                check(L.svr_rendered_total(ptr(self.geom), C.byref(R), C.byref(por), stream_ptr(self.device)),
                      "svr_rendered_total")
            else:
                check(L.svr_count_rendered(M, ptr(self.geom), C.byref(R), C.byref(por), stream_ptr(self.device)),
                      "svr_count_rendered")
            self.num_rendered, self.path_or = int(R.value), int(por.value)
        else:
            if path_or is None:
                raise ValueError("bin(capacity=...) needs path_or")
            if pair_order is None:
                check(L.svr_scan_rendered(M, ptr(self.geom), stream_ptr(self.device)), "svr_scan_rendered")
            self.num_rendered, self.path_or = int(capacity), int(path_or)
        nb = L.svr_binning_buffer_bytes(self.num_rendered, self.total_tiles)
        self.binning = _empty_bytes(nb, self.device)
        self.image = _empty_bytes(L.svr_image_buffer_bytes(self.total_pix, self.total_tiles), self.device)
        if pair_order is not None:
            check(L.svr_bin_tiles(self.views, self.n_views, self.N, self.num_rendered, ptr(pair_order.pos),
                                  pair_order.bits, ptr(self.geom), ptr(self.binning), nb, ptr(self.image),
                                  stream_ptr(self.device)), "svr_bin_tiles")
        elif rank_table is not None and rank_table.matches(self.path_or):
            check(L.svr_bin_and_sort_ranked(self.views, self.n_views, self.N, self.num_rendered, self.path_or,
                                            ptr(octpaths), ptr(rank_table.table), rank_table.bits, ptr(self.geom),
                                            ptr(self.binning), nb, ptr(self.image), stream_ptr(self.device)),
                  "svr_bin_and_sort_ranked")
        else:
            check(L.svr_bin_and_sort(self.views, self.n_views, self.N, self.num_rendered, self.path_or,
                                     ptr(octpaths), ptr(self.geom), ptr(self.binning), nb, ptr(self.image),
                                     stream_ptr(self.device)), "svr_bin_and_sort")
        return self.num_rendered

    # -------------------------------------------------------------- render
    def render(self, n_samp, need_depth, need_normal, centers, lengths, geos, rgbs, s_val, track_max_w=False,
               rgb_per_view=False):
        L = _lib.load()
        P, dev = self.total_pix, self.device
        color = torch.empty(3 * P, dtype=torch.float32, device=dev)
        depth = torch.empty(4 * P, dtype=torch.float32, device=dev) if need_depth else None
        normal = torch.empty(3 * P, dtype=torch.float32, device=dev) if need_normal else None
        T = torch.empty(P, dtype=torch.float32, device=dev)
        max_w = torch.zeros(self.N, dtype=torch.float32, device=dev) if track_max_w else None
        check(L.svr_render_fwd(self.views, self.n_views, self.N, self.num_rendered, int(n_samp), int(need_depth),
                               int(need_normal), ptr(centers), ptr(lengths), ptr(geos), ptr(rgbs),
                               self.n_views if rgb_per_view else 1, ptr(s_val), ptr(self.geom), ptr(self.binning),
                               ptr(self.image), ptr(color), ptr(depth), ptr(normal), ptr(T), ptr(max_w),
                               stream_ptr(dev)), "svr_render_fwd")
        return color, depth, normal, T, max_w

    def count_pairs(self, s_val, return_planes=False):
        """(evaluated, accepted, adjoint) (pixel, record) pair counts of this batch's forward
        (three sub-samples, depth and normal on), by the counting instance of the forward
        kernel; call after ``render`` packed the records.  Synchronises.  With
        ``return_planes`` also returns that instance's (color, depth, normal, T)."""
        L = _lib.load()
        P, dev = self.total_pix, self.device
        out = [torch.empty(n * P, dtype=torch.float32, device=dev) for n in (3, 4, 3, 1)]
        cnt = torch.zeros(3, dtype=torch.int64, device=dev)
        check(L.svr_render_fwd_count_pairs(self.views, self.n_views, self.N, self.num_rendered, ptr(s_val),
                                           ptr(self.binning), ptr(self.image), *[ptr(o) for o in out], ptr(cnt),
                                           stream_ptr(dev)), "svr_render_fwd_count_pairs")
        counts = tuple(int(x) for x in cnt.cpu().tolist())
        return (counts, tuple(out)) if return_planes else counts

    def render_backward(self, need_depth, need_normal, s_val, out_T, dcolor, ddepth, dnormal, dT,
                        lambda_R_concen=0.0, gt_color=None, drgbs=None, dvox=None, ds=None):
        L = _lib.load()
        dev = self.device
        if dvox is None:
            dvox = torch.zeros(self.N, 12, dtype=torch.float32, device=dev)
        if ds is None:
            ds = torch.zeros(1, dtype=torch.float32, device=dev)
        check(L.svr_render_bwd(self.views, self.n_views, self.N, self.num_rendered, int(need_depth),
                               int(need_normal), float(lambda_R_concen), ptr(gt_color), ptr(s_val),
                               ptr(self.binning), ptr(self.image), ptr(out_T), ptr(dcolor), ptr(ddepth),
                               ptr(dnormal), ptr(dT), ptr(dvox), ptr(drgbs), ptr(ds), stream_ptr(dev)),
              "svr_render_bwd")
        return dvox, ds

    def binned_count(self):
        """Records actually binned (min(total, capacity)); synchronises."""
        n = C.c_int64(0)
        check(_lib.load().svr_binning_count(ptr(self.binning), C.byref(n), stream_ptr(self.device)),
              "svr_binning_count")
        return int(n.value)

    def candidates_valid(self):
        """Whether the adjoint will read the forward's candidate rows (svr_binning_candidates_valid);
        synchronises."""
        v = C.c_int(0)
        check(_lib.load().svr_binning_candidates_valid(ptr(self.binning), C.byref(v), stream_ptr(self.device)),
              "svr_binning_candidates_valid")
        return bool(v.value)

    # -------------------------------------------------------------- introspection (tests)
    def status(self):
        st = C.c_uint32(0)
        check(_lib.load().svr_read_status(ptr(self.image), self.total_pix, self.total_tiles, C.byref(st),
                                          stream_ptr(self.device)), "svr_read_status")
        return int(st.value)

    def geom_fields(self):
        M = self.N * self.n_views
        nd = torch.empty(M, dtype=torch.int32, device=self.device)
        bb = torch.empty(M, 2, dtype=torch.int32, device=self.device)
        bits = torch.empty(M, dtype=torch.int32, device=self.device)
        check(_lib.load().svr_unpack_geom(ptr(self.geom), M, ptr(nd), ptr(bb), ptr(bits), stream_ptr(self.device)),
              "svr_unpack_geom")
        return nd, bb, bits

    def binning_fields(self):
        R = max(self.num_rendered, 1)
        vals = torch.empty(R, dtype=torch.int32, device=self.device)
        ranges = torch.empty(self.total_tiles, 2, dtype=torch.int32, device=self.device)
        tl = torch.empty(self.total_tiles, dtype=torch.int32, device=self.device)
        nc = torch.empty(self.total_pix, dtype=torch.int32, device=self.device)
        check(_lib.load().svr_unpack_binning(ptr(self.binning), self.num_rendered, self.total_tiles, ptr(self.image),
                                             self.total_pix, ptr(vals), ptr(ranges), ptr(tl), ptr(nc),
                                             stream_ptr(self.device)), "svr_unpack_binning")
        return vals[: self.num_rendered], ranges, tl, nc


def rank_shift(path_or):
    """Low rank bits the binning key drops for this path OR (raster.cu key_format): all 3-bit
    level groups below the lowest non-zero one but one."""
    path_or = int(path_or)
    g = 16 if path_or == 0 else ((path_or & -path_or).bit_length() - 1) // 3
    return 3 * (g - 1) if g > 0 else 0


class RankTable:
    """Dense ranks of every (voxel, octant) pair of an octree (svr_rank_table_build), for
    ``RasterState.bin(rank_table=...)``.  Valid for the octree it was built from and for
    binning calls whose path_or trims as ``path_or`` does."""

    def __init__(self, octpaths, path_or):
        L = _lib.load()
        dev = octpaths.device
        paths = octpaths.reshape(-1).to(torch.int64).contiguous()
        N = paths.numel()
        nbytes = C.c_size_t(0)
        check(L.svr_rank_table_workspace_bytes(N, C.byref(nbytes)), "svr_rank_table_workspace_bytes")
        ws = _empty_bytes(nbytes.value, dev)
        self.table = torch.empty(8 * N, dtype=torch.int32, device=dev)
        bits = C.c_int(0)
        check(L.svr_rank_table_build(N, ptr(paths), int(path_or), ptr(self.table), C.byref(bits), ptr(ws),
                                     nbytes.value, stream_ptr(dev)), "svr_rank_table_build")
        self.bits = int(bits.value)
        self.shift = rank_shift(path_or)

    def matches(self, path_or):
        return rank_shift(path_or) == self.shift


class PairOrder:
    """Position of every (voxel, octant) pair of an octree in the reference's record order
    (full octree rank, ties by voxel id then octant; svr_pair_order_build), for
    ``RasterState.bin(pair_order=...)``.  Valid for the octree it was built from."""

    def __init__(self, octpaths):
        L = _lib.load()
        dev = octpaths.device
        paths = octpaths.reshape(-1).to(torch.int64).contiguous()
        N = paths.numel()
        nbytes = C.c_size_t(0)
        check(L.svr_rank_table_workspace_bytes(N, C.byref(nbytes)), "svr_rank_table_workspace_bytes")
        ws = _empty_bytes(nbytes.value, dev)
        self.pos = torch.empty(8 * N, dtype=torch.int32, device=dev)
        bits = C.c_int(0)
        check(L.svr_pair_order_build(N, ptr(paths), ptr(self.pos), C.byref(bits), ptr(ws), nbytes.value,
                                     stream_ptr(dev)), "svr_pair_order_build")
        self.bits = int(bits.value)
        self.N = N


_PAIR_ORDER_CACHE = {}


def pair_order_for(octpaths):
    """The PairOrder of an octree, cached on the path tensor's storage and version (a new
    octree after pruning or subdivision gets a new table)."""
    key = (octpaths.data_ptr(), octpaths.numel(), octpaths._version, str(octpaths.device))
    po = _PAIR_ORDER_CACHE.get(key)
    if po is None:
        _PAIR_ORDER_CACHE.clear()
        po = PairOrder(octpaths)
        _PAIR_ORDER_CACHE[key] = po
    return po
