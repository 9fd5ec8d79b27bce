"""Batched multi-view training step on the sm_100a library.

One step renders every view of a batch forward and backward and applies the shipped SDF
regularisers and Adam (train.py:324-709 for one view at a time): corner-SDF gather, SH
colour for all views, preprocess, binning, render forward, render adjoint, gradient scatter
to grid points, SH adjoint, Laplacian + grid-Eikonal smoothness adjoints, Adam on the grid
SDF and the SH coefficients.  Each stage is one launch for the whole batch.

The upstream gradients dL/d(color, depth, normal, T) stand in for the photometric and
normal-consistency losses, which run upstream of the rasterizer and are out of scope.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_ptr
from .raster import PairOrder, RankTable, RasterState
from . import utils


def flat_views(shapes, device, align=64):
    """One zeroed float32 buffer holding a view of each shape, every view starting on a
    multiple of ``align`` elements (256 bytes): one fill zeroes them all and one collective
    exchanges them all.  The padding between views stays zero.  Returns (flat, views)."""
    offs, total = [], 0
    for shape in shapes:
        n = int(np.prod(shape)) if len(shape) else 1
        offs.append((total, n))
        total += (n + align - 1) // align * align
    flat = torch.zeros(max(total, 1), dtype=torch.float32, device=device)
    return flat, [flat[o:o + n].view(shape) for (o, n), shape in zip(offs, shapes)]


class BatchedTrainStep:

    def __init__(self, scene, cams, device="cuda", lr=(1e-3, 1e-3, 1e-4), betas=(0.1, 0.99), eps=1e-15,
                 lambda_ls=1e-3, lambda_ge=1e-3, lambda_R_concen=0.0, sh_degree=3, seed=0, fused_smoothness=True,
                 sh_dtype="f32", normal_losses=None, dense_ranks=True, binning="tiles", view_chunk=None):
        """``sh_dtype="bf16"`` stores the SH coefficients in bf16 (the precision configuration):
        colours, compositing, transmittance and every gradient stay f32, Adam keeps f32 moments
        and rounds the updated coefficients to nearest bf16.  ``normal_losses`` (a dict with
        any of lambda_dmean, dmean_ks, dmean_tol_deg, lambda_dmed; train.py:159-166, 418-425)
        adds the normal-from-depth consistency losses of the rendered batch: one launch each
        between the render forward and the adjoint, their gradients added to the upstream
        depth / normal planes the adjoint reads.  ``dense_ranks`` bins with the octree's dense
        (voxel, octant) ranks (``raster.RankTable``, built here once): the same record order
        with a narrower sort key.  ``binning="tiles"`` (default) bins with the per-tile sort
        (``raster.PairOrder``, built here once; svr_bin_tiles), ``"radix"`` with the global
        radix sort of svr_bin_and_sort; both give the same record order.  ``view_chunk=k`` renders
        the step's views k at a time (forward and adjoint of each chunk, then the smoothness
        adjoint and Adam once), so that the per-(view, voxel) state of a large batch is held for
        one chunk at a time; the gradients of all chunks are summed before Adam."""
        dev = torch.device(device)
        self.dev = dev
        t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a)).to(dev, dt)
        self.N = scene.n_vox
        self.octpath = t(scene.octpath, torch.int64)
        self.centers = t(scene.vox_center)
        self.lengths = t(scene.vox_size).reshape(-1).contiguous()
        self.is_leaf = t(scene.is_leaf, torch.uint8)
        self.vox_key = t(scene.vox_key, torch.int64)
        self.grid = t(scene.geo_grid_pts)
        if sh_dtype not in ("f32", "bf16"):
            raise ValueError("sh_dtype must be 'f32' or 'bf16'")
        self.sh_bf16 = sh_dtype == "bf16"
        sh_t = torch.bfloat16 if self.sh_bf16 else torch.float32
        self.sh0 = t(scene.sh0).to(sh_t).contiguous()
        self.shs = t(scene.shs).to(sh_t).contiguous()
        self.M_sh = 1 + scene.shs.shape[1]
        self.sh_degree = sh_degree
        self.s_val = torch.tensor([scene.s_val], dtype=torch.float32, device=dev)
        self.views = [dict(width=c.width, height=c.height, tanfovx=c.tanfovx, tanfovy=c.tanfovy, cx=c.cx, cy=c.cy,
                           near=c.near, w2c=t(c.w2c), c2w=t(c.c2w), bg=torch.zeros(3, device=dev))
                      for c in cams]
        self.V = len(cams)
        self.cam_pos = torch.stack([v["c2w"][:3, 3] for v in self.views]).contiguous()
        self.view_chunk = int(view_chunk) if view_chunk else None
        if self.view_chunk and normal_losses:
            raise ValueError("view_chunk does not take the normal-from-depth losses")
        k = self.view_chunk or self.V
        self.chunks = [(a, min(a + k, self.V)) for a in range(0, self.V, k)]
        offs = np.concatenate([[0], np.cumsum([c.width * c.height for c in cams])]).astype(np.int64)
        self.chunk_pix = [(int(offs[a]), int(offs[b])) for a, b in self.chunks]
        self.V_buf = max(b - a for a, b in self.chunks)     # views held per chunk
        self.P = sum(c.width * c.height for c in cams)
        self.rays = self.P
        self.lr, self.betas, self.eps = lr, betas, eps
        self.lambda_R = float(lambda_R_concen)
        self.params = [self.grid, self.sh0, self.shs]
        self.param_bf16 = [False, self.sh_bf16, self.sh_bf16]
        self.adam_m = [torch.zeros(p.shape, dtype=torch.float32, device=dev) for p in self.params]
        self.adam_v = [torch.zeros(p.shape, dtype=torch.float32, device=dev) for p in self.params]
        self.adam_step = 0
        # dense-grid table for the smoothness losses (rebuilt only on prune / subdivide)
        lv_max = int(scene.octlevel.max())
        self.res_pow2 = min(lv_max, 9)
        res = 1 << self.res_pow2
        self.grid_mask, self.grid_keys, self.grid2voxel = utils.valid_gradient_table(
            self.centers, self.lengths, torch.zeros(3, device=dev), scene.scene_extent, self.res_pow2, self.is_leaf)
        ext = np.float32(scene.scene_extent)
        coord = ((scene.vox_center - scene.vox_size * np.float32(0.5)) + ext * np.float32(0.5)) / ext * np.float32(res)
        self.grid_voxel_coord = t(np.round(coord))
        self.grid_voxel_size = t(np.round(scene.vox_size / ext * np.float32(res))).reshape(-1)
        self.vox_size_min_inv = float(res) / float(scene.scene_extent)
        self.active = torch.arange(self.grid_keys.numel(), dtype=torch.int32, device=dev)
        from .grid_loss_bw import dense_index
        self.grid_index = dense_index(self.grid_keys, res)
        self.lambda_ls, self.lambda_ge = lambda_ls, lambda_ge
        self.fused_smoothness = fused_smoothness
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.seed = seed
        # upstream gradients (seeded synthetic)
        g = torch.Generator(device=dev).manual_seed(seed)
        P = self.P
        self.dcolor = torch.randn(3 * P, device=dev, generator=g)
        self.ddepth = torch.randn(4 * P, device=dev, generator=g)
        self.dnormal = torch.randn(3 * P, device=dev, generator=g)
        self.dT = torch.zeros(P, device=dev)
        self.gt = torch.rand(3 * P, device=dev, generator=g) if self.lambda_R > 0 else None
        nl = dict(lambda_dmean=0.0, dmean_ks=3, dmean_tol_deg=90.0, lambda_dmed=0.0)
        nl.update(normal_losses or {})
        self.normal_losses = nl
        self.nd_on = nl["lambda_dmean"] > 0 or nl["lambda_dmed"] > 0
        if self.nd_on:
            self.ddepth_w = torch.empty_like(self.ddepth)
            self.dnormal_w = torch.empty_like(self.dnormal)
            self.nd_loss = torch.zeros(self.V, dtype=torch.float64, device=dev)
        # per-step buffers
        self.geos = torch.empty(self.N, 8, device=dev)
        self.rgbs = torch.empty(self.V_buf * self.N, 3, device=dev)
        self.dvox = torch.zeros(self.N, 12, device=dev)
        self.drgbs = torch.zeros(self.V_buf * self.N, 3, device=dev)
        self.ds = torch.zeros(1, device=dev)
        # the gradients are views into one flat buffer, so that a step zeroes them with one
        # fill and a data-parallel step exchanges them with one all-reduce (``grad_flat``)
        self.grad_flat, self.grads = flat_views([p.shape for p in self.params], dev)
        self.all_idx = torch.arange(self.N, dtype=torch.int64, device=dev)
        self.state = None
        self.ev = None
        # graph replay state: OR of every leaf's octree path (a superset of the rendered
        # paths, so the trimmed sort key stays exact for any camera), device step counter,
        # per-group Adam coefficient tables
        leaf_paths = np.asarray(scene.octpath, dtype=np.int64)[np.asarray(scene.is_leaf).astype(bool).reshape(-1)]
        self.path_or_all = int(np.bitwise_or.reduce(leaf_paths.view(np.uint64))) if leaf_paths.size else 0
        if binning not in ("tiles", "radix"):
            raise ValueError("binning is 'tiles' or 'radix'")
        self.binning = binning
        self.pair_order = PairOrder(self.octpath) if binning == "tiles" else None
        self.rank_table = RankTable(self.octpath, self.path_or_all) if dense_ranks and binning == "radix" else None
        self.graph = None
        self.graph_b = None
        self.graph_out = None
        self.capacity = None
        self.step_dev = None
        self.coef_tables = None
        self.coef_rows = 0
        self._dev_step_synced = False
        self.tuned = None

    # ------------------------------------------------------------------ one step
    def step(self, time_render=False, grad_hook=None):
        """One training step.  ``grad_hook(grads)`` runs between the adjoints and Adam (the
        data-parallel all-reduce of the gradients goes there; ``grad_flat`` holds all of them
        contiguously).  With ``time_render`` every
        stage is bracketed by CUDA events on the launching stream (see ``stage_ms``)."""
        out = self._body(False, time_render, grad_hook)
        self.adam_step += 1
        self._dev_step_synced = False
        return out

    def _body(self, graph, time_render=False, grad_hook=None):
        marks = []

        def mark(name, event=None):
            """Event mark ending stage `name`; `event` = one the library records itself."""
            if time_render:
                e = event
                if e is None:
                    e = torch.cuda.Event(enable_timing=True)
                    e.record()
                marks.append((name, e))
        mark.on = time_render

        mark("start")
        if self.view_chunk:
            return self._body_chunked(graph, mark, grad_hook, marks, time_render)
        fw = self._forward_part(graph, mark)
        return self._backward_part(graph, mark, grad_hook, fw, marks, time_render)

    def _body_chunked(self, graph, mark, grad_hook, marks, time_render):
        """One step over the views chunk by chunk: per chunk SH, preprocess, binning, render
        forward and adjoint and the SH adjoint (added up); then smoothness, the gradient
        scatter and Adam once."""
        L = _lib.load()
        st = stream_ptr(self.dev)
        N = self.N
        check(L.svr_gather_geo(N, ptr(self.all_idx), ptr(self.vox_key), ptr(self.grid), ptr(self.geos), st),
              "gather")
        self.dvox.zero_()
        self.ds.zero_()
        self.grad_flat.zero_()
        mark("gather+zero")
        sh_eval = L.svr_sh_eval_views_bf16 if self.sh_bf16 else L.svr_sh_eval_views
        gt = self.gt
        for k, ((a, b), (pa, pb)) in enumerate(zip(self.chunks, self.chunk_pix)):
            nv = b - a
            cam_pos = self.cam_pos[a:b]
            rgbs = self.rgbs[: nv * N]
            check(sh_eval(N, nv, self.sh_degree, self.M_sh, ptr(self.centers), ptr(cam_pos), ptr(self.sh0),
                          ptr(self.shs), ptr(rgbs), st), "sh views")
            state = RasterState(self.views[a:b], N, self.dev)
            state.preprocess(self.octpath, self.centers, self.lengths, self.is_leaf)
            if graph:
                state.bin(self.octpath, capacity=self.capacity[k], path_or=self.path_or_all,
                          rank_table=self.rank_table, pair_order=self.pair_order)
            else:
                state.bin(self.octpath, rank_table=self.rank_table, pair_order=self.pair_order)
            color, depth, normal, T, _ = state.render(3, True, True, self.centers, self.lengths, self.geos, rgbs,
                                                      self.s_val, rgb_per_view=True)
            drgbs = self.drgbs[: nv * N]
            drgbs.zero_()
            state.render_backward(True, True, self.s_val, T, self.dcolor[3 * pa:3 * pb], self.ddepth[4 * pa:4 * pb],
                                  self.dnormal[3 * pa:3 * pb], self.dT[pa:pb], lambda_R_concen=self.lambda_R,
                                  gt_color=None if gt is None else gt[3 * pa:3 * pb], drgbs=drgbs, dvox=self.dvox,
                                  ds=self.ds)
            check(L.svr_sh_eval_views_bw_add(N, nv, self.sh_degree, self.M_sh, ptr(self.centers), ptr(cam_pos),
                                             ptr(drgbs), ptr(self.grads[1]), ptr(self.grads[2]), st), "sh views bw")
            self.state = state
            mark(f"chunk{k}")
        G = self.grid_keys.numel()
        seed = self.seed if graph else self.seed + self.adam_step
        step_ptr = ptr(self.step_dev) if graph else None
        check(L.svr_smoothness_bw_vox(G, G, None, ptr(self.grid_keys), ptr(self.grid2voxel), 1 << self.res_pow2,
                                      ptr(self.grid_mask), ptr(self.grid_index), ptr(self.grid_voxel_coord),
                                      ptr(self.grid_voxel_size), N, ptr(self.geos), float(self.lambda_ls),
                                      float(self.lambda_ge), self.vox_size_min_inv, seed, step_ptr,
                                      ptr(self.dvox), 12, ptr(self.status), st), "smoothness")
        check(L.svr_scatter_vox_grads(N, 12, ptr(self.vox_key), ptr(self.dvox), ptr(self.grads[0]), st), "scatter")
        mark("smoothness+scatter")
        if grad_hook is not None:
            grad_hook(self.grads)
            mark("allreduce")
        self._adam(graph)
        mark("adam")
        self.ev = marks if time_render else None
        return color, T

    def _forward_part(self, graph, mark):
        """Gather, SH, preprocess, binning and the render forward of the batch."""
        L = _lib.load()
        st = stream_ptr(self.dev)
        N = self.N
        check(L.svr_gather_geo(N, ptr(self.all_idx), ptr(self.vox_key), ptr(self.grid), ptr(self.geos), st),
              "gather")
        sh_eval = L.svr_sh_eval_views_bf16 if self.sh_bf16 else L.svr_sh_eval_views
        check(sh_eval(N, self.V, self.sh_degree, self.M_sh, ptr(self.centers), ptr(self.cam_pos),
                      ptr(self.sh0), ptr(self.shs), ptr(self.rgbs), st), "sh views")
        mark("gather+sh")
        state = RasterState(self.views, N, self.dev)
        state.preprocess(self.octpath, self.centers, self.lengths, self.is_leaf)
        mark("preprocess")
        if graph:
            state.bin(self.octpath, capacity=self.capacity, path_or=self.path_or_all, rank_table=self.rank_table,
                      pair_order=self.pair_order)
        else:
            state.bin(self.octpath, rank_table=self.rank_table, pair_order=self.pair_order)
        mark("count+sort")
        pack_ev = None
        if getattr(mark, "on", False) and not graph:
            # the library records this event between its record packing and render launches
            pack_ev = torch.cuda.Event(enable_timing=True)
            pack_ev.record()   # creates the event; the library records it again after packing
            check(L.svr_set_pack_event(pack_ev.cuda_event), "pack event")
        try:
            color, depth, normal, T, _ = state.render(3, True, True, self.centers, self.lengths, self.geos,
                                                      self.rgbs, self.s_val, rgb_per_view=True)
        finally:
            if pack_ev is not None:
                L.svr_set_pack_event(None)
        if pack_ev is not None:
            mark("pack", pack_ev)
        mark("render_fwd")
        return state, color, depth, normal, T

    def _backward_part(self, graph, mark, grad_hook, fw, marks, time_render):
        """Normal losses (when on), the render adjoint, smoothness, scatter, SH adjoint and
        Adam; reads the upstream gradient planes (dcolor, ddepth, dnormal, gt)."""
        L = _lib.load()
        st = stream_ptr(self.dev)
        N = self.N
        state, color, depth, normal, T = fw
        ddepth, dnormal = self.ddepth, self.dnormal
        if self.nd_on:
            # loss_utils.py:345-407 on the rendered planes, added to the upstream gradients
            nl = self.normal_losses
            self.ddepth_w.copy_(self.ddepth)
            self.dnormal_w.copy_(self.dnormal)
            self.nd_loss.zero_()
            if nl["lambda_dmean"] > 0:
                tol = float(np.float32(np.cos(np.deg2rad(nl["dmean_tol_deg"]))))
                check(L.svr_normal_depth_loss(state.views, self.V, 0, int(nl["dmean_ks"]), tol if tol > 0 else -1.0,
                                              float(nl["lambda_dmean"]), ptr(depth), ptr(normal), ptr(T),
                                              ptr(self.nd_loss), ptr(self.ddepth_w), ptr(self.dnormal_w), st),
                      "normal-depth loss")
            if nl["lambda_dmed"] > 0:
                check(L.svr_normal_depth_loss(state.views, self.V, 1, 3, -1.0, float(nl["lambda_dmed"]), ptr(depth),
                                              ptr(normal), ptr(T), ptr(self.nd_loss), ptr(self.ddepth_w),
                                              ptr(self.dnormal_w), st), "normal-median loss")
            ddepth, dnormal = self.ddepth_w, self.dnormal_w
            mark("normal_losses")
        self.dvox.zero_()
        self.drgbs.zero_()
        self.ds.zero_()
        mark("zero")
        state.render_backward(True, True, self.s_val, T, self.dcolor, ddepth, dnormal, self.dT,
                              lambda_R_concen=self.lambda_R, gt_color=self.gt, drgbs=self.drgbs, dvox=self.dvox,
                              ds=self.ds)
        mark("render_bwd")
        G, A = self.grid_keys.numel(), self.active.numel()
        seed = self.seed if graph else self.seed + self.adam_step
        step_ptr = ptr(self.step_dev) if graph else None
        if self.fused_smoothness:
            # both adjoints in one pass, accumulated per voxel corner into dvox, then moved to
            # the grid points with the render adjoint's corner gradients
            check(L.svr_smoothness_bw_vox(G, G, None, ptr(self.grid_keys), ptr(self.grid2voxel), 1 << self.res_pow2,
                                          ptr(self.grid_mask), ptr(self.grid_index), ptr(self.grid_voxel_coord),
                                          ptr(self.grid_voxel_size), N, ptr(self.geos), float(self.lambda_ls),
                                          float(self.lambda_ge), self.vox_size_min_inv, seed, step_ptr,
                                          ptr(self.dvox), 12, ptr(self.status), st), "smoothness")
            mark("smoothness")
        self.grad_flat.zero_()
        check(L.svr_scatter_vox_grads(N, 12, ptr(self.vox_key), ptr(self.dvox), ptr(self.grads[0]), st), "scatter")
        check(L.svr_sh_eval_views_bw(N, self.V, self.sh_degree, self.M_sh, ptr(self.centers), ptr(self.cam_pos),
                                     ptr(self.drgbs), ptr(self.grads[1]), ptr(self.grads[2]), st), "sh views bw")
        mark("scatter+sh_bw")
        if not self.fused_smoothness:
            common = (G, A, ptr(self.active), ptr(self.grid_keys), ptr(self.grid2voxel), 1 << self.res_pow2,
                      ptr(self.grid_mask), ptr(self.grid_index), ptr(self.grid_voxel_coord),
                      ptr(self.grid_voxel_size), N, ptr(self.vox_key), ptr(self.grid), self.grid.numel())
            if graph:
                for fn, lam in ((L.svr_laplacian_bw_at_step, self.lambda_ls),
                                (L.svr_eikonal_bw_at_step, self.lambda_ge)):
                    check(fn(*common, float(lam), self.vox_size_min_inv, seed, step_ptr, ptr(self.grads[0]),
                             ptr(self.status), st), "grid loss")
            else:
                for fn, lam in ((L.svr_laplacian_bw, self.lambda_ls), (L.svr_eikonal_bw, self.lambda_ge)):
                    check(fn(*common, float(lam), self.vox_size_min_inv, seed, ptr(self.grads[0]),
                             ptr(self.status), st), "grid loss")
            mark("smoothness")
        if grad_hook is not None:
            grad_hook(self.grads)
            mark("allreduce")
        self._adam(graph)
        mark("adam")
        self.state = state
        self.ev = marks if time_render else None
        return color, T

    def _adam(self, graph):
        """Adam on grid / sh0 / shs: in a graph the step number comes from the device counter
        and the bias corrections from the captured tables."""
        L = _lib.load()
        st = stream_ptr(self.dev)
        if graph:
            check(L.svr_counter_add(ptr(self.step_dev), 1, st), "counter")
            for p, g, m, v, tab, bf in zip(self.params, self.grads, self.adam_m, self.adam_v, self.coef_tables,
                                           self.param_bf16):
                fn = L.svr_adam_step_bf16_at if bf else L.svr_adam_step_at
                check(fn(p.numel(), 0, 0, ptr(p), ptr(g), ptr(m), ptr(v), ptr(tab), self.coef_rows,
                         ptr(self.step_dev), self.betas[0], self.betas[1], self.eps, ptr(self.status), st), "adam")
        else:
            for p, g, m, v, lr, bf in zip(self.params, self.grads, self.adam_m, self.adam_v, self.lr, self.param_bf16):
                fn = L.svr_adam_step_bf16 if bf else L.svr_adam_step
                check(fn(p.numel(), 0, 0, ptr(p), ptr(g), ptr(m), ptr(v), float(self.adam_step + 1),
                         float(lr), self.betas[0], self.betas[1], self.eps, st), "adam")

    # ------------------------------------------------------------------ CUDA graph
    def autotune(self, reps=3, cache=None):
        """Choose the render kernels' launch configuration for this batch by timing each
        configuration on the last step's binned records (svraster_b200.autotune).  Runs one
        eager step first if none ran yet; the gradient buffers are left as a step leaves them."""
        from . import autotune as AT
        if self.state is None:
            self.step()
        st = self.state

        def fwd():
            st.render(3, True, True, self.centers, self.lengths, self.geos, self.rgbs, self.s_val,
                      rgb_per_view=True)

        color, depth, normal, T, _ = st.render(3, True, True, self.centers, self.lengths, self.geos, self.rgbs,
                                                self.s_val, rgb_per_view=True)

        def bwd():
            st.render_backward(True, True, self.s_val, T, self.dcolor, self.ddepth, self.dnormal, self.dT,
                               lambda_R_concen=self.lambda_R, gt_color=self.gt, drgbs=self.drgbs, dvox=self.dvox,
                               ds=self.ds)
        key = AT.workload_key(self.dev, self.V, self.P, self.N, st.num_rendered)
        self.tuned = AT.tune_render(fwd, bwd, reps=reps, key=key, cache=cache)
        torch.cuda.synchronize(self.dev)
        return self.tuned

    def capture(self, capacity=None, rows=1 << 20, split=False, upstream_sets=1, grad_hook=None):
        """Capture one whole step (gather, SH, preprocess, scan, duplicate, sort, pack, render
        forward and adjoint, scatter, SH adjoint, smoothness adjoints, Adam) into a CUDA graph.
        ``capacity`` bounds the records per step (default: this batch's record total, found by
        one counting pass); a replay that needs more sets status bit 8 (``graph_status``).
        ``split=True`` captures two graphs sharing one memory pool: the forward part (up to
        the render forward) and the backward part (everything that reads the upstream
        gradient planes), replayed by ``replay_forward`` / ``replay_backward`` (``replay`` runs
        both), so that a caller can refill the upstream planes while the forward part runs.  With
        ``upstream_sets=2`` (split only) one backward graph is captured per set of upstream
        planes (``upstream(i)``); ``replay_backward(i)`` reads set i, so the next step's
        planes can be copied into the other set during the whole current step.
        ``grad_hook(grads)`` is captured between the adjoints and Adam, like ``step``'s (the
        data-parallel NCCL all-reduce of ``grad_flat`` is captured into the graph with it; a
        graph holding NCCL calls must be released before the process group is destroyed).
        Returns the number of this library's kernels in the graph(s)."""
        L = _lib.load()
        if self.view_chunk and split:
            raise ValueError("a step with view_chunk is captured whole (split=False)")

        def count(views):
            probe = RasterState(views, self.N, self.dev)
            probe.preprocess(self.octpath, self.centers, self.lengths, self.is_leaf)
            R, por = C.c_int64(0), C.c_uint64(0)
            check(L.svr_count_rendered(self.N * len(views), ptr(probe.geom), C.byref(R), C.byref(por),
                                       stream_ptr(self.dev)), "count")
            return int(R.value)
        if self.view_chunk:
            self.capacity = [max(count(self.views[a:b]), 1) if capacity is None else int(capacity)
                             for a, b in self.chunks]
        else:
            if capacity is None:
                capacity = count(self.views)
            self.capacity = max(int(capacity), 1)
        self.coef_rows = int(rows)
        self.coef_tables = []
        for lr in self.lr:
            tab = np.empty((self.coef_rows, 2), np.float32)
            check(L.svr_adam_coef_table(0, float(lr), self.betas[0], self.betas[1], self.coef_rows,
                                        tab.ctypes.data_as(C.c_void_p)), "adam table")
            self.coef_tables.append(torch.from_numpy(tab).to(self.dev))
        self.step_dev = torch.full((1,), self.adam_step, dtype=torch.int64, device=self.dev)
        torch.cuda.synchronize(self.dev)
        n0 = L.svr_kernel_launches()
        # the step counter and parameters must not move during capture: capture runs no work
        nomark = lambda name: None
        if upstream_sets not in (1, 2) or (upstream_sets == 2 and not split):
            raise ValueError("upstream_sets is 1, or 2 with split=True")
        names = ("dcolor", "ddepth", "dnormal", "gt")
        sets = [tuple(getattr(self, n) for n in names)]
        if upstream_sets == 2:
            sets.append(tuple(None if t is None else t.clone() for t in sets[0]))
        self._up_sets = sets
        if split:
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._graph_fw = self._forward_part(True, nomark)
            self.graph_bs = []
            for up in sets:
                for n, t in zip(names, up):
                    setattr(self, n, t)
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, pool=self.graph.pool()):
                    self.graph_out = self._backward_part(True, nomark, grad_hook, self._graph_fw, [], False)
                self.graph_bs.append(g)
            for n, t in zip(names, sets[0]):
                setattr(self, n, t)
            self.graph_b = self.graph_bs[0]
        else:
            self.graph = torch.cuda.CUDAGraph()
            self.graph_b = None
            with torch.cuda.graph(self.graph):
                self.graph_out = self._body(True, grad_hook=grad_hook)
        self.graph_launches = int(L.svr_kernel_launches() - n0)
        torch.cuda.synchronize(self.dev)
        self._dev_step_synced = True
        return self.graph_launches

    def replay(self):
        """One step by graph replay (capture first).  Returns (color, T) of the replayed step;
        their storage is reused by the next replay."""
        if self.graph is None:
            raise RuntimeError("capture() first")
        if self.adam_step + 1 >= self.coef_rows:
            raise RuntimeError("Adam coefficient table exhausted; capture again with more rows")
        self.replay_forward()
        return self.replay_backward()

    def replay_forward(self):
        """The forward part of a step captured with ``split=True`` (or the whole step of an
        unsplit capture, whose ``replay_backward`` is then a no-op)."""
        if self.graph is None:
            raise RuntimeError("capture() first")
        if self.adam_step + 1 >= self.coef_rows:
            raise RuntimeError("Adam coefficient table exhausted; capture again with more rows")
        if not self._dev_step_synced:
            self.step_dev.fill_(self.adam_step)
            self._dev_step_synced = True
        self.graph.replay()
        if self.graph_b is None:
            self.adam_step += 1
        return self.graph_out

    def replay_backward(self, upstream_set=0):
        """The backward part of a split capture: reads the upstream gradient planes of set
        ``upstream_set`` as they are when it runs.  Returns (color, T) of the step."""
        if self.graph_b is not None:
            self.graph_bs[upstream_set].replay()
            self.adam_step += 1
        return self.graph_out

    def upstream(self, i=0):
        """The upstream tensors (dcolor, ddepth, dnormal, gt) of set i of the last capture
        (set 0 is the step's own)."""
        if getattr(self, "_up_sets", None):
            return self._up_sets[i]
        return (self.dcolor, self.ddepth, self.dnormal, self.gt)

    def graph_status(self):
        """Status words after replays: (raster status, smoothness / Adam status)."""
        torch.cuda.synchronize(self.dev)
        return self.state.status(), int(self.status.item())

    @staticmethod
    def stage_ms(marks):
        """{stage: ms} from the event marks of one timed step (call after synchronising)."""
        out = {}
        for (_, a), (name, b) in zip(marks[:-1], marks[1:]):
            out[name] = a.elapsed_time(b)
        return out

    def record_counts(self):
        """R (records) and R' (records up to tile_last) of the last step."""
        st = self.state
        _, ranges, tl, _ = st.binning_fields()
        r_prime = int((tl.to(torch.int64) - ranges[:, 0].to(torch.int64)).clamp_min(0).sum().item())
        return st.num_rendered, r_prime
