"""Python mirror of quadmap::Depthmap (include/quadmap/depthmap.h:31-89).

Same constructor arguments (note the reference's fx, cx, fy, cy order), the
same add_frames / get* methods, numpy images in and out.  All work happens
in libqm_b200.so through the C-ABI; undistortion (the reference's host-side
cv::remap, seed_matrix.cu:85) is applied here when remap maps are given.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .params import Params, QmParamsC


def _pose12(T) -> np.ndarray:
    T = np.asarray(T, dtype=np.float32)
    if T.shape == (4, 4):
        T = T[:3, :4]
    return np.ascontiguousarray(T.reshape(12), dtype=np.float32)


def _pparams(params):
    if params is None:
        return None
    if isinstance(params, Params):
        return QmParamsC.from_params(params)
    return params


class Depthmap:
    """One camera stream: Depthmap(width, height, fx, cx, fy, cy, remap_1,
    remap_2, semi2dense_ratio) as in depthmap.h:34-44."""

    def __init__(self, width, height, fx, cx, fy, cy, remap_1=None, remap_2=None,
                 semi2dense_ratio=1, params: Params | None = None, device: int = 0):
        L = _lib.lib()
        self._h = ctypes.c_void_p()
        pc = _pparams(params)
        _lib.check(L.qm_depthmap_create(ctypes.byref(self._h), int(width), int(height),
                                        float(fx), float(cx), float(fy), float(cy),
                                        int(semi2dense_ratio),
                                        ctypes.byref(pc) if pc is not None else None,
                                        int(device)))
        self.width, self.height = int(width), int(height)
        self.fx, self.fy, self.cx, self.cy = float(fx), float(fy), float(cx), float(cy)
        self.remap_1, self.remap_2 = remap_1, remap_2

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().qm_depthmap_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_frames(self, img_curr: np.ndarray, T_curr_world) -> bool:
        """Depthmap::add_frames (depthmap.h:46-47): u8 image, world->camera pose."""
        img = np.asarray(img_curr)
        if self.remap_1 is not None:
            import cv2  # host-side undistortion, as the reference's SeedMatrix::input_raw
            img = cv2.remap(img, self.remap_1, self.remap_2, cv2.INTER_LINEAR,
                            borderMode=cv2.BORDER_CONSTANT)
        img = np.ascontiguousarray(img, dtype=np.uint8)
        if img.shape != (self.height, self.width):
            raise ValueError("image shape %s != (%d, %d)" % (img.shape, self.height, self.width))
        T = _pose12(T_curr_world)
        has = ctypes.c_int(0)
        _lib.check(_lib.lib().qm_depthmap_add_frame(self._h, img.ctypes.data, img.strides[0],
                                                    T.ctypes.data, ctypes.byref(has)))
        return bool(has.value)

    def getDepthmap(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        _lib.check(_lib.lib().qm_depthmap_get_depth(self._h, out.ctypes.data, self.width))
        return out

    def getDebugmap(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        _lib.check(_lib.lib().qm_depthmap_get_debug(self._h, out.ctypes.data, self.width))
        return out

    def getVariancemap(self) -> np.ndarray:
        """Fused variance sigma^2 per pixel of the last result."""
        out = np.empty((self.height, self.width), np.float32)
        _lib.check(_lib.lib().qm_depthmap_get_variance(self._h, out.ctypes.data, self.width))
        return out

    def set_semidense(self, on: bool) -> None:
        """Run the semi-dense tracker on every frame (before the first frame)."""
        _lib.check(_lib.lib().qm_depthmap_set_semidense(self._h, 1 if on else 0))

    def getPointCloud(self) -> np.ndarray:
        """(N, 4) float32 rows (x, y, z, intensity) in world coordinates of
        the last result, as Publisher::publishPointCloud builds them
        (publisher.cpp:129-166)."""
        out = np.empty((self.height * self.width, 4), np.float32)
        n = ctypes.c_int()
        _lib.check(_lib.lib().qm_depthmap_get_point_cloud(self._h, out.ctypes.data,
                                                          self.height * self.width,
                                                          ctypes.byref(n)))
        return out[:n.value].copy()

    def getReferenceImage(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.uint8)
        _lib.check(_lib.lib().qm_depthmap_get_reference(self._h, out.ctypes.data, self.width))
        return out

    def getT_world_ref(self) -> np.ndarray:
        T = np.empty(12, np.float32)
        _lib.check(_lib.lib().qm_depthmap_get_T_world_ref(self._h, T.ctypes.data))
        return T.reshape(3, 4)

    def getFx(self):
        return self.fx

    def getFy(self):
        return self.fy

    def getCx(self):
        return self.cx

    def getCy(self):
        return self.cy

    def getWidth(self):
        return self.width

    def getHeight(self):
        return self.height


class BatchDepthmap:
    """N independent Depthmap streams (possibly of different sizes) whose dense
    pipelines run batched: one launch per stage over all streams, replayed
    from a CUDA graph (qm_batch_* in include/qm_capi.h)."""

    def __init__(self, streams, params: Params | None = None, device: int = 0):
        """streams: list of dicts with width, height, fx, fy, cx, cy and optional
        num_hyp, num_slots, semi2dense_ratio."""
        n = len(streams)
        descs = (_lib.QmStreamDesc * n)()
        for i, s in enumerate(streams):
            descs[i].width = int(s["width"])
            descs[i].height = int(s["height"])
            descs[i].cam = _lib.QmCamera(float(s["fx"]), float(s["fy"]), float(s["cx"]),
                                         float(s["cy"]))
            descs[i].num_hyp = int(s.get("num_hyp", 0))
            descs[i].num_slots = int(s.get("num_slots", 0))
            descs[i].semi2dense_ratio = int(s.get("semi2dense_ratio", 1))
        self.shapes = [(int(s["height"]), int(s["width"])) for s in streams]
        self._h = ctypes.c_void_p()
        pc = _pparams(params)
        _lib.check(_lib.lib().qm_batch_create(ctypes.byref(self._h), n, descs,
                                              ctypes.byref(pc) if pc is not None else None,
                                              int(device)))
        self.n = n

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().qm_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_frames(self, imgs, poses):
        """imgs: n u8 arrays (any row pitch, e.g. pinned host views);
        poses: (n, 12) or n world->camera poses.  Returns n booleans."""
        n = self.n
        ptrs = (ctypes.c_void_p * n)()
        strides = (ctypes.c_size_t * n)()
        keep = []
        for i, im in enumerate(imgs):
            a = np.asarray(im)
            if a.dtype != np.uint8 or a.shape != self.shapes[i] or a.strides[1] != 1:
                a = np.ascontiguousarray(a, dtype=np.uint8)
            keep.append(a)
            ptrs[i] = a.ctypes.data
            strides[i] = a.strides[0]
        T = np.ascontiguousarray(np.stack([_pose12(p) for p in poses]), dtype=np.float32)
        has = (ctypes.c_int * n)()
        _lib.check(_lib.lib().qm_batch_add_frames(self._h, ptrs, strides, T.ctypes.data, has))
        return [bool(h) for h in has]

    def submit(self, imgs, poses, outs=None):
        """Pipelined add_frames (qm_batch_submit): returns the n booleans at
        once; the depth of every stream with a result is downloaded into
        outs[i] (float32 (H, W), ideally pinned) and is complete after
        wait().  Image arrays must stay unchanged until the next submit or
        wait returns."""
        n = self.n
        ptrs = (ctypes.c_void_p * n)()
        strides = (ctypes.c_size_t * n)()
        keep = []
        for i, im in enumerate(imgs):
            a = np.asarray(im)
            if a.dtype != np.uint8 or a.shape != self.shapes[i] or a.strides[1] != 1:
                a = np.ascontiguousarray(a, dtype=np.uint8)
            keep.append(a)
            ptrs[i] = a.ctypes.data
            strides[i] = a.strides[0]
        dptrs = dstrides = None
        if outs is not None:
            for i, o in enumerate(outs):
                if o.dtype != np.float32 or o.shape != tuple(self.shapes[i]) or o.strides[1] != 4:
                    raise ValueError("output %d must be a float32 %s array" % (i, self.shapes[i]))
            dptrs = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
            dstrides = (ctypes.c_size_t * n)(*[o.strides[0] // 4 for o in outs])
            keep.extend(outs)
        T = np.ascontiguousarray(np.stack([_pose12(p) for p in poses]), dtype=np.float32)
        has = (ctypes.c_int * n)()
        _lib.check(_lib.lib().qm_batch_submit(self._h, ptrs, strides, T.ctypes.data, has,
                                              dptrs, dstrides))
        # the buffers of the last two steps may still be in use on the device
        self._inflight = (getattr(self, "_inflight", (None, None))[1], keep)
        return [bool(h) for h in has]

    def wait(self) -> None:
        _lib.check(_lib.lib().qm_batch_wait(self._h))
        self._inflight = (None, None)

    def get_depth(self, i, out: np.ndarray | None = None) -> np.ndarray:
        H, W = self.shapes[i]
        if out is None:
            out = np.empty((H, W), np.float32)
        _lib.check(_lib.lib().qm_batch_get_depth(self._h, i, out.ctypes.data,
                                                 out.strides[0] // 4))
        return out

    def get_depths(self, outs=None, streams=None) -> list:
        """Fused depth of several streams (default: all) in one call; `outs`
        are float32 (H, W) arrays with unit column stride (pinned memory
        makes the downloads fastest)."""
        streams = list(range(len(self.shapes))) if streams is None else list(streams)
        if outs is None:
            outs = [np.empty(self.shapes[i], np.float32) for i in streams]
        n = len(streams)
        for i, o in zip(streams, outs):
            if o.dtype != np.float32 or o.shape != tuple(self.shapes[i]) or o.strides[1] != 4:
                raise ValueError("output %d must be a float32 %s array" % (i, self.shapes[i]))
        idx = (ctypes.c_int * n)(*streams)
        ptrs = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
        strides = (ctypes.c_size_t * n)(*[o.strides[0] // 4 for o in outs])
        _lib.check(_lib.lib().qm_batch_get_depths(self._h, n, idx, ptrs, strides))
        return outs

    def get_variance(self, i) -> np.ndarray:
        """Fused variance sigma^2 per pixel of stream i's last result."""
        H, W = self.shapes[i]
        out = np.empty((H, W), np.float32)
        _lib.check(_lib.lib().qm_batch_get_variance(self._h, i, out.ctypes.data, W))
        return out

    def get_point_cloud(self, i) -> np.ndarray:
        """Point cloud of stream i's last result ((N, 4): x, y, z, intensity)."""
        H, W = self.shapes[i]
        out = np.empty((H * W, 4), np.float32)
        n = ctypes.c_int()
        _lib.check(_lib.lib().qm_batch_get_point_cloud(self._h, i, out.ctypes.data, H * W,
                                                       ctypes.byref(n)))
        return out[:n.value].copy()

    def get_debug(self, i) -> np.ndarray:
        H, W = self.shapes[i]
        out = np.empty((H, W), np.float32)
        _lib.check(_lib.lib().qm_batch_get_debug(self._h, i, out.ctypes.data, W))
        return out

    def run_resident(self) -> None:
        _lib.check(_lib.lib().qm_batch_run_resident(self._h))

    def set_semidense(self, on: bool) -> None:
        """Run the semi-dense tracker on every frame of every stream (before
        the first frame)."""
        _lib.check(_lib.lib().qm_batch_set_semidense(self._h, 1 if on else 0))

    def set_branches(self, k: int) -> None:
        """2: two concurrent pipeline branches over the two halves of the
        streams; 1: one sequence (results are the same)."""
        _lib.check(_lib.lib().qm_batch_set_branches(self._h, int(k)))

    def set_graphs(self, on: bool) -> None:
        _lib.check(_lib.lib().qm_batch_set_graphs(self._h, 1 if on else 0))

    def set_group_bytes(self, nbytes: int) -> None:
        """L2 budget of a BP job range (0 = all streams at once)."""
        _lib.check(_lib.lib().qm_batch_set_group_bytes(self._h, int(nbytes)))

    def set_coarse_bp(self, max_cells: int) -> None:
        """Top BP levels with at most max_cells cells in one cluster launch
        (0 = one launch per half-sweep at every level)."""
        _lib.check(_lib.lib().qm_batch_set_coarse_bp(self._h, int(max_cells)))

    def set_stagger(self, on: bool) -> None:
        """Branch i + 1 starts after branch i's cost volume (default off)."""
        _lib.check(_lib.lib().qm_batch_set_stagger(self._h, 1 if on else 0))

    TUNE_FIELDS = ("sweep_warps", "extract_warps", "row_warps", "col_lines", "cost_blocks")

    def set_autotune(self, on: bool) -> None:
        """Time candidate launch shapes per active stream set (default on)."""
        _lib.check(_lib.lib().qm_batch_set_autotune(self._h, 1 if on else 0))

    def set_tune(self, sweep_warps=8, extract_warps=8, row_warps=2, col_lines=4,
                 cost_blocks=5) -> None:
        """Fix the launch shapes (turns autotune off)."""
        t = (ctypes.c_int * 5)(sweep_warps, extract_warps, row_warps, col_lines, cost_blocks)
        _lib.check(_lib.lib().qm_batch_set_tune(self._h, t))

    def get_tune(self) -> dict:
        """Launch shapes of the last run."""
        t = (ctypes.c_int * 5)()
        _lib.check(_lib.lib().qm_batch_get_tune(self._h, t))
        return dict(zip(self.TUNE_FIELDS, list(t)))

    def last_launches(self) -> int:
        c = ctypes.c_int()
        _lib.check(_lib.lib().qm_batch_last_launches(self._h, ctypes.byref(c)))
        return c.value

    KERNEL_KINDS = ("quadtree", "cost", "pyramid", "msg_init", "bp_sweep", "extract",
                    "row_solve", "col_solve", "fuse_transform", "fuse_fill", "fuse_update")

    def stream_ptr(self) -> int:
        """cudaStream_t the batch's kernels run on (for timing events)."""
        s = ctypes.c_void_p()
        _lib.check(_lib.lib().qm_batch_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def profile(self):
        """{kind: (ms, launches)} of one eager resident run (qm_batch_profile)."""
        n = len(self.KERNEL_KINDS)
        ms = (ctypes.c_float * n)()
        cnt = (ctypes.c_int * n)()
        _lib.check(_lib.lib().qm_batch_profile(self._h, ms, cnt))
        return {k: (ms[i], cnt[i]) for i, k in enumerate(self.KERNEL_KINDS)}

    def device_depth_ptr(self, i) -> int:
        p = ctypes.c_void_p()
        _lib.check(_lib.lib().qm_batch_device_depth(self._h, i, ctypes.byref(p)))
        return p.value
