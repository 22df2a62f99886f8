"""Many views of one or more visualizations in one persistent launch.

The reference renders one camera per ``doVisualization`` (lib/isaac.hpp:2008-2061);
a server that streams several cameras, or several timesteps side by side, calls
it once per view.  ``IsaacBatch`` renders all of them with one kernel launch
whose CTAs pull screen tiles from a shared work queue, optionally as one
captured CUDA graph that also holds the per-timestep buffer updates.  Every
frame is bit-identical to the frame ``IsaacVisualization.render`` draws for the
same context and camera.

Each visualization in a batch must use the combined renderer with volume
sources only: no iso threshold, no particle source with weight, no SSAO.
"""

from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import BatchConfig, View, check

__all__ = ["IsaacBatch", "BatchConfig"]


def _torch():
    import torch

    return torch


class IsaacBatch:
    """Views ``(visualization index, width, height, projection, modelview)``
    over the visualizations ``vis``; each view renders into its own
    (height, width, 4) uint8 CUDA tensor, ``self.frames[i]``."""

    def __init__(self, vis: Sequence, views: Sequence[tuple]):
        torch = _torch()
        self.lib = _lib.load()
        self.vis = list(vis)
        self.frames = []
        arr = (View * len(views))()
        for i, (ci, w, h, proj, mv) in enumerate(views):
            out = torch.zeros((h, w, 4), dtype=torch.uint8, device="cuda")
            self.frames.append(out)
            v = arr[i]
            v.ctx_index = int(ci)
            v.width = int(w)
            v.height = int(h)
            v.projection[:] = [float(x) for x in np.asarray(proj, dtype=np.float64).reshape(16)]
            v.modelview[:] = [float(x) for x in np.asarray(mv, dtype=np.float64).reshape(16)]
            v.rgba_dev = out.data_ptr()
        ctxs = (C.c_void_p * len(self.vis))(*[x.ctx for x in self.vis])
        h = C.c_void_p()
        check(self.lib.isaacb_batch_create(ctxs, len(self.vis), arr, len(views), C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self.lib.isaacb_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _stream():
        return C.c_void_p(_torch().cuda.current_stream().cuda_stream)

    # ------------------------------------------------------------------ settings
    @property
    def config(self) -> BatchConfig:
        cfg = BatchConfig()
        check(self.lib.isaacb_batch_get_config(self.handle, C.byref(cfg)))
        return cfg

    def setConfig(self, tile_w: int = 32, tile_h: int = 8, blocks_per_sm: int = 0, skip_empty: int = -1):
        """Tile shape (256 pixels, width a multiple of 8), CTAs per SM (0 = as many
        as fit) and empty-brick skipping (-1 = decided from the last update)."""
        cfg = BatchConfig(tile_w, tile_h, blocks_per_sm, skip_empty)
        check(self.lib.isaacb_batch_set_config(self.handle, C.byref(cfg)))

    def setCamera(self, view: int, projection, modelview_m):
        p = np.ascontiguousarray(projection, dtype=np.float64).reshape(16)
        m = np.ascontiguousarray(modelview_m, dtype=np.float64).reshape(16)
        check(self.lib.isaacb_batch_set_camera(self.handle, view, p.ctypes.data_as(_lib._dp), m.ctypes.data_as(_lib._dp)))

    def setCounting(self, on: bool):
        check(self.lib.isaacb_batch_set_counting(self.handle, int(on)))

    def launchCount(self) -> int:
        """Kernels the last render or capture enqueued (a graph launch replays the captured ones)."""
        n = C.c_uint32()
        check(self.lib.isaacb_batch_get_launch_count(self.handle, C.byref(n)))
        return int(n.value)

    def samples(self) -> int:
        n = C.c_uint64()
        check(self.lib.isaacb_batch_get_samples(self.handle, self._stream(), C.byref(n)))
        return int(n.value)

    # ------------------------------------------------------------------ frames
    def render(self, update: bool = True):
        """Buffer updates of every visualization (when ``update``), then all views, asynchronously."""
        check(self.lib.isaacb_batch_render(self.handle, self._stream(), int(update)))

    def capture(self, update: bool = True):
        """Capture one batch frame as a CUDA graph (on the current, non-default stream)."""
        check(self.lib.isaacb_batch_capture(self.handle, self._stream(), int(update)))

    def launchGraph(self):
        check(self.lib.isaacb_batch_launch_graph(self.handle, self._stream()))

    def autotune_step(self, steps=(0.5, 0.75, 1.0, 1.5), threshold_db: float = 40.0, repeat: int = 3) -> dict:
        """Step schedule under a quality constraint: every view is rendered at step 0.5
        (the reference's default) as the judge, then at each candidate step; a candidate
        qualifies when every view's PSNR against its judge frame is at or above
        ``threshold_db``, and the fastest qualifying candidate (render time by CUDA
        events over ``repeat`` launches) is set on every visualization.  Frames at a
        larger step are not bit-identical to the reference's step; the report says how
        far they are."""
        from .recon import psnr

        torch = _torch()
        for v in self.vis:
            v.setStep(0.5)
        self.render(update=False)
        judge = [f.clone() for f in self.frames]
        acc = torch.zeros(1, dtype=torch.int64, device="cuda")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        results = []
        for st in steps:
            for v in self.vis:
                v.setStep(st)
            self.render(update=False)
            ps = [psnr(f, j, acc) for f, j in zip(self.frames, judge)]
            torch.cuda.synchronize()
            e0.record()
            for _ in range(repeat):
                self.render(update=False)
            e1.record()
            e1.synchronize()
            # an identical frame has infinite PSNR; the report keeps JSON-safe numbers (None)
            fin = [x for x in ps if x != float("inf")]
            results.append({"step": st, "ms": e0.elapsed_time(e1) / repeat, "psnr_min": min(fin) if fin else None,
                            "psnr_mean": sum(fin) / len(fin) if fin else None, "identical_views": len(ps) - len(fin),
                            "qualifies": min(ps) >= threshold_db})
        ok = [r for r in results if r["qualifies"]]
        best = min(ok, key=lambda r: r["ms"]) if ok else results[0]
        for v in self.vis:
            v.setStep(best["step"])
        return {"chosen_step": best["step"], "threshold_db": threshold_db, "candidates": results}

    def autotune(self) -> tuple[BatchConfig, float]:
        """Time every tile shape, CTA count and skipping choice; keep the fastest."""
        best = BatchConfig()
        ms = C.c_float()
        check(self.lib.isaacb_batch_autotune(self.handle, self._stream(), C.byref(best), C.byref(ms)))
        return best, float(ms.value)
