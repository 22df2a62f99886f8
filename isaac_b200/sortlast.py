"""Sort-last compositing across ranks: the part of ``IsaacVisualization`` that IceT
does over MPI in the reference (lib/isaac.hpp:799-830, 2015-2055), done here with
NCCL (``torch.distributed``) for the exchange and a CUDA kernel for the blend.

Each rank renders its own sub-volume (``position`` and ``local_size`` inside
``global_size``) into a full-size RGBA8 frame.  Per frame:

1. Every rank computes the distance from the camera to its sub-volume's centre
   (``rank_distance``, the reference's formula); the distances are all-gathered
   and sorted into a front-to-back order (``composite_order``; ties keep rank
   order, as the reference's ``std::multimap`` does).
2. The frame is cut into ``world`` row stripes.  One ``all_to_all_single`` sends
   stripe k of every rank to rank k.
3. Rank k blends its stripe of all ranks front to back (``isaacb_blend_ordered``:
   premultiplied "under" in 8-bit integers, IceT's BLEND composite).
4. One ``all_gather_into_tensor`` assembles the full frame on every rank.

Only step 3 computes; steps 2 and 4 move one frame's bytes per rank each, which is
IceT's "direct send" with a reduce-to-all.  The blend is a parameter so that the
exchange and ordering logic can be exercised with ``gloo`` on the CPU; on the GPU the
default is the CUDA kernel, and there is no host fallback.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check


def rank_distance(modelview, position, local_size, global_size, scale=(1.0, 1.0, 1.0)) -> float:
    """Distance from the camera to the centre of this rank's sub-volume
    (lib/isaac.hpp:2019-2028): the scaled box in normalised coordinates, w = 1,
    through the modelview (column-major [col][row]), length of all four
    components in double, returned as float32."""
    f32 = np.float32
    pos_s = [int(f32(p) * f32(s)) for p, s in zip(position, scale)]  # isaac_int3(float3 * scale)
    loc_s = [int(f32(l) * f32(s)) for l, s in zip(local_size, scale)]  # isaac_size3(float3 * scale)
    glo_s = [int(f32(g) * f32(s)) for g, s in zip(global_size, scale)]
    half_max = float(max(glo_s) // 2)  # integer division before the conversion, as in the reference
    p = np.array([(pos_s[i] + (loc_s[i] - glo_s[i]) / 2.0) / half_max for i in range(3)] + [1.0])
    m = np.asarray(modelview, dtype=np.float64).reshape(4, 4)  # [col][row]
    v = m.T @ p
    return float(np.float32(math.sqrt(float(v @ v))))


def composite_order(distances) -> list[int]:
    """Ranks front to back: ascending distance, ties in rank order."""
    d = [float(np.float32(x)) for x in distances]
    return sorted(range(len(d)), key=lambda r: (d[r], r))


def blend_cuda(stripes, order, background=None, out=None):
    """Blend ``stripes`` ((K, P, 4) uint8 CUDA tensor, image k = rank k) front to back in
    ``order`` with ``isaacb_blend_ordered``; returns a (P, 4) uint8 CUDA tensor."""
    import torch

    k, pixels = int(stripes.shape[0]), int(stripes.shape[1])
    if out is None:
        out = torch.empty((pixels, 4), dtype=torch.uint8, device=stripes.device)
    stride = pixels * 4
    base = stripes.data_ptr()
    ptrs = (C.c_void_p * k)(*[base + i * stride for i in range(k)])
    ordr = (C.c_int32 * k)(*[int(r) for r in order])
    bg = (C.c_uint8 * 4)(*background) if background is not None else None
    check(_lib.load().isaacb_blend_ordered(ptrs, k, ordr, pixels, bg, C.c_void_p(out.data_ptr()),
                                           C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return out


class SortLastCompositor:
    """Sort-last compositing of one frame per rank over a ``torch.distributed`` group."""

    def __init__(self, group=None, background=None, blend=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.background = background
        self.blend = blend if blend is not None else blend_cuda
        self.lastOrder: list[int] | None = None

    def order(self, distance: float) -> list[int]:
        """All-gather the ranks' distances and sort them front to back."""
        import torch

        dev = "cuda" if self.dist.get_backend(self.group) == "nccl" else "cpu"
        mine = torch.tensor([distance], dtype=torch.float32, device=dev)
        every = torch.empty(self.world, dtype=torch.float32, device=dev)
        self.dist.all_gather_into_tensor(every, mine, group=self.group)
        self.lastOrder = composite_order(every.cpu().tolist())
        return self.lastOrder

    def composite(self, frame, distance: float):
        """The composited (H, W, 4) uint8 frame on every rank, from this rank's
        (H, W, 4) uint8 frame (premultiplied RGBA, as the renderer writes it)."""
        import torch

        order = self.order(distance)
        h, w, _ = frame.shape
        n = self.world
        rows = -(-h // n)
        if rows * n != h:
            padded = torch.zeros((rows * n, w, 4), dtype=torch.uint8, device=frame.device)
            padded[:h] = frame
        else:
            padded = frame.contiguous()
        send = padded.reshape(n, rows * w * 4)
        recv = torch.empty_like(send)
        self.dist.all_to_all_single(recv, send, group=self.group)
        mine = self.blend(recv.reshape(n, rows * w, 4), order, self.background)
        full = torch.empty((n * rows * w, 4), dtype=torch.uint8, device=frame.device)
        self.dist.all_gather_into_tensor(full, mine.reshape(-1, 4).contiguous(), group=self.group)
        return full.reshape(n * rows, w, 4)[:h]
