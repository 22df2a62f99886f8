"""CPU restatement of the reference's sort-last compositing -- TEST INFRASTRUCTURE.

Only ``tests/`` use this module, as the checker of the CUDA blend and of the
compositor's exchange logic; nothing in the package imports it.

* ``distance`` and ``order`` restate lib/isaac.hpp:2019-2047: the sub-volume centre
  in normalised coordinates (w = 1) through the modelview, length in double, as
  float; ranks sorted by distance with ties in rank order (``std::multimap``).
* ``blend`` restates the ordered BLEND composite the reference asks of IceT
  (lib/isaac.hpp:820-826: ICET_COMPOSITE_MODE_BLEND, ICET_ORDERED_COMPOSITE, RGBA
  unsigned bytes).  IceT is a third-party dependency that is not vendored and not
  version-pinned (``Modules/FindIceT.cmake``).  Its published algorithm composites
  premultiplied colours front to back with the "under" operator; in unsigned bytes
  each channel becomes ``acc + src * (255 - acc.alpha) // 255``, kept in 8 bits.
  That rounding, and a plain front-to-back fold rather than IceT's binary-swap
  grouping, are assumptions of this restatement.  No reference test or golden
  vector pins them: parity unpinned.
"""

from __future__ import annotations

import math

import numpy as np


def distance(modelview, position, local_size, global_size, scale=(1.0, 1.0, 1.0)) -> float:
    pos = [int(np.float32(p) * np.float32(s)) for p, s in zip(position, scale)]
    loc = [int(np.float32(v) * np.float32(s)) for v, s in zip(local_size, scale)]
    glo = [int(np.float32(v) * np.float32(s)) for v, s in zip(global_size, scale)]
    half = float(max(glo) // 2)
    point = [(pos[i] + (loc[i] - glo[i]) / 2.0) / half for i in range(3)] + [1.0]
    m = np.asarray(modelview, dtype=np.float64).reshape(4, 4)  # [col][row]
    out = [sum(m[c][r] * point[c] for c in range(4)) for r in range(4)]
    return float(np.float32(math.sqrt(sum(v * v for v in out))))


def order(distances) -> list[int]:
    pairs = sorted((float(np.float32(d)), r) for r, d in enumerate(distances))
    return [r for _, r in pairs]


def blend(images, order_, background=None) -> np.ndarray:
    """``images``: list or array of (..., 4) uint8, image k = rank k; front to back in ``order_``."""
    imgs = [np.asarray(images[r], dtype=np.int64) for r in order_]
    acc = np.zeros_like(imgs[0])
    for src in imgs:
        f = 255 - acc[..., 3:4]
        acc = (acc + src * f // 255) & 0xFF
    if background is not None:
        bg = np.asarray(background, dtype=np.int64)
        f = 255 - acc[..., 3:4]
        acc = (acc + bg * f // 255) & 0xFF
    return acc.astype(np.uint8)
