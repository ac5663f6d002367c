"""ORACLE - test infrastructure only.  The translation masks that the solver's
gap-fill and slab-lattice code read off a full-range binary correlation,
restated in numpy as the checker of spk_correlate_binary_mask.  The product
never imports it.

Reference rules (engine/pack_solver/src):
- gap_fill.cpp:404-420, free translations.  The mask covers the legal box,
  whose first translation is window.first - kernel.first.  A cell is free when
  its translation lies in the correlation range and the rounded count there
  is 0.
- gap_fill.cpp:443-446, blocked offsets.  Over the whole range, a cell is
  blocked when its rounded count is non-zero.
- slab_lattice.cpp:688-691, the no-fit map: the same rule as the blocked
  offsets.

Parity is pinned on the host by tests/test_oracle_masks.py against direct
overlap sums at every translation, which involve no FFT.
"""

from __future__ import annotations

import numpy as np


def translation_mask(translation_first, shape, values, box_first, box_shape, want_zero):
    """u8 mask over the box (X fastest), from full-range values laid out X
    fastest over `shape` starting at `translation_first`."""
    tf = np.asarray(translation_first, np.int64)
    sh = np.asarray(shape, np.int64)
    bf = np.asarray(box_first, np.int64)
    bs = [int(v) for v in box_shape]
    counts = np.round(np.asarray(values, np.float64)).reshape(int(sh[2]), int(sh[1]), int(sh[0]))
    mask = np.zeros((bs[2], bs[1], bs[0]), np.uint8)
    if min(bs) == 0:
        return mask.reshape(-1)
    # Offsets of the box's cells within the range, per axis.
    off = [bf[a] - tf[a] + np.arange(bs[a], dtype=np.int64) for a in range(3)]
    inside = [(o >= 0) & (o < sh[a]) for a, o in enumerate(off)]
    zi, yi, xi = (np.nonzero(inside[2])[0], np.nonzero(inside[1])[0], np.nonzero(inside[0])[0])
    if len(zi) and len(yi) and len(xi):
        sub = counts[np.ix_(off[2][zi], off[1][yi], off[0][xi])]
        hit = (sub == 0) if want_zero else (sub != 0)
        mask[np.ix_(zi, yi, xi)] = hit.astype(np.uint8)
    return mask.reshape(-1)


def direct_counts(env_shape, ker_shape, env_first, ker_first, env, ker):
    """Overlap count at every translation of the full range by direct sums
    (small cases only): count(t) = sum_i env[i + t - (env_first - ker_first)] ker[i]."""
    es = [int(v) for v in env_shape]
    ks = [int(v) for v in ker_shape]
    e = np.asarray(env, np.int64).reshape(es[2], es[1], es[0])
    k = np.asarray(ker, np.int64).reshape(ks[2], ks[1], ks[0])
    tf = [int(env_first[a]) - int(ker_first[a]) - (ks[a] - 1) for a in range(3)]
    shape = [es[a] + ks[a] - 1 for a in range(3)]
    out = np.zeros((shape[2], shape[1], shape[0]), np.int64)
    # Translation index u along an axis places kernel cell i on environment
    # cell i + u - (K - 1).
    padded = np.zeros((es[2] + 2 * (ks[2] - 1), es[1] + 2 * (ks[1] - 1), es[0] + 2 * (ks[0] - 1)), np.int64)
    padded[ks[2] - 1:ks[2] - 1 + es[2], ks[1] - 1:ks[1] - 1 + es[1], ks[0] - 1:ks[0] - 1 + es[0]] = e
    for uz in range(shape[2]):
        for uy in range(shape[1]):
            for ux in range(shape[0]):
                out[uz, uy, ux] = int((padded[uz:uz + ks[2], uy:uy + ks[1], ux:ux + ks[0]] * k).sum())
    return tf, shape, out.reshape(-1)
