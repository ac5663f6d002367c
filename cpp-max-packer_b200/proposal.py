"""Learned orientation proposal: host mirror of the spk_proposal_* C ABI.

No counterpart in the reference.  The exhaustive method pages every catalog
orientation at every placement step (spectral.cpp:1460-1591).  The proposal
network ranks the orientations for the current layout, and a step pages only
the k best.  When none of them admits a copy, the exhaustive step decides.

Network input per sample: 2 x 32^3 channels-last floats, shaped
(32, 32, 32, 2) as (z, y, x, c):
- c = 0 is the layout's occupancy fraction pooled over the environment window;
- c = 1 is the oriented item's cells pooled to 32^3.

Architecture:
- four 3^3 convolutions with ReLU: 2->16 at stride 1, 16->32, 32->64 and
  64->64 at stride 2;
- a mean over the final 4^3 voxels;
- a linear layer 64->1.

Arithmetic is BF16 on the tensor cores with FP32 accumulation; the master
parameters and Adam are FP32.
"""

from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional, Tuple

import numpy as np

from . import _lib
from .compute import Context, default_context

P = ctypes.c_void_p
GRID = 32
VOXELS = GRID ** 3
LAYERS = ((2, 16, 1, 32), (16, 32, 2, 32), (32, 64, 2, 16), (64, 64, 2, 8))  # (cin, cout, stride, side in)


class DatasetC(ctypes.Structure):
    _fields_ = [("crops", P), ("crop_count", ctypes.c_uint64), ("items", P), ("item_count", ctypes.c_uint64),
                ("sample_crop", P), ("sample_item", P), ("sample_label", P), ("sample_count", ctypes.c_uint64)]


def _declare(lib):
    if getattr(lib, "_proposal_declared", False):
        return
    lib.spk_proposal_parameter_count.restype = ctypes.c_uint64
    lib.spk_proposal_parameter_count.argtypes = []
    lib.spk_proposal_create.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(P)]
    lib.spk_proposal_destroy.argtypes = [P]
    lib.spk_proposal_destroy.restype = None
    lib.spk_proposal_get_parameters.argtypes = [P, P, P]
    lib.spk_proposal_set_parameters.argtypes = [P, P, P]
    lib.spk_proposal_forward.argtypes = [P, P, ctypes.c_uint64, P, P]
    lib.spk_proposal_gradients.argtypes = [P, P, ctypes.c_uint64, P, P, P, P]
    lib.spk_proposal_train.argtypes = [P, P, ctypes.POINTER(DatasetC), ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_float, ctypes.c_uint64, P]
    lib.spk_session_features.argtypes = [P, P, P]
    lib.spk_session_propose.argtypes = [P, P, ctypes.c_uint32, P, P]
    lib.spk_session_greedy_proposed.argtypes = [P, P, ctypes.c_uint32, ctypes.c_uint64, P, P, P, P, P]
    lib.spk_session_greedy_proposed_margin.argtypes = [P, P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                                       ctypes.c_uint64, P, P, P, P, P, P]
    lib.spk_session_greedy_proposed_adaptive.argtypes = [P, P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, P,
                                                         P, P, P, P, P]
    lib._proposal_declared = True


def parameter_layout():
    """(name, shape) of every parameter block in the flat order."""
    out = []
    for i, (cin, cout, _, _) in enumerate(LAYERS):
        out.append((f"conv{i + 1}.weight", (cout, 27, cin)))
        out.append((f"conv{i + 1}.bias", (cout,)))
    out.append(("head.weight", (64,)))
    out.append(("head.bias", (1,)))
    return out


def split_parameters(flat: np.ndarray) -> dict:
    out, off = {}, 0
    for name, shape in parameter_layout():
        n = int(np.prod(shape))
        out[name] = flat[off:off + n].reshape(shape)
        off += n
    return out


@dataclasses.dataclass
class ProposalDataset:
    """Crops (n, 32, 32, 32), items (m, 32, 32, 32) and samples (crop, item, label)."""

    crops: np.ndarray
    items: np.ndarray
    sample_crop: np.ndarray
    sample_item: np.ndarray
    sample_label: np.ndarray


class Proposal:
    """A proposal network on the device (He-initialised from `seed`)."""

    def __init__(self, seed: int = 0, context: Optional[Context] = None):
        self.lib = _lib.lib()
        _declare(self.lib)
        self.context = context or default_context()
        handle = P()
        _lib.check(self.lib.spk_proposal_create(self.context.handle, seed, ctypes.byref(handle)),
                   "spk_proposal_create")
        self.handle = handle
        self.count = int(self.lib.spk_proposal_parameter_count())

    def close(self):
        if self.handle:
            self.lib.spk_proposal_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_parameters(self) -> np.ndarray:
        out = np.empty(self.count, np.float32)
        _lib.check(self.lib.spk_proposal_get_parameters(self.context.handle, self.handle, out.ctypes.data),
                   "spk_proposal_get_parameters")
        return out

    def set_parameters(self, flat) -> None:
        flat = np.ascontiguousarray(flat, np.float32)
        if flat.size != self.count:
            raise ValueError(f"expected {self.count} parameters, got {flat.size}")
        _lib.check(self.lib.spk_proposal_set_parameters(self.context.handle, self.handle, flat.ctypes.data),
                   "spk_proposal_set_parameters")

    def save(self, path: str) -> None:
        np.savez_compressed(path, parameters=self.get_parameters())

    def load(self, path: str) -> None:
        with np.load(path) as z:
            self.set_parameters(z["parameters"])

    @staticmethod
    def _inputs(inputs) -> np.ndarray:
        x = np.ascontiguousarray(inputs, np.float32)
        if x.ndim != 5 or x.shape[1:] != (GRID, GRID, GRID, 2):
            raise ValueError("inputs must be (batch, 32, 32, 32, 2)")
        return x

    def forward(self, inputs) -> np.ndarray:
        x = self._inputs(inputs)
        out = np.empty(x.shape[0], np.float32)
        _lib.check(self.lib.spk_proposal_forward(self.context.handle, self.handle, x.shape[0], x.ctypes.data,
                                                 out.ctypes.data), "spk_proposal_forward")
        return out

    def gradients(self, inputs, labels) -> Tuple[float, np.ndarray]:
        x = self._inputs(inputs)
        y = np.ascontiguousarray(labels, np.float32)
        loss = np.zeros(1, np.float32)
        grads = np.empty(self.count, np.float32)
        _lib.check(self.lib.spk_proposal_gradients(self.context.handle, self.handle, x.shape[0], x.ctypes.data,
                                                   y.ctypes.data, loss.ctypes.data, grads.ctypes.data),
                   "spk_proposal_gradients")
        return float(loss[0]), grads

    def train(self, data: ProposalDataset, batch: int, steps: int, learning_rate: float,
              seed: int = 0) -> np.ndarray:
        crops = np.ascontiguousarray(data.crops, np.float32)
        items = np.ascontiguousarray(data.items, np.float32)
        sc = np.ascontiguousarray(data.sample_crop, np.uint32)
        si = np.ascontiguousarray(data.sample_item, np.uint32)
        sl = np.ascontiguousarray(data.sample_label, np.float32)
        d = DatasetC(crops.ctypes.data, len(crops), items.ctypes.data, len(items), sc.ctypes.data, si.ctypes.data,
                     sl.ctypes.data, len(sl))
        losses = np.zeros(steps, np.float32)
        _lib.check(self.lib.spk_proposal_train(self.context.handle, self.handle, ctypes.byref(d), batch, steps,
                                               learning_rate, seed, losses.ctypes.data), "spk_proposal_train")
        return losses


def session_features(session) -> Tuple[np.ndarray, np.ndarray]:
    """(crop (32,32,32), items (orientations, 32,32,32)) of an open Session."""
    lib = _lib.lib()
    _declare(lib)
    O = len(session.catalog)
    crop = np.empty((GRID, GRID, GRID), np.float32)
    items = np.empty((O, GRID, GRID, GRID), np.float32)
    _lib.check(lib.spk_session_features(session.context.handle, crop.ctypes.data, items.ctypes.data),
               "spk_session_features")
    return crop, items


def session_crop(session) -> np.ndarray:
    lib = _lib.lib()
    _declare(lib)
    crop = np.empty((GRID, GRID, GRID), np.float32)
    _lib.check(lib.spk_session_features(session.context.handle, crop.ctypes.data, None), "spk_session_features")
    return crop


def propose(session, net: Proposal, k: int) -> Tuple[np.ndarray, np.ndarray]:
    """(the k best orientations, every orientation's prediction)."""
    lib = _lib.lib()
    _declare(lib)
    O = len(session.catalog)
    best = np.zeros(max(k, 1), np.uint64)
    pred = np.zeros(O, np.float32)
    _lib.check(lib.spk_session_propose(session.context.handle, net.handle, k, best.ctypes.data, pred.ctypes.data),
               "spk_session_propose")
    return best[:k], pred


def greedy_proposed(session, net: Proposal, k: int, max_steps: int):
    """Greedy fill paging the k proposed orientations per step; returns
    (placements, fallback steps)."""
    from .session import Placement

    lib = _lib.lib()
    _declare(lib)
    n = max(max_steps, 1)
    ori = np.zeros(n, np.uint64)
    t = np.zeros((n, 3), np.int64)
    scores = np.zeros(n, np.float64)
    placed = ctypes.c_uint64()
    fallbacks = ctypes.c_uint64()
    _lib.check(lib.spk_session_greedy_proposed(session.context.handle, net.handle, k, max_steps,
                                               ctypes.byref(placed), ori.ctypes.data, t.ctypes.data,
                                               scores.ctypes.data, ctypes.byref(fallbacks)),
               "spk_session_greedy_proposed")
    out = [Placement(int(ori[i]), tuple(int(v) for v in t[i]), float(scores[i])) for i in range(placed.value)]
    session.placements += out
    return out, int(fallbacks.value)


def greedy_proposed_margin(session, net: Proposal, k_min: int, k_max: int, margin: float, max_steps: int):
    """The proposed greedy paging the k_min best orientations and those
    predicted within `margin` of the k_min-th (at most k_max); returns
    (placements, fallback steps, orientations paged in all)."""
    from .session import Placement

    lib = _lib.lib()
    _declare(lib)
    n = max(max_steps, 1)
    ori = np.zeros(n, np.uint64)
    t = np.zeros((n, 3), np.int64)
    scores = np.zeros(n, np.float64)
    placed, fallbacks, paged = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    _lib.check(lib.spk_session_greedy_proposed_margin(session.context.handle, net.handle, k_min, k_max,
                                                      ctypes.c_float(margin), max_steps, ctypes.byref(placed),
                                                      ori.ctypes.data, t.ctypes.data, scores.ctypes.data,
                                                      ctypes.byref(fallbacks), ctypes.byref(paged)),
               "spk_session_greedy_proposed_margin")
    out = [Placement(int(ori[i]), tuple(int(v) for v in t[i]), float(scores[i])) for i in range(placed.value)]
    session.placements += out
    return out, int(fallbacks.value), int(paged.value)


def greedy_proposed_adaptive(session, net: Proposal, k: int, min_feasible: int, max_steps: int):
    """The proposed greedy that widens by k orientations at a time while
    fewer than `min_feasible` paged orientations admit a copy; returns
    (placements, fallback steps, widenings)."""
    from .session import Placement

    lib = _lib.lib()
    _declare(lib)
    n = max(max_steps, 1)
    ori = np.zeros(n, np.uint64)
    t = np.zeros((n, 3), np.int64)
    scores = np.zeros(n, np.float64)
    placed, fallbacks, widenings = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    _lib.check(lib.spk_session_greedy_proposed_adaptive(session.context.handle, net.handle, k, min_feasible,
                                                        max_steps, ctypes.byref(placed), ori.ctypes.data,
                                                        t.ctypes.data, scores.ctypes.data, ctypes.byref(fallbacks),
                                                        ctypes.byref(widenings)),
               "spk_session_greedy_proposed_adaptive")
    out = [Placement(int(ori[i]), tuple(int(v) for v in t[i]), float(scores[i])) for i in range(placed.value)]
    session.placements += out
    return out, int(fallbacks.value), int(widenings.value)
