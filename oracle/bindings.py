"""ORACLE bindings (test infrastructure only).

``C`` wraps liboracle.so (the plain-C restatement in spk_oracle.c);
``Ref`` wraps oracle/_ref/libspk_ref.so (the reference's own C++ compiled
here with project-written FFT and accepted-solid shims).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use them.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libspk_ref.so")
# The reference checkout, when present, is found by oracle/ref/Makefile
# (SPK_REFERENCE_ROOT, or the recipe's default); without it the prebuilt
# oracle/_ref library is used as it is.

_c = ctypes
_P = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_P)


def build_oracle() -> str:
    """Compiles spk_oracle.c (gcc) when the library is missing or stale."""
    src = os.path.join(HERE, "spk_oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_SO


def build_reference(reference_root: str | None = None) -> str | None:
    """Compiles the reference's hot-path sources in place (oracle/ref/Makefile;
    a no-op where the sources are absent)."""
    extra = [f"REF={reference_root}"] if reference_root else []
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(HERE, "ref"), *extra], check=True)
    return REF_SO if os.path.exists(REF_SO) else None


class C:
    """The plain-C restatement."""

    def __init__(self):
        self.lib = ctypes.CDLL(build_oracle() if not os.path.exists(ORACLE_SO) else ORACLE_SO)
        self.lib.oracle_fsum.restype = ctypes.c_double

    def fsum(self, values) -> float:
        v = np.ascontiguousarray(values, dtype=np.float64)
        return self.lib.oracle_fsum(_ptr(v), ctypes.c_int64(v.size))

    def correlate_int(self, blocked, kernel, origin):
        b = np.ascontiguousarray(blocked, dtype=np.int64)
        k = np.ascontiguousarray(kernel, dtype=np.int64)
        bs = np.array(b.shape[::-1], dtype=np.int64)  # arrays are [z][y][x]
        ks = np.array(k.shape[::-1], dtype=np.int64)
        o = np.array(origin, dtype=np.int64)
        first = np.zeros(3, np.int64)
        oshape = bs + ks - 1
        out = np.zeros(int(np.prod(oshape)), np.int64)
        rc = self.lib.oracle_correlate_int(_ptr(b), _ptr(bs), _ptr(k), _ptr(ks), _ptr(o), _ptr(out), _ptr(first),
                                           _ptr(np.zeros(3, np.int64)))
        if rc:
            raise OverflowError("integer correlation overflowed")
        return first, oshape, out

    def correlate(self, proximity, env_shape, ker_shape, env_first, ker_first, env, ker):
        es = np.array(env_shape, np.uint32)
        ks = np.array(ker_shape, np.uint32)
        ef = np.array(env_first, np.int64)
        kf = np.array(ker_first, np.int64)
        e = np.ascontiguousarray(env, dtype=np.float64 if proximity else np.uint8)
        k = np.ascontiguousarray(ker, dtype=np.uint8)
        oshape = es.astype(np.int64) + ks - 1
        out = np.zeros(int(np.prod(oshape)), np.float64)
        tf = np.zeros(3, np.int64)
        os_ = np.zeros(3, np.uint32)
        fn = self.lib.oracle_correlate_proximity if proximity else self.lib.oracle_correlate_binary
        fn(_ptr(es), _ptr(ks), _ptr(ef), _ptr(kf), _ptr(e), _ptr(k), _ptr(out), _ptr(tf), _ptr(os_))
        return tf, os_, out

    def broad_phase(self, lo, hi, finite, proven, clearance, capacity=None):
        """oracle_broad_phase: the uncertified pairs, (count, 2) uint32, in visiting order."""
        lo = np.ascontiguousarray(lo, np.float64).reshape(-1, 3)
        hi = np.ascontiguousarray(hi, np.float64).reshape(-1, 3)
        n = lo.shape[0]
        fin = np.ascontiguousarray(finite, np.uint8)
        prv = None if proven is None else np.ascontiguousarray(proven, np.uint8)
        cap = n * (n - 1) // 2 if capacity is None else capacity
        out = np.zeros((max(cap, 1), 2), np.uint32)
        self.lib.oracle_broad_phase.restype = ctypes.c_int64
        count = self.lib.oracle_broad_phase(_ptr(lo), _ptr(hi), _ptr(fin), None if prv is None else _ptr(prv),
                                            ctypes.c_int64(n), ctypes.c_double(clearance), _ptr(out),
                                            ctypes.c_int64(cap))
        return out[:min(count, cap)].copy(), int(count)

    def build_proximity(self, shape, occupied):
        s = np.array(shape, np.uint32)
        occ = np.ascontiguousarray(occupied, dtype=np.uint8)
        values = np.zeros(occ.size, np.float64)
        d2 = np.zeros(occ.size, np.int64)
        self.lib.oracle_build_proximity(_ptr(s), _ptr(occ), _ptr(values), _ptr(d2))
        return values, d2


class PageEntry(ctypes.Structure):
    _fields_ = [("t", ctypes.c_int64 * 3), ("score", ctypes.c_double), ("orientation", ctypes.c_uint64),
                ("binary_overlap", ctypes.c_double), ("direct_zero", ctypes.c_int32)]


class Ref:
    """The reference's own C++ (requires oracle/_ref/libspk_ref.so)."""

    def __init__(self):
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        lib = self.lib = ctypes.CDLL(REF_SO)
        lib.spkref_asset_from_stl.restype = _P
        lib.spkref_session_new.restype = _P
        self.err = ctypes.create_string_buffer(256)

    def _error(self):
        return self.err.value.decode()

    def correlate(self, proximity, env_shape, ker_shape, env_first, ker_first, env, ker):
        es = np.array(env_shape, np.uint32)
        ks = np.array(ker_shape, np.uint32)
        ef = np.array(env_first, np.int64)
        kf = np.array(ker_first, np.int64)
        e = np.ascontiguousarray(env, dtype=np.float64 if proximity else np.uint8)
        k = np.ascontiguousarray(ker, dtype=np.uint8)
        n = int(np.prod(es.astype(np.int64) + ks - 1))
        out = np.zeros(n, np.float64)
        tf = np.zeros(3, np.int64)
        os_ = np.zeros(3, np.uint32)
        report = np.zeros(3, np.float64)
        rc = self.lib.spkref_correlate(int(proximity), _ptr(es), _ptr(ks), _ptr(ef), _ptr(kf), _ptr(e), _ptr(k),
                                       _ptr(out), ctypes.c_uint64(n), _ptr(tf), _ptr(os_), _ptr(report), self.err, 256)
        if rc:
            return self._error()
        return tf, os_, out, report

    def build_proximity(self, shape, occupied):
        s = np.array(shape, np.uint32)
        occ = np.ascontiguousarray(occupied, dtype=np.uint8)
        values = np.zeros(occ.size, np.float64)
        if self.lib.spkref_build_proximity(_ptr(s), _ptr(occ), _ptr(values)):
            return None
        return values

    # --- assets and fields -------------------------------------------------
    def asset(self, stl: bytes, container: bool = False):
        handle = self.lib.spkref_asset_from_stl(stl, ctypes.c_uint64(len(stl)), int(container), self.err, 256)
        if not handle:
            raise RuntimeError(self._error())
        return RefAsset(self, handle)

    def catalog(self, mode: int, quaternions=None):
        q = np.ascontiguousarray(quaternions if quaternions is not None else np.zeros((0, 4)), np.float64)
        cap = max(len(q), 24) + 8
        out = np.zeros((cap, 4), np.float64)
        count = ctypes.c_uint64()
        rc = self.lib.spkref_catalog(mode, _ptr(q), ctypes.c_uint64(len(q)), _ptr(out), ctypes.c_uint64(cap),
                                     ctypes.byref(count))
        if rc:
            raise RuntimeError("catalog failed")
        return out[: count.value].copy()

    def session(self, obj, container, pair_clearance, wall_clearance, origin, pitch, catalog):
        box = isinstance(container, (tuple, list, np.ndarray))
        dims = np.array(container if box else (0, 0, 0), np.float64)
        o = np.array(origin, np.float64)
        q = np.ascontiguousarray(catalog, np.float64)
        handle = self.lib.spkref_session_new(
            _P(obj.handle), int(box), _ptr(dims), None if box else _P(container.handle), ctypes.c_double(pair_clearance),
            ctypes.c_double(wall_clearance), _ptr(o), ctypes.c_double(pitch), _ptr(q), ctypes.c_uint64(len(q)),
            self.err, 256)
        if not handle:
            raise RuntimeError(self._error())
        return RefSession(self, handle, len(q))


class RefAsset:
    def __init__(self, ref: Ref, handle):
        self.ref, self.handle = ref, handle

    def __del__(self):
        try:
            self.ref.lib.spkref_asset_free(_P(self.handle))
        except Exception:
            pass

    def mesh(self):
        lib = self.ref.lib
        counts = np.zeros(2, np.uint64)
        bounds = np.zeros(6, np.float64)
        lib.spkref_asset_mesh(_P(self.handle), None, ctypes.c_uint64(0), None, ctypes.c_uint64(0), _ptr(counts),
                              _ptr(bounds))
        v = np.zeros((int(counts[0]), 3), np.float64)
        t = np.zeros((int(counts[1]), 3), np.uint32)
        lib.spkref_asset_mesh(_P(self.handle), _ptr(v), ctypes.c_uint64(len(v)), _ptr(t), ctypes.c_uint64(len(t)),
                              _ptr(counts), _ptr(bounds))
        return v, t, bounds

    def voxelize_object(self, origin, pitch, q, capacity=1 << 26):
        first = np.zeros(3, np.int64)
        shape = np.zeros(3, np.uint32)
        cells = np.zeros(capacity, np.uint8)
        rc = self.ref.lib.spkref_voxelize_object(_P(self.handle), _ptr(np.array(origin, np.float64)),
                                                 ctypes.c_double(pitch), _ptr(np.array(q, np.float64)), _ptr(first),
                                                 _ptr(shape), _ptr(cells), ctypes.c_uint64(capacity), self.ref.err, 256)
        if rc:
            raise RuntimeError(self.ref._error())
        return first, shape, cells[: int(np.prod(shape.astype(np.int64)))].copy()

    def voxelize_placed(self, origin, pitch, first, shape, translation, q, clearance):
        cells = np.zeros(int(np.prod(np.array(shape, np.int64))), np.uint8)
        rc = self.ref.lib.spkref_voxelize_placed(
            _P(self.handle), _ptr(np.array(origin, np.float64)), ctypes.c_double(pitch), _ptr(np.array(first, np.int64)),
            _ptr(np.array(shape, np.uint32)), _ptr(np.array(translation, np.float64)), _ptr(np.array(q, np.float64)),
            ctypes.c_double(clearance), _ptr(cells), self.ref.err, 256)
        if rc:
            raise RuntimeError(self.ref._error())
        return cells

    def export_stl(self, translations, quaternions) -> bytes:
        """The reference's STL records of the posed copies (spkref_export_stl)."""
        t = np.ascontiguousarray(translations, np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(quaternions, np.float64).reshape(-1, 4)
        size = ctypes.c_uint64()
        self.ref.lib.spkref_export_stl(_P(self.handle), _ptr(t), _ptr(q), ctypes.c_uint64(len(t)), None,
                                       ctypes.c_uint64(0), ctypes.byref(size))
        out = np.zeros(size.value, np.uint8)
        rc = self.ref.lib.spkref_export_stl(_P(self.handle), _ptr(t), _ptr(q), ctypes.c_uint64(len(t)), _ptr(out),
                                            ctypes.c_uint64(size.value), ctypes.byref(size))
        if rc:
            raise RuntimeError(f"spkref_export_stl failed ({rc})")
        return out.tobytes()

    def bounds_pair(self, t1, q1, t2, q2, clearance):
        """validation_kernel::bounds_pair_certificate: 0 none, 1 outward-aabb, 2 other, 3 indeterminate."""
        return self.ref.lib.spkref_bounds_pair(_P(self.handle), _ptr(np.array(t1, np.float64)),
                                               _ptr(np.array(q1, np.float64)), _ptr(np.array(t2, np.float64)),
                                               _ptr(np.array(q2, np.float64)), ctypes.c_double(clearance))

    def oriented_bounds(self, q):
        out = np.zeros(6, np.float64)
        if self.ref.lib.spkref_oriented_bounds(_P(self.handle), _ptr(np.array(q, np.float64)), _ptr(out)):
            raise RuntimeError("oriented_bounds failed")
        return out


def ref_voxelize_container(ref: Ref, container, origin, pitch, first, shape, clearance):
    box = isinstance(container, (tuple, list, np.ndarray))
    cells = np.zeros(int(np.prod(np.array(shape, np.int64))), np.uint8)
    rc = ref.lib.spkref_voxelize_container(
        int(box), _ptr(np.array(container if box else (0, 0, 0), np.float64)), None if box else _P(container.handle),
        _ptr(np.array(origin, np.float64)), ctypes.c_double(pitch), _ptr(np.array(first, np.int64)),
        _ptr(np.array(shape, np.uint32)), ctypes.c_double(clearance), _ptr(cells), ref.err, 256)
    if rc:
        raise RuntimeError(ref._error())
    return cells


class RefSession:
    def __init__(self, ref: Ref, handle, orientations):
        self.ref, self.handle, self.orientations = ref, handle, orientations

    def __del__(self):
        try:
            self.ref.lib.spkref_session_free(_P(self.handle))
        except Exception:
            pass

    def page(self, orientation, cursor=None, low_overlap=False, keep_values=False):
        page = (PageEntry * 32)()
        count = ctypes.c_uint64()
        cur = PageEntry()
        if cursor is not None:
            cur = cursor
        rc = self.ref.lib.spkref_session_page(_P(self.handle), ctypes.c_uint64(orientation), int(cursor is not None),
                                              ctypes.byref(cur), int(low_overlap), page, ctypes.byref(count),
                                              int(keep_values), self.ref.err, 256)
        if rc:
            raise RuntimeError(self.ref._error())
        return [page[i] for i in range(count.value)]

    def observed(self, kind):
        meta = np.zeros(19, np.int64)
        self.ref.lib.spkref_session_observed(_P(self.handle), kind, None, ctypes.c_uint64(0), _ptr(meta))
        nbytes = int(meta[18])
        buf = np.zeros(nbytes, np.uint8)
        if self.ref.lib.spkref_session_observed(_P(self.handle), kind, _ptr(buf), ctypes.c_uint64(nbytes), _ptr(meta)):
            raise RuntimeError("no observation")
        dtype = np.uint8 if kind in (0, 2) else np.float64
        return buf.view(dtype), meta[:18].reshape(6, 3)

    def place(self, orientation, t):
        return self.ref.lib.spkref_session_place(_P(self.handle), ctypes.c_uint64(orientation),
                                                 _ptr(np.array(t, np.int64))) == 0

    def greedy(self, max_steps):
        ori = np.zeros(max_steps, np.uint64)
        t = np.zeros((max_steps, 3), np.int64)
        scores = np.zeros(max_steps, np.float64)
        placed = ctypes.c_uint64()
        rejected = ctypes.c_uint64()
        seconds = ctypes.c_double()
        rc = self.ref.lib.spkref_session_greedy(_P(self.handle), ctypes.c_uint64(max_steps), _ptr(ori), _ptr(t),
                                                _ptr(scores), ctypes.byref(placed), ctypes.byref(rejected),
                                                ctypes.byref(seconds), self.ref.err, 256)
        if rc:
            raise RuntimeError(self.ref._error())
        n = placed.value
        return ori[:n], t[:n], scores[:n], rejected.value, seconds.value


class OracleCandidate(ctypes.Structure):
    _fields_ = [("t", ctypes.c_int64 * 3), ("score", ctypes.c_double), ("direct_zero", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("orientation", ctypes.c_uint64), ("binary_overlap", ctypes.c_double)]


def oracle_page(c: C, env_first, env_shape, occupancy, proximity, kernel_first, kernel_shape, kernel, lattice,
                max_z, cmin_z, height, orientation=0, cursor=None):
    """The restated page (oracle_page in spk_oracle.c); cursor is (t, score, orientation) or None."""
    ef = np.array(env_first, np.int64)
    es = np.array(env_shape, np.uint32)
    kf = np.array(kernel_first, np.int64)
    ks = np.array(kernel_shape, np.uint32)
    occ = np.ascontiguousarray(occupancy, np.uint8).reshape(-1)
    prox = np.ascontiguousarray(proximity, np.float64).reshape(-1)
    ker = np.ascontiguousarray(kernel, np.uint8).reshape(-1)
    lat = np.array(lattice, np.float64)
    page = (OracleCandidate * 32)()
    cur = None
    if cursor is not None:
        cur = OracleCandidate()
        for a in range(3):
            cur.t[a] = int(cursor[0][a])
        cur.score = cursor[1]
        cur.orientation = cursor[2]
    n = c.lib.oracle_page(_ptr(ef), _ptr(es), _ptr(occ), _ptr(prox), _ptr(kf), _ptr(ks), _ptr(ker), _ptr(lat),
                          ctypes.c_double(max_z), ctypes.c_double(cmin_z), ctypes.c_double(height),
                          ctypes.c_uint64(orientation), ctypes.byref(cur) if cur is not None else None, page)
    if n < 0:
        raise ValueError("empty kernel")
    return [(tuple(page[i].t), page[i].score, page[i].orientation) for i in range(n)]
