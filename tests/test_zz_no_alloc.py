"""The allocation-free proximity entry point against the regular one.

spk_build_proximity_static serves callers that cannot allocate device memory
(their device memory belongs to another allocator, or their steady-state
loop must not allocate): it takes caller-owned device buffers and keeps its
scratch in one static device array.  This file is collected last so that a
failure here comes after every other test has run; it must pass both alone in
a fresh process and after the rest of the suite.
"""

import ctypes

import numpy as np
import pytest

from conftest import package

pytestmark = pytest.mark.gpu


def _static_call(shape, occupied):
    import torch

    lib = package("_lib").lib()
    occ = torch.from_numpy(np.ascontiguousarray(occupied, np.uint8)).cuda()
    out = torch.full((occ.numel(),), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    s = np.array(shape, np.uint32)
    status = lib.spk_build_proximity_static(ctypes.c_void_p(stream or None), s.ctypes.data_as(ctypes.c_void_p),
                                            ctypes.c_void_p(occ.data_ptr()), ctypes.c_void_p(out.data_ptr()))
    torch.cuda.synchronize()
    return status, out.cpu().numpy()


def test_static_entry_point_matches_regular_on_two_calls(gpu_ctx):
    compute = package("compute")
    rng = np.random.default_rng(9)
    # Two calls in a row on different shapes and densities: the second must
    # not see anything the first left in the shared scratch.
    for shape, density in [((64, 48, 40), 0.01), ((17, 33, 29), 0.2)]:
        occ = (rng.random(int(np.prod(shape))) < density).astype(np.uint8)
        status, got = _static_call(shape, occ)
        assert status == 0, package("_lib").status_code(status)
        want = compute.build_proximity(shape, occ, context=gpu_ctx)
        # The regular path is bit-exact with the reference; so must this be.
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def test_static_entry_point_rejects_fields_beyond_its_scratch():
    status, _ = _static_call((65, 4, 4), np.zeros(65 * 16, np.uint8))
    assert package("_lib").status_code(status) == "SPK_SCRATCH_LIMIT"
