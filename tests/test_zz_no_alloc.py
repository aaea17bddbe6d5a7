"""The CTF insertion for callers that cannot allocate device memory.

`rexlib_b200_insert_ctf_slices_fixed_scratch` serves callers that must not
call cudaMalloc (a program launching on a queue that must not synchronize the
device, or a caller whose device memory is budgeted up front): it takes no
workspace and uses a fixed array inside the library. These tests call it
through the C-ABI twice in a row, on different inputs, and compare each result
with the allocating entry point's on the same inputs, within the insertion
tolerance of the other GPU tests (relative L2 1e-5; bit for bit in the
deterministic mode). The file is collected last so that a run stopping at its
first failure has run every other test before it.
"""

import ctypes

import numpy as np
import pytest
import torch

from rexlib_b200 import _capi, em
from tests.cases import insertion_inputs, rel_l2

pytestmark = pytest.mark.gpu

OPTICS = em.CtfOptics(300.0, 2.7, 0.1)
PIXEL = 1.2


def _tensors(c):
    to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    V = c["numerator"].shape[0]
    num = to(c["numerator"].reshape(V, 1, *c["numerator"].shape[1:]))
    den = to(c["denominator"].reshape(V, 1, *c["denominator"].shape[1:]))
    return num, den, to(c["slices"]), to(c["transforms"]), to(c["extra"]), to(c["radial"])


WINDOWS = {
    "nearest": em.GriddingWindow.nearest(),
    "linear": em.GriddingWindow.linear(),
    # Half-width 2 is the widest Kaiser-Bessel window on the tile-major path.
    "kb2": em.GriddingWindow.kaiser_bessel(2.0, 9.0),
}


def allocating(c, deterministic, window):
    num, den, sl, tr, ctf, ra = _tensors(c)
    em.insert_ctf_slices(num, den, sl, tr, ctf, ra, window, OPTICS, PIXEL, numerator_out=num,
                         denominator_out=den, deterministic=deterministic)
    torch.cuda.synchronize()
    return num.cpu().numpy(), den.cpu().numpy()


def fixed_scratch(c, deterministic, window):
    num, den, sl, tr, ctf, ra = _tensors(c)
    desc, plan, num_out, den_out, keep = em._prepare_insertion(num, den, sl, tr, ra, window, num, den, deterministic,
                                                               extra_batches=[(ctf.shape[:-1])])
    c_view, c_strides = plan.strides(ctf, 1)
    status = _capi.load().rexlib_b200_insert_ctf_slices_fixed_scratch(
        ctypes.byref(desc), ctypes.c_void_p(c_view.data_ptr()), c_strides, OPTICS._c(), PIXEL,
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _capi.check(status)
    torch.cuda.synchronize()
    return num.cpu().numpy(), den.cpu().numpy()


@pytest.mark.parametrize("window_name", ["nearest", "linear", "kb2"])
@pytest.mark.parametrize("deterministic", [False, True])
def test_fixed_scratch_matches_the_allocating_entry_point_on_two_calls(deterministic, window_name):
    # Two calls in a row with different inputs: the second runs on the
    # scratch the first left behind. The second volume is odd (65^3), so its
    # tiles carry the tabulated volume phase.
    window = WINDOWS[window_name]
    cases = [insertion_inputs(64, 64, 300, kind="ctf", seed=101),
             insertion_inputs(65, 65, 120, volumes=2, kind="ctf", seed=102)]
    fixed = [fixed_scratch(c, deterministic, window) for c in cases]
    for c, (num, den) in zip(cases, fixed):
        want_num, want_den = allocating(c, deterministic, window)
        if deterministic:
            np.testing.assert_array_equal(num, want_num)
            np.testing.assert_array_equal(den, want_den)
        else:
            assert rel_l2(num, want_num) <= 1e-5 and rel_l2(den, want_den) <= 1e-5


def test_fixed_scratch_refuses_calls_beyond_its_size():
    # 100,000 slices of 256^2 need more than the fixed 8 MiB: refused before
    # any work, with both sizes in the message.
    c = insertion_inputs(16, 16, 1, kind="ctf", seed=103)
    num, den, sl, tr, ctf, ra = _tensors(c)
    desc, plan, *_ = em._prepare_insertion(num, den, sl, tr, ra, em.GriddingWindow.linear(), num, den, False)
    desc.slices_per_volume = 100_000
    desc.slice_extent = 256
    desc.volume_extent = 256
    status = _capi.load().rexlib_b200_insert_ctf_slices_fixed_scratch(
        ctypes.byref(desc), ctypes.c_void_p(ctf.data_ptr()), _capi.BatchStrides(0, 1), OPTICS._c(), PIXEL, None)
    assert status == _capi.INVALID_ARGUMENT
    message = _capi.load().rexlib_b200_last_error().decode()
    assert "8388608" in message and "smaller batches" in message
