"""Host logic of the Python mirror on the CPU: the batch plan of the
insertions (kept and reduced axes, per-operand strides in cores, after
slice_insertion_layout_plan.cpp:81-185), the parameter checks of the window
and the optics, the bounds and the mode switch. None of it launches a
kernel."""

import math

import pytest
import torch

from rexlib_b200 import _capi, em


def test_plan_keeps_the_accumulator_axes_and_reduces_the_others():
    # Accumulators (V=3, 1) keep axis 0; the slices (3, 5) sum over axis 1.
    plan = em._BatchPlan((3, 1), [(3, 5), (3, 5), (5,)])
    assert plan.shape == (3, 5)
    assert plan.kept == [0] and plan.reduced == [1]
    assert (plan.volumes, plan.particles) == (3, 5)


def test_plan_refuses_batches_that_do_not_broadcast():
    with pytest.raises(ValueError, match="do not broadcast"):
        em._BatchPlan((3, 1), [(4, 5)])


def test_strides_in_cores_for_contiguous_and_broadcast_operands():
    plan = em._BatchPlan((3, 1), [(3, 5), (5,)])
    # One slice per (volume, particle): contiguous cores, strides (P, 1).
    slices = torch.zeros(3, 5, 8, 5, dtype=torch.complex64)
    flat, st = plan.strides(slices, 2)
    assert tuple(flat.shape) == (3, 5, 8, 5)
    assert (st.volume, st.particle) == (5, 1)
    # Radial weights shared by every volume: the volume stride is 0.
    radial = torch.ones(5, 5)
    flat, st = plan.strides(radial, 1)
    assert (st.volume, st.particle) == (0, 1)
    # One set for everything: both strides 0.
    one = torch.ones(5)
    flat, st = plan.strides(one, 1)
    assert (st.volume, st.particle) == (0, 0)


def test_operands_the_kernels_cannot_stride_are_copied():
    plan = em._BatchPlan((2, 1), [(2, 3)])
    base = torch.arange(2 * 3 * 4 * 8, dtype=torch.float32).reshape(2, 3, 4, 8)
    # Cores (3, 8) whose batch stride (32 elements) is not a whole number of
    # cores (24): copied to contiguous cores, strides (P, 1).
    view = base[..., :3, :]
    flat, st = plan.strides(view, 2)
    assert flat[0, 0].is_contiguous() and (st.volume, st.particle) == (3, 1)
    assert torch.equal(flat, view)
    # Cores with a column stride of 2: not contiguous, so copied.
    strided = base[..., ::2]
    flat, st = plan.strides(strided, 2)
    assert flat[0, 0].is_contiguous() and torch.equal(flat, strided)


def test_window_and_optics_checks():
    with pytest.raises(ValueError, match="half-width"):
        em.GriddingWindow.kaiser_bessel(0.0, 2.0)
    with pytest.raises(ValueError, match="shape"):
        em.GriddingWindow.kaiser_bessel(2.0, math.nan)
    with pytest.raises(ValueError, match="voltage"):
        em.CtfOptics(-1.0, 2.7, 0.1)
    with pytest.raises(ValueError, match="amplitude contrast"):
        em.CtfOptics(300.0, 2.7, 1.0)
    w = em.GriddingWindow.linear()._c()
    assert (w.profile, w.half_width) == (_capi.WINDOW_TRIANGLE, 1.0)
    # The relativistic wavelength at 300 kV: 0.0196875 angstroms.
    assert abs(em.CtfOptics(300.0, 2.7, 0.1).wavelength - 0.0196875) < 1e-6


def test_bounds_and_mode(monkeypatch):
    assert em._resolve_bounds(2.5) == (-2.5, 2.5)
    assert em._resolve_bounds((-1.0, 3.0)) == (-1.0, 3.0)
    monkeypatch.delenv("REXLIB_B200_DETERMINISTIC", raising=False)
    assert em._mode(None) == _capi.INSERT_THROUGHPUT
    monkeypatch.setenv("REXLIB_B200_DETERMINISTIC", "1")
    assert em._mode(None) == _capi.INSERT_DETERMINISTIC
    assert em._mode(False) == _capi.INSERT_THROUGHPUT
    assert em._mode(True) == _capi.INSERT_DETERMINISTIC


def test_insertions_refuse_host_tensors_and_mixed_types():
    num = torch.zeros(8, 8, 5, dtype=torch.complex64)
    den = torch.zeros(8, 8, 5)
    sl = torch.zeros(2, 8, 5, dtype=torch.complex64)
    tr = torch.zeros(2, 3, 4)
    ra = torch.ones(5)
    with pytest.raises(ValueError, match="CUDA device"):
        em.insert_slices(num, den, sl, tr, ra, em.GriddingWindow.linear())
    with pytest.raises(TypeError, match="complex64 or complex128"):
        em.insert_slices(num.real, den, sl, tr, ra, em.GriddingWindow.linear())
