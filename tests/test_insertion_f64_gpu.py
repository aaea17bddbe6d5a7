"""Float64 insertions on the B200 (complex128 accumulators and slices, float64
transforms, weights and CTF parameters) against the oracle's float64
instantiation, which is bit-identical to the reference's CPU functor in
double. Only the order of the FP64 sums differs: relative L2 <= 1e-12."""

import numpy as np
import pytest
import torch

from rexlib_b200 import _capi, em
from tests.cases import insertion_inputs, rel_l2
from tests.test_insertion_gpu import OPTICS, PIXEL, WINDOWS, oracle_insert

pytestmark = pytest.mark.gpu

TOL = 1e-12


def as_f64(c):
    d = dict(c)
    for k, v in c.items():
        if isinstance(v, np.ndarray):
            d[k] = v.astype(np.complex128 if np.iscomplexobj(v) else np.float64)
    return d


def gpu_insert_f64(kind, c, window, deterministic=False):
    to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    V = c["numerator"].shape[0]
    num = to(c["numerator"].reshape(V, 1, *c["numerator"].shape[1:]))
    den = to(c["denominator"].reshape(V, 1, *c["denominator"].shape[1:]))
    args = dict(numerator_out=num, denominator_out=den, deterministic=deterministic)
    sl, tr, ra = to(c["slices"]), to(c["transforms"]), to(c["radial"])
    if kind == "plain":
        em.insert_slices(num, den, sl, tr, ra, window, **args)
    elif kind == "ctf":
        em.insert_ctf_slices(num, den, sl, tr, to(c["extra"]), ra, window, OPTICS, PIXEL, **args)
    else:
        em.insert_weighted_slices(num, den, sl, to(c["extra"]), tr, ra, window, **args)
    torch.cuda.synchronize()
    shape = c["numerator"].shape
    return num.cpu().numpy().reshape(shape), den.cpu().numpy().reshape(shape)


@pytest.mark.parametrize("kind", ["plain", "ctf", "weighted"])
@pytest.mark.parametrize("window_name", ["nearest", "linear", "kb15", "kb2"])
@pytest.mark.parametrize("n,big", [(6, 12), (5, 7), (8, 8), (7, 7), (16, 16), (12, 9)])
def test_float64_insertion_matches_oracle(cuda, kind, window_name, n, big):
    c = as_f64(insertion_inputs(n, big, 7, volumes=2, kind=kind, seed=n * 100 + big, radial_per_particle=True))
    gw, ow = WINDOWS[window_name]
    gnum, gden = gpu_insert_f64(kind, c, gw)
    assert gnum.dtype == np.complex128 and gden.dtype == np.float64
    onum, oden = oracle_insert(kind, c, ow, dtype=np.float64)
    assert rel_l2(gnum, onum) <= TOL and rel_l2(gden, oden) <= TOL, (rel_l2(gnum, onum), rel_l2(gden, oden))


@pytest.mark.parametrize("kind", ["plain", "ctf"])
@pytest.mark.parametrize("n,big", [(64, 64), (63, 63), (32, 64)])
def test_float64_insertion_larger(cuda, kind, n, big):
    c = as_f64(insertion_inputs(n, big, 40, kind=kind, seed=11, zero_accumulators=True))
    gw, ow = WINDOWS["linear"]
    gnum, gden = gpu_insert_f64(kind, c, gw)
    onum, oden = oracle_insert(kind, c, ow, dtype=np.float64)
    assert rel_l2(gnum, onum) <= TOL and rel_l2(gden, oden) <= TOL


def test_float64_is_more_accurate_than_float32(cuda):
    # Against the oracle's float64 result, the float64 insertion's error sits
    # far below the float32 insertion's.
    c32 = insertion_inputs(32, 32, 30, kind="ctf", seed=5, zero_accumulators=True)
    c64 = as_f64(c32)
    gw, ow = WINDOWS["linear"]
    g64, _ = gpu_insert_f64("ctf", c64, gw)
    o64, _ = oracle_insert("ctf", c64, ow, dtype=np.float64)
    from tests.test_insertion_gpu import gpu_insert
    g32 = gpu_insert("ctf", c32, gw)[0]
    assert rel_l2(g64, o64) * 1e5 < rel_l2(g32, o64)


def test_float64_refusals(cuda):
    c = as_f64(insertion_inputs(8, 8, 3, seed=1))
    gw = WINDOWS["linear"][0]
    with pytest.raises(_capi.RexlibB200Error, match="throughput mode") as e:
        gpu_insert_f64("plain", c, gw, deterministic=True)
    assert e.value.status == _capi.UNSUPPORTED
    with pytest.raises(_capi.RexlibB200Error, match="half-widths up to 3"):
        gpu_insert_f64("plain", c, em.GriddingWindow.kaiser_bessel(3.5, 8.0))
    # one element type for every operand
    num = torch.zeros(1, 8, 8, 5, dtype=torch.complex128, device="cuda")
    den = torch.zeros(1, 8, 8, 5, dtype=torch.float64, device="cuda")
    sl = torch.zeros(2, 8, 5, dtype=torch.complex64, device="cuda")
    tr = torch.zeros(2, 3, 4, dtype=torch.float64, device="cuda")
    ra = torch.ones(5, dtype=torch.float64, device="cuda")
    with pytest.raises(TypeError, match="slices must be torch.complex128"):
        em.insert_slices(num, den, sl, tr, ra, gw)
