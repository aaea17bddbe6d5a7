"""The array operations on the GPU, through the C-ABI, against the host.

Real add and divide, and complex add, are IEEE operations: numpy's results
are the reference's, and the kernels must give the same bits. Complex divide
is compared bit for bit with the oracle (the reference's std::complex
division, compiled by g++); for complex128 the operands stay away from the
float64 overflow and underflow limits, where libgcc rescales. NaN results
compare as NaN, whatever their payload bits; zeros compare with their signs.
"""

import numpy as np
import pytest
import torch

import oracle
from rexlib_b200 import arrays

pytestmark = pytest.mark.gpu

TYPES = [torch.float32, torch.float64, torch.complex64, torch.complex128]
NP = {torch.float32: np.float32, torch.float64: np.float64, torch.complex64: np.complex64,
      torch.complex128: np.complex128}


def same_bits(got: np.ndarray, want: np.ndarray) -> bool:
    """Equal bit for bit, NaN payloads aside."""
    assert got.dtype == want.dtype and got.shape == want.shape
    real = np.float32 if got.dtype in (np.float32, np.complex64) else np.float64
    g = got.reshape(-1).view(real)
    w = want.reshape(-1).view(real)
    nan = np.isnan(g) & np.isnan(w)
    bits = np.uint32 if real == np.float32 else np.uint64
    return bool(np.array_equal(g.view(bits)[~nan], w.view(bits)[~nan]) and (np.isnan(g) == np.isnan(w)).all())


def values(dtype, n, rng, specials=True):
    """Seeded values over many binades, with zeros of both signs,
    infinities, NaN and subnormals mixed in."""
    np_dtype = NP[dtype]
    real = np.float32 if np_dtype in (np.float32, np.complex64) else np.float64
    span = 30 if real == np.float32 else 200

    def part():
        p = (rng.standard_normal(n) * np.exp(rng.uniform(-span, span, n))).astype(real)
        if specials and n >= 64:
            # complex128 quotients are exact away from the float64 range
            # limits only (libgcc rescales there): no subnormals for them
            tiny = 1e-90 if np_dtype == np.complex128 else np.finfo(real).smallest_subnormal
            pick = rng.choice(n, size=n // 16, replace=False)
            p[pick] = rng.choice(np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1.0, tiny * 3, -tiny], real),
                                 size=pick.size)
        return p

    if np.dtype(np_dtype).kind == "c":
        out = np.empty(n, np_dtype)
        out.real = part()
        out.imag = part()
        return out
    return part()


def to_device(a: np.ndarray, offset: int = 0) -> torch.Tensor:
    """A device array holding `a`, starting `offset` elements into its
    allocation (an offset of one breaks the 16-byte alignment)."""
    t = torch.from_numpy(np.ascontiguousarray(a).reshape(-1))
    buf = torch.empty(t.numel() + offset, dtype=t.dtype, device="cuda")
    view = buf[offset:]
    view.copy_(t)
    return view.view(a.shape)


def host_result(name, x, y):
    if name == "add":
        return x + y
    if np.iscomplexobj(x):
        return oracle.divide(x, y)
    with np.errstate(all="ignore"):
        return x / y


@pytest.mark.parametrize("dtype", TYPES, ids=str)
@pytest.mark.parametrize("name", ["add", "divide"])
@pytest.mark.parametrize("n", [1, 3, 4, 1000, 65_537])
def test_binary_matches_host(cuda, dtype, name, n):
    rng = np.random.default_rng(n * 7 + TYPES.index(dtype))
    x, y = values(dtype, n, rng), values(dtype, n, rng)
    got = getattr(arrays, name)(to_device(x), to_device(y)).cpu().numpy()
    assert same_bits(got, host_result(name, x, y))


@pytest.mark.parametrize("dtype", TYPES, ids=str)
@pytest.mark.parametrize("name", ["add", "divide"])
@pytest.mark.parametrize("offsets", [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1)])
def test_binary_on_unaligned_arrays(cuda, dtype, name, offsets):
    rng = np.random.default_rng(sum(offsets) + 17)
    n = 4099
    x, y = values(dtype, n, rng), values(dtype, n, rng)
    out = to_device(np.zeros(n, NP[dtype]), offsets[2])
    getattr(arrays, name)(to_device(x, offsets[0]), to_device(y, offsets[1]), out=out)
    assert same_bits(out.cpu().numpy(), host_result(name, x, y))


@pytest.mark.parametrize("dtype", TYPES, ids=str)
@pytest.mark.parametrize("name", ["add", "divide"])
@pytest.mark.parametrize("side", ["x", "y", "both"])
def test_binary_broadcasts_one_element(cuda, dtype, name, side):
    rng = np.random.default_rng(5)
    n = 3001
    x = values(dtype, 1 if side in ("x", "both") else n, rng, specials=False)
    y = values(dtype, 1 if side in ("y", "both") else n, rng, specials=False)
    if side != "both":
        y = y.reshape(()) if side == "y" else y
        x = x.reshape(()) if side == "x" else x
    got = getattr(arrays, name)(to_device(x), to_device(y)).cpu().numpy()
    want = host_result(name, np.broadcast_to(x, np.broadcast_shapes(x.shape, y.shape)).copy(),
                       np.broadcast_to(y, np.broadcast_shapes(x.shape, y.shape)).copy())
    assert same_bits(got, want)


def test_complex_divide_special_values(cuda):
    specials = [0.0, -0.0, 1.0, -2.5, np.inf, -np.inf, np.nan, 1e-30, 3e30, 1e-40]
    for dtype in (torch.complex64, torch.complex128):
        s = np.array([complex(a, b) for a in specials for b in specials], NP[dtype])
        x, y = np.repeat(s, s.size), np.tile(s, s.size)
        got = arrays.divide(to_device(x), to_device(y)).cpu().numpy()
        assert same_bits(got, oracle.divide(x, y)), dtype


def test_divide_in_place_and_large(cuda):
    rng = np.random.default_rng(3)
    n = (1 << 24) + 5
    x = values(torch.complex64, n, rng, specials=False)
    y = values(torch.complex64, n, rng, specials=False)
    dx = to_device(x)
    arrays.divide(dx, to_device(y), out=dx)
    assert same_bits(dx.cpu().numpy(), oracle.divide(x, y))


@pytest.mark.parametrize("dtype", TYPES, ids=str)
@pytest.mark.parametrize("n", [0, 1, 5, 4096 + 3])
@pytest.mark.parametrize("offset", [0, 1])
def test_fill(cuda, dtype, n, offset):
    value = complex(1.5, -2.25) if dtype.is_complex else -3.75
    buf = torch.full((n + offset + 2,), 7, dtype=dtype, device="cuda")
    arrays.fill(buf[offset:offset + n], value)
    host = buf.cpu().numpy()
    assert (host[offset:offset + n] == NP[dtype](value)).all()
    assert (host[:offset] == 7).all() and (host[offset + n:] == 7).all()


def test_zeros_full_and_copy(cuda):
    z = arrays.zeros((3, 5, 7), torch.complex64)
    assert z.shape == (3, 5, 7) and not z.cpu().numpy().view(np.uint32).any()
    f = arrays.full((4, 6), 2.5, torch.float64)
    assert (f.cpu().numpy() == 2.5).all()
    o = arrays.ones((3, 9), torch.complex128)
    assert (o.cpu().numpy() == 1.0).all()
    c = arrays.copy(f)
    assert c.data_ptr() != f.data_ptr() and torch.equal(c, f)


def test_python_mirror_refusals(cuda):
    x = torch.ones(4, device="cuda")
    with pytest.raises(TypeError, match="share one type"):
        arrays.add(x, x.double())
    with pytest.raises(ValueError, match="one element is broadcast"):
        arrays.add(torch.ones(4, 4, device="cuda"), torch.ones(1, 4, device="cuda"))
    with pytest.raises(TypeError, match="float32, float64"):
        arrays.divide(x.half(), x.half())
    with pytest.raises(ValueError, match="contiguous"):
        arrays.add(torch.ones(4, 4, device="cuda").t(), torch.ones(4, 4, device="cuda"))


def test_transfers_round_trip(cuda):
    x = torch.randn(1000, dtype=torch.complex64)
    d = arrays.to_device(x)
    assert d.is_cuda and arrays.to_device(d) is d
    assert torch.equal(arrays.to_host(d), x)
    pinned = x.pin_memory()
    out = torch.empty_like(d)
    assert arrays.to_device_copy(pinned, out=out) is out
    torch.cuda.synchronize()
    assert torch.equal(out.cpu(), x)
    assert arrays.to_device_copy(d).data_ptr() != d.data_ptr()
