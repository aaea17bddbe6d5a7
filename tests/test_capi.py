"""The C-ABI library on the CPU: it loads, exports every entry point that
include/*.h declares, and refuses bad arguments before touching a device."""

import ctypes
import glob
import os
import re

import pytest

from rexlib_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        names.update(re.findall(r"REXLIB_B200_API\s+[\w\s\*]*?\b(rexlib_b200_\w+)\s*\(", text))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_functions()
    assert "rexlib_b200_insert_ctf_slices" in names
    assert len(names) >= 6


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    # and every declared symbol has a binding with a signature
    assert set(declared_functions()) <= set(_capi.SIGNATURES)


def test_abi_version():
    assert _capi.load().rexlib_b200_abi_version() == 2


def _descriptor(**changes):
    d = _capi.Insertion()
    d.volume_count = 1
    d.slices_per_volume = 1
    d.slice_extent = 8
    d.volume_extent = 8
    d.window = _capi.GriddingWindowC(_capi.WINDOW_TRIANGLE, 1.0, 0.0)
    d.numerator_out = d.numerator_in = 0x1000
    d.denominator_out = d.denominator_in = 0x2000
    d.slices = 0x3000
    d.transforms = 0x4000
    d.radial_weights = 0x5000
    for k, v in changes.items():
        setattr(d, k, v)
    return d


@pytest.mark.parametrize("changes, fragment", [
    ({"slice_extent": 0}, "extents must be positive"),
    ({"volume_count": -1}, "negative batch extents"),
    ({"window": _capi.GriddingWindowC(_capi.WINDOW_KAISER_BESSEL, -1.0, 2.0)}, "half-width"),
    ({"window": _capi.GriddingWindowC(_capi.WINDOW_KAISER_BESSEL, 2.0, float("nan"))}, "shape"),
    ({"window": _capi.GriddingWindowC(7, 1.0, 0.0)}, "unknown gridding profile"),
    ({"mode": 5}, "unknown insertion mode"),
    ({"slices": 0}, "null slice operand"),
    ({"numerator_out": 0x1004}, "8-byte aligned"),
])
def test_insertion_argument_checks(changes, fragment):
    lib = _capi.load()
    d = _descriptor(**changes)
    status = lib.rexlib_b200_insert_slices(ctypes.byref(d), None)
    assert status == _capi.INVALID_ARGUMENT
    assert fragment in lib.rexlib_b200_last_error().decode()


def test_ctf_optics_checks():
    lib = _capi.load()
    d = _descriptor()
    strides = _capi.BatchStrides(0, 1)
    bad = [(_capi.CtfOpticsC(-300.0, 2.7, 0.1), 1.0, "voltage"),
           (_capi.CtfOpticsC(300.0, float("inf"), 0.1), 1.0, "spherical aberration"),
           (_capi.CtfOpticsC(300.0, 2.7, 1.0), 1.0, "amplitude contrast"),
           (_capi.CtfOpticsC(300.0, 2.7, 0.1), 0.0, "pixel size")]
    for optics, pixel, fragment in bad:
        status = lib.rexlib_b200_insert_ctf_slices(ctypes.byref(d), ctypes.c_void_p(0x6000), strides, optics, pixel,
                                                   None)
        assert status == _capi.INVALID_ARGUMENT
        assert fragment in lib.rexlib_b200_last_error().decode()


def test_unsupported_sizes_are_refused():
    lib = _capi.load()
    d = _descriptor(slice_extent=4096)
    assert lib.rexlib_b200_insert_slices(ctypes.byref(d), None) == _capi.UNSUPPORTED


def test_empty_batch_needs_no_device():
    # No accumulator: nothing to copy, nothing to launch.
    lib = _capi.load()
    d = _descriptor(volume_count=0, numerator_out=0, numerator_in=0, denominator_out=0, denominator_in=0)
    assert lib.rexlib_b200_insert_slices(ctypes.byref(d), None) == _capi.OK


def test_workspace_query():
    lib = _capi.load()
    size = ctypes.c_size_t(123)
    assert lib.rexlib_b200_insertion_workspace_size(ctypes.byref(_descriptor()), ctypes.byref(size)) == _capi.OK
    assert size.value >= 0


@pytest.mark.parametrize("mode, extent, expected", [
    (_capi.INSERT_THROUGHPUT, 8, 1),       # below the tiled path's smallest volume: the slice-parallel kernel
    (_capi.INSERT_THROUGHPUT, 32, 4),      # settle, hit count, plan, tiled insertion
    (_capi.INSERT_DETERMINISTIC, 32, 3),   # settle, tile order, gather
    (_capi.INSERT_DETERMINISTIC, 8, 3),
])
def test_insertion_launch_counts(mode, extent, expected):
    # The count a bench reports as its kernel launches, answered on the host.
    lib = _capi.load()
    d = _descriptor(slice_extent=extent, volume_extent=extent, mode=mode)
    count = ctypes.c_int32(-1)
    assert lib.rexlib_b200_insertion_launches(ctypes.byref(d), ctypes.byref(count)) == _capi.OK
    assert count.value == expected


def test_float64_insertion_limits():
    # float64 (complex128 accumulators) runs the throughput mode with
    # Kaiser-Bessel half-widths up to 3; other element types are refused.
    lib = _capi.load()
    d = _descriptor(element_type=7)
    assert lib.rexlib_b200_insert_slices(ctypes.byref(d), None) == _capi.UNSUPPORTED
    assert "float32 or float64" in lib.rexlib_b200_last_error().decode()
    d = _descriptor(element_type=_capi.FLOAT64, mode=_capi.INSERT_DETERMINISTIC)
    assert lib.rexlib_b200_insert_slices(ctypes.byref(d), None) == _capi.UNSUPPORTED
    assert "throughput mode" in lib.rexlib_b200_last_error().decode()
    d = _descriptor(element_type=_capi.FLOAT64, window=_capi.GriddingWindowC(_capi.WINDOW_KAISER_BESSEL, 3.5, 2.0))
    assert lib.rexlib_b200_insert_slices(ctypes.byref(d), None) == _capi.UNSUPPORTED
    assert "half-widths up to 3" in lib.rexlib_b200_last_error().decode()
    # complex128 operands are 16-byte aligned
    d = _descriptor(element_type=_capi.FLOAT64, numerator_out=0x1008)
    assert lib.rexlib_b200_insert_slices(ctypes.byref(d), None) == _capi.INVALID_ARGUMENT
    assert "16-byte aligned" in lib.rexlib_b200_last_error().decode()
    # the slice-parallel kernel, with no workspace
    d = _descriptor(element_type=_capi.FLOAT64, slice_extent=64, volume_extent=64)
    count, size = ctypes.c_int32(-1), ctypes.c_size_t(123)
    assert lib.rexlib_b200_insertion_launches(ctypes.byref(d), ctypes.byref(count)) == _capi.OK
    assert lib.rexlib_b200_insertion_workspace_size(ctypes.byref(d), ctypes.byref(size)) == _capi.OK
    assert (count.value, size.value) == (1, 0)


def test_product_never_reaches_the_oracle():
    # The oracle is test infrastructure: no module or source of the product
    # names it, and importing the product's Python API loads no part of it.
    import subprocess
    import sys

    package = os.path.join(ROOT, "rexlib_b200")
    for dirpath, _, files in os.walk(package):
        for name in files:
            if name.endswith((".py", ".cu", ".cuh", ".h")):
                text = open(os.path.join(dirpath, name)).read()
                assert not re.search(r"\boracle\b", text), os.path.join(dirpath, name)
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        assert not re.search(r"\boracle\b", open(header).read()), header
    code = ("import sys; import rexlib_b200.em, rexlib_b200.fourier, rexlib_b200.arrays; "
            "sys.exit(1 if any(m == 'oracle' or m.startswith('oracle.') for m in sys.modules) else 0)")
    assert subprocess.run([sys.executable, "-c", code], cwd=ROOT).returncode == 0


def _standardization(**changes):
    s = _capi.Standardization()
    s.value = 0x1000
    s.keys = 0x2000
    s.images_per_key = 1
    s.batch = 2
    s.rank = 2
    s.extents[0] = s.extents[1] = 128
    s.radius = 57.6
    s.lower_bound, s.upper_bound = -3.0, 3.0
    for k, v in changes.items():
        setattr(s, k, v)
    return s


def test_standardize_rfft2_refusals():
    # The fused standardization + R2C checks its descriptor on the host.
    lib = _capi.load()
    out = ctypes.c_void_p(0x3000)
    call = lambda s, o=out: lib.rexlib_b200_standardize_rfft2(o, ctypes.byref(s), None, None)  # noqa: E731
    s = _standardization()
    s.extents[0] = s.extents[1] = 96
    assert call(s) == _capi.UNSUPPORTED and b"64, 128 or 256" in lib.rexlib_b200_last_error()
    s = _standardization(rank=3)
    s.extents[2] = 128
    assert call(s) == _capi.UNSUPPORTED
    assert call(_standardization(), None) == _capi.INVALID_ARGUMENT
    assert call(_standardization(value=0x1004)) == _capi.INVALID_ARGUMENT
    assert call(_standardization(lower_bound=1.0)) == _capi.INVALID_ARGUMENT
    assert b"either side of 0" in lib.rexlib_b200_last_error()
    assert call(_standardization(radius=-1.0)) == _capi.INVALID_ARGUMENT
    # nothing to do: no pointer is read
    assert call(_standardization(batch=0, value=0, keys=0), None) == _capi.OK


@pytest.mark.parametrize("compiler, flags", [("gcc", ["-std=c99", "-pedantic", "-x", "c"]),
                                             ("g++", ["-std=c++17", "-x", "c++"])])
def test_headers_compile_as_c_and_cpp(tmp_path, compiler, flags):
    # The boundary is plain C: a C or C++ caller (a plugin, a cgo or ctypes
    # stub) includes the headers without warnings.
    import shutil
    import subprocess

    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} is not installed")
    source = tmp_path / "use.c"
    source.write_text(
        "#include <string.h>\n"
        '#include "rexlib_b200.h"\n'
        "int main(void)\n{\n"
        "\trexlib_b200_insertion d;\n"
        "\tmemset(&d, 0, sizeof d);\n"
        "\td.element_type = REXLIB_B200_FLOAT64;\n"
        "\treturn (int)d.mode + (int)sizeof(rexlib_b200_standardization);\n}\n")
    result = subprocess.run([compiler, *flags, "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                             "-c", str(source), "-o", str(tmp_path / "use.o")], capture_output=True, text=True)
    assert result.returncode == 0, result.stderr
