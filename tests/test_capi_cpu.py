"""C ABI checks that need no GPU: exports, argument errors, no-device error."""
import os
import re

import numpy as np
import pytest

from helpers import ROOT
from tval3g import capi, workloads as W


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"\b(tval3g_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    declared = _declared("tval3g.h")
    assert "tval3g_solve" in declared and len(declared) >= 15
    for name in declared:
        assert hasattr(L, name), name
    assert set(capi.EXPORTS) <= set(declared)


def _opts():
    return W.options(2 ** 8, 2 ** 5, 1e-4, 10, tv_norm=0)


def _dense_spec(shape=(4, 4), m=5, ncols=16, layers=1):
    A = np.zeros((m, ncols), np.float32)
    return capi.dense_problem(shape, A, layers)


@pytest.mark.parametrize("case,msg", [
    ("ut", "Argument error: U and Ut must have the same size!"),
    ("u", "Argument error: the length of U must be equal to A.dim_x * layers!"),
    ("b", "Argument error: b.len must be equal to A.dim_y * layers!"),
])
def test_dense_argument_errors_match_reference(case, msg):
    """Messages and check order of check_params (2d/tval3_cpu_2d.cpp:696-713)."""
    spec = _dense_spec()
    b = np.zeros(5, np.float32)
    Ut = None
    if case == "ut":
        Ut = np.zeros(7, np.float32)
    elif case == "u":
        spec = _dense_spec(shape=(4, 5))
    elif case == "b":
        b = np.zeros(6, np.float32)
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(spec, b, _opts(), Ut=Ut)
    assert e.value.code == capi.ERR_ARGUMENT
    assert str(e.value) == msg


def test_ray_argument_errors():
    g = W.ring_geometry(16, 16)
    spec = capi.ray2d_problem((16, 16), g)
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(spec, np.zeros(10, np.float32), _opts())
    assert str(e.value) == "Argument error: b.len must be equal to A.num_emitters * A.num_receivers!"
    g2 = dict(g)
    g2["xr"] = g["xr"] + 100
    spec = capi.ray2d_problem((16, 16), g2)
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(spec, np.zeros(256, np.float32), _opts())
    # the reference indexes out of bounds here; the C ABI refuses
    assert e.value.code == capi.ERR_ARGUMENT
    spec = capi.ray2d_problem((16, 16), g)
    spec.p.layers = 2
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(spec, np.zeros(256, np.float32), _opts())
    assert str(e.value) == "Argument error: multilayer reconstruction with dynamic calculation is not supported!"


def test_3d_argument_errors():
    spec = capi.dense_problem((2, 2, 2), np.zeros((3, 8), np.float32))
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(spec, np.zeros(4, np.float32), _opts())
    assert str(e.value) == "Argument error: b.len must be equal to A.dim_y!"
    spec = capi.dense_problem((2, 2, 3), np.zeros((3, 8), np.float32))
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(spec, np.zeros(3, np.float32), _opts())
    assert str(e.value) == "Argument error: the length of U must be equal to A.dim_x!"


def test_f64_argument_errors_match_reference():
    """The double-data entry point validates like the float one (the
    reference's messages, before any device work)."""
    spec = _dense_spec()
    A64 = np.zeros((5, 16), np.float64)
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve_f64(spec, np.zeros(6), _opts(), values=A64)
    assert e.value.code == capi.ERR_ARGUMENT
    assert str(e.value) == "Argument error: b.len must be equal to A.dim_y * layers!"
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve_f64(spec, np.zeros(5), _opts(), Ut=np.zeros(7), values=A64)
    assert str(e.value) == "Argument error: U and Ut must have the same size!"
    with pytest.raises(capi.TVAL3Error) as e:   # the float A of the spec is not read
        capi.solve_f64(spec, np.zeros(5), _opts(), values=None)
    assert str(e.value) == "Argument error: A is NULL"


def test_f64_no_device_is_an_error_not_a_fallback():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve_f64(_dense_spec(), np.zeros(5), _opts(), values=np.zeros((5, 16)))
    assert e.value.code in (capi.ERR_NO_DEVICE, capi.ERR_CUDA)


def test_no_device_is_an_error_not_a_fallback():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    spec = _dense_spec()
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(spec, np.zeros(5, np.float32), _opts())
    assert e.value.code in (capi.ERR_NO_DEVICE, capi.ERR_CUDA)


def test_complex_argument_errors():
    """Complex data: the reference's size checks, layers included."""
    A = np.zeros((5, 16), np.complex64)
    spec = capi.dense_problem((4, 4), A)
    assert spec.p.complex_data == 1
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(spec, np.zeros(6, np.complex64), _opts())
    assert str(e.value) == "Argument error: b.len must be equal to A.dim_y * layers!"
    spec = capi.dense_problem((4, 8), A, layers=2)   # layers: b.len = A.dim_y * layers
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(spec, np.zeros(11, np.complex64), _opts())
    assert str(e.value) == "Argument error: b.len must be equal to A.dim_y * layers!"
    spec = capi.dense_problem((2, 2, 4), A)   # 3D: the reference's 3D size message
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(spec, np.zeros(6, np.complex64), _opts())
    assert str(e.value) == "Argument error: b.len must be equal to A.dim_y!"


def test_philox_known_answers():
    """The counter-based generator's core against the published Philox-4x32-10
    known-answer vectors (Salmon et al., SC 2011; counter, key -> output)."""
    kat = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for c, k, want in kat:
        got = W.philox4x32_10([np.array([v], np.uint64) for v in c], k)
        assert tuple(int(x[0]) for x in got) == want


@pytest.mark.parametrize("seed,offset,count,scale", [(0, 0, 1000, 1.0), (12345678901, 7, 5001, 0.25),
                                                     ((1 << 40) + 3, (1 << 33) + 1, 4099, 0.125)])
def test_gaussian_host_equals_numpy(seed, offset, count, scale):
    """tval3g_gaussian_host (C++) and the numpy restatement give the same
    stream bit for bit; any window of it equals the same slice of a longer
    draw (counter-based: offsets compose)."""
    h = capi.gaussian_host(count, seed, scale, offset)
    np.testing.assert_array_equal(h, W.philox_gaussian(seed, count, scale, offset))
    np.testing.assert_array_equal(capi.gaussian_host(count - 5, seed, scale, offset + 5), h[5:])


def test_gaussian_stream_statistics():
    z = capi.gaussian_host(1 << 20, 99)
    assert abs(z.mean()) < 5e-3 and abs(z.std() - 1) < 5e-3
    assert abs(np.mean(z ** 4) - 3) < 0.05   # Gaussian kurtosis
