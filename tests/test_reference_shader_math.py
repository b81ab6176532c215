"""The path's math pinned to the reference's own shader code.  oracle/build_oracle.py compiles
Stratum2's src/Shaders/common/rng.hlsli (xxhash32, pcg, pcg4d, RandomSampler), common.hlsli
(octahedral normal packing through D3DX_DXGIFormatConvert.inl's R16G16_SNORM conversion,
makeOrthonormal and the sampling maps) and microfacet.hlsli (GTR1, GTR2, Smith masking, VNDF
sampling, Schlick and dielectric Fresnel) as host C++ into oracle/_ref/libref_shader.so.  On
seeded inputs in each function's domain:

* the oracle's FP32 restatement equals the reference bit for bit for the integer functions, the
  packing, Schlick, the dielectric Fresnel term, makeOrthonormal and the triangle map, and within
  float rounding (1e-6 relative, 2e-5 absolute for the trigonometric sampling maps) for the rest;
* the oracle's FP64 build agrees within float tolerances (packing within one SNORM16 step);
* the device functions (s2_device_math, GPU) equal the reference bit for bit for the integer
  functions and the packing, and within float rounding for the rest (1e-5 relative; 1e-4 for
  GTR1, whose (a^2 - 1) / log(a^2) is ill-conditioned as alpha -> 1).
"""
import ctypes as C

import numpy as np
import pytest

from oracle_lib import MATH_FUNCTIONS, MATH_OUT, math_inputs, oracle, ref_shader

N = 20000
EXACT_F32 = {"xxhash32", "pcg", "pcg4d", "next_float", "pack_normal", "unpack_normal", "smith_gtr1", "schlick",
             "fresnel_dielectric", "uniform_triangle", "orthonormal"}
INTEGER = {"xxhash32", "pcg", "pcg4d", "next_float", "pack_normal"}
TRIG = {"vndf", "concentric_disc", "cos_hemisphere", "uniform_sphere"}


def _ref(fn, a):
    L = ref_shader()
    if L is None:
        pytest.skip("reference shader math not built (reference tree absent when the oracle was built)")
    r = np.zeros((len(a), MATH_OUT))
    assert L.ref_shader_math(fn, np.ascontiguousarray(a).ctypes.data, len(a), r.ctypes.data) == 0
    return r


def _oracle(fn, a, precision):
    o = np.zeros((len(a), MATH_OUT))
    assert oracle().oracle_math(fn, np.ascontiguousarray(a).ctypes.data, len(a), o.ctypes.data, precision) == 0
    return o


def _close(name, got, ref, exact, device=False):
    if exact:
        np.testing.assert_array_equal(got, ref, err_msg=name)
    elif device and name == "gtr1":
        # (a^2 - 1) / log(a^2) is ill-conditioned as alpha -> 1: one ulp of the device's logf
        # there is up to 2e-5 relative in the result
        np.testing.assert_allclose(got, ref, rtol=1e-4, atol=0, err_msg=name)
    elif device and name == "vndf":
        # the renderer is compiled with approximate division and square root (two ulp each); the
        # visible-normal map is ill-conditioned for grazing directions, where that moves the sampled
        # half vector by up to a few 1e-5
        np.testing.assert_allclose(got, ref, rtol=0, atol=5e-5, err_msg=name)
    elif name in TRIG:
        np.testing.assert_allclose(got, ref, rtol=0, atol=2e-5, err_msg=name)
    elif device:
        # the device's sqrtf / powf / division (approximate: two ulp) round near the host's
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-7, err_msg=name)
    else:
        np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-7, err_msg=name)


@pytest.mark.parametrize("fn", range(len(MATH_FUNCTIONS)), ids=MATH_FUNCTIONS)
def test_oracle_fp32_matches_reference_shader_math(fn):
    name = MATH_FUNCTIONS[fn]
    a = math_inputs(fn, N, 1)
    _close(name, _oracle(fn, a, 32), _ref(fn, a), name in EXACT_F32)


@pytest.mark.parametrize("fn", range(len(MATH_FUNCTIONS)), ids=MATH_FUNCTIONS)
def test_oracle_fp64_matches_reference_shader_math(fn):
    name = MATH_FUNCTIONS[fn]
    a = math_inputs(fn, N, 2)
    got, ref = _oracle(fn, a, 64), _ref(fn, a)
    if name == "pack_normal":
        g, r = got[:, 0].astype(np.int64), ref[:, 0].astype(np.int64)
        for sh in (0, 16):
            d = np.abs((((g >> sh) & 0xFFFF) ^ 0x8000) - (((r >> sh) & 0xFFFF) ^ 0x8000))
            assert d.max() <= 1, name
    elif name in INTEGER:
        np.testing.assert_array_equal(got, ref, err_msg=name)
    elif name in ("gtr1", "gtr2"):
        np.testing.assert_allclose(got, ref, rtol=2e-5, atol=0, err_msg=name)
    else:
        np.testing.assert_allclose(got, ref, rtol=0, atol=5e-5, err_msg=name)


@pytest.mark.gpu
@pytest.mark.parametrize("fn", range(len(MATH_FUNCTIONS)), ids=MATH_FUNCTIONS)
def test_device_math_matches_reference_shader_math(device, fn):
    from stratum2_b200 import _abi
    name = MATH_FUNCTIONS[fn]
    a = math_inputs(fn, N, 3)
    ref = _ref(fn, a)
    got = np.zeros((len(a), MATH_OUT))
    rc = _abi.lib().s2_device_math(device._h, fn, np.ascontiguousarray(a).ctypes.data, len(a), got.ctypes.data)
    assert rc == _abi.S2_OK, _abi.lib().s2_last_error(device._h)
    _close(name, got, ref, name in INTEGER, device=True)
