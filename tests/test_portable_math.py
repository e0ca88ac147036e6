"""The engine's portable sin, cos, pow and scalbn (sinksim_b200/csrc/portable_math.cuh, a restatement of fdlibm 5.3)
must equal the reference's vendored fdlibm (third_party/fdlibm of the reference, built in oracle/_ref) bit for bit,
over the sample sets of the reference's tests/test_portable_math.cpp: once compiled for the host (CPU test) and once
compiled for sm_100a (GPU test, through the C ABI)."""
import numpy as np
import pytest

import sinksim_b200 as ssb
from _support import fdlibm_ref
from samples import reference_samples


def _ref(op, x, y=None):
    lib = fdlibm_ref()
    f = {"sin": lib.fdlibm_sin, "cos": lib.fdlibm_cos}.get(op)
    if f is not None:
        return np.array([f(v) for v in x])
    if op == "pow":
        return np.array([lib.fdlibm_pow(a, b) for a, b in zip(x, y)])
    return np.array([lib.fdlibm_scalbn(a, int(b)) for a, b in zip(x, y)])


def _same_bits(a, b):
    return (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))


@pytest.fixture(scope="module")
def cases():
    trig, (px, py), (sx, sn) = reference_samples()
    return dict(sin=(trig, None, _ref("sin", trig)), cos=(trig, None, _ref("cos", trig)), pow=(px, py, _ref("pow", px, py)),
                scalbn=(sx, sn, _ref("scalbn", sx, sn)))


@pytest.mark.parametrize("op", ["sin", "cos", "pow", "scalbn"])
def test_host_build_matches_fdlibm(cases, op):
    x, y, want = cases[op]
    got = ssb.portable_math(op, x, y, device=False)
    bad = ~_same_bits(got, want)
    assert not bad.any(), f"{op}: {bad.sum()} mismatches, first at x={x[bad][0]!r}"


@pytest.mark.gpu
@pytest.mark.parametrize("op", ["sin", "cos", "pow", "scalbn"])
def test_device_build_matches_fdlibm(cases, op):
    x, y, want = cases[op]
    got = ssb.portable_math(op, x, y, device=True)
    bad = ~_same_bits(got, want)
    assert not bad.any(), f"{op}: {bad.sum()} mismatches, first at x={x[bad][0]!r}"
