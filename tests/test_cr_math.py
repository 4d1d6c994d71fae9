"""Correctly rounded helpers of the strict kernels (cr_math.cuh).

The Manning depth factor DEPTH**(1.D0/3.D0) (rhs_dg_hydro.F) in the strict
kernels and in the oracle: both must give the correctly rounded double, so
that the strict build and the oracle agree bit for bit on Manning decks.

* dgswem::pow_third (dgswem_b200/csrc/cr_math.cuh) compiled for the host with
  the strict kernels' rule (no contraction) against the quadruple-precision
  pow rounded to double;
* the oracle's evaluation (orc_pow_third) against the same;
* the C library's pow, which the reference's gfortran build calls, is within
  one ulp of that value and equal to it for all but about 1 in 1,000 depths
  (reported, not asserted).
The device build of the same source is checked through the strict kernels'
bitwise parity with the oracle on Manning decks (tests/test_parity_gpu.py).
"""
import ctypes as C
import shutil
import subprocess

import numpy as np
import pytest

from oracle_lib import lib as oracle_lib

ROOT = __import__("pathlib").Path(__file__).resolve().parents[1]
_dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("crm") / "cr_math_check.so"
    subprocess.run([gxx, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-shared", "-I",
                    str(ROOT / "dgswem_b200" / "csrc"), str(ROOT / "tests" / "native" / "cr_math_check.cpp"),
                    "-o", str(out), "-lquadmath"], check=True)
    L = C.CDLL(str(out))
    L.cr_pow_third_eval.argtypes = [_dp, C.c_long, C.c_int, _dp, _dp, _dp]
    L.cr_div3_mismatches.argtypes = [_dp, C.c_long]
    L.cr_div3_mismatches.restype = C.c_long
    return L


def samples():
    rng = np.random.default_rng(20261203)
    near = [np.nextafter(2.0 ** k, t) for k in range(-60, 60) for t in (0.0, np.inf)]
    return np.concatenate([
        10.0 ** rng.uniform(-3, 3, 400_000),          # depths of the physical range
        2.0 ** rng.uniform(-1070, 1020, 100_000),     # every binade
        np.array(near), 2.0 ** np.arange(-1074, 1023, dtype=np.float64),
        np.arange(1, 2000, dtype=np.float64) ** 3,    # exact cubes
        np.array([5e-324, 1e-310, 0.01, 0.01 + 1e-18, 1.0, 7.999999999999999, 8.0]),
    ]).astype(np.float64)


@pytest.mark.parametrize("series", [0, 1])
def test_pow_third_correctly_rounded(checker, series):
    """series=0: as the kernels call it (single-precision log deciding the
    rounding, series when undecided); series=1: the series every time."""
    xs = np.ascontiguousarray(samples())
    ours, quad, libm = (np.empty_like(xs) for _ in range(3))
    checker.cr_pow_third_eval(xs.ctypes.data_as(_dp), len(xs), series, ours.ctypes.data_as(_dp),
                              quad.ctypes.data_as(_dp), libm.ctypes.data_as(_dp))
    np.testing.assert_array_equal(ours, quad)
    off = libm != quad
    ulps = np.abs(libm.view(np.int64) - quad.view(np.int64))
    print(f"C library pow: {off.sum()} of {len(xs)} one ulp from the correctly rounded value")
    assert ulps.max() <= 1


def test_pow_third_special_values(checker):
    xs = np.array([0.0, -1.0, np.inf, np.nan])
    ours, quad, libm = (np.empty_like(xs) for _ in range(3))
    checker.cr_pow_third_eval(xs.ctypes.data_as(_dp), len(xs), 0, ours.ctypes.data_as(_dp),
                              quad.ctypes.data_as(_dp), libm.ctypes.data_as(_dp))
    np.testing.assert_array_equal(ours, libm)  # 0, NaN, inf, NaN


def test_oracle_pow_third_correctly_rounded(checker):
    L = oracle_lib()
    L.orc_pow_third.argtypes = [_dp, C.c_long, _dp]
    xs = np.ascontiguousarray(samples())
    orc = np.empty_like(xs)
    L.orc_pow_third(xs.ctypes.data_as(_dp), len(xs), orc.ctypes.data_as(_dp))
    ours, quad, libm = (np.empty_like(xs) for _ in range(3))
    checker.cr_pow_third_eval(xs.ctypes.data_as(_dp), len(xs), 0, ours.ctypes.data_as(_dp),
                              quad.ctypes.data_as(_dp), libm.ctypes.data_as(_dp))
    np.testing.assert_array_equal(orc, quad)


def test_div3_is_the_ieee_quotient(checker):
    """div3(x) and x / 3.0 bit for bit (signed zeros included) over random
    bit patterns (every exponent, both signs, subnormals) and significands
    at both ends of a binade."""
    rng = np.random.default_rng(7)
    bits = rng.integers(0, 2 ** 63, 4_000_000, dtype=np.int64) * rng.choice([1, -1], 4_000_000)
    xs = bits.view(np.float64)
    xs = xs[np.isfinite(xs)]
    k = np.arange(1_000_000, dtype=np.float64)
    edges = np.concatenate([np.ldexp(1.0 + k * 2.0 ** -52, (k % 200 - 100).astype(int)),
                            np.ldexp(2.0 - (k + 1) * 2.0 ** -52, (k % 200 - 100).astype(int)),
                            [0.0, -0.0, 5e-324, -5e-324, 1e-323, 3.0, 1.5, 2.0 ** -1022]])
    xs = np.ascontiguousarray(np.concatenate([xs, edges]))
    assert checker.cr_div3_mismatches(xs.ctypes.data_as(_dp), len(xs)) == 0
