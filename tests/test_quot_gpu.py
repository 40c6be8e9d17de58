"""fb_quot -- quotients by one divisor sharing a single division (the
azimuthal transport's q / (RhoInt + 1e-20)) -- against IEEE division,
bit for bit, on random operands over the ranges the gas takes and far
beyond them."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "dustyfargoadsg_b200", "csrc")


def _lib(tmp_path):
    so = str(tmp_path / "quot_check.so")
    subprocess.run(["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "--fmad=false",
                    "-Xcompiler", "-fPIC", "-shared", "-I" + CSRC, "-I" + os.path.join(os.path.dirname(HERE), "include"),
                    os.path.join(HERE, "native", "quot_check.cu"), "-o", so], check=True)
    return C.CDLL(so)


def test_shared_reciprocal_quotient_is_ieee_division(tmp_path):
    lib = _lib(tmp_path)
    rng = np.random.default_rng(7)
    n = 1 << 22
    # numerators: signed, 1e-12 .. 1e12; divisors: densities 1e-10 .. 1e4 plus
    # the 1e-20 guard, and random mantissas over a wide exponent range
    a = rng.choice([-1.0, 1.0], n) * 10.0 ** rng.uniform(-12, 12, n)
    d = np.where(rng.random(n) < 0.5, 10.0 ** rng.uniform(-10, 4, n) + 1e-20,
                 rng.uniform(1.0, 2.0, n) * 2.0 ** rng.integers(-200, 200, n))
    a[:1000] = rng.uniform(1.0, 2.0, 1000)   # same-binade operands
    d[:1000] = rng.uniform(1.0, 2.0, 1000)
    a[1000:2000] = 0.0
    qa, qb = np.empty(n), np.empty(n)
    mis = C.c_ulonglong()
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    assert lib.quot_check(n, dp(a), dp(d), dp(qa), dp(qb), C.byref(mis)) == 0
    assert np.array_equal(qb, a / d)            # the GPU's division is IEEE
    assert mis.value == 0 and np.array_equal(qa.view(np.int64), qb.view(np.int64))
