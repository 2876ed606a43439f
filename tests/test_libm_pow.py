"""Math.Pow on the path: the kernels' pow (mycel_b200/csrc/libm_pow.h) against the C library's pow.

Mycel.Core computes E_e = Emin + Math.Pow(rho, p)(E0 - Emin) (FemOperator.cs:100,133) and
p Math.Pow(rho, p - 1) dE (SensitivityAnalysis.cs:93-95); on Linux .NET's Math.Pow is the C library's pow.
Here the same header is compiled for the CPU (same operation sequence as the device build, every operation
rounded once) and compared bit for bit with the library's pow, which the oracle calls. The device build is
compared on the GPU in test_gpu_parity.py.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def twin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("powtwin") / "libpowtwin.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
                           "-o", out, os.path.join(HERE, "native", "libm_pow_twin.cpp")])
    lib = C.CDLL(out)
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    lib.twin_pow.argtypes = [C.c_int64, dp, dp, C.c_int64, dp]

    def f(x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(np.atleast_1d(y), dtype=np.float64)
        out = np.empty(x.size)
        lib.twin_pow(x.size, x, y, y.size, out)
        return out
    return f


def same_bits(a, b):
    a = np.asarray(a).view(np.uint64)
    b = np.asarray(b).view(np.uint64)
    nan = np.isnan(np.asarray(a).view(np.float64)) & np.isnan(np.asarray(b).view(np.float64))
    return (a == b) | nan


@pytest.mark.parametrize("p", [1.0, 2.0, 3.0, 3.5, 0.0, 2.5, 1.5, 4.0, 5.0])
def test_simp_exponents_bit_exact(oracle, twin, p):
    # densities as the SIMP loop sees them: (0, 1], and a log-uniform sweep down to 1e-12
    rng = np.random.default_rng(int(p * 10))
    x = np.concatenate([1e-9 + rng.random(400_000) * (1 - 1e-9), 10.0 ** rng.uniform(-12, 0, 200_000),
                        [1.0, 1e-9, 1e-3, 0.5, 0.3, 0.15]])
    assert same_bits(twin(x, p), oracle.math_pow(x, p)).all()


def test_wide_range_and_special_values_bit_exact(oracle, twin):
    rng = np.random.default_rng(11)
    n = 400_000
    x = np.ldexp(rng.random(n) + 0.5, rng.integers(-1074, 1024, n))
    y = rng.uniform(-60, 60, n)
    yi = np.floor(y)
    special = np.array([0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, np.nan, 0.5, 2.0, -2.0, 1e-310, -1e-310, 1e308,
                        3.0, 0.1, 5e-324, 2.0 ** -70, 2.0 ** 64])
    sx, sy = np.meshgrid(special, special)
    raw = rng.integers(0, 2 ** 63, size=(2, n), dtype=np.int64).view(np.float64)
    for xs, ys in ((x, y), (-x, yi), (sx.ravel(), sy.ravel()), (np.abs(raw[0]), raw[1]),
                   (np.abs(raw[0]), np.ldexp(rng.random(n) - 0.5, rng.integers(-20, 60, n)))):
        with np.errstate(all="ignore"):
            ok = same_bits(twin(xs, ys), oracle.math_pow(xs, ys))
        assert ok.all(), (xs[~ok][:3], ys[~ok][:3])


def test_results_near_the_subnormal_edge_bit_exact(oracle, twin):
    # exp arguments below -708: the scaled path that rounds once before scaling into the subnormal range
    rng = np.random.default_rng(5)
    x = rng.uniform(1e-3, 0.5, 300_000)
    y = rng.uniform(-1075, -700, 300_000) / np.log(x)
    assert same_bits(twin(x, y), oracle.math_pow(x, y)).all()
