"""The correctly rounded exp, log10 and pow the kernels use in place of the C
library calls micm makes (rate_constant_functions.hpp:52-136 and the step-size
factor std::pow(error, 1 / order), rosenbrock.inl:232-235).

CPU: the host build is correctly rounded on seeded samples of the arguments the
solver meets (checked against exactly rounded values from Python's decimal
module), and therefore equal to glibc's results wherever glibc rounds
correctly.  GPU: the device build returns the host build's bits."""
import ctypes as C
import math
from decimal import Decimal, getcontext

import numpy as np
import pytest

from micm_b200._native import check, lib

EXP, LOG10, POW = 0, 1, 2


def _samples(seed=11, n=4000):
    rng = np.random.default_rng(seed)
    # exp: C/T of Arrhenius terms (C in [-2000, 500] K, T in [200, 310] K) and wide arguments
    x_exp = np.concatenate([rng.uniform(-2000, 500, n) / rng.uniform(200, 310, n), rng.uniform(-700, 700, n)])
    # log10: Troe's k0 [M] / kinf ratios, 1e-12 .. 1e12, and wide values
    x_log = np.concatenate([10 ** rng.uniform(-12, 12, n), np.exp(rng.uniform(-700, 700, n))])
    # pow: (T / 300)^B, Fc^(...), and the step-size factor error^(1/order)
    b1 = rng.uniform(200, 310, n) / 300.0
    e1 = rng.uniform(-8, 8, n)
    err = 10 ** rng.uniform(-10, 3, n)
    inv_order = rng.choice([1 / 2, 1 / 3, 1 / 4], n)
    x_pow = np.concatenate([b1, err])
    y_pow = np.concatenate([e1, inv_order])
    return x_exp, x_log, x_pow, y_pow


def _host(fn, x, y=None):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = None if y is None else np.ascontiguousarray(y, dtype=np.float64)
    out = np.empty_like(x)
    check(lib().micmb_math_eval(fn, x.ctypes.data, None if y is None else y.ctypes.data, out.ctypes.data,
                                len(x), 0))
    return out


def _exact(fn, x, y=None):
    getcontext().prec = 60
    ln10 = Decimal(10).ln()
    out = np.empty(len(x))
    for i, v in enumerate(x):
        d = Decimal(float(v))
        if fn == EXP:
            r = d.exp()
        elif fn == LOG10:
            r = d.ln() / ln10
        else:
            r = (d.ln() * Decimal(float(y[i]))).exp()
        out[i] = float(r)  # float(Decimal) rounds to nearest
    return out


def test_host_build_is_correctly_rounded():
    x_exp, x_log, x_pow, y_pow = _samples()
    for fn, x, y in ((EXP, x_exp, None), (LOG10, x_log, None), (POW, x_pow, y_pow)):
        got = _host(fn, x, y)
        want = _exact(fn, x, y)
        assert np.array_equal(got, want), (fn, int(np.sum(got != want)))


def test_agrees_with_glibc_except_where_glibc_misrounds():
    x_exp, x_log, x_pow, y_pow = _samples(seed=12, n=2000)
    got = _host(POW, x_pow, y_pow)
    libc = np.array([math.pow(a, b) for a, b in zip(x_pow, y_pow)])
    diff = np.nonzero(got != libc)[0]
    assert len(diff) <= 0.005 * len(got)
    exact = _exact(POW, x_pow[diff], y_pow[diff])
    assert np.array_equal(got[diff], exact)
    got = _host(EXP, x_exp)
    libc = np.array([math.exp(v) for v in x_exp])
    assert np.mean(got == libc) >= 0.995


def test_agrees_with_the_oracles_quad_precision_functions():
    """Two independent correctly rounded implementations (this library's
    double-double code, the oracle's libquadmath evaluation) agree on every
    sample."""
    import oracle
    from micm_b200 import synthetic
    if not oracle.restatement_available():
        pytest.skip("oracle not built")
    R = oracle.Restatement(synthetic.readme_mechanism(), 3, correctly_rounded=True)
    x_exp, x_log, x_pow, y_pow = _samples(seed=14, n=20000)
    for fn, x, y in ((EXP, x_exp, None), (LOG10, x_log, None), (POW, x_pow, y_pow)):
        assert np.array_equal(_host(fn, x, y), R.math_eval(fn, x, y)), fn


def test_special_arguments():
    assert list(_host(POW, [2.0, 9.0, -3.0, 0.0, 5.0], [0.5, 0.5, 2.0, 0.25, 0.0])) == [math.sqrt(2.0), 3.0, 9.0, 0.0, 1.0]
    assert list(_host(LOG10, [1.0, 10.0, 1e-300, 1e300])) == [0.0, 1.0, -300.0, 300.0]
    assert _host(EXP, [0.0])[0] == 1.0 and math.isinf(_host(EXP, [1000.0])[0])
    assert np.isnan(_host(POW, [float("nan")], [0.25])[0])


def test_invalid_arguments():
    out = np.zeros(1)
    assert lib().micmb_math_eval(7, out.ctypes.data, None, out.ctypes.data, 1, 0) == -1
    assert lib().micmb_math_eval(POW, out.ctypes.data, None, out.ctypes.data, 1, 0) == -1


@pytest.mark.gpu
def test_device_build_equals_host_build(cuda_device):
    import torch
    x_exp, x_log, x_pow, y_pow = _samples(seed=13, n=20000)
    for fn, x, y in ((EXP, x_exp, None), (LOG10, x_log, None), (POW, x_pow, y_pow)):
        xd = torch.from_numpy(x).cuda()
        yd = None if y is None else torch.from_numpy(y).cuda()
        od = torch.empty_like(xd)
        check(lib().micmb_math_eval(fn, xd.data_ptr(), None if yd is None else yd.data_ptr(), od.data_ptr(),
                                    len(x), 1))
        assert np.array_equal(od.cpu().numpy(), _host(fn, x, y)), fn
