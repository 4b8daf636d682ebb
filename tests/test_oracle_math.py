"""The oracle's elementary functions against 50-digit decimal references."""
import ctypes
import decimal
import math

import numpy as np
import pytest

decimal.getcontext().prec = 50
D = decimal.Decimal
PI = D("3.14159265358979323846264338327950288419716939937510582097494459")


def _ulp_err(got, exact):
    return abs(got - float(exact)) / math.ulp(float(exact)) if float(exact) != 0 else abs(got)


def _dsin(x):
    s, t, n = D(0), x, 1
    while abs(t) > D(10) ** -45:
        s += t
        t = -t * x * x / ((n + 1) * (n + 2))
        n += 2
    return s


def _dcos(x):
    s, t, n = D(0), D(1), 0
    while abs(t) > D(10) ** -45:
        s += t
        t = -t * x * x / ((n + 1) * (n + 2))
        n += 2
    return s


def test_pow_faithful(oracle_lib):
    L = oracle_lib.lib()
    rng = np.random.default_rng(0)
    worst = 0.0
    for x in 10 ** rng.uniform(-2.5, 2.5, 400):
        for y in (4.2, 0.2, 0.25, 3.0 * 1.4):
            got = L.bes_oracle_pow(float(x), y)
            worst = max(worst, _ulp_err(got, (D(float(x)).ln() * D(y)).exp()))
    assert worst <= 1.0


def test_pow_recip_faithful(oracle_lib):
    """(1/x)^y as exp(-y log x), the Keller-Miksis gas-pressure term's form."""
    L = oracle_lib.lib()
    rng = np.random.default_rng(3)
    worst = 0.0
    for x in 10 ** rng.uniform(-2.5, 2.5, 400):
        for y in (4.2, 3.0 * 1.4, 1.0, 0.3):
            got = L.bes_oracle_pow_recip(float(x), y)
            worst = max(worst, _ulp_err(got, (-(D(float(x)).ln() * D(y))).exp()))
    assert worst <= 1.0


def test_exp_log_faithful(oracle_lib):
    L = oracle_lib.lib()
    rng = np.random.default_rng(1)
    for x in rng.uniform(-700, 700, 300):
        assert _ulp_err(L.bes_oracle_exp(float(x)), D(float(x)).exp()) <= 1.0
    for x in 10 ** rng.uniform(-300, 300, 300):
        assert _ulp_err(L.bes_oracle_log(float(x)), D(float(x)).ln()) <= 1.0


def test_sincospi_and_sincos_faithful(oracle_lib):
    L = oracle_lib.lib()
    rng = np.random.default_rng(2)
    s, c = ctypes.c_double(), ctypes.c_double()
    for x in rng.uniform(-2.0, 4.0, 300):
        L.bes_oracle_sincospi(float(x), ctypes.byref(s), ctypes.byref(c))
        assert _ulp_err(s.value, _dsin(PI * D(float(x)))) <= 1.0
        assert _ulp_err(c.value, _dcos(PI * D(float(x)))) <= 1.0
    for x in rng.uniform(-30.0, 30.0, 300):
        L.bes_oracle_sincos(float(x), ctypes.byref(s), ctypes.byref(c))
        assert _ulp_err(s.value, _dsin(D(float(x)))) <= 1.0
        assert _ulp_err(c.value, _dcos(D(float(x)))) <= 1.0


def test_special_values(oracle_lib):
    L = oracle_lib.lib()
    assert L.bes_oracle_pow(0.0, 4.2) == 0.0
    assert math.isinf(L.bes_oracle_pow(0.0, -4.2))
    assert L.bes_oracle_pow(-2.0, 3.0) == -8.0
    assert math.isnan(L.bes_oracle_pow(-2.0, 0.5))
    assert L.bes_oracle_pow(7.0, 0.0) == 1.0
    assert math.isinf(L.bes_oracle_exp(710.0)) and L.bes_oracle_exp(-800.0) == 0.0
    s, c = ctypes.c_double(), ctypes.c_double()
    L.bes_oracle_sincos(0.0, ctypes.byref(s), ctypes.byref(c))
    assert s.value == 0.0 and c.value == 1.0
    L.bes_oracle_sincospi(0.5, ctypes.byref(s), ctypes.byref(c))
    assert s.value == 1.0 and c.value == 0.0
