"""The kernels' shared-reciprocal division (csrc/fct_div.cuh) is bit-identical to the
native IEEE division (fct_div_check): random operands over wide exponent ranges, exactly
representable quotients, quotients next to rounding midpoints, and the special operands
that take the native fallback."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _check(torch, x, y):
    from fesom_jax_b200 import _lib
    L = _lib.lib()
    L.fct_div_check.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    L.fct_div_check.restype = C.c_int
    x, y = x.contiguous(), y.contiguous()
    res = torch.tensor([0, -1], dtype=torch.int64, device=x.device)   # {count, UINT64_MAX}
    s = torch.cuda.current_stream().cuda_stream
    _lib.check(L.fct_div_check(x.data_ptr(), y.data_ptr(), x.numel(), res.data_ptr(),
                               C.c_void_p(s)))
    count, first = res.cpu().tolist()
    return count, first


def _rand(torch, g, n, emin, emax):
    mant = 1.0 + torch.rand(n, generator=g, device="cuda", dtype=torch.float64)
    exp = torch.randint(emin, emax + 1, (n,), generator=g, device="cuda")
    sign = torch.where(torch.rand(n, generator=g, device="cuda") < 0.5, -1.0, 1.0)
    return torch.ldexp(mant * sign.double(), exp)


@pytest.mark.parametrize("emin,emax", [(-60, 60), (-500, 500), (-1074, 1023)])
def test_random_operands(torch, emin, emax):
    g = torch.Generator(device="cuda")
    g.manual_seed(1000 + emax)
    for _ in range(4):
        n = 1 << 24
        x, y = _rand(torch, g, n, emin, emax), _rand(torch, g, n, emin, emax)
        count, first = _check(torch, x, y)
        assert count == 0, (count, first, x[first].item(), y[first].item())


def test_exact_and_midpoint_quotients(torch):
    """x = q * y exactly (short mantissas), and x = RN(q * y) +- a few ulp for random q, y:
    quotients that are representable or sit next to a rounding midpoint."""
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    n = 1 << 24
    # 26-bit mantissas: products are exact
    q = torch.ldexp(torch.randint(1 << 25, 1 << 26, (n,), generator=g, device="cuda").double(),
                    torch.randint(-60, 40, (n,), generator=g, device="cuda"))
    y = torch.ldexp(torch.randint(1 << 25, 1 << 26, (n,), generator=g, device="cuda").double(),
                    torch.randint(-60, 40, (n,), generator=g, device="cuda"))
    count, first = _check(torch, q * y, y)
    assert count == 0, (count, first)
    q, y = _rand(torch, g, n, -30, 30), _rand(torch, g, n, -30, 30)
    x = q * y
    for k in (-2, -1, 1, 2):
        xi = x.view(torch.int64) + k
        count, first = _check(torch, xi.view(torch.float64), y)
        assert count == 0, (k, count, first)


def test_special_operands(torch):
    vals = [0.0, -0.0, 1.0, -1.0, 3.0, 6.0, np.inf, -np.inf, np.nan, 5e-324, -5e-324,
            2.2250738585072014e-308, 1.7976931348623157e308, 1e-300, 1e300, 2.0 ** -500,
            2.0 ** 500, 2.0 ** -501, 2.0 ** 501, 1e-16, 0.1, 1.0 / 3.0]
    a = np.array(vals)
    x, y = np.meshgrid(a, a)
    count, first = _check(torch, torch.from_numpy(x.ravel()).cuda(),
                          torch.from_numpy(y.ravel()).cuda())
    assert count == 0, (count, first, x.ravel()[first], y.ravel()[first])
