"""The parity tests' error norms fail on a NaN or Inf in any field (planted
on the CPU), and agree with the plain formulas on finite data."""
import numpy as np
import pytest

from errnorm import assert_finite, field_relerr, rel_l1_linf, relerr, state_err


def _pair():
    rng = np.random.default_rng(0)
    b = rng.random((5, 4, 6, 7)) + 1.0
    a = b + 1e-14 * rng.standard_normal(b.shape)
    return a, b


@pytest.mark.parametrize("field", [0, 2, 4])
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_planted_nonfinite_fails(field, bad):
    a, b = _pair()
    a[field, 1, 2, 3] = bad
    for f in (relerr, lambda x, y: state_err(x, y, y), field_relerr, rel_l1_linf):
        with pytest.raises(AssertionError):
            f(a, b)
    with pytest.raises(AssertionError):
        assert_finite(a)


def test_finite_values_match_plain_formulas():
    a, b = _pair()
    want = max(np.abs(a[v] - b[v]).max() / np.abs(b[v]).max() for v in range(5))
    assert relerr(a, b) == pytest.approx(want, rel=0, abs=0)
    assert relerr(a, b) < 1e-13
    assert state_err(a, b, b) < 1e-13
