"""Error norms for the parity tests that fail on any non-finite value.

Every reduction here first asserts that both operands are finite, and the
per-field errors are reduced with numpy (which propagates NaN) rather than
Python's max() (whose comparisons drop a NaN unless it is the first item).
A NaN or Inf anywhere in a GPU result therefore fails the assertion that
uses it, whichever field it lands in.
"""
import numpy as np


def to_np(a):
    """numpy view of an array or a torch tensor (copied to the host)"""
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    return np.asarray(a)


def assert_finite(*arrays, what="result"):
    for k, a in enumerate(arrays):
        a = to_np(a)
        bad = ~np.isfinite(a)
        if bad.any():
            idx = np.argwhere(bad)[0]
            raise AssertionError(f"{what}[{k}] has {int(bad.sum())} non-finite values, "
                                 f"first at {tuple(int(i) for i in idx)}: {a[tuple(idx)]}")


def field_relerr(a, b):
    """per-field max|a - b| / max|b| (first axis = field); finite inputs only"""
    a, b = to_np(a), to_np(b)
    assert_finite(a, b, what="field_relerr input")
    if a.ndim <= 1:
        return np.array([np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)])
    d = np.abs(a - b).reshape(a.shape[0], -1).max(axis=1)
    s = np.maximum(np.abs(b).reshape(b.shape[0], -1).max(axis=1), 1e-300)
    return d / s


def relerr(a, b):
    """largest per-field relative max error (fails on NaN/Inf)"""
    return float(np.max(field_relerr(a, b)))


def state_scale(u):
    """per-variable magnitude of a conserved state [nvar, ...]: density,
    sqrt(rho E) (or the largest momentum) for the momenta, total energy"""
    u = to_np(u)
    rho = np.max(np.abs(u[0]))
    en = np.max(np.abs(u[4]))
    mom = max(np.sqrt(rho * en), np.max(np.abs(u[1:4])))
    return np.array([rho, mom, mom, mom, en])


def state_errs(a, b, u):
    """per-variable max|a_v - b_v| / scale_v(u)"""
    a, b = to_np(a), to_np(b)
    assert_finite(a, b, what="state_err input")
    sc = state_scale(u)
    d = np.abs(a - b).reshape(a.shape[0], -1).max(axis=1)
    return d / sc[: a.shape[0]]


def state_err(a, b, u):
    """max over variables of max|a_v - b_v| / scale_v(u) (fails on NaN/Inf)"""
    return float(np.max(state_errs(a, b, u)))


def rel_l1_linf(a, b):
    """per-field (rel L1, rel L-inf) = sum|a-b|/sum|b|, max|a-b|/max|b|"""
    a, b = to_np(a), to_np(b)
    assert_finite(a, b, what="rel_l1_linf input")
    out = []
    for v in range(a.shape[0]):
        x, y = a[v], b[v]
        out.append((float(np.abs(x - y).sum() / max(np.abs(y).sum(), 1e-300)),
                    float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300))))
    return out
