"""The adjoint of the 2-D warm-bubble workload at its full size: 512 x 256
cells on 20 km x 10 km, WENO5 + HLLC + VIC 3x3, 200 RK3 steps at CFL 0.8 with
checkpoints every 20 steps, J = domain-integrated kinetic energy at the final
time.  dJ/dtheta'(x, z) from the hand-written adjoint (through
torch.autograd and the checkpointed rollout) is checked against FP64 central
differences of the forward path along 8 seeded random directions,
Richardson-extrapolated ((4 D(eps/2) - D(eps)) / 3, eps = 1e-3 K).
Bound: 1e-6 relative, the target for the gradients.

A weak seeded flow (0.3 m/s) is added to the bubble at rest: a resting,
horizontally uniform pressure puts every x2 face exactly on the HLLC contact
switch, where the one-sided derivatives differ and a finite difference is not
a derivative.  With SNAPB_PARITY_REPORT set, the per-direction errors and the
timings are appended there as one JSON line.
"""
import json
import os

import numpy as np
import pytest

from snapy_linfel_b200 import problems

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

NDIR = 8
TOL = 1e-6


def test_warm_bubble_512x256_200_steps_gradient_vs_finite_differences():
    from snapy_linfel_b200 import adjoint as A

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    opts, w, _ = problems.adjoint_bubble()
    cfg = opts.hydro
    assert (cfg.nx2, cfg.nx1) == (512, 256)
    rng = np.random.default_rng(4)
    k3, k2, k1 = np.meshgrid(*[np.arange(n) / n for n in cfg.shape[1:]], indexing="ij")
    w[1] = 0.3 * np.sin(2 * np.pi * (k1 + 2 * k2) + rng.uniform(0, 6.28))
    w[2] = 0.3 * np.cos(2 * np.pi * (2 * k1 - k2) + rng.uniform(0, 6.28))
    base = torch.from_numpy(w).cuda()
    rd, cp = cfg.rgas, cfg.rgas * cfg.gammad / (cfg.gammad - 1.0)
    p = base[4]
    temp0 = p / (rd * base[0])
    it = cfg.interior()

    def state(dth):
        wt = torch.cat([(p / (rd * (temp0 + dth * (p / 1.0e5) ** (rd / cp))))[None], base[1:]])
        return A.initial_state(cfg, wt)

    dth0 = torch.zeros(cfg.shape[1:], dtype=torch.float64, device="cuda")
    dts = A.cfl_steps(opts, state(dth0).detach(), nsteps=200)
    runner = A.StepRunner(opts, device="cuda")

    def J(dth):
        uT, _ = A.rollout(opts, state(dth), None, dts, checkpoint_every=20, runner=runner)
        return (0.5 * (uT[1] ** 2 + uT[2] ** 2 + uT[3] ** 2) / uT[0])[it].sum()

    x = dth0.clone().requires_grad_(True)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    j = J(x)
    e1.record()
    (grad,) = torch.autograd.grad(j, x)
    e2.record()
    torch.cuda.synchronize()
    assert bool(torch.isfinite(grad).all())
    assert float(grad.abs().max()) > 0.0
    mask = torch.zeros_like(dth0)
    mask[it] = 1.0
    gen = torch.Generator(device="cuda").manual_seed(2024)
    errs = []
    eps = 1e-3
    with torch.no_grad():
        for _ in range(NDIR):
            v = torch.randn(dth0.shape, generator=gen, device="cuda", dtype=torch.float64) * mask
            f = lambda t: float(J(dth0 + t * v))  # noqa: E731
            d1 = (f(eps) - f(-eps)) / (2 * eps)
            d2 = (f(eps / 2) - f(-eps / 2)) / eps
            fd = (4 * d2 - d1) / 3
            ad = float((grad * v).sum())
            errs.append(abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
    path = os.environ.get("SNAPB_PARITY_REPORT")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps({"case": "adjoint_bubble_512x256_200steps", "rel_err": errs,
                                 "forward_ms": e0.elapsed_time(e1),
                                 "backward_ms": e1.elapsed_time(e2)}) + "\n")
    print(f"adjoint 512x256 x 200 steps: {NDIR} directions, max rel err {max(errs):.2e}, "
          f"backward/forward {e1.elapsed_time(e2) / e0.elapsed_time(e1):.2f}")
    assert max(errs) < TOL, errs
