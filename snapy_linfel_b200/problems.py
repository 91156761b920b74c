"""Synthetic initial states for the five benchmark configurations.

Each function returns ``(MeshBlockOptions, w, r)``: the block options, the
primitive state ``hydro_w`` of shape [nvar, nc3, nc2, nc1] (ghost cells
included, before boundary fills) and the passive-scalar mixing ratios
``scalar_r`` (or None).  Seeds are fixed; the inputs stand in for the data of
the reference's examples (shock tube, Straka density current, warm bubbles)
with their shapes, sizes and value distributions.
"""
from __future__ import annotations

import numpy as np

from .config import Integration, MeshBlockOptions, make_config


def _centers(lo, hi, nx, ng):
    """Cell-centre coordinates including ghosts (uniform Cartesian)."""
    if nx <= 1:
        return np.array([0.5 * (lo + hi)])
    dx = (hi - lo) / nx
    return lo + (np.arange(nx + 2 * ng) - ng + 0.5) * dx


def _grids(cfg):
    x1 = _centers(cfg.x1min, cfg.x1max, cfg.nx1, cfg.nghost)
    x2 = _centers(cfg.x2min, cfg.x2max, cfg.nx2, cfg.nghost)
    x3 = _centers(cfg.x3min, cfg.x3max, cfg.nx3, cfg.nghost)
    X3, X2, X1 = np.meshgrid(x3, x2, x1, indexing="ij")
    return X1, X2, X3


def sod(nx1=1024):
    """1-D Sod shock tube on x1 in [0, 1] (1024 cells, WENO5 + HLLC, outflow)."""
    cfg = make_config(nx1=nx1, x1=(0.0, 1.0), gammad=1.4, recon1="weno5", shock1=True,
                      recon23="weno5", shock23=True, riemann="hllc",
                      bc=("outflow",) * 6)
    X1, _, _ = _grids(cfg)
    w = np.zeros(cfg.shape)
    w[0] = np.where(X1 < 0.5, 1.0, 0.125)
    w[4] = np.where(X1 < 0.5, 1.0, 0.1)
    opts = MeshBlockOptions(cfg, Integration(cfl=0.9, tlim=0.2))
    return opts, w, None


def _isentropic(X1, p0, theta0, grav, rd, cp):
    temp = theta0 - grav * X1 / cp
    p = p0 * (temp / theta0) ** (cp / rd)
    return temp, p


def straka(nx2=1024, nx1=128, implicit_scheme=1, riemann="lmars"):
    """2-D Straka cold-bubble density current (1024 x 128 cells, WENO5 + LMARS).

    x2 in [-25.6, 25.6] km (bubble centred at x2 = 0), x1 in [0, 6.4] km,
    R = 287, cp = 1004, g = 9.81, T' = -15 K (cos(pi L) + 1)/2 for L <= 1 as
    the reference example perturbs the temperature; nu = kappa = 75.
    """
    rd, cp, g = 287.0, 1004.0, 9.81
    cfg = make_config(nx1=nx1, nx2=nx2, x1=(0.0, 6.4e3), x2=(-25.6e3, 25.6e3),
                      gammad=cp / (cp - rd), rgas=rd, recon1="weno5", recon23="weno5",
                      riemann=riemann, implicit_scheme=implicit_scheme, grav=(-g, 0.0, 0.0),
                      nu_iso=75.0, kappa_iso=75.0, bc=("reflecting",) * 6)
    X1, X2, _ = _grids(cfg)
    temp, p = _isentropic(X1, 1.0e5, 300.0, g, rd, cp)
    L = np.sqrt(((X2 - 0.0) / 4.0e3) ** 2 + ((X1 - 3.0e3) / 2.0e3) ** 2)
    temp = temp + np.where(L <= 1, -15.0 * (np.cos(L * np.pi) + 1.0) / 2.0, 0.0)
    w = np.zeros(cfg.shape)
    w[0] = p / (rd * temp)
    w[4] = p
    return MeshBlockOptions(cfg, Integration(cfl=0.9, tlim=900.0)), w, None


def warm_bubble_3d(nx3, nx2, nx1, amp, radius, center, dx=100.0, dz=100.0,
                   riemann="lmars", implicit_scheme=1):
    """One 3-D dry warm-bubble member of the 48-member ensemble, doubly periodic."""
    rd, cp, g = 287.0, 1004.0, 9.81
    cfg = make_config(nx1=nx1, nx2=nx2, nx3=nx3, x1=(0.0, nx1 * dz), x2=(0.0, nx2 * dx),
                      x3=(0.0, nx3 * dx), gammad=cp / (cp - rd), rgas=rd, recon1="weno5",
                      recon23="weno5", riemann=riemann, implicit_scheme=implicit_scheme,
                      grav=(-g, 0.0, 0.0),
                      bc=("reflecting", "reflecting", "periodic", "periodic", "periodic",
                          "periodic"))
    X1, X2, X3 = _grids(cfg)
    temp, p = _isentropic(X1, 1.0e5, 300.0, g, rd, cp)
    c3, c2, c1 = center
    L = np.sqrt(((X3 - c3) ** 2 + (X2 - c2) ** 2 + (X1 - c1) ** 2)) / radius
    dth = np.where(L <= 1, amp * (np.cos(L * np.pi) + 1.0) / 2.0, 0.0)
    temp = temp + dth * (p / 1.0e5) ** (rd / cp)
    w = np.zeros(cfg.shape)
    w[0] = p / (rd * temp)
    w[4] = p
    return MeshBlockOptions(cfg, Integration(cfl=0.8, nlim=100)), w, None


def ensemble(n=48, seed=2024, horiz=(64, 96, 128), vert=(64, 128)):
    """48 uneven 3-D warm-bubble members drawn from a seed (config 3)."""
    rng = np.random.default_rng(seed)
    members = []
    for _ in range(n):
        nh = int(rng.choice(horiz))
        nv = int(rng.choice(vert))
        amp = rng.uniform(0.5, 3.0)
        rad = rng.uniform(1.0e3, 2.0e3)
        cx = rng.uniform(0.0, nh * 100.0)
        cy = rng.uniform(0.0, nh * 100.0)
        cz = rng.uniform(0.0, 0.5 * nv * 100.0)
        members.append(dict(nx3=nh, nx2=nh, nx1=nv, amp=amp, radius=rad,
                            center=(cy, cx, cz)))
    return members


def ensemble_members(n=48, seed=2024, horiz=(64, 96, 128), vert=(64, 128),
                     riemann="lmars", implicit_scheme=1):
    """(options, w, r) of every member of the seeded ensemble."""
    out = []
    for m in ensemble(n=n, seed=seed, horiz=horiz, vert=vert):
        out.append(warm_bubble_3d(riemann=riemann, implicit_scheme=implicit_scheme, **m))
    return out


def gaussian_random_field(shape, dx, corr, sigma, seed):
    """Seeded Gaussian random field by FFT filtering of white noise."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(shape)
    ks = [np.fft.fftfreq(n, d=d) for n, d in zip(shape, dx)]
    K = np.meshgrid(*ks, indexing="ij")
    k2 = sum(k * k for k in K)
    filt = np.exp(-0.5 * (2 * np.pi) ** 2 * k2 * corr ** 2)
    f = np.real(np.fft.ifftn(np.fft.fftn(noise) * filt))
    f -= f.mean()
    return sigma * f / max(f.std(), 1e-300)


def adjoint_bubble(nx2=512, nx1=256, seed=7):
    """2-D warm bubble of the adjoint workload (512 x 256 cells, 20 km x 10 km, HLLC)."""
    rd, cp, g = 287.0, 1004.0, 9.81
    cfg = make_config(nx1=nx1, nx2=nx2, x1=(0.0, 10.0e3), x2=(0.0, 20.0e3),
                      gammad=cp / (cp - rd), rgas=rd, recon1="weno5", recon23="weno5",
                      riemann="hllc", implicit_scheme=1, grav=(-g, 0.0, 0.0),
                      bc=("reflecting",) * 6)
    X1, X2, _ = _grids(cfg)
    temp, p = _isentropic(X1, 1.0e5, 300.0, g, rd, cp)
    L = np.sqrt((X2 - 10.0e3) ** 2 + (X1 - 2.0e3) ** 2) / 2.0e3
    dth = np.where(L <= 1, 2.0 * (np.cos(L * np.pi) + 1.0) / 2.0, 0.0)
    grf = gaussian_random_field(X1.shape[1:], (cfg.x2max / nx2, cfg.x1max / nx1), 500.0,
                                0.1, seed)
    dth = dth + grf[None]
    temp = temp + dth * (p / 1.0e5) ** (rd / cp)
    w = np.zeros(cfg.shape)
    w[0] = p / (rd * temp)
    w[4] = p
    return MeshBlockOptions(cfg, Integration(cfl=0.8, nlim=200)), w, None


def large_3d(nx3=384, nx2=384, nx1=192, seed=11, nscalar=2, implicit_scheme=1):
    """Large H2-He 3-D domain (384 x 384 x 192 cells, WENO5 + Roe, two tracers).

    R = 3777, cp = 13000, g = 24.8; dry-adiabatic below 2/3 of the height,
    isothermal above; T0 = 166 K and p0 = 1e5 Pa at the bottom (chosen here,
    the configuration does not fix them); white-noise theta' with sigma
    0.01 K; two smooth seeded tracers in [0, 1]; WENO5 + Roe.
    """
    rd, cp, g = 3777.0, 13000.0, 24.8
    dz, dx = 100.0, 200.0
    cfg = make_config(nx1=nx1, nx2=nx2, nx3=nx3, x1=(0.0, nx1 * dz), x2=(0.0, nx2 * dx),
                      x3=(0.0, nx3 * dx), gammad=cp / (cp - rd), rgas=rd, recon1="weno5",
                      recon23="weno5", riemann="roe", implicit_scheme=implicit_scheme,
                      grav=(-g, 0.0, 0.0), nscalar=nscalar, scalar_recon="weno5",
                      bc=("reflecting", "reflecting", "periodic", "periodic", "periodic",
                          "periodic"))
    x1 = _centers(cfg.x1min, cfg.x1max, nx1, cfg.nghost)
    zt = 2.0 / 3.0 * nx1 * dz
    T0, p0 = 166.0, 1.0e5
    Tt = T0 - g * zt / cp
    pt = p0 * (Tt / T0) ** (cp / rd)
    temp1 = np.where(x1 < zt, T0 - g * x1 / cp, Tt)
    p1 = np.where(x1 < zt, p0 * (np.maximum(T0 - g * x1 / cp, 1.0) / T0) ** (cp / rd),
                  pt * np.exp(-g * (x1 - zt) / (rd * Tt)))
    shape = (cfg.nc3, cfg.nc2, cfg.nc1)
    rng = np.random.default_rng(seed)
    dth = 0.01 * rng.standard_normal(shape)
    temp = temp1[None, None, :] + dth * (p1[None, None, :] / p0) ** (rd / cp)
    w = np.zeros(cfg.shape)
    w[0] = p1[None, None, :] / (rd * temp)
    w[4] = np.broadcast_to(p1[None, None, :], shape)
    r = None
    if nscalar:
        r = np.empty(cfg.scalar_shape)
        for n in range(nscalar):
            f = gaussian_random_field(shape, (dx, dx, dz), 2000.0, 1.0, seed + 1 + n)
            r[n] = (f - f.min()) / (f.max() - f.min())
    return MeshBlockOptions(cfg, Integration(cfl=0.8, nlim=50)), w, r
