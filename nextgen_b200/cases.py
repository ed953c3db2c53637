"""Canonical periodic-box cases: Taylor-Green vortex and decaying isotropic
turbulence initial states, with the solver parameters they run with.

All fields are evaluated in the caller's (lattice) cell order.
"""
import numpy as np

from .cgx import Params


def tgv_params(Ma=0.1, Re=1600.0, gamma=1.4, Pr=0.71, U0=1.0, rho0=1.0, T0=1.0, L=1.0,
               cfl=0.8, sgs="vreman"):
    """Parameters of the Taylor-Green case: P_REF = rho0 U0^2/(gamma Ma^2),
    R = P_REF/(rho0 T0), MU_REF = rho0 U0 L / Re."""
    p0 = rho0 * U0 * U0 / (gamma * Ma * Ma)
    prm = Params()
    prm.gamma = gamma
    prm.p_ref = p0
    prm.rho_ref = rho0
    prm.T_ref = T0
    prm.mu_ref = rho0 * U0 * L / Re
    prm.Pr_lam = Pr
    prm.sgs_model = 1 if sgs == "vreman" else 0
    prm.dt_mode = 1
    prm.dt_data[0] = cfl
    return prm


def tgv_state(x_cv, prm, U0=1.0):
    """Taylor-Green vortex: u = U0 sin x cos y cos z, v = -U0 cos x sin y cos z,
    w = 0, p = p0 + rho0 U0^2/16 (cos 2x + cos 2y)(cos 2z + 2), uniform T0."""
    x, y, z = x_cv[:, 0], x_cv[:, 1], x_cv[:, 2]
    u = np.empty((len(x), 3))
    u[:, 0] = U0 * np.sin(x) * np.cos(y) * np.cos(z)
    u[:, 1] = -U0 * np.cos(x) * np.sin(y) * np.cos(z)
    u[:, 2] = 0.0
    p = prm.p_ref + prm.rho_ref * U0 * U0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    R = prm.p_ref / prm.rho_ref / prm.T_ref
    rho = p / (R * prm.T_ref)
    return np.ascontiguousarray(rho), np.ascontiguousarray(u), np.ascontiguousarray(p)


def hit_params(Mt=0.3, gamma=1.4, mu=1.0e-3, Pr=0.7, cfl=0.8):
    """Decaying isotropic turbulence: uniform rho = 1, sound speed 1 (p = 1/gamma)."""
    prm = Params()
    prm.gamma = gamma
    prm.rho_ref = 1.0
    prm.T_ref = 1.0
    prm.p_ref = 1.0 / gamma
    prm.mu_ref = mu
    prm.Pr_lam = Pr
    prm.sgs_model = 1
    prm.dt_mode = 1
    prm.dt_data[0] = cfl
    return prm


def solenoidal_lattice_field(n, k0=4.0, seed=4321):
    """Random solenoidal velocity on an n^3 lattice of [0, 2pi)^3 with energy
    spectrum E(k) ~ k^4 exp(-2 (k/k0)^2): random-phase Fourier modes projected
    onto the plane normal to k.  Returns [n^3, 3] in lattice order (i fastest),
    normalised to unit rms of |u|."""
    rng = np.random.default_rng(seed)
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    kz, ky, kx = np.meshgrid(k1, k1, k1, indexing="ij")  # arrays indexed [k][j][i]
    kk = np.sqrt(kx * kx + ky * ky + kz * kz)
    kk_safe = np.where(kk == 0, 1.0, kk)
    amp = np.sqrt(kk_safe ** 4 * np.exp(-2.0 * (kk_safe / k0) ** 2) / (4 * np.pi * kk_safe ** 2))
    amp[kk == 0] = 0.0
    amp[kk > n / 2 - 1] = 0.0
    uh = (rng.standard_normal((3,) + kk.shape) + 1j * rng.standard_normal((3,) + kk.shape)) * amp
    kvec = np.stack([kx, ky, kz]) / kk_safe
    kdotu = (kvec * uh).sum(0)
    uh = uh - kvec * kdotu  # solenoidal projection
    u = np.stack([np.real(np.fft.ifftn(uh[c])) for c in range(3)], axis=-1)  # [k][j][i][3]
    u = u.reshape(-1, 3)
    u /= np.sqrt((u * u).sum(1).mean())
    return np.ascontiguousarray(u)


def hit_state(n, prm, Mt=0.3, k0=4.0, seed=4321):
    """Solenoidal field of solenoidal_lattice_field() scaled to turbulent Mach
    number Mt = sqrt(<u.u>)/c, uniform rho and T; one value per lattice cell."""
    c0 = np.sqrt(prm.gamma * prm.p_ref / prm.rho_ref)
    u = solenoidal_lattice_field(n, k0=k0, seed=seed) * (Mt * c0)
    ncv = n ** 3
    rho = np.full(ncv, prm.rho_ref)
    p = np.full(ncv, prm.p_ref)
    return rho, u, p
