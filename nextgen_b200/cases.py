"""Canonical periodic-box cases: Taylor-Green vortex, decaying isotropic
turbulence and the inviscid (isentropic) vortex, with the solver parameters
they run with.

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


def vortex_params(gamma=1.4, cfl=0.8):
    """The reference's inviscid vortex harness (IdealGasEulerSolver,
    src/charles/charles_ig.cpp:170-290): rho_inf = p_inf = 1, no viscosity and
    no SGS model, CFL time step."""
    prm = Params()
    prm.gamma = gamma
    prm.rho_ref = 1.0
    prm.p_ref = 1.0
    prm.T_ref = 1.0
    prm.mu_ref = 0.0
    prm.sgs_model = 0
    prm.dt_mode = 1
    prm.dt_data[0] = cfl
    return prm


def vortex_state(x_cv, prm, t=0.0, u_inf=0.5, Lx=10.0, Ly=10.0 * np.sqrt(3.0) / 2.0, periodic=True,
                 x0=-2.5, y0=-2.5, theta=np.pi / 3.0, e_twopi=0.32, rc=1.0):
    """calcInviscidVortexLocal (src/charles/charles_ig.cpp:88-168): the exact
    isentropic vortex at time t, of circulation parameter e_twopi (0.32, the
    reference's "strong" setting) and radius rc, started at (x0, y0) and
    advected at u_inf along theta.  On a periodic box [-Lx, Lx] x [-Ly, Ly] the
    vortex offset is wrapped into the box.  Defaults are the reference's
    (EULER_UINF 0.5, EULER_LX 10, EULER_LY 10 sqrt(3)/2).  Returns rho, u, p."""
    gamma = prm.gamma
    Ma_inf = u_inf / np.sqrt(gamma * prm.p_ref / prm.rho_ref)
    coeff = 0.5 * e_twopi * e_twopi * (gamma - 1.0) * Ma_inf * Ma_inf
    dx = x_cv[:, 0] - x0 - u_inf * np.cos(theta) * t
    dy = x_cv[:, 1] - y0 - u_inf * np.sin(theta) * t
    if periodic:
        dx = (dx + Lx) % (2.0 * Lx) - Lx
        dy = (dy + Ly) % (2.0 * Ly) - Ly
    f0 = 1.0 - (dx * dx + dy * dy) / (rc * rc)
    rho = prm.rho_ref * (1.0 - coeff * np.exp(f0)) ** (1.0 / (gamma - 1.0))
    u = np.zeros((len(dx), 3))
    u[:, 0] = u_inf * (np.cos(theta) - e_twopi * dy / rc * np.exp(f0 / 2.0))
    u[:, 1] = u_inf * (np.sin(theta) + e_twopi * dx / rc * np.exp(f0 / 2.0))
    p = prm.p_ref * (1.0 - coeff * np.exp(f0)) ** (gamma / (gamma - 1.0))
    return np.ascontiguousarray(rho), np.ascontiguousarray(u), np.ascontiguousarray(p)


def vortex_errors(x_cv, vol_cv, rho, u, rhoE, prm, t, **vortex_kw):
    """The error norms IdealGasEulerSolver::temporalHook reports
    (src/charles/charles_ig.cpp:224-288): volume-weighted L2 and Linf of
    rho - rho_exact, u - u_exact (3) and rhoE - rhoE_exact against the exact
    vortex at time t.  Returns (l2[5], linf[5])."""
    re, ue, pe = vortex_state(x_cv, prm, t=t, **vortex_kw)
    rEe = pe / (prm.gamma - 1.0) + 0.5 * re * (ue * ue).sum(1)
    d = np.column_stack([rho - re, u - ue, rhoE - rEe])
    vol = np.asarray(vol_cv)
    l2 = np.sqrt((vol[:, None] * d * d).sum(0) / vol.sum())
    linf = np.abs(d).max(0)
    return l2, linf
