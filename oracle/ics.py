"""Initial conditions evaluated at GLL points (test infrastructure only).

OseenVortex and AcousticPulse restate src/EulerIC.hpp:203-237 and :238-300;
the Taylor-Green "Given" expression restates runs/TaylorGreen/tg.ic with the
Mach number as a parameter; the isentropic vortex and the shallow-water
Gaussian bump have no built-in counterpart in the reference (they would be
"Given" parser expressions there) and follow their textbook definitions.
All return conserved variables, shape (nfields, npoints).
"""
from __future__ import annotations

import numpy as np


def oseen_vortex(x, y, x0, y0, radius, amp, Ma, gamma=1.4):
    r2 = ((x - x0) ** 2 + (y - y0) ** 2) / radius / radius
    rho = (1.0 - 0.5 * (gamma - 1.0) * Ma * Ma * np.exp(1.0 - r2)) ** (1.0 / (gamma - 1.0))
    u = -amp * (y - y0) / radius * np.exp(0.5 * (1.0 - r2))
    v = amp * (x - x0) / radius * np.exp(0.5 * (1.0 - r2))
    t = rho ** (gamma - 1.0)
    E = amp * amp * rho * t / (gamma * (gamma - 1) * Ma * Ma) + 0.5 * rho * (u * u + v * v)
    return rho, rho * u, rho * v, E


def vortex_ic(x, y, vortices, gamma=1.4, nf=4):
    """DGM "Vortex" IC: superposed Oseen vortices added to a zero field
    (src/Euler.cpp:921-937)."""
    U = np.zeros((nf, x.size))
    for (x0, y0, rad, amp, Ma) in vortices:
        r, ru, rv, E = oseen_vortex(x, y, x0, y0, rad, amp, Ma, gamma)
        U[0] += r
        U[1] += ru
        U[2] += rv
        U[nf - 1] += E
    return U


def acoustic_pulse(x, amp, x0, sigma, gamma=1.4):
    gm1 = gamma - 1.0
    Ma = 1.0
    r = np.ones_like(x)
    u = np.zeros_like(x)
    e = 1.0 / (gamma * gm1 * Ma * Ma)
    c = np.sqrt(gamma * gm1 * e)
    c3 = np.exp(-0.5 * ((x - x0) / sigma) ** 2.0)
    rp = (0.5 * c3) / (c * c)
    up = c3 * 0.5 / (1.0 * c)
    pp = 0.5 * c3
    ep = (pp / gm1 - rp * e) / 1.0
    r = r + amp * rp
    u = u + amp * up
    e = e + amp * ep
    U = np.zeros((5, x.size))
    U[0] = r
    U[1] = r * u
    U[4] = r * e + 0.5 * r * (u * u)
    return U


def isentropic_vortex(x, y, beta=5.0, x0=0.0, y0=0.0, gamma=1.4,
                      rho_inf=1.0, u_inf=1.0, v_inf=0.0, p_inf=1.0, period=None):
    """Shu's isentropic vortex (strength beta) on a free stream."""
    dx, dy = x - x0, y - y0
    if period is not None:
        dx = (dx + 0.5 * period[0]) % period[0] - 0.5 * period[0]
        dy = (dy + 0.5 * period[1]) % period[1] - 0.5 * period[1]
    r2 = dx * dx + dy * dy
    f = beta / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2))
    u = u_inf - dy * f
    v = v_inf + dx * f
    T = p_inf / rho_inf - (gamma - 1.0) * beta * beta / (8.0 * gamma * np.pi ** 2) * np.exp(1.0 - r2)
    s = p_inf / rho_inf ** gamma
    rho = (T / s) ** (1.0 / (gamma - 1.0))
    p = rho * T
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return np.stack([rho, rho * u, rho * v, E])


def taylor_green(x, y, z, Ma=0.1, gamma=1.4, rho0=1.0, U0=1.0):
    """3-D Taylor-Green vortex on [0, 2pi]^3 (same form as tg.ic with
    p0 = rho0 U0^2 / (gamma Ma^2))."""
    p0 = rho0 * U0 * U0 / (gamma * Ma * Ma)
    u = U0 * np.sin(x) * np.cos(y) * np.cos(z)
    v = -U0 * np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(x)
    p = p0 + rho0 * U0 * U0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    rho = np.full_like(x, rho0)
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, E])


def gaussian_bump(x, y, a=0.3, w=0.5, g=9.81, x0=0.0, y0=0.0):
    """Shallow water at rest with h = 1 + a exp(-r^2/w^2), geopotential form."""
    r2 = (x - x0) ** 2 + (y - y0) ** 2
    h = 1.0 + a * np.exp(-r2 / (w * w))
    return np.stack([g * h, np.zeros_like(x), np.zeros_like(x)])
