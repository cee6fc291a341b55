"""Solve requests for the pool: periodic box meshes, initial conditions from
a few parameters, and the CFL step.

A request names its physics, mesh size, order, initial-condition parameters
and end time; ``make_request`` turns it into what ``Pool.add`` takes.  The
initial conditions are the ones the reference would express as "Given"
parser expressions (src/vField.cpp:2896-2975): the isentropic vortex on a
free stream, the 3-D Taylor-Green vortex, and a Gaussian bump of still
shallow water.  The step follows dt = CFL h / ((2p+1) max(|u|+c)), taken
once from the initial state.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import EULER2D, EULER3D, SHALLOW, meshgen

_GAMMA = 1.4


def gll_points(q: int) -> np.ndarray:
    """Gauss-Lobatto-Legendre points on [-1, 1] (q of them)."""
    n = q - 1
    c = np.zeros(n + 1)
    c[-1] = 1.0
    inner = np.polynomial.legendre.legroots(np.polynomial.legendre.legder(c)) if n > 1 else np.array([])
    return np.concatenate(([-1.0], np.sort(np.real(inner)), [1.0]))


def coordinates(mesh) -> tuple:
    """GLL coordinates of a box mesh in Field layout."""
    return meshgen.gll_coordinates(mesh, gll_points(int(mesh.qorder[0])))


def vortex(x, y, beta=5.0, x0=0.0, y0=0.0, period=(10.0, 10.0), gamma=_GAMMA):
    """Isentropic vortex of strength beta on the free stream rho=1, u=1, v=0, p=1."""
    dx = (x - x0 + 0.5 * period[0]) % period[0] - 0.5 * period[0]
    dy = (y - y0 + 0.5 * period[1]) % period[1] - 0.5 * period[1]
    r2 = dx * dx + dy * dy
    f = beta / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2))
    u, v = 1.0 - dy * f, dx * f
    T = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * np.pi ** 2) * np.exp(1.0 - r2)
    rho = T ** (1.0 / (gamma - 1.0))
    p = rho * T
    return np.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)])


def taylor_green(x, y, z, Ma=0.1, gamma=_GAMMA):
    """Taylor-Green vortex on [0, 2pi]^3, rho0 = U0 = 1, p0 = 1/(gamma Ma^2)."""
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    p = 1.0 / (gamma * Ma * Ma) + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0
    return np.stack([np.ones_like(x), u, v, np.zeros_like(x), p / (gamma - 1.0) + 0.5 * (u * u + v * v)])


def bump(x, y, a=0.3, w=0.5, g=9.81):
    """Still water with depth 1 + a exp(-r^2/w^2), geopotential form phi = g h."""
    h = 1.0 + a * np.exp(-(x * x + y * y) / (w * w))
    return np.stack([g * h, np.zeros_like(x), np.zeros_like(x)])


def max_speed(U, physics: int, gamma=_GAMMA) -> float:
    """max(|u| + c) over the points of U (Field layout)."""
    r = U[0]
    if physics == SHALLOW:
        u, v = U[1] / r, U[2] / r
        return float(np.max(np.sqrt(u * u + v * v) + np.sqrt(r)))
    nd = U.shape[0] - 2
    vel2 = sum((U[1 + k] / r) ** 2 for k in range(nd))
    p = (gamma - 1.0) * (U[-1] - 0.5 * r * vel2)
    return float(np.max(np.sqrt(vel2) + np.sqrt(gamma * p / r)))


def cfl_dt(U, h: float, p: int, physics: int, cfl: float = 0.5) -> float:
    return cfl * h / ((2 * p + 1) * max_speed(U, physics))


@dataclasses.dataclass
class Request:
    """One solve: physics, n x n (x n) periodic box, order, IC parameters, end time."""
    physics: int
    n: int
    p: int
    t_end: float
    params: dict = dataclasses.field(default_factory=dict)
    arrival: float = 0.0
    mesh: object = None
    U0: np.ndarray = None
    dt: float = 0.0

    @property
    def dof(self) -> int:
        nf = 3 if self.physics == SHALLOW else (5 if self.physics == EULER3D else 4)
        d = 3 if self.physics == EULER3D else 2
        return nf * self.n ** d * (self.p + 1) ** d


def make_request(physics: int, n: int, p: int, t_end: float, cfl: float = 0.5, arrival: float = 0.0,
                 **params) -> Request:
    """Builds the mesh, the initial GLL values and the CFL step of a request.

    Euler 2-D vortex on [-5, 5]^2 (params beta, x0, y0), shallow-water bump
    on [-5, 5]^2 (a, w, g), Euler 3-D Taylor-Green on [0, 2pi]^3 (Ma)."""
    if physics == EULER3D:
        lo, hi = 0.0, 2 * np.pi
        mesh = meshgen.box(3, n, lo, hi, p)
        x, y, z = coordinates(mesh)
        U0 = taylor_green(x, y, z, Ma=params.get("Ma", 0.1))
    else:
        lo, hi = -5.0, 5.0
        mesh = meshgen.box(2, n, lo, hi, p)
        x, y, _ = coordinates(mesh)
        if physics == EULER2D:
            U0 = vortex(x, y, beta=params.get("beta", 5.0), x0=params.get("x0", 0.0), y0=params.get("y0", 0.0))
        elif physics == SHALLOW:
            U0 = bump(x, y, a=params.get("a", 0.3), w=params.get("w", 0.5), g=params.get("g", 9.81))
        else:
            raise ValueError(f"physics {physics} is not a pool physics")
    h = (hi - lo) / n
    return Request(physics, n, p, t_end, dict(params), arrival, mesh, U0, cfl_dt(U0, h, p, physics, cfl))
