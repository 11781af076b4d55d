"""Initial data evaluated on the host at a grid's node points (setup, not the hot path).

Each function returns the state in Raven's GridArray parent layout (Np, Ns, E),
column-major, ready for ``GridArray.from_numpy``.
"""

import numpy as np


def _energy(gamma, rho, rhou, p):
    return p / (gamma - 1) + sum(m * m for m in rhou) / (2 * rho)


def _pack(grid, fields):
    q = np.zeros((grid.np, len(fields), grid.E), order="F")
    for s, f in enumerate(fields):
        q[:, s, :] = f
    return q


def isentropic_vortex(grid, law, beta=5.0, u0=1.0, center=(5.0, 0.0), t=0.0):
    """Isentropic vortex of test/balancelaws/euler/isentropicvortex.jl:18-34, advected
    with velocity u0 along x; in 3-D the vortex is invariant along z."""
    g = law.gamma
    x, y = grid.points[:, 0, :], grid.points[:, 1, :]
    r0 = (x - center[0]) - u0 * t
    r1 = (y - center[1]) - 0.0 * t
    f = beta * np.exp(1 - (r0 * r0 + r1 * r1))
    rho = (1 - ((g - 1) * (f * f)) / ((16 * g) * (np.pi * np.pi))) ** (1 / (g - 1))
    c = f / (2 * np.pi)
    u = [u0 + c * (-r1), 0.0 + c * r0] + ([np.zeros_like(x)] if grid.dim == 3 else [])
    rhou = [rho * ui for ui in u]
    p = rho**g
    return _pack(grid, [rho] + rhou + [_energy(g, rho, rhou, p)])


def euler_wave(grid, law, t=0.0):
    """Density wave of test/balancelaws/euler/wave_{2,3}d.jl: u = 1 along every axis, p = 1."""
    x = grid.points
    s = x[:, 0, :]
    for d in range(1, grid.dim):
        s = s + x[:, d, :]
    rho = 2 + np.sin(np.pi * (s - float(grid.dim) * t))
    rhou = [rho * 1.0 for _ in range(grid.dim)]
    return _pack(grid, [rho] + rhou + [_energy(law.gamma, rho, rhou, 1.0)])


def advection_wave(grid, law, t=0.0):
    """2 + sin(pi (sum(x) - sum(u) t)) (test/balancelaws/advection/wave_{2,3}d.jl:18-21)."""
    x = grid.points
    s = x[:, 0, :]
    a = law.u[0]
    for d in range(1, grid.dim):
        s = s + x[:, d, :]
        a = a + law.u[d]
    return _pack(grid, [2 + np.sin(np.pi * (s - a * t))])


def sine_plus_gaussian(grid, law, sigma=0.05, center=(0.5, 0.5, 0.5)):
    """sin(2 pi x) sin(2 pi y) [sin(2 pi z)] + exp(-|x - c|^2 / (2 sigma^2))."""
    x = grid.points
    s = np.ones_like(x[:, 0, :])
    r2 = np.zeros_like(s)
    for d in range(grid.dim):
        s = s * np.sin(2 * np.pi * x[:, d, :])
        r2 = r2 + (x[:, d, :] - center[d]) ** 2
    return _pack(grid, [s + np.exp(-r2 / (2 * sigma * sigma))])


def density_pulse(grid, law, center, amplitude=0.2, width2=0.01):
    """rho = 1 + amplitude * exp(-|x - c|^2 / width2) at rest and uniform pressure 1."""
    x = grid.points
    r2 = np.zeros_like(x[:, 0, :])
    for d in range(grid.dim):
        r2 = r2 + (x[:, d, :] - center[d]) ** 2
    rho = 1 + amplitude * np.exp(-r2 / width2)
    rhou = [np.zeros_like(rho) for _ in range(grid.dim)]
    return _pack(grid, [rho] + rhou + [_energy(law.gamma, rho, rhou, 1.0)])


def max_wavespeed(grid, law, q):
    """max(|u| + c) over the nodes of an Euler state (for the CFL time step)."""
    rho = q[:, 0, :]
    rhou = [q[:, 1 + d, :] for d in range(grid.dim)]
    p = (law.gamma - 1) * (q[:, grid.dim + 1, :] - sum(m * m for m in rhou) / (2 * rho))
    speed = np.sqrt(sum((m / rho) ** 2 for m in rhou))
    return float((speed + np.sqrt(law.gamma * p / rho)).max())
