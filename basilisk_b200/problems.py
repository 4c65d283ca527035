"""Seeded synthetic inputs of the solver's benchmark workloads.

The reference publishes no data set for this path; each workload is built
from a fixed recipe with a seeded numpy Generator (PCG64).  Arrays are
finest-level values in C order (last index contiguous); face component d has
n+1 entries along d.  Geometry: unit box, origin 0, cell centre
x = (i + 0.5)*Delta (cartesian-common.h:15), face d at x = i*Delta.

  poisson_periodic_2d   128^2 periodic Poisson, alpha = 1, lambda = 0; b a sum
                        of 8 Gaussians A exp(-|x - c|^2 / w^2), c ~ U[0.2, 0.8]^2,
                        w ~ U[0.02, 0.1], A ~ N(0, 1), mean removed
  two_phase_2d          2048^2 variable-coefficient Poisson as in a two-phase
                        projection: f = (1 - tanh((r - 0.25)/(2 Delta)))/2,
                        face fraction ff = (f[i] + f[i-1])/2 with symmetric
                        ghosts, alpha = 1/rho(ff), rho(f) = f (1 - 1000) + 1000
                        (two-phase.h:48,97-99); b ~ N(0, 1); Dirichlet a = 0
  helmholtz_3d          256^3 periodic Helmholtz as viscosity/diffusion: alpha =
                        1e-2 stored on every face, lambda = -1/dt = -1000;
                        b ~ N(0, 1) smoothed by 4 weighted-Jacobi sweeps
                        u <- (1 - w) u + w (sum of 6 neighbours)/6, w = 2/3,
                        periodic wrap
  two_phase_tree        the two_phase_2d problem on a quadtree: level < 5
                        everywhere, and every cell whose centre lies within 4
                        of its own cells of the circle r = 0.25 refined, up to
                        level 11 (2:1 graded); the interface width is that of
                        the finest level on every level, b ~ N(0, 1) drawn per
                        level (the solver reads the leaves)
  random_field_2d       512^2 periodic Poisson with alpha = exp(kappa) on faces,
                        kappa a Gaussian random field (FFT, squared-exponential
                        covariance sigma^2 exp(-r^2 / (2 l^2)), l = 0.05,
                        sigma = 1), face value exp((kappa[i] + kappa[i-1])/2);
                        b as poisson_periodic_2d
"""
import math

import numpy as np


def centers(dim, n, L0=1.0, origin=(0.0, 0.0, 0.0)):
    D = L0 * (1.0 / n)
    ax = [(np.arange(n) + 0.5) * D + origin[d] for d in range(dim)]
    return list(np.meshgrid(*ax, indexing="ij"))


def gaussian_bumps(n, rng, count=8):
    x, y = centers(2, n)
    b = np.zeros((n, n))
    c = rng.uniform(0.2, 0.8, size=(count, 2))
    w = rng.uniform(0.02, 0.1, size=count)
    A = rng.standard_normal(count)
    for k in range(count):
        b += A[k] * np.exp(-((x - c[k, 0]) ** 2 + (y - c[k, 1]) ** 2) / w[k] ** 2)
    return b - b.mean()


def poisson_periodic_2d(depth=7, seed=0):
    n = 1 << depth
    rng = np.random.default_rng(seed)
    return {"dim": 2, "depth": depth, "periodic": (0, 1), "b": gaussian_bumps(n, rng),
            "alpha": None, "lambda": None, "bc": {}, "tolerance": 1e-6}


def two_phase_alpha(n, rho1=1.0, rho2=1000.0, radius=0.25, width_n=None):
    """Face coefficients of a level with n cells per side; the interface
    width is 2 Delta of a level with width_n cells (default: this one)."""
    D = 1.0 / (width_n or n)
    x, y = centers(2, n)
    r = np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2)
    f = 0.5 * (1.0 - np.tanh((r - radius) / (2.0 * D)))
    comps = []
    for d in range(2):
        fp = np.concatenate([np.take(f, [0], axis=d), f, np.take(f, [n - 1], axis=d)], axis=d)
        lo = np.take(fp, np.arange(0, n + 1), axis=d)
        hi = np.take(fp, np.arange(1, n + 2), axis=d)
        ff = (lo + hi) / 2.0
        ff = np.clip(ff, 0.0, 1.0)
        rho = ff * (rho1 - rho2) + rho2
        comps.append(1.0 / rho)
    return comps


def two_phase_2d(depth=11, seed=1):
    n = 1 << depth
    rng = np.random.default_rng(seed)
    return {"dim": 2, "depth": depth, "periodic": (), "b": rng.standard_normal((n, n)),
            "alpha": two_phase_alpha(n), "lambda": None,
            "bc": {s: ("dirichlet", 0.0) for s in range(4)}, "tolerance": 1e-6}


def smoothed_noise_3d(n, rng, sweeps=4, omega=2.0 / 3.0):
    u = rng.standard_normal((n, n, n))
    for _ in range(sweeps):
        s = np.zeros_like(u)
        for ax in range(3):
            s += np.roll(u, 1, axis=ax) + np.roll(u, -1, axis=ax)
        u = (1.0 - omega) * u + omega * s / 6.0
    return u


def helmholtz_3d(depth=8, seed=2, D=1e-2, dt=1e-3):
    n = 1 << depth
    rng = np.random.default_rng(seed)
    alpha = [np.full(tuple(n + 1 if e == d else n for e in range(3)), D) for d in range(3)]
    return {"dim": 3, "depth": depth, "periodic": (0, 1, 2),
            "b": smoothed_noise_3d(n, rng), "alpha": alpha, "lambda": -1.0 / dt,
            "bc": {}, "tolerance": 1e-8}


def gaussian_random_field(n, rng, length=0.05, sigma=1.0):
    """Periodic stationary field with covariance sigma^2 exp(-r^2/(2 l^2)),
    sampled by filtering white noise with the square root of its spectrum."""
    k = np.fft.fftfreq(n, d=1.0 / n) * 2.0 * math.pi
    kx, ky = np.meshgrid(k, k, indexing="ij")
    # spectral density of the squared-exponential kernel on the unit torus
    S = (2.0 * math.pi * length ** 2) * np.exp(-0.5 * length ** 2 * (kx ** 2 + ky ** 2))
    noise = rng.standard_normal((n, n))
    field = np.real(np.fft.ifft2(np.fft.fft2(noise) * np.sqrt(S))) * n
    field *= sigma / max(field.std(), 1e-300)
    return field


def face_exp(kappa):
    n = kappa.shape[0]
    comps = []
    for d in range(2):
        kp = np.concatenate([np.take(kappa, [n - 1], axis=d), kappa, np.take(kappa, [0], axis=d)], axis=d)
        lo = np.take(kp, np.arange(0, n + 1), axis=d)
        hi = np.take(kp, np.arange(1, n + 2), axis=d)
        comps.append(np.exp((lo + hi) / 2.0))
    return comps


def random_field_2d(depth=9, seed=3, instance=0):
    n = 1 << depth
    rng = np.random.default_rng([seed, instance])
    kappa = gaussian_random_field(n, rng)
    return {"dim": 2, "depth": depth, "periodic": (0, 1), "kappa": kappa,
            "b": gaussian_bumps(n, rng), "alpha": face_exp(kappa), "lambda": None,
            "bc": {}, "tolerance": 1e-6}


def setup(grid, prob):
    """Create the fields of ``prob`` on ``grid`` (a basilisk_b200.Grid);
    returns (a, b, alpha, lambda) with a = 0."""
    for d in prob["periodic"]:
        grid.periodic(2 * d)
    a = grid.scalar()
    for side, (kind, val) in prob["bc"].items():
        a.bc(side, kind, val)
    a.set(np.zeros(prob["b"].shape))
    b = grid.scalar(prob["b"])
    alpha = grid.face_vector(prob["alpha"]) if prob["alpha"] is not None else None
    lam = prob["lambda"]
    if lam is None:
        lam_f = None
    elif np.isscalar(lam):
        lam_f = grid.const_scalar(float(lam))
    else:
        lam_f = grid.scalar(lam)
    return a, b, alpha, lam_f


def band_refinement(depth, base, width=4.0, radius=0.25, center=(0.5, 0.5)):
    """``refine`` predicate of two_phase_tree: every cell below level base,
    and the cells whose centre lies within ``width`` cells of their own level
    of the circle, up to level depth."""
    def cond(level, x, y):
        if level < base:
            return True
        if level >= depth:
            return False
        r = math.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2)
        return abs(r - radius) < width * (1.0 / (1 << level))
    return cond


def two_phase_tree_levels(depth, seed=1):
    """Dense per-level inputs of two_phase_tree: {level: (b, alpha_x,
    alpha_y)}; the leaves of any tree of this depth read their cells."""
    rng = np.random.default_rng(seed)
    n_fine = 1 << depth
    out = {}
    for l in range(depth + 1):
        n = 1 << l
        ax, ay = two_phase_alpha(n, width_n=n_fine)
        out[l] = (rng.standard_normal((n, n)), ax, ay)
    return out


def setup_tree(grid, depth=11, base=5, seed=1):
    """two_phase_tree on ``grid`` (a basilisk_b200.TreeGrid of depth >=
    depth): refine, then create the fields; returns (a, b, alpha) with a = 0
    on every level, Dirichlet a = 0 on the four walls."""
    grid.refine(band_refinement(depth, base))
    a, b = grid.scalar(), grid.scalar()
    for side in range(4):
        a.bc(side, "dirichlet", 0.0)
    alpha = grid.face_vector()
    for l, (bl, ax, ay) in two_phase_tree_levels(grid.tree_depth, seed).items():
        b.set(bl, level=l)
        a.set(np.zeros_like(bl), level=l)
        alpha.set([ax, ay], level=l)
    return a, b, alpha
