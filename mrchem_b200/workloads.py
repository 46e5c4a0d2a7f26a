"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference measures no public dataset for this path; these generators produce the Gaussian-sum
functions the configurations describe (the same construction MRChem uses for its initial guesses:
projected sums of Gaussians, ``src/initial_guess/gto.cpp:132-170``).  Every function is returned as
an analytic parameter block ``(func_type, params)`` accepted by ``project`` of both the GPU library
and the CPU oracle.

World shared by all configurations: [-20, 20]^3 as 10^3 root boxes of edge 4 (min_scale -2,
corner (-5,-5,-5)).
"""
from __future__ import annotations

import numpy as np

FUNC_GAUSSIANS = 1

WORLD = dict(min_scale=-2, corner=(-5, -5, -5), boxes=(10, 10, 10))


def _gauss_block(coefs, alphas, centers):
    p = [float(len(coefs))]
    for c, a, r in zip(coefs, alphas, centers):
        p += [float(c), float(a), float(r[0]), float(r[1]), float(r[2]), 0.0, 0.0, 0.0]
    return FUNC_GAUSSIANS, np.array(p)


def gaussian_overlap(a, A, b, B):
    """<exp(-a|r-A|^2) | exp(-b|r-B|^2)>."""
    p = a + b
    d2 = float(np.sum((np.asarray(A) - np.asarray(B)) ** 2))
    return (np.pi / p) ** 1.5 * np.exp(-a * b / p * d2)


def normalise(coefs, alphas, centers):
    s = 0.0
    for i in range(len(coefs)):
        for j in range(len(coefs)):
            s += coefs[i] * coefs[j] * gaussian_overlap(alphas[i], centers[i], alphas[j], centers[j])
    return [c / np.sqrt(s) for c in coefs]


def poisson_density(seed=1, ngauss=3):
    """Config 1: sum of 3 normalised (unit-charge) Gaussians, exponents U[1,50], centres U[-2,2]^3."""
    rng = np.random.default_rng(seed)
    alphas = rng.uniform(1.0, 50.0, ngauss)
    centers = rng.uniform(-2.0, 2.0, (ngauss, 3))
    coefs = (alphas / np.pi) ** 1.5
    return _gauss_block(coefs, alphas, centers), dict(alphas=alphas, centers=centers, coefs=coefs)


def atom_sites(rng, n=8, box=6.0):
    return rng.uniform(-box / 2, box / 2, (n, 3))


def orbitals(n=32, seed=2, natoms=8, box=6.0):
    """Config 2: n Slater-like orbitals, each a normalised sum of 2-6 Gaussians with exponents
    log-U[0.5, 200] centred on 8 seeded atom sites in a 6 Bohr box."""
    rng = np.random.default_rng(seed)
    sites = atom_sites(rng, natoms, box)
    out = []
    for _ in range(n):
        ng = int(rng.integers(2, 7))
        alphas = np.exp(rng.uniform(np.log(0.5), np.log(200.0), ng))
        centers = sites[rng.integers(0, natoms, ng)]
        coefs = normalise(list(rng.uniform(0.5, 1.5, ng)), alphas, centers)
        out.append(_gauss_block(coefs, alphas, centers))
    return out


def helmholtz_mus(n=32, seed=2):
    """Config 2: mu_i ~ U[0.5, 3]."""
    rng = np.random.default_rng(seed + 1000)
    return rng.uniform(0.5, 3.0, n)


def density_20_atoms(seed=4, natoms=20, box=12.0, per_atom=4):
    """Config 4: 20 atoms at seeded positions in a 12 Bohr box, 4 Gaussians each, exponents
    log-U[0.3, 1e3], each Gaussian a normalised unit charge."""
    rng = np.random.default_rng(seed)
    sites = atom_sites(rng, natoms, box)
    coefs, alphas, centers = [], [], []
    for s in sites:
        for _ in range(per_atom):
            a = float(np.exp(rng.uniform(np.log(0.3), np.log(1e3))))
            alphas.append(a)
            centers.append(s)
            coefs.append((a / np.pi) ** 1.5)
    return _gauss_block(coefs, alphas, centers)
