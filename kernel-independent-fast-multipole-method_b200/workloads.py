"""Seeded synthetic point clouds and densities for the KIFMM benchmark shapes.

No public dataset is involved: every input is generated here with numpy's
PCG64 generator (``numpy.random.default_rng``), seed 0 for positions, seed 1
for densities and seed 2 for the check-target indices.  Positions are
(n, 3) float64 arrays, i.e. the reference's 3 x n column-major DblNumMat
(xyz interleaved).  The reference's own CLI driver draws uniform cube points
and U[0,1] densities (fmm3d/tt.cpp:59-78); the shapes below are the
benchmark workloads' sphere, ellipsoid and cube + Plummer clouds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

KERNEL_DOFS = {111: (1, 1), 121: (1, 1), 301: (4, 3), 311: (3, 3), 312: (3, 1), 321: (3, 3),
               322: (3, 1), 511: (3, 3), 521: (3, 3)}


def sphere(n: int, seed: int = 0):
    """Uniform on the unit sphere surface: Gaussian 3-vectors normalised.
    Normals are the positions themselves."""
    g = np.random.default_rng(seed).standard_normal((n, 3))
    p = g / np.linalg.norm(g, axis=1, keepdims=True)
    return np.ascontiguousarray(p), np.ascontiguousarray(p.copy())


def ellipsoid(n: int, seed: int = 0, axes=(1.0, 0.5, 0.25)):
    """Sphere samples scaled per axis; normals from the implicit gradient
    (x/a^2, y/b^2, z/c^2), normalised."""
    s, _ = sphere(n, seed)
    a = np.asarray(axes, np.float64)
    p = s * a
    nrm = p / (a * a)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    return np.ascontiguousarray(p), np.ascontiguousarray(nrm)


def cube(n: int, seed: int = 0):
    p = np.random.default_rng(seed).uniform(-1.0, 1.0, (n, 3))
    return np.ascontiguousarray(p), np.ascontiguousarray(p.copy())


def cube_plummer(n: int, seed: int = 0, frac: float = 0.3, scale: float = 0.1,
                 centre=(0.3, 0.2, -0.4)):
    """(1-frac) uniform in [-1,1]^3 plus frac from a Plummer ball
    (r = a / sqrt(m^(-2/3) - 1), uniform direction).  Plummer samples
    outside the open box (-1,1)^3 are redrawn, so every point lies inside
    the reference's root box (fmm3d/let3d.cpp:73)."""
    rng = np.random.default_rng(seed)
    npl = int(round(frac * n))
    nu = n - npl
    pu = rng.uniform(-1.0, 1.0, (nu, 3))
    c = np.asarray(centre, np.float64)
    out = np.empty((0, 3))
    while len(out) < npl:
        k = (npl - len(out)) * 2 + 16
        m = rng.uniform(0.0, 1.0, k)
        m = np.clip(m, 1e-12, 1.0 - 1e-12)
        r = scale / np.sqrt(m ** (-2.0 / 3.0) - 1.0)
        d = rng.standard_normal((k, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        q = c + r[:, None] * d
        ok = np.all(np.abs(q) < 1.0, axis=1)
        out = np.concatenate([out, q[ok]])
    p = np.concatenate([pu, out[:npl]])
    return np.ascontiguousarray(p), np.ascontiguousarray(p.copy())


def densities(n: int, sdof: int, dist: str = "uniform", seed: int = 1):
    rng = np.random.default_rng(seed)
    if dist == "uniform":       # U[-1, 1]
        return rng.uniform(-1.0, 1.0, n * sdof)
    if dist == "uniform01":     # U[0, 1], as fmm3d/tt.cpp:75
        return rng.uniform(0.0, 1.0, n * sdof)
    if dist == "normal":
        return rng.standard_normal(n * sdof)
    raise ValueError(dist)


def check_indices(n: int, k: int, seed: int = 2):
    return np.sort(np.random.default_rng(seed).choice(n, size=min(k, n), replace=False))


@dataclass
class Workload:
    name: str
    kt: int
    coefs: tuple
    np_: int
    ptsmax: int
    maxlevel: int
    n: int
    geometry: str
    dens: str
    nchk: int
    precision: str = "fp64"
    ctr: tuple = (0.0, 0.0, 0.0)
    rootlvl: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def sdof(self):
        return KERNEL_DOFS[self.kt][0]

    @property
    def tdof(self):
        return KERNEL_DOFS[self.kt][1]

    def points(self, n: int | None = None):
        n = self.n if n is None else n
        gen = {"sphere": sphere, "ellipsoid": ellipsoid, "cube": cube, "cube_plummer": cube_plummer}[self.geometry]
        return gen(n, 0)

    def density(self, n: int | None = None):
        n = self.n if n is None else n
        return densities(n, self.sdof, self.dens, 1)


# The five benchmark shapes.  Sources = targets throughout.
WORKLOADS = {
    "laplace_sphere_np4": Workload("laplace_sphere_np4", 111, (1.0,), 4, 100, 10, 32768, "sphere", "uniform", 1000),
    "stokes_dl_ellipsoid_np6": Workload("stokes_dl_ellipsoid_np6", 321, (1.0,), 6, 100, 10, 262144, "ellipsoid",
                                        "uniform", 1000),
    "navier_sphere_np8": Workload("navier_sphere_np8", 511, (1.0, 0.3), 8, 150, 10, 1048576, "sphere", "normal",
                                  1000),
    "laplace_cube_plummer_np6": Workload("laplace_cube_plummer_np6", 111, (1.0,), 6, 64, 10, 4194304,
                                         "cube_plummer", "uniform", 4096, precision="mixed"),
}


def surface_counts(np_: int):
    """|UE| = np^3 - (np-2)^3 and |UC| = (np+2)^3 - np^3 (fmm3d/matmgnt3d.cpp:375-398)."""
    ue = np_ ** 3 - (np_ - 2) ** 3
    uc = (np_ + 2) ** 3 - np_ ** 3
    return ue, uc


def log_uniform_sizes(k: int, lo: float = 1e4, hi: float = 5e5, seed: int = 3):
    u = np.random.default_rng(seed).uniform(math.log(lo), math.log(hi), k)
    return np.round(np.exp(u)).astype(np.int64)


def plummer_ball(n: int, seed: int = 0, scale: float = 0.1):
    """A Plummer-clustered ball of scale radius `scale` at the origin (points
    outside the open root box (-1,1)^3 redrawn)."""
    return cube_plummer(n, seed, frac=1.0, scale=scale, centre=(0.0, 0.0, 0.0))


GEOMETRIES = {"sphere": sphere, "ellipsoid": ellipsoid, "cube": cube, "cube_plummer": cube_plummer,
              "plummer_ball": plummer_ball}


def batched_instances(k: int = 64, n_stokes: int = 16, seed: int = 3, lo: float = 1e4, hi: float = 5e5):
    """The batched workload: k independent instances with log-uniform sizes in
    [lo, hi]; geometries cycle through the unit sphere surface, the uniform
    cube and the Plummer ball; n_stokes of them (seeded choice) use the Stokes
    single-layer kernel (311, mu = 1), the rest Laplace single-layer (111)."""
    sizes = log_uniform_sizes(k, lo, hi, seed)
    stokes = set(np.random.default_rng(seed + 1).choice(k, size=n_stokes, replace=False).tolist())
    geoms = ("sphere", "cube", "plummer_ball")
    out = []
    for i in range(k):
        kt = 311 if i in stokes else 111
        out.append({"index": i, "kt": kt, "coefs": (1.0,), "n": int(sizes[i]), "geometry": geoms[i % 3],
                    "seed": 100 + i})
    return out
