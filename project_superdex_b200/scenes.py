"""Seeded synthetic soft-body scenes (tet grids, materials, pins, colliders).

The reference builds soft actors from tetrahedral meshes (mochi_physics/src/mochi_soft_init.cpp)
produced offline by its mesh CLI; here every mesh is a seeded hex grid split into 6 tets per hex
(Freudenthal split along the hex diagonal), which is the workload the soft-body step is measured on.

All arrays are numpy and identical for the CUDA library and the CPU oracle.
"""
from __future__ import annotations

import dataclasses
import itertools
from typing import List, Optional, Sequence

import numpy as np

COLLIDER_PLANE = 0
COLLIDER_CAPSULE = 1


@dataclasses.dataclass
class Collider:
    """A kinematic rigid collider. Plane: p = (n, o) with d = n.x - o.
    Capsule: p = (a, b) segment end points, radius r. Both move with constant velocity `vel`."""

    type: int
    p: np.ndarray  # 6 doubles (plane uses 4)
    radius: float = 0.0
    vel: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(3))

    def as_row(self) -> np.ndarray:
        """Packed float64[11] = (type, p[6], radius, vel[3])."""
        row = np.zeros(11)
        row[0] = self.type
        row[1:7] = self.p
        row[7] = self.radius
        row[8:11] = self.vel
        return row


@dataclasses.dataclass
class Body:
    """One soft body (environment)."""

    X: np.ndarray          # (N, 3) float64 rest positions
    tets: np.ndarray       # (T, 4) int32, positively oriented
    E: np.ndarray          # (T,) float64 Young's modulus
    nu: np.ndarray         # (T,) float64 Poisson ratio
    rho: np.ndarray        # (T,) float64 density
    pin: np.ndarray        # (N,) uint8, bit c set -> DoF c pinned
    colliders: List[Collider]
    cells: tuple = (0, 0, 0)
    material: int = 0      # SoftMaterialType: 0 Neo-Hookean (Smith), 1 St. Venant-Kirchhoff, 2 linear elastic,
                           # 5 ARAP (stiffness = the tet's mu)

    @property
    def n_nodes(self) -> int:
        return int(self.X.shape[0])

    @property
    def n_tets(self) -> int:
        return int(self.tets.shape[0])

    def lame(self):
        """(lambda, mu) per tet, ComputeLameConstants (mochi_core/.../materials/material_utils.h:331)."""
        lam = self.E * self.nu / ((1.0 + self.nu) * (1.0 - 2.0 * self.nu))
        mu = self.E / (2.0 * (1.0 + self.nu))
        return lam, mu


@dataclasses.dataclass
class SceneConfig:
    """Physics and solver constants shared by all bodies of a scene."""

    dt: float = 1.0 / 240.0
    gravity: tuple = (0.0, 0.0, -9.81)
    k_contact: float = 1e9        # ContactParams::penaltyCoefficient default (contact_params.h:96)
    t_half: float = 0.005         # penaltySmoothingHalfDistance (contact_params.h:108)
    thr: float = 0.001            # penaltyThresholdDefault (contact_params.h:123)
    max_align: float = 0.0        # maxAlignmentNormals
    steps: int = 100
    mass_damping: float = 0.0     # Rayleigh massDampingCoefficient alpha [1/s]
    stiffness_damping: float = 0.0  # Rayleigh stiffnessDampingCoefficient beta [s]
    stiffness_damping_geometric: bool = False  # stiffnessDampingIncludeGeometricTerm
    # contact dissipation (ContactParams / ContactEvalConfig); the reference's default Coulomb coefficient
    # is 0.5, the workloads here are frictionless unless they say otherwise
    friction_coulomb: float = 0.0
    friction_falloff_vel: float = 0.01
    friction_viscous: float = 0.0
    contact_normal_damping: float = 0.0
    friction_model: int = 0          # 0 C1Regularized, 1 CinfRegularized
    friction_fitted_hessian: bool = True
    friction_fade: bool = True
    friction_collider_normal: bool = True
    contact_explicit_normals: bool = False
    contact_implicit_normal_force: bool = False


# Freudenthal split of a hex into 6 tets: paths 0 -> 7 through the corner cube.
def _hex_tets() -> np.ndarray:
    out = []
    for perm in itertools.permutations(range(3)):
        c = [0]
        cur = 0
        for a in perm:
            cur |= 1 << a
            c.append(cur)
        # orientation: even permutations of the axes give positive volume for corner order
        # (0, e_a, e_a+e_b, 7); odd permutations are flipped by swapping the two middle corners.
        sign = np.linalg.det(np.array([[(c[k] >> a) & 1 for a in range(3)] for k in (1, 2, 3)],
                                      dtype=float))
        if sign < 0:
            c[1], c[2] = c[2], c[1]
        out.append(c)
    return np.array(out, dtype=np.int64)


_HEX_TETS = _hex_tets()


def grid_body(nx: int, ny: int, nz: int, h: float, origin=(0.0, 0.0, 0.0), jitter: float = 0.1,
              rng: Optional[np.random.Generator] = None, E=1e5, nu=0.45, rho=1000.0,
              pin_bottom: bool = True) -> Body:
    """nx*ny*nz hex cells of edge h, 6 tets per hex, interior nodes jittered U(+-jitter*h)."""
    rng = rng if rng is not None else np.random.default_rng(0)
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    # node index = i + (nx+1) * (j + (ny+1) * k)
    ii = ii.transpose(2, 1, 0).reshape(-1)
    jj = jj.transpose(2, 1, 0).reshape(-1)
    kk = kk.transpose(2, 1, 0).reshape(-1)
    X = np.stack([ii, jj, kk], axis=1).astype(np.float64) * h + np.asarray(origin, np.float64)
    interior = (ii > 0) & (ii < nx) & (jj > 0) & (jj < ny) & (kk > 0) & (kk < nz)
    noise = rng.uniform(-jitter * h, jitter * h, size=X.shape)
    X[interior] += noise[interior]

    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ci = ci.transpose(2, 1, 0).reshape(-1)
    cj = cj.transpose(2, 1, 0).reshape(-1)
    ck = ck.transpose(2, 1, 0).reshape(-1)
    corners = np.empty((ci.size, 8), dtype=np.int64)
    for b in range(8):
        corners[:, b] = (ci + (b & 1)) + (nx + 1) * ((cj + ((b >> 1) & 1)) + (ny + 1) * (ck + ((b >> 2) & 1)))
    tets = corners[:, _HEX_TETS].reshape(-1, 4).astype(np.int32)
    T = tets.shape[0]
    Ea = np.broadcast_to(np.asarray(E, np.float64), (T,)).copy()
    nua = np.broadcast_to(np.asarray(nu, np.float64), (T,)).copy()
    rhoa = np.full(T, float(rho))
    pin = np.zeros(X.shape[0], np.uint8)
    if pin_bottom:
        pin[kk == 0] = 7
    return Body(X=X, tets=tets, E=Ea, nu=nua, rho=rhoa, pin=pin, colliders=[], cells=(nx, ny, nz))


def capsule(a, b, r, vel) -> Collider:
    p = np.zeros(6)
    p[:3] = a
    p[3:] = b
    return Collider(COLLIDER_CAPSULE, p, float(r), np.asarray(vel, np.float64))


def plane(n, o, vel=(0.0, 0.0, 0.0)) -> Collider:
    p = np.zeros(6)
    p[:3] = np.asarray(n, np.float64) / np.linalg.norm(n)
    p[3] = o
    return Collider(COLLIDER_PLANE, p, 0.0, np.asarray(vel, np.float64))


def _fingertips(rng, lo, hi, top, n=5, r=0.004, length=0.02, speed=0.05, gap=0.002):
    """n capsules just above z=top inside the xy box [lo, hi], moving down at `speed`."""
    out = []
    for _ in range(n):
        c = np.array([rng.uniform(lo[0] + length / 2, hi[0] - length / 2),
                      rng.uniform(lo[1] + length / 2, hi[1] - length / 2),
                      top + r + rng.uniform(0.0, gap)])
        th = rng.uniform(0.0, np.pi)
        axis = np.array([np.cos(th), np.sin(th), 0.0]) * (length / 2)
        d = np.array([rng.normal(0, 0.1), rng.normal(0, 0.1), -1.0])
        d *= speed / np.linalg.norm(d)
        out.append(capsule(c - axis, c + axis, r, d))
    return out


def config0(seed: int = 0):
    """Single soft cube: 10^3 cells of 0.01 m (1,331 nodes, 6,000 tets), E=1e5, nu=0.45,
    bottom pinned, gravity, dt=1/240, 100 steps, no contact."""
    rng = np.random.default_rng(seed)
    b = grid_body(10, 10, 10, 0.01, rng=rng, E=1e5, nu=0.45, rho=1000.0)
    return [b], SceneConfig(steps=100)


def config1(seed: int = 0, n: int = 64, size: float = 0.1):
    """Single large body with contact: n^3 cells over a `size` m cube (64^3: 274,625 nodes,
    1,572,864 tets); E log-uniform per tet in [1e4, 1e6], nu=0.45; 5 capsules (r=4 mm, L=20 mm)
    pressing on the top at 0.05 m/s; penalty stiffness 1e4, activation distance 1 mm; 200 steps."""
    rng = np.random.default_rng(seed)
    h = size / n
    b = grid_body(n, n, n, h, rng=rng, nu=0.45)
    b.E = np.exp(rng.uniform(np.log(1e4), np.log(1e6), size=b.n_tets))
    b.colliders = _fingertips(rng, (0, 0), (size, size), size)
    return [b], SceneConfig(k_contact=1e4, steps=200)


def config2(seed: int = 0, n_envs: int = 1024, lo: int = 8, hi: int = 40, h: float = 0.0025):
    """Batched uneven environments: per-axis cell counts U{lo..hi} (independent axes), E in
    [1e4, 1e6] and nu in [0.3, 0.48] per body, 5 capsule fingertips and a ground plane each."""
    rng = np.random.default_rng(seed)
    bodies = []
    for _ in range(n_envs):
        nx, ny, nz = (int(v) for v in rng.integers(lo, hi + 1, size=3))
        E = float(np.exp(rng.uniform(np.log(1e4), np.log(1e6))))
        nu = float(rng.uniform(0.3, 0.48))
        b = grid_body(nx, ny, nz, h, rng=rng, E=E, nu=nu, pin_bottom=False,
                      origin=(0.0, 0.0, 0.0005))
        b.colliders = [plane((0, 0, 1), 0.0)] + _fingertips(rng, (0, 0), (nx * h, ny * h), nz * h + 0.0005)
        bodies.append(b)
    return bodies, SceneConfig(steps=100)


def config4(seed: int = 0, n: int = 96, size: float = 0.1):
    """Stiff heterogeneous body: n^3 cells, nu=0.49, E log-uniform [1e4, 1e7] with 10 spherical
    inclusions (radius 5-15 cells, E x100), squeezed between two planes closing at 0.02 m/s
    plus 5 capsules; 100 steps."""
    rng = np.random.default_rng(seed)
    h = size / n
    b = grid_body(n, n, n, h, rng=rng, nu=0.49, pin_bottom=False)
    b.E = np.exp(rng.uniform(np.log(1e4), np.log(1e7), size=b.n_tets))
    cent = b.X[b.tets].mean(axis=1)
    for _ in range(10):
        c = rng.uniform(0, size, size=3)
        r = rng.uniform(5, 15) * h
        b.E[np.linalg.norm(cent - c, axis=1) < r] *= 100.0
    b.colliders = [plane((0, 0, 1), -0.0005, vel=(0, 0, 0.01)),
                   plane((0, 0, -1), -(size + 0.0005), vel=(0, 0, -0.01))]
    b.colliders += _fingertips(rng, (0, 0), (size, size), size)
    return [b], SceneConfig(steps=100)


def concat_bodies(bodies: Sequence[Body]):
    """CSR-of-environments layout: concatenated nodes/tets with per-env offsets (tets re-indexed
    to global node ids)."""
    node_off = np.zeros(len(bodies) + 1, np.int64)
    tet_off = np.zeros(len(bodies) + 1, np.int64)
    for i, b in enumerate(bodies):
        node_off[i + 1] = node_off[i] + b.n_nodes
        tet_off[i + 1] = tet_off[i] + b.n_tets
    X = np.concatenate([b.X for b in bodies])
    tets = np.concatenate([b.tets.astype(np.int64) + node_off[i] for i, b in enumerate(bodies)]).astype(np.int32)
    return node_off, tet_off, X, tets
