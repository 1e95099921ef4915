"""Seeded synthetic cavities: perturbed ellipsoids with spherical-harmonic noise.

The real-cavity workload (a watertight ~20k-triangle mesh of ~2.2 ml voxelised
at 0.5 mm) is stood in for by this generator: an icosphere (20*4^5 = 20480
triangles), radially perturbed by real spherical harmonics of degree 1-4 with
seeded coefficients (total amplitude 15 % of the radius), stretched to
sinus-like proportions and scaled to the requested volume. It is new
synthetic input, not a reference asset.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.s = seed & MASK64

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        return lo + (hi - lo) * ((self.next() >> 11) / float(1 << 53))


def icosphere(subdiv: int):
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, dtype=np.int64)


def real_sh(l: int, m: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """Real spherical harmonic Y_lm (orthonormal), theta polar, phi azimuth."""
    x = np.cos(theta)
    am = abs(m)
    # associated Legendre P_l^|m|(x) by the standard recurrence
    pmm = np.ones_like(x)
    if am > 0:
        somx2 = np.sqrt(np.maximum(0.0, (1 - x) * (1 + x)))
        fact = 1.0
        for _ in range(am):
            pmm = -pmm * fact * somx2
            fact += 2.0
    if l == am:
        plm = pmm
    else:
        pmmp1 = x * (2 * am + 1) * pmm
        if l == am + 1:
            plm = pmmp1
        else:
            for ll in range(am + 2, l + 1):
                pll = (x * (2 * ll - 1) * pmmp1 - (ll + am - 1) * pmm) / (ll - am)
                pmm, pmmp1 = pmmp1, pll
            plm = pmmp1
    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
    if m > 0:
        return math.sqrt(2) * norm * plm * np.cos(m * phi)
    if m < 0:
        return math.sqrt(2) * norm * plm * np.sin(am * phi)
    return norm * plm


@dataclass
class Cavity:
    tris: np.ndarray      # [T, 9] metres, outward winding
    volume: float         # m^3
    tip: tuple            # needle tip on the floor (inside), metres
    axis: tuple           # needle axis (unit)


def signed_volume(tris: np.ndarray) -> float:
    t = tris.reshape(-1, 3, 3)
    cr = np.cross(t[:, 1], t[:, 2])
    terms = (t[:, 0, 0] * cr[:, 0] + t[:, 0, 1] * cr[:, 1] + t[:, 0, 2] * cr[:, 2]) / 6.0
    return float(np.cumsum(terms)[-1])


def perturbed_ellipsoid(seed: int, volume_ml: float = 2.2, amplitude: float = 0.15,
                        proportions=(1.0, 2.8, 2.0), subdiv: int = 5, tilt_deg: float = 0.0) -> Cavity:
    """A watertight cavity of ``volume_ml`` with SH radial noise (degrees 1-4).

    Gravity is assumed along -y; the needle tip sits 1.5 mm above the floor
    directly below the centre and fires up, tilted by ``tilt_deg`` about z."""
    rng = SplitMix64(seed)
    v, f = icosphere(subdiv)
    theta = np.arccos(np.clip(v[:, 1], -1, 1))  # polar angle from +y
    phi = np.arctan2(v[:, 2], v[:, 0])
    pert = np.zeros(len(v))
    for l in range(1, 5):
        for m in range(-l, l + 1):
            pert += rng.uniform(-1.0, 1.0) * real_sh(l, m, theta, phi)
    pert *= amplitude / max(np.max(np.abs(pert)), 1e-12)
    r = 1.0 + pert
    pts = v * r[:, None] * np.asarray(proportions, dtype=np.float64)[None, :]
    tris = pts[f].reshape(-1, 9)
    vol = signed_volume(tris)
    if vol < 0:  # keep outward winding
        f = f[:, ::-1]
        tris = pts[f].reshape(-1, 9)
        vol = -vol
    s = (volume_ml * 1e-6 / vol) ** (1.0 / 3.0)
    pts = pts * s
    tris = pts[f].reshape(-1, 9)
    vol = signed_volume(tris)
    # floor point straight below the centre: the vertex direction closest to -y
    down = int(np.argmin(v[:, 1]))
    floor_y = pts[down, 1]
    tip = (0.0, float(floor_y + 1.5e-3), 0.0)
    a = math.radians(tilt_deg)
    axis = (math.sin(a), math.cos(a), 0.0)
    return Cavity(tris=tris, volume=vol, tip=tip, axis=axis)
