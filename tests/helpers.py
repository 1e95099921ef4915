"""Shared test helpers: build oracle solvers from resolved scenes (oracle = checker only)."""
from __future__ import annotations

import os

import numpy as np

import oracle
from sdr_b200 import scene as sc

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ASSETS = os.path.join(REPO, "tests", "golden")


def oracle_sdf(res: sc.ResolvedScene, tris=None):
    """The SDF ``SceneConfig::build`` makes (scene.rs:279-297), computed by the oracle."""
    if res.sinus is not None:
        return oracle.sdf_from_sinus(res.sinus, res.sdf_origin, res.sdf_dx, res.sdf_dims)
    if tris is None:
        tris = sc.load_mesh(res.mesh_path) * sc.MM
    return oracle.sdf_from_mesh(tris, res.sdf_dx, res.mesh_padding)


def cavity_volume(res: sc.ResolvedScene, tris=None) -> float:
    """``cavity_mesh.signed_volume().abs()`` (scene.rs:312)."""
    if res.sinus is not None:
        return oracle.sinus_mesh_volume(res.sinus)[0]
    if tris is None:
        tris = sc.load_mesh(res.mesh_path) * sc.MM
    return abs(oracle.mesh_signed_volume(tris))


def oracle_solver(res: sc.ResolvedScene, sdf=None) -> oracle.Solver:
    sdf = sdf if sdf is not None else oracle_sdf(res)
    f = res.fluid
    fl = oracle.Fluid(f.density, f.gravity, f.flip_ratio, f.particles_per_cell,
                      f.volume_stiffness, f.redistribute, f.redist_cap_factor)
    n = res.needle
    nd = oracle.Needle(n.tip, n.axis, n.radius, n.flow_rate, n.inject_until)
    s = oracle.Solver(sdf, res.sim_dx, fl, nd)
    s.set_solve(res.solve.max_iters, res.solve.tol)
    s.set_outlet(res.outlet)
    return s
