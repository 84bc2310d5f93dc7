"""The reference's diagnostic sums restated over plain arrays (test
infrastructure): Simulation::sample (src/Simulation.cpp:1140-1161) with
Species::kinetic_energy (src/Species.cpp:338-351) and Grid::node_volume
(src/Grid.cpp:26-30); Diagnostics2D::sample (src/Diagnostics.cpp:111-137) and
Diagnostics3D::sample (src/Diagnostics.cpp:205-232).  Applied to the oracle's
state they give the values the device's sample() must reproduce."""
from __future__ import annotations

import numpy as np


def kinetic_1d(mass, weight, p):
    """0.5 m w (v^2 + v_y^2 + v_z^2) summed over the live particles of one
    species (p: dict of arrays with the time-centred v)."""
    sq = p["v"] ** 2 + p["vy"] ** 2 + p["vz"] ** 2
    if "alive" in p:
        sq = sq[p["alive"] != 0]
    return float(np.sum(0.5 * mass * weight * sq))


def sample_1d(species, parts, rho, E, phi, eps, dirichlet, dx):
    """species: [(mass, weight)], parts: per-species particle dicts."""
    nx = len(rho)
    vol = np.full(nx, dx)
    if dirichlet:
        vol[0] = vol[-1] = 0.5 * dx
    ke = [kinetic_1d(m, w, p) for (m, w), p in zip(species, parts)]
    fe = float(np.sum(0.5 * eps * E * E * vol))
    l1 = float(np.sum(np.abs(rho) * vol))
    live = [int(np.sum(p["alive"] != 0)) if "alive" in p else len(p["x"]) for p in parts]
    out = {"kinetic_energy": float(sum(ke)), "field_energy": fe, "total_energy": float(sum(ke)) + fe,
           "charge_l1": l1, "live_particles": sum(live), "kinetic_by_species": ke, "live_by_species": live}
    if dirichlet:
        out["phi_left"], out["phi_right"] = float(phi[0]), float(phi[-1])
    return out


def sample_nd(species, parts, rho, E, eps, node_volume):
    """species: [(mass, weight)], parts: per-species (pos, v, vh) arrays
    ([3][n], time-centred v); E: [dims][N]; a periodic mesh's node volume is
    the cell volume (2D: area x out-of-plane depth)."""
    ke = [float(np.sum(0.5 * m * w * np.sum(p[1] ** 2, axis=0))) for (m, w), p in zip(species, parts)]
    fe = float(np.sum(0.5 * eps * np.sum(np.asarray(E) ** 2, axis=0) * node_volume))
    l1 = float(np.sum(np.abs(rho) * node_volume))
    live = [p[1].shape[1] for p in parts]
    return {"kinetic_energy": float(sum(ke)), "field_energy": fe, "total_energy": float(sum(ke)) + fe,
            "charge_l1": l1, "live_particles": sum(live), "kinetic_by_species": ke}
