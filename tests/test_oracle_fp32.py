"""Oracle mode 2 (the FP32 particle form of the 1D step) on the CPU: the stored
velocities are floats after every step, the positions stay FP64, and the run
stays within the stated bounds of the FP64 form (mode 1)."""
import numpy as np

import pyoracle as po
from apic import workloads as W
from common import load_oracle, oracle_config, rel_max


def _is_f32(a):
    return np.array_equal(a, a.astype(np.float32).astype(np.float64))


def test_mode2_stores_float_velocities_and_tracks_mode1():
    wl = W.ccp_helium(particles_per_cell=8, cells=32, seed=5, steps=10, table_rows=256)
    T = po.TableSet()
    sims = []
    for mode in (1, 2):
        s = po.Sim1D(oracle_config(wl, T), mode, 99)
        load_oracle(s, wl)
        s.initialize()
        s.step(10)
        sims.append(s)
    one, two = sims
    two.round_fp32()
    c1, n1, _ = one.collisions()
    c2, n2, _ = two.collisions()
    assert c1 == c2 and n1 == n2  # decisions do not move at float resolution
    for k in range(2):
        a, b = two.particles(k), one.particles(k)
        for key in ("vh", "vy", "vz"):
            assert _is_f32(a[key]), key
        assert not _is_f32(b["vh"])  # mode 1 keeps FP64
        if len(a["x"]) == len(b["x"]):
            assert rel_max(a["x"], b["x"]) < 1e-6
            assert rel_max(a["vh"], b["vh"]) < 1e-5
