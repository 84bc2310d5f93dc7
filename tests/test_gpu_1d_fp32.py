"""The 1D FP32 storage form (APIC_FP32_STORAGE: v_half, v_y, v_z stored as
float; position, fields and all arithmetic FP64) through the C ABI.

Parity: against oracle mode 2, which stores the same components as float at
the same points, the state agrees bit for bit except where the two FP64
evaluations (which agree to about 1e-15) straddle a float rounding boundary;
those rare one-ulp differences are bounded below.  Collision counts are exact.

Error of the form: against the FP64 oracle (mode 1), the stated bounds of the
FP32 form after 20 MCC steps of the discharge and 50 steps of the two-stream
deck."""
import numpy as np
import pytest

import apic
import pyoracle as po
from apic import workloads as W
from common import load_device, load_oracle, oracle_config, rel_max

pytestmark = pytest.mark.gpu

# fraction of values that must agree to 1e-12 with oracle mode 2, and the
# bound on the rest (a flipped float rounding perturbs one particle by about
# 6e-8 relative, which the following steps carry along)
EXACT_FRACTION = 0.99
MAX_REL = 1e-5
# error of the FP32 form against the FP64 oracle
FP32_VS_FP64 = {"x": 1e-6, "vh": 1e-5, "v": 1e-5, "vy": 1e-6, "vz": 1e-6, "field_energy": 1e-4}


def _pair(wl, seed=0x5EED):
    cfg, tabs = W.to_device_config(wl, precision=apic.FP32_STORAGE, seed=seed)
    dev = apic.Simulation1D(cfg, tabs)
    load_device(dev, wl)
    dev.initialize()
    T = po.TableSet()
    ora2 = po.Sim1D(oracle_config(wl, T), 2, seed)
    load_oracle(ora2, wl)
    ora2.initialize()
    ora1 = po.Sim1D(oracle_config(wl, T), 1, seed)
    load_oracle(ora1, wl)
    ora1.initialize()
    return dev, ora2, ora1, (T, tabs)


def _close(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(float(np.max(np.abs(b))), 1e-300) if b.size else 1.0
    d = np.abs(a - b) / scale
    return float(np.mean(d <= 1e-12)) if d.size else 1.0, float(d.max()) if d.size else 0.0


def _check_mode2(dev, ora2, nspecies):
    ora2.round_fp32()  # the device stored its read-back state as float
    for s in range(nspecies):
        a, b = dev.particles(s), ora2.particles(s)
        assert len(a["x"]) == len(b["x"])
        for k in ("x", "v", "vh", "vy", "vz"):
            frac, mx = _close(a[k], b[k])
            assert frac >= EXACT_FRACTION and mx < MAX_REL, (s, k, frac, mx)
        # the stored components really are floats
        for k in ("vh", "vy", "vz"):
            assert np.array_equal(a[k], a[k].astype(np.float32).astype(np.float64)), k


@pytest.mark.parametrize("steps", [1, 10, 50])
def test_fp32_two_stream_matches_oracle_mode2(steps):
    wl = W.two_stream(particles_per_beam=512, nx=64, seed=3, steps=50)
    dev, ora2, ora1, _keep = _pair(wl)
    dev.step(steps)
    ora2.step(steps)
    ora1.step(steps)
    _check_mode2(dev, ora2, 2)
    for a, b in zip(dev.fields(), ora2.fields()):
        assert rel_max(a, b) < MAX_REL
    # error of the FP32 form against the FP64 oracle
    for s in range(2):
        a, b = dev.particles(s), ora1.particles(s)
        for k in ("x", "vh", "v"):
            assert rel_max(a[k], b[k]) < FP32_VS_FP64[k], (k, rel_max(a[k], b[k]))
    fe = dev.sample().field_energy
    assert abs(fe - ora1.field_energy()) <= FP32_VS_FP64["field_energy"] * abs(ora1.field_energy())


def test_fp32_ccp_mcc_matches_oracle_mode2():
    """Full discharge steps with MCC and ionization products: collision
    counts exact, state as above, FP32-vs-FP64 error within the stated bounds."""
    wl = W.ccp_helium(particles_per_cell=32, cells=64, seed=11, steps=20, table_rows=1024)
    dev, ora2, ora1, _keep = _pair(wl)
    dev.step(20)
    ora2.step(20)
    ora1.step(20)
    tot = dev.collision_totals()
    c, nl, per = ora2.collisions()
    assert tot.candidates == c and tot.null_collisions == nl
    for m in range(2):
        assert list(tot.channel_collisions[m])[:3] == list(per[m])[:3]
    for s in range(2):
        b = dev.boundary_losses(s)
        l, r, _, _ = ora2.losses(s)
        assert (b.absorbed_left, b.absorbed_right) == (l, r)
    _check_mode2(dev, ora2, 2)
    c1, _, _ = ora1.collisions()
    assert abs(c1 - c) <= 0.01 * c1  # the same physics as the FP64 form
    for s in range(2):
        a, b = dev.particles(s), ora1.particles(s)
        if len(a["x"]) != len(b["x"]):
            continue  # a wall loss or product on one side only
        for k in ("x", "vy", "vz"):
            assert rel_max(a[k], b[k]) < FP32_VS_FP64[k], (s, k, rel_max(a[k], b[k]))


def test_fp32_step_group_and_readback_idempotent():
    """Grouped FP32 runs end in the state of the same runs stepped alone, and a
    read-back in the middle of a run changes nothing when repeated."""
    decks = [W.ccp_helium(particles_per_cell=16, cells=64, seed=3, table_rows=256, te_ev=12.0),
             W.two_stream(particles_per_beam=2048, nx=64, seed=4)]

    def make(wl, k):
        cfg, tabs = W.to_device_config(wl, precision=apic.FP32_STORAGE, seed=77 + k)
        sim = apic.Simulation1D(cfg, tabs)
        load_device(sim, wl)
        sim.initialize()
        return sim, tabs

    grouped = [make(wl, k) for k, wl in enumerate(decks)]
    single = [make(wl, k) for k, wl in enumerate(decks)]
    apic.step_group([g for g, _ in grouped], 7)
    for s, _ in single:
        s.step(7)
    for (g, _), (s, _), wl in zip(grouped, single, decks):
        for k in range(len(wl.species)):
            a, b = g.particles(k), s.particles(k)
            c = g.particles(k)
            for key in a:
                assert np.array_equal(a[key], b[key]), key
                assert np.array_equal(a[key], c[key]), key
