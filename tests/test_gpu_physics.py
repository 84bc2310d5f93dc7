"""Physics the device step must reproduce (kinetic validation of the 1D path):
the two-stream growth rate and the Landau damping rate against linear theory."""
import math

import numpy as np
import pytest

import apic
from apic import workloads as W
from common import load_device

pytestmark = pytest.mark.gpu


def field_energy_history(wl, steps):
    cfg, tabs = W.to_device_config(wl)
    sim = apic.Simulation1D(cfg, tabs)
    load_device(sim, wl)
    sim.initialize()
    t, fe = [0.0], [sim.sample().field_energy]
    for _ in range(steps):
        sim.step(1)
        s = sim.sample()
        t.append(s.time)
        fe.append(s.field_energy)
    sim.close()
    return np.array(t), np.array(fe)


def test_two_stream_growth_rate():
    """Symmetric cold beams at +/-1 (omega_p = 1, k = 0.5): the field energy of
    the only unstable mode grows as exp(2 gamma t), gamma = 0.3406 from
    (w^2 - a^2)^2 = 2 w_b^2 (w^2 + a^2), a = k v0, w_b^2 = 1/2."""
    a2, wb2 = 0.25, 0.5
    x = ((2 * a2 + 2 * wb2) - math.sqrt((2 * a2 + 2 * wb2) ** 2 - 4 * (a2 * a2 - 2 * wb2 * a2))) / 2
    gamma = math.sqrt(-x)
    t, fe = field_energy_history(W.two_stream(particles_per_beam=16384, nx=256, seed=1), 200)
    # linear phase of the seeded mode: after the loading noise (t < 8), before
    # saturation (t ~ 18); the beams' 0.01 thermal spread and the particle
    # noise put the measured rate about 10% under the cold-beam value (the CPU
    # restatement of the reference's step gives 0.305 on this deck)
    sel = (t >= 8.0) & (t <= 16.0)
    slope = np.polyfit(t[sel], np.log(fe[sel]), 1)[0]
    assert abs(slope / 2 - gamma) < 0.15 * gamma, (slope / 2, gamma)
    assert abs(slope / 2 - 0.3054) < 0.01, slope / 2


def test_landau_damping_rate():
    """k lambda_D = 0.5: the field energy oscillates at 2 omega_r and decays as
    exp(2 gamma t) with gamma = -0.1533; the peaks' log-linear fit over the
    first damping decade recovers it within 10%."""
    t, fe = field_energy_history(W.landau(), 300)
    peaks = [i for i in range(1, len(fe) - 1) if fe[i] > fe[i - 1] and fe[i] >= fe[i + 1] and 1.0 < t[i] < 18.0]
    assert len(peaks) >= 6
    slope = np.polyfit(t[peaks], np.log(fe[peaks]), 1)[0]
    assert abs(slope / 2 - (-0.1533)) < 0.1 * 0.1533, slope / 2
    period = 2 * np.mean(np.diff(t[peaks]))  # field energy peaks twice per period
    assert abs(2 * math.pi / period - 1.4156) < 0.05 * 1.4156
