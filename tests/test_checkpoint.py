"""1D3V checkpoints (.apc version 12) on the host: files the reference's own
Simulation::save_checkpoint wrote (the reference compiled from its sources)
are read and written back byte-identical, their parts equal what the reference
holds, and damaged files fail with the reference's messages."""
import os
import tempfile

import numpy as np
import pytest

import apic
import pyoracle as po
from apic import workloads as W


def _reference_checkpoint(wl, steps, seed=777):
    T = po.TableSet()
    cfg = po.config_from_workload(wl, T, seed=seed)
    d = tempfile.mkdtemp()
    ref = po.Ref1D(cfg, d)
    ref.initialize()
    ref.step(steps)
    path = os.path.join(d, "ref.apc")
    ref.save_checkpoint(path)
    return ref, path, T


def _decks():
    mcc = W.ccp_helium(particles_per_cell=8, cells=32, seed=11, table_rows=256, te_ev=30.0)
    rf = W.ccp_helium(particles_per_cell=8, cells=32, seed=12, table_rows=256)
    rf.models = []
    ts = W.two_stream(particles_per_beam=256, nx=32, seed=3)
    # the legacy BGK model (one "bgk" channel and its signature line)
    bgk = W.ccp_helium(particles_per_cell=8, cells=32, seed=13, table_rows=64, te_ev=4.0, bgk=(2.0e8, 3.0e5))
    return {"mcc": (mcc, 12), "rf": (rf, 30), "two_stream": (ts, 20), "bgk": (bgk, 25)}


@pytest.mark.parametrize("case", ["mcc", "rf", "two_stream", "bgk"])
def test_reference_checkpoint_round_trip_is_byte_identical(case, tmp_path):
    if not po.reference_available():
        pytest.skip("reference library not built on this host")
    wl, steps = _decks()[case]
    ref, path, _keep = _reference_checkpoint(wl, steps)
    c = apic.Checkpoint(path)
    out = str(tmp_path / "again.apc")
    c.write(out)
    assert open(out, "rb").read() == open(path, "rb").read()
    info = c.info()
    assert info.step == steps and abs(info.time - ref.time()) == 0.0
    assert info.nspecies == len(wl.species)
    for s in range(len(wl.species)):
        p = c.particles(s)
        r = ref.particles(s)
        for k in ("x", "v", "vy", "vz", "vh"):
            assert np.array_equal(p[k], r[k]), (s, k)
        assert np.array_equal(p["alive"], r["alive"])
        name, n, loss, work = c.species(s)
        l, rr, el, er = ref.losses(s)
        assert (loss.absorbed_left, loss.absorbed_right) == (l, rr)
        assert loss.kinetic_energy_left == el and loss.kinetic_energy_right == er
        assert work == ref.electric_work(s)
    cand, nulls, per = ref.collisions()
    assert (info.candidates, info.null_collisions) == (cand, nulls)
    assert [c.channel(k)[0] for k in range(info.nchannels)] == list(per)


def test_damaged_checkpoints_fail_with_the_reference_messages(tmp_path):
    if not po.reference_available():
        pytest.skip("reference library not built on this host")
    wl, steps = _decks()["rf"]
    _ref, path, _keep = _reference_checkpoint(wl, 3)
    text = open(path).read()
    cases = {
        "magic": (text.replace("AuroraPIC-checkpoint-v12", "not-a-checkpoint", 1), "invalid checkpoint magic in:"),
        "old": (text.replace("AuroraPIC-checkpoint-v12", "AuroraPIC-checkpoint-v11", 1), "is not supported"),
        "dimension": (text.replace("dimension 1", "dimension 2", 1), "checkpoint dimension does not match 1D simulation"),
        "truncated": (text[: len(text) - 200], "failed while reading checkpoint:"),
        "no_rng": (text.replace("\nrng ", "\nrnq ", 1), "checkpoint missing rng state"),
    }
    for name, (body, msg) in cases.items():
        p = tmp_path / f"{name}.apc"
        p.write_text(body)
        with pytest.raises(apic.ApicError) as e:
            apic.Checkpoint(str(p))
        assert msg in str(e.value), (name, str(e.value))


def _oracle_from_checkpoint(wl, c, seed, T):
    ora = po.Sim1D(po.config_from_workload(wl, T), 1, seed)
    for s in range(len(wl.species)):
        p = c.particles(s)
        ora.load(s, p["x"], p["v"], p["vh"], p["vy"], p["vz"], p["alive"])
    info = c.info()
    ora.initialize_fields(info.time, info.step)
    return ora


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["rf", "mcc", "bgk"])
def test_device_restart_from_a_reference_checkpoint(case, tmp_path):
    """A device run restarted from a file the reference wrote matches the
    oracle restarted from the same file: FP64 state within 1e-11 after 10
    more steps, collision counts exact (the oracle's device-form streams), the
    file's totals carried forward."""
    if not po.reference_available():
        pytest.skip("reference library not built on this host")
    from common import rel_max
    wl, steps = _decks()[case]
    _ref, path, T = _reference_checkpoint(wl, steps)
    c = apic.Checkpoint(path)
    seed = 0x5EED
    cfg, tabs = W.to_device_config(wl, seed=seed)
    dev = apic.Simulation1D(cfg, tabs)
    dev.load_checkpoint(c)
    ora = _oracle_from_checkpoint(wl, c, seed, T)
    dev.step(10)
    ora.step(10)
    for s in range(len(wl.species)):
        a, b = dev.particles(s), ora.particles(s)
        assert len(a["x"]) == len(b["x"])
        for k in ("x", "v", "vh", "vy", "vz"):
            assert rel_max(a[k], b[k]) < 1e-11, (s, k)
    tot = dev.collision_totals()
    info = c.info()
    cand, nulls, per = ora.collisions()
    assert tot.candidates - info.candidates == cand and tot.null_collisions - info.null_collisions == nulls
    assert dev.sample().step == info.step + 10
    dev.close()


@pytest.mark.gpu
def test_device_checkpoint_loads_in_the_reference(tmp_path):
    """A checkpoint the device writes is read by the reference's own
    load_checkpoint, and the reference then holds exactly the device's
    particles, step and time."""
    if not po.reference_available():
        pytest.skip("reference library not built on this host")
    wl, steps = _decks()["mcc"]
    ref, path, T = _reference_checkpoint(wl, steps)
    meta = apic.Checkpoint(path)
    cfg, tabs = W.to_device_config(wl, seed=3)
    dev = apic.Simulation1D(cfg, tabs)
    dev.load_checkpoint(meta)
    dev.step(7)
    out = str(tmp_path / "device.apc")
    dev.save_checkpoint(meta, out)
    mine = apic.Checkpoint(out)
    again = str(tmp_path / "again.apc")
    mine.write(again)
    assert open(again, "rb").read() == open(out, "rb").read()
    ref.load_checkpoint(out)
    assert abs(ref.time() - dev.time) == 0.0
    for s in range(len(wl.species)):
        a, b = dev.particles(s), ref.particles(s)
        for k in ("x", "v", "vh", "vy", "vz"):
            assert np.array_equal(a[k], b[k]), (s, k)
    dev.close()
