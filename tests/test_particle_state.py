"""AuroraPIC particle-state files (.aps version 1) on the host: the library's
reader and writer against the reference's own (load_external_particle_state,
write_external_particle_state) compiled from its sources, and against a
committed file the reference wrote.  Records bit-exact, signatures equal,
written files byte-identical, the reference's error messages."""
import os

import numpy as np
import pytest

import apic
import pyoracle as po

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _state(dim, seed, counts=(("electrons", 7), ("ions", 5), ("beam", 3))):
    rng = np.random.default_rng(seed)
    sp = {}
    for name, n in counts:
        pos = rng.uniform(0.0, 1.0, (3, n)) * [[0.02], [0.01], [0.005]]
        vel = rng.standard_normal((3, n)) * 1e5
        if dim < 3:
            pos[2] = 0.0
        if dim == 1:
            pos[1] = 0.0
            vel[1:] = 0.0
        vel[0, 0] = -0.0  # signed zero survives both ways
        sp[name] = (pos, vel)
    return sp


def _need_ref():
    if not po.reference_available():
        pytest.skip("reference library not built")


@pytest.mark.parametrize("dim,units", [(1, apic.NORMALIZED), (2, apic.SI), (3, apic.SI)])
def test_reader_matches_reference_writer(tmp_path, dim, units):
    _need_ref()
    sp = _state(dim, 10 + dim)
    path = str(tmp_path / "ref.aps")
    sig = po.ref_aps_write(path, dim, int(units == apic.SI), sp)
    st = apic.ParticleState(path)
    assert (st.dimension, st.units, st.particle_count, st.signature) == (dim, units, 15, sig)
    assert list(st.species) == sorted(sp)
    for name, (pos, vel) in sp.items():
        assert np.array_equal(st.species[name][0], pos) and np.array_equal(st.species[name][1], vel)
        assert np.array_equal(np.signbit(st.species[name][1]), np.signbit(vel))


@pytest.mark.parametrize("dim,units", [(1, apic.NORMALIZED), (2, apic.NORMALIZED), (3, apic.SI)])
def test_writer_is_byte_identical_to_reference(tmp_path, dim, units):
    _need_ref()
    sp = _state(dim, 20 + dim)
    a, b = str(tmp_path / "ours.aps"), str(tmp_path / "ref.aps")
    sig = apic.ParticleState.write(a, dim, units, sp)
    ref_sig = po.ref_aps_write(b, dim, int(units == apic.SI), sp)
    assert sig == ref_sig
    assert open(a, "rb").read() == open(b, "rb").read()
    rsig, recs = po.ref_aps_read(a)
    assert rsig == sig
    for (pos, vel), name in zip(recs, sorted(sp)):
        assert np.array_equal(pos, sp[name][0]) and np.array_equal(vel, sp[name][1])


def test_committed_reference_file():
    """A file the reference wrote (tests/golden/state_2d.aps) and its signature."""
    g = np.load(os.path.join(GOLDEN, "state_2d.npz"))
    st = apic.ParticleState(os.path.join(GOLDEN, "state_2d.aps"))
    assert st.signature == int(g["signature"]) and st.dimension == 2 and st.units == apic.SI
    for k, name in enumerate(sorted(st.species)):
        assert np.array_equal(st.species[name][0], g[f"pos{k}"]) and np.array_equal(st.species[name][1], g[f"vel{k}"])


@pytest.mark.parametrize("body,message", [
    ("AuroraPIC-particle-state-v2\n", "invalid external particle-state magic"),
    ("AuroraPIC-particle-state-v1\ndimension 4\n", "invalid dimension"),
    ("AuroraPIC-particle-state-v1\ndimension 2\nunits cgs\n", "invalid units 'cgs'"),
    ("AuroraPIC-particle-state-v1\ndimension 2\nunits si\nweighting per_particle\n", "weighting species_constant"),
    ("AuroraPIC-particle-state-v1\ndimension 2\nunits si\nweighting species_constant\n"
     "velocity_staggering time_centered\nparticle_count 1\nrecords\nparticle e 0 0 1 0 0 0\nend\n",
     "nonzero inactive z position"),
    ("AuroraPIC-particle-state-v1\ndimension 1\nunits si\nweighting species_constant\n"
     "velocity_staggering time_centered\nparticle_count 1\nrecords\nparticle e 0 0 0 1 2 0\nend\n",
     "1D1V external particle state has nonzero inactive components"),
    ("AuroraPIC-particle-state-v1\ndimension 2\nunits si\nweighting species_constant\n"
     "velocity_staggering time_centered\nparticle_count 1\nrecords\nparticle e 0 0 0 1 2 0\nend\nextra\n",
     "trailing data"),
    ("AuroraPIC-particle-state-v1\ndimension 2\nunits si\nweighting species_constant\n"
     "velocity_staggering time_centered\nparticle_count 2\nrecords\nparticle e 0 0 0 1 2 0\nend\n",
     "expected key 'particle'"),
    ("AuroraPIC-particle-state-v1\ndimension 2\nunits si\nweighting species_constant\n"
     "velocity_staggering time_centered\nparticle_count 1\nrecords\nparticle e 0 0 0 1 nan 0\nend\n",
     "invalid external particle record 0"),
])
def test_rejects_like_the_reference(tmp_path, body, message):
    path = str(tmp_path / "bad.aps")
    open(path, "w").write(body)
    with pytest.raises(apic.ApicError, match=message):
        apic.ParticleState(path)
    if po.reference_available():
        with pytest.raises(RuntimeError, match=message):
            po.ref_aps_read(path)


def test_writer_refuses_to_overwrite(tmp_path):
    sp = _state(2, 3)
    path = str(tmp_path / "s.aps")
    apic.ParticleState.write(path, 2, apic.SI, sp)
    with pytest.raises(apic.ApicError, match="already exists"):
        apic.ParticleState.write(path, 2, apic.SI, sp)
    apic.ParticleState.write(path, 2, apic.SI, sp, overwrite=True)
