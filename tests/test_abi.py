"""The C ABI library loads and exports every entry point include/*.h declares;
host-side behaviour that needs no GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import apic
from apic import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            text = open(os.path.join(inc, fn)).read()
            names |= set(re.findall(r"APIC_EXPORT\s+[\w\s\*]+?\b(apic_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = apic.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version():
    lib = apic.lib()
    assert b"sm_100a" in lib.apic_version()
    for code in range(11):
        assert lib.apic_status_string(code)


@pytest.mark.skipif(apic.lib().apic_device_count() > 0, reason="checks the no-device path")
def test_create_without_device_fails_loudly():
    wl = W.two_stream(particles_per_beam=64, nx=16)
    cfg, tabs = W.to_device_config(wl)
    with pytest.raises(apic.ApicError) as e:
        apic.Simulation1D(cfg, tabs)
    assert e.value.status == 10  # APIC_ERR_NO_DEVICE, never a CPU fallback


def test_workload_shapes():
    wl = W.ccp_helium()
    assert wl.nx == 513 and len(wl.species) == 2
    assert all(len(s.x) == 262144 for s in wl.species)
    assert abs(wl.dt - 1.0 / (400 * 13.56e6)) < 1e-24
    # max_frequency * dt stays well below 1 (the reference requires <= 0.1 for swarms)
    for m in wl.models:
        assert m.max_frequency * wl.dt < 0.1
    ts = W.two_stream()
    assert ts.nx == 256 and sum(len(s.x) for s in ts.species) == 32768
    assert np.all((ts.species[0].x >= 0) & (ts.species[0].x < ts.length))


def test_ctypes_structs_match_the_c_header(tmp_path):
    """Every struct the Python binding passes across the ABI has the C size."""
    names = {"apic_mcc_channel": apic.McChannel, "apic_mcc_model": apic.MccModel, "apic_config1d": apic.Config1D,
             "apic_config_nd": apic.ConfigND, "apic_sample_nd": apic.SampleND,
             "apic_swarm_config": apic.SwarmConfig, "apic_swarm_result": apic.SwarmResult,
             "apic_swarm_request": apic.SwarmRequest, "apic_swarm_server_config": apic.SwarmServerConfig}
    src = tmp_path / "sizes.c"
    body = "".join(f'    printf("{n} %zu\\n", sizeof({n}));\n' for n in names)
    src.write_text('#include <stdio.h>\n#include "aurorapic_b200.h"\nint main(void) {\n' + body + "    return 0;\n}\n")
    exe = tmp_path / "sizes"
    import subprocess
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    got = dict(zip(out[0::2], map(int, out[1::2])))
    for n, cls in names.items():
        assert got[n] == C.sizeof(cls), (n, got[n], C.sizeof(cls))


def test_swarm_request_validation_on_cpu():
    """Server creation needs a device; its absence is reported, never hidden."""
    spec = W.swarm_c5(particles=1000, steps=100, burn_in_steps=50)
    cfg, gas, tabs = W.to_device_swarm(spec)
    if apic.lib().apic_device_count() > 0:
        pytest.skip("checks the no-device path")
    with pytest.raises(apic.ApicError):
        apic.swarm_run(cfg, gas, [10.0])


def build_facade_check(tmp_path):
    import subprocess
    exe = tmp_path / "facade_check"
    subprocess.run(["g++", "-std=c++20", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "facade_check.cpp"), "-L", os.path.dirname(apic.library_path()),
                    "-laurorapic_b200", "-Wl,-rpath," + os.path.dirname(apic.library_path()), "-o", str(exe)],
                   check=True)
    return exe


def test_cpp20_facade_compiles_and_maps_errors(tmp_path):
    """The C++20 facade (include/aurorapic_b200.hpp) builds against the
    library; without a device, creation raises runtime_error and a bad
    configuration keeps the reference's invalid_argument."""
    import subprocess
    if apic.lib().apic_device_count() > 0:
        pytest.skip("checks the no-device path")
    out = subprocess.run([str(build_facade_check(tmp_path))], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "invalid_argument: simulation dt must be positive and finite" in out.stdout


@pytest.mark.parametrize("walls,msg", [
    (((1, 1, 0), None, (0,) * 6), "3D meshes are periodic or Dirichlet on every axis"),
    (((1, 1, 1), (0.0, 1.0, 0.0, 0.0), (0,) * 6), "3D Dirichlet walls are grounded"),
    (((1, 1, 1), None, (0, 0, 0, 0, 0, 7)), "unknown particle boundary"),
])
def test_3d_wall_configuration_checks(walls, msg):
    """A 3D mesh is periodic or Dirichlet as a whole, with grounded walls
    (Simulation3DConfig's single field boundary, src/Mesh3D.cpp:37-48,
    src/FieldSolver.cpp:351-372); create rejects anything else before it looks
    for a device."""
    cfg = apic.config_nd(dims=3, n=(9, 9, 9), length=(1.0, 1.0, 1.0), dt=0.1,
                         species=[(-1.0, 1.0, 1.0, 16)], walls=walls)
    with pytest.raises(apic.ApicError) as e:
        apic.SimulationND(cfg)
    assert msg in str(e.value)


@pytest.mark.parametrize("bgk,models,msg", [
    ((-1.0, 1.0), False, "collision frequency must be non-negative and finite"),
    ((float("nan"), 1.0), False, "collision frequency must be non-negative and finite"),
    ((1.0, -2.0), False, "neutral_temperature_velocity must be non-negative and finite"),
    ((1.0e8, 1.0e5), True, "named collision models cannot be combined with the legacy collision model"),
])
def test_bgk_configuration_checks(bgk, models, msg):
    """The legacy BGK model's checks (src/Simulation.cpp:95-100, :388-392) run
    in create before it looks for a device."""
    from apic import workloads as W
    wl = W.ccp_helium(particles_per_cell=2, cells=8, seed=1, steps=1, table_rows=16, bgk=bgk)
    if models:
        wl.models = W.ccp_helium(particles_per_cell=2, cells=8, seed=1, steps=1, table_rows=16).models
    cfg, tabs = W.to_device_config(wl)
    with pytest.raises(apic.ApicError) as e:
        apic.Simulation1D(cfg, tabs)
    assert msg in str(e.value)
