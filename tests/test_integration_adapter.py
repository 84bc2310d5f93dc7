"""The reference-side adapter of the integration guide (its C++ code block)
compiles against the
reference's own public headers and this library's C ABI, so a drift of either
side's field names breaks this test rather than a maintainer's build.  The
reference tree's location comes from oracle/Makefile (APIC_REFERENCE or its
default); the test is skipped where the tree is absent."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reference_include():
    try:
        out = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"], check=True,
                             capture_output=True, text=True).stdout.strip()
    except (OSError, subprocess.CalledProcessError):
        return None
    inc = os.path.join(out, "include")
    return inc if os.path.isfile(os.path.join(inc, "pic", "Simulation.hpp")) else None


def _adapter_source():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    section = text[text.index("## The adapter a maintainer adds"):]
    m = re.search(r"```cpp\n(.*?)```", section, re.S)
    assert m, "INTEGRATION.md has no adapter code block"
    return m.group(1)


def test_integration_adapter_compiles_against_the_reference_headers(tmp_path):
    inc = _reference_include()
    if inc is None:
        pytest.skip("reference source tree not present on this host")
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "adapter.cpp"
    src.write_text("#include <stdexcept>\n#include <string>\n#include <vector>\n" + _adapter_source())
    r = subprocess.run([gxx, "-std=c++20", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), "-I", inc,
                        str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
