"""CPU check of the build: no kernel is defined in both CUDA translation units.

The FP64 unit (phl_runtime.cu, no FMA contraction) and the FP32 split unit (phl_split.cu,
contraction and approximate division) include the same kernel templates.  The host stub of a
template kernel is a weak symbol, so one instantiated in both units under the same name would be
linked once for two device images, and which image a launch runs would depend on module load
order -- an FP64 launch could silently run FMA-contracted code.  Each unit therefore puts its
kernels in a namespace of its own; this test reads the symbol tables of the two objects and
fails if any function of namespace phl is defined in both.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "phlegethon_b200", "_build")


def defined_symbols(obj):
    out = subprocess.run(["nm", "-C", "--defined-only", obj], check=True, capture_output=True, text=True).stdout
    names = set()
    for line in out.splitlines():
        parts = line.split(None, 2)
        if len(parts) == 3 and parts[1] in ("T", "W", "V", "u"):
            names.add(parts[2])
    return names


@pytest.mark.skipif(shutil.which("nm") is None, reason="binutils nm not installed")
def test_no_kernel_defined_in_two_units():
    import importlib
    importlib.import_module("phlegethon_b200.build").build(force=False)
    a = defined_symbols(os.path.join(BUILD, "phl_runtime.o"))
    b = defined_symbols(os.path.join(BUILD, "phl_split.o"))
    shared = sorted(s for s in a & b if re.search(r"\bphl::", s) and not s.startswith(("typeinfo", "vtable")))
    assert not shared, shared[:10]
    # the per-unit namespaces are in place (an FP64 kernel and a split kernel of each kind)
    assert any("phl::fp64_unit::k_dt<" in s for s in a)
    assert any("phl::fp64_unit::k_init_thermo<" in s for s in a)
    assert not any("k_dt<" in s or "k_init_thermo<" in s for s in b)
