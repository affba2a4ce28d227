"""CPU checks of the C-ABI library: it loads, exports every declared entry point, and refuses
to run without a CUDA device (no CPU fallback)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "phl_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:int|void|const char|void \*)\s*\*?\s*(phl_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib_path():
    import importlib
    return importlib.import_module("phlegethon_b200.build").build(force=False)


def test_library_exports_every_declared_symbol(lib_path):
    lib = C.CDLL(lib_path)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from phlegethon_b200 import abi
    assert sorted(abi.EXPORTS) == names


def test_abi_version_and_errors(lib_path):
    from phlegethon_b200 import abi
    lib = abi.load_library(lib_path)
    assert lib.phl_abi_version() == abi.ABI_VERSION
    assert lib.phl_error_string(-1).decode().startswith("invalid")


def test_no_cpu_fallback(lib_path):
    """Without a GPU, phl_init reports PHL_E_NO_DEVICE instead of running anything on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from phlegethon_b200 import abi, problems
    cfg, _ = problems.hot_bubble_2d(16)
    with pytest.raises(abi.PhlError) as e:
        abi.Simulation(cfg)
    assert e.value.code == -5


def test_invalid_config_rejected_before_device_use(lib_path):
    from phlegethon_b200 import abi, problems
    lib = abi.load_library(lib_path)
    cfg, _ = problems.hot_bubble_2d(16)
    s = abi.make_config_struct(cfg)
    s.nvars = 99
    ctx = C.c_void_p()
    assert lib.phl_init(C.byref(s), C.byref(ctx)) == -1
    s = abi.make_config_struct(cfg)
    s.abi_version = 12345
    assert lib.phl_init(C.byref(s), C.byref(ctx)) == -1


def test_bench_algorithmic_bytes():
    """Algorithmic HBM bytes per zone-update used for the roofline (derivations in bench.py)."""
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location("bench", os.path.join(os.path.dirname(__file__), "..", "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    from phlegethon_b200 import problems
    cfg, _ = problems.stratified_3d(8)
    assert bench.step_bytes_per_cell(cfg.replace(precision="fp64")) == 888 + 8 * 3 * 2 * 7 * 3
    assert bench.step_bytes_per_cell(cfg.replace(precision="fp32_split")) == 776
    cfgm, _ = problems.stratified_3d(8, mhd=True)
    assert bench.step_bytes_per_cell(cfgm.replace(precision="fp32_split")) == 2072
    # roofline numerators: algorithmic bytes, below the materialised traffic model
    assert bench.algorithmic_bytes_per_cell("stratified_mhd", "fp32_split") == 904
    assert bench.algorithmic_bytes_per_cell("stratified_mhd", "fp64") == 1120
    assert bench.algorithmic_bytes_per_cell("stratified", "fp32_split") == 712
    assert bench.algorithmic_bytes_per_cell("hot_bubble", "fp64") == 448
    name, launches = bench.stage_kernels(cfgm.replace(precision="fp32_split"), "fp32_split")
    assert "k_face_split_mhd" in name and launches == 3 * (3 + 3 + 3 + 1) + 2


def test_python_binding_matches_header_arity(lib_path):
    """Every entry point bound in phlegethon_b200.abi takes as many arguments as its prototype
    in include/phl_gpu.h declares (a drifted binding would pass garbage across the ABI)."""
    from phlegethon_b200 import abi
    lib = abi.load_library(lib_path)
    src = open(os.path.join(ROOT, "include", "phl_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    protos = dict(re.findall(r"\b(phl_\w+)\s*\(([^()]*)\)\s*;", src, flags=re.S))
    assert set(abi.EXPORTS) <= set(protos)
    for name in abi.EXPORTS:
        params = protos[name].strip()
        n = 0 if params in ("", "void") else len(params.split(","))
        assert len(getattr(lib, name).argtypes) == n, name


def test_bench_reference_arm_line():
    """`bench.py --impl reference` (the oracle on the host's cores) prints one JSON line with the
    contract's keys and the GPU arm's workload keys; the 256^2 hot bubble keeps it short."""
    import json
    import subprocess
    import sys
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config",
                        "hot_bubble", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "zone-updates/s" and d["value"] > 0
    assert d["config"]["workload"] == "hot_bubble" and d["config"]["n"] == 256
    assert d["config"]["cells"] == 256 * 256
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
