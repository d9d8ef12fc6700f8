"""The C-ABI library loads and exports every symbol include/psb200.h declares;
the pybind11 module exposes the reference module's names; without a GPU every
compute call fails loudly (no CPU fallback)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "psb200.h"
LIB = ROOT / "psacking_b200" / "libpsb200.so"

REFERENCE_EXPORTS = [  # spectral_packing/bindings.cpp:681-924
    "fft_search_placement", "fft_search_placement_with_cache", "place_in_tray", "dft_conv3",
    "dft_corr3", "calculate_distance", "collision_grid", "make_tight", "get_bounds",
    "gpu_tray_init", "gpu_tray_cleanup", "gpu_tray_is_initialized", "gpu_tray_search",
    "fft_search_batch", "fft_search_batch_interlocking_free", "interlocking_free_positions",
    "voxelize_stl", "save_vox",
]


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(psb_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "psb_tray_search" in syms and "psb_pack" in syms and len(syms) >= 18


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(LIB))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    lib.psb_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.psb_version()
    n = ctypes.c_int(-1)
    assert lib.psb_device_count(ctypes.byref(n)) == 0 and n.value >= 0


def test_core_module_mirrors_reference(core):
    for name in REFERENCE_EXPORTS:
        assert callable(getattr(core, name)), name
    assert core.VOXEL_RESOLUTION == 128
    assert core.HEIGHT_PENALTY == 1e8
    assert core.__version__ == "0.1.0"
    import psacking_b200 as p
    for name in REFERENCE_EXPORTS + ["save_vox", "voxelize_stl", "BinPacker"]:
        assert hasattr(p, name), name


def test_core_save_vox_writes_the_package_encoding(core, tmp_path):
    from psacking_b200.vox import encode_vox
    g = np.zeros((3, 4, 5), np.int32)
    g[0, 1, 2] = 1
    g[2, 3, 4] = 8
    core.save_vox(g, str(tmp_path / "a.vox"))
    assert (tmp_path / "a.vox").read_bytes() == encode_vox(g)


def test_wrong_dimensions_raise(core):
    # bindings.cpp:75-78 / tests/test_bindings.py:276-284
    with pytest.raises(RuntimeError, match="3-dimensional"):
        core.fft_search_placement(np.ones((3, 3), np.int32), np.zeros((5, 5, 5), np.int32))


def test_host_utilities(core):
    from oracle import psb_oracle as O
    g = np.zeros((5, 5, 5), np.int32)
    g[1:3, 0:2, 1:4] = 1
    assert core.get_bounds(g) == ((1, 0, 1), (2, 1, 3))
    assert core.make_tight(g).shape == (2, 2, 3)
    assert core.get_bounds(np.zeros((2, 2, 2), np.int32)) == O.bounds(np.zeros((2, 2, 2)))
    with pytest.raises(ValueError):
        core.make_tight(np.zeros((2, 2, 2), np.int32))


def test_no_gpu_fails_loudly(core):
    if core.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(RuntimeError, match="CUDA"):
        core.calculate_distance(np.zeros((4, 4, 4), np.int32))
    with pytest.raises(RuntimeError):
        core.fft_search_placement(np.ones((2, 2, 2), np.int32), np.zeros((6, 6, 6), np.int32))


def test_context_calls_from_threads_are_serialised(core):
    """The module's process-wide search context is guarded by a mutex that
    is only waited for with the GIL released, and the engine's cached
    contexts of the stateless searches by a call lock: calls that use them
    from several Python threads at once neither deadlock nor crash.  Without
    a GPU every such call raises, which exercises the locks on the error
    path too."""
    import threading
    if core.device_count() > 0:
        pytest.skip("a GPU is visible (the GPU tests cover the context itself)")
    tray = np.zeros((6, 6, 6), np.int32)
    phi = np.zeros_like(tray)
    item = np.ones((2, 2, 2), np.int32)
    errors, done = [], []

    def worker(k):
        for g in range(20):
            for call in (lambda: core.gpu_tray_init(tray, phi),
                         lambda: core.fft_search_batch([item], tray, phi, 1000 * k + g),
                         lambda: core.fft_search_placement_with_cache(item, tray, phi, 1000 * k + g),
                         lambda: core.gpu_tray_search(item),
                         lambda: core.fft_search_placement(item, tray)):
                try:
                    call()
                except RuntimeError as e:
                    errors.append(str(e))
            core.gpu_tray_is_initialized()
            core.gpu_tray_cleanup()
        done.append(k)
    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    assert sorted(done) == [0, 1, 2, 3]
    assert len(errors) == 4 * 20 * 5
    assert not core.gpu_tray_is_initialized()


def test_is_cuda_available_reports_the_device(core):
    import psacking_b200 as p
    assert p.is_cuda_available() == (core.device_count() > 0)


def test_product_never_reaches_the_oracle():
    """The oracle is test infrastructure only: no module of the package
    imports it, no native source includes or links anything under oracle/,
    and importing the whole package (every module) leaves it unloaded."""
    import ast
    import subprocess
    import sys
    pkg = ROOT / "psacking_b200"
    for py in pkg.rglob("*.py"):
        tree = ast.parse(py.read_text())
        for node in ast.walk(tree):
            names = []
            if isinstance(node, ast.Import):
                names = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom) and node.level == 0:
                names = [node.module or ""]
            assert not any(n.split(".")[0] == "oracle" for n in names), (py, names)
    for src in list((pkg / "csrc").iterdir()) + [pkg / "build.py"]:
        text = src.read_text()
        assert "oracle/" not in text and '"oracle' not in text, src
    mods = sorted(p.stem for p in pkg.glob("*.py") if p.stem != "__init__")
    code = ("import importlib, sys, psacking_b200\n"
            f"for m in {mods!r}:\n"
            "    importlib.import_module('psacking_b200.' + m)\n"
            "print(sorted(k for k in sys.modules if k.split('.')[0] == 'oracle'))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "[]"


def test_header_cites_each_entry_point():
    """Every declaration in include/psb200.h sits under a comment that
    cites the reference interface it replaces (file:line) or says that it
    has no counterpart in the reference."""
    text = HEADER.read_text()
    decls = list(re.finditer(r"^(?:int|void|const char\*)\s+(psb_[a-z0-9_]+)\(", text, re.M))
    assert len(decls) >= 50
    prev, section, missing = 0, "", []
    for m in decls:
        chunk = text[prev:m.start()]
        prev = m.end()
        if "/* ----" in chunk:
            section = chunk[chunk.rfind("/* ----"):]
        if not re.search(r"\.(cpp|cu|py|h):\d|counterpart|[Rr]eplaces", chunk + section):
            missing.append(m.group(1))
    assert not missing, missing
