"""CPU checks of the C ABI library: it loads without a GPU and exports every function
that include/*.h declares; calls that need no device report errors cleanly."""
import ctypes
import importlib
import re
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT

N = importlib.import_module("2023_render_engine_b200._native")


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:RT_API\s+)?(?:int|void|const char\s*\*)\s+(rt_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_functions():
    assert {"rt_trace_closest", "rt_scene_commit", "rt_context_create"} <= declared_functions()


def test_library_exports_every_declared_symbol():
    lib = N.load()
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = declared_functions() - exported
    assert not missing, missing
    for name in declared_functions():
        assert getattr(lib, name) is not None


def test_python_binding_covers_declarations():
    assert declared_functions() <= set(N.SIGNATURES)


def test_abi_version_and_errors_without_gpu():
    lib = N.load()
    assert lib.rt_abi_version() == 2
    # null arguments are rejected before any device work
    assert lib.rt_scene_commit(None) == 1
    assert "null" in N.last_error()
    assert lib.rt_trace_counts(None, None, 0, 0, None) == 1
    assert "rt_trace_counts" in N.last_error()
    assert lib.rt_render_stage_times(None, None, 0) == 1
    assert "rt_render_stage_times" in N.last_error()
    h = ctypes.c_void_p()
    st = lib.rt_context_create(0, ctypes.byref(h))
    import torch

    if not torch.cuda.is_available():
        assert st != 0  # no device here: a clean error, not a crash
