"""CPU tests of the C-ABI boundary: the library loads and exports every entry
point declared in include/*.h (no compute calls: this host has no GPU)."""
import ctypes
import glob
import os
import re

from alpine_b200 import build, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(alpine_gpu_\w+)\s*\(", src))
    return sorted(names)


def test_library_builds_and_loads():
    path = build.build()
    assert os.path.exists(path)
    gpu.lib()


def test_every_declared_symbol_is_exported():
    names = _declared()
    assert len(names) >= 12, names
    L = ctypes.CDLL(build.build())
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_header_is_plain_c():
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        raw = open(h).read()
        code = re.sub(r"/\*.*?\*/", "", raw, flags=re.S)
        assert "torch" not in code and "std::" not in code and "class " not in code, h
        assert 'extern "C"' in raw, h


def test_create_without_gpu_fails_cleanly():
    """No GPU here: create must return an error code, not crash."""
    import torch

    if torch.cuda.is_available():
        return
    L = gpu.lib()
    h = ctypes.c_void_p()
    cfg = gpu.Config(0, 0, 0, 8)
    rc = L.alpine_gpu_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc != 0 and not h.value
