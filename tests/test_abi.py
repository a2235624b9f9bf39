"""The C-ABI library loads and exports every entry point include/pdb200.h declares (no GPU call)."""
import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared():
    text = (ROOT / "include" / "pdb200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pd_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(pd):
    pd.build()
    import ctypes
    lib = ctypes.CDLL(str(pd._native.LIB_PATH))
    names = declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(pd._native.LIB_PATH)], capture_output=True, text=True)
    exported = set(re.findall(r" T (pd_\w+)", out.stdout))
    assert set(names) <= exported


def test_python_binding_covers_the_header(pd):
    assert set(declared()) == set(pd._native.EXPORTED)


def test_no_cpu_fallback(pd, monkeypatch, tmp_path):
    # the product fails loudly when the CUDA library is missing
    import importlib
    n = pd._native
    monkeypatch.setattr(n, "_lib", None)
    monkeypatch.setattr(n, "LIB_PATH", tmp_path / "missing.so")
    try:
        n.lib()
    except RuntimeError as e:
        assert "no CPU fallback" in str(e)
    else:
        raise AssertionError("loading a missing library must fail")


def test_status_strings(pd):
    pd.build()
    L = pd._native.lib()
    assert L.pd_version() >= 100
    assert L.pd_strerror(3).decode() == "outer cluster list capacity exceeded"
