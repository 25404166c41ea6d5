"""The product never routes through the oracle.

The oracle (oracle/, the CPU restatement of rblas's GEMM) is the checker
only: the package's sources never name it, and the built library links
nothing of it (its dynamic dependencies are the C/C++ runtime only; the
CUDA runtime is linked statically and the driver is reached at run time)."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "rblas_b200")


def test_package_sources_never_name_the_oracle():
    hits = []
    for dirpath, _, files in os.walk(PKG):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".rs", ".toml")):
                path = os.path.join(dirpath, f)
                if "oracle" in open(path, errors="replace").read():
                    hits.append(os.path.relpath(path, ROOT))
    assert not hits, f"product sources that name the oracle: {hits}"


def test_library_links_no_oracle_code():
    lib = os.path.join(PKG, "librblas_b200.so")
    if not os.path.exists(lib):
        pytest.skip("library not built")
    readelf = shutil.which("readelf")
    if not readelf:
        pytest.skip("readelf not available")
    out = subprocess.run([readelf, "-d", lib], capture_output=True, text=True, check=True).stdout
    needed = [ln.split("[", 1)[1].rstrip("]") for ln in out.splitlines() if "(NEEDED)" in ln]
    assert needed, "no dynamic dependencies listed"
    assert not [n for n in needed if "oracle" in n], needed
    allowed = ("libstdc++", "libm.", "libgcc_s", "libc.", "ld-linux", "libdl", "libpthread", "librt")
    assert all(n.startswith(allowed) for n in needed), needed


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """Without librblas_b200.so the binding raises at load time; nothing
    falls back to another implementation."""
    from rblas_b200 import _lib

    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "librblas_b200.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError, match="no CPU fallback"):
        _lib.load()
