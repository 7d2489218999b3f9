"""The C ABI: the library loads and exports every function declared in include/*.h; without a GPU
it refuses cleanly (no CPU fallback); the CLI drop-in starts."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

from conftest import PKG, ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            before = text[:m.start()].rstrip()
            # a declaration: preceded by a type (identifier or '*'), not a keyword/macro use
            if name in ("if", "for", "while", "switch", "return", "sizeof", "defined"):
                continue
            if before.endswith(("*", ")")) and not before.endswith("(*"):
                pass
            if re.search(r"[A-Za-z0-9_\*]\s*$", before) and not before.endswith("(*"):
                names.add(name)
    # function-pointer parameter names are not exports
    return sorted(n for n in names if n not in ("setup", "cleanup", "f_seq", "f_par"))


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(os.path.join(PKG, "libgnncolor.so"))
    names = declared_functions()
    assert "gc_color" in names and "jones_plassmann_internal" in names and "cgnn_graph_sage_16_par" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert hasattr(lib, "layers")  # the reference's global model depth (src/gnn.c:18)


def test_no_gpu_means_no_fallback():
    import gnn_coloring as gcn
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(gcn.GCError) as e:
        gcn.Context(0)
    assert e.value.name == "GC_ERR_NODEV"


def test_status_strings():
    import gnn_coloring as gcn
    for code in range(10):
        assert gcn.lib.gc_status_string(code)


def test_cli_starts():
    exe = os.path.join(PKG, "cli", "coloring")
    r = subprocess.run([exe, "-h"], capture_output=True, text=True, timeout=30)
    assert r.returncode == 0 and "Usage" in r.stdout
    r = subprocess.run([exe, "-g", "/nonexistent.mtx"], capture_output=True, text=True, timeout=30)
    assert r.returncode == 1 and "Unable to open file" in r.stdout
    r = subprocess.run([exe, "-x"], capture_output=True, text=True, timeout=30)
    assert r.returncode == 1


REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "coloring_main")


def test_reference_main_links_against_the_library_alone():
    """INTEGRATION.md option 2: the reference's unmodified src/main.c, compiled against include/ and
    linked against libgnncolor.so (oracle/Makefile builds it where the reference sources exist),
    needs nothing else of the reference and starts without a GPU."""
    if not os.path.exists(REF_MAIN):
        pytest.skip("the reference's main.c was not compiled here (reference sources absent at build time)")
    ldd = subprocess.run(["ldd", REF_MAIN], capture_output=True, text=True, timeout=60).stdout
    assert "libgnncolor.so" in ldd and "libref" not in ldd, ldd
    r = subprocess.run([REF_MAIN, "-h"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.startswith("GNN-based greedy graph coloring")
