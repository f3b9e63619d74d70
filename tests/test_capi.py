"""The C-ABI library loads and exports every declared entry point (CPU only)."""
import ctypes
import re
from pathlib import Path

import pytest

import lpa_b200 as L

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(lpa_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "lpa_create" in names and "lpa_iterate" in names and "lpa_decode_csr" in names
    assert len(names) >= 30


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    lib = ctypes.CDLL(str(L.LIB_PATH))
    assert hasattr(lib, name), name


def test_library_binds_every_symbol_at_load():
    """Immediate binding in a fresh process: no symbol is left undefined for a
    later call to trip over."""
    import subprocess
    import sys

    code = f"import ctypes, os; ctypes.CDLL({str(L.LIB_PATH)!r}, mode=os.RTLD_NOW)"
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr


def test_status_strings():
    lib = L.lib()
    for s in L.Status:
        assert lib.lpa_status_str(int(s))
    assert b"sm_100a" in lib.lpa_version()


def test_create_without_device_or_bad_args_fails_loudly():
    """No CPU fallback: without a usable device lpa_create reports an error."""
    import torch
    g = L.HostGraph.road(8, 8).compress(0, 128)
    desc = g.desc()
    if not torch.cuda.is_available():
        with pytest.raises(L.LpaError) as e:
            L.Propagator(g)
        assert e.value.status in (L.Status.NO_DEVICE, L.Status.CUDA)
    # invalid descriptors are rejected before any device work
    bad = L.GraphDesc()
    ctypes.memmove(ctypes.byref(bad), ctypes.byref(desc), ctypes.sizeof(desc))
    bad.num_compressed = desc.num_vertices + 1
    out = ctypes.c_void_p()
    assert L.lib().lpa_create(ctypes.byref(bad), None, ctypes.byref(out)) == L.Status.INVALID_ARG
