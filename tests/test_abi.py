"""The C-ABI library loads and exports every entry point include/*.h declares
(no device work: this runs without a GPU)."""
import ctypes
import re

import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(khrr_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("khrr_create", "khrr_accel", "khrr_phi", "khrr_integ_time", "khrr_step",
                 "khrr_upload_state", "khrr_conservation"):
        assert must in names


def test_library_exports_every_declared_symbol(libkhrr):
    missing = [n for n in declared_functions() if not hasattr(libkhrr, n)]
    assert not missing, f"not exported: {missing}"


def test_abi_version_and_status_names(libkhrr):
    import khrr
    L = khrr.lib()
    assert L.khrr_abi_version() == 1
    assert L.khrr_status_name(5) == b"KHRR_ERR_TIMEOUT"
    assert L.khrr_status_name(0) == b"KHRR_OK"


def test_create_without_gpu_reports_unsupported(libkhrr):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import khrr
    with pytest.raises(khrr.KhrrError) as e:
        khrr.Context(0)
    assert e.value.status == 8


def test_null_context_is_rejected(libkhrr):
    import khrr
    L = khrr.lib()
    assert L.khrr_forces(None, 1) == 1
    assert L.khrr_step(None, 0.002, 1, 0) == 1
    assert L.khrr_last_error(None) == b"null context"
