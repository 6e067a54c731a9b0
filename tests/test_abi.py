"""C ABI surface (CPU only: loads the library, calls nothing that computes)."""
import ctypes as C
import os
import re

import paddi_b200 as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(paddi_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_function():
    L = P.lib()
    declared = _declared_functions()
    assert declared, "no declarations found"
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing


def test_bindings_cover_the_header():
    assert set(_declared_functions()) <= set(P._SIGS), \
        set(_declared_functions()) - set(P._SIGS)


def test_abi_version_and_status_strings():
    L = P.lib()
    assert L.paddi_abi_version() == 2
    assert P.status_string(P.PADDI_OK) == "ok"
    assert "invalid" in P.status_string(P.PADDI_ERR_INVALID_ARG)
    assert P.status_string(12345) == "unknown status"


def test_default_options():
    o = P._Opts()
    P.lib().paddi_opts_default(C.byref(o))
    assert o.struct_size == C.sizeof(P._Opts)
    assert (o.segment_len, o.phase1_chunks, o.iter_cap) == (256, 12, 200)


def test_null_arguments_are_rejected_without_a_device():
    L = P.lib()
    assert L.paddi_ctx_create(None, None) == P.PADDI_ERR_INVALID_ARG
    assert L.paddi_ctx_destroy(None) == P.PADDI_ERR_INVALID_ARG
    assert L.paddi_palmad(None, None, 0, 0, 0, None, None, 0, None) == P.PADDI_ERR_INVALID_ARG
    o = P._Opts()
    L.paddi_opts_default(C.byref(o))
    o.struct_size = 3  # wrong struct size
    h = C.c_void_p()
    assert L.paddi_ctx_create(C.byref(h), C.byref(o)) in (P.PADDI_ERR_INVALID_ARG,
                                                          P.PADDI_ERR_NO_DEVICE)


def test_unsupported_tile_rows_are_refused_without_a_device():
    L = P.lib()
    o = P._Opts()
    L.paddi_opts_default(C.byref(o))
    assert o.tile_rows == 0
    o.tile_rows = 128  # only 0 (by length) and 64 are accepted
    h = C.c_void_p()
    assert L.paddi_ctx_create(C.byref(h), C.byref(o)) == P.PADDI_ERR_UNSUPPORTED


def test_cli_usage_without_arguments():
    import subprocess
    exe = os.path.join(ROOT, "paddi_b200", "paddi-main")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
