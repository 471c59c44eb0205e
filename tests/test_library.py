"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(nova_b200_\w+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for required in ("nova_b200_create", "nova_b200_upload_scene", "nova_b200_build_bvh", "nova_b200_render",
                     "nova_b200_trace", "nova_b200_bake_irradiance", "nova_b200_get_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from axomae_b200 import native
    lib = native.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_create_reports_status_without_gpu():
    """Without a visible GPU the context cannot be created and the call says so (NOT_GPU_BUILD);
    with a GPU it succeeds.  Either way no compute is issued."""
    import torch
    from axomae_b200 import native
    h = ctypes.c_void_p()
    st = native.lib().nova_b200_create(ctypes.byref(h), 0)
    if torch.cuda.is_available():
        assert st == 0
        native.lib().nova_b200_destroy(h)
    else:
        assert st == 10  # NOT_GPU_BUILD, nova::ERROR_STATE numbering


def test_status_numbering_matches_reference_enum():
    from axomae_b200 import native
    assert native.STATUS[0] == "SUCCESS" and native.STATUS[9] == "SCENE_NOT_PROCESSED"
    assert native.STATUS[15] == "INVALID_ARGUMENT" and native.STATUS[16] == "RENDERER_EXCEPTION"


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """With the library absent the bindings raise at the first call; there is no other path."""
    from axomae_b200 import native
    monkeypatch.setattr(native, "_lib", None)
    monkeypatch.setattr(native, "LIB_PATH", str(tmp_path / "libnova_b200.so"))
    with pytest.raises(ImportError, match="not built"):
        native.lib()
    with pytest.raises(ImportError):
        native.Context(0)


def test_c_abi_from_plain_c():
    """tests/cpp/cabi_caller.c: the header compiles as C99 (-pedantic) and a C program links the
    library and gets its status codes (no device work)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "cpp")], check=True)
    r = subprocess.run([os.path.join(ROOT, "tests", "cpp", "_build", "cabi_caller")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
