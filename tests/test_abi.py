"""The C ABI: libaxr.so loads without a GPU and exports every symbol
include/axr.h declares; the product package never imports the oracle."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "axr.h")
LIB = os.path.join(ROOT, "axi_visualizer_b200", "libaxr.so")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(axr_\w+)\s*\(", src)))


def test_header_lists_match_binding():
    from axi_visualizer_b200._lib import EXPORTS
    assert sorted(EXPORTS) == declared()


@pytest.mark.parametrize("lang,std", [("c", "-std=c99"), ("c++", "-std=c++11")])
def test_header_is_plain_c_and_cpp(lang, std, tmp_path):
    """The boundary header compiles warning-free as pedantic C99 and as
    C++11, with no CUDA or torch headers on the include path."""
    cc = "gcc" if lang == "c" else "g++"
    try:
        subprocess.run([cc, "--version"], capture_output=True, check=True)
    except (OSError, subprocess.CalledProcessError):
        pytest.skip(f"{cc} not available")
    src = tmp_path / "use_axr.c"
    src.write_text('#include "axr.h"\nint main(void) { return 0; }\n')
    r = subprocess.run([cc, "-x", lang, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                        os.path.dirname(HEADER), "-c", str(src), "-o", str(tmp_path / "use_axr.o")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_library_loads_and_exports_all_symbols():
    if not os.path.exists(LIB):
        from axi_visualizer_b200 import build
        build.build()
    L = ctypes.CDLL(LIB)
    missing = [s for s in declared() if not hasattr(L, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(axr_\w+)\b", out))
    assert set(declared()) <= exported


def test_binding_signatures_cover_exports():
    from axi_visualizer_b200 import _lib
    L = _lib.lib()
    for name in _lib.EXPORTS:
        fn = getattr(L, name)
        assert fn.argtypes is not None or name == "axr_last_error"


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from axi_visualizer_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "libaxr.so"))
    with pytest.raises(_lib.AxrError):
        _lib.lib()


def test_product_does_not_use_the_oracle():
    pkg = os.path.join(ROOT, "axi_visualizer_b200")
    for dp, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h")):
                txt = open(os.path.join(dp, f)).read()
                assert not re.search(r"^\s*(import|from)\s+oracle\b", txt, flags=re.M), f
                assert "liboracle" not in txt and "_ref/" not in txt, f


def test_errors_without_gpu_are_reported():
    """axr_create on a machine without a usable device returns an error code
    and a message instead of crashing (skipped where a GPU exists)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    from axi_visualizer_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    rc = L.axr_create(64, 64, 0, ctypes.byref(h))
    assert rc != 0 and L.axr_last_error()
    assert L.axr_create(60, 64, 0, ctypes.byref(h)) == -1     # width not a multiple of 16


def test_entry_points_refuse_a_null_handle():
    """Without a handle every entry point returns an error code and leaves a
    message, before any CUDA call (so this runs without a GPU)."""
    from axi_visualizer_b200 import _lib
    L = _lib.lib()
    f3 = (ctypes.c_float * 9)()
    calls = [
        ("axr_transform", (None, 0, f3, f3, f3, 0, -1)),
        ("axr_translate", (None, 0, f3, 0, -1)),
        ("axr_vert_light", (None, None, 0, None, None, 0, None, None, 0, None, None, None, 0, 0.2)),
        ("axr_get_vertices", (None, 0, None, None, None)),
        ("axr_ssao", (None, f3, 9)),
        ("axr_dof", (None, 8.0)),
        ("axr_bloom", (None,)),
        ("axr_gamma", (None, 1.0)),
    ]
    for name, args in calls:
        rc = getattr(L, name)(*args)
        assert rc < 0, name
        assert b"null handle" in L.axr_last_error(), name
