"""The C-ABI library loads on any host and exports every symbol the public
headers declare (no compute calls: those need a GPU)."""
import ctypes
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(zb_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_headers_declare_functions():
    names = declared_functions()
    assert "zb_swe2d_step" in names and "zb_version" in names


def test_library_exports_every_declared_symbol():
    from zoomy_b200 import _lib as L
    lib = L.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"libzb.so lacks {missing}"


def test_bindings_cover_every_declared_symbol():
    from zoomy_b200 import _lib as L
    bound = {n for n, _, _ in L.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_struct_layouts_match_header():
    from zoomy_b200 import _lib as L
    assert ctypes.sizeof(L.ZbCtrl) == 128
    # zb_swe2d_cfg: field offsets follow the C declaration order
    assert L.ZbSwe2dCfg.dx.offset == 24
    assert L.ZbSwe2dCfg.bc.offset == 56


def test_cfg_struct_matches_the_c_compiler(tmp_path):
    """Every field offset of the ctypes mirror of zb_swe2d_cfg and its size,
    against what gcc lays out from the header."""
    import shutil
    import subprocess
    from zoomy_b200 import _lib as L
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    names = [f[0] for f in L.ZbSwe2dCfg._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include "zb.h"\nint main(void) {\n'
                   + "".join(f'  printf("%zu\\n", offsetof(zb_swe2d_cfg, {n}));\n'
                             for n in names)
                   + '  printf("%zu\\n", sizeof(zb_swe2d_cfg));\n  return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    want = [getattr(L.ZbSwe2dCfg, n).offset for n in names] + [ctypes.sizeof(L.ZbSwe2dCfg)]
    assert got == want


def test_version_string():
    from zoomy_b200 import _lib as L
    assert b"sm_100a" in L.load().zb_version()


def test_cuda_required_without_gpu(monkeypatch):
    import torch
    from zoomy_b200 import _lib as L
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        L.require_cuda()
