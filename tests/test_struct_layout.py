"""The C ABI's structs as C compilers lay them out, against the ctypes and numpy
mirrors that the Python package passes across the boundary (no GPU).

A cgo, bindgen or N-API caller compiles include/dgann.h as plain C, so the
header is compiled here with gcc as C99.  Each struct's size and each field's
offset must equal the ctypes Structure in pydiskann_b200/_lib.py; the request
record that Server.run_trace builds with numpy must equal DgRequest.
"""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from pydiskann_b200 import _lib
from pydiskann_b200.serve import _REQ_DTYPE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = {
    "DgFilterOp": _lib.FilterOp,
    "DgIndexDesc": _lib.IndexDesc,
    "DgSearchParams": _lib.SearchParams,
    "DgSpfreshDesc": _lib.SpfreshDesc,
    "DgSpfreshParams": _lib.SpfreshParams,
    "DgServerConfig": _lib.ServerConfig,
    "DgRequest": _lib.Request,
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    lines = []
    for cname, cls in STRUCTS.items():
        lines.append(f'printf("{cname} . %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    src = ("#include <stddef.h>\n#include <stdio.h>\n#include \"dgann.h\"\nint main(void) {\n  "
           + "\n  ".join(lines) + "\n  return 0;\n}\n")
    d = tmp_path_factory.mktemp("layout")
    (d / "layout.c").write_text(src)
    exe = d / "layout"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(d / "layout.c"), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    lay = {}
    for line in out.splitlines():
        s, f, v = line.split()
        lay.setdefault(s, {})[f] = int(v)
    return lay


@pytest.mark.parametrize("cname", list(STRUCTS))
def test_ctypes_mirror_matches_c(c_layout, cname):
    cls = STRUCTS[cname]
    assert C.sizeof(cls) == c_layout[cname]["."], f"sizeof({cname})"
    for f, _ in cls._fields_:
        assert getattr(cls, f).offset == c_layout[cname][f], f"offsetof({cname}, {f})"


def test_numpy_request_record_matches_c(c_layout):
    want = [c_layout["DgRequest"][f] for f, _ in _lib.Request._fields_]
    got = [_REQ_DTYPE.fields[n][1] for n in _REQ_DTYPE.names]
    assert got == want
    assert _REQ_DTYPE.itemsize == c_layout["DgRequest"]["."]
