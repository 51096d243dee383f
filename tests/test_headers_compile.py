"""The C-ABI headers (include/cupf_b200.h, include/cupf_mlp.h) are what a cgo,
JNI or ctypes binding includes: they must compile on their own as C11 and as
C++17, warnings as errors."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

INCLUDE = Path(__file__).resolve().parents[1] / "include"
SNIPPET = """#include <string.h>
#include "cupf_b200.h"
#include "cupf_mlp.h"
int main(void) {
  cls_config c;
  pf_options o;
  memset(&c, 0, sizeof c);
  memset(&o, 0, sizeof o);
  o.custom = c;
  return (int)sizeof(pf_nr_config) == 0;
}
"""


@pytest.mark.parametrize("compiler,std,lang", [("gcc", "c11", "c"), ("g++", "c++17", "c++")])
def test_headers_compile_standalone(tmp_path, compiler, std, lang):
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not installed")
    src = tmp_path / "use_headers.c"
    src.write_text(SNIPPET)
    r = subprocess.run([compiler, f"-std={std}", "-Wall", "-Wextra", "-Werror", "-pedantic", f"-I{INCLUDE}",
                        "-x", lang, "-fsyntax-only", str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def _c_layouts(tmp_path, pairs):
    """sizeof and every field offset of the named C structs, from gcc."""
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "cupf_b200.h"', 'int main(void) {']
    for cname, fields in pairs:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layouts.c"
    exe = tmp_path / "layouts"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", f"-I{INCLUDE}", str(src), "-o", str(exe)], check=True)
    out = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        name, key, val = line.split()
        out[(name, key)] = int(val)
    return out


def test_ctypes_layouts_match_the_header(tmp_path):
    """The ctypes mirrors in cupf/_capi.py have the size and field offsets of
    the C structs, so the Python binding and a C caller pass the same bytes."""
    if shutil.which("gcc") is None:
        pytest.skip("gcc not installed")
    import sys
    sys.path.insert(0, str(INCLUDE.parent / "gpu-powerflow_b200"))
    from cupf import _capi

    mirrors = {"cls_config": _capi.ClsConfig, "pf_options": _capi.PfOptions, "pf_nr_config": _capi.PfNRConfig,
               "pf_solve_options": _capi.PfSolveOptions, "pf_adjoint_options": _capi.PfAdjointOptions,
               "pf_adjoint_result": _capi.PfAdjointResult, "pf_info_t": _capi.PfInfo}
    pairs = [(c, [f[0] for f in py._fields_]) for c, py in mirrors.items()]
    c = _c_layouts(tmp_path, pairs)
    for cname, py in mirrors.items():
        assert ctypes.sizeof(py) == c[(cname, "size")], cname
        for f in py._fields_:
            assert getattr(py, f[0]).offset == c[(cname, f[0])], (cname, f[0])
