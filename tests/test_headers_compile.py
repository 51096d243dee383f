"""The C-ABI headers (include/cupf_b200.h, include/cupf_mlp.h) are what a cgo,
JNI or ctypes binding includes: they must compile on their own as C11 and as
C++17, warnings as errors."""
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
