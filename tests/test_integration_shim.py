"""The reference-side binding shown in INTEGRATION.md (a drop-in
`symbfact_min_id` over the C-ABI) compiles against include/gsofa.h and
links against libgsofa.so, with a main() that calls it the way the
reference's main.cu does (CPU only: compiled and linked, not run)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_shim_compiles_and_links(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    shim = [b for b in blocks if "inline void symbfact_min_id" in b]
    assert len(shim) == 1
    (tmp_path / "gsofa_symbfact_shim.hpp").write_text(shim[0])
    (tmp_path / "main.cpp").write_text(
        '#include "gsofa_symbfact_shim.hpp"\n'
        "int main(int argc, char** argv) {\n"
        "    ull_t fill_count = 0, teps = 0;\n"
        "    double time = 0;\n"
        "    int nsup = 0;\n"
        "    if (argc > 1) symbfact_min_id(argc, argv, 0, fill_count, time, nsup, teps);\n"
        '    printf("%llu %g %d %llu\\n", fill_count, time, nsup, teps);\n'
        "    return 0;\n"
        "}\n")
    lib = os.path.join(ROOT, "gsofatpds_b200")
    out = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                          str(tmp_path / "main.cpp"), "-L", lib, "-lgsofa",
                          "-Wl,-rpath," + lib, "-o", str(tmp_path / "main")],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr


def test_c_examples_compile_and_link(tmp_path):
    """The C snippets of INTEGRATION.md (handle API, serving) compile inside a
    main() against include/gsofa.h and link against libgsofa.so."""
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```c\n(.*?)```", text, flags=re.S)
    assert len(blocks) >= 2
    lib = os.path.join(ROOT, "gsofatpds_b200")
    strip = [("\n".join(l for l in b.splitlines() if not l.startswith("#include")))
             for b in blocks]
    # the serving snippet uses the handle-API one's ctx and opts
    serving = "gsofa_ctx* ctx = NULL; gsofa_opts o; gsofa_opts_default(&o);\n" + strip[1]
    for k, body in enumerate([strip[0], serving]):
        src = ('#include <stdio.h>\n#include <stdlib.h>\n#include "gsofa.h"\n'
               "int n = 0; long long nnz = 0; int *row_begin, *row_end, *col;\n"
               "int main(void) {\n" + body + "\nreturn 0;\n}\n")
        (tmp_path / ("ex%d.c" % k)).write_text(src)
        out = subprocess.run(["gcc", "-std=c11", "-Wall", "-Wno-unused-variable",
                              "-I", os.path.join(ROOT, "include"), str(tmp_path / ("ex%d.c" % k)),
                              "-L", lib, "-lgsofa", "-Wl,-rpath," + lib,
                              "-o", str(tmp_path / ("ex%d" % k))],
                             capture_output=True, text=True, timeout=120)
        assert out.returncode == 0, (k, out.stderr)
