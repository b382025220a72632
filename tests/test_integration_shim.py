"""The reference-side binding (include/gsofa_symbfact_shim.hpp, a drop-in
`symbfact_min_id` over the C-ABI) compiles against include/gsofa.h and
links against libgsofa.so, with a main() that calls it the way the
reference's main.cu does; the C examples under include/examples compile and
link too (CPU only: compiled and linked, not run)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "gsofatpds_b200")


def _need_lib():
    if not os.path.exists(os.path.join(LIB, "libgsofa.so")):
        pytest.skip("libgsofa.so not built")


def test_shim_compiles_and_links(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    _need_lib()
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
    out = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", INC,
                          str(tmp_path / "main.cpp"), "-L", LIB, "-lgsofa",
                          "-Wl,-rpath," + LIB, "-o", str(tmp_path / "main")],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr


@pytest.mark.parametrize("name", ["handle_api.c", "serving.c"])
def test_c_examples_compile_and_link(tmp_path, name):
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    _need_lib()
    out = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", INC,
                          os.path.join(INC, "examples", name), "-L", LIB, "-lgsofa",
                          "-Wl,-rpath," + LIB, "-o", str(tmp_path / "ex")],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
