"""The C-ABI library loads and exports every function include/*.h declares.

No GPU needed: this only opens libpfb200.so and resolves symbols.
"""
import ctypes
import os
import re

import pfb200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")

# C++-linkage helpers (declared outside extern "C") are matched by substring.
_CPP_LINKAGE = {"trial_div_launch"}


def _declared_functions():
    names = set()
    for fn in sorted(os.listdir(INC)):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(INC, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        src = re.sub(r"#[^\n]*", "", src)
        src = re.sub(r"typedef[^;]*;", "", src)
        for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{}]*)\)\s*;", src):
            name = m.group(1)
            if name in ("if", "while", "for", "return", "sizeof"):
                continue
            names.add(name)
    return names


def test_library_loads():
    L = pfb200.lib()
    assert pfb200.mask_bytes(100) == 313 * 4
    assert pfb200.mask_bytes(9999) == ((9999 * 9999 + 31) // 32) * 4


def test_every_declared_symbol_is_exported():
    L = pfb200.lib()
    declared = _declared_functions()
    assert "trial_div_gpu" in declared and "pfb_sieve_run" in declared
    missing = []
    for name in sorted(declared):
        if name in _CPP_LINKAGE:
            out = os.popen(f"nm -D --defined-only {pfb200.LIB_PATH}").read()
            if name not in out:
                missing.append(name)
            continue
        try:
            getattr(L, name)
        except AttributeError:
            missing.append(name)
    assert not missing, missing


def test_missing_library_raises_instead_of_falling_back(tmp_path):
    """With the shared library absent, the binding's first call raises
    ImportError (there is no CPU path to fall back to).  A fresh interpreter
    with the package's library path pointed at an empty folder."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import pfb200; pfb200.LIB_PATH = %r\n"
            "try:\n    pfb200.mask_bytes(100)\nexcept ImportError as e:\n    print('raised', e)\n"
            % (os.path.join(ROOT, "prime-finder_b200"), str(tmp_path / "libpfb200.so")))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120).stdout
    assert out.startswith("raised") and "is missing" in out


def test_headers_serve_c_callers(tmp_path):
    """The reference's callers are C (worker.c, tests/test_gpu.c): every
    header in include/*.h compiles as strict C99, and a C program linked
    against the library runs calls that need no GPU."""
    import subprocess
    src = tmp_path / "caller.c"
    headers = sorted(f for f in os.listdir(INC) if f.endswith(".h"))
    src.write_text("".join('#include "%s"\n' % h for h in headers) + """
#include <stdio.h>
int main(void) {
    printf("%zu %d\\n", pfb_sieve_mask_bytes(100), trial_div_gpu(NULL, 1, 1, 1, NULL, NULL));
    return 0;
}
""")
    exe = str(tmp_path / "caller")
    libdir = os.path.dirname(pfb200.LIB_PATH)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", INC, str(src), "-o", exe,
                         "-L", libdir, "-lpfb200", "-Wl,-rpath," + libdir], capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.split() == ["1252", "-1"], (r.stdout, r.stderr)


def test_cpp_surface_compiles_and_links(tmp_path):
    """bench_mr_gpu.cu-style C++ callers of batch_mod_ctx.cuh and
    miller_rabin_runner.cuh (tests/cpp/mr_api_demo.cpp) compile and link
    against the library; running them needs a GPU (test_cpp_api_gpu.py)."""
    import subprocess
    exe = str(tmp_path / "mr_api_demo")
    libdir = os.path.dirname(pfb200.LIB_PATH)
    cc = subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-I", INC, "-I", "/usr/local/cuda/include",
                         os.path.join(ROOT, "tests", "cpp", "mr_api_demo.cpp"), "-o", exe,
                         "-L", libdir, "-lpfb200", "-Wl,-rpath," + libdir], capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
