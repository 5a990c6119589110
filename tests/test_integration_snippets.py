"""The C calls that INTEGRATION.md shows a reference-side caller compile
against include/ with warnings as errors and link against libtk.so (every
symbol resolves).  Nothing is executed: no GPU is needed."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# the free variables the snippets use, as a caller would hold them
PARAMS = """int16_t *d_buf, int npoly, tk_stream_t stream,
    int16_t *d_s, const int16_t *h_polys, void *h_packed, const void *d_packed,
    int16_t *d_out, size_t n2, size_t n3, size_t n4,
    const int16_t *A2, const int16_t *A3, const int16_t *A4,
    const int16_t *s2, const int16_t *s3, const int16_t *s4,
    const int16_t *e2, const int16_t *e3, const int16_t *e4,
    int16_t *out2, int16_t *out3, int16_t *out4,
    int k, size_t njobs, const int16_t *h_A, const int16_t *h_s, const int16_t *h_e,
    int16_t *h_out"""


def c_blocks():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```c\n(.*?)```", text, flags=re.S)


def test_integration_c_snippets_compile_and_link(tk, tmp_path):
    blocks = c_blocks()
    assert len(blocks) >= 3
    src = "#include <stdint.h>\n#include <stdio.h>\n#include \"tk_ntt.h\"\n"
    for i, body in enumerate(blocks):
        src += f"void snippet_{i}({PARAMS}) {{\n{body}\n}}\n"
    c = tmp_path / "snippets.c"
    c.write_text(src)
    so = tmp_path / "libsnippets.so"
    lib_dir = os.path.join(ROOT, "tensorkyber_b200")
    cmd = ["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-Wno-unused-parameter",
           "-Wno-unused-variable", "-Wno-unused-but-set-variable",
           "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(so),
           "-L", lib_dir, "-ltk", "-Wl,--no-undefined"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-3000:]
