"""The C calls a reference-side caller makes (tests/integration/
caller_snippets.c, the calls the integration guide shows) compile against
include/ with warnings as errors and link against libtk.so (every symbol
resolves).  Nothing is executed: no GPU is needed."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_integration_c_snippets_compile_and_link(tk, tmp_path):
    src = os.path.join(ROOT, "tests", "integration", "caller_snippets.c")
    so = tmp_path / "libsnippets.so"
    lib_dir = os.path.join(ROOT, "tensorkyber_b200")
    cmd = ["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "include"), src, "-o", str(so),
           "-L", lib_dir, "-ltk", "-Wl,--no-undefined"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-3000:]
    nm = subprocess.run(["nm", "-D", "--undefined-only", str(so)], capture_output=True,
                        text=True, timeout=60).stdout
    for sym in ("tk_ntt", "tk_invntt", "tk_ntt_small", "tk_ntt_packed", "tk_pack_small",
                "tk_matvec", "tk_matvec_host_noalloc", "tk_server_create"):
        assert f" {sym}\n" in nm + "\n", sym
