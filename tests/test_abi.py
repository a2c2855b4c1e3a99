"""The C ABI library loads and exports every symbol its headers declare."""
import os
import re
import subprocess

from molspin_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for hdr in ("msgpu.h", "msgpu_host.h"):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(msgpu_\w+)\s*\(", text))
    return names


def test_all_declared_symbols_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (msgpu_\w+)", out))
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = declared - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    for name in declared:
        assert hasattr(L.lib, name)


def test_library_targets_sm100a():
    out = subprocess.run(["cuobjdump", "--list-elf", L.LIB_PATH], capture_output=True, text=True)
    if out.returncode == 0:
        assert "sm_100a" in out.stdout


def test_null_context_errors():
    assert L.lib.msgpu_last_error(None) == b"null context"
    assert L.lib.msgpu_run(None, None) == L.MSGPU_ERR_INVALID
    assert L.lib.msgpu_upload_hamiltonian_csr(None, 4, None, None, None) == L.MSGPU_ERR_INVALID


def test_package_import_does_not_load_the_library():
    # a fresh checkout builds through `python -m molspin_b200.build`, which
    # imports the package before libmsgpu.so exists
    code = ("import sys, molspin_b200, molspin_b200.build; "
            "assert 'molspin_b200._lib' not in sys.modules; "
            "molspin_b200.HSPropagatorB200; assert 'molspin_b200._lib' in sys.modules")
    subprocess.run([os.sys.executable, "-c", code], cwd=ROOT, check=True)


C_CONSUMER = r"""
#include <stdio.h>
#include <string.h>
#include "msgpu.h"
#include "msgpu_host.h"

int main(void)
{
    double t[8];
    long n = msgpu_host_time_grid(3.0, 1.0, t, 8);
    if (n != 4 || t[0] != 0.0 || t[3] != 3.0) return 1;
    if (strcmp(msgpu_last_error(NULL), "null context") != 0) return 2;
    if (msgpu_run(NULL, NULL) != MSGPU_ERR_INVALID) return 3;
    if (msgpu_launch_count(NULL) != 0) return 4;
    printf("ok %ld\n", n);
    return 0;
}
"""


def test_headers_are_plain_c_and_link(tmp_path):
    # A C99 caller (the language of a cgo / JNI / ctypes shim) compiles against
    # both headers with warnings as errors, links against the library and
    # calls host entry points and the null-context error paths.
    src = tmp_path / "consumer.c"
    src.write_text(C_CONSUMER)
    exe = tmp_path / "consumer"
    libdir = os.path.dirname(L.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                    "-L", libdir, "-lmsgpu", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, (out.returncode, out.stderr)
    assert out.stdout.strip() == "ok 4"
