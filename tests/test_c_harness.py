"""The C ABI from a plain C program (tests/c_harness.c): compiled with gcc
against include/inmsom_gpu.h and linked with the library, it calls the
entries with Fortran-layout arrays and checks what they return; it needs
no GPU (the device entry must fail cleanly without one)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_program_calls_the_abi(tmp_path):
    from inmsom_elfs_b200 import _lib, build
    build.build()
    exe = tmp_path / "c_harness"
    libdir = _lib.LIB_PATH.parent
    subprocess.run(["gcc", "-std=c99", "-O1", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "c_harness.c"), f"-L{libdir}", "-linmsom_gpu", f"-Wl,-rpath,{libdir}",
                    "-lm", "-o", str(exe)], check=True)
    scratch = tmp_path / "files"
    scratch.mkdir()
    r = subprocess.run([str(exe), str(scratch)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
