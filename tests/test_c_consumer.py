"""The C ABI from plain C99 (tests/c/abi_consumer.c): include/ladds_gpu.h
compiles as C, the library links, and its host-only entry points work from C."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_c99_consumer(tmp_path):
    from ladds_b200 import build

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lib = build.build_gpu()
    exe = str(tmp_path / "abi_consumer")
    libdir = os.path.dirname(lib)
    cmd = [cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "c", "abi_consumer.c"), "-o", exe, "-L", libdir, "-lladds_gpu",
           f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "abi_consumer: ok" in r.stdout
