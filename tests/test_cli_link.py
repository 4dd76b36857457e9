"""The reference's command-line front end (cli/main.cpp), unchanged, compiles
against this library's headers (include/grrt/api.h forwards to
include/grrt_api.h) and links against libgrrt.so: the drop-in claim for the
caller side. CPU only: the CLI's --help runs without a GPU, and a render on a
machine without one ends with the library's error rather than a crash.

Needs the reference sources (GRRT_REFERENCE, else the tree this build
environment mounts); skipped where they are absent.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("GRRT_REFERENCE", "/root/reference")
CLI = os.path.join(REF, "cli", "main.cpp")


@pytest.fixture(scope="module")
def cli(tmp_path_factory, grrt):
    if not os.path.exists(CLI):
        pytest.skip("reference sources not present")
    out = str(tmp_path_factory.mktemp("cli") / "grrt-cli")
    libdir = os.path.dirname(grrt.LIB_PATH)
    cmd = ["/usr/bin/g++", "-std=c++23", "-O1", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(REF, "third_party"),
           # GCC 13 lacks <print>; the shim provides std::print/println over std::format
           "-I", os.path.join(ROOT, "oracle", "shim"),
           CLI, "-L", libdir, "-lgrrt", f"-Wl,-rpath,{libdir}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


def test_reference_cli_links_unchanged(cli):
    # every symbol the CLI calls resolves in libgrrt.so
    r = subprocess.run(["ldd", "-r", cli], capture_output=True, text=True)
    assert "undefined symbol" not in r.stdout + r.stderr
    assert "libgrrt.so" in r.stdout
    h = subprocess.run([cli, "--help"], capture_output=True, text=True, timeout=60)
    assert h.returncode == 0 and "--help" in h.stdout


def test_reference_cli_without_gpu_reports_the_error(cli, grrt, tmp_path):
    if grrt.cuda_available():
        pytest.skip("a GPU is present; this case covers a machine without one")
    r = subprocess.run([cli, "--width", "8", "--height", "8", "--output", str(tmp_path / "o")],
                       capture_output=True, text=True, timeout=120, cwd=tmp_path)
    assert r.returncode != 0 and "no CUDA device" in (r.stdout + r.stderr)
