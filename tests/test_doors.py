"""The two doors a reference user comes in through: the C++ classes
(include/linking_number_certificate.h:63-66, the per-pair functions of
src/compute_link.h:62-181) and the `verifycurves` command line
(src/main.cpp:14-99, src/define_args.h:9-55).

The C++ drop-in headers are compiled into a small program that links
libfln.so; the CLI runs on every golden input with both methods, and its
output file must equal the reference's golden certificate byte for byte.
The host-only parts (certificate I/O, diffs, flag parsing) run on the CPU;
the rest needs a GPU.
"""
import os
import subprocess

import pytest

from conftest import FIXTURES, GOLDEN, REPO, golden_bcc
from fastlinkingnumbers_b200._native import LIB_DIR

CLI = os.path.join(LIB_DIR, "verifycurves")


@pytest.fixture(scope="module")
def shim_exe(tmp_path_factory):
    d = tmp_path_factory.mktemp("shim")
    exe = str(d / "shim_check")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "cpp", "shim_check.cpp"), "-L", LIB_DIR, "-lfln",
                    f"-Wl,-rpath,{LIB_DIR}", "-o", exe], check=True)
    return exe


def _run_shim(exe, mode, golden_dir):
    golden_bcc("knittubebroken", golden_dir)
    r = subprocess.run([exe, mode, GOLDEN, golden_dir], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr


def test_cpp_shim_host(shim_exe, golden_dir):
    _run_shim(shim_exe, "host", golden_dir)


@pytest.mark.gpu
def test_cpp_shim_compute(shim_exe, golden_dir):
    _run_shim(shim_exe, "gpu", golden_dir)


def test_cli_flag_errors(golden_dir, tmp_path):
    r = subprocess.run([CLI, "--no_such_flag=1"], capture_output=True, text=True)
    assert r.returncode == 2 and "unknown command line flag" in r.stderr
    # The method is checked after the import and before any device work.
    path = golden_bcc("knittubebroken", golden_dir)
    r = subprocess.run([CLI, "--input", path, "--method", "fastest", "--output", str(tmp_path / "o.txt")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "Invalid method: 'fastest'." in r.stderr
    r = subprocess.run([CLI, "--input", str(tmp_path / "missing.bcc")], capture_output=True, text=True)
    assert r.returncode == 1 and "Unable to open BCC file" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("method", ["directsum", "barneshut"])
def test_cli_certificates_match_golden(name, method, golden_dir, tmp_path):
    out = tmp_path / "cert.txt"
    r = subprocess.run([CLI, "--input", golden_bcc(name, golden_dir), "--output", str(out), "--method", method],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    with open(os.path.join(GOLDEN, "certificates", name + ".txt"), "rb") as f:
        assert out.read_bytes() == f.read()


@pytest.mark.gpu
def test_cli_compare_and_diffs(golden_dir, tmp_path):
    # README.md:100-126: verifycurves on knittubebroken with --comparewith the
    # knittubeinit certificate writes the differing pair and its curves.
    dp, dc, out = tmp_path / "dp.txt", tmp_path / "dc.txt", tmp_path / "o.txt"
    r = subprocess.run([CLI, "--input", golden_bcc("knittubebroken", golden_dir), "--output", str(out),
                        "--method", "directsum", "--comparewith",
                        os.path.join(GOLDEN, "certificates", "knittubeinit.txt"), "--diffpairs", str(dp),
                        "--diffcurves", str(dc)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert dp.read_text() == "5,6,-2\n" and dc.read_text() == "5\n6\n"
    # --nodiscretize: the control polygons themselves are summed, which on the
    # broken knitted tube gives other integers; they must be the oracle's
    # (the reference's pipeline with discretize = false).
    from oracle import pyoracle
    path = golden_bcc("knittubebroken", golden_dir)
    want, _, _ = pyoracle.Oracle().load_bcc(path).certificate(True, discretize=False)
    for method in ("directsum", "barneshut"):
        r = subprocess.run([CLI, "--input", path, "--output", str(out), "--nodiscretize", "--method", method],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        assert out.read_text() == want and want.count("\n") > 2
