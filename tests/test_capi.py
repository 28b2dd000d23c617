"""The C ABI library: loads, exports every symbol include/fln.h declares, and
its host-only entry points (certificate I/O, comparison, argument checks)
behave like the reference. No kernel runs here."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import GOLDEN, REPO
from fastlinkingnumbers_b200 import FlnError, LinkingNumberCertificate
from fastlinkingnumbers_b200 import _native as N


def _declared():
    hdr = open(os.path.join(REPO, "include", "fln.h")).read()
    return sorted(set(re.findall(r"\b(fln_[a-z_]+)\s*\(", hdr)))


def test_exports_every_declared_symbol():
    lib = ctypes.CDLL(N.LIB_PATH)
    declared = _declared()
    assert set(declared) == set(N.EXPORTED)
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    for name in declared:
        assert re.search(r"\bT %s$" % name, out, re.M), name


def test_status_strings_and_defaults():
    L = N.load()
    assert L.fln_abi_version() == 3
    assert L.fln_status_string(0) == b"ok"
    p = N.default_params()
    assert (p.barnes_hut_init_beta, p.barnes_hut_beta_limit, p.epssq) == (2.0, 10.0, 1e-24)
    assert (p.target_error, p.error_est_scale, p.fp64_margin) == (0.1, 0.05, 0.25)


def test_certificate_io_and_diffs(tmp_path):
    # README.md:100-126: knittubebroken vs knittubeinit -> "5,6,-2" and "5\n6\n".
    broken = LinkingNumberCertificate(os.path.join(GOLDEN, "certificates", "knittubebroken.txt"))
    init = LinkingNumberCertificate(os.path.join(GOLDEN, "certificates", "knittubeinit.txt"))
    assert broken.text() == "39\n5,6,-2\n" and init.text() == "39\n"
    assert broken != init and broken == LinkingNumberCertificate(
        os.path.join(GOLDEN, "certificates", "knittubebroken.txt"))
    dp, dc = str(tmp_path / "dp.txt"), str(tmp_path / "dc.txt")
    broken.ExportDiffsToFiles(dp, dc, init)
    assert open(dp).read() == "5,6,-2\n"
    assert open(dc).read() == "5\n6\n"
    out = str(tmp_path / "c.txt")
    broken.ExportToFile(out)
    assert open(out).read() == "39\n5,6,-2\n"
    assert broken.entries().tolist() == [[5, 6, -2]]


def test_diff_size_mismatch_message(tmp_path):
    a = tmp_path / "a.txt"
    a.write_text("3\n0,1,1\n")
    b = tmp_path / "b.txt"
    b.write_text("4\n")
    dp = str(tmp_path / "dp.txt")
    LinkingNumberCertificate(str(a)).ExportDiffsToFiles(dp, "[none]", LinkingNumberCertificate(str(b)))
    assert open(dp).read().startswith("Unable to compare")


def test_certificate_read_sums_duplicates_and_prunes(tmp_path):
    f = tmp_path / "d.txt"
    f.write_text("5\n1,2,3\n1,2,-3\n0,4,2\n")
    assert LinkingNumberCertificate(str(f)).text() == "5\n0,4,2\n"


def test_argument_checks_without_device():
    L = N.load()
    h = ctypes.c_void_p()
    st = L.fln_ctx_create(0, None, ctypes.byref(h))
    if st == 0:
        L.fln_ctx_destroy(h)
        pytest.skip("a CUDA device is visible")
    assert st == 5  # FLN_ERR_NO_DEVICE, not a crash
    with pytest.raises(FlnError):
        N.check(L.fln_certificate_load(b"/nonexistent/x.txt", ctypes.byref(h)))
