"""Shared pytest configuration: the `gpu` marker and fixture helpers."""
import lzma
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
FIXTURES = ["glove", "knittubeinit", "knittubebroken", "blenderobj", "houdiniobj"]
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden_bcc(name: str, tmp_dir: str) -> str:
    """Decompresses tests/golden/inputs/<name>.bcc.xz into tmp_dir; returns the path."""
    out = os.path.join(tmp_dir, name + ".bcc")
    if not os.path.exists(out):
        with lzma.open(os.path.join(GOLDEN, "inputs", name + ".bcc.xz"), "rb") as f, open(out, "wb") as g:
            g.write(f.read())
    return out


def golden_certificate(name: str) -> str:
    with open(os.path.join(GOLDEN, "certificates", name + ".txt")) as f:
        return f.read()


@pytest.fixture(scope="session")
def golden_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("golden"))
