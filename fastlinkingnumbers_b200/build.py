"""Builds libfln.so and the verifycurves CLI in-tree with nvcc (sm_100a) and g++.

Usage: python -m fastlinkingnumbers_b200.build [--clean]
"""
import os
import subprocess
import sys

CSRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc")


def build(clean: bool = False, jobs: int = 8) -> None:
    if clean:
        subprocess.run(["make", "-s", "-C", CSRC, "clean"], check=True)
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", CSRC], check=True)


if __name__ == "__main__":
    build(clean="--clean" in sys.argv)
