"""The C-ABI libraries load without a GPU and export every symbol their
headers declare."""
import ctypes
import os
import re
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(REPO, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if not n.startswith("__")))


def exported(so):
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True).stdout
    return set(l.split()[-1] for l in out.splitlines() if " T " in l)


@pytest.mark.parametrize("header,so", [
    ("jacquard_b200.h", "jacquard_b200/libjacquard_b200.so"),
    ("jacquard_frontend.h", "jacquard_b200/libjq_frontend.so"),
])
def test_library_exports_every_declared_symbol(header, so):
    path = os.path.join(REPO, so)
    ctypes.CDLL(path)  # loads on a machine without a GPU
    names = declared(header)
    assert names, header
    missing = [n for n in names if n not in exported(path)]
    assert not missing, missing


def test_reference_symbols_present():
    syms = exported(os.path.join(REPO, "jacquard_b200/libjacquard_b200.so"))
    for n in ("simulate_v1_noninteractive_simple_scan_cuda", "simulate_v1_noninteractive_timed_cuda"):
        assert n in syms
