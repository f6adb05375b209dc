"""The tile order of the persistent TMA hop kernels, checked on the host.

tests/c/tile_order.cpp includes the header the kernels use
(plqcd_b200/csrc/tile_order.cuh) and checks, for every kind of launch (one
parity, full lattice, RHS tiles), a range of lattice shapes and tile heights,
the default (z, t) blocks and every block the environment can set, that the
items map onto the tiles one to one with every coordinate in range."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tile_order_is_a_bijection(tmp_path):
    exe = tmp_path / "tile_order"
    src = os.path.join(ROOT, "tests", "c", "tile_order.cpp")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "plqcd_b200", "csrc"),
                        src, "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout[-2000:]
    assert " 0 failures" in r.stdout
