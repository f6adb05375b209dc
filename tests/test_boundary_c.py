"""The drop-in boundary seen from C: a C caller compiles and links against
include/ and libplqcd_b200.so alone, the reference's own driver
(tests/test_hopping.c) compiles and links unchanged, plqcd_g has the
reference's member layout, and (GPU) the C caller's eo+oe output equals the
oracle's.

The reference's driver calls MPI for its timing (tests/test_hopping.c:293,
303-304); it is compiled here with the single-rank MPI header of oracle/,
as a caller would with mpicc. Tests that need the reference's sources skip
when they are absent (PLQCD_REFERENCE_ROOT)."""
import os
import subprocess

import numpy as np
import pytest

import plqcd_b200 as P
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.dirname(P.LIB_PATH)
CDIR = os.path.join(ROOT, "tests", "c")
MPI_STUB = os.path.join(ROOT, "oracle", "mpi_stub")

# offsets of struct _PLQCD_GLOBAL_PARAMS in the reference's default build
# (include/plqcd_global_params.h:67-205 without AVX_SPLIT / MIC), LP64
REFERENCE_LAYOUT = {
    "sizeof": 416, "nprocs": 0, "nthread": 16, "cpr": 20, "npr": 36, "LX": 68, "LY": 72, "LZ": 76, "LT": 80,
    "latdims": 84, "VOLUME": 100, "Vmic_split": 104, "Vavx_split": 108, "Vsse_split": 112, "face": 116,
    "ipt_eo": 136, "ipt_lex": 144, "nn_bnde": 152, "nn_bndo": 216, "iup": 280, "idn": 288, "ipt_eo_yzt": 296,
    "ipt_lex_yzt": 304, "ipt_eo_sse_split": 312, "ipt_lex_sse_split": 320, "iup_sse_split": 328,
    "idn_sse_split": 336, "phip": 344, "phim": 376, "ALIGN": 408, "init": 412,
}


def _run(cmd, **kw):
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    assert r.returncode == 0, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return r.stdout


def _layout(exe):
    out = _run([str(exe)])
    return {k: int(v) for k, v in (line.split() for line in out.splitlines())}


def _reference_tree():
    root = O.reference_root()
    if not root or not os.path.exists(os.path.join(root, "include", "plqcd_global_params.h")):
        pytest.skip("reference sources not present")
    return root


def build_c_caller(tmp_path):
    exe = tmp_path / "hop_caller"
    _run(["gcc", "-std=gnu99", "-O2", "-Wall", "-Werror", "-I", INC, os.path.join(CDIR, "hop_caller.c"),
          "-L", LIBDIR, "-lplqcd_b200", f"-Wl,-rpath,{LIBDIR}", "-lm", "-o", str(exe)])
    return exe


def test_struct_layout_is_the_references(tmp_path):
    exe = tmp_path / "offsets"
    _run(["gcc", "-std=gnu99", "-Wall", "-Werror", "-I", INC, os.path.join(CDIR, "struct_offsets.c"), "-o", str(exe)])
    assert _layout(exe) == REFERENCE_LAYOUT


def test_struct_layout_equals_reference_header(tmp_path):
    root = _reference_tree()
    exe = tmp_path / "offsets_ref"
    _run(["gcc", "-std=gnu99", "-fcommon", "-w", "-I", os.path.join(root, "include"), "-I", MPI_STUB,
          os.path.join(CDIR, "struct_offsets.c"), "-o", str(exe)])
    assert _layout(exe) == REFERENCE_LAYOUT


def test_c_caller_compiles_and_links(tmp_path):
    exe = build_c_caller(tmp_path)
    assert exe.exists()
    # the executable resolves every symbol it uses from the library
    out = _run(["nm", "-u", str(exe)])
    for sym in ("init_plqcd", "amalloc", "plqcd_hopping_matrix_eo_sse3_assymbly",
                "plqcd_hopping_matrix_oe_sse3_assymbly"):
        assert sym in out


def test_reference_driver_compiles_and_links_unchanged(tmp_path):
    """tests/test_hopping.c of the reference, as its Makefile builds the
    plain-C variant (-DASSYMBLY, OpenMP), against include/ and the library
    instead of lib/*.c."""
    root = _reference_tree()
    exe = tmp_path / "hopping"
    # the driver's own code draws a maybe-uninitialized warning at -O2; every
    # declaration it takes from the headers must be there
    _run(["gcc", "-std=gnu99", "-fopenmp", "-O2", "-Werror=implicit-function-declaration",
          "-Werror=incompatible-pointer-types", "-Werror=int-conversion", "-DASSYMBLY", "-I", INC, "-I", MPI_STUB,
          os.path.join(root, "tests", "test_hopping.c"), "-L", LIBDIR, "-lplqcd_b200", f"-Wl,-rpath,{LIBDIR}",
          "-lm", "-o", str(exe)])
    out = _run(["nm", "-u", str(exe)])
    assert "plqcd_hopping_matrix_eo_sse3_assymbly" in out and "init_plqcd" in out


@pytest.mark.gpu
@pytest.mark.parametrize("L", [(8, 8, 8, 16), (4, 6, 8, 10)])
def test_c_caller_matches_oracle(cuda, tmp_path, L):
    exe = build_c_caller(tmp_path)
    V = O.volume(L)
    rng = np.random.default_rng(31)
    q, u = O.gaussian_spinor(V, rng), O.random_su3(4 * V, rng)
    fin, fout = tmp_path / "fields.bin", tmp_path / "out.bin"
    with open(fin, "wb") as f:
        f.write(np.ascontiguousarray(q).tobytes())
        f.write(np.ascontiguousarray(u).tobytes())
    inp = O.write_input_file(L)
    try:
        env = dict(os.environ, PLQCD_DEVICE="0")
        _run([str(exe), inp, str(fin), str(fout)], env=env)
    finally:
        os.unlink(inp)
    got = np.fromfile(fout, dtype=np.complex128).reshape(V, 12)
    want = O.Restatement().hop("full", L, q, u)
    err = float(np.abs(got - want).max() / np.abs(want).max())
    assert err <= 1e-14, err
