"""C-ABI library: loads, exports every declared symbol, host-side behaviour.

Runs without a GPU: only host-side entry points are called (init_plqcd
geometry, helpers, utils, error reporting)."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import plqcd_b200 as P
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = P.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", P.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"
    assert "plqcd_g" in exported
    for n in declared_functions():
        getattr(L, n)
    # the Python binding covers every declared function
    assert set(declared_functions()) <= set(P.exported_symbols())


def test_declared_function_list_is_complete():
    names = declared_functions()
    for n in ["init_plqcd", "finalize_plqcd", "ipr", "comp_cpr", "set_npr", "lex2cart", "cart2lex",
              "set_geometry", "find_site", "print_params", "amalloc", "afree", "alloc", "stop_watch",
              "plqcd_hopping_matrix_eo_sse3_assymbly", "plqcd_hopping_matrix_oe_sse3_assymbly",
              "plqcd_hopping_matrix_eo_sse3_intrin_blocking", "plqcd_dslash", "plqcd_dslash_full"]:
        assert n in names


class GlobalParams(ctypes.Structure):
    """Mirror of struct _PLQCD_GLOBAL_PARAMS in include/plqcd_global_params.h."""
    _fields_ = [("nprocs", ctypes.c_int * 4), ("nthread", ctypes.c_int), ("cpr", ctypes.c_int * 4),
                ("npr", ctypes.c_int * 8), ("LX", ctypes.c_int), ("LY", ctypes.c_int), ("LZ", ctypes.c_int),
                ("LT", ctypes.c_int), ("latdims", ctypes.c_int * 4), ("VOLUME", ctypes.c_int),
                ("Vmic_split", ctypes.c_int), ("Vavx_split", ctypes.c_int), ("Vsse_split", ctypes.c_int),
                ("face", ctypes.c_int * 4), ("ipt_eo", ctypes.POINTER(ctypes.c_int)),
                ("ipt_lex", ctypes.POINTER(ctypes.c_int)), ("nn_bnde", ctypes.c_void_p * 8),
                ("nn_bndo", ctypes.c_void_p * 8), ("iup", ctypes.POINTER(ctypes.POINTER(ctypes.c_int))),
                ("idn", ctypes.POINTER(ctypes.POINTER(ctypes.c_int))),
                ("ipt_eo_yzt", ctypes.POINTER(ctypes.c_int)), ("ipt_lex_yzt", ctypes.POINTER(ctypes.c_int)),
                ("ipt_eo_sse_split", ctypes.c_void_p), ("ipt_lex_sse_split", ctypes.c_void_p),
                ("iup_sse_split", ctypes.c_void_p), ("idn_sse_split", ctypes.c_void_p),
                ("phip", ctypes.c_void_p * 4), ("phim", ctypes.c_void_p * 4), ("ALIGN", ctypes.c_int),
                ("init", ctypes.c_int)]


def g():
    return GlobalParams.in_dll(P.lib(), "plqcd_g")


@pytest.fixture
def initialised(tmp_path):
    path = O.write_input_file((4, 6, 8, 10), nthreads=2, align=6)
    P.finalize_plqcd()
    assert P.init_plqcd(path) == 0, P.last_error()
    yield
    P.finalize_plqcd()
    os.unlink(path)


def test_init_reads_input_and_builds_reference_tables(initialised):
    gp = g()
    assert gp.init == 1
    assert list(gp.latdims) == [4, 6, 8, 10] and gp.VOLUME == 1920
    assert gp.ALIGN == 6 and gp.nthread == 2 and list(gp.face) == [0, 0, 0, 0]
    gold = np.load(os.path.join(GOLD, "geom_4x6x8x10.npz"))
    V = gp.VOLUME
    assert np.array_equal(np.ctypeslib.as_array(gp.ipt_eo, (V,)), gold["ipt_eo"])
    assert np.array_equal(np.ctypeslib.as_array(gp.ipt_lex, (V,)), gold["ipt_lex"])
    iup = np.array([[gp.iup[i][m] for m in range(4)] for i in range(V)])
    idn = np.array([[gp.idn[i][m] for m in range(4)] for i in range(V)])
    assert np.array_equal(iup, gold["iup"]) and np.array_equal(idn, gold["idn"])


def test_geometry_helpers(initialised):
    L = P.lib()
    x = (ctypes.c_int * 4)(3, 5, 7, 9)
    ix = L.cart2lex(x)
    assert ix == 3 + 4 * (5 + 6 * (7 + 8 * 9))
    y = (ctypes.c_int * 4)()
    L.lex2cart(ix, y)
    assert list(y) == [3, 5, 7, 9]
    pid, xeo = ctypes.c_int(), ctypes.c_int()
    L.find_site(x, ctypes.byref(pid), ctypes.byref(xeo))
    assert pid.value == 0 and xeo.value == g().ipt_eo[ix]
    n = (ctypes.c_int * 4)(0, 0, 0, 0)
    assert L.ipr(n) == 0
    L.comp_cpr(0, n)
    assert list(n) == [0, 0, 0, 0]
    assert list(g().npr) == [0] * 8
    # out-of-range inputs are reported, not fatal (the reference exit()s)
    bad = (ctypes.c_int * 4)(4, 0, 0, 0)
    assert L.cart2lex(bad) == -1
    assert "out of bounds" in P.last_error()
    assert L.ipr((ctypes.c_int * 4)(1, 0, 0, 0)) == -1


def test_yzt_tables(initialised):
    gp = g()
    Vyzt = 6 * 8 * 10
    eo = np.ctypeslib.as_array(gp.ipt_eo_yzt, (Vyzt,))
    lex = np.ctypeslib.as_array(gp.ipt_lex_yzt, (Vyzt,))
    assert np.array_equal(lex[eo], np.arange(Vyzt))
    y, z, t = np.meshgrid(np.arange(6), np.arange(8), np.arange(10), indexing="ij")
    il = (y + 6 * z + 48 * t).ravel()
    par = ((y + z + t) % 2).ravel()
    assert np.all((eo[il] < Vyzt // 2) == (par == 0))


def test_print_params_format(initialised, tmp_path):
    libc = ctypes.CDLL(None)
    libc.fopen.restype = ctypes.c_void_p
    libc.fopen.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    libc.fclose.argtypes = [ctypes.c_void_p]
    p = tmp_path / "params.txt"
    fp = libc.fopen(str(p).encode(), b"w")
    P.lib().print_params(fp)
    libc.fclose(fp)
    text = p.read_text()
    assert "grid of processes: nprocs0 1 nprocs1 1 nprocs2 1 nprocs3 1" in text
    assert "Local lattice size: lx 4 ly 6 lz 8 lt 10, local volume 1920" in text
    assert "memory alignment in bytes: ALIGN 6" in text
    rows = [l for l in text.splitlines() if re.match(r"^\s+\d+(\s+\d+){13}\s*$", l)]
    assert len(rows) == 1920


@pytest.mark.parametrize("content,msg", [
    ("L0 5\nL1 4\nL2 4\nL3 4\n", ">= 4 and even"),
    ("L0 2\nL1 4\nL2 4\nL3 4\n", ">= 4 and even"),
    ("L0 4\nL1 4\nL2 4\nL3 4\nNPROC0 3\n", "1 or even"),
    ("L0 4\nL1 4\nL2 4\nL3 4\nNPROC3 2\n", "one process"),
])
def test_init_rejects_bad_input(tmp_path, content, msg):
    P.finalize_plqcd()
    p = tmp_path / "bad.input"
    p.write_text(content)
    assert P.init_plqcd(str(p)) != 0
    assert msg in P.last_error()
    assert g().init == 0


def test_init_missing_file():
    P.finalize_plqcd()
    assert P.init_plqcd("/nonexistent/input") != 0
    assert "cannot open" in P.last_error()


def test_hopping_before_init_fails_cleanly():
    P.finalize_plqcd()
    V = 256
    q = np.zeros((V, 12), complex)
    u = np.zeros((4 * V, 9), complex)
    t = P.lib().plqcd_hopping_matrix_eo_sse3_assymbly(q.ctypes.data, q.ctypes.data, u.ctypes.data)
    assert t < 0 and "before init_plqcd" in P.last_error()


def test_amalloc_alignment_and_afree():
    L = P.lib()
    for p in (4, 6, 12, 16):
        a = L.amalloc(1000, p)
        assert a and a % (1 << p) == 0
        ctypes.memset(a, 7, 1000)
        L.afree(a)
    assert L.amalloc(0, 4) is None
    assert L.amalloc(16, -1) is None
    L.afree(12345)  # unknown address: ignored
    b = L.alloc(4096, 64)
    assert b % 64 == 0
    ctypes.CDLL(None).free(ctypes.c_void_p(b))


def test_stop_watch_seconds_and_tags():
    L = P.lib()
    t0 = L.stop_watch(0.0)
    assert t0 > 1.6e9
    assert 0 <= L.stop_watch(t0) < 5
    a, b = L.mpi_permanent_tag(), L.mpi_permanent_tag()
    assert b == a + 1
    t = L.mpi_tag()
    assert t > 16383


def test_device_api_without_gpu_reports_error():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    with pytest.raises(P.PlqcdError, match="no CUDA device"):
        P.Lattice((4, 4, 4, 4))


@pytest.mark.parametrize("n", [0, 1, 12 * 257, 5_000_001])
def test_split_converters_roundtrip(n):
    """plqcd_aos_to_split / plqcd_split_to_aos: planes hold exactly the real
    and imaginary parts, and merging restores the array bit for bit (the
    largest case runs the multi-threaded path)."""
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    re, im = P.aos_to_split(a)
    assert np.array_equal(re, a.real) and np.array_equal(im, a.imag)
    b = np.zeros_like(a)
    P.split_to_aos(re, im, b)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_split_converters_reject_null():
    assert P.lib().plqcd_aos_to_split(None, None, None, 4) == P.ERR_ARG
    assert "bad argument" in P.last_error()
    x = np.zeros(4)
    assert P.lib().plqcd_split_to_aos(x.ctypes.data, x.ctypes.data, x.ctypes.data, -1) == P.ERR_ARG


def test_packed_field_types_known_answers(tmp_path):
    """include/su3_256.h and su3_512.h (the reference's two- and four-lane
    packed types, include/su3_256.h:14-191, su3_512.h:12-216): a C program
    compiled against the headers checks every lane of every element after
    packing and that unpacking restores the objects; the headers also
    compile as C++."""
    exe = tmp_path / "packed_types"
    src = os.path.join(ROOT, "tests", "c", "packed_types.c")
    r = subprocess.run(["gcc", "-std=c11", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), src,
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    cxx = tmp_path / "t.cpp"
    cxx.write_text('#include "su3_256.h"\n#include "su3_512.h"\nint main() { return 0; }\n')
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(cxx)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_print_params_matches_reference_golden(tmp_path):
    """print_params writes byte for byte what the reference's print_params
    (lib/start.c:1346-1428) wrote for the same 4^4 single-process setup
    (fixture from tests/golden/make_golden.py)."""
    P.finalize_plqcd()
    path = O.write_input_file((4, 4, 4, 4), nthreads=1, align=6)
    try:
        assert P.init_plqcd(path) == 0, P.last_error()
        libc = ctypes.CDLL(None)
        libc.fopen.restype = ctypes.c_void_p
        libc.fopen.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        libc.fclose.argtypes = [ctypes.c_void_p]
        out = tmp_path / "params.txt"
        fp = libc.fopen(str(out).encode(), b"w")
        P.lib().print_params(fp)
        libc.fclose(fp)
    finally:
        os.unlink(path)
        P.finalize_plqcd()
    want = open(os.path.join(GOLD, "print_params_4x4x4x4.txt"), "rb").read()
    assert out.read_bytes() == want


@pytest.mark.parametrize("lanes", [2, 4])
def test_python_lane_packing_matches_the_header_converters(tmp_path, lanes):
    """plqcd_b200.pack_lanes lays out spinors and links exactly as the
    packed-type converters do when driven like the reference's test driver
    (pairs / quadruples of consecutive even/odd sites), so the lane-packed
    entry points are tested on the layout legacy callers build."""
    so = tmp_path / "pack.so"
    r = subprocess.run(["gcc", "-std=c11", "-O2", "-shared", "-fPIC", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "c", "pack_arrays.c"), "-o", str(so)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lib = ctypes.CDLL(str(so))
    V = 64
    rng = np.random.default_rng(lanes)
    q = rng.standard_normal((V, 12)) + 1j * rng.standard_normal((V, 12))
    u = rng.standard_normal((4 * V, 9)) + 1j * rng.standard_normal((4 * V, 9))
    pq, pu = np.zeros_like(q), np.zeros_like(u)
    lib.pack_spinors(lanes, q.ctypes.data_as(ctypes.c_void_p), pq.ctypes.data_as(ctypes.c_void_p), V)
    lib.pack_links(lanes, u.ctypes.data_as(ctypes.c_void_p), pu.ctypes.data_as(ctypes.c_void_p), V)
    assert np.array_equal(pq.reshape(-1), P.pack_lanes(q, lanes).reshape(-1))
    assert np.array_equal(pu.reshape(-1), P.pack_lanes(u.reshape(V, 36), lanes).reshape(-1))
    assert np.array_equal(P.unpack_lanes(P.pack_lanes(q, lanes)), q)
