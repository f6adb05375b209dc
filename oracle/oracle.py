"""CPU oracles for the Wilson hopping matrix -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, always as the checker (or as the timed CPU
reference), never as the thing measured or shipped.

Three independent implementations are wrapped here:

* ``Restatement``: oracle/hop_oracle.c, a gather-form restatement of the
  reference's plain-C pair (lib/dirac.c:35-408 eo, 414-791 oe) with a
  bug-compatible ``compat`` mode, plus an FP64 CG on the even/odd Schur
  operator.
* ``CompiledReference``: the reference's own lib/dirac.c + lib/start.c +
  lib/utils.c compiled by oracle/build_ref.sh, either with the two one-line
  fixes ("patched") or exactly as shipped ("shipped").
* ``naive_hop``: a numpy evaluation of the operator from explicit gamma
  matrices (the basis implied by lib/dirac.c:95-114/163-195/269-311/371-398)
  with ``np.roll`` neighbours on the lexicographic lattice.

Field layout (the reference's API layout, include/su3.h:52-75): a spinor
field is complex128 of shape (V, 12) with index 3*spin+colour, a gauge field
is complex128 of shape (4V, 9), link (i, mu) at row 4*i+mu, row-major 3x3.
Site index i is the even/odd index of lib/start.c:406-433.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)


def reference_root() -> str:
    """Root of the reference's sources: $PLQCD_REFERENCE_ROOT, else the
    default of the build recipe (oracle/build_ref.sh --root). Only the
    recipe and the tests that compile the reference's own files use it; no
    GPU test, smoke() or bench.py reads the reference's sources."""
    r = os.environ.get("PLQCD_REFERENCE_ROOT")
    if r:
        return r
    out = subprocess.run(["bash", os.path.join(HERE, "build_ref.sh"), "--root"], capture_output=True, text=True)
    return out.stdout.strip()


def build(root: str | None = None) -> None:
    """Compile the oracles (oracle/build_ref.sh)."""
    subprocess.run(["bash", os.path.join(HERE, "build_ref.sh"), root or reference_root()], check=True)


def _dims(L):
    a = (ctypes.c_int * 4)(*[int(x) for x in L])
    return a


def _dptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(_c_dbl_p)


def volume(L) -> int:
    return int(L[0]) * int(L[1]) * int(L[2]) * int(L[3])


# ---------------------------------------------------------------------------
# random inputs (seeded numpy; the product has its own device generator)
# ---------------------------------------------------------------------------

def random_su3(n: int, rng: np.random.Generator) -> np.ndarray:
    """n random SU(3) matrices, shape (n, 9): Gaussian complex 3x3, rows 0,1
    Gram-Schmidt orthonormalised, row 2 = conj(row0 x row1)."""
    a = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    r0 = a[:, 0, :]
    r0 = r0 / np.linalg.norm(r0, axis=1, keepdims=True)
    r1 = a[:, 1, :] - np.sum(np.conj(r0) * a[:, 1, :], axis=1, keepdims=True) * r0
    r1 = r1 / np.linalg.norm(r1, axis=1, keepdims=True)
    r2 = np.conj(np.cross(r0, r1))
    return np.ascontiguousarray(np.stack([r0, r1, r2], axis=1).reshape(n, 9))


def gaussian_spinor(V: int, rng: np.random.Generator) -> np.ndarray:
    """V i.i.d. N(0,1) complex spinors, shape (V, 12)."""
    return np.ascontiguousarray(rng.standard_normal((V, 12)) + 1j * rng.standard_normal((V, 12)))


def uniform_spinor(V: int, rng: np.random.Generator) -> np.ndarray:
    """Uniform [0,1) real and imaginary parts, as the reference's driver
    fills its fields (tests/test_hopping.c:193-213)."""
    return np.ascontiguousarray(rng.random((V, 12)) + 1j * rng.random((V, 12)))


# ---------------------------------------------------------------------------
# restatement (oracle/hop_oracle.c)
# ---------------------------------------------------------------------------

class Restatement:
    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "libhop_oracle.so")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.orc_geometry.argtypes = [_c_int_p, _c_int_p, _c_int_p, _c_int_p, _c_int_p]
        for f in (L.orc_hop_eo, L.orc_hop_oe):
            f.argtypes = [_c_int_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, ctypes.c_int, ctypes.c_int]
        L.orc_wilson.argtypes = [_c_int_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, ctypes.c_double, ctypes.c_int]
        L.orc_cg_solve.argtypes = [_c_int_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int, _c_dbl_p, ctypes.c_int]
        L.orc_cg_solve.restype = ctypes.c_int

    def geometry(self, L):
        V = volume(L)
        ipt_eo = np.zeros(V, np.int32)
        ipt_lex = np.zeros(V, np.int32)
        iup = np.zeros((V, 4), np.int32)
        idn = np.zeros((V, 4), np.int32)
        ip = lambda a: a.ctypes.data_as(_c_int_p)
        self.lib.orc_geometry(_dims(L), ip(ipt_eo), ip(ipt_lex), ip(iup), ip(idn))
        return ipt_eo, ipt_lex, iup, idn

    def hop(self, which: str, L, qin: np.ndarray, u: np.ndarray, qout: np.ndarray | None = None,
            compat: bool = False, nthreads: int = 0) -> np.ndarray:
        """which in {'eo', 'oe', 'full'}; returns the full-length output
        array (the other half is left as given in ``qout`` or zero)."""
        V = volume(L)
        qin = np.ascontiguousarray(qin, np.complex128)
        u = np.ascontiguousarray(u, np.complex128)
        assert qin.shape == (V, 12) and u.shape == (4 * V, 9)
        out = np.zeros((V, 12), np.complex128) if qout is None else np.array(qout, np.complex128, copy=True)
        if which in ("eo", "full"):
            self.lib.orc_hop_eo(_dims(L), _dptr(qin), _dptr(out), _dptr(u), int(compat), nthreads)
        if which in ("oe", "full"):
            self.lib.orc_hop_oe(_dims(L), _dptr(qin), _dptr(out), _dptr(u), int(compat), nthreads)
        return out

    def wilson(self, L, u, x, kappa, nthreads: int = 0):
        out = np.zeros_like(x)
        self.lib.orc_wilson(_dims(L), _dptr(u), _dptr(np.ascontiguousarray(x)), _dptr(out), kappa, nthreads)
        return out

    def cg_solve(self, L, u, b, kappa, tol=1e-10, maxiter=10000, nthreads: int = 0):
        """Solve D x = b, D = 1 - kappa H, by even/odd preconditioned CG on
        Mhat^dag Mhat. Returns (x, iterations, true relative residual)."""
        x = np.zeros_like(b)
        rel = ctypes.c_double(0)
        it = self.lib.orc_cg_solve(_dims(L), _dptr(u), _dptr(np.ascontiguousarray(b)), _dptr(x), kappa, tol,
                                   maxiter, ctypes.byref(rel), nthreads)
        return x, it, rel.value


# ---------------------------------------------------------------------------
# compiled reference (oracle/_ref, built by oracle/build_ref.sh)
# ---------------------------------------------------------------------------

class CompiledReference:
    """The reference's plain-C hopping pair, compiled from its own sources.

    variant 'patched': _vector_minus_assign fixed (include/su3.h:135-138) and
    the oe forward link fixed (lib/dirac.c:643); 'shipped': as distributed.
    """

    def __init__(self, variant: str = "patched"):
        path = os.path.join(REF_DIR, f"libplqcd_ref_{variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run oracle/build_ref.sh")
        self.variant = variant
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.oracle_ref_setup.argtypes = [ctypes.c_int] * 5
        L.oracle_ref_setup.restype = ctypes.c_int
        L.oracle_ref_set_threads.argtypes = [ctypes.c_int]
        for f in (L.plqcd_hopping_matrix_eo_sse3_assymbly, L.plqcd_hopping_matrix_oe_sse3_assymbly):
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            f.restype = ctypes.c_double
        L.oracle_ref_tables.argtypes = [_c_int_p] * 4
        self.dims = None

    def tables(self, L):
        """(ipt_eo, ipt_lex, iup, idn) as built by the reference's
        set_geometry (lib/start.c:406-526)."""
        self.setup(L)
        V = volume(L)
        ipt_eo = np.zeros(V, np.int32)
        ipt_lex = np.zeros(V, np.int32)
        iup = np.zeros((V, 4), np.int32)
        idn = np.zeros((V, 4), np.int32)
        ip = lambda a: a.ctypes.data_as(_c_int_p)
        self.lib.oracle_ref_tables(ip(ipt_eo), ip(ipt_lex), ip(iup), ip(idn))
        return ipt_eo, ipt_lex, iup, idn

    def setup(self, L, nthreads: int = 1):
        L = tuple(int(x) for x in L)
        if self.dims != L:
            rc = self.lib.oracle_ref_setup(*L, int(nthreads))
            if rc != 0:
                raise RuntimeError("oracle_ref_setup failed")
            self.dims = L
        self.lib.oracle_ref_set_threads(int(nthreads))

    def hop(self, which: str, L, qin: np.ndarray, u: np.ndarray, qout: np.ndarray | None = None,
            nthreads: int = 1):
        """Returns (qout, seconds) where seconds is the sum of the
        reference's own return values (lib/dirac.c:405-407)."""
        self.setup(L, nthreads)
        V = volume(L)
        qin = np.ascontiguousarray(qin, np.complex128)
        u = np.ascontiguousarray(u, np.complex128)
        assert qin.shape == (V, 12) and u.shape == (4 * V, 9)
        out = np.zeros((V, 12), np.complex128) if qout is None else np.array(qout, np.complex128, copy=True)
        t = 0.0
        if which in ("eo", "full"):
            t += self.lib.plqcd_hopping_matrix_eo_sse3_assymbly(qin.ctypes.data, out.ctypes.data, u.ctypes.data)
        if which in ("oe", "full"):
            t += self.lib.plqcd_hopping_matrix_oe_sse3_assymbly(qin.ctypes.data, out.ctypes.data, u.ctypes.data)
        return out, t


# ---------------------------------------------------------------------------
# naive numpy evaluation from explicit gamma matrices
# ---------------------------------------------------------------------------

def gamma_matrices() -> list[np.ndarray]:
    """gamma_mu implied by the reference's projections: the forward term
    uses (1 - gamma_mu) psi(x+mu), the backward term (1 + gamma_mu) psi(x-mu)
    (lib/dirac.c:95-114, 163-195 with the rebuild of 269-311, 371-398)."""
    i = 1j
    g0 = np.array([[0, 0, -1, 0], [0, 0, 0, -1], [-1, 0, 0, 0], [0, -1, 0, 0]], complex)
    g1 = np.array([[0, 0, 0, -i], [0, 0, -i, 0], [0, i, 0, 0], [i, 0, 0, 0]], complex)
    g2 = np.array([[0, 0, 0, -1], [0, 0, 1, 0], [0, 1, 0, 0], [-1, 0, 0, 0]], complex)
    g3 = np.array([[0, 0, -i, 0], [0, 0, 0, i], [i, 0, 0, 0], [0, -i, 0, 0]], complex)
    return [g0, g1, g2, g3]


GAMMA5 = np.diag([1, 1, -1, -1]).astype(complex)


def naive_hop(L, qin: np.ndarray, u: np.ndarray, ipt_lex: np.ndarray) -> np.ndarray:
    """Full-lattice H psi (both parities) from the formula
    sum_mu U_mu(x)(1-g_mu)psi(x+mu) + U_mu(x-mu)^dag (1+g_mu) psi(x-mu)."""
    V = volume(L)
    shape = (L[3], L[2], L[1], L[0])            # lexicographic, x fastest
    axis = {0: 3, 1: 2, 2: 1, 3: 0}
    psi = np.empty((V, 4, 3), complex)
    psi[ipt_lex] = qin.reshape(V, 4, 3)
    psi = psi.reshape(shape + (4, 3))
    U = np.empty((V, 4, 3, 3), complex)
    U[ipt_lex] = u.reshape(V, 4, 3, 3)
    U = U.reshape(shape + (4, 3, 3))
    out = np.zeros_like(psi)
    one = np.eye(4)
    for mu, g in enumerate(gamma_matrices()):
        ax = axis[mu]
        fwd = np.roll(psi, -1, axis=ax)           # psi(x+mu)
        bwd = np.roll(psi, +1, axis=ax)           # psi(x-mu)
        Ub = np.roll(U[..., mu, :, :], +1, axis=ax)   # U_mu(x-mu)
        pf = np.einsum("st,...tc->...sc", one - g, fwd)
        pb = np.einsum("st,...tc->...sc", one + g, bwd)
        out += np.einsum("...ab,...sb->...sa", U[..., mu, :, :], pf)
        out += np.einsum("...ba,...sb->...sa", np.conj(Ub), pb)
    out = out.reshape(V, 12)
    res = np.empty_like(out)
    res[:] = out[ipt_lex]
    return res


def lex_to_eo(field_lex: np.ndarray, ipt_lex: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(field_lex[ipt_lex])


def write_input_file(L, nthreads: int = 1, align: int = 6, nprocs=(1, 1, 1, 1)) -> str:
    """Key-value input file in the format init_plqcd reads
    (lib/start.c:84-107; tests/test.input)."""
    fd, path = tempfile.mkstemp(suffix=".input")
    with os.fdopen(fd, "w") as f:
        for k in range(4):
            f.write(f"L{k} {int(L[k])}\n")
        for k in range(4):
            f.write(f"NPROC{k} {int(nprocs[k])}\n")
        f.write(f"NTHREAD {int(nthreads)}\nALIGN {int(align)}\n")
    return path
