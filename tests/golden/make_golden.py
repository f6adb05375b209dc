"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own plain-C hopping pair (lib/dirac.c:35-791),
compiled from the read-only reference sources by oracle/build_ref.sh into
oracle/_ref/, on seeded inputs, and stores inputs and outputs:

  hop_4x4x4x4.npz   qin, u (random SU(3)), qout_patched, qout_shipped,
                    and the reference's geometry tables
  hop_8x8x8x16_summary.npz  seeds + per-(spin,colour) sums and norms of
                    the 8^3x16 outputs (the full arrays are too large to
                    commit; the inputs are regenerated from the seed)
  geom_4x6x8x10.npz the reference's ipt_eo/ipt_lex/iup/idn tables on a
                    lattice with four different extents
  print_params_4x4x4x4.txt  the text the reference's print_params
                    (lib/start.c:1346-1428) writes for a 4^4 lattice, one
                    process, one thread, ALIGN 6

The patched build fixes include/su3.h:135-138 and lib/dirac.c:643; the
shipped build is the reference as distributed. Usage (needs oracle/_ref):
    python tests/golden/make_golden.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402


def summarize(q):
    q = q.reshape(-1, 12)
    return np.stack([q.sum(axis=0), np.sqrt((np.abs(q) ** 2).sum(axis=0)) + 0j])


def main():
    P = O.CompiledReference("patched")
    S = O.CompiledReference("shipped")

    L = (4, 4, 4, 4)
    V = O.volume(L)
    rng = np.random.default_rng(20121)
    qin = O.gaussian_spinor(V, rng)
    u = O.random_su3(4 * V, rng)
    qp, _ = P.hop("full", L, qin, u)
    qs, _ = S.hop("full", L, qin, u)
    ipt_eo, ipt_lex, iup, idn = P.tables(L)
    np.savez_compressed(os.path.join(HERE, "hop_4x4x4x4.npz"), L=np.array(L), qin=qin, u=u,
                        qout_patched=qp, qout_shipped=qs, ipt_eo=ipt_eo, ipt_lex=ipt_lex, iup=iup, idn=idn)

    L = (8, 8, 8, 16)
    V = O.volume(L)
    seed = 1234
    rng = np.random.default_rng(seed)
    qin = O.gaussian_spinor(V, rng)
    u = O.random_su3(4 * V, rng)
    qp, _ = P.hop("full", L, qin, u, nthreads=4)
    qs, _ = S.hop("full", L, qin, u, nthreads=4)
    np.savez_compressed(os.path.join(HERE, "hop_8x8x8x16_summary.npz"), L=np.array(L), seed=seed,
                        qin_summary=summarize(qin), u_sum=u.sum(axis=0),
                        patched_summary=summarize(qp), shipped_summary=summarize(qs),
                        patched_probe=qp[::97], shipped_probe=qs[::97])

    L = (4, 6, 8, 10)
    ipt_eo, ipt_lex, iup, idn = P.tables(L)
    np.savez_compressed(os.path.join(HERE, "geom_4x6x8x10.npz"), L=np.array(L), ipt_eo=ipt_eo,
                        ipt_lex=ipt_lex, iup=iup, idn=idn)
    L = (4, 4, 4, 4)
    P.setup(L, 1)
    libc = ctypes.CDLL(None)
    libc.fopen.restype = ctypes.c_void_p
    libc.fopen.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    libc.fclose.argtypes = [ctypes.c_void_p]
    P.lib.print_params.argtypes = [ctypes.c_void_p]
    fp = libc.fopen(os.path.join(HERE, "print_params_4x4x4x4.txt").encode(), b"w")
    P.lib.print_params(fp)
    libc.fclose(fp)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
