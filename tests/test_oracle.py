"""The CPU oracle pinned against the reference's own outputs.

Golden fixtures in tests/golden/ were produced by the reference's plain-C
hopping pair (lib/dirac.c:35-791) compiled from its sources
(tests/golden/make_golden.py, oracle/build_ref.sh): the "patched" build with
the two one-line fixes and the "shipped" build as distributed.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_restatement_matches_reference_patched_bitexact(restatement):
    g = np.load(os.path.join(GOLD, "hop_4x4x4x4.npz"))
    L = tuple(g["L"])
    out = restatement.hop("full", L, g["qin"], g["u"])
    # same operation order as the reference's plain C: bit-identical
    assert np.array_equal(out, g["qout_patched"])


def test_restatement_compat_matches_reference_shipped_bitexact(restatement):
    g = np.load(os.path.join(GOLD, "hop_4x4x4x4.npz"))
    L = tuple(g["L"])
    out = restatement.hop("full", L, g["qin"], g["u"], compat=True)
    assert np.array_equal(out, g["qout_shipped"])


def test_shipped_differs_only_where_the_bugs_act(restatement):
    g = np.load(os.path.join(GOLD, "hop_4x4x4x4.npz"))
    p, s = g["qout_patched"], g["qout_shipped"]
    V = p.shape[0]
    # eo half: spins 0,1 agree exactly, spins 2,3 differ (include/su3.h:135-138)
    assert np.array_equal(p[: V // 2, :6], s[: V // 2, :6])
    assert np.abs(p[: V // 2, 6:] - s[: V // 2, 6:]).max() > 0.1
    # oe half: also wrong forward links (lib/dirac.c:643), so spins 0,1 differ
    assert np.abs(p[V // 2:, :6] - s[V // 2:, :6]).max() > 0.1


def test_restatement_matches_summary_8x8x8x16(restatement):
    g = np.load(os.path.join(GOLD, "hop_8x8x8x16_summary.npz"))
    L = tuple(g["L"])
    V = O.volume(L)
    rng = np.random.default_rng(int(g["seed"]))
    qin = O.gaussian_spinor(V, rng)
    u = O.random_su3(4 * V, rng)
    # the regenerated inputs are the ones the fixture was made from
    np.testing.assert_allclose(O_summary(qin), g["qin_summary"], rtol=1e-13)
    out = restatement.hop("full", L, qin, u)
    np.testing.assert_allclose(O_summary(out), g["patched_summary"], rtol=1e-12, atol=1e-9)
    assert np.array_equal(out[::97], g["patched_probe"])
    outc = restatement.hop("full", L, qin, u, compat=True)
    assert np.array_equal(outc[::97], g["shipped_probe"])


def O_summary(q):
    q = q.reshape(-1, 12)
    return np.stack([q.sum(axis=0), np.sqrt((np.abs(q) ** 2).sum(axis=0)) + 0j])


@pytest.mark.parametrize("fname", ["hop_4x4x4x4.npz", "geom_4x6x8x10.npz"])
def test_geometry_tables_match_reference(restatement, fname):
    g = np.load(os.path.join(GOLD, fname))
    L = tuple(g["L"])
    ipt_eo, ipt_lex, iup, idn = restatement.geometry(L)
    assert np.array_equal(ipt_eo, g["ipt_eo"])
    assert np.array_equal(ipt_lex, g["ipt_lex"])
    assert np.array_equal(iup, g["iup"])
    assert np.array_equal(idn, g["idn"])


def test_naive_gamma_formula_matches_golden(restatement):
    g = np.load(os.path.join(GOLD, "hop_4x4x4x4.npz"))
    L = tuple(g["L"])
    out = O.naive_hop(L, g["qin"], g["u"], g["ipt_lex"])
    np.testing.assert_allclose(out, g["qout_patched"], rtol=0, atol=1e-13)


def test_gamma_basis_properties():
    gs = O.gamma_matrices()
    for a, ga in enumerate(gs):
        np.testing.assert_allclose(ga, ga.conj().T)           # hermitian
        for b, gb in enumerate(gs):
            ac = ga @ gb + gb @ ga
            np.testing.assert_allclose(ac, 2 * np.eye(4) * (a == b), atol=1e-15)
    np.testing.assert_allclose(gs[0] @ gs[1] @ gs[2] @ gs[3], O.GAMMA5)


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (4, 6, 4, 8)])
def test_gamma5_hermiticity_oracle(restatement, L):
    # <phi, H psi> = <g5 H g5 phi, psi> on the full lattice
    V = O.volume(L)
    rng = np.random.default_rng(3)
    u = O.random_su3(4 * V, rng)
    phi, psi = O.gaussian_spinor(V, rng), O.gaussian_spinor(V, rng)
    g5 = np.array([1] * 6 + [-1] * 6)
    lhs = np.vdot(phi, restatement.hop("full", L, psi, u))
    rhs = np.vdot(g5 * restatement.hop("full", L, g5 * phi, u), psi)
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)


def test_unit_gauge_point_source_kat(restatement):
    """Point source with U = 1: non-zero output at exactly the 8 neighbours,
    with the spin structure (1 -/+ g_mu) (the neighbour pattern of the
    reference's tests/test_comms.c:167-497, with links and gammas)."""
    L = (4, 4, 4, 6)
    V = O.volume(L)
    u = np.tile(np.eye(3, dtype=complex).reshape(1, 9), (4 * V, 1))
    ipt_eo, ipt_lex, iup, idn = restatement.geometry(L)
    src_site, s, c = 5, 2, 1
    q = np.zeros((V, 12), complex)
    q[src_site, 3 * s + c] = 1.0
    out = restatement.hop("full", L, q, u)
    nz = set(np.nonzero(np.abs(out).sum(axis=1))[0])
    assert nz == set(iup[src_site]) | set(idn[src_site])
    gs = O.gamma_matrices()
    for mu in range(4):
        # the site whose +mu neighbour is the source gets (1 - g_mu) e_s
        y = idn[src_site, mu]
        np.testing.assert_allclose(out[y].reshape(4, 3)[:, c], (np.eye(4) - gs[mu])[:, s], atol=1e-15)
        y = iup[src_site, mu]
        np.testing.assert_allclose(out[y].reshape(4, 3)[:, c], (np.eye(4) + gs[mu])[:, s], atol=1e-15)


def test_oracle_cg_converges_small(restatement):
    L = (4, 4, 4, 4)
    V = O.volume(L)
    rng = np.random.default_rng(7)
    u = O.random_su3(4 * V, rng)
    b = O.gaussian_spinor(V, rng)
    x, it, rel = restatement.cg_solve(L, u, b, 0.12, tol=1e-10)
    assert rel < 1e-10
    r = b - restatement.wilson(L, u, x, 0.12)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10
    assert 5 < it < 200
