"""Parity of the sm_100a hopping kernels with the oracle, through the C-ABI.

FP64 results must match the reference's operator to 1e-14 relative
(max |diff| / max |value|); reduced precisions are bounded in relative L2
against the FP64 kernel."""
import ctypes
import os

import numpy as np
import pytest

import plqcd_b200 as P
from oracle import oracle as O
from tests.gpu_util import dev_bytes, field_from_host, field_to_host, new_lattice, rel_l2, relmax, to_dev

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL64 = 1e-14


@pytest.fixture
def dropin(cuda):
    paths = []

    def init(L):
        P.finalize_plqcd()
        p = O.write_input_file(L)
        paths.append(p)
        assert P.init_plqcd(p) == 0, P.last_error()

    yield init
    P.finalize_plqcd()
    os.environ.pop("PLQCD_REF_COMPAT", None)
    for p in paths:
        os.unlink(p)


def test_dropin_golden_4x4x4x4(dropin):
    g = np.load(os.path.join(GOLD, "hop_4x4x4x4.npz"))
    L = tuple(g["L"])
    dropin(L)
    qout = np.zeros_like(g["qin"])
    t1 = P.hopping_matrix("eo", g["qin"], qout, g["u"])
    t2 = P.hopping_matrix("oe", g["qin"], qout, g["u"])
    assert t1 > 0 and t2 > 0
    assert relmax(qout, g["qout_patched"]) < TOL64


def test_dropin_compat_reproduces_shipped_reference(dropin):
    g = np.load(os.path.join(GOLD, "hop_4x4x4x4.npz"))
    dropin(tuple(g["L"]))
    os.environ["PLQCD_REF_COMPAT"] = "1"
    qout = np.zeros_like(g["qin"])
    P.hopping_matrix("eo", g["qin"], qout, g["u"])
    P.hopping_matrix("oe", g["qin"], qout, g["u"])
    assert relmax(qout, g["qout_shipped"]) < TOL64


@pytest.mark.parametrize("L", [(8, 8, 8, 16), (4, 6, 8, 10), (6, 4, 4, 4), (16, 8, 4, 4)])
@pytest.mark.parametrize("fill", ["su3", "uniform"])
def test_dropin_matches_oracle(dropin, restatement, L, fill):
    dropin(L)
    V = O.volume(L)
    rng = np.random.default_rng(11)
    if fill == "su3":
        q, u = O.gaussian_spinor(V, rng), O.random_su3(4 * V, rng)
    else:  # the reference driver's fill: rand()/RAND_MAX, links not SU(3)
        q, u = O.uniform_spinor(V, rng), O.uniform_spinor(4 * V, rng)[:, :9].copy()
    want = restatement.hop("full", L, q, u)
    got = np.full_like(q, np.nan)
    P.hopping_matrix("eo", q, got, u, variant="sse3_intrin")
    # only the even half is written by eo
    assert np.isnan(got[V // 2:]).all() and not np.isnan(got[: V // 2]).any()
    P.hopping_matrix("oe", q, got, u, variant="sse3_intrin_blocking")
    assert relmax(got, want) < TOL64


def test_dropin_gauge_cache_sees_in_place_update(dropin, restatement):
    L = (4, 4, 4, 8)
    dropin(L)
    V = O.volume(L)
    rng = np.random.default_rng(5)
    q, u = O.gaussian_spinor(V, rng), O.random_su3(4 * V, rng)
    out = np.zeros_like(q)
    P.hopping_matrix("eo", q, out, u)
    u[:] = O.random_su3(4 * V, rng)            # same address, new links
    P.lib().plqcd_gauge_update(u.ctypes.data)
    P.hopping_matrix("eo", q, out, u)
    want = restatement.hop("eo", L, q, u)
    assert relmax(out[: V // 2], want[: V // 2]) < TOL64


def test_dropin_reads_links_on_every_call_by_default(dropin, restatement):
    """Without a registration the drop-in call reads the link array every
    time, as the reference does: one link changed in place (far from any
    sampled word) shows up in the next call's output."""
    L = (4, 4, 4, 8)
    dropin(L)
    V = O.volume(L)
    rng = np.random.default_rng(6)
    q, u = O.gaussian_spinor(V, rng), O.random_su3(4 * V, rng)
    out = np.zeros_like(q)
    P.hopping_matrix("eo", q, out, u)
    P.hopping_matrix("eo", q, out, u)
    k = 4 * (V // 2 + 37) + 2                 # U_z at odd site 37, read by the even outputs
    u[k] = O.random_su3(1, rng)[0]
    P.hopping_matrix("eo", q, out, u)
    want = restatement.hop("eo", L, q, u)
    assert relmax(out[: V // 2], want[: V // 2]) < TOL64
    _, h2d, _ = P.dropin_last_stats()
    assert h2d >= 4 * V * 144                 # the links went up again


def test_dropin_registered_links_are_uploaded_once(dropin, restatement):
    """plqcd_gauge_update(u) registers the array: later calls reuse the
    device copy (only the spinor parity goes up) until the next
    plqcd_gauge_update, which picks up links changed in place."""
    L = (4, 4, 4, 8)
    dropin(L)
    V = O.volume(L)
    rng = np.random.default_rng(7)
    q, u = O.gaussian_spinor(V, rng), O.random_su3(4 * V, rng)
    P.lib().plqcd_gauge_update(u.ctypes.data)
    out = np.zeros_like(q)
    P.hopping_matrix("eo", q, out, u)
    P.hopping_matrix("eo", q, out, u)
    _, h2d, _ = P.dropin_last_stats()
    assert h2d < 4 * V * 144                  # spinor parity only
    assert relmax(out[: V // 2], restatement.hop("eo", L, q, u)[: V // 2]) < TOL64
    u[4 * (V // 2 + 11) + 1] = O.random_su3(1, rng)[0]
    P.lib().plqcd_gauge_update(u.ctypes.data)
    P.hopping_matrix("eo", q, out, u)
    assert relmax(out[: V // 2], restatement.hop("eo", L, q, u)[: V // 2]) < TOL64


def _pinned(lib, shape):
    """complex128 array on amalloc'd (pinned) host memory, and its block"""
    n = int(np.prod(shape)) * 16
    p = lib.amalloc(n, 6)
    a = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_double)), (n // 8,)).view(np.complex128)
    return a.reshape(shape), p


@pytest.mark.parametrize("chunks", ["ramp", "1", "3", "16", "64"])
def test_dropin_pipeline_graph_and_chunking(dropin, restatement, monkeypatch, chunks):
    """Pinned host arrays: the first call runs the chunked copy/compute
    pipeline eagerly, the second captures it as a CUDA graph, later calls
    replay it. Every call, for every chunk count, gives the oracle's result
    and the same bits as the eager pipeline; a new output array is a new
    graph (no stale pointers)."""
    L = (8, 8, 4, 16)
    dropin(L)
    V = O.volume(L)
    lib = P.lib()
    rng = np.random.default_rng(17)
    qin, pq = _pinned(lib, (V, 12))
    u, pu = _pinned(lib, (4 * V, 9))
    qin[:] = O.gaussian_spinor(V, rng)
    u[:] = O.random_su3(4 * V, rng)
    want = restatement.hop("full", L, qin, u)
    if chunks == "ramp":  # the default plan: 1, 1, 2, ... slab chunks from both ends
        monkeypatch.delenv("PLQCD_DROPIN_CHUNKS", raising=False)
    else:
        monkeypatch.setenv("PLQCD_DROPIN_CHUNKS", chunks)
    outs = []
    try:
        for graph in ("0", "1"):
            monkeypatch.setenv("PLQCD_DROPIN_GRAPH", graph)
            for _ in range(3):
                qout, po = _pinned(lib, (V, 12))
                for rep in range(3):
                    qout[:] = 0
                    P.hopping_matrix("eo", qin, qout, u)
                    P.hopping_matrix("oe", qin, qout, u)
                    assert relmax(qout, want) < TOL64
                    outs.append(np.array(qout))
                lib.afree(po)
    finally:
        lib.afree(pq)
        lib.afree(pu)
    assert all(bool((o == outs[0]).all()) for o in outs)


def _device_setup(L, seed=1):
    lat = new_lattice(L)
    g64 = P.Gauge(lat, P.F64, 18)
    g64.random(seed)
    u = g64.store_host()
    return lat, g64, u


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (8, 4, 6, 10), (16, 16, 16, 32)])
@pytest.mark.parametrize("recon", [18, 12])
def test_device_dslash_f64_matches_oracle(cuda, restatement, L, recon):
    lat, g64, u = _device_setup(L)
    g = g64 if recon == 18 else P.Gauge(lat, P.F64, 12)
    if recon == 12:
        g.copy_from(g64)
    V = lat.V
    q = O.gaussian_spinor(V, np.random.default_rng(2))
    want = restatement.hop("full", L, q, u)
    fe, fo = field_from_host(lat, q, 0, P.F64), field_from_host(lat, q, 1, P.F64)
    oe_, oo_ = dev_bytes(lat.spinor_bytes(P.F64)), dev_bytes(lat.spinor_bytes(P.F64))
    lat.dslash(g, oe_, fo, P.EVEN, P.F64)
    lat.dslash(g, oo_, fe, P.ODD, P.F64)
    got = field_to_host(lat, oe_, P.F64, 0)
    got[V // 2:] = field_to_host(lat, oo_, P.F64, 1)[V // 2:]
    # 12-real storage rebuilds row 2 in FP64: agreement at rounding level
    assert relmax(got, want) < (TOL64 if recon == 18 else 1e-13)


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (8, 6, 4, 10)])
def test_full_lattice_kernel_equals_two_halves(cuda, L):
    lat, g64, u = _device_setup(L, 3)
    bs = lat.spinor_bytes(P.F64)
    fe, fo = dev_bytes(bs), dev_bytes(bs)
    lat.spinor_gaussian(fe, P.F64, 0, 9)
    lat.spinor_gaussian(fo, P.F64, 1, 9)
    a_e, a_o, b_e, b_o = (dev_bytes(bs) for _ in range(4))
    lat.dslash(g64, a_e, fo, 0, P.F64)
    lat.dslash(g64, a_o, fe, 1, P.F64)
    lat.dslash_full(g64, b_e, b_o, fe, fo, P.F64)
    lat.synchronize()
    assert bool((a_e == b_e).all()) and bool((a_o == b_o).all())


@pytest.mark.parametrize("prec,recon,tol", [(P.F32, 18, 2e-6), (P.F32, 12, 3e-6), (P.F16, 12, 2e-3),
                                            (P.BF16, 12, 1.5e-2)])
def test_reduced_precision_error(cuda, prec, recon, tol):
    L = (8, 8, 8, 16)
    lat, g64, u = _device_setup(L, 4)
    g = P.Gauge(lat, prec, recon)
    g.copy_from(g64)
    V = lat.V
    q = O.gaussian_spinor(V, np.random.default_rng(8))
    f64 = field_from_host(lat, q, 1, P.F64)
    ref = dev_bytes(lat.spinor_bytes(P.F64))
    lat.dslash(g64, ref, f64, 0, P.F64)
    flo = dev_bytes(lat.spinor_bytes(prec))
    lat.spinor_convert(flo, prec, f64, P.F64)
    out = dev_bytes(lat.spinor_bytes(prec))
    lat.dslash(g, out, flo, 0, prec)
    want = field_to_host(lat, ref, P.F64, 0)[: V // 2]
    got = field_to_host(lat, out, prec, 0)[: V // 2]
    err = rel_l2(got, want)
    assert err < tol, err


def test_xpay_and_gamma5_flags(cuda, restatement):
    L = (4, 4, 6, 8)
    lat, g64, u = _device_setup(L, 6)
    V = lat.V
    rng = np.random.default_rng(12)
    q, x = O.gaussian_spinor(V, rng), O.gaussian_spinor(V, rng)
    g5 = np.array([1.0] * 6 + [-1.0] * 6)
    fin = field_from_host(lat, q, 1, P.F64)
    fx = field_from_host(lat, x, 0, P.F64)
    out = dev_bytes(lat.spinor_bytes(P.F64))
    a, b = -0.0144, 1.0
    lat.dslash_xpay(g64, out, fin, 0, P.F64, a, fx, b, flags=P.DSLASH_G5_IN | P.DSLASH_G5_OUT)
    got = field_to_host(lat, out, P.F64, 0)[: V // 2]
    h = restatement.hop("eo", L, g5 * q, u)[: V // 2]
    want = b * x[: V // 2] + a * (g5 * h)
    assert relmax(got, want) < TOL64


def test_point_source_kat_gpu(cuda, restatement):
    L = (4, 4, 4, 6)
    lat = new_lattice(L)
    g = P.Gauge(lat, P.F64, 18)
    g.unit()
    V = lat.V
    _, _, iup, idn = restatement.geometry(L)
    src, s, c = V // 2 + 7, 3, 2  # an odd site
    q = np.zeros((V, 12), complex)
    q[src, 3 * s + c] = 1.0
    fo = field_from_host(lat, q, 1, P.F64)
    out = dev_bytes(lat.spinor_bytes(P.F64))
    lat.dslash(g, out, fo, 0, P.F64)
    got = field_to_host(lat, out, P.F64, 0)[: V // 2]
    nz = set(np.nonzero(np.abs(got).sum(axis=1))[0])
    assert nz == set(iup[src]) | set(idn[src])
    gs = O.gamma_matrices()
    for mu in range(4):
        np.testing.assert_allclose(got[idn[src, mu]].reshape(4, 3)[:, c], (np.eye(4) - gs[mu])[:, s], atol=0)
        np.testing.assert_allclose(got[iup[src, mu]].reshape(4, 3)[:, c], (np.eye(4) + gs[mu])[:, s], atol=0)


def test_random_gauge_is_su3(cuda):
    lat, g64, u = _device_setup((4, 4, 4, 8), 21)
    U = u.reshape(-1, 3, 3)
    eye = np.eye(3)
    assert np.abs(np.einsum("nab,ncb->nac", U, U.conj()) - eye).max() < 1e-14
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-14
    # a different seed gives different links; the same seed the same links
    g2 = P.Gauge(lat, P.F64, 18)
    g2.random(21)
    assert np.array_equal(g2.store_host(), u)
    g2.random(22)
    assert not np.allclose(g2.store_host(), u)


def test_gauge_and_spinor_roundtrips(cuda):
    L = (4, 6, 4, 8)
    lat = new_lattice(L)
    V = lat.V
    rng = np.random.default_rng(4)
    u = O.random_su3(4 * V, rng)
    g = P.Gauge(lat, P.F64, 18)
    g.load_host(u)
    assert np.array_equal(g.store_host(), u)
    g12 = P.Gauge(lat, P.F64, 12)
    g12.load_host(u)
    np.testing.assert_allclose(g12.store_host(), u, atol=1e-15)
    gd = P.Gauge(lat, P.F64, 18)
    gd.load_device(to_dev(u))
    assert np.array_equal(gd.store_host(), u)
    q = O.gaussian_spinor(V, rng)
    for par in (0, 1):
        f = field_from_host(lat, q, par, P.F64)
        back = field_to_host(lat, f, P.F64, par)
        sl = slice(0, V // 2) if par == 0 else slice(V // 2, V)
        assert np.array_equal(back[sl], q[sl])
    f = field_from_host(lat, q, 0, P.F64)
    for prec, tol in ((P.F32, 1e-7), (P.F16, 1e-3), (P.BF16, 8e-3)):
        lo = dev_bytes(lat.spinor_bytes(prec))
        lat.spinor_convert(lo, prec, f, P.F64)
        back = field_to_host(lat, lo, prec, 0)[: V // 2]
        assert rel_l2(back, q[: V // 2]) < tol


def test_gamma5_hermiticity_and_gauge_covariance_large(cuda):
    """Size-independent properties at 16^3x32 on device-generated fields:
    <phi_e, H_eo psi_o> = <g5 H_oe g5 phi_e, psi_o>; and H transforms
    covariantly under a random local SU(3) rotation."""
    L = (16, 16, 16, 32)
    lat, g64, u = _device_setup(L, 31)
    V = lat.V
    bs = lat.spinor_bytes(P.F64)
    phi, psi = dev_bytes(bs), dev_bytes(bs)
    lat.spinor_gaussian(phi, P.F64, 0, 1)
    lat.spinor_gaussian(psi, P.F64, 1, 2)
    a, b = dev_bytes(bs), dev_bytes(bs)
    lat.dslash(g64, a, psi, 0, P.F64)                                     # H_eo psi
    lat.dslash(g64, b, phi, 1, P.F64, flags=P.DSLASH_G5_IN | P.DSLASH_G5_OUT)  # g5 H_oe g5 phi
    ph = field_to_host(lat, phi, P.F64, 0)[: V // 2]
    ps = field_to_host(lat, psi, P.F64, 1)[V // 2:]
    A = field_to_host(lat, a, P.F64, 0)[: V // 2]
    B = field_to_host(lat, b, P.F64, 1)[V // 2:]
    lhs, rhs = np.vdot(ph, A), np.vdot(B, ps)
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)

    # gauge covariance: U'_mu(x) = G(x) U_mu(x) G(x+mu)^dag, psi' = G psi
    from oracle.oracle import random_su3
    rng = np.random.default_rng(5)
    G = random_su3(V, rng).reshape(V, 3, 3)
    R = O.Restatement()
    _, _, iup, _ = R.geometry(L)
    U = u.reshape(V, 4, 3, 3)
    Up = np.einsum("nab,nmbc,nmdc->nmad", G, U, G[iup].conj()).reshape(4 * V, 9)
    q = np.concatenate([ph, ps])
    qp = np.einsum("nab,nsb->nsa", G, q.reshape(V, 4, 3)).reshape(V, 12)
    gp = P.Gauge(lat, P.F64, 18)
    gp.load_host(np.ascontiguousarray(Up))
    fo = field_from_host(lat, qp, 1, P.F64)
    out = dev_bytes(bs)
    lat.dslash(gp, out, fo, 0, P.F64)
    got = field_to_host(lat, out, P.F64, 0)[: V // 2]
    want = np.einsum("nab,nsb->nsa", G[: V // 2], A.reshape(-1, 4, 3)).reshape(-1, 12)
    assert relmax(got, want) < 1e-13


def test_dropin_32x32x32x64_matches_oracle(dropin, restatement):
    """The benchmark size, element-wise against the oracle (FP64, 1e-14)."""
    L = (32, 32, 32, 64)
    lat, g64, u = _device_setup(L, 1234)
    V = lat.V
    bs = lat.spinor_bytes(P.F64)
    fe, fo = dev_bytes(bs), dev_bytes(bs)
    lat.spinor_gaussian(fe, P.F64, 0, 77)
    lat.spinor_gaussian(fo, P.F64, 1, 77)
    q = field_to_host(lat, fe, P.F64, 0)
    q[V // 2:] = field_to_host(lat, fo, P.F64, 1)[V // 2:]
    del lat, g64, fe, fo
    dropin(L)
    got = np.zeros_like(q)
    P.hopping_matrix("eo", q, got, u)
    P.hopping_matrix("oe", q, got, u)
    want = restatement.hop("full", L, q, u)
    assert relmax(got, want) < TOL64


@pytest.mark.parametrize("prec", [P.F64, P.F32, P.F16, P.BF16])
def test_spinor_norm2_batched(cuda, prec):
    import torch
    L = (8, 8, 4, 6)
    lat = new_lattice(L)
    V = lat.V
    rng = np.random.default_rng(17)
    nf = 5
    bs = lat.spinor_bytes(prec)
    block = dev_bytes(nf * bs)
    want = []
    for f in range(nf):
        q = O.gaussian_spinor(V, rng) * (f + 1)
        src = field_from_host(lat, q, 0, P.F64)
        lat.spinor_convert(block[f * bs:(f + 1) * bs], prec, src, P.F64)
        back = field_to_host(lat, block[f * bs:(f + 1) * bs], prec, 0)[: V // 2]
        want.append(float(np.sum(np.abs(back) ** 2)))
    out = torch.zeros(nf, dtype=torch.float64, device="cuda")
    lat.spinor_norm2(block, prec, nf, out)
    lat.synchronize()
    got = out.cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=1e-12)
    out2 = torch.zeros(nf, dtype=torch.float64, device="cuda")
    lat.spinor_norm2(block, prec, nf, out2)
    lat.synchronize()
    assert bool((out == out2).all())  # fixed summation order: reproducible


@pytest.mark.parametrize("prec,recon,tol", [(P.F64, 18, 1e-14), (P.F64, 12, 1e-13), (P.F32, 12, 1e-6),
                                            (P.F16, 12, 1e-3), (P.BF16, 12, 1e-2)])
@pytest.mark.parametrize("nrhs", [1, 3, 8])
def test_multi_rhs_equals_single_rhs(cuda, prec, recon, tol, nrhs):
    """Each field of a multi-RHS block gives what the single-RHS kernel gives
    (same arithmetic; tolerance covers compiler contraction differences)."""
    L = (8, 4, 6, 8)
    lat, g64, u = _device_setup(L, 13)
    g = P.Gauge(lat, prec, recon)
    g.copy_from(g64)
    bs = lat.spinor_bytes(prec)
    blk_in, blk_out, blk_x = dev_bytes(nrhs * bs), dev_bytes(nrhs * bs), dev_bytes(nrhs * bs)
    for r in range(nrhs):
        lat.spinor_gaussian(blk_in[r * bs:(r + 1) * bs], prec, 1, 100 + r)
        lat.spinor_gaussian(blk_x[r * bs:(r + 1) * bs], prec, 0, 200 + r)
    for xpay in (False, True):
        flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT if xpay else 0
        if xpay:
            lat.dslash_mrhs_xpay(g, blk_out, blk_in, nrhs, 0, prec, -0.0144, blk_x, 1.0, flags)
        else:
            lat.dslash_mrhs(g, blk_out, blk_in, nrhs, 0, prec)
        for r in range(nrhs):
            one = dev_bytes(bs)
            sl = slice(r * bs, (r + 1) * bs)
            if xpay:
                lat.dslash_xpay(g, one, blk_in[sl], 0, prec, -0.0144, blk_x[sl], 1.0, flags)
            else:
                lat.dslash(g, one, blk_in[sl], 0, prec)
            a = field_to_host(lat, blk_out[sl], prec, 0)[: lat.V // 2]
            b = field_to_host(lat, one, prec, 0)[: lat.V // 2]
            assert relmax(a, b) <= tol, (r, xpay, relmax(a, b))


@pytest.mark.parametrize("variant,block", [(1, 128), (2, 64), (4, 128), (100, 128), (102, 64), (103, 64),
                                           (1022, 64), (1042, 128)])
@pytest.mark.parametrize("prec,recon,tol", [(P.F64, 18, 1e-14), (P.F32, 12, 1e-6), (P.F16, 12, 1e-3)])
def test_multi_rhs_every_variant(cuda, monkeypatch, variant, block, prec, recon, tol):
    """Each launch variant of the multi-RHS kernel (RHS tile 1/2/4, RHS folded
    into the single-RHS kernels' grid, pipelined RHS tiles), forced past the
    tuner, agrees with the single-RHS kernel for every field of the block."""
    if prec == P.F64 and variant in (4, 1042):
        pytest.skip("no four-RHS FP64 tile (register file)")
    L = (8, 4, 6, 8)
    nrhs = 5
    lat, g64, u = _device_setup(L, 21)
    g = g64 if (prec, recon) == (P.F64, 18) else P.Gauge(lat, prec, recon)
    if g is not g64:
        g.copy_from(g64)
    bs = lat.spinor_bytes(prec)
    blk_in, blk_out, blk_x = dev_bytes(nrhs * bs), dev_bytes(nrhs * bs), dev_bytes(nrhs * bs)
    for r in range(nrhs):
        lat.spinor_gaussian(blk_in[r * bs:(r + 1) * bs], prec, 0, 300 + r)
        lat.spinor_gaussian(blk_x[r * bs:(r + 1) * bs], prec, 1, 400 + r)
    monkeypatch.setenv("PLQCD_MRHS_VARIANT", str(variant))
    monkeypatch.setenv("PLQCD_MRHS_BLOCK", str(block))
    flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT
    lat.dslash_mrhs_xpay(g, blk_out, blk_in, nrhs, 1, prec, 0.37, blk_x, -1.5, flags)
    monkeypatch.delenv("PLQCD_MRHS_VARIANT")
    for r in range(nrhs):
        sl = slice(r * bs, (r + 1) * bs)
        one = dev_bytes(bs)
        lat.dslash_xpay(g, one, blk_in[sl], 1, prec, 0.37, blk_x[sl], -1.5, flags)
        a = field_to_host(lat, blk_out[sl], prec, 1)[lat.V // 2:]
        b = field_to_host(lat, one, prec, 1)[lat.V // 2:]
        assert relmax(a, b) <= tol, (variant, r, relmax(a, b))


@pytest.mark.parametrize("variant", [2002, 2022, 2032, 2102, 2122])
@pytest.mark.parametrize("nrhs", [1, 2, 5, 8])
@pytest.mark.parametrize("prec,recon", [(P.F32, 18), (P.F32, 12), (P.F16, 12), (P.BF16, 12)])
@pytest.mark.parametrize("xpay", [False, True])
def test_multi_rhs_pair_kernel_is_bit_identical(cuda, monkeypatch, variant, nrhs, prec, recon, xpay):
    """The RHS-pair kernels (two RHS on the lanes of packed FP32
    instructions: 2002 direct loads, 2022 / 2032 cp.async pipeline of depth
    2 / 3, 2102 / 2122 with at most 128 registers), forced past the tuner, store the same bytes as the single-RHS
    kernel for every field of the block, an odd last RHS included."""
    L = (8, 4, 6, 8)
    lat, g64, u = _device_setup(L, 23)
    g = P.Gauge(lat, prec, recon)
    g.copy_from(g64)
    bs = lat.spinor_bytes(prec)
    blk_in, blk_out, blk_x = dev_bytes(nrhs * bs), dev_bytes(nrhs * bs), dev_bytes(nrhs * bs)
    for r in range(nrhs):
        lat.spinor_gaussian(blk_in[r * bs:(r + 1) * bs], prec, 1, 500 + r)
        lat.spinor_gaussian(blk_x[r * bs:(r + 1) * bs], prec, 0, 600 + r)
    monkeypatch.setenv("PLQCD_MRHS_VARIANT", str(variant))
    monkeypatch.setenv("PLQCD_MRHS_BLOCK", "64")
    flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT
    if xpay:
        lat.dslash_mrhs_xpay(g, blk_out, blk_in, nrhs, 0, prec, -0.29, blk_x, 1.25, flags)
    else:
        lat.dslash_mrhs(g, blk_out, blk_in, nrhs, 0, prec)
    monkeypatch.delenv("PLQCD_MRHS_VARIANT")
    for r in range(nrhs):
        sl = slice(r * bs, (r + 1) * bs)
        one = dev_bytes(bs)
        if xpay:
            lat.dslash_xpay(g, one, blk_in[sl], 0, prec, -0.29, blk_x[sl], 1.25, flags)
        else:
            lat.dslash(g, one, blk_in[sl], 0, prec)
        lat.synchronize()
        assert bool((blk_out[sl] == one).all()), (r, prec, recon, xpay)


@pytest.mark.parametrize("variant", [4208, 4204, 4308, 4304])
@pytest.mark.parametrize("nrhs", [4, 5, 11])
@pytest.mark.parametrize("recon", [18, 12])
@pytest.mark.parametrize("xpay", [False, True])
def test_multi_rhs_f64_link_sharing_kernel_is_bit_identical(cuda, monkeypatch, variant, nrhs, recon, xpay):
    """The FP64 link-sharing kernel (4000 + 100 * ring depth + RHS per block:
    a block's warps are RHS of the same 32 sites and read each link from
    shared memory), forced past the tuner, stores the same bytes as the
    single-RHS kernel for every field, with a partial last RHS group and a
    half volume (720) that is not a multiple of 32 sites."""
    L = (6, 4, 6, 10)
    lat, g64, u = _device_setup(L, 29)
    g = g64 if recon == 18 else P.Gauge(lat, P.F64, 12)
    if g is not g64:
        g.copy_from(g64)
    bs = lat.spinor_bytes(P.F64)
    blk_in, blk_out, blk_x = dev_bytes(nrhs * bs), dev_bytes(nrhs * bs), dev_bytes(nrhs * bs)
    for r in range(nrhs):
        lat.spinor_gaussian(blk_in[r * bs:(r + 1) * bs], P.F64, 0, 700 + r)
        lat.spinor_gaussian(blk_x[r * bs:(r + 1) * bs], P.F64, 1, 800 + r)
    monkeypatch.setenv("PLQCD_MRHS_VARIANT", str(variant))
    flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT
    if xpay:
        lat.dslash_mrhs_xpay(g, blk_out, blk_in, nrhs, 1, P.F64, -0.0144, blk_x, 1.0, flags)
    else:
        lat.dslash_mrhs(g, blk_out, blk_in, nrhs, 1, P.F64)
    monkeypatch.delenv("PLQCD_MRHS_VARIANT")
    for r in range(nrhs):
        sl = slice(r * bs, (r + 1) * bs)
        one = dev_bytes(bs)
        if xpay:
            lat.dslash_xpay(g, one, blk_in[sl], 1, P.F64, -0.0144, blk_x[sl], 1.0, flags)
        else:
            lat.dslash(g, one, blk_in[sl], 1, P.F64)
        lat.synchronize()
        assert bool((blk_out[sl] == one).all()), (variant, r)


@pytest.mark.parametrize("tiles,nrhs", [(1, 8), (1, 12), (2, 16), (2, 20), (4, 32), (1, 3)])
@pytest.mark.parametrize("prec,tol", [(P.F16, 2e-3), (P.BF16, 1.6e-2)])
@pytest.mark.parametrize("xpay", [False, True])
def test_multi_rhs_tensor_core_kernel(cuda, monkeypatch, tiles, nrhs, prec, tol, xpay):
    """The tensor-core multi-RHS kernel (mma.sync m16n8k8, 16-bit operands,
    FP32 accumulation; variant 3000 + RHS tiles of 8 per warp), forced past
    the tuner, agrees with the scalar single-RHS kernel for every field of
    the block within the 16-bit storage error (relative L2), including
    partial tiles, the xpay / gamma5 epilogue and both output parities."""
    L = (8, 4, 6, 8)
    lat, g64, u = _device_setup(L, 23)
    g = P.Gauge(lat, prec, 12)
    g.copy_from(g64)
    bs = lat.spinor_bytes(prec)
    for par in (0, 1):
        blk_in, blk_out, blk_x = dev_bytes(nrhs * bs), dev_bytes(nrhs * bs), dev_bytes(nrhs * bs)
        for r in range(nrhs):
            lat.spinor_gaussian(blk_in[r * bs:(r + 1) * bs], prec, 1 - par, 500 + r)
            lat.spinor_gaussian(blk_x[r * bs:(r + 1) * bs], prec, par, 600 + r)
        flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT if xpay else 0
        monkeypatch.setenv("PLQCD_MRHS_VARIANT", str(3000 + tiles))
        if xpay:
            lat.dslash_mrhs_xpay(g, blk_out, blk_in, nrhs, par, prec, 0.37, blk_x, -1.5, flags)
        else:
            lat.dslash_mrhs(g, blk_out, blk_in, nrhs, par, prec)
        monkeypatch.delenv("PLQCD_MRHS_VARIANT")
        half = slice(0, lat.V // 2) if par == 0 else slice(lat.V // 2, lat.V)
        for r in range(nrhs):
            sl = slice(r * bs, (r + 1) * bs)
            one = dev_bytes(bs)
            if xpay:
                lat.dslash_xpay(g, one, blk_in[sl], par, prec, 0.37, blk_x[sl], -1.5, flags)
            else:
                lat.dslash(g, one, blk_in[sl], par, prec)
            a = field_to_host(lat, blk_out[sl], prec, par)[half]
            b = field_to_host(lat, one, prec, par)[half]
            assert rel_l2(a, b) <= tol, (par, r, rel_l2(a, b))


@pytest.mark.parametrize("variant", ["sse3_intrin_nohalfspinor", "avx_nohalfspinor", "single_mic_split",
                                     "single_mic_split_nohalfspinor", "single_mic_split_nohalfspinor_short"])
def test_split_layout_entry_points(dropin, restatement, variant):
    """Split real/imaginary names (reference include/dirac.h:31-32, 39-40,
    55-62) compute the same operator as the AoS ones; the *_short names
    read link rows 0,1 only (exact for SU(3) links)."""
    L = (4, 6, 8, 10)
    dropin(L)
    V = O.volume(L)
    rng = np.random.default_rng(31)
    q, u = O.gaussian_spinor(V, rng), O.random_su3(4 * V, rng)
    want = restatement.hop("full", L, q, u)
    got = np.zeros_like(q)
    P.hopping_matrix_split("eo", q, got, u, variant)
    P.hopping_matrix_split("oe", q, got, u, variant)
    tol = 1e-13 if variant.endswith("short") else TOL64
    assert relmax(got, want) < tol
    if variant.endswith("short"):
        # row 2 really is rebuilt: garbage in row 2 of the input changes nothing
        u2 = u.copy()
        u2[:, 6:] = 123.0
        P.lib().plqcd_gauge_update(None)
        got2 = np.zeros_like(q)
        P.hopping_matrix_split("eo", q, got2, u2, variant)
        P.hopping_matrix_split("oe", q, got2, u2, variant)
        assert relmax(got2, want) < tol


def test_shipped_selftest(cuda):
    assert P.lib().plqcd_selftest(0, 1) == 0, P.last_error()


@pytest.mark.parametrize("variant,block", [(0, 64), (2, 64), (2, 128), (3, 64), (12, 64), (12, 128), (13, 64),
                                           (13, 128)])
@pytest.mark.parametrize("prec,recon,tol", [(P.F64, 18, 1e-14), (P.F32, 12, 1e-6), (P.F16, 12, 1e-3),
                                            (P.BF16, 12, 1e-2)])
def test_dslash_every_load_strategy(cuda, monkeypatch, variant, block, prec, recon, tol):
    """Each load strategy of the single-RHS kernel, forced past the tuner
    (direct, cp.async pipeline depth 2/3, two sites per thread, also on
    packed FP32 lanes), matches the
    FP64 oracle-checked kernel within the precision's tolerance, with the
    xpay and gamma5 epilogue and on a lattice whose half volume is not a
    multiple of the block."""
    if variant >= 12 and prec == P.F64:
        pytest.skip("two sites per thread is built for 32/16-bit formats")
    L = (6, 4, 6, 10)
    lat, g64, u = _device_setup(L, 41)
    g = g64 if (prec, recon) == (P.F64, 18) else P.Gauge(lat, prec, recon)
    if g is not g64:
        g.copy_from(g64)
    bs = lat.spinor_bytes(prec)
    a, x, o = dev_bytes(bs), dev_bytes(bs), dev_bytes(bs)
    lat.spinor_gaussian(a, prec, 0, 5)
    lat.spinor_gaussian(x, prec, 1, 6)
    flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT
    monkeypatch.setenv("PLQCD_DSLASH_STAGES", "0")
    monkeypatch.setenv("PLQCD_DSLASH_BLOCK", "128")
    ref = dev_bytes(bs)
    lat.dslash_xpay(g, ref, a, 1, prec, 0.25, x, -2.0, flags)
    monkeypatch.setenv("PLQCD_DSLASH_STAGES", str(variant))
    monkeypatch.setenv("PLQCD_DSLASH_BLOCK", str(block))
    lat.dslash_xpay(g, o, a, 1, prec, 0.25, x, -2.0, flags)
    want = field_to_host(lat, ref, prec, 1)[lat.V // 2:]
    got = field_to_host(lat, o, prec, 1)[lat.V // 2:]
    assert relmax(got, want) <= tol


@pytest.mark.parametrize("prec,recon", [(P.F32, 18), (P.F32, 12), (P.F16, 12), (P.BF16, 12)])
def test_packed_lanes_bit_identical(cuda, monkeypatch, prec, recon):
    """Packed FP32 lanes (FFMA2) round every lane as the scalar arithmetic
    does: the one-site cp.async kernel (variant 2, spin pairs of one site on
    the two lanes), two sites per thread with scalar arithmetic (variant 12)
    and on packed lanes (variant 13) give the same bits, for a plain hop and
    for the xpay / gamma5 epilogue, on a lattice whose half volume leaves a
    ragged last tile."""
    L = (6, 4, 6, 10)
    lat, g64, u = _device_setup(L, 49)
    g = P.Gauge(lat, prec, recon)
    g.copy_from(g64)
    bs = lat.spinor_bytes(prec)
    a, x = dev_bytes(bs), dev_bytes(bs)
    lat.spinor_gaussian(a, prec, 0, 15)
    lat.spinor_gaussian(x, prec, 1, 16)
    flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT
    outs = {}
    for v, blk in (("2", "64"), ("12", "64"), ("13", "64"), ("13", "128"), ("13", "32")):
        monkeypatch.setenv("PLQCD_DSLASH_STAGES", v)
        monkeypatch.setenv("PLQCD_DSLASH_BLOCK", blk)
        o1, o2 = dev_bytes(bs), dev_bytes(bs)
        lat.dslash(g, o1, a, 1, prec)
        lat.dslash_xpay(g, o2, a, 1, prec, 0.25, x, -2.0, flags)
        lat.synchronize()
        outs[v + "/" + blk] = (o1, o2)
    ref = outs["2/64"]
    for k, (o1, o2) in outs.items():
        assert bool((o1 == ref[0]).all()) and bool((o2 == ref[1]).all()), k


# TMA-staged kernels: variant 1000 * kind + 100 * ring depth + rows per tile;
# kind 1 stages every direction on its own, kinds 2-5 stage the own-line rows
# once per tile (2, 3: in 1 or 2 buffers of their own; 4, 5: the same with
# one tile-load box per ring stage)
TMA_CASES = [((16, 8, 4, 6), 1204), ((16, 8, 4, 6), 1308), ((16, 8, 6, 4), 1404), ((32, 8, 4, 4), 1602),
             ((8, 8, 4, 4), 1208), ((32, 16, 4, 2), 1216),
             ((16, 8, 4, 6), 2104), ((16, 8, 4, 6), 2208), ((16, 8, 6, 4), 3204), ((32, 8, 4, 4), 2302),
             ((8, 8, 4, 4), 3108), ((32, 16, 4, 2), 2116), ((16, 4, 4, 4), 2404),
             ((16, 8, 4, 6), 4204), ((16, 8, 4, 6), 4308), ((16, 8, 6, 4), 5204), ((32, 8, 4, 4), 4602),
             ((8, 8, 4, 4), 5308), ((16, 4, 4, 4), 4404)]


@pytest.mark.parametrize("L,variant", TMA_CASES)
@pytest.mark.parametrize("prec,recon", [(P.F64, 18), (P.F64, 12), (P.F32, 18), (P.F32, 12), (P.F16, 12),
                                        (P.BF16, 12)])
def test_tma_kernel_bit_identical(cuda, monkeypatch, L, variant, prec, recon):
    """The TMA-staged kernels (tile loads of whole rows into a shared-memory
    ring, one producer warp) compute exactly what the gather kernel
    computes: bit-identical outputs for the full lattice, for one parity with
    the xpay and gamma5 epilogue, and no stage wait runs out."""
    lat, g64, u = _device_setup(L, 43)
    g = g64 if (prec, recon) == (P.F64, 18) else P.Gauge(lat, prec, recon)
    if g is not g64:
        g.copy_from(g64)
    bs = lat.spinor_bytes(prec)
    fe, fo, x = dev_bytes(bs), dev_bytes(bs), dev_bytes(bs)
    lat.spinor_gaussian(fe, prec, 0, 7)
    lat.spinor_gaussian(fo, prec, 1, 8)
    lat.spinor_gaussian(x, prec, 1, 9)
    flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT
    outs = {}
    for v in ("2", str(variant)):
        monkeypatch.setenv("PLQCD_DSLASH_STAGES", v)
        monkeypatch.setenv("PLQCD_DSLASH_BLOCK", "64")
        oe, oo, ox = dev_bytes(bs), dev_bytes(bs), dev_bytes(bs)
        lat.dslash_full(g, oe, oo, fe, fo, prec)
        lat.dslash_xpay(g, ox, fe, 1, prec, 0.25, x, -2.0, flags)
        lat.synchronize()  # raises if a stage wait ran out
        outs[v] = (oe, oo, ox)
    for a, b in zip(outs["2"], outs[str(variant)]):
        assert bool((a == b).all())


def test_tma_kernel_matches_oracle(cuda, restatement):
    """Full-lattice TMA kernel against the C restatement of the reference."""
    L = (16, 8, 6, 4)
    lat, g64, u = _device_setup(L, 44)
    V = lat.V
    q = O.gaussian_spinor(V, np.random.default_rng(5))
    want = restatement.hop("full", L, q, u)
    fe, fo = field_from_host(lat, q, 0, P.F64), field_from_host(lat, q, 1, P.F64)
    bs = lat.spinor_bytes(P.F64)
    oe, oo = dev_bytes(bs), dev_bytes(bs)
    os.environ["PLQCD_DSLASH_STAGES"] = "1408"
    try:
        lat.dslash_full(g64, oe, oo, fe, fo, P.F64)
        lat.synchronize()
    finally:
        os.environ.pop("PLQCD_DSLASH_STAGES", None)
    got = field_to_host(lat, oe, P.F64, 0)
    got[V // 2:] = field_to_host(lat, oo, P.F64, 1)[V // 2:]
    assert relmax(got, want) < TOL64


def test_tma_kernel_rejects_misfit_tiles(cuda, monkeypatch):
    """A tile that does not divide the lattice (rows per tile not dividing L1,
    or not a whole number of warps), an unknown kernel kind or a ring too
    short for its kernel is refused on the host with an argument error;
    nothing is launched."""
    lat, g64, u = _device_setup((6, 4, 6, 10), 45)
    bs = lat.spinor_bytes(P.F64)
    a, o = dev_bytes(bs), dev_bytes(bs)
    for v in ("1408", "1203", "2203", "3008", "4104", "6204"):
        monkeypatch.setenv("PLQCD_DSLASH_STAGES", v)
        with pytest.raises(P.PlqcdError):
            lat.dslash(g64, o, a, 0, P.F64)


def test_tma_kernel_bit_identical_at_benchmark_size(cuda, monkeypatch):
    """At the benchmark lattice (32^3x64) the TMA configurations the tuner
    picks among there (blocked tile order) give the same bits as the
    cp.async kernel for the full lattice and for one parity."""
    L = (32, 32, 32, 64)
    lat = new_lattice(L)
    g64 = P.Gauge(lat, P.F64, 18)
    g64.random(46)
    bs = lat.spinor_bytes(P.F64)
    fe, fo = dev_bytes(bs), dev_bytes(bs)
    lat.spinor_gaussian(fe, P.F64, 0, 11)
    lat.spinor_gaussian(fo, P.F64, 1, 12)
    outs = {}
    variants = ("1204", "2204", "4304", "2216")
    for v in ("2",) + variants:
        monkeypatch.setenv("PLQCD_DSLASH_STAGES", v)
        monkeypatch.setenv("PLQCD_DSLASH_BLOCK", "64")
        for rep in range(2 if v != "2" else 1):  # repeats: the same bits every launch
            oe, oo, o1 = dev_bytes(bs), dev_bytes(bs), dev_bytes(bs)
            lat.dslash_full(g64, oe, oo, fe, fo, P.F64)
            lat.dslash(g64, o1, fe, P.ODD, P.F64)
            lat.synchronize()
            outs[(v, rep)] = (oe, oo, o1)
    for v in variants:
        for rep in range(2):
            for a, b in zip(outs[("2", 0)], outs[(v, rep)]):
                assert bool((a == b).all()), (v, rep)


@pytest.mark.parametrize("variant", ["intrin_256", "intrin_512", "single_mic", "single_mic_short"])
def test_lane_packed_entry_points(dropin, restatement, variant):
    """The lane-packed names (spinor_256/512, su3_256/512 arrays) compute the
    reference's operator on the packed layout; eo writes only the even
    objects of qout, oe only the odd ones; a changed link array is picked
    up through plqcd_gauge_update."""
    L = (8, 4, 6, 4)
    dropin(L)
    V = O.volume(L)
    rng = np.random.default_rng(29)
    q, u = O.gaussian_spinor(V, rng), O.random_su3(4 * V, rng)
    want = restatement.hop("full", L, q, u)
    got = np.full_like(q, np.nan)
    P.hopping_matrix_packed("eo", q, got, u, variant)
    assert np.isnan(got[V // 2:]).all() and not np.isnan(got[: V // 2]).any()
    P.hopping_matrix_packed("oe", q, got, u, variant)
    tol = 1e-13 if variant.endswith("short") else TOL64
    assert relmax(got, want) < tol
    u2 = O.random_su3(4 * V, rng)
    P.lib().plqcd_gauge_update(None)
    P.hopping_matrix_packed("eo", q, got, u2, variant)
    P.hopping_matrix_packed("oe", q, got, u2, variant)
    assert relmax(got, restatement.hop("full", L, q, u2)) < tol


def test_misaligned_fields_are_refused(cuda):
    """Field pointers that are not 16-byte aligned are refused with an
    argument error before any launch (the kernels use 16-byte vector and
    tile loads); nothing runs on the device with them."""
    L = (4, 4, 4, 4)
    lat, g64, u = _device_setup(L, 47)
    bs = lat.spinor_bytes(P.F64)
    buf = dev_bytes(bs + 64)
    ok = buf.data_ptr()
    bad = ok + 8
    for call in (lambda: lat.dslash(g64, bad, ok + 16, 0, P.F64),
                 lambda: lat.dslash(g64, ok, bad, 0, P.F64),
                 lambda: lat.dslash_xpay(g64, ok, ok + 16, 0, P.F64, 1.0, bad, 1.0),
                 lambda: lat.dslash_full(g64, ok, ok + 16, bad, ok + 32, P.F64),
                 lambda: lat.spinor_gaussian(bad, P.F64, 0, 1),
                 lambda: lat.spinor_convert(bad, P.F32, ok, P.F64)):
        with pytest.raises(P.PlqcdError, match="aligned"):
            call()
    lat.synchronize()


@pytest.mark.parametrize("variant", ["1204", "1308", "2204", "3104", "4304"])
def test_tma_kernel_on_whole_slice_ranges(cuda, monkeypatch, variant):
    """On a site range of whole t-slices (a slab interior, a pipeline chunk)
    the TMA kernel writes the same bits as the gather kernel on that range
    and leaves the other sites of the output untouched."""
    L = (16, 8, 4, 6)
    lat, g64, u = _device_setup(L, 48)
    S = (L[0] // 2) * L[1] * L[2]
    bs = lat.spinor_bytes(P.F64)
    fin, x = dev_bytes(bs), dev_bytes(bs)
    lat.spinor_gaussian(fin, P.F64, 1, 3)
    lat.spinor_gaussian(x, P.F64, 0, 4)
    outs = {}
    for v in ("2", variant):
        monkeypatch.setenv("PLQCD_DSLASH_STAGES", v)
        monkeypatch.setenv("PLQCD_DSLASH_BLOCK", "64")
        o = dev_bytes(bs)
        o.fill_(7)
        lat.dslash_sites(g64, o, fin, 0, P.F64, S, 4 * S, P.DSLASH_G5_IN, 0.5, x, -1.0)
        lat.synchronize()
        outs[v] = o
    assert bool((outs["2"] == outs[variant]).all())
    import torch
    plane = outs[variant].view(12, -1)      # 12 planes of Vh * 16 bytes
    assert bool((plane[:, :S * 16] == 7).all()) and bool((plane[:, 5 * S * 16:] == 7).all())
    assert not bool((plane[:, S * 16:5 * S * 16] == 7).all())
    del torch


@pytest.mark.parametrize("variant", ["1204", "2204", "4304"])
def test_tma_wait_that_runs_out_reports_timeout(cuda, monkeypatch, variant):
    """Failure detection of the bounded stage waits: with the test hook on,
    each consumer warp of the TMA kernels waits (limit 200 us) on a barrier
    that nothing completes. The wait runs out, the kernel returns after its
    tile loads in flight have landed, plqcd_lattice_synchronize reports
    PLQCD_ERR_TIMEOUT and clears the flag, and the next normal launch gives
    the gather kernel's bits again."""
    L = (16, 8, 6, 4)
    lat, g64, u = _device_setup(L, 48)
    bs = lat.spinor_bytes(P.F64)
    fe, fo = dev_bytes(bs), dev_bytes(bs)
    lat.spinor_gaussian(fe, P.F64, 0, 13)
    lat.spinor_gaussian(fo, P.F64, 1, 14)
    monkeypatch.setenv("PLQCD_DSLASH_BLOCK", "64")
    monkeypatch.setenv("PLQCD_DSLASH_STAGES", "2")
    re_, ro_ = dev_bytes(bs), dev_bytes(bs)
    lat.dslash_full(g64, re_, ro_, fe, fo, P.F64)
    lat.synchronize()
    monkeypatch.setenv("PLQCD_DSLASH_STAGES", variant)
    lib = P.lib()
    oe, oo = dev_bytes(bs), dev_bytes(bs)
    P.check(lib.plqcd_tma_timeout_test(1, 200_000))
    try:
        P.check(lib.plqcd_dslash_full(lat.handle, g64.handle, oe.data_ptr(), oo.data_ptr(), fe.data_ptr(),
                                      fo.data_ptr(), P.F64))
        rc = lib.plqcd_lattice_synchronize(lat.handle)
        msg = P.last_error()
    finally:
        P.check(lib.plqcd_tma_timeout_test(0, 0))
    assert rc == P.ERR_TIMEOUT, (rc, msg)
    assert "TMA stage wait ran out" in msg
    assert lib.plqcd_lattice_synchronize(lat.handle) == 0   # flag cleared, context usable
    lat.dslash_full(g64, oe, oo, fe, fo, P.F64)
    lat.synchronize()
    assert bool((oe == re_).all()) and bool((oo == ro_).all())


def _mrhs_tma_case(L, nrhs, seed, par):
    lat, g64, u = _device_setup(L, seed)
    bs = lat.spinor_bytes(P.F64)
    blk_in, blk_out, blk_x = dev_bytes(nrhs * bs), dev_bytes(nrhs * bs), dev_bytes(nrhs * bs)
    for r in range(nrhs):
        lat.spinor_gaussian(blk_in[r * bs:(r + 1) * bs], P.F64, par ^ 1, 900 + r)
        lat.spinor_gaussian(blk_x[r * bs:(r + 1) * bs], P.F64, par, 950 + r)
    return lat, g64, bs, blk_in, blk_out, blk_x


# variant = 100000 * RHS per tile + 1000 * kind + 100 * ring depth + rows per tile
@pytest.mark.parametrize("L,nrhs,variant", [
    ((8, 4, 6, 8), 8, 402102), ((8, 4, 6, 8), 8, 402202), ((8, 4, 6, 8), 8, 404202), ((8, 4, 6, 8), 8, 404302),
    ((8, 4, 6, 8), 8, 802101), ((8, 4, 6, 8), 8, 804201), ((8, 4, 6, 8), 8, 202104), ((8, 4, 6, 8), 12, 402202),
    ((16, 4, 4, 6), 8, 202202), ((16, 4, 4, 6), 6, 204202), ((12, 8, 4, 4), 16, 802204)])
@pytest.mark.parametrize("recon", [18, 12])
@pytest.mark.parametrize("xpay", [False, True])
def test_multi_rhs_tma_rhs_tile_kernel_is_bit_identical(cuda, monkeypatch, L, nrhs, variant, recon, xpay):
    """The TMA-staged FP64 multi-RHS hop with RHS tiles (several RHS of the
    block per tile, each tile's links staged once for all of them; own-line
    kinds 2 and 4), forced past the tuner, stores the same bytes as the
    single-RHS kernel for every field of the block: several RHS groups,
    tiles of 1, 2 and 4 rows, a tile that covers all of y (the rows on either
    side wrap onto it), both link formats."""
    par = 1 if xpay else 0
    lat, g64, bs, blk_in, blk_out, blk_x = _mrhs_tma_case(L, nrhs, 61 + recon, par)
    g = g64 if recon == 18 else P.Gauge(lat, P.F64, 12)
    if g is not g64:
        g.copy_from(g64)
    monkeypatch.setenv("PLQCD_MRHS_VARIANT", str(variant))
    flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT
    if xpay:
        lat.dslash_mrhs_xpay(g, blk_out, blk_in, nrhs, par, P.F64, -0.0144, blk_x, 1.0, flags)
    else:
        lat.dslash_mrhs(g, blk_out, blk_in, nrhs, par, P.F64)
    lat.synchronize()
    monkeypatch.delenv("PLQCD_MRHS_VARIANT")
    for r in range(nrhs):
        sl = slice(r * bs, (r + 1) * bs)
        one = dev_bytes(bs)
        if xpay:
            lat.dslash_xpay(g, one, blk_in[sl], par, P.F64, -0.0144, blk_x[sl], 1.0, flags)
        else:
            lat.dslash(g, one, blk_in[sl], par, P.F64)
        lat.synchronize()
        assert bool((blk_out[sl] == one).all()), (variant, r)


def test_multi_rhs_tma_xpay_repeats_bit_identical_at_scale(cuda, monkeypatch):
    """Persistent CTAs with many tiles each (16^3x32, 32 RHS, tiles of 4 RHS x
    2 rows, 4 CTAs per SM): every repeat of the xpay hop gives the bytes of
    the cp.async multi-RHS kernel. The producer must fence the async proxy
    after a buffer's release and before its refill (the consumers read it
    through the generic proxy); without that fence every repeat of this case
    had tiles refilled under their readers."""
    L, nrhs = (16, 16, 16, 32), 32
    lat, g64, bs, blk_in, blk_out, blk_x = _mrhs_tma_case(L, nrhs, 81, 0)
    flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT
    ref = dev_bytes(nrhs * bs)
    monkeypatch.setenv("PLQCD_MRHS_VARIANT", "102")
    monkeypatch.setenv("PLQCD_MRHS_BLOCK", "64")
    lat.dslash_mrhs_xpay(g64, ref, blk_in, nrhs, 0, P.F64, -0.0144, blk_x, 1.0, flags)
    monkeypatch.setenv("PLQCD_MRHS_VARIANT", "402202")
    for rep in range(3):
        blk_out.zero_()
        lat.dslash_mrhs_xpay(g64, blk_out, blk_in, nrhs, 0, P.F64, -0.0144, blk_x, 1.0, flags)
        lat.synchronize()
        assert bool((blk_out == ref).all()), rep


def test_multi_rhs_tma_rhs_tile_rejects_tiles_that_do_not_fit(cuda, monkeypatch):
    """RHS tiles that do not divide the block, or whose tile exceeds 256
    consumer threads, are refused with a message; nothing is launched."""
    lat, g64, bs, blk_in, blk_out, blk_x = _mrhs_tma_case((8, 4, 6, 8), 6, 3, 0)
    for variant, msg in ((402202, "does not divide"), (202203, "does not fit")):
        monkeypatch.setenv("PLQCD_MRHS_VARIANT", str(variant))
        rc = P.lib().plqcd_dslash_mrhs(lat.handle, g64.handle, blk_out.data_ptr(), blk_in.data_ptr(), 6, 0, P.F64, 0)
        assert rc == -1 and msg in P.last_error(), (variant, P.last_error())
    monkeypatch.delenv("PLQCD_MRHS_VARIANT")


def test_multi_rhs_tma_wait_that_runs_out_reports_timeout(cuda, monkeypatch):
    """The bounded stage waits of the RHS-tile kernel: with the test hook on,
    the consumer waits run out, synchronize reports PLQCD_ERR_TIMEOUT, and
    the next launch gives the single-RHS kernel's bytes again."""
    nrhs = 8
    lat, g64, bs, blk_in, blk_out, blk_x = _mrhs_tma_case((16, 8, 6, 4), nrhs, 71, 0)
    ref = dev_bytes(nrhs * bs)
    for r in range(nrhs):
        sl = slice(r * bs, (r + 1) * bs)
        lat.dslash(g64, ref[sl], blk_in[sl], 0, P.F64)
    lat.synchronize()
    monkeypatch.setenv("PLQCD_MRHS_VARIANT", "402202")
    lib = P.lib()
    P.check(lib.plqcd_tma_timeout_test(1, 200_000))
    try:
        P.check(lib.plqcd_dslash_mrhs(lat.handle, g64.handle, blk_out.data_ptr(), blk_in.data_ptr(), nrhs, 0,
                                      P.F64, 0))
        rc = lib.plqcd_lattice_synchronize(lat.handle)
        msg = P.last_error()
    finally:
        P.check(lib.plqcd_tma_timeout_test(0, 0))
    assert rc == P.ERR_TIMEOUT, (rc, msg)
    assert lib.plqcd_lattice_synchronize(lat.handle) == 0
    lat.dslash_mrhs(g64, blk_out, blk_in, nrhs, 0, P.F64)
    lat.synchronize()
    monkeypatch.delenv("PLQCD_MRHS_VARIANT")
    assert bool((blk_out == ref).all())


def test_tma_timeout_test_hook_rejects_bad_limits(cuda):
    lib = P.lib()
    for ns in (0, 999, 3_000_000_000):
        assert lib.plqcd_tma_timeout_test(1, ns) == -1
        assert "outside 1 us .. 2 s" in P.last_error()
    assert lib.plqcd_tma_timeout_test(0, 0) == 0
