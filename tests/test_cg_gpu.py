"""Even/odd preconditioned Wilson CG on the GPU: FP64 and mixed precision.

The oracle is the FP64 CPU CG on the restated operator (oracle/hop_oracle.c);
every solution is also checked independently on the host, in FP64, against
the full-lattice operator D = 1 - kappa H of the oracle."""
import numpy as np
import pytest

import plqcd_b200 as P
from oracle import oracle as O
from tests.gpu_util import dev_bytes, field_from_host, field_to_host, new_lattice

pytestmark = pytest.mark.gpu
KAPPA = 0.12


def _setup(L, seed=3):
    lat = new_lattice(L)
    g64 = P.Gauge(lat, P.F64, 18)
    g64.random(seed)
    u = g64.store_host()
    b = O.gaussian_spinor(lat.V, np.random.default_rng(seed + 1))
    return lat, g64, u, b


def _solve(lat, g64, gs, b, **kw):
    bs = lat.spinor_bytes(P.F64)
    be, bo = field_from_host(lat, b, 0, P.F64), field_from_host(lat, b, 1, P.F64)
    xe, xo = dev_bytes(bs), dev_bytes(bs)
    info = P.invert_cg(lat, g64, gs, xe, xo, be, bo, P.cg_param(kappa=KAPPA, **kw))
    x = field_to_host(lat, xe, P.F64, 0)
    x[lat.V // 2:] = field_to_host(lat, xo, P.F64, 1)[lat.V // 2:]
    return x, info


def _host_residual(restatement, L, u, x, b):
    r = b - restatement.wilson(L, u, x, KAPPA)
    return float(np.linalg.norm(r) / np.linalg.norm(b))


def test_cg_f64_matches_oracle_cg(cuda, restatement):
    L = (8, 8, 8, 16)
    lat, g64, u, b = _setup(L)
    x, info = _solve(lat, g64, None, b, tol=1e-10)
    assert info.converged and info.schur_residual <= 1e-10
    assert info.true_residual < 1e-9
    assert _host_residual(restatement, L, u, x, b) < 1e-9
    xo, it, rel = restatement.cg_solve(L, u, b, KAPPA, tol=1e-10)
    assert rel < 1e-9
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8
    # same Krylov recursion in the same precision: same iteration count (+-1)
    assert abs(info.iterations - it) <= 1


@pytest.mark.parametrize("prec,recon", [(P.F32, 18), (P.F32, 12), (P.F16, 12), (P.BF16, 12)])
def test_cg_mixed_precision_reaches_f64_residual(cuda, restatement, prec, recon):
    L = (8, 8, 8, 16)
    lat, g64, u, b = _setup(L, 5)
    gs = P.Gauge(lat, prec, recon)
    gs.copy_from(g64)
    x, info = _solve(lat, g64, gs, b, tol=1e-10, sloppy_prec=prec)
    assert info.converged and info.schur_residual <= 1e-10
    assert info.reliable_updates >= 1
    assert _host_residual(restatement, L, u, x, b) < 1e-9
    x64, _ = _solve(lat, g64, None, b, tol=1e-10)
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-8


def test_cg_zero_source(cuda):
    L = (4, 4, 4, 8)
    lat, g64, u, b = _setup(L)
    x, info = _solve(lat, g64, None, np.zeros_like(b))
    assert info.converged and np.all(x == 0)


def test_cg_reports_non_convergence(cuda):
    L = (4, 4, 4, 8)
    lat, g64, u, b = _setup(L)
    bs = lat.spinor_bytes(P.F64)
    be, bo = field_from_host(lat, b, 0, P.F64), field_from_host(lat, b, 1, P.F64)
    xe, xo = dev_bytes(bs), dev_bytes(bs)
    info = P.invert_cg(lat, g64, None, xe, xo, be, bo, P.cg_param(kappa=KAPPA, max_iter=3), raise_on_error=False)
    assert not info.converged and info.iterations == 3
    assert "not converged" in P.last_error()


def test_cg_larger_lattice_mixed_f16(cuda, restatement):
    L = (16, 16, 16, 32)
    lat, g64, u, b = _setup(L, 9)
    gs = P.Gauge(lat, P.F16, 12)
    gs.copy_from(g64)
    x, info = _solve(lat, g64, gs, b, tol=1e-10, sloppy_prec=P.F16)
    assert info.converged and info.true_residual < 1e-9
    assert _host_residual(restatement, L, u, x, b) < 1e-9


def test_tuner_persists_choices(cuda, tmp_path):
    import ctypes
    L = (8, 8, 4, 4)
    lat = new_lattice(L)
    g = P.Gauge(lat, P.F32, 12)
    g.random(1)
    bs = lat.spinor_bytes(P.F32)
    a, b = dev_bytes(bs), dev_bytes(bs)
    lat.spinor_gaussian(a, P.F32, 1, 1)
    lat.dslash(g, b, a, 0, P.F32)
    first = b.clone()
    lat.dslash(g, b, a, 0, P.F32)
    lat.synchronize()
    assert bool((first == b).all())
    n = P.lib().plqcd_tune_count()
    assert n >= 1
    path = str(tmp_path / "tune.json").encode()
    assert P.lib().plqcd_tune_save(path) == 0
    text = open(path.decode()).read()
    assert "dslash|p1|r12|half|8x8x4x4" in text
    key = [l for l in text.splitlines() if "dslash|p1|r12|half|8x8x4x4" in l][0].split('"')[3]
    v, blk, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    assert P.lib().plqcd_tune_get(key.encode(), ctypes.byref(v), ctypes.byref(blk), ctypes.byref(ms)) == 0
    assert v.value in (0, 2, 3) and blk.value in (64, 128, 256) and ms.value > 0
