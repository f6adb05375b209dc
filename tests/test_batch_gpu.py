"""Batched multi-RHS, multi-lattice CG (plqcd_invert_cg_batch), eager and as
one CUDA-graph launch: every RHS must reach the FP64 residual and agree with
the single-RHS solver; residuals are re-checked on the host with the
oracle's full-lattice operator."""
import numpy as np
import pytest

import plqcd_b200 as P
from oracle import oracle as O
from tests.gpu_util import dev_bytes, field_to_host, new_lattice

pytestmark = pytest.mark.gpu
KAPPA = 0.12


def _lattice_item(L, nrhs, seed, sloppy):
    lat = new_lattice(L)
    g64 = P.Gauge(lat, P.F64, 18)
    g64.random(seed)
    gs = None
    if sloppy != P.F64:
        gs = P.Gauge(lat, sloppy, 12)
        gs.copy_from(g64)
    bs = lat.spinor_bytes(P.F64)
    be, bo, xe, xo = (dev_bytes(nrhs * bs) for _ in range(4))
    for r in range(nrhs):
        lat.spinor_gaussian(be[r * bs:(r + 1) * bs], P.F64, 0, seed * 100 + r)
        lat.spinor_gaussian(bo[r * bs:(r + 1) * bs], P.F64, 1, seed * 100 + r)
    return dict(lat=lat, g64=g64, g_sloppy=gs, nrhs=nrhs, x_even=xe, x_odd=xo, b_even=be, b_odd=bo)


def _host_field(item, blk_e, blk_o, r):
    lat = item["lat"]
    bs = lat.spinor_bytes(P.F64)
    sl = slice(r * bs, (r + 1) * bs)
    f = field_to_host(lat, blk_e[sl], P.F64, 0)
    f[lat.V // 2:] = field_to_host(lat, blk_o[sl], P.F64, 1)[lat.V // 2:]
    return f


@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("sloppy", [P.F16, P.F32, P.F64])
def test_batch_solves_every_rhs(cuda, restatement, use_graph, sloppy):
    items = [_lattice_item((8, 8, 8, 16), 3, 3, sloppy), _lattice_item((4, 6, 4, 8), 2, 5, sloppy)]
    info, res = P.invert_cg_batch(items, P.cg_param(kappa=KAPPA, tol=1e-10, sloppy_prec=sloppy), use_graph)
    assert info.converged and info.max_schur_residual <= 1e-10
    assert info.graph_launches == (1 if use_graph else 0)
    assert max(res) < 1e-9 and len(res) == 5
    if sloppy != P.F64:
        assert info.reliable_updates >= 1
    for it in items:
        lat = it["lat"]
        u = it["g64"].store_host()
        bs = lat.spinor_bytes(P.F64)
        for r in range(it["nrhs"]):
            x = _host_field(it, it["x_even"], it["x_odd"], r)
            b = _host_field(it, it["b_even"], it["b_odd"], r)
            rr = np.linalg.norm(b - restatement.wilson(lat.dims, u, x, KAPPA)) / np.linalg.norm(b)
            assert rr < 1e-9
            # the single-RHS solver gives the same solution
            xe1, xo1 = dev_bytes(bs), dev_bytes(bs)
            sl = slice(r * bs, (r + 1) * bs)
            P.invert_cg(lat, it["g64"], None, xe1, xo1, it["b_even"][sl], it["b_odd"][sl],
                        P.cg_param(kappa=KAPPA, tol=1e-10))
            x1 = field_to_host(lat, xe1, P.F64, 0)
            x1[lat.V // 2:] = field_to_host(lat, xo1, P.F64, 1)[lat.V // 2:]
            assert np.linalg.norm(x - x1) / np.linalg.norm(x1) < 1e-8


def test_batch_reports_non_convergence(cuda):
    items = [_lattice_item((4, 4, 4, 8), 2, 7, P.F32)]
    info, res = P.invert_cg_batch(items, P.cg_param(kappa=KAPPA, tol=1e-10, sloppy_prec=P.F32, max_iter=2),
                                  True, raise_on_error=False)
    assert not info.converged and info.iterations == 2
    assert "not converged" in P.last_error()


def test_batch_rejects_mismatched_sloppy_gauge(cuda):
    it = _lattice_item((4, 4, 4, 8), 1, 9, P.F16)
    info, _ = P.invert_cg_batch([it], P.cg_param(kappa=KAPPA, sloppy_prec=P.F32), True, raise_on_error=False)
    assert "sloppy gauge does not match" in P.last_error()


@pytest.mark.parametrize("variant", [2102, 2022])
def test_batch_fused_sums_match_separate_passes(cuda, monkeypatch, tmp_path, variant):
    """With RHS-pair kernels as the sloppy hops, the batched solver moves
    |t|^2 and r -= alpha Ap, |r|^2 into the hops' epilogues, and the restart
    of a reliable update (|r|^2 fused, retired RHS pairs skipped). The solves
    (5 RHS: a partial RHS pair; Vh = 96: a partial site block) agree with the
    separate passes (PLQCD_MCG_FUSED=0) and reach the FP64 residual."""
    import json
    prm = P.cg_param(kappa=KAPPA, tol=1e-10, sloppy_prec=P.F16)
    items = [_lattice_item((8, 8, 8, 16), 5, 11, P.F16), _lattice_item((4, 6, 4, 8), 2, 13, P.F16)]
    P.invert_cg_batch(items, P.cg_param(kappa=KAPPA, tol=1e-10, sloppy_prec=P.F16, max_iter=2), True,
                      raise_on_error=False)  # tunes every configuration
    path = str(tmp_path / "tune.json")
    assert P.lib().plqcd_tune_save(path.encode()) == 0
    lines = []
    for line in open(path):
        e = json.loads(line)
        if f"dslash_mrhs|p{P.F16}|r12|" in e["key"]:  # plain and xpay hops
            e["variant"], e["block"] = variant, 64
        lines.append(json.dumps(e))
    open(path, "w").write("\n".join(lines) + "\n")
    P.lib().plqcd_tune_clear()
    assert P.lib().plqcd_tune_load(path.encode()) == 0
    try:
        sols = {}
        for fused in ("1", "0"):
            monkeypatch.setenv("PLQCD_MCG_FUSED", fused)
            info, res = P.invert_cg_batch(items, prm, True)
            assert info.converged and info.max_schur_residual <= 1e-10 and max(res) < 1e-9
            sols[fused] = (info.iterations, [_host_field(it, it["x_even"], it["x_odd"], r)
                                             for it in items for r in range(it["nrhs"])])
        assert abs(sols["1"][0] - sols["0"][0]) <= 1
        for a, b in zip(sols["1"][1], sols["0"][1]):
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-8
    finally:
        P.lib().plqcd_tune_clear()
