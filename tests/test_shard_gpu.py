"""t-slab decomposition on the GPU (plqcd_b200/shard.py): N slabs held in
one process on one device (LocalTransport copies the ghost slices), so the
kernels, the ghost slices and the site ranges of the multi-GPU hop run here;
the transport between processes is covered by tests/test_shard_cpu.py.

The sharded hop runs the single-device kernels on the same data, so its
output is bit-identical to the unsharded hop; the sharded CG matches
plqcd_invert_cg."""
import numpy as np
import pytest

import plqcd_b200 as P
from plqcd_b200 import shard as SH
from oracle import oracle as O
from tests.gpu_util import dev_bytes, field_from_host, field_to_host, new_lattice, relmax

pytestmark = pytest.mark.gpu
_STREAMS = []  # side streams of the per-slab-stream tests (kept alive)


def _global(L, seed):
    lat = new_lattice(L)
    g64 = P.Gauge(lat, P.F64, 18)
    g64.random(seed)
    u = g64.store_host()
    q = O.gaussian_spinor(lat.V, np.random.default_rng(seed))
    return lat, g64, u, q


def _shards(L, N, u, prec, recon, own_streams=False):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    side = [torch.cuda.Stream() for _ in range(N - 1)] if own_streams else []
    _STREAMS.extend(side)
    shards = [SH.ShardedLattice(L, r, N, 0, stream if (r == 0 or not own_streams) else side[r - 1].cuda_stream)
              for r in range(N)]
    gauges = [s.gauge_from_global(u, prec, recon) for s in shards]
    SH.exchange_gauge(shards, gauges, SH.LocalTransport(N))
    return shards, gauges


def _gather(shards, fields, parity, prec, V):
    out = np.full((V, 12), np.nan + 0j)
    for s, f in zip(shards, fields):
        idx, vals = s.export_interior(f, parity, prec)
        out[idx] = vals
    return out


@pytest.mark.parametrize("N,own_streams", [(1, False), (2, False), (4, False), (4, True)])
@pytest.mark.parametrize("prec,recon", [(P.F64, 18), (P.F32, 12), (P.F16, 12)])
def test_sharded_hop_is_bit_identical(cuda, N, own_streams, prec, recon):
    L = (8, 8, 4, 16)
    lat, g64, u, q = _global(L, 31)
    g = g64 if (prec, recon) == (P.F64, 18) else P.Gauge(lat, prec, recon)
    if g is not g64:
        g.copy_from(g64)
    shards, gauges = _shards(L, N, u, prec, recon, own_streams)
    T = SH.LocalTransport(N)
    flags = P.DSLASH_G5_IN | P.DSLASH_G5_OUT
    for p in (P.EVEN, P.ODD):
        # single device: out = 0.25 g5 H g5-in + (-2) x
        fin = field_from_host(lat, q, 1 - p, prec)
        fx = field_from_host(lat, np.conj(q), p, prec)
        fo = dev_bytes(lat.spinor_bytes(prec))
        lat.dslash(g, fo, fin, p, prec)
        fox = dev_bytes(lat.spinor_bytes(prec))
        lat.dslash_xpay(g, fox, fin, p, prec, 0.25, fx, -2.0, flags)
        want = field_to_host(lat, fo, prec, p)[p * lat.Vh:(p + 1) * lat.Vh]
        wantx = field_to_host(lat, fox, prec, p)[p * lat.Vh:(p + 1) * lat.Vh]
        ins = [s.import_global(q, 1 - p, prec) for s in shards]
        xs = [s.import_global(np.conj(q), p, prec) for s in shards]
        outs = [s.field(prec) for s in shards]
        outx = [s.field(prec) for s in shards]
        SH.dslash(shards, gauges, outs, ins, p, prec, T)
        SH.dslash(shards, gauges, outx, ins, p, prec, T, flags, 0.25, xs, -2.0)
        got = _gather(shards, outs, p, prec, lat.V)[p * lat.Vh:(p + 1) * lat.Vh]
        gotx = _gather(shards, outx, p, prec, lat.V)[p * lat.Vh:(p + 1) * lat.Vh]
        assert not np.isnan(got).any()
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
        assert np.array_equal(gotx.view(np.uint64), wantx.view(np.uint64))


def test_sharded_hop_matches_oracle(cuda, restatement):
    L = (4, 4, 4, 12)
    lat, g64, u, q = _global(L, 32)
    want = restatement.hop("full", L, q, u)
    shards, gauges = _shards(L, 3, u, P.F64, 18)
    T = SH.LocalTransport(3)
    got = np.full_like(q, np.nan)
    for p in (P.EVEN, P.ODD):
        ins = [s.import_global(q, 1 - p) for s in shards]
        outs = [s.field(P.F64) for s in shards]
        SH.dslash(shards, gauges, outs, ins, p, P.F64, T)
        part = _gather(shards, outs, p, P.F64, lat.V)
        got[p * lat.Vh:(p + 1) * lat.Vh] = part[p * lat.Vh:(p + 1) * lat.Vh]
    assert relmax(got, want) < 1e-14


@pytest.mark.parametrize("N,own_streams", [(2, False), (4, False), (4, True)])
def test_sharded_cg_matches_single_device_cg(cuda, N, own_streams):
    L = (8, 8, 4, 16)
    kappa, tol = 0.12, 1e-10
    lat, g64, u, q = _global(L, 33)
    bs = lat.spinor_bytes(P.F64)
    be, bo = field_from_host(lat, q, 0, P.F64), field_from_host(lat, q, 1, P.F64)
    xe, xo = dev_bytes(bs), dev_bytes(bs)
    info = P.invert_cg(lat, g64, None, xe, xo, be, bo, P.cg_param(kappa=kappa, tol=tol))
    want = field_to_host(lat, xe, P.F64, 0)
    want[lat.Vh:] = field_to_host(lat, xo, P.F64, 1)[lat.Vh:]

    shards, gauges = _shards(L, N, u, P.F64, 18, own_streams)
    T = SH.LocalTransport(N)
    b_e = [s.import_global(q, 0) for s in shards]
    b_o = [s.import_global(q, 1) for s in shards]
    x_e, x_o, iters, res = SH.cg_solve(shards, gauges, b_e, b_o, kappa, T, tol)
    got = _gather(shards, x_e, 0, P.F64, lat.V)
    got[lat.Vh:] = _gather(shards, x_o, 1, P.F64, lat.V)[lat.Vh:]
    assert res <= tol
    assert abs(iters - info.iterations) <= 2, (iters, info.iterations)
    assert relmax(got, want) < 1e-8


def test_site_range_vector_ops_match_torch(cuda):
    """plqcd_sites_norm2 / cg_update / xpay / sub_norm2 on a site range of
    F64 fields against the same operations written in torch FP64; sites
    outside the range are untouched; scalars come from device memory."""
    import torch
    L = (8, 4, 6, 8)
    lat = new_lattice(L)
    lib = P.lib()
    Vh = lat.Vh
    bs = lat.spinor_bytes(P.F64)
    fs = [dev_bytes(bs) for _ in range(5)]
    for k, f in enumerate(fs):
        lat.spinor_gaussian(f, P.F64, 0, 70 + k)
    x, r, p, ap, z = fs
    v = lambda f: f.view(torch.float64).view(12, Vh, 2)
    h0, n = 37, Vh - 80
    sl = slice(h0, h0 + n)
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    coef = torch.tensor([2.5, 1.25], dtype=torch.float64, device="cuda")
    x0, r0, p0, ap0 = (v(f).clone() for f in (x, r, p, ap))
    P.check(lib.plqcd_sites_norm2(lat.handle, p.data_ptr(), h0, n, out.data_ptr()))
    P.check(lib.plqcd_sites_cg_update(lat.handle, x.data_ptr(), r.data_ptr(), p.data_ptr(), ap.data_ptr(), h0, n,
                                      coef.data_ptr(), out[1:].data_ptr()))
    lat.synchronize()
    alpha = 2.0
    want_x, want_r = x0.clone(), r0.clone()
    want_x[:, sl] += alpha * p0[:, sl]
    want_r[:, sl] -= alpha * ap0[:, sl]
    assert torch.allclose(v(x), want_x, rtol=0, atol=1e-14) and torch.allclose(v(r), want_r, rtol=0, atol=1e-14)
    assert abs(out[0].item() - (p0[:, sl] ** 2).sum().item()) <= 1e-12 * out[0].item()
    assert abs(out[1].item() - (want_r[:, sl] ** 2).sum().item()) <= 1e-12 * out[1].item()
    P.check(lib.plqcd_sites_xpay(lat.handle, p.data_ptr(), r.data_ptr(), h0, n, coef.data_ptr()))
    P.check(lib.plqcd_sites_sub_norm2(lat.handle, z.data_ptr(), x.data_ptr(), r.data_ptr(), h0, n,
                                      out[2:].data_ptr()))
    lat.synchronize()
    want_p = p0.clone()
    want_p[:, sl] = v(r)[:, sl] + alpha * p0[:, sl]
    assert torch.allclose(v(p), want_p, rtol=0, atol=1e-14)
    d = v(x)[:, sl] - v(r)[:, sl]
    assert torch.allclose(v(z)[:, sl], d, rtol=0, atol=1e-14)
    assert abs(out[2].item() - (d ** 2).sum().item()) <= 1e-12 * out[2].item()
    # twice in a row: the reduction scratch is left clean
    P.check(lib.plqcd_sites_norm2(lat.handle, p.data_ptr(), h0, n, out[3:].data_ptr()))
    P.check(lib.plqcd_sites_norm2(lat.handle, p.data_ptr(), h0, n, out[3:].data_ptr()))
    lat.synchronize()
    assert abs(out[3].item() - (want_p[:, sl] ** 2).sum().item()) <= 1e-12 * out[3].item()
    assert lib.plqcd_sites_norm2(lat.handle, p.data_ptr(), Vh - 4, 8, out.data_ptr()) == P.ERR_ARG


def test_copy_segments_one_launch(cuda):
    """plqcd_copy_segments copies every segment of its table and refuses
    segments that are not 16-byte aligned."""
    import ctypes
    import torch
    lat = new_lattice((4, 4, 4, 4))
    src = torch.arange(4096, dtype=torch.int32, device="cuda").view(torch.uint8)
    dst = torch.zeros_like(src)
    # destinations back to back (no overlap), sources overlapping
    segs = [(dst.data_ptr() + 8 * k * (k + 1), src.data_ptr() + 16 * k * 5, 16 * (k + 1)) for k in range(20)]
    SH.copy_segments(lat, segs)
    lat.synchronize()
    for d, s, b in segs:
        o_d, o_s = d - dst.data_ptr(), s - src.data_ptr()
        assert bool((dst[o_d:o_d + b] == src[o_s:o_s + b]).all())
    n = 1
    bad = (ctypes.c_void_p * n)(dst.data_ptr() + 8)
    ok = (ctypes.c_void_p * n)(src.data_ptr())
    nb = (ctypes.c_size_t * n)(16)
    assert P.lib().plqcd_copy_segments(lat.handle, n, bad, ok, nb) == P.ERR_ARG
