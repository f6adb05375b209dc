"""plqcd_spinor_norm2_noalloc: the batched norm without any device allocation.

It serves callers that cannot allocate device memory: applications whose
device memory all comes from their own pool or budget, and latency-bound
loops that cannot take cudaFree's device-wide synchronisation. Its result
must equal plqcd_spinor_norm2's,
which gets its scratch from the lattice workspace, call after call: the
static scratch keeps the previous call's contents and must not leak into
the next result. Collected last so that a failure here stops a -x run only
after every other test has run; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

import plqcd_b200 as P
from oracle import oracle as O
from tests.gpu_util import dev_bytes, field_from_host, new_lattice

pytestmark = pytest.mark.gpu
RTOL = 1e-12  # the tolerance of the batched-norm tests


@pytest.mark.parametrize("prec", [P.F64, P.F16])
def test_noalloc_norm2_matches_workspace_norm2_twice(cuda, prec):
    import torch
    L = (8, 8, 8, 16)
    lat = new_lattice(L)
    rng = np.random.default_rng(2026)
    nf = 6
    bs = lat.spinor_bytes(prec)
    block = dev_bytes(nf * bs)
    for f in range(nf):
        src = field_from_host(lat, O.gaussian_spinor(lat.V, rng) * (1 + f), f % 2, P.F64)
        lat.spinor_convert(block[f * bs:(f + 1) * bs], prec, src, P.F64)
    ref = torch.zeros(nf, dtype=torch.float64, device="cuda")
    P.check(P.lib().plqcd_spinor_norm2(lat.handle, block.data_ptr(), prec, nf, ref.data_ptr()))
    for call in range(2):
        out = torch.full((nf,), -1.0, dtype=torch.float64, device="cuda")
        P.check(P.lib().plqcd_spinor_norm2_noalloc(lat.handle, block.data_ptr(), prec, nf, out.data_ptr()))
        lat.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=RTOL, err_msg=f"call {call}")
    # a smaller batch after a larger one: stale partials must not leak in
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    P.check(P.lib().plqcd_spinor_norm2_noalloc(lat.handle, block.data_ptr(), prec, 2, out.data_ptr()))
    lat.synchronize()
    np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy()[:2], rtol=RTOL)


def test_noalloc_norm2_rejects_batches_beyond_its_scratch(cuda):
    import torch
    lat = new_lattice((4, 4, 4, 4))
    limit = 32  # PLQCD_NORM2_NOALLOC_MAX_FIELDS
    bs = lat.spinor_bytes(P.F64)
    block = dev_bytes((limit + 1) * bs)
    out = torch.zeros(limit + 1, dtype=torch.float64, device="cuda")
    for n in (0, limit + 1):
        rc = P.lib().plqcd_spinor_norm2_noalloc(lat.handle, block.data_ptr(), P.F64, n, out.data_ptr())
        assert rc == -1
        assert "outside 1..32" in P.last_error()
    block.zero_()
    P.check(P.lib().plqcd_spinor_norm2_noalloc(lat.handle, block.data_ptr(), P.F64, limit, out.data_ptr()))
    lat.synchronize()
    assert float(out[:limit].abs().max()) == 0.0
