"""Host logic of the t-slab decomposition (plqcd_b200/shard.py), on CPU.

The slab geometry maps every local site to the global site it holds; the
ghost-slice exchange moves the right bytes between ranks. The exchange runs
as two and four gloo ranks (127.0.0.1) over CPU tensors whose bytes encode
(plane, global slice): after the exchange every ghost slice holds exactly the
neighbour's boundary slice."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from plqcd_b200.shard import SPINOR_PLANES, GAUGE_PLANES, SlabGeometry
import plqcd_b200 as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _coords(L, eo):
    """(x, y, z, t) of global even/odd indices."""
    L0, L1, L2, L3 = L
    Vh = L0 * L1 * L2 * L3 // 2
    p, h = eo // Vh, eo % Vh
    xh, row = h % (L0 // 2), h // (L0 // 2)
    y, z, t = row % L1, (row // L1) % L2, row // (L1 * L2)
    x = 2 * xh + ((y + z + t + p) & 1)
    return x, y, z, t


@pytest.mark.parametrize("L,N", [((4, 4, 4, 8), 1), ((4, 4, 4, 8), 2), ((4, 6, 2, 16), 4), ((8, 4, 4, 12), 3)])
def test_slabs_cover_the_lattice_once(L, N):
    V = int(np.prod(L))
    seen = np.zeros(V, int)
    for r in range(N):
        geo = SlabGeometry(L, r, N)
        g = geo.local_to_global_sites()
        ghost = geo.ghost_mask()
        seen[g[~ghost]] += 1
        x, y, z, t = _coords(L, g)
        # local parity = global parity + 1
        p_loc = np.arange(2 * geo.Vh) // geo.Vh
        assert np.all(((x + y + z + t) & 1) == p_loc ^ 1)
        # ghost slices hold the neighbours' boundary slices
        tl = (np.arange(2 * geo.Vh) % geo.Vh) // geo.S
        assert np.all(t[tl == 0] == (geo.t0 - 1) % L[3])
        assert np.all(t[tl == geo.Lt + 1] == (geo.t0 + geo.Lt) % L[3])
        assert np.all((t[~ghost] >= geo.t0) & (t[~ghost] < geo.t0 + geo.Lt))
    assert np.all(seen == 1)


def test_local_neighbours_are_global_neighbours():
    """A local site's t-neighbour (t' +- 1, same x y z) is its global
    t-neighbour; its x/y/z neighbours wrap as in the global lattice."""
    L, N = (4, 4, 2, 8), 2
    for r in range(N):
        geo = SlabGeometry(L, r, N)
        g = geo.local_to_global_sites()
        gx = np.stack(_coords(L, g), 1)
        lx = np.stack(_coords(geo.local_dims, np.arange(2 * geo.Vh)), 1)
        # index local sites by local coordinates
        key = lambda c: ((c[:, 3] * L[2] + c[:, 2]) * L[1] + c[:, 1]) * L[0] + c[:, 0]
        order = np.full(int(np.prod(geo.local_dims)), -1)
        order[key(lx)] = np.arange(len(lx))
        inner = (lx[:, 3] >= 1) & (lx[:, 3] <= geo.Lt)
        for mu, ext in enumerate(geo.local_dims):
            for s in (+1, -1):
                nb = lx.copy()
                nb[:, mu] = (nb[:, mu] + s) % ext
                j = order[key(nb)]
                want = gx.copy()
                want[:, mu] = (want[:, mu] + s) % L[mu]
                assert np.array_equal(gx[j][inner], want[inner])


def test_slab_rejects_uneven_splits():
    with pytest.raises(P.PlqcdError):
        SlabGeometry((4, 4, 4, 8), 0, 3)
    with pytest.raises(P.PlqcdError):
        SlabGeometry((4, 4, 4, 6), 0, 2)   # odd slab thickness
    with pytest.raises(P.PlqcdError):
        SlabGeometry((4, 4, 4, 8), 0, 8)   # one slice per rank


WORKER = r"""
import os, sys
sys.path.insert(0, {root!r})
import numpy as np, torch, torch.distributed as dist
from plqcd_b200.shard import SlabGeometry, DistTransport, SPINOR_PLANES, GAUGE_PLANES
import plqcd_b200 as P
dist.init_process_group("gloo", init_method="env://", timeout=__import__("datetime").timedelta(seconds=60))
r, N = dist.get_rank(), dist.get_world_size()
L = (4, 4, 2, 4 * N)
geo = SlabGeometry(L, r, N)
T = DistTransport()
def fill(planes, nsites):
    # byte value of (plane k, local slice tl) = code of (k, global slice) for interior slices, 0 in ghosts
    f = torch.zeros(sum(planes) * nsites, dtype=torch.uint8)
    for tl in range(1, geo.Lt + 1):
        for k, (o, n) in enumerate(geo.plane_slices(planes, nsites, tl)):
            f[o:o + n] = (7 * k + 3 * ((geo.t0 + tl - 1) % L[3]) + 1) % 251
    return f
ok = True
for prec in (P.F64, P.F16):
    planes = SPINOR_PLANES[prec]
    f = fill(planes, geo.Vh)
    T.start(geo, f, geo.spinor_groups(prec)).wait()
    for tl, gt in ((0, (geo.t0 - 1) % L[3]), (geo.Lt + 1, (geo.t0 + geo.Lt) % L[3])):
        for k, (o, n) in enumerate(geo.plane_slices(planes, geo.Vh, tl)):
            ok &= bool((f[o:o + n] == (7 * k + 3 * gt + 1) % 251).all())
    # interior untouched
    g = fill(planes, geo.Vh)
    for tl in range(1, geo.Lt + 1):
        for (o, n) in geo.plane_slices(planes, geo.Vh, tl):
            ok &= bool((f[o:o + n] == g[o:o + n]).all())
# gauge: lower ghost only
ne, eb = GAUGE_PLANES[(P.F64, 18)]
planes = [eb] * (8 * ne)
f = fill(planes, geo.Vh)
T.start(geo, f, geo.gauge_groups(P.F64, 18), lower=True, upper=False).wait()
for k, (o, n) in enumerate(geo.plane_slices(planes, geo.Vh, 0)):
    ok &= bool((f[o:o + n] == (7 * k + 3 * ((geo.t0 - 1) % L[3]) + 1) % 251).all())
for (o, n) in geo.plane_slices(planes, geo.Vh, geo.Lt + 1):
    ok &= bool((f[o:o + n] == 0).all())
print("OK" if ok else "FAIL", flush=True)
dist.destroy_process_group()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("nproc", [2, 4])
def test_ghost_exchange_over_gloo(nproc):
    port = _free_port()
    code = WORKER.format(root=ROOT)
    procs = []
    for r in range(nproc):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(nproc), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    for p in procs:
        o, e = p.communicate(timeout=180)
        assert p.returncode == 0, e[-2000:]
        assert o.strip().endswith("OK"), o + e[-2000:]
