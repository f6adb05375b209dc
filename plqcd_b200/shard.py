"""A lattice held in t-slabs by several devices: ghost-slice exchange, the
hopping matrix and the even/odd CG on top of it.

The reference decomposes the lattice over an MPI process grid and exchanges
half-spinor faces inside every hop (lib/dirac.c:124-131, 203-228; face
tables nn_bnde/nn_bndo, include/plqcd_global_params.h:119-132). Here the
lattice is cut along t only, one slab per rank (one process per GPU):

* rank r of N holds global t in [r*Lt, (r+1)*Lt), Lt = L3 / N, even;
* its local lattice is (L0, L1, L2, Lt + 2): local slice t' = 0 and
  t' = Lt + 1 are ghosts holding global slices r*Lt - 1 and (r+1)*Lt
  (periodic), the interior is t' = 1 .. Lt;
* local half-site h = xh + L0/2 (y + L1 (z + L2 t')); since t' = t - r*Lt + 1
  and r*Lt is even, a site's local parity is its global parity plus one, so
  the field of global parity p is stored as the local field of parity 1 - p;
* one hop: the input field's first and last interior slices go to the ranks
  below and above. A t-slice is contiguous in every SoA plane, so the slice
  of a group of planes is one strided (planes x slice-bytes) view: packed
  with one copy, sent with one send, unpacked with one copy. The interior
  slices that do not touch a ghost are computed meanwhile, then the two
  boundary slices; the kernels are the single-device ones, run on site ranges
  (plqcd_dslash_sites), with the periodic wrap never reached in t;
* links: the backward t-link of slice t' = 1 sits in ghost slice 0, filled
  once per gauge field from the rank below;
* streams: every slab's kernels and torch work run on its lattice's stream.
  Slabs held by one process may each have their own stream: an exchange
  then waits for all of them (on the first slab's stream) and they wait for
  it, so the hops of the slabs run side by side on the device.

Transports move the ghost slices: DistTransport (torch.distributed
point-to-point, NCCL between GPUs, gloo on the host) and LocalTransport (all
slabs in one process on one device, for tests and single-GPU runs).
"""
from __future__ import annotations

import numpy as np

from . import BF16, F16, F32, F64, Gauge, Lattice, PlqcdError

# bytes of one site in each SoA plane of a one-parity spinor field
SPINOR_PLANES = {F64: [16] * 12, F32: [16] * 6, F16: [16, 16, 16, 4], BF16: [16, 16, 16, 4]}
# (elements per link, bytes per element) of the gauge formats; a field is
# planes[2 parities][4 mu][elements][Vh]
GAUGE_PLANES = {(F64, 18): (9, 16), (F64, 12): (6, 16), (F32, 18): (9, 8), (F32, 12): (3, 16), (F16, 12): (3, 8),
                (BF16, 12): (3, 8)}


class SlabGeometry:
    """Index arithmetic of one rank's slab (no device objects)."""

    def __init__(self, L, rank: int, nranks: int):
        L = tuple(int(v) for v in L)
        if nranks < 1 or L[3] % nranks or (L[3] // nranks) % 2 or L[3] // nranks < 2:
            raise PlqcdError(f"t extent {L[3]} does not split into {nranks} even slabs of >= 2 slices")
        if any(v < 2 or v % 2 for v in L):
            raise PlqcdError(f"lattice extents must be even and >= 2: {L}")
        self.L, self.rank, self.nranks = L, rank, nranks
        self.Lt = L[3] // nranks
        self.t0 = rank * self.Lt                      # first global t of the slab
        self.local_dims = (L[0], L[1], L[2], self.Lt + 2)
        self.L0h = L[0] // 2
        self.S = self.L0h * L[1] * L[2]               # half-sites of one t-slice
        self.Vh = self.S * (self.Lt + 2)              # local half volume, ghosts included
        self.below = (rank - 1) % nranks
        self.above = (rank + 1) % nranks

    @staticmethod
    def local_parity(global_parity: int) -> int:
        return global_parity ^ 1

    def interior(self):
        """(h_begin, h_count) of the interior slices."""
        return self.S, self.S * self.Lt

    def slice_range(self, tl: int):
        return tl * self.S, self.S

    def plane_slices(self, plane_bytes, nsites: int, tl: int):
        """Byte ranges (offset, length) of local slice tl in every plane of a
        field whose planes hold nsites sites of plane_bytes[k] bytes each."""
        out, off = [], 0
        for eb in plane_bytes:
            out.append((off + tl * self.S * eb, self.S * eb))
            off += nsites * eb
        return out

    def spinor_slices(self, prec: int, tl: int):
        return self.plane_slices(SPINOR_PLANES[prec], self.Vh, tl)

    def spinor_groups(self, prec: int):
        """Plane groups (byte offset, planes, element bytes) of a one-parity
        field: planes of equal element size that follow each other."""
        return _groups(SPINOR_PLANES[prec], self.Vh)

    def gauge_groups(self, prec: int, recon: int):
        ne, eb = GAUGE_PLANES[(prec, recon)]
        return _groups([eb] * (8 * ne), self.Vh)

    def cols(self, tl: int, eb: int):
        """Byte columns of local slice tl in a plane of eb-byte elements."""
        return slice(tl * self.S * eb, (tl + 1) * self.S * eb)

    # ---- API-layout (host) mapping between global and local arrays --------
    def local_to_global_sites(self):
        """For every local even/odd site index (API layout: parity-major),
        the global even/odd index of the site it holds."""
        L0, L1, L2, L3 = self.L
        Lt2 = self.Lt + 2
        Vl = 2 * self.Vh
        idx = np.arange(Vl)
        p_loc, h = idx // self.Vh, idx % self.Vh
        xh = h % self.L0h
        row = h // self.L0h
        y = row % L1
        z = (row // L1) % L2
        tl = row // (L1 * L2)
        assert tl.max() < Lt2
        x = 2 * xh + ((y + z + tl + p_loc) & 1)
        t = (self.t0 + tl - 1) % L3
        p_g = (x + y + z + t) & 1
        Vh_g = L0 * L1 * L2 * L3 // 2
        return p_g * Vh_g + x // 2 + self.L0h * (y + L1 * (z + L2 * t))

    def local_links_from_global(self, u_global: np.ndarray, ghosts: bool = True) -> np.ndarray:
        """Local API-layout link array (4 V_local, 9) from the global one;
        ghost slices zero unless `ghosts`."""
        g = self.local_to_global_sites()
        u = u_global.reshape(-1, 4, 9)[g].copy()
        if not ghosts:
            u[self.ghost_mask()] = 0
        return u.reshape(-1, 9)

    def local_spinor_from_global(self, q_global: np.ndarray, ghosts: bool = True) -> np.ndarray:
        q = q_global[self.local_to_global_sites()].copy()
        if not ghosts:
            q[self.ghost_mask()] = 0
        return q

    def ghost_mask(self) -> np.ndarray:
        """True for local API-layout sites in a ghost slice."""
        h = np.arange(2 * self.Vh) % self.Vh
        tl = h // self.S
        return (tl == 0) | (tl == self.Lt + 1)


def _groups(plane_bytes, nsites):
    out, off, i = [], 0, 0
    while i < len(plane_bytes):
        eb, n = plane_bytes[i], 0
        while i < len(plane_bytes) and plane_bytes[i] == eb:
            n, i = n + 1, i + 1
        out.append((off, n, eb))
        off += n * nsites * eb
    return out


def _view(field, geo: SlabGeometry, group):
    """(planes, Vh * eb) byte view of one plane group of a field."""
    off, n, eb = group
    return field[off:off + n * geo.Vh * eb].view(n, geo.Vh * eb)


def segment_tables(segs):
    """[(dst_ptr, src_ptr, nbytes), ...] as the argument arrays of
    plqcd_copy_segments, PLQCD_COPY_MAX_SEGMENTS segments per table."""
    import ctypes
    tables = []
    for k in range(0, len(segs), 128):
        part = segs[k:k + 128]
        n = len(part)
        tables.append((n, (ctypes.c_void_p * n)(*[d for d, _, _ in part]),
                       (ctypes.c_void_p * n)(*[s_ for _, s_, _ in part]),
                       (ctypes.c_size_t * n)(*[b for _, _, b in part])))
    return tables


def copy_segments(lat, segs):
    """Device copies [(dst_ptr, src_ptr, nbytes), ...] on the lattice's
    stream, PLQCD_COPY_MAX_SEGMENTS per launch (plqcd_copy_segments).
    `segs` may also be the result of segment_tables."""
    from . import check, lib
    tables = segs if segs and len(segs[0]) == 4 else segment_tables(segs)
    for n, dst, src, nb in tables:
        check(lib().plqcd_copy_segments(lat.handle, n, dst, src, nb))


class LocalTransport:
    """All slabs in one process (one device): ghost slices are copied."""

    def __init__(self, nranks: int):
        self.nranks = nranks
        self._tables = {}  # segment tables of the fields exchanged so far

    def exchange(self, geos, fields, groups, lower: bool = True, upper: bool = True, lat=None):
        """fields[r]: torch uint8 tensor of rank r's field; groups: its plane
        groups (SlabGeometry.spinor_groups / gauge_groups). With `lat` (device
        fields): every plane's slice of every slab and direction in one
        plqcd_copy_segments launch on lat's stream (the segment table of a set
        of field addresses is built once); otherwise one strided copy per
        plane group and direction."""
        if lat is not None and fields and fields[0].is_cuda:
            key = (tuple(f.data_ptr() for f in fields), tuple(tuple(g) for g in groups), lower, upper,
                   tuple((g.L, g.rank, g.nranks) for g in geos))
            tables = self._tables.get(key)
            if tables is not None:
                copy_segments(lat, tables)
                return
            segs = []
            for r, geo in enumerate(geos):
                base = fields[r].data_ptr()
                for off, n, eb in groups:
                    nbytes = geo.S * eb
                    for k in range(n):
                        plane = off + k * geo.Vh * eb
                        if lower:  # my last interior slice -> ghost 0 of the rank above
                            up = geos[geo.above]
                            segs.append((fields[geo.above].data_ptr() + plane + 0 * up.S * eb,
                                         base + plane + geo.Lt * geo.S * eb, nbytes))
                        if upper:  # my first interior slice -> ghost Lt+1 of the rank below
                            dn = geos[geo.below]
                            segs.append((fields[geo.below].data_ptr() + plane + (dn.Lt + 1) * dn.S * eb,
                                         base + plane + 1 * geo.S * eb, nbytes))
            tables = segment_tables(segs)
            if len(self._tables) >= 256:
                self._tables.clear()
            self._tables[key] = tables
            copy_segments(lat, tables)
            return
        for r, geo in enumerate(geos):
            for gr in groups:
                src = _view(fields[r], geo, gr)
                eb = gr[2]
                if lower:  # my last interior slice -> ghost 0 of the rank above
                    up = geos[geo.above]
                    _view(fields[geo.above], up, gr)[:, up.cols(0, eb)].copy_(src[:, geo.cols(geo.Lt, eb)])
                if upper:  # my first interior slice -> ghost Lt+1 of the rank below
                    dn = geos[geo.below]
                    _view(fields[geo.below], dn, gr)[:, dn.cols(dn.Lt + 1, eb)].copy_(src[:, geo.cols(1, eb)])


class _Exchange:
    """Sends and receives of one exchange in flight: wait() completes them
    and copies the received slices into the ghost slices."""

    def __init__(self, works, unpack):
        self.works, self.unpack = works, unpack

    def wait(self):
        for w in self.works:
            w.wait()
        for dst, buf in self.unpack:
            dst.copy_(buf)


class DistTransport:
    """One slab per process: ghost slices travel by torch.distributed
    point-to-point operations (NCCL between GPUs, gloo on the host). Per plane
    group and direction the boundary slice is packed into one contiguous
    buffer (one strided copy), sent with one send, received into one buffer
    and unpacked into the ghost slice; all sends and receives of an exchange
    go in one batch."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group

    def start(self, geo: SlabGeometry, field, groups, lower: bool = True, upper: bool = True) -> _Exchange:
        """Post the sends and receives of one exchange; call .wait() on the
        result before reading the ghost slices."""
        import torch
        dist = self.dist
        if geo.nranks == 1:
            LocalTransport(1).exchange([geo], [field], groups, lower, upper)
            return _Exchange([], [])
        grank = lambda r: dist.get_global_rank(self.group, r) if self.group is not None else r
        ops, unpack = [], []
        for gr in groups:
            v, eb = _view(field, geo, gr), gr[2]
            for on, src_tl, ghost_tl, to, frm in ((lower, geo.Lt, 0, geo.above, geo.below),
                                                 (upper, 1, geo.Lt + 1, geo.below, geo.above)):
                if not on:
                    continue
                send = v[:, geo.cols(src_tl, eb)].contiguous()
                recv = torch.empty_like(send)
                ops.append(dist.P2POp(dist.isend, send, grank(to), self.group))
                ops.append(dist.P2POp(dist.irecv, recv, grank(frm), self.group))
                unpack.append((v[:, geo.cols(ghost_tl, eb)], recv))
        return _Exchange(dist.batch_isend_irecv(ops) if ops else [], unpack)

    @staticmethod
    def wait(ex: _Exchange):
        ex.wait()


class ShardedLattice:
    """One rank's slab on its device: a local Lattice of (L0, L1, L2, Lt+2)
    plus the geometry. Fields are torch uint8 device tensors of
    lat.spinor_bytes(prec) bytes in the local parity (global parity ^ 1)."""

    def __init__(self, L, rank: int, nranks: int, device: int = 0, stream: int | None = None):
        self.geo = SlabGeometry(L, rank, nranks)
        self.lat = Lattice(self.geo.local_dims, device, stream)

    def field(self, prec: int):
        """Zeroed field, allocated and cleared on the slab's stream."""
        import torch
        with torch.cuda.stream(_torch_stream(self.lat)):
            return torch.zeros(self.lat.spinor_bytes(prec), dtype=torch.uint8, device=f"cuda:{self.lat.device}")

    def import_global(self, q_global: np.ndarray, global_parity: int, prec: int = F64, ghosts: bool = False):
        """Device field of one global parity from a global API-layout array."""
        import torch
        q = self.geo.local_spinor_from_global(q_global, ghosts)
        with torch.cuda.stream(_torch_stream(self.lat)):
            aos = torch.from_numpy(q).to(f"cuda:{self.lat.device}")
        f = self.field(prec)
        self.lat.spinor_import(aos, self.geo.local_parity(global_parity), f, prec)
        return f

    def export_interior(self, f, global_parity: int, prec: int = F64) -> tuple[np.ndarray, np.ndarray]:
        """(global even/odd indices, API-layout values) of the interior sites
        of a field of one global parity."""
        import torch
        with torch.cuda.stream(_torch_stream(self.lat)):
            aos = torch.zeros((2 * self.geo.Vh, 12), dtype=torch.complex128, device=f"cuda:{self.lat.device}")
        p = self.geo.local_parity(global_parity)
        self.lat.spinor_export(f, prec, p, aos)
        self.lat.synchronize()
        h0, n = self.geo.interior()
        loc = p * self.geo.Vh + np.arange(h0, h0 + n)
        return self.geo.local_to_global_sites()[loc], aos.cpu().numpy()[loc]

    def gauge_from_global(self, u_global: np.ndarray, prec: int = F64, recon: int = 18) -> Gauge:
        """Local gauge field (ghost slices zero: fill them with
        exchange_gauge) from the global API-layout link array."""
        u = self.geo.local_links_from_global(u_global, ghosts=False)
        g64 = Gauge(self.lat, F64, 18)
        g64.load_host(np.ascontiguousarray(u))
        if (prec, recon) == (F64, 18):
            return g64
        g = Gauge(self.lat, prec, recon)
        g.copy_from(g64)
        return g


def _wrap(ptr: int, nbytes: int, device: int):
    """uint8 torch tensor over device memory the library owns."""
    import torch

    class _Arr:
        pass
    a = _Arr()
    a.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}
    return torch.as_tensor(a, device=f"cuda:{device}")


def _torch_stream(lat: Lattice):
    """The lattice's CUDA stream as a torch stream (0: the default stream)."""
    import torch
    dev = f"cuda:{lat.device}"
    if not lat.stream:
        return torch.cuda.default_stream(dev)
    return torch.cuda.ExternalStream(lat.stream, device=dev)


class _StreamSet:
    """The distinct streams of a list of slabs with one reusable event per
    stream (a wait takes the event's state when it is issued, so an event
    can be recorded again at once)."""

    def __init__(self, lats):
        import torch
        self.streams = [_torch_stream(lat) for lat in lats]
        self.events = [torch.cuda.Event() for _ in lats]

    def join(self):
        for st, ev in zip(self.streams[1:], self.events[1:]):
            ev.record(st)
            self.streams[0].wait_event(ev)

    def fork(self):
        ev = self.events[0]
        ev.record(self.streams[0])
        for st in self.streams[1:]:
            st.wait_event(ev)


_STREAM_SETS: dict = {}


def _streams(shards):
    """The _StreamSet of the slabs' distinct streams (first slab's first),
    or None when they all share one stream."""
    key = tuple(sh.lat.stream for sh in shards) + (shards[0].lat.device,)
    ss = _STREAM_SETS.get(key, 0)
    if ss == 0:
        firsts = {}
        for sh in shards:
            firsts.setdefault(sh.lat.stream, sh.lat)
        ss = _StreamSet(list(firsts.values())) if len(firsts) > 1 else None
        _STREAM_SETS[key] = ss
    return ss


def join_streams(shards):
    """The first slab's stream waits for the work queued on every other
    slab's stream (no-op when all slabs share one stream)."""
    ss = _streams(shards)
    if ss is not None:
        ss.join()


def fork_streams(shards):
    """Every slab's stream waits for the work queued on the first slab's
    stream (no-op when all slabs share one stream)."""
    ss = _streams(shards)
    if ss is not None:
        ss.fork()


def exchange_gauge(shards, gauges, transport):
    """Fill ghost slice 0 of every shard's gauge field (the backward t-link
    of the first interior slice) from the rank below."""
    views = [_wrap(g.data, g.lat.gauge_bytes(g.prec, g.recon), g.lat.device) for g in gauges]
    groups = shards[0].geo.gauge_groups(gauges[0].prec, gauges[0].recon)
    if isinstance(transport, LocalTransport):
        join_streams(shards)
        transport.exchange([s.geo for s in shards], views, groups, lower=True, upper=False, lat=shards[0].lat)
        fork_streams(shards)
    else:
        transport.start(shards[0].geo, views[0], groups, lower=True, upper=False).wait()


def dslash(shards, gauges, outs, ins, out_parity: int, prec: int, transport, flags: int = 0, a: float = 1.0,
           xs=None, b: float = 0.0):
    """out = a H in (+ b x) on every shard's interior, out_parity global.
    shards/gauges/outs/ins/xs: one entry per slab this process holds (all N
    with LocalTransport, one with DistTransport). Slab k's output is written
    on slab k's stream; slabs of one process may share a stream or have one
    each (their hops then overlap on the device)."""
    p = SlabGeometry.local_parity(out_parity)
    groups = shards[0].geo.spinor_groups(prec)
    xs = xs if xs is not None else [None] * len(shards)
    if isinstance(transport, LocalTransport):
        # the exchange (on the first slab's stream) follows every slab's
        # earlier work; each slab's hop then runs on its own stream, so the
        # launches of slabs with separate streams overlap
        join_streams(shards)
        transport.exchange([s.geo for s in shards], ins, groups, lat=shards[0].lat)
        fork_streams(shards)
        for s, g, o, i, x in zip(shards, gauges, outs, ins, xs):
            h0, n = s.geo.interior()
            s.lat.dslash_sites(g, o, i, p, prec, h0, n, flags, a, x, b)
        return
    (s,), (g,), (o,), (i,), (x,) = shards, gauges, outs, ins, xs
    geo = s.geo
    ex = transport.start(geo, i, groups)
    # slices 2 .. Lt-1 need no ghost: computed while the exchange runs
    if geo.Lt > 2:
        s.lat.dslash_sites(g, o, i, p, prec, 2 * geo.S, (geo.Lt - 2) * geo.S, flags, a, x, b)
    ex.wait()
    for tl in (1, geo.Lt):
        h0, n = geo.slice_range(tl)
        s.lat.dslash_sites(g, o, i, p, prec, h0, n, flags, a, x, b)


# ---------------------------------------------------------------------------
# even/odd CG over the slabs (FP64)
# ---------------------------------------------------------------------------

class _Slabs:
    """The fields of one logical spinor over the slabs this process holds.
    Vector updates and interior dot products are the library's site-range
    kernels (plqcd_sites_*) on each slab's interior; a dot product over all
    slabs is the sum of the slabs' partial results, all-reduced over the
    ranks on the device (one NCCL all-reduce of one double). The scalars of
    the recursion live in a small device array `st`; the host reads one
    value when it needs to steer."""

    # slots of st: cg_update reads (st[RR], st[PAP]) as (rr, pAp); xpay
    # reads (st[RRN], st[RR_COPY]) as (rr_new, rr)
    RR, PAP, RRN, RR_COPY, AUX = 0, 1, 2, 3, 4

    def __init__(self, shards, transport):
        import torch
        self.shards, self.transport = shards, transport
        self.dev = f"cuda:{shards[0].lat.device}"
        # torch work of the solver (partial sums, scalar copies, the
        # all-reduce) runs on the slabs' stream, ordered with the kernels
        self.stream = _torch_stream(shards[0].lat)
        with torch.cuda.stream(self.stream):
            self.st = torch.zeros(8, dtype=torch.float64, device=self.dev)
            self.part = torch.zeros((len(shards), 1), dtype=torch.float64, device=self.dev)

    def new(self):
        return [s.field(F64) for s in self.shards]

    def _ptr(self, slot: int) -> int:
        return self.st.data_ptr() + 8 * slot

    def _finish(self, slot: int):
        """st[slot] = the sum of the slabs' partials, over every rank."""
        import torch
        join_streams(self.shards)
        with torch.cuda.stream(self.stream):
            torch.sum(self.part[:, 0], dim=0, keepdim=True, out=self.st[slot:slot + 1])
            if not isinstance(self.transport, LocalTransport):
                self.transport.dist.all_reduce(self.st[slot:slot + 1], group=self.transport.group)

    def _each(self, fn, *fields):
        from . import check, lib
        fork_streams(self.shards)  # the scalars and fields the first stream produced
        for k, s in enumerate(self.shards):
            h0, n = s.geo.interior()
            check(fn(lib(), s.lat.handle, h0, n, k, *[f[k].data_ptr() for f in fields]))

    def norm2(self, fs, slot: int):
        self._each(lambda L, lat, h0, n, k, x: L.plqcd_sites_norm2(lat, x, h0, n, self.part[k].data_ptr()), fs)
        self._finish(slot)

    def cg_update(self, x, r, p, ap):
        """alpha = st[RR] / st[PAP]; x += alpha p; r -= alpha Ap; st[RRN] = |r|^2"""
        self._each(lambda L, lat, h0, n, k, xx, rr, pp, aa: L.plqcd_sites_cg_update(
            lat, xx, rr, pp, aa, h0, n, self._ptr(self.RR), self.part[k].data_ptr()), x, r, p, ap)
        self._finish(self.RRN)

    def xpay(self, r, p):
        """beta = st[RRN] / st[RR]; p = r + beta p; then st[RR] = st[RRN]"""
        import torch
        with torch.cuda.stream(self.stream):
            self.st[self.RR_COPY] = self.st[self.RR]
        self._each(lambda L, lat, h0, n, k, pp, rr: L.plqcd_sites_xpay(lat, pp, rr, h0, n, self._ptr(self.RRN)),
                   p, r)
        with torch.cuda.stream(self.stream):
            self.st[self.RR] = self.st[self.RRN]

    def sub_norm2(self, x, y, z, slot: int):
        """z = x - y; st[slot] = |z|^2"""
        self._each(lambda L, lat, h0, n, k, zz, xx, yy: L.plqcd_sites_sub_norm2(
            lat, zz, xx, yy, h0, n, self.part[k].data_ptr()), z, x, y)
        self._finish(slot)

    def value(self, slot: int) -> float:
        import torch
        with torch.cuda.stream(self.stream):
            return float(self.st[slot].item())

    def copy(self, src, dst):
        import torch
        join_streams(self.shards)
        with torch.cuda.stream(self.stream):
            for s_, d in zip(src, dst):
                d.copy_(s_)
        fork_streams(self.shards)


def cg_solve(shards, g64s, b_even, b_odd, kappa: float, transport, tol: float = 1e-10, max_iter: int = 10000):
    """Solve D x = b, D = 1 - kappa H, on the slabs: even/odd CG on
    Mhat^dag Mhat with Mhat = 1 - kappa^2 H_eo H_oe (gamma5-hermitian, so
    Mhat^dag = g5 Mhat g5, folded into the hopping kernels), convergence on
    the FP64 Schur residual |b' - Mhat x_e| / |b'| <= tol, then
    x_o = b_o + kappa H_oe x_e; the same algorithm as plqcd_invert_cg in
    FP64. b_even/b_odd: lists of per-slab fields of global parity 0 / 1.
    Returns (x_even, x_odd, iterations, schur_residual). The hops are the
    library's kernels with one ghost exchange each; the vector updates and
    interior dot products are the library's site-range kernels
    (plqcd_sites_*), each dot product summed over the ranks with one
    all-reduce on the device; the host reads one scalar per iteration."""
    from . import DSLASH_G5_IN, DSLASH_G5_OUT, EVEN, ODD
    S = _Slabs(shards, transport)

    def hop(outs, ins, parity, flags=0, a=1.0, xs=None, b=0.0):
        dslash(shards, g64s, outs, ins, parity, F64, transport, flags, a, xs, b)

    tmp_o = S.new()

    def mhat(outs, ins, dagger):
        fin = DSLASH_G5_IN if dagger else 0
        fout = DSLASH_G5_OUT if dagger else 0
        hop(tmp_o, ins, ODD, fin)
        hop(outs, tmp_o, EVEN, fout, -kappa * kappa, ins, 1.0)

    bprime, rhs = S.new(), S.new()
    hop(bprime, b_odd, EVEN, 0, kappa, b_even, 1.0)
    S.norm2(bprime, S.AUX)
    bp2 = S.value(S.AUX)
    x_e, x_o = S.new(), S.new()
    if not bp2 > 0:
        hop(x_o, x_e, ODD, 0, kappa, b_odd, 1.0)
        return x_e, x_o, 0, 0.0
    mhat(rhs, bprime, True)
    r, p, t, Ap, r64 = S.new(), S.new(), S.new(), S.new(), S.new()
    S.copy(rhs, r)
    S.copy(rhs, p)
    S.norm2(r, S.RR)
    target = tol * tol * S.value(S.RR)
    sr2 = bp2
    it = 0
    for it in range(1, max_iter + 1):
        mhat(t, p, False)
        S.norm2(t, S.PAP)
        mhat(Ap, t, True)
        S.cg_update(x_e, r, p, Ap)          # alpha from the device, st[RRN] = |r|^2
        if S.value(S.RRN) <= target:        # the one host read of an iteration
            # FP64 Schur residual decides convergence
            mhat(t, x_e, False)
            S.sub_norm2(bprime, t, r64, S.AUX)
            sr2 = S.value(S.AUX)
            if sr2 <= tol * tol * bp2:
                break
            mhat(r, r64, True)
            S.norm2(r, S.RRN)
            if S.value(S.RRN) <= target:
                target *= 0.25
        S.xpay(r, p)                        # beta = rr_new / rr from the device
    hop(x_o, x_e, ODD, 0, kappa, b_odd, 1.0)
    join_streams(shards)  # the solution is complete on the first slab's stream
    return x_e, x_o, it, (sr2 / bp2) ** 0.5
