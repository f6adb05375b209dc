"""plqcd_b200 -- Python binding of the B200 Wilson hopping-matrix library.

The product is the C-ABI shared library ``libplqcd_b200.so`` built from
``plqcd_b200/csrc`` (``python -m plqcd_b200.build``); this module only binds
it with ctypes. There is no Python or CPU fallback: importing fails loudly
when the library is missing.

Two layers mirror the C headers in ``include/``:

* the reference's drop-in entry points (``include/dirac.h``,
  ``include/start.h``): ``init_plqcd``, ``hopping_matrix_eo/oe`` on host
  numpy arrays in the API layout (reference lib/dirac.c:35-791);
* the device-resident API (``include/plqcd_b200.h``): ``Lattice``,
  ``Gauge`` and functions taking device pointers (e.g. ``tensor.data_ptr()``
  of a torch CUDA tensor).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libplqcd_b200.so")

F64, F32, F16, BF16 = 0, 1, 2, 3
EVEN, ODD = 0, 1
DSLASH_COMPAT, DSLASH_G5_IN, DSLASH_G5_OUT = 1, 2, 4
PREC_NAMES = {F64: "f64", F32: "f32", F16: "f16", BF16: "bf16"}
SPINOR_BYTES_PER_SITE = {F64: 192, F32: 96, F16: 52, BF16: 52}

OK = 0
ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_STATE, ERR_TIMEOUT, ERR_NOCONV, ERR_NODEV = -1, -2, -3, -4, -5, -6, -7


class PlqcdError(RuntimeError):
    pass


_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_u64 = ctypes.c_uint64
_sz = ctypes.c_size_t
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)

# name: (restype, argtypes)
_SIGS = {
    # include/start.h
    "init_plqcd": (_i, [_i, ctypes.POINTER(ctypes.c_char_p)]),
    "finalize_plqcd": (None, []),
    "ipr": (_i, [_ip]),
    "comp_cpr": (None, [_i, _ip]),
    "set_npr": (None, []),
    "lex2cart": (None, [_i, _ip]),
    "cart2lex": (_i, [_ip]),
    "set_geometry": (None, []),
    "find_site": (None, [_ip, _ip, _ip]),
    "print_params": (None, [_vp]),
    # include/utils.h
    "alloc": (_vp, [_sz, _sz]),
    "amalloc": (_vp, [_sz, _i]),
    "afree": (None, [_vp]),
    "mpi_permanent_tag": (_i, []),
    "mpi_tag": (_i, []),
    "stop_watch": (_d, [_d]),
    # include/dirac.h
    "plqcd_hopping_matrix_eo_sse3_assymbly": (_d, [_vp, _vp, _vp]),
    "plqcd_hopping_matrix_oe_sse3_assymbly": (_d, [_vp, _vp, _vp]),
    "plqcd_hopping_matrix_eo_sse3_intrin": (_d, [_vp, _vp, _vp]),
    "plqcd_hopping_matrix_oe_sse3_intrin": (_d, [_vp, _vp, _vp]),
    "plqcd_hopping_matrix_eo_sse3_intrin_blocking": (_d, [_vp, _vp, _vp]),
    "plqcd_hopping_matrix_oe_sse3_intrin_blocking": (_d, [_vp, _vp, _vp]),
    **{f"plqcd_hopping_matrix_{p}_{v}": (_d, [_vp] * 6)
       for p in ("eo", "oe")
       for v in ("sse3_intrin_nohalfspinor", "avx_nohalfspinor", "single_mic_split",
                 "single_mic_split_nohalfspinor", "single_mic_split_nohalfspinor_short")},
    # include/plqcd_b200.h
    "plqcd_last_error": (ctypes.c_char_p, []),
    "plqcd_last_status": (_i, []),
    "plqcd_clear_error": (None, []),
    "plqcd_version": (ctypes.c_char_p, []),
    "plqcd_lattice_create": (_i, [_ip, _i, _vp, ctypes.POINTER(_vp)]),
    "plqcd_lattice_destroy": (_i, [_vp]),
    "plqcd_lattice_set_stream": (_i, [_vp, _vp]),
    "plqcd_lattice_stream": (_vp, [_vp]),
    "plqcd_lattice_synchronize": (_i, [_vp]),
    "plqcd_lattice_half_volume": (ctypes.c_long, [_vp]),
    "plqcd_lattice_last_kernel_ms": (_d, [_vp]),
    "plqcd_spinor_bytes": (_sz, [_vp, _i]),
    "plqcd_gauge_bytes": (_sz, [_vp, _i, _i]),
    "plqcd_gauge_create": (_i, [_vp, _i, _i, ctypes.POINTER(_vp)]),
    "plqcd_gauge_destroy": (_i, [_vp]),
    "plqcd_gauge_data": (_vp, [_vp]),
    "plqcd_gauge_load_host": (_i, [_vp, _vp]),
    "plqcd_gauge_load_device": (_i, [_vp, _vp]),
    "plqcd_gauge_store_host": (_i, [_vp, _vp]),
    "plqcd_gauge_random": (_i, [_vp, _u64]),
    "plqcd_gauge_unit": (_i, [_vp]),
    "plqcd_gauge_copy": (_i, [_vp, _vp]),
    "plqcd_spinor_import": (_i, [_vp, _vp, _i, _vp, _i]),
    "plqcd_spinor_export": (_i, [_vp, _vp, _i, _i, _vp]),
    "plqcd_spinor_convert": (_i, [_vp, _vp, _i, _vp, _i]),
    "plqcd_spinor_gaussian": (_i, [_vp, _vp, _i, _i, _u64]),
    "plqcd_spinor_norm2": (_i, [_vp, _vp, _i, _i, _vp]),
    "plqcd_spinor_norm2_noalloc": (_i, [_vp, _vp, _i, _i, _vp]),
    "plqcd_dslash": (_i, [_vp, _vp, _vp, _vp, _i, _i, ctypes.c_uint]),
    "plqcd_dslash_xpay": (_i, [_vp, _vp, _vp, _vp, _i, _i, ctypes.c_uint, _d, _vp, _d]),
    "plqcd_dslash_full": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i]),
    "plqcd_dslash_sites": (_i, [_vp, _vp, _vp, _vp, _i, _i, ctypes.c_uint, ctypes.c_double, _vp, ctypes.c_double,
                               ctypes.c_long, ctypes.c_long]),
    "plqcd_dslash_mrhs": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, ctypes.c_uint]),
    "plqcd_dslash_mrhs_xpay": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, ctypes.c_uint, _d, _vp, _d]),
    "plqcd_tune_enable": (_i, [_i]),
    "plqcd_tune_clear": (_i, []),
    "plqcd_tune_save": (_i, [ctypes.c_char_p]),
    "plqcd_tune_load": (_i, [ctypes.c_char_p]),
    "plqcd_tune_count": (_i, []),
    "plqcd_tune_get": (_i, [ctypes.c_char_p, _ip, _ip, _dp]),
    "plqcd_selftest": (_i, [_i, _i]),
    "plqcd_gauge_update": (_i, [_vp]),
    "plqcd_tma_timeout_test": (_i, [_i, ctypes.c_ulonglong]),
    "plqcd_sites_norm2": (_i, [_vp, _vp, ctypes.c_long, ctypes.c_long, _vp]),
    "plqcd_sites_cg_update": (_i, [_vp, _vp, _vp, _vp, _vp, ctypes.c_long, ctypes.c_long, _vp, _vp]),
    "plqcd_sites_xpay": (_i, [_vp, _vp, _vp, ctypes.c_long, ctypes.c_long, _vp]),
    "plqcd_sites_sub_norm2": (_i, [_vp, _vp, _vp, _vp, ctypes.c_long, ctypes.c_long, _vp]),
    "plqcd_copy_segments": (_i, [_vp, _i, _vp, _vp, _vp]),
    "plqcd_dropin_last_stats": (_i, [_dp, _dp, _dp]),
    "plqcd_aos_to_split": (_i, [_vp, _vp, _vp, ctypes.c_long]),
    **{f"plqcd_hopping_matrix_{w}_{v}": (ctypes.c_double, [_vp, _vp, _vp])
       for w in ("eo", "oe") for v in ("intrin_256", "intrin_512", "single_mic", "single_mic_short")},
    "plqcd_split_to_aos": (_i, [_vp, _vp, _vp, ctypes.c_long]),
}

_lib = None


def exported_symbols() -> list[str]:
    return list(_SIGS)


def lib() -> ctypes.CDLL:
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PlqcdError(f"{LIB_PATH} not found: build it with `python -m plqcd_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return (lib().plqcd_last_error() or b"").decode()


def check(rc: int) -> None:
    if rc != OK:
        raise PlqcdError(f"plqcd error {rc}: {last_error()}")


def _dims(L):
    return (ctypes.c_int * 4)(*[int(x) for x in L])


def _ptr(x) -> int | None:
    """Device or host address of a torch tensor, numpy array or int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    raise TypeError(f"cannot take the address of {type(x)}")


# ---------------------------------------------------------------------------
# drop-in layer (include/start.h, include/dirac.h)
# ---------------------------------------------------------------------------

def init_plqcd(input_file: str) -> int:
    argv = (ctypes.c_char_p * 3)(b"plqcd", input_file.encode(), None)
    return lib().init_plqcd(2, argv)


def finalize_plqcd() -> None:
    lib().finalize_plqcd()


def hopping_matrix(which: str, qin: np.ndarray, qout: np.ndarray, u: np.ndarray, variant: str = "sse3_assymbly") -> float:
    """Call plqcd_hopping_matrix_{eo,oe}_<variant> on host arrays in the API
    layout (complex128 (V, 12) spinors, (4V, 9) links). Returns the
    library's elapsed seconds; raises on a negative return."""
    for a in (qin, qout, u):
        assert a.dtype == np.complex128 and a.flags.c_contiguous
    f = getattr(lib(), f"plqcd_hopping_matrix_{which}_{variant}")
    t = f(qin.ctypes.data, qout.ctypes.data, u.ctypes.data)
    if t < 0:
        raise PlqcdError(f"hopping matrix failed: {last_error()}")
    return t


PACKED_LANES = {"intrin_256": 2, "intrin_512": 4, "single_mic": 4, "single_mic_short": 4}


def pack_lanes(a: np.ndarray, lanes: int) -> np.ndarray:
    """API-layout objects (n, E) -> lane-packed (n/lanes, E, lanes): the
    layout of arrays of spinor_256/512 (E = 12) or su3_256/512 (E = 9 per
    link, 36 per site) built by the copy_*_256/512 converters."""
    n, E = a.shape
    return np.ascontiguousarray(a.reshape(n // lanes, lanes, E).transpose(0, 2, 1))


def unpack_lanes(p: np.ndarray) -> np.ndarray:
    m, E, lanes = p.shape
    return np.ascontiguousarray(p.transpose(0, 2, 1).reshape(m * lanes, E))


def hopping_matrix_packed(which: str, qin: np.ndarray, qout: np.ndarray, u: np.ndarray, variant: str) -> float:
    """The lane-packed entry points on API-layout arrays: qin/u are packed
    for the call, the output objects unpacked back into qout (only the output
    parity changes)."""
    lanes = PACKED_LANES[variant]
    V = qin.shape[0]
    pq, po = pack_lanes(qin, lanes), pack_lanes(qout, lanes)
    pu = pack_lanes(u.reshape(V, 36), lanes)
    f = getattr(lib(), f"plqcd_hopping_matrix_{which}_{variant}")
    t = f(pq.ctypes.data, po.ctypes.data, pu.ctypes.data)
    if t < 0:
        raise PlqcdError(f"hopping matrix failed: {last_error()}")
    qout[:] = unpack_lanes(po)
    return t


def aos_to_split(a: np.ndarray):
    """(re, im) planes of a complex128 API-layout array, by the library's
    converter (plqcd_aos_to_split)."""
    a = np.ascontiguousarray(a, np.complex128)
    re, im = np.empty(a.shape, np.float64), np.empty(a.shape, np.float64)
    check(lib().plqcd_aos_to_split(a.ctypes.data, re.ctypes.data, im.ctypes.data, a.size))
    return re, im


def split_to_aos(re: np.ndarray, im: np.ndarray, out: np.ndarray) -> np.ndarray:
    """Merge split planes into the complex128 array `out` (plqcd_split_to_aos)."""
    assert out.dtype == np.complex128 and out.flags.c_contiguous and re.size == im.size == out.size
    re, im = np.ascontiguousarray(re, np.float64), np.ascontiguousarray(im, np.float64)
    check(lib().plqcd_split_to_aos(re.ctypes.data, im.ctypes.data, out.ctypes.data, out.size))
    return out


def hopping_matrix_split(which: str, qin: np.ndarray, qout: np.ndarray, u: np.ndarray,
                         variant: str = "sse3_intrin_nohalfspinor") -> float:
    """The split real/imaginary entry points on the same arrays: the complex
    inputs are split into planes, the output planes are merged back into
    qout (only the output parity changes)."""
    qre, qim = aos_to_split(qin)
    ure, uim = aos_to_split(u)
    ore, oim = aos_to_split(qout)
    f = getattr(lib(), f"plqcd_hopping_matrix_{which}_{variant}")
    t = f(ore.ctypes.data, oim.ctypes.data, ure.ctypes.data, uim.ctypes.data, qre.ctypes.data, qim.ctypes.data)
    if t < 0:
        raise PlqcdError(f"hopping matrix failed: {last_error()}")
    split_to_aos(ore, oim, qout)
    return t


def dropin_last_stats():
    k, h, d = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    check(lib().plqcd_dropin_last_stats(ctypes.byref(k), ctypes.byref(h), ctypes.byref(d)))
    return k.value, h.value, d.value


# ---------------------------------------------------------------------------
# device-resident layer (include/plqcd_b200.h)
# ---------------------------------------------------------------------------

class Lattice:
    """A plqcd_lattice: geometry, CUDA stream and scratch of one lattice."""

    def __init__(self, dims, device: int = 0, stream: int | None = None):
        self.dims = tuple(int(x) for x in dims)
        h = _vp()
        check(lib().plqcd_lattice_create(_dims(self.dims), device, stream, ctypes.byref(h)))
        self.handle = h
        self.device = device
        self.Vh = int(lib().plqcd_lattice_half_volume(h))
        self.V = 2 * self.Vh

    @property
    def stream(self) -> int:
        """The lattice's CUDA stream handle (0: the legacy default stream)."""
        return int(lib().plqcd_lattice_stream(self.handle) or 0)

    def close(self):
        if self.handle:
            lib().plqcd_lattice_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(lib().plqcd_lattice_synchronize(self.handle))

    @property
    def stream(self) -> int:
        return lib().plqcd_lattice_stream(self.handle) or 0

    def spinor_bytes(self, prec: int) -> int:
        return int(lib().plqcd_spinor_bytes(self.handle, prec))

    def gauge_bytes(self, prec: int, recon: int) -> int:
        return int(lib().plqcd_gauge_bytes(self.handle, prec, recon))

    # spinor helpers -------------------------------------------------------
    def spinor_import(self, aos_dev, parity: int, dst, prec: int):
        check(lib().plqcd_spinor_import(self.handle, _ptr(aos_dev), parity, _ptr(dst), prec))

    def spinor_export(self, src, prec: int, parity: int, aos_dev):
        check(lib().plqcd_spinor_export(self.handle, _ptr(src), prec, parity, _ptr(aos_dev)))

    def spinor_convert(self, dst, dprec: int, src, sprec: int):
        check(lib().plqcd_spinor_convert(self.handle, _ptr(dst), dprec, _ptr(src), sprec))

    def spinor_norm2(self, fields, prec: int, nfields: int, out_dev):
        check(lib().plqcd_spinor_norm2(self.handle, _ptr(fields), prec, nfields, _ptr(out_dev)))

    def spinor_gaussian(self, dst, prec: int, parity: int, seed: int):
        check(lib().plqcd_spinor_gaussian(self.handle, _ptr(dst), prec, parity, seed))

    # hopping ----------------------------------------------------------------
    def dslash(self, gauge: "Gauge", out, inp, out_parity: int, prec: int, flags: int = 0):
        check(lib().plqcd_dslash(self.handle, gauge.handle, _ptr(out), _ptr(inp), out_parity, prec, flags))

    def dslash_xpay(self, gauge: "Gauge", out, inp, out_parity: int, prec: int, a: float, x, b: float,
                    flags: int = 0):
        check(lib().plqcd_dslash_xpay(self.handle, gauge.handle, _ptr(out), _ptr(inp), out_parity, prec, flags,
                                      a, _ptr(x), b))

    def dslash_mrhs(self, gauge: "Gauge", out, inp, nrhs: int, out_parity: int, prec: int, flags: int = 0):
        check(lib().plqcd_dslash_mrhs(self.handle, gauge.handle, _ptr(out), _ptr(inp), nrhs, out_parity, prec,
                                      flags))

    def dslash_mrhs_xpay(self, gauge: "Gauge", out, inp, nrhs: int, out_parity: int, prec: int, a: float, x,
                         b: float, flags: int = 0):
        check(lib().plqcd_dslash_mrhs_xpay(self.handle, gauge.handle, _ptr(out), _ptr(inp), nrhs, out_parity, prec,
                                           flags, a, _ptr(x), b))

    def dslash_sites(self, gauge: "Gauge", out, inp, out_parity: int, prec: int, h_begin: int, h_count: int,
                     flags: int = 0, a: float = 1.0, x=None, b: float = 0.0):
        """out[h] = a H in (+ b x) on output half-sites [h_begin, h_begin + h_count)."""
        check(lib().plqcd_dslash_sites(self.handle, gauge.handle, _ptr(out), _ptr(inp), out_parity, prec, flags,
                                       a, _ptr(x) if x is not None else None, b, h_begin, h_count))

    def dslash_full(self, gauge: "Gauge", out_even, out_odd, in_even, in_odd, prec: int):
        check(lib().plqcd_dslash_full(self.handle, gauge.handle, _ptr(out_even), _ptr(out_odd), _ptr(in_even),
                                      _ptr(in_odd), prec))


class Gauge:
    """A plqcd_gauge: device gauge field owned by the library."""

    def __init__(self, lat: Lattice, prec: int = F64, recon: int = 18):
        h = _vp()
        check(lib().plqcd_gauge_create(lat.handle, prec, recon, ctypes.byref(h)))
        self.handle = h
        self.lat = lat
        self.prec = prec
        self.recon = recon

    def close(self):
        if self.handle:
            lib().plqcd_gauge_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def data(self) -> int:
        return lib().plqcd_gauge_data(self.handle)

    def load_host(self, u: np.ndarray):
        assert u.dtype == np.complex128 and u.flags.c_contiguous and u.shape == (4 * self.lat.V, 9)
        check(lib().plqcd_gauge_load_host(self.handle, u.ctypes.data))

    def load_device(self, u_dev):
        check(lib().plqcd_gauge_load_device(self.handle, _ptr(u_dev)))

    def store_host(self) -> np.ndarray:
        u = np.empty((4 * self.lat.V, 9), np.complex128)
        check(lib().plqcd_gauge_store_host(self.handle, u.ctypes.data))
        return u

    def random(self, seed: int):
        check(lib().plqcd_gauge_random(self.handle, seed))

    def unit(self):
        check(lib().plqcd_gauge_unit(self.handle))

    def copy_from(self, src: "Gauge"):
        check(lib().plqcd_gauge_copy(self.handle, src.handle))


# ---------------------------------------------------------------------------
# solver (include/plqcd_b200.h: plqcd_invert_cg)
# ---------------------------------------------------------------------------

class CgParam(ctypes.Structure):
    _fields_ = [("kappa", ctypes.c_double), ("tol", ctypes.c_double), ("max_iter", ctypes.c_int),
                ("sloppy_prec", ctypes.c_int), ("delta", ctypes.c_double), ("verbose", ctypes.c_int)]


class CgInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("reliable_updates", ctypes.c_int), ("converged", ctypes.c_int),
                ("schur_residual", ctypes.c_double), ("true_residual", ctypes.c_double),
                ("seconds", ctypes.c_double), ("sloppy_hops", ctypes.c_double), ("f64_hops", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_SIGS.update({
    "plqcd_cg_param_default": (None, [ctypes.POINTER(CgParam)]),
    "plqcd_invert_cg": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(CgParam), ctypes.POINTER(CgInfo)]),
})


def cg_param(**kw) -> CgParam:
    p = CgParam()
    lib().plqcd_cg_param_default(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def invert_cg(lat: Lattice, g64: Gauge, g_sloppy: Gauge | None, x_even, x_odd, b_even, b_odd,
              param: CgParam, raise_on_error: bool = True) -> CgInfo:
    info = CgInfo()
    rc = lib().plqcd_invert_cg(lat.handle, g64.handle, g_sloppy.handle if g_sloppy else None, _ptr(x_even),
                               _ptr(x_odd), _ptr(b_even), _ptr(b_odd), ctypes.byref(param), ctypes.byref(info))
    if rc != OK and raise_on_error:
        raise PlqcdError(f"plqcd error {rc}: {last_error()}")
    return info


class SolveItem(ctypes.Structure):
    _fields_ = [("lat", _vp), ("g64", _vp), ("g_sloppy", _vp), ("nrhs", ctypes.c_int),
                ("x_even", _vp), ("x_odd", _vp), ("b_even", _vp), ("b_odd", _vp)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("reliable_updates", ctypes.c_int), ("converged", ctypes.c_int),
                ("max_schur_residual", ctypes.c_double), ("max_true_residual", ctypes.c_double),
                ("seconds", ctypes.c_double), ("graph_launches", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_SIGS.update({
    "plqcd_invert_cg_batch": (_i, [ctypes.POINTER(SolveItem), _i, ctypes.POINTER(CgParam), _i,
                                   ctypes.POINTER(BatchInfo), _dp]),
})


def invert_cg_batch(items, param: CgParam, use_graph: bool = True, raise_on_error: bool = True):
    """items: list of dicts with lat, g64, g_sloppy, nrhs, x_even, x_odd,
    b_even, b_odd. Returns (BatchInfo, per-RHS true residuals)."""
    arr = (SolveItem * len(items))()
    n = 0
    for k, it in enumerate(items):
        arr[k].lat = it["lat"].handle
        arr[k].g64 = it["g64"].handle
        arr[k].g_sloppy = it["g_sloppy"].handle if it.get("g_sloppy") else None
        arr[k].nrhs = it["nrhs"]
        for f in ("x_even", "x_odd", "b_even", "b_odd"):
            setattr(arr[k], f, _ptr(it[f]))
        n += it["nrhs"]
    res = (ctypes.c_double * n)()
    info = BatchInfo()
    rc = lib().plqcd_invert_cg_batch(arr, len(items), ctypes.byref(param), int(use_graph), ctypes.byref(info), res)
    if rc != OK and raise_on_error:
        raise PlqcdError(f"plqcd error {rc}: {last_error()}")
    return info, list(res)
