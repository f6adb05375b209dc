"""Helpers for the GPU parity tests: device buffers (torch, plumbing only)
and transfers through the library's C-ABI layout converters."""
import numpy as np

import plqcd_b200 as P


def torch():
    import torch as t
    return t


def new_lattice(L):
    t = torch()
    return P.Lattice(L, 0, t.cuda.current_stream().cuda_stream)


def dev_bytes(n):
    t = torch()
    return t.empty(int(n), dtype=t.uint8, device="cuda")


def to_dev(a: np.ndarray):
    t = torch()
    return t.from_numpy(np.ascontiguousarray(a)).to("cuda")


def field_from_host(lat, q: np.ndarray, parity: int, prec: int):
    """Host API-layout spinor array (V, 12) -> device field of one parity."""
    aos = to_dev(q)
    f = dev_bytes(lat.spinor_bytes(prec))
    lat.spinor_import(aos, parity, f, prec)
    return f


def field_to_host(lat, f, prec: int, parity: int) -> np.ndarray:
    """Device field of one parity -> (V, 12) host array with that half set."""
    t = torch()
    aos = t.zeros((lat.V, 12), dtype=t.complex128, device="cuda")
    lat.spinor_export(f, prec, parity, aos)
    lat.synchronize()
    return aos.cpu().numpy()


def relmax(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
