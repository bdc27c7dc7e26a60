"""ctypes wrapper for the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg as the parity checker; the product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


class Params(C.Structure):
    _fields_ = [
        ("min_size", C.c_uint32), ("max_size", C.c_uint32), ("shift", C.c_uint32),
        ("bits_alfa", C.c_uint32), ("bits_beta", C.c_uint32), ("zero_threshold", C.c_uint32),
        ("max_alfa", C.c_double), ("t_rms", C.c_double), ("has_lambda", C.c_int32),
        ("pad_", C.c_int32), ("lambda_", C.c_double),
    ]


class Options(C.Structure):
    _fields_ = [("allowed_modes", C.c_uint8 * 4), ("adaptive_density", C.c_int32),
                ("residual_adaptive", C.c_int32), ("residual_qstep", C.c_float),
                ("method", C.c_int32), ("rd_candidates", C.c_uint32)]


METHODS = {"exhaustive": 0, "fisher": 1}


class Moments(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("s0", "s1_x4", "s2_x16", "t0", "t1_x4", "t2")]


class Candidate(C.Structure):
    _fields_ = [
        ("dom_row", C.c_uint32), ("dom_col", C.c_uint32), ("isometry", C.c_uint32),
        ("qalfa", C.c_uint32), ("qbeta", C.c_uint32), ("valid", C.c_uint32),
        ("rms", C.c_double), ("m", Moments),
    ]


class Leaf(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in (
        "row", "col", "size", "mode", "qalfa", "qbeta", "isometry", "dom_row", "dom_col")] + [
        ("qgx", C.c_int32), ("qgy", C.c_int32)]


class Header(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in (
        "bits_alfa", "bits_beta", "min_size", "max_size", "shift", "width", "height",
        "int_max_alfa")] + [("residual_qstep", C.c_float)]


CANDIDATE_DTYPE = np.dtype([
    ("dom_row", "<u4"), ("dom_col", "<u4"), ("isometry", "<u4"), ("qalfa", "<u4"),
    ("qbeta", "<u4"), ("valid", "<u4"), ("rms", "<f8"), ("s0", "<i8"), ("s1_x4", "<i8"),
    ("s2_x16", "<i8"), ("t0", "<i8"), ("t1_x4", "<i8"), ("t2", "<i8")])
LEAF_DTYPE = np.dtype([(n, "<u4") for n in (
    "row", "col", "size", "mode", "qalfa", "qbeta", "isometry", "dom_row", "dom_col")] + [
    ("qgx", "<i4"), ("qgy", "<i4")])
assert CANDIDATE_DTYPE.itemsize == C.sizeof(Candidate)
assert LEAF_DTYPE.itemsize == C.sizeof(Leaf)

_lib = None


def build() -> None:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.POINTER
        L.orc_contract.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
        L.orc_fit_f64.argtypes = [P(Moments), C.c_double, C.c_uint32, C.c_uint32,
                                  P(C.c_uint32), P(C.c_uint32), P(C.c_double)]
        L.orc_best_beta.argtypes = [C.c_int64, C.c_int64, C.c_uint32]
        L.orc_best_beta.restype = C.c_uint32
        L.orc_search.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32,
                                 C.c_uint32, C.c_uint32, C.c_uint32, P(Params), C.c_uint32,
                                 C.c_void_p, P(C.c_uint32), P(C.c_uint64)]
        L.orc_search_grid.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                      P(Params), C.c_void_p, C.c_void_p, C.c_int]
        L.orc_search_blocks.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                        C.c_uint32, P(Params), C.c_void_p, C.c_void_p, C.c_size_t,
                                        C.c_void_p, C.c_void_p, C.c_int]
        L.orc_fisher_search_blocks.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                               C.c_uint32, P(Params), C.c_void_p, C.c_void_p,
                                               C.c_size_t, C.c_void_p, C.c_void_p, C.c_int]
        L.orc_fisher_classify_domains.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                                  C.c_uint32, C.c_void_p, C.c_void_p]
        L.orc_encode.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, P(Params), P(Options),
                                 P(Header), P(C.c_void_p), P(C.c_size_t), P(C.c_void_p),
                                 P(C.c_size_t), P(C.c_uint64), P(C.c_uint64), C.c_int]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_decode.argtypes = [P(Header), C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                 C.c_uint32, C.c_void_p]
        L.orc_ycbcr.argtypes = [C.c_void_p] * 3 + [C.c_size_t] + [C.c_void_p] * 3
        L.orc_rgb_from_ycbcr.argtypes = [C.c_void_p] * 3 + [C.c_size_t] + [C.c_void_p] * 3
        L.orc_downsample_box.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
        L.orc_upsample_nearest.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                           C.c_uint32, C.c_uint32]
        L.orc_mse.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.orc_mse.restype = C.c_double
        L.orc_forward_dct2d.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
        L.orc_inverse_dct2d.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
        L.orc_dead_zone_quantize.argtypes = [C.c_double, C.c_double, C.c_double]
        L.orc_dead_zone_quantize.restype = C.c_int32
        L.orc_dead_zone_dequantize.argtypes = [C.c_int32, C.c_double, C.c_double]
        L.orc_dead_zone_dequantize.restype = C.c_double
        L.orc_ifs_parse.argtypes = [C.c_void_p, C.c_size_t, P(Header), P(C.c_void_p),
                                    P(C.c_size_t)]
        L.orc_ifs_write.argtypes = [P(Header), C.c_void_p, C.c_size_t, P(C.c_void_p),
                                    P(C.c_size_t)]
        L.orc_leaf_bits.argtypes = [P(Header), C.c_void_p, C.c_size_t, P(Leaf)]
        L.orc_leaf_bits.restype = C.c_double
        L.orc_decode_until_stable.argtypes = [P(Header), C.c_void_p, C.c_size_t, C.c_void_p,
                                              C.c_size_t, C.c_uint8, C.c_uint32, C.c_void_p,
                                              P(C.c_uint32)]
        L.orc_zoom_leaves.argtypes = [P(Header), C.c_void_p, C.c_size_t, C.c_double, P(Header),
                                      C.c_void_p]
        L.orc_refine_params.argtypes = [P(Header), C.c_void_p, C.c_size_t, C.c_void_p,
                                        C.c_void_p]
        L.orc_refine_eval.argtypes = [P(Header), C.c_void_p, C.c_size_t, C.c_void_p,
                                      C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_uint32, C.c_uint32, C.c_void_p, P(C.c_double),
                                      C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def make_params(min_size=4, max_size=16, shift=4, bits_alfa=4, bits_beta=7, max_alfa=1.0,
                t_rms=8.0, zero_threshold=0, lam=None) -> Params:
    return Params(min_size, max_size, shift, bits_alfa, bits_beta, zero_threshold, max_alfa,
                  t_rms, 0 if lam is None else 1, 0, 0.0 if lam is None else float(lam))


def _u8(img: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(img, dtype=np.uint8)
    assert a.ndim == 2
    return a


def contract(img: np.ndarray) -> np.ndarray:
    a = _u8(img)
    h, w = a.shape
    out = np.zeros((h // 2, w // 2), dtype=np.int32)
    lib().orc_contract(a.ctypes.data, w, h, out.ctypes.data)
    return out


def fit_f64(s0, s1_x4, s2_x16, t0, t1_x4, t2, max_alfa=1.0, bits_alfa=4, bits_beta=7):
    m = Moments(s0, s1_x4, s2_x16, t0, t1_x4, t2)
    qa, qb, rms = C.c_uint32(), C.c_uint32(), C.c_double()
    lib().orc_fit_f64(C.byref(m), max_alfa, bits_alfa, bits_beta, C.byref(qa), C.byref(qb),
                      C.byref(rms))
    return qa.value, qb.value, rms.value


def best_beta(range_sum: int, pixel_count: int, bits_beta: int = 7) -> int:
    return lib().orc_best_beta(range_sum, pixel_count, bits_beta)


def search(img, row, col, size, shift, params: Params, k=1, contracted=None):
    """search_top_k for one block: (candidates structured array, evals).  `contracted` (the
    (h/2, w/2) int32 contraction of another plane of the same size) replaces the domain pool
    of `img`'s own contraction: ranges from `img`, domains from that plane."""
    a = _u8(img)
    h, w = a.shape
    cd = None
    if contracted is not None:
        cd = np.ascontiguousarray(contracted, dtype=np.int32)
        if cd.shape != (h // 2, w // 2):
            raise ValueError("the contracted plane must be (h/2, w/2)")
    out = np.zeros(k, dtype=CANDIDATE_DTYPE)
    n, ev = C.c_uint32(), C.c_uint64()
    rc = lib().orc_search(a.ctypes.data, w, h, None if cd is None else cd.ctypes.data, row, col,
                          size, shift, C.byref(params), k, out.ctypes.data, C.byref(n),
                          C.byref(ev))
    if rc:
        raise ValueError(f"orc_search failed: {rc}")
    return out[: n.value], ev.value


def search_grid(img, size, shift, params: Params, nthreads=0):
    """search_block over every aligned size x size block, row-major."""
    a = _u8(img)
    h, w = a.shape
    nb = (h // size) * (w // size)
    out = np.zeros(nb, dtype=CANDIDATE_DTYPE)
    ev = np.zeros(nb, dtype=np.uint64)
    rc = lib().orc_search_grid(a.ctypes.data, w, h, size, shift, C.byref(params), out.ctypes.data,
                               ev.ctypes.data, nthreads)
    if rc:
        raise ValueError(f"orc_search_grid failed: {rc}")
    return out, ev


def search_blocks(img, size, shift, params: Params, rows, cols, nthreads=0):
    a = _u8(img)
    h, w = a.shape
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    out = np.zeros(len(rows), dtype=CANDIDATE_DTYPE)
    ev = np.zeros(len(rows), dtype=np.uint64)
    rc = lib().orc_search_blocks(a.ctypes.data, w, h, size, shift, C.byref(params),
                                 rows.ctypes.data, cols.ctypes.data, len(rows), out.ctypes.data,
                                 ev.ctypes.data, nthreads)
    if rc:
        raise ValueError(f"orc_search_blocks failed: {rc}")
    return out, ev


def fisher_search_blocks(img, size, shift, params: Params, rows, cols, nthreads=0):
    """Fisher::index at (size, shift), then Fisher::candidates + search_block_fitted per block:
    (candidates, evals per block)."""
    a = _u8(img)
    h, w = a.shape
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    out = np.zeros(len(rows), dtype=CANDIDATE_DTYPE)
    ev = np.zeros(len(rows), dtype=np.uint64)
    rc = lib().orc_fisher_search_blocks(a.ctypes.data, w, h, size, shift, C.byref(params),
                                        rows.ctypes.data, cols.ctypes.data, len(rows),
                                        out.ctypes.data, ev.ctypes.data, nthreads)
    if rc:
        raise ValueError(f"orc_fisher_search_blocks failed: {rc}")
    return out, ev


def fisher_classify_domains(img, size, shift):
    """(bucket, isometry) of every domain position at (size, shift), raster order."""
    a = _u8(img)
    h, w = a.shape
    n = ((h - 2 * size) // shift + 1) * ((w - 2 * size) // shift + 1)
    bucket = np.zeros(n, np.uint8)
    iso = np.zeros(n, np.uint8)
    rc = lib().orc_fisher_classify_domains(a.ctypes.data, w, h, size, shift, bucket.ctypes.data,
                                           iso.ctypes.data)
    if rc:
        raise ValueError(f"orc_fisher_classify_domains failed: {rc}")
    return bucket, iso


def encode(img, params: Params, allowed_modes=(1, 0, 1, 0), adaptive_density=False, nthreads=0,
           residual_adaptive=False, residual_qstep=0.0, method="exhaustive", rd_candidates=1):
    """encode_image_with_search with ExhaustiveSearch (or the Fisher provider):
    (header, leaves, residuals, search_evals, warmup_evals); `residuals` holds the levels of
    the mode-3 leaves, size*size each, in leaf order."""
    a = _u8(img)
    h, w = a.shape
    opts = Options((C.c_uint8 * 4)(*allowed_modes), int(adaptive_density), int(residual_adaptive),
                   float(residual_qstep), METHODS[method], int(rd_candidates))
    hdr = Header()
    ptr, n = C.c_void_p(), C.c_size_t()
    rptr, rn = C.c_void_p(), C.c_size_t()
    sev, wev = C.c_uint64(), C.c_uint64()
    rc = lib().orc_encode(a.ctypes.data, w, h, C.byref(params), C.byref(opts), C.byref(hdr),
                          C.byref(ptr), C.byref(n), C.byref(rptr), C.byref(rn), C.byref(sev),
                          C.byref(wev), nthreads)
    if rc:
        raise ValueError(f"orc_encode failed: {rc}")
    leaves = np.frombuffer(C.string_at(ptr, n.value * LEAF_DTYPE.itemsize), dtype=LEAF_DTYPE).copy()
    resid = np.frombuffer(C.string_at(rptr, rn.value * 4), dtype=np.int32).copy()
    lib().orc_free(ptr)
    lib().orc_free(rptr)
    return hdr, leaves, resid, sev.value, wev.value


def decode(hdr: Header, leaves: np.ndarray, iterations: int = 10, residuals=None) -> np.ndarray:
    leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
    res = np.ascontiguousarray(residuals if residuals is not None else np.zeros(0), dtype=np.int32)
    out = np.zeros((hdr.height, hdr.width), dtype=np.uint8)
    rc = lib().orc_decode(C.byref(hdr), leaves.ctypes.data, len(leaves), res.ctypes.data, len(res),
                          iterations, out.ctypes.data)
    if rc:
        raise ValueError(f"orc_decode failed: {rc}")
    return out


def _convert(fn, planes):
    a, b, c = (np.ascontiguousarray(p, dtype=np.uint8) for p in planes)
    outs = [np.empty_like(a) for _ in range(3)]
    fn(a.ctypes.data, b.ctypes.data, c.ctypes.data, a.size, *[o.ctypes.data for o in outs])
    return tuple(outs)


def ycbcr(r, g, b):
    return _convert(lib().orc_ycbcr, (r, g, b))


def rgb_from_ycbcr(y, cb, cr):
    return _convert(lib().orc_rgb_from_ycbcr, (y, cb, cr))


def downsample_box(plane):
    a = _u8(plane)
    h, w = a.shape
    out = np.empty(((h + 1) // 2, (w + 1) // 2), np.uint8)
    lib().orc_downsample_box(a.ctypes.data, w, h, out.ctypes.data)
    return out


def upsample_nearest(plane, width, height):
    a = _u8(plane)
    sh, sw = a.shape
    out = np.empty((height, width), np.uint8)
    lib().orc_upsample_nearest(a.ctypes.data, sw, sh, out.ctypes.data, width, height)
    return out


def mse(a, b) -> float:
    x, y = _u8(a), _u8(b)
    assert x.shape == y.shape
    return float(lib().orc_mse(x.ctypes.data, y.ctypes.data, x.size))


def forward_dct2d(block: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(block, dtype=np.float64)
    out = np.empty_like(b)
    lib().orc_forward_dct2d(b.ctypes.data, b.shape[0], out.ctypes.data)
    return out


def inverse_dct2d(coeffs: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    out = np.empty_like(c)
    lib().orc_inverse_dct2d(c.ctypes.data, c.shape[0], out.ctypes.data)
    return out


def dead_zone_quantize(x: float, step: float, dz: float) -> int:
    return int(lib().orc_dead_zone_quantize(x, step, dz))


def dead_zone_dequantize(level: int, step: float, dz: float) -> float:
    return float(lib().orc_dead_zone_dequantize(level, step, dz))


def ifs_parse(data: bytes):
    buf = np.frombuffer(data, dtype=np.uint8)
    hdr = Header()
    ptr, n = C.c_void_p(), C.c_size_t()
    rc = lib().orc_ifs_parse(buf.ctypes.data, len(data), C.byref(hdr), C.byref(ptr), C.byref(n))
    if rc:
        raise ValueError(f"orc_ifs_parse failed: {rc}")
    leaves = np.frombuffer(C.string_at(ptr, n.value * LEAF_DTYPE.itemsize), dtype=LEAF_DTYPE).copy()
    lib().orc_free(ptr)
    return hdr, leaves


def ifs_write(hdr: Header, leaves: np.ndarray) -> bytes:
    leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
    ptr, n = C.c_void_p(), C.c_size_t()
    rc = lib().orc_ifs_write(C.byref(hdr), leaves.ctypes.data, len(leaves), C.byref(ptr),
                             C.byref(n))
    if rc:
        raise ValueError(f"orc_ifs_write failed: {rc}")
    data = C.string_at(ptr, n.value)
    lib().orc_free(ptr)
    return data


def pgm_bytes(img: np.ndarray) -> bytes:
    h, w = img.shape
    return b"P5\n%d %d\n255\n" % (w, h) + np.ascontiguousarray(img, dtype=np.uint8).tobytes()


def refine_params(hdr: Header, leaves: np.ndarray):
    """The leaves' dequantised (s, o) in f64 (s = 0 without a domain, both 0 for mode 1)."""
    leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
    s, o = np.zeros(len(leaves)), np.zeros(len(leaves))
    lib().orc_refine_params(C.byref(hdr), leaves.ctypes.data, len(leaves), s.ctypes.data,
                            o.ctypes.data)
    return s, o


def refine_eval(hdr: Header, leaves: np.ndarray, target, s, o, residuals=None,
                fwd_iters: int = 600, adj_iters: int = 600):
    """The refinement model in f64: (loss, x*, dL/ds, dL/do) after fwd_iters forward steps
    from the flat-128 seed and adj_iters adjoint steps from zero."""
    leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
    res = np.ascontiguousarray(residuals if residuals is not None else np.zeros(0), dtype=np.int32)
    t = np.ascontiguousarray(target, dtype=np.uint8)
    s = np.ascontiguousarray(s, dtype=np.float64)
    o = np.ascontiguousarray(o, dtype=np.float64)
    x = np.zeros((hdr.height, hdr.width))
    gs, go = np.zeros(len(leaves)), np.zeros(len(leaves))
    loss = C.c_double()
    rc = lib().orc_refine_eval(C.byref(hdr), leaves.ctypes.data, len(leaves), res.ctypes.data,
                               len(res), t.ctypes.data, s.ctypes.data, o.ctypes.data, fwd_iters,
                               adj_iters, x.ctypes.data, C.byref(loss), gs.ctypes.data,
                               go.ctypes.data)
    if rc:
        raise ValueError(f"orc_refine_eval failed: {rc}")
    return loss.value, x, gs, go


def decode_until_stable(hdr: Header, leaves: np.ndarray, threshold: int, max_iterations: int,
                        residuals=None):
    """decode_until_stable (ifs.rs:321-343): (plane, iterations used)."""
    leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
    res = np.ascontiguousarray(residuals if residuals is not None else np.zeros(0), dtype=np.int32)
    out = np.zeros((hdr.height, hdr.width), dtype=np.uint8)
    used = C.c_uint32()
    rc = lib().orc_decode_until_stable(C.byref(hdr), leaves.ctypes.data, len(leaves),
                                       res.ctypes.data, len(res), threshold, max_iterations,
                                       out.ctypes.data, C.byref(used))
    if rc:
        raise ValueError(f"orc_decode_until_stable failed: {rc}")
    return out, used.value


def zoom_leaves(hdr: Header, leaves: np.ndarray, factor: float):
    """zoom_leaves (ifs.rs:370-392): (zoomed header, zoomed leaves)."""
    leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
    out = np.zeros(len(leaves), dtype=LEAF_DTYPE)
    h2 = Header()
    lib().orc_zoom_leaves(C.byref(hdr), leaves.ctypes.data, len(leaves), factor, C.byref(h2),
                          out.ctypes.data)
    return h2, out
