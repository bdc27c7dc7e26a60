"""mars_b200: the Mars fractal codec's domain-range block search and decode on B200.

Python mirror of the reference's search-provider boundary (daleobrien/mars,
crates/mars-codec/src/encode.rs:530-602): `Context.search_provider(plane, params)` plays
the provider factory `make_search(&Contracted)`, and the returned `GpuSearch.search()` is
`SearchProvider::search` -- same request (row, col, size, shift), same outcome (winning
candidate or None, evals).  Everything runs through libmars_b200.so (include/mars_b200.h);
there is no CPU path: without a CUDA device the calls raise `MarsError`.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import build as _build

_HERE = os.path.dirname(os.path.abspath(__file__))

MARS_OK = 0
ERRORS = {-1: "EINVAL", -2: "ENODEV", -3: "ECUDA", -4: "ENOMEM", -5: "ENOTFOUND",
          -6: "ETIMEOUT", -7: "EFORMAT", -8: "EUNSUPPORTED"}


class MarsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    """EncodeParams (encode.rs:27-52)."""
    _fields_ = [
        ("min_size", C.c_uint32), ("max_size", C.c_uint32), ("shift", C.c_uint32),
        ("bits_alfa", C.c_uint32), ("bits_beta", C.c_uint32), ("zero_threshold", C.c_uint32),
        ("max_alfa", C.c_double), ("t_rms", C.c_double), ("has_lambda", C.c_int32),
        ("reserved", C.c_int32), ("lambda_", C.c_double),
    ]


class Options(C.Structure):
    """EncodeOptions (encode.rs:78-109): allowed modes, adaptive density, residual
    quantisation (LambdaAdaptive when residual_adaptive, else Fixed(residual_qstep), 0 = 8),
    the final walk's search method and rd_candidates (0/1 = the single winner)."""
    _fields_ = [("allowed_modes", C.c_uint8 * 4), ("adaptive_density", C.c_int32),
                ("residual_adaptive", C.c_int32), ("residual_qstep", C.c_float),
                ("method", C.c_int32), ("rd_candidates", C.c_uint32)]


# MethodName (crates/mars-search/src/lib.rs): the search provider of the final walk.
METHODS = {"exhaustive": 0, "fisher": 1}


class Header(C.Structure):
    """mars_format::Header: the ifs geometry plus the binary32 residual step (0 = 8)."""
    _fields_ = [(n, C.c_uint32) for n in (
        "bits_alfa", "bits_beta", "min_size", "max_size", "shift", "width", "height",
        "int_max_alfa")] + [("residual_qstep", C.c_float)]


class Counters(C.Structure):
    _fields_ = [("search_evals", C.c_uint64), ("warmup_evals", C.c_uint64)]


class RefineReport(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("loss_start", "loss_end", "psnr_plain",
                                          "psnr_refined")] + [
        (n, C.c_uint32) for n in ("steps", "improving_steps", "changed_leaves", "accepted")]


CANDIDATE_DTYPE = np.dtype([
    ("dom_row", "<u4"), ("dom_col", "<u4"), ("isometry", "<u4"), ("qalfa", "<u4"),
    ("qbeta", "<u4"), ("valid", "<u4"), ("rms", "<f8"), ("s0", "<i8"), ("s1_x4", "<i8"),
    ("s2_x16", "<i8"), ("t0", "<i8"), ("t1_x4", "<i8"), ("t2", "<i8")])
LEAF_DTYPE = np.dtype([(n, "<u4") for n in (
    "row", "col", "size", "mode", "qalfa", "qbeta", "isometry", "dom_row", "dom_col")] + [
    ("qgx", "<i4"), ("qgy", "<i4")])

# Every symbol include/mars_b200.h declares (tests check the library exports them all).
EXPORTS = (
    "mars_last_error", "mars_version", "mars_ctx_create", "mars_ctx_destroy",
    "mars_ctx_set_stream", "mars_ctx_launch_count", "mars_ctx_set_search_path",
    "mars_search_table_build",
    "mars_search_table_lookup", "mars_search_table_evals", "mars_search_table_exact_fits",
    "mars_search_table_free", "mars_search_blocks", "mars_search_blocks_device",
    "mars_search_nodes_device", "mars_encode", "mars_leaves_free", "mars_decode",
    "mars_ifs_parse", "mars_ifs_write", "mars_bytes_free", "mars_search_blocks_noalloc",
    "mars_decode_plan_create", "mars_decode_plan_run", "mars_decode_plan_free",
    "mars_format_write", "mars_format_read", "mars_entropy_encode", "mars_entropy_decode",
    "mars_residuals_free", "mars_indexed_table_build", "mars_ycbcr_device",
    "mars_rgb_from_ycbcr_device", "mars_downsample_box_device", "mars_upsample_nearest_device",
    "mars_mse_device", "mars_search_table_build_ranked", "mars_search_table_lookup_ranked",
    "mars_search_plan_create", "mars_search_plan_run", "mars_search_plan_run_device",
    "mars_indexed_plan_create",
    "mars_search_plan_table", "mars_search_plan_evals", "mars_search_plan_launches",
    "mars_search_plan_kernel_ms",
    "mars_search_plan_free", "mars_decode_until_stable", "mars_decode_plan_run_until_stable",
    "mars_zoom_leaves", "mars_encode_planned",
    "mars_refine_plan_create", "mars_refine_params", "mars_refine_forward",
    "mars_refine_backward", "mars_refine_run", "mars_refine_plan_free",
    "mars_search_blocks_cross_device", "mars_refine_domains",
)

_lib = None


def lib_path() -> str:
    return _build.LIB


def lib():
    """Load libmars_b200.so (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_build.LIB) or _build.stale():
        _build.build()
    L = C.CDLL(_build.LIB)
    P, vp, u32, u64, sz = C.POINTER, C.c_void_p, C.c_uint32, C.c_uint64, C.c_size_t
    L.mars_last_error.restype = C.c_char_p
    L.mars_version.restype = C.c_char_p
    L.mars_ctx_create.argtypes = [P(vp), C.c_int]
    L.mars_ctx_destroy.argtypes = [vp]
    L.mars_ctx_destroy.restype = None
    L.mars_ctx_set_stream.argtypes = [vp, vp]
    L.mars_ctx_launch_count.argtypes = [vp]
    L.mars_ctx_launch_count.restype = u64
    L.mars_ctx_set_search_path.argtypes = [vp, C.c_int32]
    L.mars_search_table_build.argtypes = [vp, vp, u32, u32, P(Params), C.c_int32, P(vp)]
    L.mars_indexed_table_build.argtypes = [vp, vp, u32, u32, P(Params), C.c_int32, C.c_int32,
                                           P(vp)]
    L.mars_search_table_lookup.argtypes = [vp, u32, u32, u32, u32, vp, P(u64)]
    L.mars_decode_until_stable.argtypes = [vp, P(Header), vp, sz, vp, sz, C.c_uint8, u32, vp,
                                            P(u32)]
    L.mars_decode_plan_run_until_stable.argtypes = [vp, C.c_uint8, u32, vp, P(u32)]
    L.mars_zoom_leaves.argtypes = [P(Header), vp, sz, C.c_double, P(Header), vp]
    L.mars_encode_planned.argtypes = [vp, vp, P(Options), P(Header), P(vp), P(sz), P(vp), P(sz),
                                      P(Counters)]
    L.mars_search_plan_create.argtypes = [vp, u32, u32, P(Params), P(vp)]
    L.mars_indexed_plan_create.argtypes = [vp, u32, u32, P(Params), C.c_int32, P(vp)]
    L.mars_search_plan_run.argtypes = [vp, vp, P(vp)]
    L.mars_search_plan_run_device.argtypes = [vp, vp]
    L.mars_search_plan_table.argtypes = [vp, P(vp)]
    L.mars_search_plan_evals.argtypes = [vp]
    L.mars_search_plan_evals.restype = u64
    L.mars_search_plan_launches.argtypes = [vp]
    L.mars_search_plan_launches.restype = u64
    L.mars_search_plan_kernel_ms.argtypes = [vp, C.POINTER(C.c_float)]
    L.mars_search_plan_free.argtypes = [vp]
    L.mars_search_plan_free.restype = None
    L.mars_search_table_build_ranked.argtypes = [vp, vp, u32, u32, P(Params), C.c_int32, u32, P(vp)]
    L.mars_search_table_lookup_ranked.argtypes = [vp, u32, u32, u32, u32, u32, vp, P(u32), P(u64)]
    L.mars_search_table_evals.argtypes = [vp]
    L.mars_search_table_evals.restype = u64
    L.mars_search_table_exact_fits.argtypes = [vp]
    L.mars_search_table_exact_fits.restype = u64
    L.mars_search_table_free.argtypes = [vp]
    L.mars_search_table_free.restype = None
    L.mars_search_blocks.argtypes = [vp, vp, u32, u32, u32, u32, P(Params), vp, vp, sz, vp, vp]
    L.mars_search_blocks_device.argtypes = [vp, vp, u32, u32, u32, u32, P(Params), vp, vp, sz, vp]
    L.mars_search_nodes_device.argtypes = [vp, vp, u32, u32, P(Params), vp, sz, P(sz), P(u64)]
    L.mars_search_blocks_noalloc.argtypes = [vp, u32, u32, u32, u32, P(Params), vp, vp, sz, vp, vp]
    L.mars_encode.argtypes = [vp, vp, u32, u32, P(Params), P(Options), P(Header), P(vp), P(sz),
                              P(vp), P(sz), P(Counters)]
    L.mars_leaves_free.argtypes = [vp]
    L.mars_leaves_free.restype = None
    L.mars_decode.argtypes = [vp, P(Header), vp, sz, vp, sz, u32, vp]
    L.mars_decode_plan_create.argtypes = [vp, P(Header), vp, sz, vp, sz, P(vp)]
    L.mars_decode_plan_run.argtypes = [vp, u32, vp]
    L.mars_decode_plan_free.argtypes = [vp]
    L.mars_decode_plan_free.restype = None
    L.mars_ifs_parse.argtypes = [vp, sz, P(Header), P(vp), P(sz)]
    L.mars_ifs_write.argtypes = [P(Header), vp, sz, P(vp), P(sz)]
    L.mars_bytes_free.argtypes = [vp]
    L.mars_bytes_free.restype = None
    L.mars_format_write.argtypes = [P(Header), vp, sz, vp, sz, P(vp), P(sz)]
    L.mars_format_read.argtypes = [vp, sz, P(Header), P(vp), P(sz), P(vp), P(sz)]
    L.mars_residuals_free.argtypes = [vp]
    L.mars_residuals_free.restype = None
    L.mars_ycbcr_device.argtypes = [vp, vp, vp, vp, sz, vp, vp, vp]
    L.mars_rgb_from_ycbcr_device.argtypes = [vp, vp, vp, vp, sz, vp, vp, vp]
    L.mars_downsample_box_device.argtypes = [vp, vp, u32, u32, vp]
    L.mars_upsample_nearest_device.argtypes = [vp, vp, u32, u32, vp, u32, u32]
    L.mars_mse_device.argtypes = [vp, vp, vp, sz, P(C.c_double)]
    fp, dp = P(C.c_float), P(C.c_double)
    L.mars_refine_plan_create.argtypes = [vp, P(Header), vp, sz, vp, sz, vp, P(vp)]
    L.mars_refine_params.argtypes = [vp, vp, vp]
    L.mars_refine_forward.argtypes = [vp, vp, vp, u32, C.c_double, vp, dp, P(u32)]
    L.mars_refine_backward.argtypes = [vp, u32, C.c_double, vp, vp, P(u32), dp]
    L.mars_refine_run.argtypes = [vp, u32, C.c_float, u32, vp, P(RefineReport)]
    L.mars_search_blocks_cross_device.argtypes = [vp, vp, vp, u32, u32, u32, u32, P(Params),
                                                  vp, vp, sz, vp]
    L.mars_refine_domains.argtypes = [vp, P(Params), P(Header), vp, sz, vp, sz, vp, u32, u32,
                                      vp, P(RefineReport)]
    L.mars_refine_plan_free.argtypes = [vp]
    L.mars_refine_plan_free.restype = None
    L.mars_entropy_encode.argtypes = [vp, sz, P(vp), P(sz)]
    L.mars_entropy_decode.argtypes = [vp, sz, vp, sz, vp]
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != MARS_OK:
        raise MarsError(rc, (lib().mars_last_error() or b"").decode())


def make_params(min_size=4, max_size=16, shift=4, bits_alfa=4, bits_beta=7, max_alfa=1.0,
                t_rms=8.0, zero_threshold=0, lam: Optional[float] = None) -> Params:
    """EncodeParams with the encmars defaults (crates/mars-cli/src/bin/encmars.rs:185-205)."""
    return Params(min_size, max_size, shift, bits_alfa, bits_beta, zero_threshold, max_alfa,
                  t_rms, 0 if lam is None else 1, 0, 0.0 if lam is None else float(lam))


def _plane(img) -> np.ndarray:
    a = np.ascontiguousarray(img, dtype=np.uint8)
    if a.ndim != 2:
        raise ValueError("a plane is a 2-D uint8 array")
    return a


@dataclass
class Candidate:
    """Candidate (encode.rs:236-244)."""
    dom_row: int
    dom_col: int
    isometry: int
    qalfa: int
    qbeta: int
    rms: float
    moments: tuple


@dataclass
class SearchOutcome:
    """SearchOutcome (encode.rs:543-546)."""
    candidate: Optional[Candidate]
    evals: int


class GpuSearch:
    """SearchProvider over a table the GPU filled for every node of one plane."""

    def __init__(self, ctx: "Context", handle: int, width: int, height: int):
        self._ctx = ctx
        self._h = C.c_void_p(handle)
        self.width, self.height = width, height

    def search_many(self, rows, cols, size: int, shift: int):
        """SearchProvider::search for many nodes of one size: (candidates, evals) arrays."""
        out = np.zeros(len(rows), dtype=CANDIDATE_DTYPE)
        evals = np.zeros(len(rows), dtype=np.uint64)
        ev = C.c_uint64()
        for i, (r, c) in enumerate(zip(rows, cols)):
            check(lib().mars_search_table_lookup(self._h, int(r), int(c), size, shift,
                                                 out[i:i + 1].ctypes.data, C.byref(ev)))
            evals[i] = ev.value
        return out, evals

    def search_candidates(self, row: int, col: int, size: int, shift: int, max_: int):
        """SearchProvider::search_candidates: (structured array of up to max_ candidates
        ascending by (rms, reference order), evals)."""
        out = np.zeros(max(max_, 1), dtype=CANDIDATE_DTYPE)
        n, ev = C.c_uint32(), C.c_uint64()
        check(lib().mars_search_table_lookup_ranked(self._h, row, col, size, shift, max_,
                                                    out.ctypes.data, C.byref(n), C.byref(ev)))
        return out[: n.value], ev.value

    def search(self, row: int, col: int, size: int, shift: int) -> SearchOutcome:
        out = np.zeros(1, dtype=CANDIDATE_DTYPE)
        ev = C.c_uint64()
        check(lib().mars_search_table_lookup(self._h, row, col, size, shift, out.ctypes.data,
                                             C.byref(ev)))
        c = out[0]
        if not c["valid"]:
            return SearchOutcome(None, ev.value)
        return SearchOutcome(Candidate(int(c["dom_row"]), int(c["dom_col"]), int(c["isometry"]),
                                       int(c["qalfa"]), int(c["qbeta"]), float(c["rms"]),
                                       tuple(int(c[k]) for k in ("s0", "s1_x4", "s2_x16", "t0",
                                                                 "t1_x4", "t2"))), ev.value)

    @property
    def evals(self) -> int:
        return lib().mars_search_table_evals(self._h)

    @property
    def exact_fits(self) -> int:
        return lib().mars_search_table_exact_fits(self._h)

    def close(self) -> None:
        if self._h:
            lib().mars_search_table_free(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One device context (a CUDA stream plus cached device memory)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().mars_ctx_create(C.byref(h), device))
        self._h = h
        self.device = device

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self) -> None:
        for plan in getattr(self, "_plans", {}).values():
            plan.close()
        self._plans = {}
        if self._h:
            lib().mars_ctx_destroy(self._h)
            self._h = C.c_void_p(None)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int) -> None:
        check(lib().mars_ctx_set_stream(self._h, C.c_void_p(stream_ptr)))

    def set_search_path(self, path: str) -> None:
        """'auto' (tensor cores wherever a level allows), 'simt' (CUDA cores only), 'boxes'
        (tensor cores, operand stages loaded as per-phase boxes, the 2x2 box folded into K
        at every size), 'fold' (tensor cores, the fold at every size instead of the
        split-digit contracted operand at sizes 16..64) or 'per_level' (tensor cores, one
        correlation launch per level instead of the all-levels persistent launch of search
        plans and tables)."""
        check(lib().mars_ctx_set_search_path(self._h, {"auto": 0, "simt": 1, "tc": 2,
                                                       "boxes": 3, "fold": 4,
                                                       "per_level": 5}[path]))

    @property
    def launches(self) -> int:
        return lib().mars_ctx_launch_count(self._h)

    def search_provider(self, img, params: Params, adaptive_density: bool = False,
                        method: str = "exhaustive", k: int = 1) -> GpuSearch:
        """The provider factory: ExhaustiveSearch (ranking the best k of every node when
        k > 1), or IndexedSearchProvider::build for a classified method ("fisher")."""
        a = _plane(img)
        h, w = a.shape
        t = C.c_void_p()
        if k != 1:
            if method != "exhaustive":
                raise ValueError("only the exhaustive search ranks candidates")
            check(lib().mars_search_table_build_ranked(self._h, a.ctypes.data, w, h,
                                                       C.byref(params), int(adaptive_density),
                                                       int(k), C.byref(t)))
        elif method == "exhaustive":
            check(lib().mars_search_table_build(self._h, a.ctypes.data, w, h, C.byref(params),
                                                int(adaptive_density), C.byref(t)))
        else:
            check(lib().mars_indexed_table_build(self._h, a.ctypes.data, w, h, C.byref(params),
                                                 int(adaptive_density), METHODS[method],
                                                 C.byref(t)))
        return GpuSearch(self, t.value, w, h)

    def search_plan(self, width: int, height: int, params: Params,
                    method: str = "exhaustive") -> "SearchPlan":
        """A graph-captured provider factory for repeated planes of one geometry
        (mars_indexed_plan_create; "fisher" for the classified search)."""
        h = C.c_void_p()
        check(lib().mars_indexed_plan_create(self._h, width, height, C.byref(params),
                                             METHODS[method], C.byref(h)))
        return SearchPlan(self, h.value, width, height)

    def search_blocks(self, img, size: int, shift: int, params: Params, rows, cols):
        """search_block for each (rows[i], cols[i]): (candidates, evals) arrays."""
        a = _plane(img)
        h, w = a.shape
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        cols = np.ascontiguousarray(cols, dtype=np.uint32)
        out = np.zeros(len(rows), dtype=CANDIDATE_DTYPE)
        ev = np.zeros(len(rows), dtype=np.uint64)
        check(lib().mars_search_blocks(self._h, a.ctypes.data, w, h, size, shift, C.byref(params),
                                       rows.ctypes.data, cols.ctypes.data, len(rows),
                                       out.ctypes.data, ev.ctypes.data))
        return out, ev

    def search_grid(self, img, size: int, shift: int, params: Params):
        a = _plane(img)
        h, w = a.shape
        rr, cc = np.meshgrid(np.arange(h // size) * size, np.arange(w // size) * size, indexing="ij")
        return self.search_blocks(a, size, shift, params, rr.ravel(), cc.ravel())

    def encode(self, img, params: Params, allowed_modes=(1, 0, 1, 0), adaptive_density=False,
               residual_adaptive=False, residual_qstep=0.0, method="exhaustive",
               rd_candidates=1):
        """encode_image_with_search with the GPU provider: (header, leaves, residuals,
        counters); `residuals` holds the levels of the mode-3 leaves, size*size each, in
        leaf order."""
        a = _plane(img)
        h, w = a.shape
        opts = Options((C.c_uint8 * 4)(*allowed_modes), int(adaptive_density),
                       int(residual_adaptive), float(residual_qstep), METHODS[method],
                       int(rd_candidates))
        return _encode_call(lambda *out: lib().mars_encode(
            self._h, a.ctypes.data, w, h, C.byref(params), C.byref(opts), *out))

    def encode_many(self, images, params: Params, workers: int = 3, **options):
        """encode() over many planes, `workers` at a time: the C ABI is thread-safe, so one
        plane's host walks overlap another's GPU search.  Exhaustive single-winner encodes
        without adaptive density go through a search plan per plane size."""
        from concurrent.futures import ThreadPoolExecutor
        planned = (options.get("method", "exhaustive") == "exhaustive"
                   and options.get("rd_candidates", 1) <= 1
                   and not (params.has_lambda and options.get("adaptive_density", False)))
        plans = {}
        if planned:
            for im in images:
                shape = _plane(im).shape
                if shape not in plans:
                    plans[shape] = self.cached_plan(shape[1], shape[0], params)
        modes = options.pop("allowed_modes", (1, 0, 1, 0))

        def one(im):
            if planned:
                return plans[_plane(im).shape].encode(
                    im, allowed_modes=modes,
                    residual_adaptive=options.get("residual_adaptive", False),
                    residual_qstep=options.get("residual_qstep", 0.0))
            return self.encode(im, params, allowed_modes=modes, **options)

        with ThreadPoolExecutor(max(1, workers)) as ex:
            return list(ex.map(one, images))

    def cached_plan(self, width: int, height: int, params: Params) -> "SearchPlan":
        """A search plan kept by the context for its lifetime, one per (size, params)."""
        key = (width, height, bytes(params))
        if not hasattr(self, "_plans"):
            self._plans = {}
        if key not in self._plans:
            self._plans[key] = self.search_plan(width, height, params)
        return self._plans[key]

    # ---- colour input and metric (device kernels; host arrays staged through torch) ----

    def _dev(self, arr):
        import torch
        return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.uint8).ravel()).to(
            f"cuda:{self.device}")

    def _convert(self, planes, inverse: bool):
        import torch
        a, b, c = (self._dev(p) for p in planes)
        outs = [torch.empty_like(a) for _ in range(3)]
        fn = lib().mars_rgb_from_ycbcr_device if inverse else lib().mars_ycbcr_device
        check(fn(self._h, a.data_ptr(), b.data_ptr(), c.data_ptr(), a.numel(),
                 outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr()))
        torch.cuda.synchronize()
        shape = np.asarray(planes[0]).shape
        return tuple(o.cpu().numpy().reshape(shape) for o in outs)

    def ycbcr(self, r, g, b):
        """metrics::ycbcr (crates/mars-core/src/metrics.rs:377-430): BT.601 full-range Y, Cb,
        Cr planes of three RGB planes."""
        return self._convert((r, g, b), False)

    def rgb_from_ycbcr(self, y, cb, cr):
        """metrics::rgb_from_ycbcr (metrics.rs:432-460)."""
        return self._convert((y, cb, cr), True)

    def downsample_box(self, plane):
        """color::downsample_box (crates/mars-codec/src/color.rs:60-83)."""
        import torch
        h, w = np.asarray(plane).shape
        src = self._dev(plane)
        dst = torch.empty(((h + 1) // 2) * ((w + 1) // 2), dtype=torch.uint8, device=src.device)
        check(lib().mars_downsample_box_device(self._h, src.data_ptr(), w, h, dst.data_ptr()))
        torch.cuda.synchronize()
        return dst.cpu().numpy().reshape((h + 1) // 2, (w + 1) // 2)

    def upsample_nearest(self, plane, width: int, height: int):
        """color::upsample_nearest (color.rs:85-101)."""
        import torch
        sh, sw = np.asarray(plane).shape
        src = self._dev(plane)
        dst = torch.empty(width * height, dtype=torch.uint8, device=src.device)
        check(lib().mars_upsample_nearest_device(self._h, src.data_ptr(), sw, sh, dst.data_ptr(),
                                                 width, height))
        torch.cuda.synchronize()
        return dst.cpu().numpy().reshape(height, width)

    def mse(self, a, b) -> float:
        """metrics::mse (metrics.rs:29-48): exact integer SSE / pixel count."""
        if np.asarray(a).shape != np.asarray(b).shape:
            raise ValueError("MSE requires identical dimensions")
        da, db = self._dev(a), self._dev(b)
        out = C.c_double()
        check(lib().mars_mse_device(self._h, da.data_ptr(), db.data_ptr(), da.numel(),
                                    C.byref(out)))
        return out.value

    def decode_plan(self, hdr: Header, leaves: np.ndarray, residuals=None) -> "DecodePlan":
        leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
        res = _residuals(residuals)
        h = C.c_void_p()
        check(lib().mars_decode_plan_create(self._h, C.byref(hdr), leaves.ctypes.data,
                                            len(leaves), res.ctypes.data, len(res), C.byref(h)))
        return DecodePlan(h.value)

    def refine_plan(self, hdr: Header, leaves: np.ndarray, target, residuals=None) -> "RefinePlan":
        """The attractor-refinement plan of a leaf list against its target plane."""
        leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
        res = _residuals(residuals)
        t = np.ascontiguousarray(target, dtype=np.uint8)
        if t.shape != (hdr.height, hdr.width):
            raise ValueError("the target must be a (height, width) plane")
        h = C.c_void_p()
        check(lib().mars_refine_plan_create(self._h, C.byref(hdr), leaves.ctypes.data,
                                            len(leaves), res.ctypes.data, len(res),
                                            t.ctypes.data, C.byref(h)))
        return RefinePlan(h.value, leaves, hdr)

    def refine_domains(self, params: Params, hdr: Header, leaves: np.ndarray, target,
                       residuals=None, passes: int = 3, decode_iterations: int = 12):
        """mars_refine_domains: -> (leaves, RefineReport).  Every mode-2 leaf is searched
        again with its range block from `target` and the domain pool from the decode of the
        current list; a pass is kept only when the exact decode improves."""
        leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
        res = _residuals(residuals)
        t = np.ascontiguousarray(target, dtype=np.uint8)
        if t.shape != (hdr.height, hdr.width):
            raise ValueError("the target must be a (height, width) plane")
        out = np.zeros(len(leaves), LEAF_DTYPE)
        rep = RefineReport()
        check(lib().mars_refine_domains(self._h, C.byref(params), C.byref(hdr),
                                        leaves.ctypes.data, len(leaves), res.ctypes.data,
                                        len(res), t.ctypes.data, passes, decode_iterations,
                                        out.ctypes.data, C.byref(rep)))
        return out, rep

    def decode_until_stable(self, hdr: Header, leaves: np.ndarray, threshold: int,
                            max_iterations: int, residuals=None):
        """decode_until_stable (ifs.rs:321-353): (plane, iterations used)."""
        leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
        res = _residuals(residuals)
        out = np.zeros((hdr.height, hdr.width), dtype=np.uint8)
        used = C.c_uint32()
        check(lib().mars_decode_until_stable(self._h, C.byref(hdr), leaves.ctypes.data,
                                             len(leaves), res.ctypes.data, len(res), threshold,
                                             max_iterations, out.ctypes.data, C.byref(used)))
        return out, used.value

    def decode(self, hdr: Header, leaves: np.ndarray, iterations: int = 10,
               residuals=None) -> np.ndarray:
        leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
        res = _residuals(residuals)
        out = np.zeros((hdr.height, hdr.width), dtype=np.uint8)
        check(lib().mars_decode(self._h, C.byref(hdr), leaves.ctypes.data, len(leaves),
                                res.ctypes.data, len(res), iterations, out.ctypes.data))
        return out


def _encode_call(call):
    """Runs a mars_encode-shaped call and returns (header, leaves, residuals, counters)."""
    hdr, cnt = Header(), Counters()
    ptr, n = C.c_void_p(), C.c_size_t()
    rptr, rn = C.c_void_p(), C.c_size_t()
    check(call(C.byref(hdr), C.byref(ptr), C.byref(n), C.byref(rptr), C.byref(rn),
               C.byref(cnt)))
    leaves = np.frombuffer(C.string_at(ptr, n.value * LEAF_DTYPE.itemsize),
                           dtype=LEAF_DTYPE).copy()
    resid = np.frombuffer(C.string_at(rptr, rn.value * 4), dtype=np.int32).copy()
    lib().mars_leaves_free(ptr)
    lib().mars_residuals_free(rptr)
    return hdr, leaves, resid, cnt


def _residuals(residuals) -> np.ndarray:
    return np.ascontiguousarray(residuals if residuals is not None else np.zeros(0),
                                dtype=np.int32)


class DecodePlan:
    """A leaf list prepared for repeated device decodes (mars_decode_plan_*)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    def run(self, iterations: int, d_out_ptr: int) -> None:
        check(lib().mars_decode_plan_run(self._h, iterations, C.c_void_p(d_out_ptr)))

    def close(self) -> None:
        if self._h:
            lib().mars_decode_plan_free(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SearchPlan:
    """mars_search_plan_*: every level of one plane's search as one CUDA-graph launch."""

    def __init__(self, ctx: "Context", handle: int, width: int, height: int):
        self._ctx = ctx
        self._h = C.c_void_p(handle)
        self.width, self.height = width, height

    @property
    def evals(self) -> int:
        return lib().mars_search_plan_evals(self._h)

    @property
    def launches(self) -> int:
        return lib().mars_search_plan_launches(self._h)

    @property
    def kernel_ms(self) -> float:
        """Device time of the last completed replay's all-levels correlation launch
        (mars_search_plan_kernel_ms)."""
        v = C.c_float()
        check(lib().mars_search_plan_kernel_ms(self._h, C.byref(v)))
        return v.value

    def run(self, img) -> GpuSearch:
        a = _plane(img)
        if a.shape != (self.height, self.width):
            raise ValueError("plane shape differs from the plan's")
        t = C.c_void_p()
        check(lib().mars_search_plan_run(self._h, a.ctypes.data, C.byref(t)))
        return GpuSearch(self._ctx, t.value, self.width, self.height)

    def run_device(self, d_plane_ptr: int) -> None:
        check(lib().mars_search_plan_run_device(self._h, C.c_void_p(d_plane_ptr)))

    def encode(self, img, allowed_modes=(1, 0, 1, 0), residual_adaptive=False,
               residual_qstep=0.0):
        """mars_encode_planned: (header, leaves, residuals, counters)."""
        a = _plane(img)
        if a.shape != (self.height, self.width):
            raise ValueError("plane shape differs from the plan's")
        opts = Options((C.c_uint8 * 4)(*allowed_modes), 0, int(residual_adaptive),
                       float(residual_qstep), 0, 1)
        return _encode_call(lambda *out: lib().mars_encode_planned(
            self._h, a.ctypes.data, C.byref(opts), *out))

    def table(self) -> GpuSearch:
        t = C.c_void_p()
        check(lib().mars_search_plan_table(self._h, C.byref(t)))
        return GpuSearch(self._ctx, t.value, self.width, self.height)

    def close(self) -> None:
        if self._h:
            lib().mars_search_plan_free(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefinePlan:
    """mars_refine_*: the decode map's fixed point and its adjoint gradient on the device."""

    def __init__(self, handle: int, leaves: np.ndarray, hdr: Header):
        self._h = C.c_void_p(handle)
        self.n = len(leaves)
        self.shape = (hdr.height, hdr.width)

    def params(self):
        """The leaves' dequantised (s, o) as float32 arrays."""
        s, o = np.zeros(self.n, np.float32), np.zeros(self.n, np.float32)
        check(lib().mars_refine_params(self._h, s.ctypes.data, o.ctypes.data))
        return s, o

    def forward(self, s, o, max_iters: int = 400, tol: float = 1e-4, want_x: bool = False):
        """-> (loss, iterations, x* or None)."""
        s = np.ascontiguousarray(s, np.float32)
        o = np.ascontiguousarray(o, np.float32)
        if len(s) != self.n or len(o) != self.n:
            raise ValueError("s and o need one value per leaf")
        x = np.zeros(self.shape, np.float32) if want_x else None
        loss, it = C.c_double(), C.c_uint32()
        check(lib().mars_refine_forward(self._h, s.ctypes.data, o.ctypes.data, max_iters, tol,
                                        x.ctypes.data if want_x else None, C.byref(loss),
                                        C.byref(it)))
        return loss.value, it.value, x

    def backward(self, max_iters: int = 400, tol: float = 1e-6):
        """-> (dL/ds, dL/do, iterations, relative residual) at the last forward's x*."""
        gs, go = np.zeros(self.n, np.float32), np.zeros(self.n, np.float32)
        it, res = C.c_uint32(), C.c_double()
        check(lib().mars_refine_backward(self._h, max_iters, tol, gs.ctypes.data, go.ctypes.data,
                                         C.byref(it), C.byref(res)))
        return gs, go, it.value, res.value

    def run(self, steps: int = 20, lr: float = 0.5, decode_iterations: int = 10):
        """-> (leaves, RefineReport): the refined list if it decodes better, else the input."""
        out = np.zeros(self.n, LEAF_DTYPE)
        rep = RefineReport()
        check(lib().mars_refine_run(self._h, steps, lr, decode_iterations, out.ctypes.data,
                                    C.byref(rep)))
        return out, rep

    def close(self) -> None:
        if self._h:
            lib().mars_refine_plan_free(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def zoom_leaves(hdr: Header, leaves: np.ndarray, factor: float):
    """zoom_leaves (ifs.rs:356-392): (zoomed header, zoomed leaves); mode-3 leaves come back
    as mode 2 at any factor but 1 (their residual is dropped)."""
    leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
    out = np.zeros(len(leaves), dtype=LEAF_DTYPE)
    h2 = Header()
    check(lib().mars_zoom_leaves(C.byref(hdr), leaves.ctypes.data, len(leaves), factor,
                                 C.byref(h2), out.ctypes.data))
    return h2, out


def ifs_parse(data: bytes):
    buf = np.frombuffer(data, dtype=np.uint8)
    hdr = Header()
    ptr, n = C.c_void_p(), C.c_size_t()
    check(lib().mars_ifs_parse(buf.ctypes.data, len(data), C.byref(hdr), C.byref(ptr), C.byref(n)))
    leaves = np.frombuffer(C.string_at(ptr, n.value * LEAF_DTYPE.itemsize), dtype=LEAF_DTYPE).copy()
    lib().mars_leaves_free(ptr)
    return hdr, leaves


EVENT_DTYPE = np.dtype([("field", "u1"), ("pad", "u1", 3), ("disambiguator", "<u4"),
                        ("alphabet", "<u4"), ("symbol", "<u4")])

LEGACY_QSTEP = 8.0


def qstep_from_lambda(lam: float) -> float:
    """ResidualQstep::from_lambda (crates/mars-codec/src/quant.rs:36-52), as binary32."""
    step = math.sqrt(max(lam, 0.0)) * math.sqrt(6.0 / math.log(2.0))
    return float(np.float32(min(max(step, 1.0), 65535.0)))


def format_write(hdr: Header, leaves: np.ndarray, residuals=None) -> bytes:
    """mars_format::write (mars_format.rs:232-300): the .mars v0 bytes of (hdr, leaves);
    the residual step is the header's (0 = 8)."""
    leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
    res = _residuals(residuals)
    ptr, n = C.c_void_p(), C.c_size_t()
    check(lib().mars_format_write(C.byref(hdr), leaves.ctypes.data, len(leaves), res.ctypes.data,
                                  len(res), C.byref(ptr), C.byref(n)))
    data = C.string_at(ptr, n.value)
    lib().mars_bytes_free(ptr)
    return data


def format_read(data: bytes):
    """mars_format::read (mars_format.rs:302-400) -> (header, leaves, residuals)."""
    buf = np.frombuffer(data, dtype=np.uint8)
    hdr = Header()
    ptr, n = C.c_void_p(), C.c_size_t()
    rptr, rn = C.c_void_p(), C.c_size_t()
    check(lib().mars_format_read(buf.ctypes.data, len(data), C.byref(hdr), C.byref(ptr),
                                 C.byref(n), C.byref(rptr), C.byref(rn)))
    leaves = np.frombuffer(C.string_at(ptr, n.value * LEAF_DTYPE.itemsize), dtype=LEAF_DTYPE).copy()
    resid = np.frombuffer(C.string_at(rptr, rn.value * 4), dtype=np.int32).copy()
    lib().mars_leaves_free(ptr)
    lib().mars_residuals_free(rptr)
    return hdr, leaves, resid


def entropy_encode(events) -> bytes:
    """mars_entropy::encode over (field, disambiguator, alphabet, symbol) tuples."""
    ev = np.zeros(len(events), EVENT_DTYPE)
    for i, (f, d, a, s) in enumerate(events):
        ev[i]["field"], ev[i]["disambiguator"], ev[i]["alphabet"], ev[i]["symbol"] = f, d, a, s
    ptr, n = C.c_void_p(), C.c_size_t()
    check(lib().mars_entropy_encode(ev.ctypes.data, len(ev), C.byref(ptr), C.byref(n)))
    data = C.string_at(ptr, n.value)
    lib().mars_bytes_free(ptr)
    return data


def entropy_decode(data: bytes, shape) -> list:
    """Decoder::next for each (field, disambiguator, alphabet) of `shape`, in order."""
    ev = np.zeros(len(shape), EVENT_DTYPE)
    for i, (f, d, a) in enumerate(shape):
        ev[i]["field"], ev[i]["disambiguator"], ev[i]["alphabet"] = f, d, a
    out = np.zeros(len(shape), np.uint32)
    buf = np.frombuffer(data, dtype=np.uint8)
    check(lib().mars_entropy_decode(buf.ctypes.data, len(data), ev.ctypes.data, len(ev),
                                    out.ctypes.data))
    return [int(x) for x in out]


def psnr_from_mse(mse: float) -> Optional[float]:
    """metrics::psnr_from_mse (metrics.rs:57-59): 10 log10(255^2 / mse); None when the planes
    are identical."""
    return 10.0 * math.log10(255.0 * 255.0 / mse) if mse > 0.0 else None


def ifs_write(hdr: Header, leaves: np.ndarray) -> bytes:
    leaves = np.ascontiguousarray(leaves, dtype=LEAF_DTYPE)
    ptr, n = C.c_void_p(), C.c_size_t()
    check(lib().mars_ifs_write(C.byref(hdr), leaves.ctypes.data, len(leaves), C.byref(ptr),
                               C.byref(n)))
    data = C.string_at(ptr, n.value)
    lib().mars_bytes_free(ptr)
    return data
