"""Colour encode/decode over the library: the host side of crates/mars-codec/src/color.rs.

`encode_color` follows encode_color_image_with_residual_quantisation (color.rs:400-490)
without lambda regions or chroma desaturation: BT.601 full-range Y/Cb/Cr on the device
(metrics.rs:377-430), 4:2:0 box-downsampled chroma (color.rs:60-83) unless 4:4:4 is asked
for, each plane encoded with the GPU search provider (Y with the luma parameters, Cb/Cr with
the chroma ones), written as .mars v0 streams and wrapped in the MARC container
(color.rs:369-373, 778-829).  `decode_color` is decode_color_image (color.rs:492-528):
per-plane GPU decodes, nearest-neighbour chroma upsampling and the inverse transform.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

from . import (Context, Params, format_read, format_write, zoom_leaves)

COLOR_MAGIC = b"MARC"
COLOR_VERSION = 0
MODE_GRAY, MODE_RGB_444, MODE_RGB_420 = 0, 1, 2


def write_container(mode: int, streams) -> bytes:
    """write_container (color.rs:778-790): magic, version, mode, count, (u32 length, bytes)*."""
    out = bytearray(COLOR_MAGIC + bytes([COLOR_VERSION, mode, len(streams)]))
    for s in streams:
        out += struct.pack("<I", len(s)) + s
    return bytes(out)


def read_container(data: bytes):
    """read_container (color.rs:792-829) -> (mode, streams); ValueError on malformed input."""
    if len(data) < 7:
        raise ValueError("truncated")
    if data[:4] != COLOR_MAGIC:
        raise ValueError("bad magic")
    if data[4] != COLOR_VERSION:
        raise ValueError(f"unsupported version {data[4]}")
    mode, count, off, streams = data[5], data[6], 7, []
    for _ in range(count):
        if off + 4 > len(data):
            raise ValueError("truncated")
        (n,) = struct.unpack_from("<I", data, off)
        off += 4
        if off + n > len(data):
            raise ValueError(f"section claims {n} bytes but only {len(data) - off} remain")
        streams.append(bytes(data[off:off + n]))
        off += n
    return mode, streams


@dataclass
class ColorEncodeParams:
    """ColorEncodeParams without regions: luma and chroma EncodeParams, 4:2:0 or 4:4:4."""
    y: Params
    chroma: Params
    subsampling: str = "420"
    allowed_modes: tuple = (1, 1, 1, 1)
    adaptive_density: bool = False
    residual_adaptive: bool = False
    residual_qstep: float = 0.0
    method: str = "exhaustive"


@dataclass
class ColorEncodeStats:
    y_bytes: int = 0
    cb_bytes: int = 0
    cr_bytes: int = 0
    y_evals: int = 0
    cb_evals: int = 0
    cr_evals: int = 0
    planes: dict = field(default_factory=dict)


def _encode_plane(ctx: Context, plane, params: Params, p: ColorEncodeParams):
    hdr, leaves, res, cnt = ctx.encode(plane, params, allowed_modes=p.allowed_modes,
                                       adaptive_density=p.adaptive_density,
                                       residual_adaptive=p.residual_adaptive,
                                       residual_qstep=p.residual_qstep, method=p.method)
    return format_write(hdr, leaves, res), cnt.search_evals


def encode_color(ctx: Context, image: np.ndarray, p: ColorEncodeParams):
    """An (h, w) gray or (h, w, 3) RGB uint8 image -> (MARC bytes, stats)."""
    img = np.ascontiguousarray(image, dtype=np.uint8)
    stats = ColorEncodeStats()
    if img.ndim == 2:
        data, stats.y_evals = _encode_plane(ctx, img, p.y, p)
        stats.y_bytes = len(data)
        return write_container(MODE_GRAY, [data]), stats
    y, cb, cr = ctx.ycbcr(img[..., 0], img[..., 1], img[..., 2])
    if p.subsampling == "420":
        mode, cb, cr = MODE_RGB_420, ctx.downsample_box(cb), ctx.downsample_box(cr)
    elif p.subsampling == "444":
        mode = MODE_RGB_444
    else:
        raise ValueError("subsampling is '420' or '444'")
    # The planes are independent encodes; the C ABI is thread-safe, so one plane's host
    # walks overlap another's search on the device.
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(3) as pool:
        jobs = [pool.submit(_encode_plane, ctx, pl, prm, p)
                for pl, prm in ((y, p.y), (cb, p.chroma), (cr, p.chroma))]
        (yb, stats.y_evals), (cbb, stats.cb_evals), (crb, stats.cr_evals) = [j.result() for j in jobs]
    stats.y_bytes, stats.cb_bytes, stats.cr_bytes = len(yb), len(cbb), len(crb)
    stats.planes = {"y": y, "cb": cb, "cr": cr}
    return write_container(mode, [yb, cbb, crb]), stats


def _decode_planes(ctx: Context, data: bytes, iterations: int, zoom: float, threshold):
    mode, streams = read_container(data)
    planes, used = [], 0
    for s in streams:
        hdr, leaves, res = format_read(s)
        if zoom != 1.0:
            hdr, leaves = zoom_leaves(hdr, leaves, zoom)
            res = None  # zoom_leaves drops the residuals (its mode-3 leaves became mode 2)
        if threshold is None:
            planes.append(ctx.decode(hdr, leaves, iterations, res))
            used = iterations
        else:
            plane, n = ctx.decode_until_stable(hdr, leaves, threshold, iterations, res)
            planes.append(plane)
            used = max(used, n)
    return mode, planes, used


def _assemble(ctx: Context, mode: int, planes):
    if mode == MODE_GRAY:
        return planes[0]
    if mode not in (MODE_RGB_444, MODE_RGB_420) or len(planes) != 3:
        raise ValueError(f"unknown mode {mode}")
    y, cb, cr = planes
    h, w = y.shape
    if mode == MODE_RGB_420:
        cb, cr = ctx.upsample_nearest(cb, w, h), ctx.upsample_nearest(cr, w, h)
    r, g, b = ctx.rgb_from_ycbcr(y, cb, cr)
    return np.stack([r, g, b], axis=-1)


def decode_color_zoomed(ctx: Context, data: bytes, iterations: int, zoom: float) -> np.ndarray:
    """decode_color_image_zoomed (color.rs:530-573): every plane's leaves zoomed
    (zoom_leaves) before the decode."""
    mode, planes, _ = _decode_planes(ctx, data, iterations, zoom, None)
    return _assemble(ctx, mode, planes)


def decode_color_auto(ctx: Context, data: bytes, threshold: int, max_iterations: int,
                      zoom: float = 1.0):
    """decode_color_image_auto (color.rs:575-629): each plane decoded until stable; returns
    (image, the largest plane's iteration count)."""
    mode, planes, used = _decode_planes(ctx, data, max_iterations, zoom, threshold)
    return _assemble(ctx, mode, planes), used


def decode_color(ctx: Context, data: bytes, iterations: int = 10) -> np.ndarray:
    """decode_color_image (color.rs:492-528): gray (h, w) or RGB (h, w, 3)."""
    mode, streams = read_container(data)
    planes = []
    for s in streams:
        hdr, leaves, res = format_read(s)
        planes.append(ctx.decode(hdr, leaves, iterations, res))
    if mode == MODE_GRAY:
        return planes[0]
    if mode not in (MODE_RGB_444, MODE_RGB_420) or len(planes) != 3:
        raise ValueError(f"unknown mode {mode}")
    y, cb, cr = planes
    h, w = y.shape
    if mode == MODE_RGB_420:
        cb, cr = ctx.upsample_nearest(cb, w, h), ctx.upsample_nearest(cr, w, h)
    r, g, b = ctx.rgb_from_ycbcr(y, cb, cr)
    return np.stack([r, g, b], axis=-1)
