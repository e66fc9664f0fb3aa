"""ctypes bindings of the CPU oracle (test infrastructure only).

The oracle is a scalar C++ restatement of the hpvcd (Rust) reconstruction
path (oracle/hpvcd_oracle.cpp).  Only tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py use it, always as the checker or the timed CPU
reference, never as the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from hpvcd_b200 import abi  # noqa: E402

_lib = None

i32, u32, vp = C.c_int32, C.c_uint32, C.c_void_p


class DequantParams(C.Structure):
    _fields_ = [("factor", C.c_int64), ("add", C.c_int64), ("shift", C.c_int32), ("pad", C.c_int32),
                ("clip_min", C.c_int64), ("clip_max", C.c_int64)]


class TsParams(C.Structure):
    _fields_ = [("dq", DequantParams), ("tr_add", C.c_int32), ("tr_shift", C.c_int32)]


class Planes(C.Structure):
    _fields_ = [("y", vp), ("cb", vp), ("cr", vp)]


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "_build", "libhpvcd_oracle.so")
        if not os.path.exists(path):
            from oracle import build_oracle
            build_oracle.build()
        L = C.CDLL(path)
        L.orc_max_log2_tr_range.restype = i32
        L.orc_dct_matrix_entry.restype = i32
        for name in ("orc_normalize_luma_offset", "orc_derive_chroma_offset", "orc_qp_prime",
                     "orc_qpc", "orc_clamp_qpy", "orc_deblock_luma_segment",
                     "orc_recon_picture", "orc_mc_picture", "orc_deblock_picture",
                     "orc_sao_picture", "orc_decode_batch"):
            getattr(L, name).restype = i32
        L.orc_decode_batch.argtypes = [C.POINTER(abi.Picture), u32, C.POINTER(abi.Output),
                                       C.POINTER(Planes), vp, i32]
        L.orc_recon_picture.argtypes = [C.POINTER(abi.Picture), C.POINTER(Planes)]
        L.orc_deblock_picture.argtypes = [C.POINTER(abi.Picture), C.POINTER(Planes)]
        L.orc_sao_picture.argtypes = [C.POINTER(abi.Picture), C.POINTER(Planes)]
        L.orc_mc_picture.argtypes = [C.POINTER(abi.Picture), C.POINTER(Planes), i32, C.POINTER(Planes)]
        L.orc_set_disabled_slices.argtypes = [vp]
        L.orc_set_disabled_slices.restype = None
        L.orc_decode_grid_reference.argtypes = [C.POINTER(abi.Picture), u32, C.POINTER(abi.Output), vp, i32, i32]
        L.orc_decode_grid_reference.restype = i32
        _lib = L
    return _lib


def set_disabled_slices(slices) -> None:
    """Slice indexes whose deblocking is disabled in later oracle decodes
    (decode.rs:1934 / :1979 / :2060 `sd.disabled`); None or [] clears."""
    flags = np.zeros(256, np.uint8)
    for s in slices or ():
        flags[s] = 1
    lib().orc_set_disabled_slices(_p(flags) if flags.any() else None)


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def dequant_params(n, qp_prime, bd, ext=False) -> DequantParams:
    p = DequantParams()
    lib().orc_dequant_params_get(i32(n), i32(qp_prime), i32(bd), i32(int(ext)), C.byref(p))
    return p


def ts_params(n, qp_prime, bd, ext=False) -> TsParams:
    p = TsParams()
    lib().orc_ts_params_get(i32(n), i32(qp_prime), i32(bd), i32(int(ext)), C.byref(p))
    return p


def dequant(levels, n, params, scaling=None, dc=16, i16=False, ts=False) -> np.ndarray:
    lv = np.ascontiguousarray(levels, dtype=np.int32)
    out = np.zeros(n * n, np.int32)
    sc = None if scaling is None else np.ascontiguousarray(scaling, dtype=np.uint8)
    fn = lib().orc_dequant_ts if ts else lib().orc_dequant
    fn(_p(lv), i32(n), C.byref(params), None if sc is None else _p(sc), i32(dc), i32(int(i16)), _p(out))
    return out


def rext_residual_ops(res, n, rotate=False, rdpcm=None, i16=False) -> np.ndarray:
    """decode.rs:8418-8446 on a copy of `res` (rdpcm: None, 0 horizontal, 1 vertical)."""
    r = np.ascontiguousarray(res, dtype=np.int32).reshape(-1).copy()
    lib().orc_rext_residual_ops(_p(r), i32(n), i32(int(rotate)), i32(-1 if rdpcm is None else rdpcm),
                                i32(int(i16)))
    return r


def scaling_select(scaling, comp, n, inter, tskip):
    """decode.rs:5874-5899: (first entry, DC) of the list a TB uses, or None
    for the flat scale.  `scaling` is an abi.Scaling."""
    first, dc = C.c_int32(), C.c_int32()
    ok = lib().orc_scaling_select(C.byref(scaling), i32(comp), i32(n), i32(int(inter)), i32(int(tskip)),
                                  C.byref(first), C.byref(dc))
    return (first.value, dc.value) if ok else None


def inv_dct(coeff, n, bd, max_range=15, nx=None, i16=False) -> np.ndarray:
    c = np.ascontiguousarray(coeff, dtype=np.int32).reshape(-1)
    out = np.zeros(n * n, np.int32)
    lib().orc_inv_dct(_p(c), i32(n), i32(bd), i32(max_range), i32(n if nx is None else nx),
                      i32(int(i16)), _p(out))
    return out


def inv_dst4(coeff, bd, max_range=15, i16=False) -> np.ndarray:
    c = np.ascontiguousarray(coeff, dtype=np.int32).reshape(-1)
    out = np.zeros(16, np.int32)
    lib().orc_inv_dst4(_p(c), i32(bd), i32(max_range), i32(int(i16)), _p(out))
    return out


def dct_matrix(n) -> np.ndarray:
    return np.array([[lib().orc_dct_matrix_entry(n, k, m) for m in range(n)] for k in range(n)],
                    dtype=np.int64)


def narrow_i32_to_i16(src) -> np.ndarray:
    s = np.ascontiguousarray(src, dtype=np.int32)
    d = np.zeros(s.size, np.int16)
    lib().orc_narrow_i32_to_i16(_p(s), _p(d), i32(s.size))
    return d


def intra_filter(above, left, n, mode, is_luma, smoothing, strong, bd):
    a = np.ascontiguousarray(above, dtype=np.uint16)
    l_ = np.ascontiguousarray(left, dtype=np.uint16)
    fa = np.zeros(2 * n + 1, np.uint16)
    fl = np.zeros(2 * n + 1, np.uint16)
    lib().orc_intra_filter(_p(a), _p(l_), i32(n), i32(mode), i32(int(is_luma)), i32(int(smoothing)),
                           i32(int(strong)), i32(bd), _p(fa), _p(fl))
    return fa, fl


def intra_predict(mode, above, left, n, is_luma, bd) -> np.ndarray:
    a = np.ascontiguousarray(above, dtype=np.uint16)
    l_ = np.ascontiguousarray(left, dtype=np.uint16)
    out = np.zeros(n * n, np.uint16)
    lib().orc_intra_predict(i32(mode), _p(a), _p(l_), i32(n), i32(int(is_luma)), i32(bd), _p(out))
    return out


def intra_substitute(raw_above, raw_left, raw_corner, n, neutral):
    ra = np.ascontiguousarray(raw_above, dtype=np.int32)
    rl = np.ascontiguousarray(raw_left, dtype=np.int32)
    a = np.zeros(2 * n + 1, np.uint16)
    l_ = np.zeros(2 * n + 1, np.uint16)
    lib().orc_intra_substitute(_p(ra), _p(rl), i32(raw_corner), i32(n), i32(neutral), _p(a), _p(l_))
    return a, l_


def uni_mc_weighted(src, w, h, bd, weight, offset, log2_denom) -> np.ndarray:
    s = np.ascontiguousarray(src, dtype=np.int16)
    d = np.zeros(w * h, np.uint16)
    lib().orc_uni_mc_weighted(_p(s), i32(w), i32(h), i32(w), i32(h), i32(bd), i32(weight),
                              i32(offset), i32(log2_denom), _p(d), i32(w))
    return d


def bi_mc_weighted(s0, s1, w, h, bd, w0, o0, w1, o1, log2_denom) -> np.ndarray:
    a = np.ascontiguousarray(s0, dtype=np.int16)
    b = np.ascontiguousarray(s1, dtype=np.int16)
    d = np.zeros(w * h, np.uint16)
    lib().orc_bi_mc_weighted(_p(a), _p(b), i32(w), i32(h), i32(w), i32(h), i32(bd), i32(w0), i32(o0),
                             i32(w1), i32(o1), i32(log2_denom), _p(d), i32(w))
    return d


def luma_interp(ref, width, height, x0, y0, fx, fy, w, h, bd) -> np.ndarray:
    r = np.ascontiguousarray(ref, dtype=np.uint16)
    d = np.zeros(w * h, np.int16)
    lib().orc_luma_interp(_p(r), i32(width), i32(width), i32(height), i32(x0), i32(y0), i32(fx),
                          i32(fy), i32(w), i32(h), i32(bd), _p(d))
    return d


def chroma_interp(ref, width, height, x0, y0, fx, fy, w, h, bd) -> np.ndarray:
    r = np.ascontiguousarray(ref, dtype=np.uint16)
    d = np.zeros(w * h, np.int16)
    lib().orc_chroma_interp(_p(r), i32(width), i32(width), i32(height), i32(x0), i32(y0), i32(fx),
                            i32(fy), i32(w), i32(h), i32(bd), _p(d))
    return d


def apply_luma_decision(plane, stride, vertical, edge, scan, decision, tc, maxv) -> None:
    assert plane.dtype == np.uint16 and plane.flags["C_CONTIGUOUS"]
    lib().orc_apply_luma_decision(_p(plane), i32(stride), i32(int(vertical)), i32(edge), i32(scan),
                                  i32(decision), i32(tc), i32(maxv))


def sao_edge(dst, src, w, h, x0, y0, x_end, y_end, offsets, eo_class, bd) -> None:
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    lib().orc_sao_edge(_p(dst), _p(src), i32(w), i32(h), i32(x0), i32(y0), i32(x_end), i32(y_end),
                       _p(off), i32(eo_class), i32(bd))


def yuv_to_rgb16(y, cb, cr, width, height, chroma_idc, bd, dw, dh, matrix, full_range,
                 crop_left=0, crop_top=0) -> np.ndarray:
    Y = np.ascontiguousarray(y, dtype=np.uint16)
    CB = np.ascontiguousarray(cb, dtype=np.uint16)
    CR = np.ascontiguousarray(cr, dtype=np.uint16)
    out = np.zeros(dw * dh * 3, np.uint16)
    lib().orc_yuv_to_rgb16(_p(Y), _p(CB), _p(CR), i32(width), i32(height), i32(chroma_idc), i32(bd),
                           i32(dw), i32(dh), i32(crop_left), i32(crop_top), i32(matrix),
                           i32(int(full_range)), _p(out))
    return out


def yuv_canvas_layout(pics, out):
    """Per canvas of a canvas output: (offset, width, height, chroma_idc,
    bytes per sample); RGB8 canvases have chroma_idc None and 3 bytes per
    pixel, native ones the format of their first picture."""
    n_c = out.n_canvases or 1
    cv = (abi.Canvas * out.n_canvases).from_address(out.canvases) if out.n_canvases else None
    place = (abi.TilePlace * len(pics)).from_address(out.place)
    res, off = [], 0
    for k in range(n_c):
        w, h = (cv[k].width, cv[k].height) if cv is not None else (out.canvas_w, out.canvas_h)
        matrix = cv[k].matrix if cv is not None else out.matrix
        if out.kind == abi.OUT_RGB8 and matrix != abi.CANVAS_NATIVE:
            res.append((off, w, h, None, 3))
            off += w * h * 3
            continue
        idc, bps = 0, 1
        for i, p in enumerate(pics):
            if place[i].canvas == k:
                idc, bps = p.chroma_idc, 1 if p.bit_depth_y <= 8 and p.bit_depth_c <= 8 else 2
                break
        sw = 2 if idc in (1, 2) else 1
        sh = 2 if idc == 1 else 1
        cw, ch = ((w + sw - 1) // sw, (h + sh - 1) // sh) if idc else (0, 0)
        res.append((off, w, h, idc, bps))
        off += (w * h + 2 * cw * ch) * bps
    return res, off


def yuv_canvas_bytes(pics, out) -> int:
    return yuv_canvas_layout(pics, out)[1]


def decode_batch(pics, out=None, want_planes=True, threads=1):
    """Oracle decode of a list of abi.Picture; returns (planes list, rgb canvas or None)."""
    n = len(pics)
    arr = (abi.Picture * n)(*pics)
    planes = []
    pl_arr = (Planes * n)()
    for i, p in enumerate(pics):
        w, h = p.width, p.height
        sw = 2 if p.chroma_idc in (1, 2) else 1   # SubWidthC
        sh = 2 if p.chroma_idc == 1 else 1        # SubHeightC
        cw, ch = ((w + sw - 1) // sw, (h + sh - 1) // sh) if p.chroma_idc else (0, 0)
        y = np.zeros((h, w), np.uint16)
        cb = np.zeros((ch, cw), np.uint16)
        cr = np.zeros((ch, cw), np.uint16)
        planes.append((y, cb, cr))
        if want_planes:
            pl_arr[i] = Planes(_p(y), _p(cb) if cb.size else None, _p(cr) if cr.size else None)
    rgb = None
    if out is not None and out.kind == abi.OUT_RGB8 and not out.n_canvases and out.matrix != abi.CANVAS_NATIVE:
        rot = out.orientation in (abi.ORIENT_ROTATE90, abi.ORIENT_ROTATE270)
        rgb = np.zeros((out.canvas_w, out.canvas_h, 3) if rot else (out.canvas_h, out.canvas_w, 3), np.uint8)
    elif out is not None and out.kind in (abi.OUT_RGB8, abi.OUT_YUV_CANVAS):
        rgb = np.zeros(yuv_canvas_bytes(pics, out), np.uint8)
    rc = lib().orc_decode_batch(arr, u32(n), C.byref(out) if out is not None else None,
                                pl_arr if want_planes else None,
                                _p(rgb) if rgb is not None else None, i32(threads))
    abi.check(rc, "orc_decode_batch")
    return planes, rgb


def canvas_bytes(out) -> int:
    """Bytes of the RGB8 canvases of an output description."""
    if out.n_canvases:
        cv = (abi.Canvas * out.n_canvases).from_address(out.canvases)
        return sum(c.width * c.height * 3 for c in cv)
    return out.canvas_w * out.canvas_h * 3


def decode_grid_reference(pics, out, threads: int, simd: bool, dst=None):
    """The reference's parallel CPU decode (grid-row jobs, banded filters and
    colour conversion on a work-stealing pool) of intra / residual tiles onto
    RGB8 canvases, with the scalar or the AVX2 kernels; returns the canvas
    bytes (into `dst` when given)."""
    n = len(pics)
    arr = (abi.Picture * n)(*pics)
    rgb = dst if dst is not None else np.zeros(canvas_bytes(out), np.uint8)
    rc = lib().orc_decode_grid_reference(arr, n, C.byref(out), _p(rgb), threads, int(simd))
    if rc != 0:
        raise abi.HpvcdError(rc, "orc_decode_grid_reference")
    return rgb
