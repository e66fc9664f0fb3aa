"""ctypes mirror of include/hpvcd_gpu.h and the library loaders.

The structs here must match the C header byte for byte; tests/test_abi.py
checks every size and field offset against the compiled library's own
`sizeof` report.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

LIB_PATH = os.path.join(HERE, "libhpvcd_b200.so")
SYNTH_PATH = os.path.join(HERE, "libhpvcd_synth.so")

# status codes (hpvcd_status)
OK = 0
ERR_BITSTREAM = 1
ERR_ALLOC = 2
ERR_LIMIT = 3
ERR_UNSUPPORTED = 4
ERR_TIMEOUT = 5
ERR_CUDA = 6
ERR_INVALID_ARG = 7
ERR_BUSY = 8

STATUS_NAMES = {
    OK: "OK",
    ERR_BITSTREAM: "Bitstream",
    ERR_ALLOC: "AllocationFailed",
    ERR_LIMIT: "LimitExceeded",
    ERR_UNSUPPORTED: "Unsupported",
    ERR_TIMEOUT: "Timeout",
    ERR_CUDA: "Cuda",
    ERR_INVALID_ARG: "InvalidArgument",
    ERR_BUSY: "Busy",
}

TU_CBF, TU_TSKIP, TU_INTRA, TU_TQB = 0x01, 0x02, 0x04, 0x08
TU_ROTATE, TU_RDPCM_H, TU_RDPCM_V, TU_PCM = 0x10, 0x20, 0x40, 0x80
CELL_EXEMPT = 0x01
CELL_INTER = 0x02
PU_L0, PU_L1 = 0x01, 0x02
MAX_REFS = 16

PIC_STRONG_SMOOTHING = 0x0001
PIC_SMOOTHING_DISABLED = 0x0002
PIC_DEBLOCK = 0x0004
PIC_SAO_LUMA = 0x0008
PIC_SAO_CHROMA = 0x0010
PIC_PRED_IN_PLANE = 0x0020
PIC_INTER = 0x0040
PIC_CROSS_COMPONENT = 0x0080
PIC_SAO_NO_ACROSS_SLICES = 0x0100
PIC_SAO_NO_ACROSS_TILES = 0x0200
PIC_CONSTRAINED_INTRA = 0x0400
PIC_PCM = 0x0800
PIC_COEFF8 = 0x1000
PIC_STORE_MASK = 0x00FF0000


def PIC_STORE_DPB(e: int) -> int:
    """hpvcd_picture.flags bits storing the decoded picture into DPB entry e."""
    return (e + 1) << 16


def REF_DPB(e: int) -> int:
    """hpvcd_picture.ref_slot value naming DPB entry e."""
    return -2 - e


DPB_MAX_READERS = 64

OUT_YUV, OUT_RGB8, OUT_YUV_CANVAS = 0, 1, 2
MATRIX_IDENTITY, MATRIX_BT709, MATRIX_BT470BG = 0, 1, 5
MATRIX_SMPTE170M, MATRIX_YCGCO, MATRIX_BT2020NCL = 6, 8, 9
CANVAS_NATIVE = 0x100  # hpvcd_canvas.matrix: native YCbCr planes on an RGB8 output
OUTPUT_CANVAS_ONLY = 0x1  # hpvcd_output.options: RGB8 canvases only, final planes not kept

STAGE_RECON, STAGE_DEBLOCK, STAGE_SAO, STAGE_OUTPUT = 0x1, 0x2, 0x4, 0x8
STAGE_ALL = 0xF
STAGE_GRAPH = 0x100

# Schedule selector network (include/hpvcd_gpu.h).
FEATURES = 16
MLP_HIDDEN = 64
MLP_MAX_VARIANTS = 32
MLP_NO_PICK = 0xFFFFFFFF

# Fixed per-device scratch of hpvcd_decode_noalloc (bytes).
NOALLOC_SCRATCH_BYTES = 12 * 1024 * 1024 + 256 * 1024

SYNTH_RESIDUAL, SYNTH_INTRA, SYNTH_INTER = 0, 1, 2


class HpvcdError(RuntimeError):
    """Error raised for a non-zero hpvcd_status (maps to the reference's DecodeError)."""

    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)} ({status})")


class Tu(C.Structure):
    _fields_ = [
        ("x", C.c_uint16), ("y", C.c_uint16), ("coeff_off", C.c_uint32),
        ("log2n", C.c_uint8), ("comp", C.c_uint8), ("flags", C.c_uint8), ("mode", C.c_uint8),
        ("qp_y", C.c_int8), ("cqp_off", C.c_int8), ("nx", C.c_uint8), ("res_scale", C.c_int8),
    ]


TU_DTYPE = np.dtype([
    ("x", "<u2"), ("y", "<u2"), ("coeff_off", "<u4"), ("log2n", "u1"), ("comp", "u1"),
    ("flags", "u1"), ("mode", "u1"), ("qp_y", "i1"), ("cqp_off", "i1"), ("nx", "u1"), ("res_scale", "i1"),
])


PU_DTYPE = np.dtype([
    ("x", "<u2"), ("y", "<u2"), ("w", "<u2"), ("h", "<u2"), ("mv", "<i2", (2, 2)), ("ref_idx", "i1", (2,)),
    ("flags", "u1"), ("rsvd", "u1"),
])


class Cell(C.Structure):
    _fields_ = [("bs_v", C.c_uint8), ("bs_h", C.c_uint8), ("qp_y", C.c_int8), ("flags", C.c_uint8)]


CELL_DTYPE = np.dtype([("bs_v", "u1"), ("bs_h", "u1"), ("qp_y", "i1"), ("flags", "u1")])


class SaoComp(C.Structure):
    _fields_ = [
        ("type_idx", C.c_uint8), ("band_pos", C.c_uint8), ("eo_class", C.c_uint8),
        ("rsvd", C.c_uint8), ("offsets", C.c_int16 * 4),
    ]


class SaoCtb(C.Structure):
    _fields_ = [("comp", SaoComp * 3)]


SAO_DTYPE = np.dtype([("comp", [("type_idx", "u1"), ("band_pos", "u1"), ("eo_class", "u1"),
                                ("rsvd", "u1"), ("offsets", "<i2", (4,))], (3,))])


class Pu(C.Structure):
    _fields_ = [
        ("x", C.c_uint16), ("y", C.c_uint16), ("w", C.c_uint16), ("h", C.c_uint16),
        ("mv", (C.c_int16 * 2) * 2), ("ref_idx", C.c_int8 * 2), ("flags", C.c_uint8),
        ("rsvd", C.c_uint8),
    ]


class WpEntry(C.Structure):
    _fields_ = [("luma_w", C.c_int16), ("luma_o", C.c_int16), ("cb_w", C.c_int16),
                ("cb_o", C.c_int16), ("cr_w", C.c_int16), ("cr_o", C.c_int16)]


class WpTable(C.Structure):
    _fields_ = [("luma_log2_denom", C.c_uint8), ("chroma_log2_denom", C.c_uint8),
                ("rsvd", C.c_uint8 * 2), ("e", (WpEntry * MAX_REFS) * 2)]


class Picture(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("chroma_idc", C.c_uint8), ("bit_depth_y", C.c_uint8), ("bit_depth_c", C.c_uint8),
        ("log2_ctb", C.c_uint8), ("flags", C.c_uint32),
        ("beta_offset_div2", C.c_int8), ("tc_offset_div2", C.c_int8),
        ("pps_cb_qp_offset", C.c_int8), ("pps_cr_qp_offset", C.c_int8),
        ("n_tus", C.c_uint32), ("n_pus", C.c_uint32), ("n_coeffs", C.c_uint64),
        ("tus", C.c_void_p), ("ctu_tu_start", C.c_void_p), ("coeffs", C.c_void_p),
        ("cells", C.c_void_p), ("sao", C.c_void_p), ("pus", C.c_void_p), ("wp", C.c_void_p),
        ("ref_slot", (C.c_int32 * MAX_REFS) * 2),
        ("pred", C.c_void_p * 3),
        ("scaling", C.c_void_p),
        ("ctb_region", C.c_void_p),
        ("slice_deblock", C.c_void_p),
    ]


class Scaling(C.Structure):
    _fields_ = [("m", ((C.c_uint8 * 64) * 6) * 4), ("dc", (C.c_uint8 * 6) * 4)]


class TilePlace(C.Structure):
    _fields_ = [("dst_x", C.c_uint32), ("dst_y", C.c_uint32), ("crop_w", C.c_uint32),
                ("crop_h", C.c_uint32), ("canvas", C.c_uint32)]


ORIENT_NORMAL, ORIENT_FLIP_H, ORIENT_ROTATE180, ORIENT_FLIP_V = 1, 2, 3, 4
ORIENT_TRANSPOSE, ORIENT_ROTATE90, ORIENT_TRANSVERSE, ORIENT_ROTATE270 = 5, 6, 7, 8


class Canvas(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("matrix", C.c_uint32),
                ("full_range", C.c_uint32), ("orientation", C.c_uint32)]


class Output(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("matrix", C.c_uint32), ("full_range", C.c_uint32),
                ("canvas_w", C.c_uint32), ("canvas_h", C.c_uint32), ("place", C.c_void_p),
                ("host_dst", C.c_void_p), ("host_dst_bytes", C.c_uint64),
                ("n_canvases", C.c_uint32), ("canvases", C.c_void_p), ("canvas_dst", C.c_void_p),
                ("orientation", C.c_uint32), ("options", C.c_uint32)]


class ServerCfg(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_inflight", C.c_uint32), ("max_batch_pictures", C.c_uint32),
                ("max_batch_bytes", C.c_uint64), ("hbm_budget", C.c_uint64), ("batching", C.c_uint32),
                ("batch_window_us", C.c_uint32)]


class Request(C.Structure):
    _fields_ = [("pics", C.c_void_p), ("n_pics", C.c_uint32), ("place", C.c_void_p),
                ("canvas", Canvas), ("dst", C.c_void_p), ("dst_bytes", C.c_uint64), ("user", C.c_uint64),
                ("flags", C.c_uint32)]


REQ_ZERO_COPY = 0x1


class Completion(C.Structure):
    _fields_ = [("user", C.c_uint64), ("status", C.c_int32), ("batch_pictures", C.c_uint32),
                ("latency_ms", C.c_double), ("queue_ms", C.c_double)]


class GpuCfg(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_inflight", C.c_uint32), ("hbm_budget", C.c_uint64)]


class Sched(C.Structure):
    _fields_ = [("idct", C.c_uint32), ("chroma_warps", C.c_uint32),
                ("recon_ctas_per_sm", C.c_uint32), ("wave", C.c_uint32)]


class SynthCfg(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64), ("width", C.c_uint32), ("height", C.c_uint32),
        ("kind", C.c_uint32), ("chroma_idc", C.c_uint32), ("bit_depth", C.c_uint32),
        ("log2_ctb", C.c_uint32), ("pic_flags", C.c_uint32),
        ("cu_split_p", C.c_float), ("tu_split_p", C.c_float), ("cbf_p", C.c_float),
        ("zero_frac", C.c_float), ("laplace_scale", C.c_float), ("tskip_p", C.c_float),
        ("tqb_p", C.c_float), ("sao_p", C.c_float),
        ("qp_min", C.c_int32), ("qp_max", C.c_int32),
        ("beta_offset_div2", C.c_int32), ("tc_offset_div2", C.c_int32),
        ("cb_qp_offset", C.c_int32), ("cr_qp_offset", C.c_int32),
        ("intra_cu_p", C.c_float), ("bi_p", C.c_float), ("mv_sd", C.c_float),
        ("mv_pad", C.c_float), ("weighted", C.c_uint32), ("n_refs", C.c_uint32),
        ("tu_mix", C.c_float * 4),
        ("scaling", C.c_uint32), ("rext", C.c_uint32), ("tskip_log2_max", C.c_uint32),
        ("ccp_p", C.c_float), ("regions", C.c_uint32), ("pcm_p", C.c_float),
        ("bitstream", C.c_uint32), ("sign_hiding", C.c_uint32),
    ]


# include/hpvcd_syntax.h
SLICE_TSKIP = 0x0001
SLICE_TQ_BYPASS = 0x0002
SLICE_CU_QP_DELTA = 0x0004
SLICE_SIGN_HIDING = 0x0008
SLICE_SAO_LUMA = 0x0010
SLICE_SAO_CHROMA = 0x0020
SLICE_DEBLOCK = 0x0040
SLICE_STRONG_SMOOTHING = 0x0080
SLICE_EBSP = 0x0100


class SliceParams(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("chroma_idc", C.c_uint8), ("bit_depth_y", C.c_uint8), ("bit_depth_c", C.c_uint8),
        ("log2_ctb", C.c_uint8), ("log2_min_cb", C.c_uint8), ("log2_min_tb", C.c_uint8),
        ("log2_max_tb", C.c_uint8), ("max_th_depth_intra", C.c_uint8),
        ("diff_cu_qp_delta_depth", C.c_uint8), ("log2_max_tskip", C.c_uint8),
        ("pps_cb_qp_offset", C.c_int8), ("pps_cr_qp_offset", C.c_int8),
        ("slice_qp", C.c_int8), ("slice_cb_qp_offset", C.c_int8), ("slice_cr_qp_offset", C.c_int8),
        ("beta_offset_div2", C.c_int8), ("tc_offset_div2", C.c_int8), ("rsvd", C.c_uint8 * 3),
        ("flags", C.c_uint32), ("scaling", C.c_void_p),
    ]


def _load(path: str, what: str) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(
            f"{what} not built: {path} is missing (run `python -c 'import __graft_entry__ as g; g.build()'`)"
        )
    return C.CDLL(path)


_lib = None
_synth = None


def lib() -> C.CDLL:
    """The CUDA back end (libhpvcd_b200.so).  Raises ImportError when it is not built."""
    global _lib
    if _lib is None:
        L = _load(LIB_PATH, "CUDA back end")
        vp, u32, i32, u64 = C.c_void_p, C.c_uint32, C.c_int32, C.c_uint64
        sig = {
            "hpvcd_abi_version": (u32, []),
            "hpvcd_status_string": (C.c_char_p, [C.c_int]),
            "hpvcd_kernel_launch_count": (u64, []),
            "hpvcd_last_error_string": (C.c_char_p, []),
            "hpvcd_gpu_create": (i32, [C.POINTER(GpuCfg), C.POINTER(vp)]),
            "hpvcd_gpu_destroy": (i32, [vp]),
            "hpvcd_gpu_submit": (i32, [vp, C.POINTER(Picture), u32, C.POINTER(Output), C.POINTER(u64)]),
            "hpvcd_gpu_wait": (i32, [vp, u64, i32]),
            "hpvcd_gpu_output_size": (i32, [vp, u64, C.POINTER(u64)]),
            "hpvcd_gpu_read": (i32, [vp, u64, vp, u64]),
            "hpvcd_plan_create": (i32, [C.POINTER(Picture), u32, C.POINTER(Output), C.POINTER(Sched), C.POINTER(vp)]),
            "hpvcd_plan_destroy": (i32, [vp]),
            "hpvcd_plan_launch": (i32, [vp, u32, vp]),
            "hpvcd_plan_planes": (i32, [vp, u32, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
            "hpvcd_plan_canvas": (i32, [vp, C.POINTER(vp), C.POINTER(u64)]),
            "hpvcd_plan_device_status": (i32, [vp, vp]),
            "hpvcd_plan_launches_per_run": (u32, [vp]),
            "hpvcd_abi_sizeof": (u64, [C.c_char_p]),
            "hpvcd_copy": (i32, [vp, vp, u64, vp]),
            "hpvcd_gpu_packed_size": (u64, [C.POINTER(Picture), u32]),
            "hpvcd_server_create": (i32, [C.POINTER(ServerCfg), C.POINTER(vp)]),
            "hpvcd_server_submit": (i32, [vp, C.POINTER(Request)]),
            "hpvcd_server_poll": (u32, [vp, C.POINTER(Completion), u32, i32]),
            "hpvcd_server_pending": (u32, [vp]),
            "hpvcd_server_destroy": (i32, [vp]),
            "hpvcd_gpu_pack_inputs": (i32, [C.POINTER(Picture), u32, vp, u64, C.POINTER(Picture)]),
            "hpvcd_decode_noalloc": (i32, [C.POINTER(Picture), C.POINTER(vp), vp, vp]),
            "hpvcd_plan_set_sched": (i32, [vp, C.POINTER(Sched)]),
            "hpvcd_plan_set_wait_test": (i32, [vp, u32, i32]),
            "hpvcd_plan_features": (i32, [vp, u32, u32, vp, vp]),
            "hpvcd_plan_autotune": (i32, [vp, C.POINTER(Sched), u32, u32, u32, u32, vp, C.POINTER(C.c_float),
                                          C.POINTER(u32)]),
            "hpvcd_plan_select": (i32, [vp, vp, C.POINTER(Sched), u32, vp, C.POINTER(u32)]),
            "hpvcd_mlp_create": (i32, [u32, u64, C.POINTER(vp)]),
            "hpvcd_mlp_destroy": (i32, [vp]),
            "hpvcd_mlp_param_count": (u32, [vp]),
            "hpvcd_mlp_variants": (u32, [vp]),
            "hpvcd_mlp_get_params": (i32, [vp, vp, C.c_int]),
            "hpvcd_mlp_set_params": (i32, [vp, vp]),
            "hpvcd_mlp_forward": (i32, [vp, vp, u32, vp, vp]),
            "hpvcd_mlp_grad": (i32, [vp, vp, vp, u32, vp, vp, vp]),
            "hpvcd_mlp_adam_step": (i32, [vp, C.c_float, vp]),
            "hpvcd_mlp_train": (i32, [vp, vp, vp, u32, u32, u32, C.c_float, u64, vp, C.POINTER(C.c_float)]),
            "hpvcd_mlp_pick": (i32, [vp, vp, u32, vp, C.POINTER(u32)]),
            "hpvcd_mlp_set_domain": (i32, [vp, vp, vp]),
            "hpvcd_gpu_set_selector": (i32, [vp, vp, C.POINTER(Sched), u32]),
            "hpvcd_gpu_selector_picks": (i32, [vp, C.POINTER(u64), u32]),
            "hpvcd_gpu_set_sched": (i32, [vp, C.POINTER(Sched)]),
            "hpvcd_server_set_selector": (i32, [vp, vp, C.POINTER(Sched), u32]),
            "hpvcd_server_selector_picks": (i32, [vp, C.POINTER(u64), u32]),
            "hpvcd_batch_features": (i32, [C.POINTER(Picture), u32, C.POINTER(C.c_float)]),
            "hpvcd_dpb_create": (i32, [i32, u32, C.POINTER(vp)]),
            "hpvcd_dpb_destroy": (i32, [vp]),
            "hpvcd_gpu_set_dpb": (i32, [vp, vp]),
            "hpvcd_syntax_decode": (i32, [C.POINTER(SliceParams), vp, u64, C.POINTER(vp)]),
            "hpvcd_syntax_decode_batch": (i32, [u32, C.POINTER(SliceParams), C.POINTER(vp), C.POINTER(u64), u32,
                                                C.POINTER(vp), C.POINTER(i32)]),
            "hpvcd_syntax_picture": (i32, [vp, C.POINTER(Picture)]),
            "hpvcd_syntax_bins": (u64, [vp]),
            "hpvcd_syntax_free": (None, [vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def synth_lib() -> C.CDLL:
    """The host-only synthetic input generator (libhpvcd_synth.so)."""
    global _synth
    if _synth is None:
        L = _load(SYNTH_PATH, "synthetic generator")
        L.hpvcd_synth_default_cfg.argtypes = [C.POINTER(SynthCfg)]
        L.hpvcd_synth_default_cfg.restype = None
        L.hpvcd_synth_new.restype = C.c_void_p
        L.hpvcd_synth_new.argtypes = []
        L.hpvcd_synth_free.argtypes = [C.c_void_p]
        L.hpvcd_synth_free.restype = None
        L.hpvcd_synth_add.argtypes = [C.c_void_p, C.POINTER(SynthCfg)]
        L.hpvcd_synth_add.restype = C.c_int32
        L.hpvcd_synth_count.argtypes = [C.c_void_p]
        L.hpvcd_synth_count.restype = C.c_uint32
        L.hpvcd_synth_get.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(Picture)]
        L.hpvcd_synth_get.restype = C.c_int32
        L.hpvcd_synth_slice.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(SliceParams),
                                        C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]
        L.hpvcd_synth_slice.restype = C.c_int32
        _synth = L
    return _synth


def check(status: int, what: str) -> None:
    if status != OK:
        detail = ""
        if status == ERR_CUDA and _lib is not None:
            detail = " [" + (_lib.hpvcd_last_error_string() or b"").decode(errors="replace") + "]"
        raise HpvcdError(status, what + detail)
