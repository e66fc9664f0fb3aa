"""The C ABI library loads, exports every entry point include/hpvcd_gpu.h
declares, and the ctypes structs match the C layout (no GPU needed)."""
import ctypes as C
import os
import re

from hpvcd_b200 import abi

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
HEADERS = [os.path.join(INCLUDE, h) for h in ("hpvcd_gpu.h", "hpvcd_syntax.h")]


def declared_functions():
    text = "".join(open(h).read() for h in HEADERS)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hpvcd_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("hpvcd_gpu_create", "hpvcd_gpu_submit", "hpvcd_gpu_wait", "hpvcd_gpu_read",
              "hpvcd_plan_create", "hpvcd_plan_launch"):
        assert n in names


def test_library_exports_every_declared_symbol():
    L = abi.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version_and_status_strings():
    L = abi.lib()
    assert L.hpvcd_abi_version() == 1
    assert b"bitstream" in L.hpvcd_status_string(abi.ERR_BITSTREAM)


def test_struct_layouts_match():
    L = abi.lib()
    pairs = {
        "hpvcd_tu": abi.Tu, "hpvcd_cell": abi.Cell, "hpvcd_sao_comp": abi.SaoComp,
        "hpvcd_sao_ctb": abi.SaoCtb, "hpvcd_pu": abi.Pu, "hpvcd_wp_entry": abi.WpEntry,
        "hpvcd_wp_table": abi.WpTable, "hpvcd_picture": abi.Picture,
        "hpvcd_tile_place": abi.TilePlace, "hpvcd_output": abi.Output,
        "hpvcd_gpu_cfg": abi.GpuCfg, "hpvcd_sched": abi.Sched, "hpvcd_canvas": abi.Canvas,
        "hpvcd_server_cfg": abi.ServerCfg, "hpvcd_request": abi.Request,
        "hpvcd_completion": abi.Completion, "hpvcd_scaling": abi.Scaling,
        "hpvcd_slice_params": abi.SliceParams,
    }
    for name, cls in pairs.items():
        assert L.hpvcd_abi_sizeof(name.encode()) == C.sizeof(cls), name
    assert abi.TU_DTYPE.itemsize == 16 and abi.CELL_DTYPE.itemsize == 4 and abi.SAO_DTYPE.itemsize == 36


def test_invalid_arguments_without_gpu():
    L = abi.lib()
    assert L.hpvcd_gpu_create(None, None) == abi.ERR_INVALID_ARG
    assert L.hpvcd_plan_launch(None, abi.STAGE_ALL, None) == abi.ERR_INVALID_ARG
    assert L.hpvcd_gpu_read(None, 1, None, 0) == abi.ERR_INVALID_ARG


def test_pack_inputs_through_the_copy_pool_is_exact():
    """hpvcd_gpu_pack_inputs spreads its copies over the host copy pool in
    1 MiB pieces (here: the 48 tiles of a 4032x3024 grid, ~27 MB); every part
    of every picture lands at its descriptor, byte for byte."""
    import numpy as np

    from hpvcd_b200 import synth
    g = synth.config1_grid(seed=3)
    pics = g.synth.pictures()
    keep = synth.narrow_coeffs(pics[:10])  # int8 pools for some, int16 for the rest
    L = abi.lib()
    arr = (abi.Picture * len(pics))(*pics)
    nb = L.hpvcd_gpu_packed_size(arr, len(pics))
    assert nb > 8 << 20
    buf = np.full(nb, 0xA5, np.uint8)
    out = (abi.Picture * len(pics))()
    assert L.hpvcd_gpu_pack_inputs(arr, len(pics), buf.ctypes.data_as(C.c_void_p), nb, out) == abi.OK
    lo, hi = buf.ctypes.data, buf.ctypes.data + nb
    for p, q in zip(pics, out):
        geo = synth.geometry(p)
        ctbs = geo["ctb_cols"] * geo["ctb_rows"]
        for name, n in (("tus", p.n_tus * C.sizeof(abi.Tu)), ("ctu_tu_start", (ctbs + 1) * 4),
                        ("coeffs", p.n_coeffs * (1 if p.flags & abi.PIC_COEFF8 else 2)),
                        ("cells", geo["gw"] * geo["gh"] * C.sizeof(abi.Cell)),
                        ("sao", ctbs * C.sizeof(abi.SaoCtb))):
            src, dst = getattr(p, name), getattr(q, name)
            if not n:
                continue
            src = C.cast(src, C.c_void_p).value
            dst = C.cast(dst, C.c_void_p).value
            assert lo <= dst and dst + n <= hi, name
            assert C.string_at(dst, n) == C.string_at(src, n), name
    del keep
