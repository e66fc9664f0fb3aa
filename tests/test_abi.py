"""The C ABI library loads, exports every entry point include/hpvcd_gpu.h
declares, and the ctypes structs match the C layout (no GPU needed)."""
import ctypes as C
import os
import re

from hpvcd_b200 import abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "hpvcd_gpu.h")


def declared_functions():
    text = open(HEADER).read()
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
    }
    for name, cls in pairs.items():
        assert L.hpvcd_abi_sizeof(name.encode()) == C.sizeof(cls), name
    assert abi.TU_DTYPE.itemsize == 16 and abi.CELL_DTYPE.itemsize == 4 and abi.SAO_DTYPE.itemsize == 36


def test_invalid_arguments_without_gpu():
    L = abi.lib()
    assert L.hpvcd_gpu_create(None, None) == abi.ERR_INVALID_ARG
    assert L.hpvcd_plan_launch(None, abi.STAGE_ALL, None) == abi.ERR_INVALID_ARG
    assert L.hpvcd_gpu_read(None, 1, None, 0) == abi.ERR_INVALID_ARG
