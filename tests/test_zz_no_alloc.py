"""hpvcd_decode_noalloc: one picture decoded with no allocation, its scratch in
a fixed array of the library's device memory, against the plan entry point
(hpvcd_plan_create / hpvcd_plan_launch) on the same device-resident inputs.

Integer reconstruction: the tolerance is zero (bit-exact planes).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from hpvcd_b200 import abi, synth

pytestmark = pytest.mark.gpu

TOLERANCE = 0  # sample values must match exactly


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _plane_shapes(p):
    g = synth.geometry(p)
    shapes = [(g["h"], g["w"])]
    if p.chroma_idc:
        shapes += [(g["ch"], g["cw"])] * 2
    return shapes, g["bytes_per_sample"]


class NoAllocOut:
    """Caller-owned device planes and status word for one call."""

    def __init__(self, torch, p):
        self.shapes, self.bps = _plane_shapes(p)
        self.planes = [torch.empty(h * w * self.bps, dtype=torch.uint8, device="cuda")
                       for h, w in self.shapes]
        self.status = torch.full((1,), -1, dtype=torch.int32, device="cuda")

    def ptrs(self):
        arr = (C.c_void_p * 3)()
        for c, t in enumerate(self.planes):
            arr[c] = t.data_ptr()
        return arr

    def host(self):
        dt = np.uint8 if self.bps == 1 else np.uint16
        return [t.cpu().numpy().view(dt).reshape(s) for t, s in zip(self.planes, self.shapes)]


def _call(L, dev_pic, out, stream) -> int:
    return L.hpvcd_decode_noalloc(C.byref(dev_pic), out.ptrs(), C.c_void_p(out.status.data_ptr()),
                                  C.c_void_p(stream.cuda_stream))


def _pictures():
    s = synth.SynthSet()
    cfgs = [
        synth.intra_cfg(9101, 512, 512, bit_depth=10, chroma_idc=1),            # deblock + SAO
        synth.intra_cfg(9102, 328, 200, bit_depth=8, chroma_idc=3, sao=False,   # odd size, no SAO
                        tskip_p=0.2, tqb_p=0.05),
        synth.residual_cfg(9103, 256, 256, bit_depth=8, chroma_idc=1),          # prediction in plane
        synth.intra_cfg(9104, 384, 256, bit_depth=12, chroma_idc=0),            # 4:0:0
    ]
    cfgs[3].log2_ctb = 4
    # 4:4:4 with cross-component prediction, RExt rotation / RDPCM and scaling lists
    rx = synth.intra_cfg(9105, 256, 192, bit_depth=10, chroma_idc=3, tskip_p=0.3, tqb_p=0.05, scaling=True)
    rx.ccp_p, rx.rext, rx.tskip_log2_max = 0.5, 7, 5
    cfgs.append(rx)
    for c in cfgs:
        s.add(c)
    return s, s.pictures()


def test_noalloc_matches_plan_entry_point_on_consecutive_calls():
    torch = _torch()
    from hpvcd_b200.gpu import DevicePlan
    L = abi.lib()
    keep, pics = _pictures()
    plan = DevicePlan(pics)                       # the existing entry point
    plan.launch()
    assert plan.status() == abi.OK
    expect = [plan.planes(i) for i in range(len(pics))]

    stream = torch.cuda.current_stream()
    # warm-up call: first call on the device does the set-up
    w = NoAllocOut(torch, pics[0])
    assert _call(L, plan.dev_pics[0], w, stream) == abi.OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    launches0 = L.hpvcd_kernel_launch_count()

    # consecutive calls on one stream, no synchronisation between them; the
    # first picture twice to show the scratch is reset per call
    order = [0, 1, 2, 3, 4, 0]
    outs = [NoAllocOut(torch, pics[i]) for i in order]
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    for i, o in zip(order, outs):
        rc = _call(L, plan.dev_pics[i], o, stream)
        assert rc == abi.OK, L.hpvcd_last_error_string()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free1, "device memory changed during the calls"
    assert free1 <= free0
    assert L.hpvcd_kernel_launch_count() > launches0
    for i, o in zip(order, outs):
        assert int(o.status.item()) == 0
        got = o.host()
        for c, (g, e) in enumerate(zip(got, expect[i])):
            diff = np.abs(g.astype(np.int32) - e.astype(np.int32))
            assert diff.max(initial=0) <= TOLERANCE, f"picture {i} component {c}"


def test_noalloc_matches_the_oracle():
    """The no-allocation planes of two pictures (one with deblocking and SAO,
    one 4:4:4 with cross-component prediction and RExt tools) against the
    CPU oracle directly, not only against the plan entry point."""
    torch = _torch()
    from hpvcd_b200.gpu import DevicePlan
    from oracle import oracle as O
    L = abi.lib()
    keep, pics = _pictures()
    plan = DevicePlan(pics)  # uploads the inputs; its own launches are not used here
    ref, _ = O.decode_batch(pics)
    stream = torch.cuda.current_stream()
    for i in (0, 4):
        for _ in range(2):  # two calls in a row on the shared scratch
            o = NoAllocOut(torch, pics[i])
            assert _call(L, plan.dev_pics[i], o, stream) == abi.OK, L.hpvcd_last_error_string()
            torch.cuda.synchronize()
            assert int(o.status.item()) == 0
            for c, g in enumerate(o.host()):
                diff = np.abs(g.astype(np.int32) - ref[i][c].astype(np.int32))
                assert diff.max(initial=0) <= TOLERANCE, f"picture {i} component {c}"


def test_noalloc_largest_stated_picture_fits():
    torch = _torch()
    from hpvcd_b200.gpu import DevicePlan
    L = abi.lib()
    s = synth.SynthSet()
    c = synth.intra_cfg(9201, 1024, 1024, bit_depth=12, chroma_idc=3)  # 4:4:4, 16-bit samples, SAO
    c.log2_ctb = 4
    s.add(c)
    pics = s.pictures()
    plan = DevicePlan(pics)
    plan.launch()
    assert plan.status() == abi.OK
    expect = plan.planes(0)
    stream = torch.cuda.current_stream()
    for _ in range(2):
        o = NoAllocOut(torch, pics[0])
        assert _call(L, plan.dev_pics[0], o, stream) == abi.OK, L.hpvcd_last_error_string()
        torch.cuda.synchronize()
        assert int(o.status.item()) == 0
        for g, e in zip(o.host(), expect):
            assert np.array_equal(g, e)


def test_noalloc_rejects_what_it_cannot_hold():
    torch = _torch()
    L = abi.lib()
    s = synth.SynthSet()
    s.add(synth.intra_cfg(9301, 2048, 1024, bit_depth=12, chroma_idc=3))  # needs ~24 MiB
    big = s.picture(0)
    dummy = (C.c_void_p * 3)(256, 512, 768)
    rc = L.hpvcd_decode_noalloc(C.byref(big), dummy, None, None)
    assert rc == abi.ERR_LIMIT
    msg = L.hpvcd_last_error_string().decode()
    assert "bytes of scratch" in msg and str(abi.NOALLOC_SCRATCH_BYTES) in msg

    s.add(synth.inter_cfg(9302, 256, 128))
    inter = s.picture(1)
    assert L.hpvcd_decode_noalloc(C.byref(inter), dummy, None, None) == abi.ERR_UNSUPPORTED

    s.add(synth.intra_cfg(9303, 256, 128))
    ok = s.picture(2)
    stored = abi.Picture()
    C.pointer(stored)[0] = ok
    stored.flags |= abi.PIC_STORE_DPB(0)  # DPB stores belong to a context's submits
    assert L.hpvcd_decode_noalloc(C.byref(stored), dummy, None, None) == abi.ERR_UNSUPPORTED
    assert b"decoded-picture buffer" in L.hpvcd_last_error_string()
    bad = (C.c_void_p * 3)(256 + 16, 512, 768)  # misaligned luma plane
    assert L.hpvcd_decode_noalloc(C.byref(ok), bad, None, None) == abi.ERR_INVALID_ARG
    assert L.hpvcd_decode_noalloc(None, dummy, None, None) == abi.ERR_INVALID_ARG
    del torch
