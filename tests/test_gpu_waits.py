"""Bounded wavefront waits of the reconstruction kernel.

The reference's wavefront rows always publish (wpp.rs:168-172), so a wait
there can only end.  Here a CTU waits on flags other CTAs write; every such
wait is bounded and, when it runs out, sets the device error word and
returns.  These tests make a wait run out without faulting anything: one CTU
is left out of the plan's work list (hpvcd_plan_set_wait_test), so it never
publishes, and the waits of the CTUs predicting from it are cut to 100 000
polls.  The launch must complete, report HPVCD_ERR_TIMEOUT, write nothing
outside the picture's place on the canvas, and leave the CTUs that cannot
see the missing one bit-exact; restoring the list decodes the whole picture
bit-exactly again in the same context.
"""
import ctypes

import numpy as np
import pytest

from hpvcd_b200 import abi, synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from hpvcd_b200.gpu import DevicePlan  # noqa: E402
from oracle import oracle as O  # noqa: E402

# polls per wait before it gives up: short enough for a quick test, far
# longer than any wait for a CTU that is being reconstructed (one CTU walk
# is a fraction of a millisecond)
SPIN = 100_000


def wavefront_order(cols: int, rows: int):
    """CTUs in the plan's work-list order: by x + 2y, then y."""
    out = []
    for t in range(cols + 2 * rows + 1):
        for y in range(rows):
            x = t - 2 * y
            if 0 <= x < cols:
                out.append((x, y))
    return out


@pytest.mark.parametrize("wave", [0, 1], ids=["per_quadrant", "whole_ctu"])
def test_wait_runs_out_and_the_launch_returns(wave):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(7001, 512, 512, bit_depth=10, chroma_idc=1))
    pics = s.pictures()
    # the tile sits at (64, 32) of a 640 x 576 canvas: the border must stay 0
    place = (abi.TilePlace * 1)(abi.TilePlace(64, 32, 512, 512))
    out = abi.Output(abi.OUT_RGB8, abi.MATRIX_SMPTE170M, 1, 640, 576, ctypes.cast(place, ctypes.c_void_p))
    plan = DevicePlan(pics, out, sched=abi.Sched(0, 0, 0, wave))
    ref_planes, ref_rgb = O.decode_batch(pics, out)

    order = wavefront_order(8, 8)
    plan.set_wait_test(SPIN, order.index((2, 2)))
    plan.launch()
    torch.cuda.synchronize()  # returns: every wait ended
    assert plan.status() == abi.ERR_TIMEOUT

    got = plan.planes(0)
    # CTU rows 0 and 1 never read CTU (2, 2); deblocking and SAO reach at
    # most 3 + 1 luma rows (1 + 1 chroma rows) past a CTU row
    assert np.array_equal(got[0][:120].astype(np.uint16), ref_planes[0][0][:120])
    for c in (1, 2):
        assert np.array_equal(got[c][:56].astype(np.uint16), ref_planes[0][c][:56])
    canvas = plan.canvas()
    inside = np.zeros(canvas.shape[:2], bool)
    inside[32:32 + 512, 64:64 + 512] = True
    assert not canvas[~inside].any(), "samples written outside the picture's place"
    assert np.array_equal(canvas[32:32 + 120, 64:64 + 512], ref_rgb[32:32 + 120, 64:64 + 512])

    # the context stays usable: the full list decodes the picture bit-exactly
    plan.set_wait_test(0, -1)
    plan.launch()
    assert plan.status() == abi.OK
    got = plan.planes(0)
    for c in range(3):
        assert np.array_equal(got[c].astype(np.uint16), ref_planes[0][c])
    assert np.array_equal(plan.canvas(), ref_rgb)
    plan.close()


def test_wait_test_rejects_bad_entries():
    s = synth.SynthSet()
    s.add(synth.intra_cfg(7002, 128, 128, bit_depth=8))
    plan = DevicePlan(s.pictures())
    L = abi.lib()
    assert L.hpvcd_plan_set_wait_test(plan._h, 10, 4) == abi.ERR_INVALID_ARG  # 2 x 2 CTUs: entries 0..3
    assert L.hpvcd_plan_set_wait_test(plan._h, 10, -2) == abi.ERR_INVALID_ARG
    assert L.hpvcd_plan_set_wait_test(None, 10, 0) == abi.ERR_INVALID_ARG
    plan.close()
