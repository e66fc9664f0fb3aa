"""The CPU reference arm: the reference's parallel structure (grid-row jobs,
banded deblocking / SAO / colour conversion on a work-stealing pool) with
the scalar kernels and with the AVX2 set, against the serial oracle decode
of the same tiles.  Integer work: the canvases must be identical."""
import numpy as np
import pytest

from hpvcd_b200 import abi, synth
from oracle import oracle as O

CASES = [
    dict(w=1100, h=700, bd=10, idc=1),                       # 3 x 2 tiles, cropped, 10-bit 4:2:0
    dict(w=640, h=512, bd=8, idc=1, tskip_p=0.3, tqb_p=0.1),  # 8-bit: i16 storage, exempt cells
    dict(w=512, h=520, bd=12, idc=3),                        # 12-bit 4:4:4 (extended dequant range)
    dict(w=600, h=448, bd=8, idc=0),                         # 4:0:0
    dict(w=512, h=512, bd=10, idc=1, scaling=True),          # scaling lists
    dict(w=1024, h=512, bd=8, idc=2, ctb=5),                 # 4:2:2, CTB 32
    dict(w=520, h=264, bd=10, idc=1, ctb=4),                 # CTB 16, ragged
]


def grid(case, seed):
    kw = {k: case[k] for k in ("tskip_p", "tqb_p", "scaling") if k in case}
    g = synth.make_grid(case["w"], case["h"], seed=seed, bit_depth=case["bd"], chroma_idc=case["idc"], **kw)
    if "ctb" in case:
        s = synth.SynthSet()
        g2 = synth.Grid(case["w"], case["h"], 512, s, [])
        for r in range(g.rows):
            for col in range(g.cols):
                c = synth.intra_cfg(seed * 100003 + r * g.cols + col, 512, 512, case["bd"], case["idc"], **kw)
                c.log2_ctb = case["ctb"]
                s.add(c)
                g2.places.append((col * 512, r * 512, 512, 512))
        g = g2
    return g


@pytest.mark.parametrize("k", range(len(CASES)))
def test_reference_arm_matches_the_oracle(k):
    g = grid(CASES[k], seed=300 + k)
    out, keep = synth.grid_output(g, matrix=abi.MATRIX_BT709 if k % 2 else abi.MATRIX_SMPTE170M,
                                  full_range=bool(k % 3))
    pics = g.synth.pictures()
    _, ref = O.decode_batch(pics, out, want_planes=False)
    for simd in (False, True):
        got = O.decode_grid_reference(pics, out, threads=4, simd=simd)
        assert np.array_equal(got.reshape(ref.shape), ref), f"simd={simd}"


def test_reference_arm_single_thread_and_many():
    g = grid(CASES[0], seed=77)
    out, keep = synth.grid_output(g)
    pics = g.synth.pictures()
    _, ref = O.decode_batch(pics, out, want_planes=False)
    for threads in (1, 2, 8):
        got = O.decode_grid_reference(pics, out, threads=threads, simd=True)
        assert np.array_equal(got.reshape(ref.shape), ref), threads
