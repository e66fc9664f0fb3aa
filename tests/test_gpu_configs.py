"""Bit-exact parity at the benchmark configurations' own shapes.

The other parity tests use small pictures; these decode the shapes the
benchmark workloads state, through the C ABI, against the CPU oracle:

* the inter video GOP: one 1920x1080 8-bit 4:2:0 intra frame and 31 inter
  frames with up to 4 references, 40 % bi-predicted PUs and explicit
  weighted prediction in one frame in ten (the sequence the inter benchmark
  times), decoded as one plan and frame by frame through the device DPB;
* the schedule-selector frames: 3840x2160 10-bit 4:2:0, one intra and one
  inter frame of the selector workload;
* the mixed-size serving workload: a seeded draw of images (sizes 256..4096,
  8 / 10 bit, 4:2:0 / 4:4:4) including a 4096-wide 10-bit 4:4:4 image,
  through the continuous-batching server with the learned schedule;
* a slice whose deblocking is disabled, folded by the host into zero
  boundary strengths, against the reference's own per-slice skip;
* the 4032x3024 grid decoded from its coded I slices (host syntax decode,
  then the GPU).

Integer work: the tolerance is zero.
"""
import ctypes as C

import numpy as np
import pytest

from hpvcd_b200 import abi, synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from hpvcd_b200.gpu import DevicePlan, Dpb, GpuDecoder, split_planes  # noqa: E402
from oracle import oracle as O  # noqa: E402


def assert_planes_equal(gpu_planes, ref_planes, what=""):
    for i, (g, r) in enumerate(zip(gpu_planes, ref_planes)):
        for c in range(3):
            if r[c].size == 0:
                continue
            gc = g[c].astype(np.uint16)
            if not np.array_equal(gc, r[c]):
                d = np.argwhere(gc != r[c])
                y, x = d[0]
                raise AssertionError(f"{what} picture {i} comp {c}: {len(d)} samples differ, first at "
                                     f"(x={x}, y={y}) gpu={gc[y, x]} oracle={r[c][y, x]}")


# --- inter video: 1920x1080, 32 frames, 4 references ----------------------
def inter_gop(seed=1000, n_frames=32, w=1920, h=1080):
    """The inter benchmark's sequence (bench.py --workload inter, rank 0)."""
    s = synth.SynthSet()
    s.add(synth.intra_cfg(seed, w, h, bit_depth=8, chroma_idc=1))
    for i in range(1, n_frames):
        s.add(synth.inter_cfg(seed + i, w, h, bit_depth=8, weighted=(i % 10 == 5), n_refs=4))
    return s, s.pictures()


def frame_by_frame(pics, in_flight=2, entries=32):
    """One frame per submit; frame k is stored in DPB entry k % entries and
    reads its references from theirs (the sequence's references reach back
    up to the intra frame, so every frame keeps its own entry)."""
    out = []
    with GpuDecoder(0, max_inflight=in_flight) as d, Dpb(0, entries) as dpb:
        d.set_dpb(dpb)
        pend = []
        for k, p in enumerate(pics):
            q = abi.Picture()
            C.pointer(q)[0] = p
            q.flags = p.flags | abi.PIC_STORE_DPB(k % entries)
            for l in range(2):
                for r in range(abi.MAX_REFS):
                    sv = p.ref_slot[l][r]
                    assert sv < 0 or k - sv < entries
                    q.ref_slot[l][r] = abi.REF_DPB(sv % entries) if sv >= 0 else -1
            pend.append((d.submit([q]), q))
            if len(pend) >= in_flight:
                t, qq = pend.pop(0)
                d.wait(t)
                out += split_planes([qq], d.read(t))
        for t, qq in pend:
            d.wait(t)
            out += split_planes([qq], d.read(t))
        d.set_dpb(None)
    return out


def test_inter_gop_1080p_32_frames_plan_and_dpb():
    keep, pics = inter_gop()
    assert len(pics) == 32 and all(p.flags & abi.PIC_INTER for p in pics[1:])
    assert max(max(p.ref_slot[0][r] for r in range(abi.MAX_REFS)) for p in pics[1:]) >= 0
    ref, _ = O.decode_batch(pics, threads=8)
    plan = DevicePlan(pics)
    plan.launch()
    assert plan.status() == abi.OK
    assert_planes_equal([plan.planes(i) for i in range(len(pics))], ref, "inter GOP plan")
    plan.close()
    assert_planes_equal(frame_by_frame(pics), ref, "inter GOP frame by frame")


# --- selector workload: 3840x2160 10-bit frames ---------------------------
def test_selector_frames_3840x2160():
    from hpvcd_b200 import selector
    specs = selector.frame_specs(40, seed=424242)
    intra = next(sp for sp in specs if sp.intra)
    inter = next(sp for sp in specs if not sp.intra and sp.weighted is False)
    refs = selector.RefPictures(upload=False)
    for sp in (intra, inter):
        keep, pics, fi = selector.build_frame(sp, refs)
        assert (pics[fi].width, pics[fi].height, pics[fi].bit_depth_y) == (3840, 2160, 10)
        ref, _ = O.decode_batch(pics, threads=8)
        for sched in (None, selector.SCHEDULES[7]):
            plan = DevicePlan(pics, sched=sched)
            plan.launch()
            assert plan.status() == abi.OK
            assert_planes_equal([plan.planes(fi)], [ref[fi]], f"4K {'intra' if sp.intra else 'inter'} frame")
            plan.close()


# --- serving mix: sizes to 4096, 10-bit 4:4:4 among them ------------------
def test_serving_mix_with_learned_schedule_to_4096():
    from hpvcd_b200 import selector, serving
    from hpvcd_b200.gpu import Server
    specs = synth.config2_images(seed=31, n_images=8)
    specs.append((4096, 2368, 10, 3))  # a 4096-wide 10-bit 4:4:4 image
    s = synth.SynthSet()
    imgs = []
    for k, (w, h, bd, idc) in enumerate(specs):
        g = synth.make_grid(w, h, seed=5000 + k, bit_depth=bd, chroma_idc=idc, synth=s)
        first = len(s) - g.cols * g.rows
        imgs.append(serving.Image(w, h, [s.picture(first + i) for i in range(g.cols * g.rows)], g.places,
                                  abi.MATRIX_SMPTE170M if k % 3 else abi.MATRIX_BT709, bool(k % 2)))
    assert any(im.width == 4096 and im.pics[0].chroma_idc == 3 and im.pics[0].bit_depth_y == 10 for im in imgs)
    mlp = selector.Mlp.load()
    with Server(0, max_inflight=2, batching=True, batch_window_us=100000) as srv:
        srv.set_selector(mlp, selector.SCHEDULES)
        for k, im in enumerate(imgs):
            srv.submit(im.pics, im.places, im.width, im.height, user=k, matrix=im.matrix,
                       full_range=im.full_range)
        got = {}
        while len(got) < len(imgs):
            for c in srv.poll(16, timeout_ms=120000):
                assert c["status"] == abi.OK
                got[c["user"]] = c["image"]
        assert sum(srv.selector_picks(selector.K + 1)) > 0
    for k, im in enumerate(imgs):
        out, kk = synth.grid_output(synth.Grid(im.width, im.height, 512, s, im.places), matrix=im.matrix,
                                    full_range=im.full_range)
        _, ref = O.decode_batch(im.pics, out, want_planes=False, threads=8)
        assert np.array_equal(got[k], ref), f"image {k} {im.width}x{im.height}"


# --- slice with deblocking disabled: the host's fold ----------------------
def test_disabled_slice_folded_into_boundary_strengths():
    s = synth.SynthSet()
    c = synth.intra_cfg(777, 512, 384, bit_depth=10, chroma_idc=1)
    c.regions = 1  # three slices with their own deblocking offsets
    s.add(c)
    p = s.picture(0)
    g = synth.geometry(p)
    regions = np.ctypeslib.as_array((C.c_uint16 * (g["ctb_cols"] * g["ctb_rows"])).from_address(p.ctb_region))
    slice_of = (regions >> 8).reshape(g["ctb_rows"], g["ctb_cols"])
    assert (slice_of == 1).any()
    try:
        O.set_disabled_slices([1])  # the reference skips every segment whose q sample is in slice 1
        ref, _ = O.decode_batch([p])
    finally:
        O.set_disabled_slices(None)
    # the host's fold: boundary strengths of the cells of slice 1 are zero
    cells = np.ctypeslib.as_array((C.c_uint8 * (g["gw"] * g["gh"] * 4)).from_address(p.cells)).copy()
    cells = cells.view(abi.CELL_DTYPE).reshape(g["gh"], g["gw"])
    ctb = 1 << p.log2_ctb
    ys, xs = np.mgrid[0:g["gh"], 0:g["gw"]]
    in_slice = slice_of[(ys * 4) // ctb, (xs * 4) // ctb] == 1
    folded = cells.copy()
    folded["bs_v"][in_slice] = 0
    folded["bs_h"][in_slice] = 0
    q = abi.Picture()
    C.pointer(q)[0] = p
    q.cells = folded.ctypes.data
    with GpuDecoder(0) as d:
        got = d.decode_yuv([q])
    assert_planes_equal(got, ref, "slice with deblocking disabled")
    # and the fold matters: without it the result differs
    plain, _ = O.decode_batch([p])
    assert any(not np.array_equal(a, b) for a, b in zip(plain[0], ref[0]))


# --- the 4032x3024 grid from its coded slices ------------------------------
def test_grid_from_coded_slices_bitstream_to_rgb8():
    """Bitstream -> pixels: the 48 I slices of the grid parsed by the host
    syntax decode (hpvcd_syntax_decode_batch), the parsed buffers decoded on
    the GPU through hpvcd_gpu_submit, against the CPU oracle on the buffers
    the writer generated."""
    from hpvcd_b200.syntax import decode_batch
    g = synth.config1_grid(seed=21)
    parsed = decode_batch(synth.grid_slices(g), threads=8)
    out, keep = synth.grid_output(g)
    with GpuDecoder(0) as d:
        rgb = d.decode_rgb8([x.picture() for x in parsed], out)
    _, ref = O.decode_batch(g.synth.pictures(), out, want_planes=False, threads=8)
    assert np.array_equal(rgb, ref)
    for x in parsed:
        x.close()
