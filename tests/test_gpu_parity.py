"""Bit-exact parity of the CUDA reconstruction path against the CPU oracle.

Every test calls through the C ABI (libhpvcd_b200.so) with seeded synthetic
flat buffers and compares plane for plane (and the RGB8 canvas) with the
oracle restatement of the reference's scalar decode.  Integer work: the
tolerance is zero.
"""
import ctypes
import numpy as np
import pytest

from hpvcd_b200 import abi, synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from hpvcd_b200.gpu import DevicePlan, GpuDecoder, split_planes  # noqa: E402
from oracle import oracle as O  # noqa: E402

C_u8 = ctypes.c_uint8


@pytest.fixture(scope="module")
def dec():
    d = GpuDecoder(0)
    yield d
    d.close()


def assert_planes_equal(gpu_planes, ref_planes, what=""):
    for i, (g, r) in enumerate(zip(gpu_planes, ref_planes)):
        for c in range(3):
            gc = g[c].astype(np.uint16)
            rc = r[c]
            if rc.size == 0:
                continue
            if not np.array_equal(gc, rc):
                diff = np.argwhere(gc != rc)
                y, x = diff[0]
                raise AssertionError(
                    f"{what} picture {i} comp {c}: {len(diff)} samples differ, first at (x={x}, y={y}) "
                    f"gpu={gc[y, x]} oracle={rc[y, x]}")


def run_yuv(dec, pics, what):
    gpu = dec.decode_yuv(pics)
    ref, _ = O.decode_batch(pics)
    assert_planes_equal(gpu, ref, what)


# --- residual-only reconstruction (512x512 8-bit, seeded prediction) -------
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_residual_picture(dec, seed):
    s = synth.SynthSet()
    s.add(synth.residual_cfg(seed))
    run_yuv(dec, s.pictures(), "residual")


def test_residual_picture_10bit_444(dec):
    s = synth.SynthSet()
    s.add(synth.residual_cfg(5, 256, 192, bit_depth=10, chroma_idc=3))
    run_yuv(dec, s.pictures(), "residual 10-bit 4:4:4")


# --- int8 level pools (HPVCD_PIC_COEFF8), host buffers and device plans ----
def test_int8_level_pool(dec):
    """Narrowed pools decode bit-exactly through hpvcd_gpu_submit (the packed
    input sized by the flag) and through a device plan, mixed in one batch
    with pictures that keep their int16 pool."""
    s = synth.SynthSet()
    s.add(synth.intra_cfg(404, 320, 192, bit_depth=8))      # the inter pictures predict from it
    for i in range(1, 3):
        s.add(synth.inter_cfg(404 + i, 320, 192, bit_depth=8, weighted=(i == 2), n_refs=1))
    s.add(synth.intra_cfg(401, 320, 192, bit_depth=10, chroma_idc=1))
    s.add(synth.intra_cfg(402, 192, 128, bit_depth=8, chroma_idc=3))
    s.add(synth.residual_cfg(403, 256, 128, bit_depth=8))
    pics = s.pictures()
    lv = synth.coeffs_of(pics[4])
    lv[np.argmax(np.abs(lv))] = 300            # this one keeps int16
    ref, _ = O.decode_batch(pics)
    keep = synth.narrow_coeffs(pics)
    assert len(keep) >= 4 and not pics[4].flags & abi.PIC_COEFF8
    assert_planes_equal(dec.decode_yuv(pics), ref, "int8 pools, host submit")
    plan = DevicePlan(pics)
    plan.launch()
    assert plan.status() == abi.OK
    assert_planes_equal([plan.planes(i) for i in range(len(pics))], ref, "int8 pools, device plan")
    plan.close()


# --- intra pictures: prediction + residual + deblock + SAO -----------------
@pytest.mark.parametrize("bd,idc", [(8, 1), (10, 1), (8, 3), (10, 3), (8, 0)])
def test_intra_tile(dec, bd, idc):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(10 + bd + idc, 512, 512, bit_depth=bd, chroma_idc=idc))
    run_yuv(dec, s.pictures(), f"intra bd={bd} idc={idc}")


def test_intra_recon_only(dec):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(21, 256, 256, bit_depth=10, sao=False, deblock=False))
    run_yuv(dec, s.pictures(), "intra recon only")


def test_intra_tskip_tqb_exempt(dec):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(22, 256, 256, bit_depth=8, tskip_p=0.5, tqb_p=0.2))
    s.add(synth.intra_cfg(23, 256, 256, bit_depth=10, tskip_p=0.5, tqb_p=0.2))
    run_yuv(dec, s.pictures(), "tskip/tqb")


@pytest.mark.parametrize("w,h,log2_ctb", [(200, 136, 6), (96, 64, 4), (328, 168, 5), (8, 8, 6), (1080 // 4 * 4, 72, 6)])
def test_intra_odd_sizes_and_ctb(dec, w, h, log2_ctb):
    s = synth.SynthSet()
    c = synth.intra_cfg(30 + w, w, h, bit_depth=10)
    c.log2_ctb = log2_ctb
    s.add(c)
    run_yuv(dec, s.pictures(), f"intra {w}x{h} ctb {1 << log2_ctb}")


def test_intra_qp_offsets_and_deblock_offsets(dec):
    s = synth.SynthSet()
    c = synth.intra_cfg(40, 256, 256, bit_depth=10)
    c.cb_qp_offset, c.cr_qp_offset = -5, 7
    c.beta_offset_div2, c.tc_offset_div2 = 3, -2
    c.qp_min, c.qp_max = 0, 51
    s.add(c)
    c2 = synth.intra_cfg(41, 128, 128, bit_depth=10)
    c2.qp_min, c2.qp_max = -12, 51  # negative QpY allowed at 10-bit
    s.add(c2)
    run_yuv(dec, s.pictures(), "qp offsets")


def test_intra_no_strong_smoothing_and_smoothing_disabled(dec):
    s = synth.SynthSet()
    c = synth.intra_cfg(42, 256, 256)
    c.pic_flags &= ~abi.PIC_STRONG_SMOOTHING
    s.add(c)
    c = synth.intra_cfg(43, 256, 256)
    c.pic_flags |= abi.PIC_SMOOTHING_DISABLED
    s.add(c)
    run_yuv(dec, s.pictures(), "smoothing flags")


def test_batch_of_mixed_pictures(dec):
    s = synth.SynthSet()
    for i, (w, h, bd, idc) in enumerate([(512, 512, 8, 1), (256, 384, 10, 3), (192, 128, 8, 3),
                                         (512, 320, 10, 1), (64, 64, 8, 1)]):
        s.add(synth.intra_cfg(50 + i, w, h, bit_depth=bd, chroma_idc=idc))
    run_yuv(dec, s.pictures(), "mixed batch")


# --- RGB8 canvas of a grid (decode_heic_rgb8 path) --------------------------
@pytest.mark.parametrize("matrix,full", [(abi.MATRIX_SMPTE170M, True), (abi.MATRIX_BT709, False),
                                         (abi.MATRIX_BT2020NCL, True), (abi.MATRIX_IDENTITY, True),
                                         (abi.MATRIX_YCGCO, True)])
def test_grid_rgb8(dec, matrix, full):
    g = synth.make_grid(1000, 700, seed=3, bit_depth=10, chroma_idc=1)
    out, keep = synth.grid_output(g, matrix=matrix, full_range=full)
    pics = g.synth.pictures()
    rgb = dec.decode_rgb8(pics, out)
    _, ref = O.decode_batch(pics, out, want_planes=False)
    assert np.array_equal(rgb, ref)


def test_full_4032x3024_grid_rgb8(dec):
    g = synth.config1_grid(seed=7)
    out, keep = synth.grid_output(g)
    pics = g.synth.pictures()
    rgb = dec.decode_rgb8(pics, out)
    _, ref = O.decode_batch(pics, out, want_planes=False, threads=8)
    assert rgb.shape == (3024, 4032, 3)
    assert np.array_equal(rgb, ref)


def test_grid_8bit_444_and_mono(dec):
    for bd, idc in ((8, 3), (8, 0), (12, 1)):
        g = synth.make_grid(700, 600, seed=9 + idc, bit_depth=bd, chroma_idc=idc)
        out, keep = synth.grid_output(g)
        pics = g.synth.pictures()
        rgb = dec.decode_rgb8(pics, out)
        _, ref = O.decode_batch(pics, out, want_planes=False)
        assert np.array_equal(rgb, ref), (bd, idc)


# --- inter: motion compensation with bi / weighted prediction --------------
@pytest.mark.parametrize("weighted", [False, True])
def test_inter_sequence(dec, weighted):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(60, 320, 192, bit_depth=8))
    for i in range(1, 5):
        s.add(synth.inter_cfg(60 + i, 320, 192, weighted=weighted))
    run_yuv(dec, s.pictures(), f"inter weighted={weighted}")


def test_inter_10bit(dec):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(70, 256, 136, bit_depth=10))
    for i in range(1, 4):
        s.add(synth.inter_cfg(70 + i, 256, 136, bit_depth=10, weighted=(i == 2)))
    run_yuv(dec, s.pictures(), "inter 10-bit")


# --- device plans: repeated launches give identical output ----------------
def test_device_plan_repeat_and_status():
    g = synth.make_grid(1024, 512, seed=11, bit_depth=10)
    out, keep = synth.grid_output(g)
    pics = g.synth.pictures()
    plan = DevicePlan(pics, out)
    plan.launch()
    a = plan.canvas()
    plan.launch()
    plan.launch()
    b = plan.canvas()
    assert plan.status() == abi.OK
    assert np.array_equal(a, b)
    _, ref = O.decode_batch(pics, out, want_planes=False)
    assert np.array_equal(a, ref)
    plan.close()


def test_ticket_reuse_same_layout(dec):
    # Same layout, different content: the cached plan is rebound.
    outs = []
    for seed in (1, 2):
        g = synth.make_grid(600, 600, seed=seed, bit_depth=8)
        out, keep = synth.grid_output(g)
        pics = g.synth.pictures()
        rgb = dec.decode_rgb8(pics, out)
        _, ref = O.decode_batch(pics, out, want_planes=False)
        assert np.array_equal(rgb, ref)
        outs.append(rgb)
    assert not np.array_equal(outs[0], outs[1])


def test_errors_map_to_status(dec):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(80, 64, 64))
    bad = s.picture(0)
    bad.chroma_idc = 4     # no such chroma format
    with pytest.raises(abi.HpvcdError) as e:
        dec.submit([bad])
    assert e.value.status == abi.ERR_UNSUPPORTED
    bad = s.picture(0)
    bad.bit_depth_y = bad.bit_depth_c = 14   # above the supported 12 bits
    with pytest.raises(abi.HpvcdError) as e:
        dec.submit([bad])
    assert e.value.status == abi.ERR_UNSUPPORTED
    # a reference of another size (motion compensation would read outside it)
    s2 = synth.SynthSet()
    s2.add(synth.intra_cfg(81, 128, 64, bit_depth=8))
    s2.add(synth.inter_cfg(82, 128, 128))
    with pytest.raises(abi.HpvcdError) as e:
        dec.submit(s2.pictures())
    assert e.value.status == abi.ERR_BITSTREAM
    p2 = s.picture(0)
    p2.width = 0
    with pytest.raises(abi.HpvcdError) as e:
        dec.submit([p2])
    assert e.value.status == abi.ERR_LIMIT


def test_malformed_tb_is_reported(dec):
    # A TB record pointing outside its CTU must not be reconstructed; the
    # device reports a Bitstream error instead of writing out of bounds.
    s = synth.SynthSet()
    s.add(synth.intra_cfg(81, 128, 128))
    p = s.picture(0)
    tus = synth.tus_of(p)
    coded = np.nonzero(tus["flags"] & abi.TU_CBF)[0]
    tus[coded[0]]["x"] = 4000  # far outside
    t = dec.submit([p])
    dec.wait(t)
    with pytest.raises(abi.HpvcdError) as e:
        dec.read(t)
    assert e.value.status == abi.ERR_BITSTREAM


def test_packed_pinned_inputs_and_direct_output(dec):
    from hpvcd_b200.gpu import pack_pinned, pinned_empty
    g = synth.make_grid(1100, 900, seed=12, bit_depth=10)
    out, keep = synth.grid_output(g)
    pics = g.synth.pictures()
    packed, pkeep = pack_pinned(pics)
    nb = out.canvas_w * out.canvas_h * 3
    dst, dkeep = pinned_empty(nb)
    out.host_dst = dst.ctypes.data
    out.host_dst_bytes = nb
    t = dec.submit(packed, out)
    dec.wait(t)
    dec.read(t, dst)
    _, ref = O.decode_batch(pics, out, want_planes=False)
    assert np.array_equal(dst.reshape(ref.shape), ref)


def _image(seed, w, h, bd, idc, synth_set):
    """One image as 512x512 grid tiles; returns (pics, places)."""
    g = synth.make_grid(w, h, seed=seed, bit_depth=bd, chroma_idc=idc, synth=synth_set)
    first = len(synth_set) - g.cols * g.rows
    pics = [synth_set.picture(first + i) for i in range(g.cols * g.rows)]
    return pics, g.places


def test_multi_canvas_batch(dec):
    s = synth.SynthSet()
    specs = [(1, 700, 500, 8, 1, abi.MATRIX_SMPTE170M, 1), (2, 512, 512, 10, 3, abi.MATRIX_BT709, 0),
             (3, 300, 900, 8, 1, abi.MATRIX_BT2020NCL, 1)]
    pics, places, canv = [], [], []
    for k, (seed, w, h, bd, idc, m, fr) in enumerate(specs):
        p, pl = _image(seed, w, h, bd, idc, s)
        pics += p
        places += [(x, y, cw, ch, k) for (x, y, cw, ch) in pl]
        canv.append(abi.Canvas(w, h, m, fr))
    import ctypes as C
    pl_arr = (abi.TilePlace * len(places))(*[abi.TilePlace(*t) for t in places])
    cv_arr = (abi.Canvas * len(canv))(*canv)
    out = abi.Output(abi.OUT_RGB8, 0, 0, 0, 0, C.cast(pl_arr, C.c_void_p), None, 0, len(canv),
                     C.cast(cv_arr, C.c_void_p))
    t = dec.submit(pics, out)
    dec.wait(t)
    got = dec.read(t)
    _, ref = O.decode_batch(pics, out, want_planes=False)
    assert got.size == ref.size and np.array_equal(got, ref)


def test_server_alone_equals_in_mix():
    from hpvcd_b200.gpu import Server
    s = synth.SynthSet()
    imgs = [(_image(100 + i, w, h, bd, idc, s), w, h) for i, (w, h, bd, idc) in
            enumerate([(640, 448, 10, 1), (1024, 768, 8, 1), (512, 1100, 8, 3), (256, 256, 10, 1), (900, 600, 8, 1)])]
    # alone: one request, plain path
    with Server(0, max_inflight=1, batching=False) as plain:
        alone = []
        for k, ((pics, places), w, h) in enumerate(imgs):
            plain.submit(pics, places, w, h, user=k)
            (c,) = plain.poll(1, timeout_ms=60000)
            assert c["status"] == abi.OK
            alone.append(c["image"].copy())
    # in the mix: all submitted at once to a batching server
    with Server(0, max_inflight=2, batching=True, batch_window_us=200000) as srv:
        for k, ((pics, places), w, h) in enumerate(imgs):
            srv.submit(pics, places, w, h, user=k)
        got = {}
        while len(got) < len(imgs):
            for c in srv.poll(16, timeout_ms=60000):
                assert c["status"] == abi.OK
                got[c["user"]] = c
    assert max(c["batch_pictures"] for c in got.values()) > max(len(p) for (p, _), _, _ in imgs)
    for k, ((pics, places), w, h) in enumerate(imgs):
        assert np.array_equal(got[k]["image"], alone[k]), k
        # and both equal the oracle's decode of the image
        out, keep = synth.grid_output(synth.Grid(w, h, 512, s, places))
        _, ref = O.decode_batch(pics, out, want_planes=False)
        assert np.array_equal(alone[k], ref), k


def test_plan_graph_replay_matches():
    g = synth.make_grid(1024, 700, seed=13, bit_depth=8)
    out, keep = synth.grid_output(g)
    pics = g.synth.pictures()
    plan = DevicePlan(pics, out)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        before = abi.lib().hpvcd_kernel_launch_count()
        plan.launch(abi.STAGE_ALL | abi.STAGE_GRAPH, s)
        plan.launch(abi.STAGE_ALL | abi.STAGE_GRAPH, s)
        s.synchronize()
        counted = abi.lib().hpvcd_kernel_launch_count() - before
    assert counted == 2 * plan.launches_per_run
    got = plan.canvas()
    _, ref = O.decode_batch(pics, out, want_planes=False)
    assert np.array_equal(got, ref)
    plan.close()


def test_server_zero_copy_matches_oracle():
    from hpvcd_b200.gpu import Server, pack_pinned, pinned_empty
    s = synth.SynthSet()
    imgs = [(_image(200 + i, w, h, 10 if i % 2 else 8, 1, s), w, h) for i, (w, h) in
            enumerate([(640, 448), (1100, 700), (300, 300)])]
    keep = []
    with Server(0, max_inflight=2, batching=True, batch_window_us=200000) as srv:
        for k, ((pics, places), w, h) in enumerate(imgs):
            packed, kp = pack_pinned(pics)
            dst, kd = pinned_empty(w * h * 3)
            keep.append((kp, kd))
            srv.submit(packed, places, w, h, user=k, dst=dst.reshape(h, w, 3), zero_copy_keep=(kp, kd))
        got = {}
        while len(got) < len(imgs):
            for c in srv.poll(16, timeout_ms=60000):
                assert c["status"] == abi.OK
                got[c["user"]] = c
    assert max(c["batch_pictures"] for c in got.values()) > max(len(p) for (p, _), _, _ in imgs)
    for k, ((pics, places), w, h) in enumerate(imgs):
        out, kk = synth.grid_output(synth.Grid(w, h, 512, s, places))
        _, ref = O.decode_batch(pics, out, want_planes=False)
        assert np.array_equal(got[k]["image"], ref), k


# --- schedule variants: every knob combination gives the same pixels -------
def _dense_cfg(cfg):
    cfg.qp_min, cfg.qp_max = 4, 14      # fine quantisation: large dequantised values
    cfg.zero_frac = 0.2                 # dense blocks (butterfly path without zero rows)
    cfg.laplace_scale = 60.0
    cfg.tu_split_p = 0.2                # mostly 16x16 / 32x32 TBs
    return cfg


def test_schedule_variants_bit_exact():
    s = synth.SynthSet()
    s.add(_dense_cfg(synth.intra_cfg(80, 320, 256, bit_depth=8, chroma_idc=1)))    # i16 wrap at 8 bits
    s.add(_dense_cfg(synth.intra_cfg(81, 256, 192, bit_depth=12, chroma_idc=3)))   # 32x32 chroma TBs
    s.add(synth.intra_cfg(82, 512, 512, bit_depth=10, chroma_idc=1))
    s.add(_dense_cfg(synth.residual_cfg(83, 256, 256, bit_depth=10)))              # in-plane add path
    pics = s.pictures()
    ref, _ = O.decode_batch(pics)
    plan = DevicePlan(pics)
    for idct in (0, 1, 2):      # matrix, butterflies, integer tensor cores
        for cw in (1, 2, 3):    # wavefront build: two warps, three, three register-capped
            for ctas in (0, 1):
                for wave in (0, 1):   # quadrant-level / whole-CTU wavefront
                    plan.set_sched(abi.Sched(idct, cw, ctas, wave))
                    plan.launch()
                    assert plan.status() == abi.OK
                    got = [plan.planes(i) for i in range(len(pics))]
                    assert_planes_equal(got, ref, f"idct={idct} chroma_warps={cw} ctas={ctas} wave={wave}")
    with pytest.raises(abi.HpvcdError):
        plan.set_sched(abi.Sched(0, 1, 0, 2))
    with pytest.raises(abi.HpvcdError):
        plan.set_sched(abi.Sched(3, 1, 0, 0))
    with pytest.raises(abi.HpvcdError):
        plan.set_sched(abi.Sched(0, 4, 0, 0))
    plan.close()


def test_schedule_variants_inter_bit_exact():
    s = synth.SynthSet()
    s.add(_dense_cfg(synth.intra_cfg(90, 320, 192, bit_depth=8)))
    for i in range(1, 4):
        s.add(_dense_cfg(synth.inter_cfg(90 + i, 320, 192, weighted=(i == 2))))
    pics = s.pictures()
    ref, _ = O.decode_batch(pics)
    plan = DevicePlan(pics)
    for sched in (abi.Sched(1, 2, 0, 0), abi.Sched(1, 1, 1, 0), abi.Sched(0, 2, 0, 0), abi.Sched(1, 2, 0, 1)):
        plan.set_sched(sched)
        plan.launch()
        assert plan.status() == abi.OK
        assert_planes_equal([plan.planes(i) for i in range(len(pics))], ref, "inter variants")
    plan.close()


def test_concurrent_groups_direct_and_graph():
    """A batch of 20 independent tiles runs as concurrent groups (one stream
    each, forked from and joined into the launching stream), launched
    directly and replayed as a CUDA graph: both equal the oracle."""
    g = synth.make_grid(2560, 2048, seed=17, bit_depth=10)   # 5 x 4 tiles of 512
    out, keep = synth.grid_output(g)
    pics = g.synth.pictures()
    assert len(pics) == 20
    _, ref = O.decode_batch(pics, out, want_planes=False, threads=8)
    plan = DevicePlan(pics, out)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        plan.launch(abi.STAGE_ALL, s)
        s.synchronize()
        assert plan.status(s) == abi.OK
        assert np.array_equal(plan.canvas(), ref)
        before = abi.lib().hpvcd_kernel_launch_count()
        plan.launch(abi.STAGE_ALL | abi.STAGE_GRAPH, s)
        plan.launch(abi.STAGE_ALL | abi.STAGE_GRAPH, s)
        s.synchronize()
        assert abi.lib().hpvcd_kernel_launch_count() - before == 2 * plan.launches_per_run
        assert plan.status(s) == abi.OK
    assert np.array_equal(plan.canvas(), ref)
    # stages launched one at a time give the same picture
    for st_ in (abi.STAGE_RECON, abi.STAGE_DEBLOCK, abi.STAGE_SAO, abi.STAGE_OUTPUT):
        plan.launch(st_)
    torch.cuda.synchronize()
    assert np.array_equal(plan.canvas(), ref)
    plan.close()


# --- edge cases: empty residuals, no records, minimum and ragged sizes ----
def test_intra_without_coded_residual(dec):
    s = synth.SynthSet()
    c = synth.intra_cfg(110, 512, 256, bit_depth=10)
    c.cbf_p = 0.0          # prediction only: every TB uncoded
    s.add(c)
    run_yuv(dec, s.pictures(), "no coded residual")


def test_picture_without_records(dec):
    import ctypes as C
    s = synth.SynthSet()
    c = synth.residual_cfg(111, 256, 128, bit_depth=8)
    s.add(c)
    p = s.picture(0)
    q = abi.Picture()
    C.pointer(q)[0] = p
    q.n_tus = 0            # prediction in the plane, nothing to add
    q.n_coeffs = 0
    run_yuv(dec, [q], "no records")


@pytest.mark.parametrize("w,h,log2_ctb", [(8, 8, 4), (8, 8, 6), (4096, 16, 4), (16, 2048, 5), (1032, 24, 6)])
def test_minimum_and_ragged_sizes(dec, w, h, log2_ctb):
    s = synth.SynthSet()
    c = synth.intra_cfg(112 + w + h, w, h, bit_depth=10, chroma_idc=1)
    c.log2_ctb = log2_ctb
    s.add(c)
    run_yuv(dec, s.pictures(), f"{w}x{h} ctb{1 << log2_ctb}")


def test_many_ctus_ctb16(dec):
    s = synth.SynthSet()
    c = synth.intra_cfg(113, 1024, 1024, bit_depth=8, chroma_idc=1)
    c.log2_ctb = 4         # 4096 CTUs, a 191-step wavefront
    s.add(c)
    run_yuv(dec, s.pictures(), "ctb16 1024x1024")


def test_mixed_edge_batch(dec):
    import ctypes as C
    s = synth.SynthSet()
    for i, (w, h, bd, idc, ctb) in enumerate([(8, 8, 8, 1, 4), (520, 264, 10, 3, 5), (64, 1024, 12, 0, 6),
                                              (1024, 8, 8, 1, 4), (256, 256, 10, 1, 6)]):
        c = synth.intra_cfg(120 + i, w, h, bit_depth=bd, chroma_idc=idc)
        c.log2_ctb = ctb
        if i == 4:
            c.cbf_p = 0.0
        s.add(c)
    r = synth.residual_cfg(130, 128, 64, bit_depth=8)
    s.add(r)
    pics = s.pictures()
    q = abi.Picture()
    C.pointer(q)[0] = pics[-1]
    q.n_tus = 0
    q.n_coeffs = 0
    pics[-1] = q
    run_yuv(dec, pics, "mixed edge batch")


# --- decoded-picture buffer: frame-by-frame submits predict from HBM ------
def _frame_by_frame(pics, in_flight):
    """Submit each picture alone; reference pictures come from the DPB
    (picture k is stored into entry k, batch index j becomes REF_DPB(j))."""
    import ctypes as C
    from hpvcd_b200.gpu import Dpb
    with GpuDecoder(0, max_inflight=in_flight) as d, Dpb(0, entries=len(pics)) as dpb:
        d.set_dpb(dpb)
        tickets, out = [], []
        for k, p in enumerate(pics):
            q = abi.Picture()
            C.pointer(q)[0] = p
            q.flags = p.flags | abi.PIC_STORE_DPB(k)
            for l in range(2):
                for r in range(abi.MAX_REFS):
                    s = p.ref_slot[l][r]
                    q.ref_slot[l][r] = abi.REF_DPB(s) if s >= 0 else -1
            tickets.append((d.submit([q]), q))
            if len(tickets) >= in_flight:
                t, qq = tickets.pop(0)
                d.wait(t)
                out += split_planes([qq], d.read(t))
        for t, qq in tickets:
            d.wait(t)
            out += split_planes([qq], d.read(t))
        d.set_dpb(None)
    return out


@pytest.mark.parametrize("in_flight", [1, 2])
def test_dpb_frame_by_frame_matches_batch(in_flight):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(140, 320, 192, bit_depth=8))
    for i in range(1, 6):
        s.add(synth.inter_cfg(140 + i, 320, 192, weighted=(i == 3)))
    pics = s.pictures()
    ref, _ = O.decode_batch(pics)
    assert_planes_equal(_frame_by_frame(pics, in_flight), ref, f"dpb in_flight={in_flight}")


def test_dpb_rejects_empty_entry(dec):
    import ctypes as C
    from hpvcd_b200.gpu import Dpb
    s = synth.SynthSet()
    s.add(synth.intra_cfg(150, 128, 64, bit_depth=8))
    s.add(synth.inter_cfg(151, 128, 64))
    pics = s.pictures()
    q = abi.Picture()
    C.pointer(q)[0] = pics[1]
    q.ref_slot[0][0] = abi.REF_DPB(3)  # never stored
    with GpuDecoder(0) as d, Dpb(0, entries=4) as dpb:
        with pytest.raises(abi.HpvcdError) as ei:
            d.submit([q])          # no DPB attached
        assert ei.value.status == abi.ERR_INVALID_ARG
        d.set_dpb(dpb)
        with pytest.raises(abi.HpvcdError) as ei:
            d.submit([q])          # entry 3 empty
        assert ei.value.status == abi.ERR_INVALID_ARG
        d.set_dpb(None)


# --- scaling lists (scaling_list_enabled_flag with signalled matrices) -----
@pytest.mark.parametrize("bd,idc", [(8, 1), (10, 3), (12, 0)])
def test_scaling_lists_intra(dec, bd, idc):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(160 + bd, 384, 256, bit_depth=bd, chroma_idc=idc, tskip_p=0.3, tqb_p=0.05,
                          scaling=True))
    run_yuv(dec, s.pictures(), f"scaling lists {bd}-bit idc {idc}")


def test_scaling_lists_residual_and_inter(dec):
    s = synth.SynthSet()
    r = synth.residual_cfg(170, 256, 128, bit_depth=10)
    r.scaling = 1
    s.add(r)
    run_yuv(dec, s.pictures(), "scaling lists residual")
    s = synth.SynthSet()
    s.add(synth.intra_cfg(171, 320, 192, bit_depth=8, scaling=True))
    for i in range(1, 4):
        s.add(synth.inter_cfg(171 + i, 320, 192, weighted=(i == 2), scaling=True))
    run_yuv(dec, s.pictures(), "scaling lists inter")


def test_scaling_lists_large_transform_skip(dec):
    """RExt transform skip above 4x4 keeps the flat scale (decode.rs:5882-5888)."""
    import ctypes as C
    s = synth.SynthSet()
    s.add(synth.intra_cfg(175, 256, 256, bit_depth=10, scaling=True))
    p = s.picture(0)
    tus = np.ctypeslib.as_array((C.c_uint8 * (p.n_tus * 16)).from_address(p.tus)).view(abi.TU_DTYPE).copy()
    coded = (tus["flags"] & abi.TU_CBF) != 0
    big = coded & (tus["log2n"] >= 3) & ((tus["flags"] & abi.TU_TQB) == 0)
    pick = np.flatnonzero(big)[::3]
    assert pick.size > 10
    tus["flags"][pick] |= abi.TU_TSKIP
    q = abi.Picture()
    C.pointer(q)[0] = p
    q.tus = tus.ctypes.data
    run_yuv(dec, [q], "transform skip 8x8..32x32 with scaling lists")


def test_scaling_lists_plan_and_server():
    from hpvcd_b200.gpu import Server, pack_pinned, pinned_empty
    g = synth.make_grid(1024, 512, seed=177, bit_depth=10, scaling=True)
    out, keep = synth.grid_output(g)
    pics = g.synth.pictures()
    _, ref = O.decode_batch(pics, out, want_planes=False)
    plan = DevicePlan(pics, out)
    plan.launch()
    torch.cuda.synchronize()
    assert np.array_equal(plan.canvas(), ref)
    plan.close()
    kp_all = []
    with Server(0, max_inflight=2, batching=True, batch_window_us=100000) as srv:
        srv.submit(pics, g.places, g.out_w, g.out_h, user=0)
        packed, kp = pack_pinned(pics)
        dst, kd = pinned_empty(g.out_w * g.out_h * 3)
        kp_all.append((kp, kd))
        srv.submit(packed, g.places, g.out_w, g.out_h, user=1, dst=dst.reshape(g.out_h, g.out_w, 3),
                   zero_copy_keep=(kp, kd))
        got = {}
        while len(got) < 2:
            for c in srv.poll(4, timeout_ms=60000):
                assert c["status"] == abi.OK
                got[c["user"]] = c
    for k in (0, 1):
        assert np.array_equal(got[k]["image"], ref), k


# --- RExt residual tools: rotation, implicit / explicit RDPCM, large TS -----
@pytest.mark.parametrize("bd,idc", [(8, 1), (10, 3), (12, 1)])
def test_rext_rotation_rdpcm_intra(dec, bd, idc):
    s = synth.SynthSet()
    for k in range(2):
        c = synth.intra_cfg(180 + bd + k, 384, 256, bit_depth=bd, chroma_idc=idc, tskip_p=0.5, tqb_p=0.1,
                            scaling=(k == 1))
        c.rext = 7
        c.tskip_log2_max = 5
        s.add(c)
    pics = s.pictures()
    tus = np.concatenate([np.ctypeslib.as_array((C_u8 * (p.n_tus * 16)).from_address(p.tus))
                          .view(abi.TU_DTYPE) for p in pics])
    assert (tus["flags"] & abi.TU_ROTATE).any() and (tus["flags"] & (abi.TU_RDPCM_H | abi.TU_RDPCM_V)).any()
    run_yuv(dec, pics, f"rext intra {bd}-bit idc {idc}")


def test_rext_explicit_rdpcm_inter(dec):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(190, 320, 192, bit_depth=10))
    for i in range(1, 4):
        c = synth.inter_cfg(190 + i, 320, 192, bit_depth=10, weighted=(i == 2))
        c.tskip_p, c.tqb_p, c.rext, c.tskip_log2_max = 0.5, 0.1, 7, 4
        s.add(c)
    run_yuv(dec, s.pictures(), "rext inter explicit rdpcm")


# --- cross-component prediction (4:4:4 RExt) -------------------------------
@pytest.mark.parametrize("bd", [8, 10, 12])
def test_cross_component_intra(dec, bd):
    s = synth.SynthSet()
    c = synth.intra_cfg(200 + bd, 384, 256, bit_depth=bd, chroma_idc=3, tskip_p=0.2, tqb_p=0.05)
    c.ccp_p = 0.6
    s.add(c)
    c2 = synth.intra_cfg(210 + bd, 256, 256, bit_depth=bd, chroma_idc=3, tskip_p=0.3, tqb_p=0.05, scaling=True,
                         cbf_p=0.5)
    c2.ccp_p, c2.rext, c2.tskip_log2_max = 0.6, 7, 5
    s.add(c2)
    pics = s.pictures()
    assert all(p.flags & abi.PIC_CROSS_COMPONENT for p in pics)
    tus = np.ctypeslib.as_array((C_u8 * (pics[1].n_tus * 16)).from_address(pics[1].tus)).view(abi.TU_DTYPE)
    ccp_only = (tus["res_scale"] != 0) & ((tus["flags"] & abi.TU_CBF) == 0)
    assert ccp_only.any()           # chroma residual from luma alone
    run_yuv(dec, pics, f"cross-component {bd}-bit")


def test_cross_component_inter_and_plan(dec):
    s = synth.SynthSet()
    c0 = synth.intra_cfg(220, 320, 192, bit_depth=10, chroma_idc=3)
    c0.ccp_p = 0.5
    s.add(c0)
    for i in range(1, 4):
        c = synth.inter_cfg(220 + i, 320, 192, bit_depth=10, weighted=(i == 2))
        c.chroma_idc = 3
        c.ccp_p, c.tskip_p, c.rext = 0.5, 0.3, 7
        s.add(c)
    pics = s.pictures()
    run_yuv(dec, pics, "cross-component inter")
    ref, _ = O.decode_batch(pics)
    plan = DevicePlan(pics)
    plan.launch()
    torch.cuda.synchronize()
    assert plan.status() == abi.OK
    assert_planes_equal([plan.planes(i) for i in range(len(pics))], ref, "cross-component plan")
    plan.close()


# --- 4:2:2: two stacked square chroma TBs, chroma CTU half as wide as tall --
@pytest.mark.parametrize("bd,log2_ctb", [(8, 6), (10, 5), (12, 4)])
def test_422_intra(dec, bd, log2_ctb):
    s = synth.SynthSet()
    c = synth.intra_cfg(230 + bd, 392, 264, bit_depth=bd, chroma_idc=2, tskip_p=0.2, tqb_p=0.05,
                        scaling=(bd == 10))
    c.log2_ctb = log2_ctb
    c.rext, c.tskip_log2_max = 7, 3
    s.add(c)
    run_yuv(dec, s.pictures(), f"4:2:2 {bd}-bit ctb {1 << log2_ctb}")


def test_422_residual_inter_and_rgb(dec):
    s = synth.SynthSet()
    s.add(synth.residual_cfg(240, 256, 128, bit_depth=8, chroma_idc=2))
    run_yuv(dec, s.pictures(), "4:2:2 residual")
    s = synth.SynthSet()
    s.add(synth.intra_cfg(241, 320, 192, bit_depth=8, chroma_idc=2))
    for i in range(1, 4):
        c = synth.inter_cfg(241 + i, 320, 192, bit_depth=8, weighted=(i == 2))
        c.chroma_idc = 2
        s.add(c)
    run_yuv(dec, s.pictures(), "4:2:2 inter")
    g = synth.make_grid(1100, 700, seed=245, bit_depth=10, chroma_idc=2)
    out, keep = synth.grid_output(g, matrix=abi.MATRIX_BT709, full_range=False)
    pics = g.synth.pictures()
    t = dec.submit(pics, out)
    dec.wait(t)
    got = dec.read(t)
    _, ref = O.decode_batch(pics, out, want_planes=False)
    assert np.array_equal(got.reshape(ref.shape), ref)


def test_mixed_formats_one_batch(dec):
    """4:2:0, 4:2:2, 4:4:4 and 4:0:0 pictures share one launch (the 4:4:4
    shared-memory layout holds every format)."""
    s = synth.SynthSet()
    for i, idc in enumerate([1, 2, 3, 0, 2, 1, 2, 3]):
        s.add(synth.intra_cfg(250 + i, 256, 192, bit_depth=8 if i % 2 else 10, chroma_idc=idc))
    run_yuv(dec, s.pictures(), "mixed chroma formats")
    s = synth.SynthSet()
    for i, idc in enumerate([1, 2, 1, 2]):
        s.add(synth.intra_cfg(260 + i, 256, 192, bit_depth=8, chroma_idc=idc))
    run_yuv(dec, s.pictures(), "4:2:0 + 4:2:2")


# --- slices and tiles: intra availability and SAO across their boundaries --
@pytest.mark.parametrize("regions,idc,no_across", [(1, 1, 0), (1, 2, abi.PIC_SAO_NO_ACROSS_SLICES),
                                                  (2, 3, abi.PIC_SAO_NO_ACROSS_TILES),
                                                  (2, 1, abi.PIC_SAO_NO_ACROSS_SLICES | abi.PIC_SAO_NO_ACROSS_TILES)])
def test_slices_and_tiles(dec, regions, idc, no_across):
    s = synth.SynthSet()
    for k, (w, h, ctb) in enumerate([(384, 320, 6), (264, 200, 5)]):
        c = synth.intra_cfg(410 + 7 * regions + idc + k, w, h, bit_depth=10 if k else 8, chroma_idc=idc)
        c.log2_ctb = ctb
        c.regions = regions
        c.pic_flags |= no_across
        s.add(c)
    pics = s.pictures()
    assert all(p.ctb_region for p in pics)
    run_yuv(dec, pics, f"regions {regions} idc {idc} flags {no_across:#x}")
    ref, _ = O.decode_batch(pics)
    plan = DevicePlan(pics)
    plan.launch()
    torch.cuda.synchronize()
    assert_planes_equal([plan.planes(i) for i in range(len(pics))], ref, "regions plan")
    for cw in (1, 2, 3):  # every wavefront build with the slice / tile tests compiled in
        plan.set_sched(abi.Sched(0, cw, 0, 0))
        plan.launch()
        assert plan.status() == abi.OK
        assert_planes_equal([plan.planes(i) for i in range(len(pics))], ref, f"regions plan, build {cw}")
    plan.close()


def test_tiles_through_the_server():
    from hpvcd_b200.gpu import Server, pack_pinned, pinned_empty
    s = synth.SynthSet()
    places = []
    for k, (x, y) in enumerate([(0, 0), (512, 0), (0, 256), (512, 256)]):
        c = synth.intra_cfg(421 + k, 512, 256, bit_depth=10)
        c.regions = 2 if k % 2 else 1
        c.pic_flags |= abi.PIC_SAO_NO_ACROSS_TILES | abi.PIC_SAO_NO_ACROSS_SLICES
        s.add(c)
        places.append((x, y, 512, 256))
    pics = s.pictures()
    out, keep = synth.grid_output(synth.Grid(1024, 512, 512, s, places))
    _, ref = O.decode_batch(pics, out, want_planes=False)
    kp_all = []
    with Server(0, max_inflight=2, batching=True, batch_window_us=100000) as srv:
        srv.submit(pics, places, 1024, 512, user=0)
        packed, kp = pack_pinned(pics)
        dst, kd = pinned_empty(1024 * 512 * 3)
        kp_all.append((kp, kd))
        srv.submit(packed, places, 1024, 512, user=1, dst=dst.reshape(512, 1024, 3), zero_copy_keep=(kp, kd))
        got = {}
        while len(got) < 2:
            for c in srv.poll(4, timeout_ms=60000):
                assert c["status"] == abi.OK
                got[c["user"]] = c
    for k in (0, 1):
        assert np.array_equal(got[k]["image"], ref), k


# --- constrained intra prediction -------------------------------------------
@pytest.mark.parametrize("bd,idc", [(8, 1), (10, 2), (10, 3)])
def test_constrained_intra(dec, bd, idc):
    s = synth.SynthSet()
    c0 = synth.intra_cfg(510 + bd + idc, 320, 192, bit_depth=bd, chroma_idc=idc)
    c0.pic_flags |= abi.PIC_CONSTRAINED_INTRA
    s.add(c0)
    for i in range(1, 4):
        c = synth.inter_cfg(510 + bd + idc + i, 320, 192, bit_depth=bd, intra_cu_p=0.4, weighted=(i == 2))
        c.chroma_idc = idc
        c.pic_flags |= abi.PIC_CONSTRAINED_INTRA
        if i == 3:
            c.regions = 1
        s.add(c)
    run_yuv(dec, s.pictures(), f"constrained intra {bd}-bit idc {idc}")


# --- native YCbCr canvas output (decode_heic_yuv of a grid) -----------------
@pytest.mark.parametrize("bd,idc", [(10, 1), (8, 1), (8, 2), (12, 3), (10, 0)])
def test_yuv_canvas_grid(dec, bd, idc):
    from hpvcd_b200.gpu import yuv_canvas_planes
    g = synth.make_grid(1100, 700, seed=600 + bd + idc, bit_depth=bd, chroma_idc=idc)
    pics = g.synth.pictures()
    out, keep = synth.grid_output(g)
    out.kind = abi.OUT_YUV_CANVAS
    t = dec.submit(pics, out)
    dec.wait(t)
    got = dec.read(t)
    _, ref = O.decode_batch(pics, out, want_planes=False)
    assert got.size == ref.size and np.array_equal(got, ref)
    (Y, Cb, Cr), = yuv_canvas_planes(pics, out, got)
    assert Y.shape == (700, 1100)


def test_yuv_canvas_multi_and_plan():
    import ctypes as C
    from hpvcd_b200.gpu import yuv_canvas_planes
    s = synth.SynthSet()
    pics, places, canv = [], [], []
    for k, (seed, w, h, bd, idc) in enumerate([(1, 700, 500, 8, 1), (2, 512, 512, 10, 3), (3, 300, 900, 8, 2)]):
        p, pl = _image(620 + seed, w, h, bd, idc, s)
        pics += p
        places += [(x, y, cw, ch, k) for (x, y, cw, ch) in pl]
        canv.append(abi.Canvas(w, h, 0, 0))
    pl_arr = (abi.TilePlace * len(places))(*[abi.TilePlace(*t) for t in places])
    cv_arr = (abi.Canvas * len(canv))(*canv)
    out = abi.Output(abi.OUT_YUV_CANVAS, 0, 0, 0, 0, C.cast(pl_arr, C.c_void_p), None, 0, len(canv),
                     C.cast(cv_arr, C.c_void_p))
    _, ref = O.decode_batch(pics, out, want_planes=False)
    plan = DevicePlan(pics, out)
    st = torch.cuda.Stream()          # graph capture needs a non-default stream
    with torch.cuda.stream(st):
        plan.launch(abi.STAGE_ALL | abi.STAGE_GRAPH, st)
        plan.launch(abi.STAGE_ALL | abi.STAGE_GRAPH, st)
    torch.cuda.synchronize()
    ptr, nb = plan.canvas_ptr()
    got = np.empty(nb, np.uint8)
    abi.check(abi.lib().hpvcd_copy(got.ctypes.data_as(C.c_void_p), C.c_void_p(ptr), nb, None), "copy")
    assert nb == ref.size and np.array_equal(got, ref)
    assert [y.shape for y, _, _ in yuv_canvas_planes(pics, out, got)] == [(500, 700), (512, 512), (900, 300)]
    plan.close()


def test_yuv_canvas_rejects_mixed_formats(dec):
    s = synth.SynthSet()
    s.add(synth.intra_cfg(630, 256, 256, bit_depth=8, chroma_idc=1))
    s.add(synth.intra_cfg(631, 256, 256, bit_depth=10, chroma_idc=1))
    pics = s.pictures()
    g = synth.Grid(512, 256, 256, s, [(0, 0, 256, 256), (256, 0, 256, 256)])
    out, keep = synth.grid_output(g)
    out.kind = abi.OUT_YUV_CANVAS
    with pytest.raises(abi.HpvcdError) as e:
        dec.submit(pics, out)
    assert e.value.status == abi.ERR_INVALID_ARG


def test_rgb_with_alpha_and_gain_map_canvases(dec):
    """One submit: a 10-bit grid image to RGB8, its 8-bit 4:0:0 alpha plane
    and a half-size 4:2:0 gain map at native depth (CANVAS_NATIVE canvases),
    also DMA'd straight into per-canvas page-locked buffers."""
    import ctypes as C
    from hpvcd_b200.gpu import canvas_views, pinned_empty
    s = synth.SynthSet()
    W, H = 1100, 700
    img, img_pl = _image(640, W, H, 10, 1, s)
    alpha, alpha_pl = _image(641, W, H, 8, 0, s)
    gm, gm_pl = _image(642, W // 2, H // 2, 10, 1, s)
    pics = img + alpha + gm
    places = ([(x, y, cw, ch, 0) for (x, y, cw, ch) in img_pl] + [(x, y, cw, ch, 1) for (x, y, cw, ch) in alpha_pl]
              + [(x, y, cw, ch, 2) for (x, y, cw, ch) in gm_pl])
    canv = [abi.Canvas(W, H, abi.MATRIX_SMPTE170M, 1), abi.Canvas(W, H, abi.CANVAS_NATIVE, 0),
            abi.Canvas(W // 2, H // 2, abi.CANVAS_NATIVE, 0)]
    pl_arr = (abi.TilePlace * len(places))(*[abi.TilePlace(*t) for t in places])
    cv_arr = (abi.Canvas * 3)(*canv)
    out = abi.Output(abi.OUT_RGB8, 0, 0, 0, 0, C.cast(pl_arr, C.c_void_p), None, 0, 3, C.cast(cv_arr, C.c_void_p))
    _, ref = O.decode_batch(pics, out, want_planes=False)
    t = dec.submit(pics, out)
    dec.wait(t)
    got = dec.read(t)
    assert got.size == ref.size and np.array_equal(got, ref)
    rgb, (a, acb, acr), (gy, gcb, gcr) = canvas_views(pics, out, got)
    assert rgb.shape == (H, W, 3) and a.shape == (H, W) and a.dtype == np.uint8 and acb.size == 0
    assert gy.shape == (H // 2, W // 2) and gy.dtype == np.uint16 and gcb.shape == (H // 4, W // 4)
    # the same into one page-locked buffer per canvas
    sizes = [v.nbytes if isinstance(v, np.ndarray) else sum(x.nbytes for x in v) for v in (rgb, (a, acb, acr),
                                                                                           (gy, gcb, gcr))]
    bufs = [pinned_empty(nb) for nb in sizes]
    dsts = (C.c_void_p * 3)(*[b.ctypes.data for b, _ in bufs])
    out.canvas_dst = C.cast(dsts, C.c_void_p)
    t = dec.submit(pics, out)
    dec.wait(t)
    assert abi.lib().hpvcd_gpu_read(dec._h, t, None, 0) == abi.OK  # nothing to copy: already in place
    assert np.array_equal(np.concatenate([b for b, _ in bufs]), ref)


# --- orientation (irot / imir) of the output canvases ------------------------
@pytest.mark.parametrize("orient", [2, 3, 4, 5, 6, 8])
def test_oriented_canvases(dec, orient):
    import ctypes as C
    s = synth.SynthSet()
    W, H = 1100, 700
    img, img_pl = _image(650 + orient, W, H, 10, 1, s)
    alpha, alpha_pl = _image(660 + orient, W, H, 8, 0, s)
    pics = img + alpha
    places = [(x, y, cw, ch, 0) for (x, y, cw, ch) in img_pl] + [(x, y, cw, ch, 1) for (x, y, cw, ch) in alpha_pl]
    canv = [abi.Canvas(W, H, abi.MATRIX_BT709, 0, orient), abi.Canvas(W, H, abi.CANVAS_NATIVE, 0, orient)]
    pl_arr = (abi.TilePlace * len(places))(*[abi.TilePlace(*t) for t in places])
    cv_arr = (abi.Canvas * 2)(*canv)
    out = abi.Output(abi.OUT_RGB8, 0, 0, 0, 0, C.cast(pl_arr, C.c_void_p), None, 0, 2, C.cast(cv_arr, C.c_void_p))
    _, ref = O.decode_batch(pics, out, want_planes=False)
    t = dec.submit(pics, out)
    dec.wait(t)
    got = dec.read(t)
    assert got.size == ref.size and np.array_equal(got, ref)
    g = synth.make_grid(1100, 700, seed=670 + orient, bit_depth=8, chroma_idc=2)
    out2, keep = synth.grid_output(g)
    out2.kind = abi.OUT_YUV_CANVAS
    out2.orientation = orient
    p2 = g.synth.pictures()
    _, ref2 = O.decode_batch(p2, out2, want_planes=False)
    t = dec.submit(p2, out2)
    dec.wait(t)
    assert np.array_equal(dec.read(t), ref2)


# --- I_PCM coding units ------------------------------------------------------
@pytest.mark.parametrize("bd,idc", [(8, 1), (10, 2), (12, 3), (10, 0)])
def test_pcm_cus(dec, bd, idc):
    s = synth.SynthSet()
    c = synth.intra_cfg(710 + bd + idc, 320, 256, bit_depth=bd, chroma_idc=idc)
    c.pcm_p = 0.3
    s.add(c)
    pics = s.pictures()
    tus = np.ctypeslib.as_array((C_u8 * (pics[0].n_tus * 16)).from_address(pics[0].tus)).view(abi.TU_DTYPE)
    assert (tus["flags"] & abi.TU_PCM).any()
    run_yuv(dec, pics, f"I_PCM {bd}-bit idc {idc}")


def test_pcm_in_inter_pictures(dec):
    s = synth.SynthSet()
    c0 = synth.intra_cfg(720, 320, 192, bit_depth=8)
    c0.pcm_p = 0.2
    s.add(c0)
    for i in range(1, 4):
        c = synth.inter_cfg(720 + i, 320, 192, intra_cu_p=0.4, weighted=(i == 2))
        c.pcm_p = 0.3
        s.add(c)
    run_yuv(dec, s.pictures(), "I_PCM in inter pictures")


# --- error paths of the added tools ------------------------------------------
def test_added_tools_reject_malformed_inputs(dec):
    import ctypes as C
    from hpvcd_b200.gpu import Dpb
    # cross-component chroma TB whose TU has no matching luma record: the
    # kernel's own check reports it, nothing is written out of place
    s = synth.SynthSet()
    c = synth.intra_cfg(730, 128, 128, bit_depth=10, chroma_idc=3)
    c.ccp_p = 0.9
    s.add(c)
    p = s.picture(0)
    tus = np.ctypeslib.as_array((C_u8 * (p.n_tus * 16)).from_address(p.tus)).view(abi.TU_DTYPE).copy()
    k = int(np.flatnonzero((tus["comp"] > 0) & (tus["res_scale"] != 0))[0])
    for back in (1, 2, 3):
        if k - back >= 0 and tus["comp"][k - back] == 0:
            tus["x"][k - back] += 4          # the luma record moves away
    q = abi.Picture()
    C.pointer(q)[0] = p
    q.tus = tus.ctypes.data
    with pytest.raises(abi.HpvcdError) as e:
        t = dec.submit([q])
        dec.wait(t)
        dec.read(t)
    assert e.value.status == abi.ERR_BITSTREAM
    # constrained intra prediction needs the cells
    q2 = abi.Picture()
    C.pointer(q2)[0] = p
    q2.flags |= abi.PIC_CONSTRAINED_INTRA
    q2.flags &= ~abi.PIC_DEBLOCK
    q2.cells = None
    with pytest.raises(abi.HpvcdError) as e:
        dec.submit([q2])
    assert e.value.status == abi.ERR_INVALID_ARG
    # a DPB store into an entry the DPB does not have
    q3 = abi.Picture()
    C.pointer(q3)[0] = p
    q3.flags = (p.flags & ~abi.PIC_CROSS_COMPONENT) | abi.PIC_STORE_DPB(5)
    with GpuDecoder(0) as d2, Dpb(0, entries=2) as dpb:
        d2.set_dpb(dpb)
        with pytest.raises(abi.HpvcdError) as e:
            d2.submit([q3])
        assert e.value.status == abi.ERR_INVALID_ARG
        d2.set_dpb(None)
    # an output kind that does not exist
    g = synth.make_grid(256, 256, seed=731, bit_depth=8, tile=256)
    out, keep = synth.grid_output(g)
    out.kind = 7
    with pytest.raises(abi.HpvcdError) as e:
        dec.submit(g.synth.pictures(), out)
    assert e.value.status == abi.ERR_INVALID_ARG
