"""Pin the CPU oracle against the reference's own unit-test known answers.

The reference (hpvcd, Rust) cannot be compiled in this image, and it ships no
golden decoded images.  Its in-tree unit tests are the only known answers for
the reconstruction path; each test below restates one of them (cited by
file:line) against the oracle, plus algebraic cross-checks of the transform
(the partial butterfly of transform.rs must equal the plain matrix product of
the H.265 basis) and an independent pure-Python restatement of the luma
deblocking filter on the reference's own step-edge inputs.
"""
import numpy as np
import pytest

from oracle import oracle as O


# --- transform.rs:1389-1395 extended_precision_uses_component_dynamic_range
def test_max_log2_transform_dynamic_range():
    L = O.lib()
    assert L.orc_max_log2_tr_range(8, 0) == 15
    assert L.orc_max_log2_tr_range(8, 1) == 15
    assert L.orc_max_log2_tr_range(10, 1) == 16
    assert L.orc_max_log2_tr_range(12, 1) == 18


# --- transform.rs:1397-1411 extended_dequant_preserves_values_above_i16
def test_extended_dequant_preserves_values_above_i16():
    p = O.dequant_params(4, 75, 12, ext=True)
    assert p.clip_min == -262_144 and p.clip_max == 262_143
    out = O.dequant(np.ones(16, np.int32), 4, p)
    assert out[0] > 32767
    assert np.all(out == out[0])


# --- transform.rs:1413-1419 extended_transform_skip_uses_extended_dynamic_range
def test_transform_skip_shift():
    assert O.ts_params(32, 0, 12, ext=False).tr_shift == -2
    assert O.ts_params(32, 0, 12, ext=True).tr_shift == 1


# --- transform.rs:1421-1429 extended_inverse_transform_accepts_full_12bit_range
def test_extended_inverse_transform_full_range():
    c = np.zeros(16, np.int32)
    c[0] = (1 << 18) - 1
    out = O.inv_dct(c, 4, 12, max_range=18, nx=1)
    assert np.all(out != np.iinfo(np.int32).min)
    assert np.any(out != 0)


# --- transform.rs:1441-1664 validate_dequant_backend, restated as the
# i16-storage kernels agreeing with the i32 ones truncated to i16, over the
# same bit depths, QPs and the reference's SAFE / STRESS level tables.
SAFE = [0, 1, -1, 2, -2, 3, -3, 7, -7, 15, -15, 31, -31, 63, -63, 5]
STRESS = [0, 1, -1, 255, -255, 4095, -4095, 32767, -32767, 100_000, -100_000, 1_000_000,
          -1_000_000, 17, -33, 511]
SCALING_COEFFS = np.array([0, 1, 2, 3, 4, 8, 16, 32, 64, 127, 255, 17, 5, 9, 23, 41] + [16] * 48,
                          np.uint8)


@pytest.mark.parametrize("bd", [8, 10, 12])
@pytest.mark.parametrize("stress", [False, True])
def test_dequant_i16_vs_i32(bd, stress):
    levels = np.array(STRESS if stress else SAFE, np.int32)
    max_qp = 51 + 6 * (bd - 8)
    for qp in (0, max_qp // 2, max_qp):
        tp = O.ts_params(4, qp, bd)
        for scaling in (None, SCALING_COEFFS):
            a32 = O.dequant(levels, 4, tp.dq, scaling)
            a16 = O.dequant(levels, 4, tp.dq, scaling, i16=True)
            assert np.array_equal(a16, a32.astype(np.int16).astype(np.int32))
            t32 = O.dequant(levels, 4, tp, scaling, ts=True)
            t16 = O.dequant(levels, 4, tp, scaling, ts=True, i16=True)
            assert np.array_equal(t16, t32.astype(np.int16).astype(np.int32))
            # clip: every dequantised value is inside the normative range
            assert a32.min() >= tp.dq.clip_min and a32.max() <= tp.dq.clip_max


def test_dequant_formula_spot_values():
    # transform.rs:764-776: clip((clip(l) * factor + add) >> shift)
    p = O.dequant_params(8, 30, 8)  # bd_shift = 8 + 3 + 10 - 15 = 6
    assert p.shift == 6 and p.add == 32
    assert p.factor == 40 * (1 << 5) * 16
    out = O.dequant(np.array([1, -1, 3, 0] + [0] * 60, np.int32), 8, p)
    f = p.factor
    assert out[0] == (1 * f + 32) >> 6
    assert out[1] == (-f + 32) >> 6
    assert out[2] == (3 * f + 32) >> 6


# --- reconstruct.rs:255-280 narrow_i32_to_i16 saturates
def test_narrow_saturates():
    src = [np.iinfo(np.int32).min, -32769, -32768, -1, 0, 1, 32767, 32768, np.iinfo(np.int32).max]
    d = O.narrow_i32_to_i16(src)
    assert d.tolist() == [-32768, -32768, -32768, -1, 0, 1, 32767, 32767, 32767]


# --- intra.rs:378-406 disabled_reference_smoothing_preserves_samples
def test_intra_smoothing_disabled_preserves():
    n = 8
    above = np.array([100 + i * i for i in range(2 * n + 1)], np.uint16)
    left = np.array([100 + 3 * i * i for i in range(2 * n + 1)], np.uint16)
    fa, fl = O.intra_filter(above, left, n, 0, True, False, True, 10)
    assert np.array_equal(fa, above) and np.array_equal(fl, left)


# --- intra.rs:408-448 disabled_reference_smoothing_skips_strong_filter
def test_intra_strong_filter_disabled_and_enabled():
    n = 32
    above = np.full(2 * n + 1, 777, np.uint16)
    left = np.full(2 * n + 1, 555, np.uint16)
    above[0], above[n], above[2 * n] = 100, 200, 300
    left[0], left[n], left[2 * n] = 100, 250, 400
    fa, fl = O.intra_filter(above, left, n, 0, True, False, True, 10)
    assert np.array_equal(fa, above) and np.array_equal(fl, left)
    fa, fl = O.intra_filter(above, left, n, 0, True, True, True, 10)
    assert not np.array_equal(fa, above) and not np.array_equal(fl, left)


# --- mc.rs:742-758 weighted prediction known answers
def test_weighted_uni_107():
    assert O.uni_mc_weighted([100 << 4], 1, 1, 10, 1, 7, 0)[0] == 107


def test_weighted_bi_152():
    assert O.bi_mc_weighted([100 << 4], [200 << 4], 1, 1, 10, 1, 7, 1, -3, 0)[0] == 152


# --- inter.rs:303-330 weighted-prediction offset normalisation
def test_wp_offsets():
    L = O.lib()
    assert L.orc_normalize_luma_offset(7, 8, 0) == 7
    assert L.orc_normalize_luma_offset(7, 10, 0) == 28
    assert L.orc_normalize_luma_offset(-128, 12, 0) == -2048
    assert L.orc_normalize_luma_offset(7, 10, 1) == 7
    assert L.orc_normalize_luma_offset(511, 10, 1) == 511
    assert L.orc_normalize_luma_offset(-512, 10, 1) == -512
    assert L.orc_derive_chroma_offset(3, 5, 2, 10, 0) == -116
    assert L.orc_derive_chroma_offset(3, 5, 2, 10, 1) == -125


# --- decode.rs:8284-8311 QP derivations
def test_qp_helpers():
    L = O.lib()
    assert L.orc_qp_prime(-12, 10) == 0
    assert L.orc_qp_prime(-24, 12) == 0
    assert L.orc_qp_prime(0, 10) == 12
    assert L.orc_qp_prime(51, 12) == 75
    assert L.orc_qpc(-12, 1, 10) == -12
    assert L.orc_qpc(-24, 1, 12) == -24
    assert L.orc_qp_prime(L.orc_qpc(-12, 1, 10), 10) == 0
    assert L.orc_qp_prime(L.orc_qpc(-24, 3, 12), 12) == 0
    assert L.orc_clamp_qpy(-1, 8) == 0
    assert L.orc_clamp_qpy(-12, 10) == -12
    assert L.orc_clamp_qpy(-13, 10) == -12
    assert L.orc_clamp_qpy(-24, 12) == -24
    assert L.orc_clamp_qpy(90, 12) == 51
    # H.265 Table 8-10 (decode.rs:7599-7613) for 4:2:0
    assert [L.orc_qpc(q, 1, 8) for q in (29, 30, 34, 35, 39, 43, 44, 57)] == [
        29, 29, 33, 33, 35, 37, 38, 51]


# --- decode.rs:8313-8331 plane_prediction_load_copies_rows_and_zero_pads_edges
def test_load_plane_block_clipped():
    import ctypes as C
    plane = np.arange(20, dtype=np.uint16)
    full = np.full(9, 65535, np.uint16)
    O.lib().orc_load_block_clipped(plane.ctypes.data_as(C.c_void_p), 5, 5, 4, 1, 1, 3,
                                   full.ctypes.data_as(C.c_void_p))
    assert full.tolist() == [6, 7, 8, 11, 12, 13, 16, 17, 18]
    clipped = np.full(16, 65535, np.uint16)
    O.lib().orc_load_block_clipped(plane.ctypes.data_as(C.c_void_p), 5, 5, 4, 3, 2, 4,
                                   clipped.ctypes.data_as(C.c_void_p))
    assert clipped.tolist() == [13, 14, 0, 0, 18, 19, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0]


# --- sao.rs:1049-1064 gated_eo_applies_when_all_available (all neighbours in picture)
def test_sao_eo_local_min():
    src = np.array([10, 5, 10, 5], np.uint16)
    dst = src.copy()
    O.sao_edge(dst, src, 4, 1, 0, 0, 4, 1, [7, 0, 0, 0], 0, 8)
    assert dst[1] == 12
    assert dst[0] == 10 and dst[3] == 5  # picture-border samples untouched (sao.rs:304-311)


# --- yuv.rs:700-756 identity matrix known answers
def test_yuv_identity_full_range():
    out = O.yuv_to_rgb16([20, 21], [30, 31], [10, 11], 2, 1, 3, 8, 2, 1, 0, True)
    assert out.tolist() == [10, 20, 30, 11, 21, 31]


def test_yuv_identity_12bit():
    out = O.yuv_to_rgb16([0x123], [0x234], [0x345], 1, 1, 3, 12, 1, 1, 0, True)
    assert out.tolist() == [0x345, 0x123, 0x234]


def test_yuv_identity_limited_range():
    out = O.yuv_to_rgb16([16, 235], [16, 240], [16, 240], 2, 1, 3, 8, 2, 1, 0, False)
    assert out.tolist() == [0, 0, 0, 255, 255, 255]


# --- transform.rs:67-413: the odd-part rows and the 4-point core are entries
# of the H.265 basis matrix the oracle generates.
def test_dct_basis_matches_reference_rows():
    t4, t8, t16, t32 = (O.dct_matrix(n) for n in (4, 8, 16, 32))
    assert t4[:, 0].tolist() == [64, 83, 64, 36]   # idct_raw_4: 64, 83, 64, 36
    assert t8[1::2, 0].tolist() == [89, 75, 50, 18]  # idct_odd_8 row 0
    assert t8[1::2, 3].tolist() == [18, -50, 75, -89]  # idct_odd_8 row 3
    assert t16[1::2, 0].tolist() == [90, 87, 80, 70, 57, 43, 25, 9]  # idct_odd_16 row 0
    assert t16[1::2, 7].tolist() == [9, -25, 43, -57, 70, -80, 87, -90]  # row 7
    assert t32[1::2, 0].tolist() == [90, 90, 88, 85, 82, 78, 73, 67, 61, 54, 46, 38, 31, 22, 13, 4]
    assert t32[1::2, 15].tolist() == [4, -13, 22, -31, 38, -46, 54, -61, 67, -73, 78, -82, 85,
                                      -88, 90, -90]  # idct_odd_32 row 15
    for t in (t4, t8, t16, t32):  # near-orthogonality of the integer basis (within 1%)
        g = (t @ t.T).astype(np.float64)
        norm = 64.0 * 64.0 * t.shape[0]
        assert np.all(np.abs(np.diag(g) - norm) < 0.01 * norm)
        assert np.all(np.abs(g - np.diag(np.diag(g))) < 0.01 * norm)


def _matrix_idct(coeff, n, bd, nx, i16):
    t = O.dct_matrix(n)
    c = coeff.reshape(n, n).astype(np.int64).copy()
    c[:, nx:] = 0
    tmp = np.clip((t.T @ c + 64) >> 7, -32768, 32767)  # columns
    sh = 20 - bd
    out = (tmp @ t + (1 << (sh - 1))) >> sh  # rows
    out = out.reshape(-1)
    return out.astype(np.int16).astype(np.int64) if i16 else out


@pytest.mark.parametrize("n", [4, 8, 16, 32])
@pytest.mark.parametrize("bd", [8, 10])
def test_butterfly_equals_matrix_form(n, bd):
    rng = np.random.default_rng(n * 100 + bd)
    for trial in range(20):
        c = rng.integers(-32768, 32768, n * n).astype(np.int32)
        if trial % 2:
            c[rng.random(n * n) < 0.85] = 0
        nx = int(rng.integers(1, n + 1))
        got = O.inv_dct(c, n, bd, nx=nx, i16=bd == 8)
        assert np.array_equal(got.astype(np.int64), _matrix_idct(c, n, bd, nx, bd == 8))


DST4 = np.array([[29, 55, 74, 84], [74, 74, 0, -74], [84, -29, -74, 55], [55, -84, 74, -29]],
                np.int64)


def test_dst_equals_matrix_form():
    rng = np.random.default_rng(7)
    for bd in (8, 10):
        for _ in range(50):
            c = rng.integers(-32768, 32768, 16).astype(np.int32)
            tmp = np.clip((DST4.T @ c.reshape(4, 4).astype(np.int64) + 64) >> 7, -32768, 32767)
            sh = 20 - bd
            ref = ((tmp @ DST4 + (1 << (sh - 1))) >> sh).reshape(-1)
            if bd == 8:
                ref = ref.astype(np.int16).astype(np.int64)
            assert np.array_equal(O.inv_dst4(c, bd, i16=bd == 8).astype(np.int64), ref)


# --- deblock.rs:1220-1287: the reference's step-edge inputs, decisions and
# tc values, checked against an independent restatement of H.265 8.7.2.5.7.
def _py_apply(p, q, dec, tc, maxv):
    p = list(p)
    q = list(q)  # p[0] = p0 ... p[3] = p3
    P, Q = p[:], q[:]
    clip = lambda v, lo, hi: max(lo, min(hi, v))
    if dec == 1:
        p0, p1, p2, p3 = p
        q0, q1, q2, q3 = q
        c = lambda o, v: clip(clip(v, o - 2 * tc, o + 2 * tc), 0, maxv)
        P[0] = c(p0, (p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3)
        P[1] = c(p1, (p2 + p1 + p0 + q0 + 2) >> 2)
        P[2] = c(p2, (2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3)
        Q[0] = c(q0, (p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3)
        Q[1] = c(q1, (p0 + q0 + q1 + q2 + 2) >> 2)
        Q[2] = c(q2, (p0 + q0 + q1 + 3 * q2 + 2 * q3 + 4) >> 3)
    else:
        d = dec - 2
        do_p1, do_q1 = (d >> 1) & 1, d & 1
        p0, p1, p2 = p[0], p[1], p[2]
        q0, q1, q2 = q[0], q[1], q[2]
        delta0 = (9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4
        if abs(delta0) < tc * 10:
            delta = clip(delta0, -tc, tc)
            P[0] = clip(p0 + delta, 0, maxv)
            Q[0] = clip(q0 - delta, 0, maxv)
            if do_p1:
                P[1] = clip(p1 + clip((((p2 + p0 + 1) >> 1) - p1 + delta) >> 1, -(tc >> 1), tc >> 1), 0, maxv)
            if do_q1:
                Q[1] = clip(q1 + clip((((q2 + q0 + 1) >> 1) - q1 - delta) >> 1, -(tc >> 1), tc >> 1), 0, maxv)
    return P, Q


@pytest.mark.parametrize("tc", [1, 2, 3, 5, 8, 14])
@pytest.mark.parametrize("maxv", [255, 1023])
def test_luma_deblock_step_edges(tc, maxv):
    w = 16
    for pv, qv in [(0, 255), (10, 240), (60, 190), (128, 132), (300, 700)]:
        pv, qv = min(pv, maxv), min(qv, maxv)
        for dec in (1, 2, 3, 4, 5):  # strong, weak(p1,q1 combos)
            for vertical in (True, False):
                if vertical:
                    base = np.where(np.arange(w)[None, :] < 8, pv, qv).repeat(4, 0).astype(np.uint16)
                else:
                    base = np.where(np.arange(16)[:, None] < 8, pv, qv).repeat(w, 1).astype(np.uint16)
                pl = np.ascontiguousarray(base.copy())
                O.apply_luma_decision(pl, w, vertical, 8, 0, dec, tc, maxv)
                for line in range(4):
                    if vertical:
                        p = [int(base[line, 7 - k]) for k in range(4)]
                        q = [int(base[line, 8 + k]) for k in range(4)]
                        gp = [int(pl[line, 7 - k]) for k in range(4)]
                        gq = [int(pl[line, 8 + k]) for k in range(4)]
                    else:
                        p = [int(base[7 - k, line]) for k in range(4)]
                        q = [int(base[8 + k, line]) for k in range(4)]
                        gp = [int(pl[7 - k, line]) for k in range(4)]
                        gq = [int(pl[8 + k, line]) for k in range(4)]
                    P, Q = _py_apply(p, q, dec, tc, maxv)
                    assert gp == P and gq == Q, (pv, qv, dec, vertical, line)


def _constant_lists(values):
    """ScalingList::test_constant_lists (config.rs): every size's matrix
    `matrix_id` filled with values[matrix_id], DC the same."""
    s = O.abi.Scaling()
    for size_id in range(4):
        for mid, v in enumerate(values):
            for i in range(64):
                s.m[size_id][mid][i] = v
            s.dc[size_id][mid] = v
    return s


def test_scaling_list_selection_uses_prediction_mode_and_ts_size():
    # decode.rs scaling_list_selection_uses_prediction_mode_and_ts_size
    lists = _constant_lists([10, 20, 30, 40, 50, 60])
    assert O.scaling_select(lists, 1, 8, inter=False, tskip=False) == (20, 20)
    assert O.scaling_select(lists, 1, 8, inter=True, tskip=False) == (50, 50)
    assert O.scaling_select(lists, 0, 4, inter=False, tskip=True) is not None
    assert O.scaling_select(lists, 0, 8, inter=False, tskip=True) is None
    assert O.scaling_select(lists, 0, 32, inter=True, tskip=True) is None
    assert O.scaling_select(lists, 2, 32, inter=True, tskip=False) == (60, 60)


@pytest.mark.parametrize("n", [8, 16, 32])
def test_scaled_dequant_upsamples_the_8x8_list(n):
    # transform.rs:668-683: 8x8 list replicated over n/8 x n/8 blocks, DC
    # entry at (0, 0) from 16x16 up; factor = factor/16 * m.
    rng = np.random.default_rng(n)
    m8 = rng.integers(1, 256, 64).astype(np.uint8)
    dc = 77
    levels = rng.integers(-300, 300, n * n).astype(np.int32)
    p = O.dequant_params(n, 33, 10)
    got = O.dequant(levels, n, p, m8, dc=dc)
    rep = n // 8
    m = np.repeat(np.repeat(m8.reshape(8, 8), rep, 0), rep, 1).astype(np.int64).reshape(-1)
    if n >= 16:
        m[0] = dc
    f = (p.factor // 16) * m
    want = np.clip((levels.astype(np.int64) * f + p.add) >> p.shift, p.clip_min, p.clip_max)
    assert np.array_equal(got, want)


def test_rext_residual_ops():
    # decode.rs:8418-8446: rotation reverses the block; vertical RDPCM adds
    # the row above, horizontal the sample to the left; i16 storage wraps.
    r = np.arange(16, dtype=np.int32)
    assert np.array_equal(O.rext_residual_ops(r, 4, rotate=True), r[::-1])
    v = O.rext_residual_ops(r, 4, rdpcm=1).reshape(4, 4)
    assert np.array_equal(v, np.cumsum(r.reshape(4, 4), axis=0))
    h = O.rext_residual_ops(r, 4, rdpcm=0).reshape(4, 4)
    assert np.array_equal(h, np.cumsum(r.reshape(4, 4), axis=1))
    both = O.rext_residual_ops(r, 4, rotate=True, rdpcm=0).reshape(4, 4)
    assert np.array_equal(both, np.cumsum(r[::-1].reshape(4, 4), axis=1))
    big = np.full(64, 30000, np.int32)
    w = O.rext_residual_ops(big, 8, rdpcm=1, i16=True).reshape(8, 8)
    want = (np.cumsum(big.reshape(8, 8).astype(np.int64), axis=0) + 32768) % 65536 - 32768
    assert np.array_equal(w, want)
    assert np.array_equal(O.rext_residual_ops(big, 8, rdpcm=1).reshape(8, 8), np.cumsum(big.reshape(8, 8), axis=0))


@pytest.mark.parametrize("bd,idc", [(8, 1), (10, 2), (12, 3), (8, 0)])
def test_yuv_canvas_stitch_matches_planes(bd, idc):
    """lib.rs:871-991: the oracle's native YUV canvas is the tiles' planes
    copied to their grid positions (checked here against numpy slicing of
    the same decode, crops at the canvas edge included)."""
    import ctypes as C
    from hpvcd_b200 import synth
    from hpvcd_b200.gpu import yuv_canvas_planes
    g = synth.make_grid(200, 136, seed=7 + bd + idc, bit_depth=bd, chroma_idc=idc, tile=64, sao=False)
    pics = g.synth.pictures()
    out, keep = synth.grid_output(g)
    out.kind = O.abi.OUT_YUV_CANVAS
    planes, raw = O.decode_batch(pics, out)
    (Y, Cb, Cr), = yuv_canvas_planes(pics, out, raw)
    sw, sh = (2 if idc in (1, 2) else 1), (2 if idc == 1 else 1)
    want = [np.zeros(Y.shape, np.uint16), np.zeros(Cb.shape, np.uint16), np.zeros(Cr.shape, np.uint16)]
    for pl, (x, y, cw, ch) in zip(planes, g.places):
        for c in range(3 if idc else 1):
            s_w, s_h = (sw, sh) if c else (1, 1)
            W = want[c]
            dx, dy = x // s_w, y // s_h
            tw, th = -(-cw // s_w), -(-ch // s_h)
            tw, th = min(tw, W.shape[1] - dx), min(th, W.shape[0] - dy)
            W[dy:dy + th, dx:dx + tw] = pl[c][:th, :tw]
    for c, got in enumerate((Y, Cb, Cr)):
        assert np.array_equal(got.astype(np.uint16), want[c]), c


@pytest.mark.parametrize("orient", range(0, 9))
def test_orientation_of_the_oracle_canvas(orient):
    """lib.rs:2065-2200: FlipH / Rotate180 / FlipV / Rotate90 (clockwise) /
    Rotate270 move the pixels; Normal, Transpose and Transverse leave them
    (the reference's rotate_luma / rotate_buf).  Checked on RGB8 and on a
    native 4:2:0 canvas against numpy flips and rotations of the normal one."""
    from hpvcd_b200 import synth
    from hpvcd_b200.gpu import canvas_views
    g = synth.make_grid(136, 72, seed=31, bit_depth=8, chroma_idc=1, tile=64, sao=False)
    pics = g.synth.pictures()
    turn = {2: np.fliplr, 3: lambda a: np.rot90(a, 2), 4: np.flipud, 6: lambda a: np.rot90(a, -1),
            8: lambda a: np.rot90(a, 1)}.get(orient, lambda a: a)

    def planes(out, raw):
        views = canvas_views(pics, out, raw.reshape(-1))
        return [p.copy() for v in views for p in (v if isinstance(v, tuple) else (v,))]

    for kind in (O.abi.OUT_RGB8, O.abi.OUT_YUV_CANVAS):
        out, keep = synth.grid_output(g)
        out.kind = kind
        _, base = O.decode_batch(pics, out, want_planes=False)
        normal = planes(out, base)
        out.orientation = orient
        _, got = O.decode_batch(pics, out, want_planes=False)
        for p0, p1 in zip(normal, planes(out, got)):
            assert np.array_equal(turn(p0), p1)


def test_int8_level_pool_decodes_the_same():
    """HPVCD_PIC_COEFF8 is a transport format: a picture whose levels all
    fit in int8 decodes identically from the narrowed pool (intra, residual-
    only and inter pictures, 8 and 10 bit, 4:2:0 and 4:4:4), and a picture
    with a level outside [-128, 127] keeps its int16 pool."""
    from hpvcd_b200 import abi, synth
    s = synth.SynthSet()
    s.add(synth.intra_cfg(304, 160, 96, bit_depth=8))       # the inter pictures predict from it
    for i in range(1, 3):
        s.add(synth.inter_cfg(304 + i, 160, 96, bit_depth=8, weighted=(i == 2), n_refs=1))
    s.add(synth.intra_cfg(301, 192, 128, bit_depth=10, chroma_idc=1))
    s.add(synth.intra_cfg(302, 128, 128, bit_depth=8, chroma_idc=3))
    s.add(synth.residual_cfg(303, 128, 96, bit_depth=8))
    pics = s.pictures()
    want, _ = O.decode_batch(pics)
    keep = synth.narrow_coeffs(pics)
    assert len(keep) >= 4 and sum(1 for p in pics if p.flags & abi.PIC_COEFF8) == len(keep)
    got, _ = O.decode_batch(pics)
    for a, b in zip(want, got):
        for pa, pb in zip(a, b):
            assert np.array_equal(pa, pb)
    # a level beyond int8 keeps the int16 pool
    s2 = synth.SynthSet()
    s2.add(synth.intra_cfg(311, 64, 64, bit_depth=10))
    p2 = s2.pictures()
    lv = synth.coeffs_of(p2[0])
    if lv.size:
        lv[np.argmax(np.abs(lv))] = 200
        assert synth.narrow_coeffs(p2) == [] and not p2[0].flags & abi.PIC_COEFF8
