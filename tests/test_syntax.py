"""Host syntax decode (include/hpvcd_syntax.h) against the seeded CABAC writer.

The reference's CABAC engine and coding-tree syntax (src/cabac/engine.rs,
src/cabac/residual_full.rs:392, src/decode.rs:1507-3620) cannot run here (no
Rust toolchain) and it ships no coded bitstreams for this path, so the
decoder is checked against an independent writer: the generator draws the
picture (CU / TU quadtrees, intra modes, QPs, levels, SAO), writes it as the
slice data of one I slice (csrc/synth.cpp SliceWriter) and keeps the flat
buffers that slice stands for.  The decoder (csrc/syntax.cpp) parses the
bytes back; every flat buffer must come out byte for byte.  Writer and
decoder share only the normative tables (csrc/cabac_tables.h).  On top, the
CPU oracle decodes the parsed buffers to the same pixels as the generated
ones (bitstream -> pixels), and malformed slices end in a status code.

No GPU needed.
"""
import ctypes as C

import numpy as np
import pytest

from hpvcd_b200 import abi, synth
from hpvcd_b200.syntax import SyntaxPicture, decode_batch


def flat_buffers(p: abi.Picture) -> dict:
    g = synth.geometry(p)
    ctbs = g["ctb_cols"] * g["ctb_rows"]
    out = {f: getattr(p, f) for f in ("width", "height", "chroma_idc", "bit_depth_y", "bit_depth_c", "log2_ctb",
                                       "flags", "beta_offset_div2", "tc_offset_div2", "pps_cb_qp_offset",
                                       "pps_cr_qp_offset", "n_tus", "n_pus", "n_coeffs")}
    out["tus"] = C.string_at(p.tus, p.n_tus * 16)
    out["ctu_tu_start"] = C.string_at(p.ctu_tu_start, (ctbs + 1) * 4)
    out["coeffs"] = C.string_at(p.coeffs, p.n_coeffs * 2) if p.n_coeffs else b""
    out["cells"] = C.string_at(p.cells, g["gw"] * g["gh"] * 4)
    out["sao"] = C.string_at(p.sao, ctbs * 36) if p.sao else None
    out["scaling"] = C.string_at(p.scaling, C.sizeof(abi.Scaling)) if p.scaling else None
    return out


def assert_same(gen: abi.Picture, dec: abi.Picture):
    a, b = flat_buffers(gen), flat_buffers(dec)
    for k in a:
        if a[k] == b[k]:
            continue
        if k == "tus":
            ta, tb = np.frombuffer(a[k], abi.TU_DTYPE), np.frombuffer(b[k], abi.TU_DTYPE)
            i = next(i for i in range(min(len(ta), len(tb))) if ta[i].tobytes() != tb[i].tobytes())
            raise AssertionError(f"TB record {i}: written {ta[i]} parsed {tb[i]}")
        raise AssertionError(f"{k} differs")


def roundtrip(cfg: abi.SynthCfg):
    s = synth.SynthSet()
    cfg.bitstream = 1
    s.add(cfg)
    sp, data = s.slice(0)
    d = SyntaxPicture.decode(sp, data)
    return s, d, sp, data


CASES = {
    "tile_512_10bit_420": dict(seed=1, width=512, height=512, bit_depth=10, chroma_idc=1),
    "8bit_420_small": dict(seed=2, width=64, height=64, bit_depth=8, chroma_idc=1),
    "8bit_444": dict(seed=3, width=256, height=192, bit_depth=8, chroma_idc=3),
    "mono_ragged": dict(seed=4, width=200, height=120, bit_depth=8, chroma_idc=0),
    "tskip_tqbypass": dict(seed=5, width=256, height=256, bit_depth=10, chroma_idc=1, tskip_p=0.3, tqb_p=0.2),
    "12bit": dict(seed=7, width=256, height=256, bit_depth=12, chroma_idc=1),
    "no_sao_no_deblock": dict(seed=8, width=192, height=128, bit_depth=8, chroma_idc=1, sao=False, deblock=False),
    "scaling_lists": dict(seed=9, width=128, height=128, bit_depth=10, chroma_idc=1, scaling=True),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_parsed_buffers_equal_written(name):
    s, d, sp, data = roundtrip(synth.intra_cfg(**CASES[name]))
    assert len(data) > 16 and d.bins > 8 * len(data) // 2
    assert_same(s.picture(0), d.picture())


@pytest.mark.parametrize("log2_ctb", [4, 5, 6])
@pytest.mark.parametrize("hiding", [0, 1])
def test_ctb_sizes_and_sign_hiding(log2_ctb, hiding):
    c = synth.intra_cfg(100 + log2_ctb * 2 + hiding, 320, 192, bit_depth=8, chroma_idc=1, tskip_p=0.2)
    c.log2_ctb = log2_ctb
    c.sign_hiding = hiding
    s, d, sp, _ = roundtrip(c)
    assert bool(sp.flags & abi.SLICE_SIGN_HIDING) == bool(hiding)
    assert_same(s.picture(0), d.picture())


def test_seeded_mix():
    """Sizes, bit depths, chroma formats, CTB sizes, QP offsets and tools drawn per seed."""
    for seed in range(10, 34):
        c = synth.intra_cfg(seed, 8 * (8 + seed % 50), 8 * (8 + (seed * 7) % 50), bit_depth=8 + 2 * (seed % 3),
                            chroma_idc=[0, 1, 3][seed % 3], tskip_p=0.2 * (seed % 2),
                            tqb_p=0.1 * (seed % 4 == 0))
        c.log2_ctb = 4 + seed % 3
        c.tskip_log2_max = 2 + seed % 4
        c.sign_hiding = seed % 2
        c.cb_qp_offset = seed % 5 - 2
        c.cr_qp_offset = 2 - seed % 5
        c.qp_min, c.qp_max = 10 + seed % 7, 40 + seed % 9
        s, d, _, _ = roundtrip(c)
        assert_same(s.picture(0), d.picture())


def test_writer_normalises_what_the_syntax_cannot_carry():
    """A CU without coded residual has no cu_qp_delta: its QP is the
    prediction; SAO fields the syntax does not code are zero."""
    c = synth.intra_cfg(41, 256, 256, bit_depth=10, chroma_idc=1, cbf_p=0.3)
    plain = synth.SynthSet()
    plain.add(c)
    s, d, sp, _ = roundtrip(c)
    a, b = flat_buffers(plain.picture(0)), flat_buffers(s.picture(0))
    assert a["coeffs"] == b["coeffs"]                  # levels untouched (no sign hiding)
    assert a["cells"] != b["cells"]                    # some QPs became the prediction
    ta, tb = np.frombuffer(a["tus"], abi.TU_DTYPE), np.frombuffer(b["tus"], abi.TU_DTYPE)
    assert (ta[["x", "y", "log2n", "comp", "flags", "mode", "nx"]] == tb[["x", "y", "log2n", "comp", "flags",
                                                                           "mode", "nx"]]).all()
    assert sp.flags & abi.SLICE_CU_QP_DELTA and sp.flags & abi.SLICE_EBSP


def test_grid_batch_decode_and_pixels_from_bitstream():
    """The config-1 grid's tiles: 48 slices parsed on a thread pool give the
    flat buffers the benchmark decodes; three of them decode on the CPU
    oracle to the same pixels as the generated buffers."""
    from oracle import oracle as O
    g = synth.config1_grid(seed=11)
    slices = synth.grid_slices(g)
    assert len(slices) == 48
    parsed = decode_batch(slices, threads=4)
    gen = g.synth.pictures()
    for a, d in zip(gen, parsed):
        assert_same(a, d.picture())
    for i in (0, 7, 47):
        ref, _ = O.decode_batch([gen[i]])
        got, _ = O.decode_batch([parsed[i].picture()])
        for c in range(3):
            assert np.array_equal(ref[0][c], got[0][c])
    for d in parsed:
        d.close()


def test_unescaped_bytes_parse_too():
    s, d, sp, data = roundtrip(synth.intra_cfg(12, 128, 128, bit_depth=8, chroma_idc=1))
    rbsp, zeros, i = bytearray(), 0, 0
    for b in data:  # strip emulation_prevention_three_byte
        if zeros >= 2 and b == 3:
            zeros = 0
            continue
        zeros = zeros + 1 if b == 0 else 0
        rbsp.append(b)
    sp2 = abi.SliceParams()
    C.pointer(sp2)[0] = sp
    sp2.flags &= ~abi.SLICE_EBSP
    d2 = SyntaxPicture.decode(sp2, bytes(rbsp))
    assert_same(s.picture(0), d2.picture())


def test_malformed_slices_end_in_a_status():
    s, d, sp, data = roundtrip(synth.intra_cfg(13, 256, 256, bit_depth=8, chroma_idc=1))
    for cut in (0, 1, len(data) // 3, len(data) - 40):
        with pytest.raises(abi.HpvcdError) as e:
            SyntaxPicture.decode(sp, data[:cut])
        assert e.value.status == abi.ERR_BITSTREAM
    rng = np.random.default_rng(5)
    for k in range(20):  # arbitrary bytes: a status or a picture, never a crash
        junk = rng.integers(0, 256, size=int(rng.integers(1, 4000)), dtype=np.uint8).tobytes()
        try:
            SyntaxPicture.decode(sp, junk).close()
        except abi.HpvcdError as e:
            assert e.status == abi.ERR_BITSTREAM
    bad = abi.SliceParams()
    C.pointer(bad)[0] = sp
    bad.chroma_idc = 2
    with pytest.raises(abi.HpvcdError) as e:
        SyntaxPicture.decode(bad, data)
    assert e.value.status == abi.ERR_UNSUPPORTED
    bad.chroma_idc = 1
    bad.width = 100  # not a multiple of the minimum CB
    with pytest.raises(abi.HpvcdError) as e:
        SyntaxPicture.decode(bad, data)
    assert e.value.status == abi.ERR_INVALID_ARG


def test_writer_rejects_what_one_i_slice_cannot_hold():
    for kw in (dict(chroma_idc=2), ):
        c = synth.intra_cfg(14, 128, 128, bit_depth=8, **kw)
        c.bitstream = 1
        with pytest.raises(abi.HpvcdError):
            synth.SynthSet().add(c)
    c = synth.inter_cfg(15, 128, 128)
    c.bitstream = 1
    with pytest.raises(abi.HpvcdError):
        synth.SynthSet().add(c)
