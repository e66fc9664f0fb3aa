"""Seeded synthetic inputs for the benchmark configurations.

The reference publishes no benchmark corpus for this path, and the HEIF/HEVC
files its demo reads are not shipped, so every workload is synthetic: a
seeded generator (csrc/synth.cpp) emits the flat per-picture buffers the host
syntax decode of hpvcd would produce (TB records, per-4x4 deblocking maps,
per-CTB SAO parameters, PUs) with the shapes and value distributions of the
configurations below.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi


def default_cfg() -> abi.SynthCfg:
    c = abi.SynthCfg()
    abi.synth_lib().hpvcd_synth_default_cfg(C.byref(c))
    return c


class SynthSet:
    """Owns generated pictures; descriptors point into native memory it keeps alive."""

    def __init__(self):
        self._h = C.c_void_p(abi.synth_lib().hpvcd_synth_new())
        if not self._h:
            raise MemoryError("hpvcd_synth_new failed")

    def add(self, cfg: abi.SynthCfg) -> int:
        r = abi.synth_lib().hpvcd_synth_add(self._h, C.byref(cfg))
        if r < 0:
            raise abi.HpvcdError(-r, "hpvcd_synth_add")
        return r

    def __len__(self) -> int:
        return abi.synth_lib().hpvcd_synth_count(self._h)

    def picture(self, i: int) -> abi.Picture:
        p = abi.Picture()
        abi.check(abi.synth_lib().hpvcd_synth_get(self._h, i, C.byref(p)), "hpvcd_synth_get")
        return p

    def pictures(self) -> list[abi.Picture]:
        return [self.picture(i) for i in range(len(self))]

    def slice(self, i: int) -> tuple[abi.SliceParams, bytes]:
        """Slice data of picture i written in bitstream mode (cfg.bitstream)
        and the slice parameters it was written with."""
        sp = abi.SliceParams()
        ptr, n = C.c_void_p(), C.c_uint64()
        abi.check(abi.synth_lib().hpvcd_synth_slice(self._h, i, C.byref(sp), C.byref(ptr), C.byref(n)),
                  "hpvcd_synth_slice")
        return sp, C.string_at(ptr.value, n.value)

    def close(self):
        if self._h:
            abi.synth_lib().hpvcd_synth_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Views of a descriptor's buffers (host pointers only).
# ---------------------------------------------------------------------------

def tus_of(p: abi.Picture) -> np.ndarray:
    if p.n_tus == 0:
        return np.zeros(0, abi.TU_DTYPE)
    buf = (C.c_uint8 * (p.n_tus * abi.TU_DTYPE.itemsize)).from_address(p.tus)
    return np.frombuffer(buf, dtype=abi.TU_DTYPE)


def pus_of(p: abi.Picture) -> np.ndarray:
    if p.n_pus == 0:
        return np.zeros(0, abi.PU_DTYPE)
    buf = (C.c_uint8 * (p.n_pus * abi.PU_DTYPE.itemsize)).from_address(p.pus)
    return np.frombuffer(buf, dtype=abi.PU_DTYPE)


def coeffs_of(p: abi.Picture) -> np.ndarray:
    """The picture's level pool (int16, or int8 with PIC_COEFF8)."""
    if p.n_coeffs == 0:
        return np.zeros(0, np.int16)
    if p.flags & abi.PIC_COEFF8:
        return np.frombuffer((C.c_int8 * p.n_coeffs).from_address(p.coeffs), dtype=np.int8)
    buf = (C.c_int16 * p.n_coeffs).from_address(p.coeffs)
    return np.frombuffer(buf, dtype=np.int16)


def narrow_coeffs(pics) -> list:
    """Host transport choice: every picture whose levels all lie in
    [-128, 127] gets an int8 copy of its pool (PIC_COEFF8), half the bytes
    to copy.  Returns the new pools, which must outlive the pictures' use."""
    keep = []
    for p in pics:
        if p.n_coeffs == 0 or p.flags & abi.PIC_COEFF8:
            continue
        lv = coeffs_of(p)
        if lv.min() < -128 or lv.max() > 127:
            continue
        c8 = np.ascontiguousarray(lv.astype(np.int8))
        keep.append(c8)
        p.coeffs = c8.ctypes.data
        p.flags |= abi.PIC_COEFF8
    return keep


def geometry(p: abi.Picture) -> dict:
    ctb = 1 << p.log2_ctb
    sw = 2 if p.chroma_idc in (1, 2) else 1   # SubWidthC
    sh = 2 if p.chroma_idc == 1 else 1        # SubHeightC
    cw, ch = ((p.width + sw - 1) // sw, (p.height + sh - 1) // sh) if p.chroma_idc else (0, 0)
    return dict(w=p.width, h=p.height, cw=cw, ch=ch, sub=sw, sub_w=sw, sub_h=sh,
                ctb_cols=(p.width + ctb - 1) // ctb, ctb_rows=(p.height + ctb - 1) // ctb,
                gw=(p.width + 3) // 4, gh=(p.height + 3) // 4,
                bytes_per_sample=1 if p.bit_depth_y <= 8 else 2)


# ---------------------------------------------------------------------------
# Benchmark configurations.
# ---------------------------------------------------------------------------

def residual_cfg(seed: int, width=512, height=512, bit_depth=8, chroma_idc=1) -> abi.SynthCfg:
    """Plain residual reconstruction: quadtree TBs 4..32 (p=0.5 per level),
    DST for 4x4 luma, QP uniform 22..37 per TB, ~85% zeros before a random
    last position, Laplacian(8) non-zeros, seeded uniform prediction."""
    c = default_cfg()
    c.seed = seed
    c.width, c.height = width, height
    c.kind = abi.SYNTH_RESIDUAL
    c.bit_depth = bit_depth
    c.chroma_idc = chroma_idc
    c.pic_flags = 0
    return c


def intra_cfg(seed: int, width=512, height=512, bit_depth=10, chroma_idc=1, sao=True,
              deblock=True, tskip_p=0.0, tqb_p=0.0, cbf_p=0.9, scaling=False,
              bitstream=False) -> abi.SynthCfg:
    """Intra still tile: random CU (64..8) and TU (32..4) quadtrees, modes
    uniform over 35, coefficients as the residual case, deblocking on, SAO
    with random band/edge types and offsets in [-7, 7].  `bitstream`: also
    written as an H.265 I slice by the seeded CABAC writer (SynthSet.slice),
    the flat buffers being what the syntax decode of that slice yields."""
    c = default_cfg()
    c.seed = seed
    c.width, c.height = width, height
    c.kind = abi.SYNTH_INTRA
    c.bit_depth = bit_depth
    c.chroma_idc = chroma_idc
    c.cbf_p = cbf_p
    c.scaling = int(scaling)
    c.tskip_p = tskip_p
    c.tqb_p = tqb_p
    c.sao_p = 0.7 if sao else 0.0
    flags = abi.PIC_STRONG_SMOOTHING
    if deblock:
        flags |= abi.PIC_DEBLOCK
    if sao:
        flags |= abi.PIC_SAO_LUMA | abi.PIC_SAO_CHROMA
    c.pic_flags = flags
    c.bitstream = int(bitstream)
    return c


def inter_cfg(seed: int, width=1920, height=1080, bit_depth=8, weighted=False, n_refs=4,
              intra_cu_p=0.1, bi_p=0.4, scaling=False) -> abi.SynthCfg:
    c = intra_cfg(seed, width, height, bit_depth=bit_depth, chroma_idc=1, scaling=scaling)
    c.kind = abi.SYNTH_INTER
    c.weighted = int(weighted)
    c.n_refs = n_refs
    c.intra_cu_p = intra_cu_p
    c.bi_p = bi_p
    c.mv_sd = 16.0
    c.mv_pad = 80.0
    return c


@dataclass
class Grid:
    """A HEIC grid: tiles of tile x tile decoded as independent pictures and
    stitched (cropped at the right / bottom edge) onto an out_w x out_h canvas."""
    out_w: int
    out_h: int
    tile: int = 512
    synth: SynthSet = field(default_factory=SynthSet)
    places: list = field(default_factory=list)

    @property
    def cols(self) -> int:
        return -(-self.out_w // self.tile)

    @property
    def rows(self) -> int:
        return -(-self.out_h // self.tile)


def make_grid(out_w: int, out_h: int, seed: int, bit_depth=10, chroma_idc=1, tile=512,
              synth: SynthSet | None = None, **kw) -> Grid:
    g = Grid(out_w, out_h, tile, synth if synth is not None else SynthSet())
    for r in range(g.rows):
        for col in range(g.cols):
            cfg = intra_cfg(seed * 100003 + r * g.cols + col, tile, tile, bit_depth, chroma_idc, **kw)
            g.synth.add(cfg)
            g.places.append((col * tile, r * tile, tile, tile))
    return g


def grid_output(g: Grid, matrix=abi.MATRIX_SMPTE170M, full_range=True, places=None):
    """hpvcd_output for an RGB8 canvas; returns (output, keepalive array)."""
    pl = places if places is not None else g.places
    arr = (abi.TilePlace * len(pl))(*[abi.TilePlace(*t) for t in pl])
    out = abi.Output(abi.OUT_RGB8, matrix, int(full_range), g.out_w, g.out_h,
                     C.cast(arr, C.c_void_p))
    return out, arr


def config1_grid(seed: int = 0, bitstream: bool = True) -> Grid:
    """4032x3024 10-bit 4:2:0 still as an 8x6 grid of 512x512 tiles, each
    tile also written as an I slice by the seeded CABAC writer."""
    return make_grid(4032, 3024, seed, bit_depth=10, chroma_idc=1, bitstream=bitstream)


def grid_slices(g: Grid) -> list:
    """[(hpvcd_slice_params, slice bytes)] of a grid made in bitstream mode."""
    return [g.synth.slice(i) for i in range(len(g.synth))]


def config2_images(seed: int = 0, n_images: int = 256, max_side: int = 4096):
    """Mixed batch: sizes uniform 256..max_side step 64, 70% 8-bit / 30% 10-bit,
    80% 4:2:0 / 20% 4:4:4, each split into 512x512 grid tiles.  Returns a
    list of (width, height, bit_depth, chroma_idc)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_images):
        w = int(rng.integers(4, max_side // 64 + 1)) * 64
        h = int(rng.integers(4, max_side // 64 + 1)) * 64
        bd = 8 if rng.random() < 0.7 else 10
        idc = 1 if rng.random() < 0.8 else 3
        out.append((w, h, bd, idc))
    return out
