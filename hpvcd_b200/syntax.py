"""Host syntax decode of H.265 I slices into the flat buffers the GPU back end
takes (include/hpvcd_syntax.h): the host half of the reference's
`decode_heic` path (CABAC engine src/cabac/engine.rs:219, coding-tree syntax
src/decode.rs:2495-3620, residual_coding src/cabac/residual_full.rs:392).
"""
from __future__ import annotations

import ctypes as C

from . import abi


class SyntaxPicture:
    """One decoded slice; owns the flat buffers its descriptor points at."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    @classmethod
    def decode(cls, params: abi.SliceParams, data: bytes) -> "SyntaxPicture":
        h = C.c_void_p()
        buf = C.create_string_buffer(data, len(data))
        st = abi.lib().hpvcd_syntax_decode(C.byref(params), C.cast(buf, C.c_void_p), len(data), C.byref(h))
        if st != abi.OK:
            raise abi.HpvcdError(st, "hpvcd_syntax_decode: " + abi.lib().hpvcd_last_error_string().decode())
        return cls(h)

    def picture(self) -> abi.Picture:
        p = abi.Picture()
        abi.check(abi.lib().hpvcd_syntax_picture(self._h, C.byref(p)), "hpvcd_syntax_picture")
        return p

    @property
    def bins(self) -> int:
        return int(abi.lib().hpvcd_syntax_bins(self._h))

    def close(self) -> None:
        if self._h:
            abi.lib().hpvcd_syntax_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def decode_batch(slices, threads: int = 0) -> list[SyntaxPicture]:
    """Decode [(params, bytes), ...] on up to `threads` host threads (0: all)."""
    n = len(slices)
    params = (abi.SliceParams * n)(*[sp for sp, _ in slices])
    bufs = [C.create_string_buffer(d, len(d)) for _, d in slices]
    data = (C.c_void_p * n)(*[C.cast(b, C.c_void_p) for b in bufs])
    sizes = (C.c_uint64 * n)(*[len(d) for _, d in slices])
    outs = (C.c_void_p * n)()
    sts = (C.c_int32 * n)()
    st = abi.lib().hpvcd_syntax_decode_batch(n, params, data, sizes, threads, outs, sts)
    res = [SyntaxPicture(C.c_void_p(outs[i])) if outs[i] else None for i in range(n)]
    if st != abi.OK:
        for r in res:
            if r is not None:
                r.close()
        raise abi.HpvcdError(st, "hpvcd_syntax_decode_batch: " + abi.lib().hpvcd_last_error_string().decode())
    return res
