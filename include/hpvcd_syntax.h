/*
 * hpvcd_syntax.h -- host syntax decode of an H.265 I slice into the flat
 * per-picture buffers of hpvcd_gpu.h.
 *
 * The reference decoder parses slice data on the host with its CABAC engine
 * (src/cabac/engine.rs:219 `decode_bin`, contexts src/cabac/contexts.rs:67)
 * and the coding-tree syntax of `FullDecoder` (src/decode.rs:1507
 * `parse_sao`, :2495 `coding_quadtree`, :2585 `coding_unit`, :3315
 * `transform_tree`, :3478 `transform_unit`, src/cabac/residual_full.rs:392
 * `residual_coding`), filling the per-TU arguments of its reconstruction
 * calls as it goes.  These entry points do the same parse and emit, instead
 * of calls, the flat buffers the GPU back end takes in one hpvcd_gpu_submit:
 * TB records in decode order with resolved intra modes and QpY, dense levels,
 * per-4x4 deblocking cells and per-CTB SAO parameters.
 *
 * Scope: one slice covering the picture (one tile), I slices, chroma 4:0:0 /
 * 4:2:0 / 4:4:4, 8..12 bits, CTBs 16..64, TBs 4..32, transform skip (up to
 * log2_max_tskip), cu_transquant_bypass, cu_qp_delta with any quantization
 * group size, sign data hiding, SAO and deblocking parameters.  Not handled
 * (HPVCD_ERR_UNSUPPORTED): P/B slices, several slices or tiles, wavefront
 * entry points, I_PCM, palette, 4:2:2, cu_chroma_qp_offset and the range
 * extension's residual tools (implicit / explicit RDPCM, cross-component
 * prediction, persistent Rice adaptation, transform-skip contexts).
 *
 * Parameter sets and the slice header are parsed by the caller (the
 * reference keeps them in src/config.rs and parse_slice_header_full,
 * src/decode.rs:7713); hpvcd_slice_params carries the fields the slice data
 * depends on.  The bytes are slice_segment_data() of one NAL unit: from the
 * first byte after the slice header's byte_alignment() to the end of the
 * NAL unit, with emulation-prevention bytes (HPVCD_SLICE_EBSP) or without.
 */
#ifndef HPVCD_SYNTAX_H
#define HPVCD_SYNTAX_H

#include <stdint.h>

#include "hpvcd_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* hpvcd_slice_params.flags */
#define HPVCD_SLICE_TSKIP 0x0001u            /* transform_skip_enabled_flag (PPS)          */
#define HPVCD_SLICE_TQ_BYPASS 0x0002u        /* transquant_bypass_enabled_flag (PPS)       */
#define HPVCD_SLICE_CU_QP_DELTA 0x0004u      /* cu_qp_delta_enabled_flag (PPS)             */
#define HPVCD_SLICE_SIGN_HIDING 0x0008u      /* sign_data_hiding_enabled_flag (PPS)        */
#define HPVCD_SLICE_SAO_LUMA 0x0010u         /* slice_sao_luma_flag                        */
#define HPVCD_SLICE_SAO_CHROMA 0x0020u       /* slice_sao_chroma_flag                      */
#define HPVCD_SLICE_DEBLOCK 0x0040u          /* !slice_deblocking_filter_disabled_flag     */
#define HPVCD_SLICE_STRONG_SMOOTHING 0x0080u /* strong_intra_smoothing_enabled_flag (SPS)  */
#define HPVCD_SLICE_EBSP 0x0100u             /* bytes carry emulation_prevention_three_byte */

typedef struct hpvcd_slice_params {
    /* sequence parameter set */
    uint32_t width, height;   /* pic_width / pic_height_in_luma_samples          */
    uint8_t chroma_idc;       /* 0, 1 or 3                                        */
    uint8_t bit_depth_y;      /* 8..12                                            */
    uint8_t bit_depth_c;
    uint8_t log2_ctb;         /* CtbLog2SizeY, 4..6                               */
    uint8_t log2_min_cb;      /* MinCbLog2SizeY, 3..log2_ctb                      */
    uint8_t log2_min_tb;      /* MinTbLog2SizeY, 2..                              */
    uint8_t log2_max_tb;      /* MaxTbLog2SizeY, ..5                              */
    uint8_t max_th_depth_intra; /* max_transform_hierarchy_depth_intra            */
    /* picture parameter set */
    uint8_t diff_cu_qp_delta_depth;
    uint8_t log2_max_tskip;   /* Log2MaxTransformSkipSize (2 without RExt)        */
    int8_t pps_cb_qp_offset, pps_cr_qp_offset;
    /* slice header */
    int8_t slice_qp;          /* SliceQpY = 26 + init_qp_minus26 + slice_qp_delta */
    int8_t slice_cb_qp_offset, slice_cr_qp_offset;
    int8_t beta_offset_div2, tc_offset_div2;  /* slice (else PPS) deblocking offsets */
    uint8_t rsvd[3];
    uint32_t flags;           /* HPVCD_SLICE_*                                    */
    const hpvcd_scaling* scaling; /* resolved scaling lists, or NULL (flat);      */
                                  /* copied into the decoded picture              */
} hpvcd_slice_params;

typedef struct hpvcd_syntax_pic hpvcd_syntax_pic;

/* Parse one slice.  On success *out owns the picture's flat buffers. */
hpvcd_status hpvcd_syntax_decode(const hpvcd_slice_params* params, const uint8_t* data, uint64_t bytes,
                                 hpvcd_syntax_pic** out);

/* Parse n independent slices (grid tiles, frames of an all-intra batch) on
 * up to `threads` host threads (0 = hardware threads); status per slice in
 * st[i] (may be NULL), first failure returned.  out[i] is NULL for a slice
 * that failed. */
hpvcd_status hpvcd_syntax_decode_batch(uint32_t n, const hpvcd_slice_params* params, const uint8_t* const* data,
                                       const uint64_t* bytes, uint32_t threads, hpvcd_syntax_pic** out,
                                       hpvcd_status* st);

/* The decoded picture: a hpvcd_picture whose pointers are host pointers into
 * buffers owned by `p` (valid until hpvcd_syntax_free), ready for
 * hpvcd_gpu_submit. */
hpvcd_status hpvcd_syntax_picture(const hpvcd_syntax_pic* p, hpvcd_picture* out);

/* Bins decoded (context-coded, bypass, terminate) for the last parse of p. */
uint64_t hpvcd_syntax_bins(const hpvcd_syntax_pic* p);

void hpvcd_syntax_free(hpvcd_syntax_pic* p);

#ifdef __cplusplus
}
#endif

#endif
