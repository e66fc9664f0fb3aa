/*
 * hpvcd_oracle.h -- CPU oracle for the hpvcd reconstruction path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a scalar C++ restatement of the
 * reference decoder's reconstruction kernels (hpvcd, Rust): transform.rs,
 * reconstruct.rs, intra.rs, mc.rs, inter.rs (offset normalisation),
 * deblock.rs plus the serial deblocking driver in decode.rs, sao.rs plus the
 * serial SAO driver in decode.rs, and yuv.rs / lib.rs (RGB conversion, rgb8
 * narrowing, grid stitching).  Each function cites the reference file:line it
 * restates.  The reference itself cannot be built here (no Rust toolchain), so
 * the restatement is pinned by the reference's own unit-test known answers
 * (see tests/test_oracle_kat.py) rather than by running the reference.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library; the product path never does.
 */
#ifndef HPVCD_ORACLE_H
#define HPVCD_ORACLE_H

#include <stdint.h>

#include "../include/hpvcd_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_dequant_params {
    int64_t factor, add;
    int32_t shift, pad;
    int64_t clip_min, clip_max;
} orc_dequant_params;

typedef struct orc_ts_params {
    orc_dequant_params dq;
    int32_t tr_add, tr_shift;
} orc_ts_params;

/* transform.rs */
/* The reference's parallel CPU decode of intra / residual tiles onto RGB8
 * canvases: grid-row jobs on a work-stealing pool, banded deblocking / SAO /
 * colour conversion, scalar or AVX2 kernels (simd != 0). */
int32_t orc_decode_grid_reference(const hpvcd_picture* pics, uint32_t n, const hpvcd_output* out, uint8_t* rgb,
                                  int32_t threads, int32_t simd);
/* Slices whose deblocking is disabled (flags[256] by slice index, NULL
 * clears): the reference's SliceDeblock.disabled, a test input. */
void orc_set_disabled_slices(const uint8_t* flags);
int32_t orc_max_log2_tr_range(int32_t bd, int32_t ext);
void orc_dequant_params_get(int32_t n, int32_t qp_prime, int32_t bd, int32_t ext,
                            orc_dequant_params* out);
void orc_ts_params_get(int32_t n, int32_t qp_prime, int32_t bd, int32_t ext, orc_ts_params* out);
void orc_dequant(const int32_t* levels, int32_t n, const orc_dequant_params* p,
                 const uint8_t* scaling /* NULL = flat */, int32_t scaling_dc, int32_t i16_store,
                 int32_t* out);
/* decode.rs:8418-8446: rotate, then RDPCM (dir 1 vertical, 0 horizontal,
 * -1 none), in place on an n*n residual. */
void orc_rext_residual_ops(int32_t* res, int32_t n, int32_t rotate, int32_t dir, int32_t i16s);
/* decode.rs:5874-5899: 1 and the selected list's first entry and DC when a
 * list applies, 0 for the flat scale. */
int32_t orc_scaling_select(const hpvcd_scaling* s, int32_t comp, int32_t n, int32_t inter, int32_t tskip,
                           int32_t* first, int32_t* dc);
void orc_dequant_ts(const int32_t* levels, int32_t n, const orc_ts_params* p,
                    const uint8_t* scaling, int32_t scaling_dc, int32_t i16_store, int32_t* out);
void orc_inv_dct(const int32_t* coeff, int32_t n, int32_t bd, int32_t max_range, int32_t nx,
                 int32_t i16_store, int32_t* out);
void orc_inv_dst4(const int32_t* coeff, int32_t bd, int32_t max_range, int32_t i16_store,
                  int32_t* out);
int32_t orc_dct_matrix_entry(int32_t n, int32_t k, int32_t m);

/* reconstruct.rs */
void orc_add_residual(uint16_t* dst, int32_t stride, const uint16_t* pred, const int32_t* res,
                      int32_t n, int32_t valid_w, int32_t valid_h, int32_t bd);
void orc_narrow_i32_to_i16(const int32_t* src, int16_t* dst, int32_t count);

/* intra.rs */
void orc_intra_substitute(const int32_t* raw_above /* 2n, -1 = unavailable */,
                          const int32_t* raw_left, int32_t raw_corner, int32_t n,
                          int32_t neutral, uint16_t* above_out, uint16_t* left_out);
void orc_intra_filter(const uint16_t* above, const uint16_t* left, int32_t n, int32_t mode,
                      int32_t is_luma, int32_t smoothing_enabled, int32_t strong, int32_t bd,
                      uint16_t* fa, uint16_t* fl);
void orc_intra_predict(int32_t mode, const uint16_t* above, const uint16_t* left, int32_t n,
                       int32_t is_luma, int32_t bd, uint16_t* out);

/* mc.rs */
void orc_luma_interp(const uint16_t* ref, int32_t stride, int32_t width, int32_t height,
                     int32_t x0, int32_t y0, int32_t fx, int32_t fy, int32_t w, int32_t h,
                     int32_t bd, int16_t* dst);
void orc_chroma_interp(const uint16_t* ref, int32_t stride, int32_t width, int32_t height,
                       int32_t x0, int32_t y0, int32_t fx, int32_t fy, int32_t w, int32_t h,
                       int32_t bd, int16_t* dst);
void orc_uni_mc(const int16_t* src, int32_t w, int32_t h, int32_t valid_w, int32_t valid_h,
                int32_t bd, uint16_t* dst, int32_t stride);
void orc_bi_mc(const int16_t* s0, const int16_t* s1, int32_t w, int32_t h, int32_t valid_w,
               int32_t valid_h, int32_t bd, uint16_t* dst, int32_t stride);
void orc_uni_mc_weighted(const int16_t* src, int32_t w, int32_t h, int32_t valid_w,
                         int32_t valid_h, int32_t bd, int32_t weight, int32_t offset,
                         int32_t log2_denom, uint16_t* dst, int32_t stride);
void orc_bi_mc_weighted(const int16_t* s0, const int16_t* s1, int32_t w, int32_t h,
                        int32_t valid_w, int32_t valid_h, int32_t bd, int32_t w0, int32_t o0,
                        int32_t w1, int32_t o1, int32_t log2_denom, uint16_t* dst,
                        int32_t stride);

/* inter.rs */
int32_t orc_normalize_luma_offset(int32_t offset, int32_t bd, int32_t high_precision);
int32_t orc_derive_chroma_offset(int32_t delta, int32_t weight, int32_t log2_denom, int32_t bd,
                                 int32_t high_precision);

/* decode.rs QP helpers */
int32_t orc_qp_prime(int32_t qp, int32_t bd);
int32_t orc_qpc(int32_t qpi, int32_t chroma_idc, int32_t bd);
int32_t orc_clamp_qpy(int32_t qp, int32_t bd);

/* deblock.rs: one 4-line luma segment; `vertical` selects the edge direction.
 * `plane` is a 16-bit plane of stride `stride`; (edge, scan) as in the serial
 * driver.  Returns the decision 0 skip, 1 strong, 2 weak. */
int32_t orc_deblock_luma_segment(uint16_t* plane, int32_t stride, int32_t vertical,
                                 int32_t edge, int32_t scan, int32_t beta, int32_t tc,
                                 int32_t maxv);
/* apply_luma_decision (deblock.rs:582) with an explicit decision
 * (1 strong, 2..5 weak with do_p1/do_q1 = (d-2)>>1&1 / (d-2)&1). */
void orc_apply_luma_decision(uint16_t* plane, int32_t stride, int32_t vertical, int32_t edge,
                             int32_t scan, int32_t decision, int32_t tc, int32_t maxv);

/* sao.rs */
void orc_sao_edge(uint16_t* dst, const uint16_t* src, int32_t w, int32_t h, int32_t x0,
                  int32_t y0, int32_t x_end, int32_t y_end, const int32_t* offsets,
                  int32_t eo_class, int32_t bd);
void orc_sao_band(uint16_t* dst, const uint16_t* src, int32_t w, int32_t x0, int32_t y0,
                  int32_t x_end, int32_t y_end, const int32_t* offsets, int32_t band_pos,
                  int32_t bd);

/* yuv.rs: convert a (width x height) picture window to RGB16 samples or RGB8
 * per `out8` (8-bit source) / Luma for mono.  Writes dw*dh*3 samples. */
void orc_yuv_to_rgb16(const uint16_t* y, const uint16_t* cb, const uint16_t* cr, int32_t width,
                      int32_t height, int32_t chroma_idc, int32_t bd, int32_t dw, int32_t dh,
                      int32_t crop_left, int32_t crop_top, int32_t matrix, int32_t full_range,
                      uint16_t* out);

/* ------------------------------------------------------------------------ */
/* Picture level.  Planes are 16-bit here (the reference keeps u16 planes    */
/* until `into_native`, yuv.rs:121).                                         */
/* ------------------------------------------------------------------------ */
typedef struct orc_planes {
    uint16_t* y;
    uint16_t* cb;
    uint16_t* cr;
} orc_planes;

/* decode.rs:4441 load_plane_block_clipped (zero padding outside the plane). */
void orc_load_block_clipped(const uint16_t* plane, int32_t stride, int32_t width, int32_t height,
                            int32_t x0, int32_t y0, int32_t n, uint16_t* pred);
/* Reconstruct the TB records of a picture in decode order (intra prediction,
 * inter residual add, PRED_IN_PLANE residual add).  `planes` must hold the
 * motion-compensated prediction (inter) or the seeded prediction
 * (PRED_IN_PLANE) on entry.  Returns 0 or an hpvcd_status. */
int32_t orc_recon_picture(const hpvcd_picture* pic, orc_planes* planes);
/* Motion compensation of all PUs of `pic` from the reference pictures
 * `refs[slot]` (decoded planes, same geometry). */
int32_t orc_mc_picture(const hpvcd_picture* pic, const orc_planes* refs, int32_t n_refs,
                       orc_planes* planes);
/* Serial deblocking (decode.rs:1774-2146). */
int32_t orc_deblock_picture(const hpvcd_picture* pic, orc_planes* planes);
/* Serial SAO (decode.rs:2258-2493). */
int32_t orc_sao_picture(const hpvcd_picture* pic, orc_planes* planes);
/* Full decode of a batch and optional RGB8 canvas (lib.rs:1610-1715,
 * lib.rs:1964-1999).  `planes_out[i]` receive the final planes (16-bit) when
 * non-NULL.  `threads` > 1 decodes pictures in parallel (grid rows in the
 * reference, lib.rs:1680).  Pictures with references decode in order. */
int32_t orc_decode_batch(const hpvcd_picture* pics, uint32_t n, const hpvcd_output* out,
                         orc_planes* planes_out, uint8_t* rgb_canvas, int32_t threads);

#ifdef __cplusplus
}
#endif

#endif
