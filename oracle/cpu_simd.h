// cpu_simd.h -- AVX2 kernels of the CPU reference arm (test infrastructure).
//
// The reference picks SIMD kernels by CPU feature through its ExecContext
// (exec.rs:31-77; the AVX2 set in avx/mod.rs).  These are this project's own
// AVX2 implementations of the same kernels, each exact to the scalar
// restatement in hpvcd_oracle.cpp (checked by tests/test_cpu_simd.py):
//   inv_dct        transform.rs:489-532 inv_dct_n_into (16x16 / 32x32,
//                  non-extended range) as 16-bit pair products
//   add_residual   reconstruct.rs:214-251 add_residual_generic
//   intra_predict  intra.rs:257-372 predict_into
//   sao_band       sao.rs:205-233
//   sao_edge       sao.rs:266-330 (no slice / tile restriction)
//   rgb_row        yuv.rs:232 / :327 (Q13, BT.601 / BT.709 / BT.2020 rows)
// Nothing in the product path uses them.
#pragma once

#include <stdint.h>

namespace orc_simd {

bool available();  // the CPU has AVX2

// n in {16, 32}, coefficients in int16 range (dequantised, max_range 15),
// columns >= nx zero; same outputs as the scalar inv_dct.
void inv_dct(const int32_t* coeff, int n, int bd, int nx, bool i16s, int32_t* out);
void add_residual(uint16_t* dst, int stride, const uint16_t* pred, const int32_t* res, int n, int valid_w,
                  int valid_h, int bd);
void intra_predict(int mode, const uint16_t* above, const uint16_t* left, int n, bool is_luma, int bd,
                   uint16_t* out);
void sao_band(uint16_t* dst, const uint16_t* src, int w, int x0, int y0, int x_end, int y_end,
              const int32_t* off, int band_pos, int bd);
void sao_edge(uint16_t* dst, const uint16_t* src, int w, int h, int x0, int y0, int x_end, int y_end,
              const int32_t* off, int eo_class, int bd);
// One row of YCbCr -> RGB16 (Q13; matrices with cr_to_r etc.; not identity /
// YCgCo): xs = first output column, count pixels; luma row / chroma row
// pointers already positioned; sub_w 1 or 2.
void rgb_row(const uint16_t* Y, const uint16_t* Cb, const uint16_t* Cr, int x_first, int count, int width,
             int cw, int sub_w, int bd, int32_t k_y, int32_t y_black, int32_t neutral, int32_t cr_to_r,
             int32_t cb_to_g, int32_t cr_to_g, int32_t cb_to_b, int32_t cmax, uint16_t* out);

}  // namespace orc_simd
