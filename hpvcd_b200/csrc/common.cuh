// common.cuh -- device-side picture table and helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hpvcd_gpu.h"

namespace hpvcd {

// Device view of one picture of a plan.  Built on the host from an
// hpvcd_picture (device pointers) plus the plan's own buffers.
struct DevPic {
    // geometry
    int32_t w, h, cw, ch, gw, gh;
    int32_t idc, sub_w, sub_h;  // sub_* = 1 or 2
    int32_t bd, bd_c, bps;      // bps: bytes per stored sample (1 when bd == 8)
    int32_t log2_ctb, ctb_cols, ctb_rows;
    uint32_t flags;
    int32_t beta_offset_div2, tc_offset_div2, pps_cb_qp_offset, pps_cr_qp_offset;
    // inputs
    const hpvcd_tu* tus;
    const uint32_t* ctu_start;
    const int16_t* coeffs;
    const hpvcd_cell* cells;
    const hpvcd_sao_ctb* sao;
    const hpvcd_pu* pus;
    const hpvcd_scaling* scaling;  // NULL: flat scale
    const uint16_t* ctb_region;    // slice << 8 | tile per CTB, NULL: one region
    const int8_t* slice_deblock;   // 256 x {beta, tc} offsets (div2) per slice, NULL: picture values
    uint32_t n_tus, n_pus;
    uint64_t n_coeffs;
    hpvcd_wp_table wp;
    int32_t has_wp;
    int32_t ref_pic[2][HPVCD_MAX_REFS];  // index of the reference picture in the plan, -1 none
    // planes: `rec` receives reconstruction and deblocking; `fin` is the
    // final picture after SAO (equal to `rec` when SAO does not run).
    void* rec[3];
    void* fin[3];
    int16_t* res[3];        // int16 residual planes of intra TBs (k_residual -> k_recon)
    int32_t res_stride[3];  // row stride of res[c] in samples (multiple of 16)
    uint32_t* ready;  // wavefront progress: 4 words per CTU, one level (0..4) per component
    // output placement on its RGB canvas
    int32_t dst_x, dst_y, crop_w, crop_h;
    uint64_t canvas_off;  // byte offset of the picture's canvas in the output
    int32_t canvas_w, canvas_h, matrix, full_range;
    int32_t orientation;  // HPVCD_ORIENT_* of the canvas (0 normal)
    int32_t needs_wavefront;
    int32_t write_fin;  // the tile filter kernel writes the final planes (else only the canvas)
};

// Work item of the reconstruction kernel: one CTU of one picture.
struct CtuItem {
    uint32_t pic;
    uint16_t cx, cy;
};

// Device error word bits.
enum : uint32_t {
    DEV_ERR_TIMEOUT = 1u,
    DEV_ERR_BITSTREAM = 2u,
};

__device__ __forceinline__ int clamp3i(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ int load_sample(const void* plane, int bps, size_t idx) {
    return bps == 1 ? (int)((const uint8_t*)plane)[idx] : (int)((const uint16_t*)plane)[idx];
}
__device__ __forceinline__ void store_sample(void* plane, int bps, size_t idx, int v) {
    if (bps == 1)
        ((uint8_t*)plane)[idx] = (uint8_t)v;
    else
        ((uint16_t*)plane)[idx] = (uint16_t)v;
}
// L2-only load (bypasses L1): used for samples another CTA published.
__device__ __forceinline__ int load_sample_cg(const void* plane, int bps, size_t idx) {
    return bps == 1 ? (int)__ldcg((const unsigned char*)plane + idx)
                    : (int)__ldcg((const unsigned short*)plane + idx);
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// qp helpers: decode.rs:5753-5771, :5868-5871, :7599-7613
__device__ __forceinline__ int qp_bd_offset(int bd) { return 6 * (bd - 8); }
__device__ __forceinline__ int qp_prime(int qp, int bd) {
    const int off = qp_bd_offset(bd);
    return clamp3i(qp + off, 0, 51 + off);
}
__device__ __forceinline__ int qpc_map(int qpi, int idc, int bd) {
    qpi = clamp3i(qpi, -qp_bd_offset(bd), 57);
    if (idc != 1) return qpi < 51 ? qpi : 51;
    if (qpi < 30) return qpi;
    if (qpi > 43) return qpi - 6;
    // H.265 Table 8-10 for qPi 30..43: 29 30 31 32 33 33 34 34 35 35 36 36 37 37
    const int i = qpi - 30;
    return i < 4 ? 29 + i : 33 + ((i - 4) >> 1);
}

}  // namespace hpvcd

// Launch bookkeeping shared by all translation units.
extern "C" void hpvcd_note_launches(uint32_t n);
