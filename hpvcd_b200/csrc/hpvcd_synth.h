/*
 * hpvcd_synth.h -- seeded synthetic producer of the flat per-picture buffers
 * (include/hpvcd_gpu.h) that the host syntax decode of hpvcd would emit.
 *
 * There is no public benchmark suite for this path; inputs are synthetic with
 * the shapes and value distributions of the benchmark configurations:
 * random CU / TU quadtrees, intra modes uniform over 35, per-CU QP, int16
 * levels with a random last-significant position, mostly zero before it and
 * Laplacian-distributed non-zeros, deblocking metadata (boundary strengths and
 * QP per 4x4 cell), random SAO parameters and, for inter pictures, PUs with
 * Gaussian quarter-pel motion vectors, bi-prediction and explicit weights.
 */
#ifndef HPVCD_SYNTH_H
#define HPVCD_SYNTH_H

#include <stdint.h>

#include "../../include/hpvcd_gpu.h"
#include "../../include/hpvcd_syntax.h"

#ifdef __cplusplus
extern "C" {
#endif

#define HPVCD_SYNTH_RESIDUAL 0u /* PRED_IN_PLANE picture: seeded prediction + residual TBs */
#define HPVCD_SYNTH_INTRA 1u    /* all-intra picture                                      */
#define HPVCD_SYNTH_INTER 2u    /* inter picture referencing earlier pictures             */

typedef struct hpvcd_synth_cfg {
    uint64_t seed;
    uint32_t width, height;
    uint32_t kind;            /* HPVCD_SYNTH_*                                   */
    uint32_t chroma_idc;      /* 0, 1, 3                                         */
    uint32_t bit_depth;       /* luma = chroma bit depth                         */
    uint32_t log2_ctb;        /* 4..6                                            */
    uint32_t pic_flags;       /* HPVCD_PIC_* added to the picture                */
    float cu_split_p;         /* CU quadtree split probability per level         */
    float tu_split_p;         /* TU quadtree split probability per level         */
    float cbf_p;              /* probability that a TB carries coefficients      */
    float zero_frac;          /* fraction of zeros before the last position      */
    float laplace_scale;      /* scale of the non-zero level magnitudes          */
    float tskip_p;            /* probability of transform skip for 4x4 TBs       */
    float tqb_p;              /* probability that a CU is transquant-bypass      */
    float sao_p;              /* probability that a CTB component has SAO on     */
    int32_t qp_min, qp_max;   /* QpY range (uniform per CU)                      */
    int32_t beta_offset_div2, tc_offset_div2;
    int32_t cb_qp_offset, cr_qp_offset;
    /* inter */
    float intra_cu_p;         /* probability that a CU of an inter picture is intra */
    float bi_p;               /* probability of bi-prediction                       */
    float mv_sd;              /* motion-vector standard deviation in luma pixels    */
    float mv_pad;             /* MVs are clamped to the picture plus this padding   */
    uint32_t weighted;        /* explicit weighted prediction table                 */
    uint32_t n_refs;          /* references: the n_refs previous pictures           */
    /* TB-size mix: area fractions of 4x4, 8x8, 16x16, 32x32 TBs that the TU
     * quadtree aims at (per-level split probabilities derived from it); all
     * zero -> tu_split_p at every level. */
    float tu_mix[4];
    /* 1: random scaling lists (hpvcd_scaling, entries 1..255 rising with
     * frequency, DC 1..255), drawn from their own seeded stream so the rest
     * of the picture is the same as without them. */
    uint32_t scaling;
    /* RExt residual tools (bit mask): 1 transform_skip_rotation_enabled,
     * 2 implicit_rdpcm_enabled, 4 explicit_rdpcm_enabled (inter CUs draw
     * none / horizontal / vertical per transform-skip or bypass TB). */
    uint32_t rext;
    /* log2_max_transform_skip_block_size (2..5; 0 -> 2): transform skip is
     * drawn for coded TBs up to this size. */
    uint32_t tskip_log2_max;
    /* 4:4:4 only: cross_component_prediction_enabled; probability that a
     * chroma TB of a TU with coded luma gets a non-zero res_scale. */
    float ccp_p;
    /* Slices and tiles (hpvcd_picture.ctb_region): 1 = three slices split at
     * random CTB addresses in raster order, 2 = a uniform 2x2 tile grid with
     * one slice per tile.  0 = one slice and tile. */
    uint32_t regions;
    /* Probability that an 8x8..32x32 intra CU is I_PCM (random samples at a
     * random PCM bit depth, pcm_loop_filter_disabled drawn per CU). */
    float pcm_p;
    /* 1: also write the picture as the slice data of one H.265 I slice with
     * the seeded CABAC writer (hpvcd_synth_slice).  The flat buffers are then
     * exactly what the syntax decode of that slice yields: a coding unit
     * without coded residual takes the predicted QP (no cu_qp_delta to carry
     * its own), SAO fields the syntax does not code are zero and, with
     * sign_hiding, the sign of each hidden level follows the parity rule.
     * Needs an all-intra picture, chroma 4:0:0 / 4:2:0 / 4:4:4, no PCM,
     * regions or range-extension tools. */
    uint32_t bitstream;
    uint32_t sign_hiding; /* bitstream mode: sign_data_hiding_enabled_flag */
} hpvcd_synth_cfg;

typedef struct hpvcd_synth hpvcd_synth;

/* Default configuration of the residual-only 512x512 8-bit case. */
void hpvcd_synth_default_cfg(hpvcd_synth_cfg* cfg);
hpvcd_synth* hpvcd_synth_new(void);
void hpvcd_synth_free(hpvcd_synth* s);
/* Generate one picture; returns its index or a negative hpvcd_status. */
int32_t hpvcd_synth_add(hpvcd_synth* s, const hpvcd_synth_cfg* cfg);
uint32_t hpvcd_synth_count(const hpvcd_synth* s);
/* Descriptor of picture i; pointers stay valid until hpvcd_synth_free. */
int32_t hpvcd_synth_get(const hpvcd_synth* s, uint32_t i, hpvcd_picture* out);
/* Slice data of picture i (bitstream mode, with emulation prevention) and the
 * slice parameters it was written with; HPVCD_ERR_INVALID_ARG when the
 * picture was generated without it.  The bytes stay valid until
 * hpvcd_synth_free. */
int32_t hpvcd_synth_slice(const hpvcd_synth* s, uint32_t i, hpvcd_slice_params* params, const uint8_t** data,
                          uint64_t* bytes);

#ifdef __cplusplus
}
#endif

#endif
