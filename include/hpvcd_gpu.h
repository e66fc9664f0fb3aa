/*
 * hpvcd_gpu.h -- C ABI of the B200 reconstruction back end for hpvcd.
 *
 * The reference decoder (hpvcd, Rust) keeps bitstream demux, parameter sets,
 * CABAC and syntax decode on the host.  Everything that turns parsed syntax
 * into pixels -- dequantisation, inverse DCT/DST and transform skip, intra
 * prediction with reconstruction, motion compensation with weighted
 * prediction, deblocking, SAO and YCbCr->RGB -- runs behind this ABI on the
 * GPU.  In the reference those steps are the function-pointer slots of
 * `ExecContext` (src/exec.rs:31-77), called once per transform block from
 * `FullDecoder::transform_unit` (src/decode.rs:3478) and once per picture from
 * `FullDecoder::finish_with` (src/decode.rs:1440) and
 * `yuv_to_rgb_window_with_color_pool` (src/yuv.rs:533).  A GPU launch per TU
 * would be hopeless, so the seam here is per picture / per batch of pictures:
 * the host fills the flat buffers below while parsing and hands a whole
 * picture (or a whole HEIC grid) over in one call.
 *
 * Everything is plain C: fixed-size integer structs, pointers and sizes.  No
 * function here throws, aborts or panics; every entry point returns an
 * `hpvcd_status`, which maps onto the reference's `DecodeError`
 * (src/error.rs:30-60).
 */
#ifndef HPVCD_GPU_H
#define HPVCD_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HPVCD_ABI_VERSION 1u

/* ------------------------------------------------------------------------ */
/* Status codes.  Mapping onto src/error.rs `DecodeError`:                   */
/*   HPVCD_ERR_BITSTREAM   -> DecodeError::Bitstream (malformed flat buffers) */
/*   HPVCD_ERR_ALLOC       -> DecodeError::AllocationFailed { what, bytes }   */
/*   HPVCD_ERR_LIMIT       -> DecodeError::LimitExceeded { what, .. }         */
/*   HPVCD_ERR_UNSUPPORTED -> DecodeError::Unsupported                        */
/* The remaining codes have no reference counterpart (device-side failures). */
/* ------------------------------------------------------------------------ */
typedef enum hpvcd_status {
    HPVCD_OK = 0,
    HPVCD_ERR_BITSTREAM = 1,
    HPVCD_ERR_ALLOC = 2,
    HPVCD_ERR_LIMIT = 3,
    HPVCD_ERR_UNSUPPORTED = 4,
    HPVCD_ERR_TIMEOUT = 5,     /* a bounded device-side wait ran out          */
    HPVCD_ERR_CUDA = 6,        /* a CUDA runtime call failed                  */
    HPVCD_ERR_INVALID_ARG = 7, /* NULL pointer, bad handle, bad size          */
    HPVCD_ERR_BUSY = 8         /* ticket not finished within the wait budget  */
} hpvcd_status;

/* ------------------------------------------------------------------------ */
/* Flat per-picture buffers (the output contract of the host syntax decode). */
/* ------------------------------------------------------------------------ */

/* hpvcd_tu.flags */
#define HPVCD_TU_CBF 0x01u   /* coded residual present (cbf_luma / cbf_cb / cbf_cr) */
#define HPVCD_TU_TSKIP 0x02u /* transform_skip_flag                                  */
#define HPVCD_TU_INTRA 0x04u /* block of an intra CU (prediction from neighbours)    */
#define HPVCD_TU_TQB 0x08u   /* cu_transquant_bypass: residual = levels verbatim     */
/* RExt residual modification of a transform-skip or transquant-bypass TB, as
 * the host resolved it (decode.rs:4356-4374 rext_post_ops, applied by
 * apply_rext_residual_ops, decode.rs:8418-8446): ROTATE reverses the 4x4
 * residual (transform_skip_rotation_enabled, intra); RDPCM_V / RDPCM_H
 * accumulate it down the columns / along the rows (implicit for intra modes
 * 26 / 10, explicit_rdpcm_dir for inter CUs).  Ignored on other TBs. */
#define HPVCD_TU_ROTATE 0x10u
#define HPVCD_TU_RDPCM_H 0x20u
#define HPVCD_TU_RDPCM_V 0x40u
/* I_PCM coding unit (decode.rs:2768-2839 decode_pcm_cu): the record's n*n
 * levels are the reconstructed samples (pcm_sample << (BitDepth -
 * PcmBitDepth)); no prediction, no transform.  One record per component
 * (4:2:2 chroma: two stacked), flagged CBF | INTRA | PCM, on pictures flagged
 * HPVCD_PIC_PCM. */
#define HPVCD_TU_PCM 0x80u

/*
 * One transform block, or one "mark decoded" record.  Records of a picture are
 * stored in decode order, grouped per CTU in raster order (ctu_tu_start).
 *
 * - Intra luma TB      : predict (intra.rs), dequant + inverse transform, add,
 *                        mark the luma 4x4 cells decoded (decode.rs:4724-4907).
 * - Intra chroma TB    : predict, dequant + inverse DCT, add (decode.rs:5280).
 * - Inter TB with CBF  : prediction already in the plane (motion compensation),
 *                        add residual, mark decoded (decode.rs:4738-4745).
 * - Record without CBF and without INTRA: marks its square decoded only; this
 *   is how the end of an inter CU is signalled (decode.rs:6546-6548).  Such a
 *   record may have log2n up to 6.
 *
 * x, y are in samples of the component plane.  For 4:2:0, a group of four 4x4
 * luma TBs is followed by one 4x4 chroma TB per chroma component at the
 * parent's position (decode.rs:3601-3609).  For 4:2:2 every chroma TB of the
 * 4:2:0 layout is two square TBs stacked vertically, the upper one first,
 * all Cb TBs before the Cr TBs (decode.rs:5030-5060), with the intra mode
 * already mapped by the 4:2:2 table (decode.rs:3265-3280).
 */
typedef struct hpvcd_tu {
    uint16_t x, y;
    uint32_t coeff_off; /* element offset of the n*n row-major int16 levels   */
    uint8_t log2n;      /* 2..5 for coded TBs                                  */
    uint8_t comp;       /* 0 = Y, 1 = Cb, 2 = Cr                               */
    uint8_t flags;      /* HPVCD_TU_*                                          */
    uint8_t mode;       /* intra prediction mode 0..34 (chroma: resolved mode) */
    int8_t qp_y;        /* QpY of the coding unit (may be negative, bd > 8)    */
    int8_t cqp_off;     /* chroma TBs: slice + CU chroma QP offset             */
    uint8_t nx;         /* max_x + 1 from residual_coding (columns >= nx zero) */
    int8_t res_scale;   /* chroma TBs of HPVCD_PIC_CROSS_COMPONENT pictures:   */
                        /* ResScaleVal of cross_comp_pred (0, +-1, 2, 4, 8)    */
} hpvcd_tu; /* 16 bytes */

/* hpvcd_cell.flags */
#define HPVCD_CELL_EXEMPT 0x01u /* tqb CU, or I_PCM CU with pcm_loop_filter_disabled */
#define HPVCD_CELL_INTER 0x02u  /* cell of an inter CU (motion map !is_intra)          */

/*
 * Per 4x4 luma cell deblocking metadata (decode.rs:101-335 maps qp_y_map,
 * edge_v/bs_v, edge_h/bs_h, tqb/pcm).  bs_v / bs_h hold the boundary strength
 * of the cell's left / top edge after the host applied the edge flag and the
 * slice / tile gating of `deblock_bs_v` / `deblock_bs_h` (decode.rs:1670-1712):
 * 0 means "not a filtered edge".
 */
typedef struct hpvcd_cell {
    uint8_t bs_v;
    uint8_t bs_h;
    int8_t qp_y;
    uint8_t flags;
} hpvcd_cell; /* 4 bytes */

/* SAO parameters of one CTB component (decode.rs:66-72 `SaoCtb`). */
typedef struct hpvcd_sao_comp {
    uint8_t type_idx; /* 0 off, 1 band offset, 2 edge offset                */
    uint8_t band_pos; /* band offset: first of the four bands (0..31)        */
    uint8_t eo_class; /* edge offset: 0 hor, 1 ver, 2 135 deg, 3 45 deg      */
    uint8_t rsvd;
    int16_t offsets[4]; /* already sign-resolved and scaled (decode.rs:1560-1612) */
} hpvcd_sao_comp; /* 12 bytes */

typedef struct hpvcd_sao_ctb {
    hpvcd_sao_comp comp[3];
} hpvcd_sao_ctb; /* 36 bytes */

/* hpvcd_pu.flags */
#define HPVCD_PU_L0 0x01u
#define HPVCD_PU_L1 0x02u

/* One inter prediction block (decode.rs:7000 `motion_compensate`). */
typedef struct hpvcd_pu {
    uint16_t x, y, w, h;  /* luma samples                                     */
    int16_t mv[2][2];     /* [list][x,y], quarter-pel luma units              */
    int8_t ref_idx[2];    /* index into the picture's reference lists          */
    uint8_t flags;        /* HPVCD_PU_L0 | HPVCD_PU_L1                         */
    uint8_t rsvd;
} hpvcd_pu; /* 20 bytes */

/* Explicit weighted prediction (inter.rs:141 `PredWeightTable`), offsets in
 * reconstructed-sample units (already normalised as inter.rs:33-58 does). */
#define HPVCD_MAX_REFS 16
typedef struct hpvcd_wp_entry {
    int16_t luma_w, luma_o;
    int16_t cb_w, cb_o;
    int16_t cr_w, cr_o;
} hpvcd_wp_entry; /* 12 bytes */

typedef struct hpvcd_wp_table {
    uint8_t luma_log2_denom;
    uint8_t chroma_log2_denom;
    uint8_t rsvd[2];
    hpvcd_wp_entry e[2][HPVCD_MAX_REFS];
} hpvcd_wp_table;

/* Scaling lists of a picture (config.rs:373 `ScalingList`, the PPS list when
 * present, else the SPS list; decode.rs:5874-5899), resolved by the host:
 * m[size_id][matrix_id] is what `ScalingList::matrix` returns (8x8 raster;
 * the 4x4 lists use the first 16 entries, 4x4 raster), dc[size_id][matrix_id]
 * the DC value of the 16x16 / 32x32 lists.  size_id = log2(TB size) - 2;
 * matrix_id = component + 3 for TBs of inter CUs.  Transform-skip TBs larger
 * than 4x4 use the flat scale, as the reference does. */
typedef struct hpvcd_scaling {
    uint8_t m[4][6][64];
    uint8_t dc[4][6];
} hpvcd_scaling; /* 1560 bytes */

/* hpvcd_picture.flags */
#define HPVCD_PIC_STRONG_SMOOTHING 0x0001u   /* strong_intra_smoothing_enabled_flag   */
#define HPVCD_PIC_SMOOTHING_DISABLED 0x0002u /* RExt intra_smoothing_disabled_flag     */
#define HPVCD_PIC_DEBLOCK 0x0004u            /* run the deblocking filter              */
#define HPVCD_PIC_SAO_LUMA 0x0008u           /* slice_sao_luma_flag                    */
#define HPVCD_PIC_SAO_CHROMA 0x0010u         /* slice_sao_chroma_flag                  */
#define HPVCD_PIC_PRED_IN_PLANE 0x0020u      /* planes hold the prediction on entry:   */
                                             /* every TB only adds its residual        */
#define HPVCD_PIC_INTER 0x0040u              /* picture has motion-compensated PUs     */
/* cross_component_prediction_enabled_flag (4:4:4): a chroma TB with
 * res_scale != 0 adds (res_scale * ((rY << BitDepthC) >> BitDepthY)) >> 3 of
 * its TU's luma residual rY (decode.rs:5488-5504), also when it has no coded
 * residual of its own (decode.rs:5428).  The TU's luma TB is one of the three
 * records before the chroma record. */
#define HPVCD_PIC_CROSS_COMPONENT 0x0080u
/* SAO edge offset does not use neighbours across a slice / tile boundary
 * (slice_loop_filter_across_slices_enabled_flag = 0 /
 * loop_filter_across_tiles_enabled_flag = 0; sao.rs:380-414); needs
 * hpvcd_picture.ctb_region. */
#define HPVCD_PIC_SAO_NO_ACROSS_SLICES 0x0100u
#define HPVCD_PIC_SAO_NO_ACROSS_TILES 0x0200u
/* constrained_intra_pred_flag: intra prediction treats samples of cells
 * flagged HPVCD_CELL_INTER as unavailable (decode.rs:4641-4649); needs
 * cells. */
#define HPVCD_PIC_CONSTRAINED_INTRA 0x0400u
/* pcm_enabled_flag: records may carry HPVCD_TU_PCM. */
#define HPVCD_PIC_PCM 0x0800u
/* coeffs holds int8 levels: the host narrows a picture whose every level
 * lies in [-128, 127] and so copies half the pool; n_coeffs and
 * hpvcd_tu.coeff_off still count levels. */
#define HPVCD_PIC_COEFF8 0x1000u
/* Store the decoded picture into entry e of the context's DPB (hpvcd_dpb)
 * after it is reconstructed; bits 16..23 of flags, 0 = no store. */
#define HPVCD_PIC_STORE_DPB(e) ((uint32_t)((e) + 1) << 16)
#define HPVCD_PIC_STORE_MASK 0x00ff0000u
/* hpvcd_picture.ref_slot value naming DPB entry e (a picture decoded by an
 * earlier submit); values >= 0 name pictures of the same batch, -1 none. */
#define HPVCD_REF_DPB(e) (-2 - (int32_t)(e))

/*
 * One coded picture (one HEIC grid tile, one still image, or one video frame).
 * Pointers are host pointers for hpvcd_gpu_submit and device pointers for the
 * hpvcd_plan_* entry points.  Planes are stored without padding: luma stride =
 * width, chroma stride = width / SubWidthC, one byte per sample when the bit
 * depth is 8 and two bytes otherwise.
 */
typedef struct hpvcd_picture {
    uint32_t width, height; /* coded luma size (multiple of the minimum CB)   */
    uint8_t chroma_idc;     /* 0 mono, 1 4:2:0, 2 4:2:2, 3 4:4:4               */
    uint8_t bit_depth_y;    /* 8..12                                           */
    uint8_t bit_depth_c;
    uint8_t log2_ctb; /* 4..6                                              */
    uint32_t flags;   /* HPVCD_PIC_*                                       */
    int8_t beta_offset_div2;
    int8_t tc_offset_div2;
    int8_t pps_cb_qp_offset;
    int8_t pps_cr_qp_offset;
    uint32_t n_tus;
    uint32_t n_pus;
    uint64_t n_coeffs;
    const hpvcd_tu* tus;           /* n_tus                                  */
    const uint32_t* ctu_tu_start;  /* ctb_cols * ctb_rows + 1 prefix offsets  */
    const int16_t* coeffs;         /* n_coeffs (int8 with HPVCD_PIC_COEFF8)  */
    const hpvcd_cell* cells;       /* ceil(w/4) * ceil(h/4), NULL -> no deblock */
    const hpvcd_sao_ctb* sao;      /* ctb_cols * ctb_rows, NULL -> no SAO     */
    const hpvcd_pu* pus;           /* n_pus, inter pictures only              */
    const hpvcd_wp_table* wp;      /* NULL -> default weighted prediction     */
    int32_t ref_slot[2][HPVCD_MAX_REFS]; /* reference: batch index (< this one), */
                                         /* HPVCD_REF_DPB(e), or -1               */
    const void* pred[3];           /* PRED_IN_PLANE: initial Y/Cb/Cr planes   */
    const hpvcd_scaling* scaling;  /* NULL -> flat (scaling_list_enabled = 0) */
    /* Slices and tiles: per CTB in raster order, slice_idx << 8 | tile_id.
     * Intra prediction never reads a CTB of another slice or tile
     * (decode.rs:4651-4690 same_slice / same_tile); SAO follows the
     * HPVCD_PIC_SAO_NO_ACROSS_* flags; deblocking gating is folded into the
     * cells' boundary strengths by the host.  NULL -> one slice, one tile. */
    const uint16_t* ctb_region;
    /* Per-slice deblocking offsets (decode.rs:1762 slice_deblock_at): 256
     * pairs {slice_beta_offset_div2, slice_tc_offset_div2} indexed by the
     * slice of ctb_region; an edge uses the pair of the slice holding its q
     * sample.  NULL (or no ctb_region) -> beta/tc_offset_div2 above. */
    const int8_t* slice_deblock;
} hpvcd_picture;

/* Output of a batch.  RGB8 is the `decode_heic_rgb8` path (lib.rs:1964):
 * Q13 YCbCr->RGB (yuv.rs:187-393) then `>> (bit_depth - 8)`.  Pictures are
 * placed on an output canvas as grid tiles (lib.rs:1610 `stitch_grid_band`);
 * the part of a tile outside the canvas is cropped. */
#define HPVCD_OUT_YUV 0u  /* per-picture planes                              */
#define HPVCD_OUT_RGB8 1u /* packed RGB8 canvas                               */
/* Native YCbCr canvas, the `decode_heic_yuv` grid path (lib.rs:993-1091
 * fill_native_grid_yuv / stitch_native_yuv_band): per canvas its Y plane
 * (width x height), then Cb and Cr (ceil(width / SubWidthC) x
 * ceil(height / SubHeightC)), one byte per sample at 8 bits, two otherwise.
 * A canvas takes the chroma format and bit depth of its pictures (all equal;
 * 8-bit 4:0:0 when none is placed on it).  Picture i fills
 * ceil(crop_w / SubWidthC) x ceil(crop_h / SubHeightC) chroma samples from
 * (dst_x / SubWidthC, dst_y / SubHeightC), rows and columns past the picture
 * repeating its last one; matrix and range are not used. */
#define HPVCD_OUT_YUV_CANVAS 2u

/* Matrix coefficients as in src/color.rs `MatrixCoefficients` (H.273 values). */
#define HPVCD_MATRIX_IDENTITY 0u
#define HPVCD_MATRIX_BT709 1u
#define HPVCD_MATRIX_BT470BG 5u
#define HPVCD_MATRIX_SMPTE170M 6u
#define HPVCD_MATRIX_YCGCO 8u
#define HPVCD_MATRIX_BT2020NCL 9u

typedef struct hpvcd_tile_place {
    uint32_t dst_x, dst_y;   /* top-left on the canvas                         */
    uint32_t crop_w, crop_h; /* visible tile size (SPS conformance window size) */
    uint32_t canvas;         /* canvas index (0 when the output has one)       */
} hpvcd_tile_place; /* 20 bytes */

/* One output image of a batch: its size and colour description (the SPS VUI
 * of its tiles, lib.rs:1801-1815). */
typedef struct hpvcd_canvas {
    uint32_t width, height;  /* the image as stored (before orientation)      */
    uint32_t matrix;         /* HPVCD_MATRIX_*, or HPVCD_CANVAS_NATIVE         */
    uint32_t full_range;
    uint32_t orientation;    /* HPVCD_ORIENT_* (0 = normal)                    */
} hpvcd_canvas;

/* Orientation of a canvas (metadata.rs:31 `Orientation`, EXIF numbering,
 * from the HEIF irot / imir boxes), applied to the finished canvas as
 * lib.rs:2017-2110 apply_orientation does: the output holds the oriented
 * image, height x width for ROTATE90 / ROTATE270.  TRANSPOSE and TRANSVERSE
 * leave the samples in their stored places (the reference's rotate_luma /
 * rotate_buf treat them so); a native canvas rotates each plane. */
#define HPVCD_ORIENT_NORMAL 1u
#define HPVCD_ORIENT_FLIP_H 2u
#define HPVCD_ORIENT_ROTATE180 3u
#define HPVCD_ORIENT_FLIP_V 4u
#define HPVCD_ORIENT_TRANSPOSE 5u
#define HPVCD_ORIENT_ROTATE90 6u
#define HPVCD_ORIENT_TRANSVERSE 7u
#define HPVCD_ORIENT_ROTATE270 8u

/* hpvcd_canvas.matrix of an RGB8 output: this canvas receives its pictures'
 * native YCbCr planes, laid out as an HPVCD_OUT_YUV_CANVAS canvas, instead
 * of RGB8.  One submit then returns an image in RGB8 together with its
 * auxiliary images at native depth: the alpha plane (a 4:0:0 picture, Y
 * only; lib.rs:470-527 decode_alpha_plane_native) and the gain map
 * (lib.rs:555 DecodedGainMapImage planes). */
#define HPVCD_CANVAS_NATIVE 0x100u

typedef struct hpvcd_output {
    uint32_t kind;           /* HPVCD_OUT_*                                    */
    uint32_t matrix;         /* HPVCD_MATRIX_* (single canvas)                 */
    uint32_t full_range;     /* video_full_range_flag (single canvas)          */
    uint32_t canvas_w, canvas_h; /* single canvas                              */
    const hpvcd_tile_place* place; /* one per picture (RGB8 only)              */
    void* host_dst;          /* optional: page-locked caller buffer that       */
                             /* receives the output directly (then             */
                             /* hpvcd_gpu_read copies nothing)                 */
    uint64_t host_dst_bytes;
    /* Several canvases (n_canvases > 0): the output is canvases[0], then
     * canvases[1], ... each packed RGB8 width*height*3 bytes, and
     * place[i].canvas selects the canvas of picture i.  canvas_w / canvas_h /
     * matrix / full_range are then ignored. */
    uint32_t n_canvases;
    const hpvcd_canvas* canvases;
    /* Optional per-canvas destinations (n_canvases entries, page-locked):
     * each canvas is DMA'd straight into its own buffer; host_dst is then
     * unused and hpvcd_gpu_read copies nothing. */
    void* const* canvas_dst;
    uint32_t orientation;     /* single canvas: HPVCD_ORIENT_* (0 = normal)    */
    uint32_t options;         /* HPVCD_OUTPUT_* bits (0 = none)                */
} hpvcd_output;

/* hpvcd_output.options: an RGB8 output keeps only its canvases.  The final
 * YCbCr planes of a picture are then not written to device memory when no
 * later picture of the batch predicts from it, it is not stored into a
 * decoded-picture buffer and its canvas is an RGB8 one; hpvcd_plan_planes
 * still returns their addresses, but their contents are undefined.  Saves
 * the plane write (1.5 samples per pixel) of a decode whose product is the
 * canvas. */
#define HPVCD_OUTPUT_CANVAS_ONLY 0x1u

/* ------------------------------------------------------------------------ */
/* Library information.                                                     */
/* ------------------------------------------------------------------------ */
uint32_t hpvcd_abi_version(void);
const char* hpvcd_status_string(int status);
/* Number of kernel launches issued by this process so far (all entry points). */
uint64_t hpvcd_kernel_launch_count(void);
/* Text of the last CUDA runtime error this thread turned into a status. */
const char* hpvcd_last_error_string(void);

/* ------------------------------------------------------------------------ */
/* Host-buffer API: the drop-in under `decode_heic` / `VideoDecoder`.        */
/* Replaces, per picture batch, the per-TU ExecContext calls made from       */
/* decode.rs:3478-5426, `finish_with` (decode.rs:1440) and the grid stitch   */
/* `fill_grid_bands` / `stitch_grid_band` (lib.rs:1680 / lib.rs:1610).       */
/* A context is internally synchronised: any thread may submit.             */
/* ------------------------------------------------------------------------ */
typedef struct hpvcd_gpu hpvcd_gpu;
typedef uint64_t hpvcd_ticket;
struct hpvcd_sched; /* schedule knobs, defined with the plan API below   */
struct hpvcd_mlp;   /* selector network, declared with schedule selection */

typedef struct hpvcd_gpu_cfg {
    int32_t device;           /* CUDA device ordinal                          */
    uint32_t max_inflight;    /* concurrent tickets (streams), 0 -> 4         */
    uint64_t hbm_budget;      /* bytes this context may hold, 0 -> 80% free   */
} hpvcd_gpu_cfg;

hpvcd_status hpvcd_gpu_create(const hpvcd_gpu_cfg* cfg, hpvcd_gpu** out);
hpvcd_status hpvcd_gpu_destroy(hpvcd_gpu* ctx);
/* Copy the host buffers of `n` pictures to the device, reconstruct them and
 * start the copy of the requested output back.  Pageable host buffers are
 * only read during the call (staging copy).  Buffers in page-locked memory
 * are copied by DMA straight from where they are, one transfer per run of
 * buffers laid out as hpvcd_gpu_pack_inputs lays them out, and must stay
 * valid until the ticket completes.  Returns HPVCD_ERR_ALLOC when the batch does not fit the HBM budget
 * (the caller may retry later). */
hpvcd_status hpvcd_gpu_submit(hpvcd_gpu* ctx, const hpvcd_picture* pics, uint32_t n,
                              const hpvcd_output* out, hpvcd_ticket* ticket);
/* Size of the packed input layout of a batch, and the packing itself: copies
 * every host buffer of `pics` into `dst` (bytes >= the size) and rewrites
 * `out_pics` to point there.  A packed batch in page-locked memory is
 * uploaded with one DMA by hpvcd_gpu_submit. */
uint64_t hpvcd_gpu_packed_size(const hpvcd_picture* pics, uint32_t n);
hpvcd_status hpvcd_gpu_pack_inputs(const hpvcd_picture* pics, uint32_t n, void* dst, uint64_t bytes,
                                   hpvcd_picture* out_pics);
/* Wait at most timeout_ms (negative: forever) for a ticket. */
hpvcd_status hpvcd_gpu_wait(hpvcd_gpu* ctx, hpvcd_ticket ticket, int32_t timeout_ms);
/* Bytes of output a finished ticket holds (RGB8 canvas, or all YUV planes
 * of all pictures concatenated). */
hpvcd_status hpvcd_gpu_output_size(hpvcd_gpu* ctx, hpvcd_ticket ticket, uint64_t* bytes);
/* Copy a finished ticket's output into caller memory and release the ticket. */
hpvcd_status hpvcd_gpu_read(hpvcd_gpu* ctx, hpvcd_ticket ticket, void* dst, uint64_t bytes);
/* Per-batch schedule selection for this context: a submit that finds no
 * other ticket in flight computes the batch's features, runs the selector
 * network and launches the picked candidate -- on the host (hpvcd_batch_
 * features and a host copy of the bf16 weights, no device round trip) for
 * batches of up to 512k records, else on the device with a short host wait
 * for the pick; the same pick either way.  Submits made while other tickets
 * run take the fixed schedule (hpvcd_gpu_set_sched).  The weights are copied
 * here: a network trained further needs another call.  mlp NULL -> no
 * selection.  n must equal the network's output count. */
hpvcd_status hpvcd_gpu_set_selector(hpvcd_gpu* ctx, struct hpvcd_mlp* mlp, const struct hpvcd_sched* cands,
                                    uint32_t n);
/* counts[k]: batches that ran candidate k; counts[K] (n > K): batches
 * outside the network's domain -- features out of its range, or submitted
 * while other tickets of the context ran (it was trained on batches decoded
 * alone) -- which ran the context's fixed schedule (hpvcd_gpu_set_sched). */
hpvcd_status hpvcd_gpu_selector_picks(hpvcd_gpu* ctx, uint64_t* counts, uint32_t n);
/* The schedule of this context's submits while no selector is set (NULL:
 * the default, all-zero schedule). */
hpvcd_status hpvcd_gpu_set_sched(hpvcd_gpu* ctx, const struct hpvcd_sched* sched);

/* Decoded-picture buffer in HBM across submits, for video decoded frame by
 * frame (dpb.rs:79-454 and video.rs:1045-1379 keep reference pictures on the
 * host and clone planes per slice; here they never leave the device).  A
 * submit stores pictures flagged HPVCD_PIC_STORE_DPB(e) into entry e after
 * decoding them, and pictures of later submits predict from entry e through
 * ref_slot = HPVCD_REF_DPB(e).  Ordering across the context's tickets is
 * kept on the device (a store waits for earlier batches reading the entry;
 * a batch waits for the store that filled an entry it reads).  Within one
 * submit, references to pictures of the same batch use batch indices.  One
 * DPB serves one context. */
#define HPVCD_DPB_MAX_READERS 64
typedef struct hpvcd_dpb hpvcd_dpb;
hpvcd_status hpvcd_dpb_create(int32_t device, uint32_t entries, hpvcd_dpb** out);
/* Waits for the entries' pending copies, then frees them. */
hpvcd_status hpvcd_dpb_destroy(hpvcd_dpb* dpb);
/* The DPB this context's submits store into and predict from (NULL: none);
 * it must outlive the context's tickets. */
hpvcd_status hpvcd_gpu_set_dpb(hpvcd_gpu* ctx, hpvcd_dpb* dpb);

/* ------------------------------------------------------------------------ */
/* Device-buffer API (plans).  The picture descriptors point at device      */
/* memory that stays valid while the plan lives.  A plan owns its own        */
/* device scratch (work queues, wavefront progress words, ping-pong        */
/* planes) and output.                                                     */
/* hpvcd_plan_launch only enqueues kernels on `stream` (no allocation, no    */
/* synchronisation), so it can be captured into a CUDA graph.               */
/* ------------------------------------------------------------------------ */
typedef struct hpvcd_plan hpvcd_plan;

/* Stage selection for hpvcd_plan_launch. */
#define HPVCD_STAGE_RECON 0x01u   /* residual / intra / inter reconstruction    */
#define HPVCD_STAGE_DEBLOCK 0x02u /* deblocking filter                          */
#define HPVCD_STAGE_SAO 0x04u     /* sample adaptive offset                     */
#define HPVCD_STAGE_OUTPUT 0x08u  /* RGB8 canvas conversion                     */
#define HPVCD_STAGE_ALL 0x0Fu
#define HPVCD_STAGE_GRAPH 0x100u /* replay the selected stages as a CUDA graph    */
                                 /* captured on first use (stream must not be   */
                                 /* the legacy default stream)                   */

/* Schedule knobs chosen by the autotuner / schedule selector.  They never
 * change pixels, only speed.  All zero is the default schedule. */
typedef struct hpvcd_sched {
    uint32_t idct;              /* k_residual inverse transform of 16x16 / 32x32 TBs: 0 integer
                                   tensor-core products (int16 operands split exactly into int8
                                   halves), 1 even-odd butterflies, 2 matrix product with all-zero
                                   rows / columns skipped */
    uint32_t chroma_warps;      /* build of the wavefront kernel: 2 one warp per chroma component
                                   (three warps per CTA), 1 one warp for Cb, then Cr (two warps
                                   per CTA: more CTAs per SM), 3 three warps with at most 80
                                   registers per thread (8 CTAs per SM instead of 5: for batches
                                   with thousands of CTUs ready at once), 0 three warps, the
                                   register-capped build for a wave with more CTUs ready at once
                                   than the plain build's CTAs hold */
    uint32_t recon_ctas_per_sm; /* persistent wavefront CTAs per SM (0 -> occupancy max) */
    uint32_t wave;              /* wavefront synchronisation: 0 per quadrant (a CTU is walked while
                                   its left / above-right neighbours still are), 1 whole CTUs (one
                                   wait per CTU: fewer polls when tickets share the SMs) */
} hpvcd_sched;

hpvcd_status hpvcd_plan_create(const hpvcd_picture* dev_pics, uint32_t n,
                               const hpvcd_output* out, const hpvcd_sched* sched,
                               hpvcd_plan** plan);
hpvcd_status hpvcd_plan_destroy(hpvcd_plan* plan);
/* Enqueue the selected stages on `stream` (a cudaStream_t, NULL = default). */
hpvcd_status hpvcd_plan_launch(hpvcd_plan* plan, uint32_t stages, void* stream);
/* Device pointers of the reconstructed planes of picture i (valid after the
 * launch completes) and of the RGB8 canvas. */
hpvcd_status hpvcd_plan_planes(hpvcd_plan* plan, uint32_t i, void** y, void** cb, void** cr);
hpvcd_status hpvcd_plan_canvas(hpvcd_plan* plan, void** rgb, uint64_t* bytes);
/* Device-side error word of the last launch (0 = none); HPVCD_ERR_TIMEOUT when
 * a wavefront wait gave up.  Synchronises with the plan's last launch. */
hpvcd_status hpvcd_plan_device_status(hpvcd_plan* plan, void* stream);
/* Number of kernel launches one hpvcd_plan_launch(HPVCD_STAGE_ALL) issues. */
uint32_t hpvcd_plan_launches_per_run(const hpvcd_plan* plan);
/* Schedule of the plan's next launches (NULL = default); drops CUDA graphs
 * captured with the previous schedule.  Pixels do not depend on it. */
hpvcd_status hpvcd_plan_set_sched(hpvcd_plan* plan, const hpvcd_sched* sched);
/* Test hook of the bounded device waits.  No reference counterpart (the
 * reference's WPP rows always publish, wpp.rs:168-172).  Every wavefront
 * wait of the plan's later launches gives up after spin_limit polls (0 = the
 * default, 2^22 polls of >= 64 ns each); drop_ctu >= 0 leaves that entry of
 * the plan's CTU work list (wavefront order) out of the launches, -1 restores
 * it.  A dropped CTU is never reconstructed, so the waits of the CTUs that
 * predict from it run out and the launch completes with HPVCD_ERR_TIMEOUT in
 * hpvcd_plan_device_status.  Synchronous; drops captured CUDA graphs. */
hpvcd_status hpvcd_plan_set_wait_test(hpvcd_plan* plan, uint32_t spin_limit, int32_t drop_ctu);

/* ------------------------------------------------------------------------ */
/* Schedule selection: exhaustive autotuning and a learned selector.  No    */
/* reference counterpart (the reference picks SIMD kernels by CPU feature  */
/* only, src/exec.rs).  Pixels never depend on the schedule.               */
/* ------------------------------------------------------------------------ */
#define HPVCD_FEATURES 16      /* per-batch statistics the selector reads      */
#define HPVCD_MLP_HIDDEN 64    /* 16 -> 64 -> 64 -> K                          */
#define HPVCD_MLP_MAX_VARIANTS 32
#define HPVCD_MLP_NO_PICK 0xffffffffu /* features outside the network's domain */

/* Features of pictures [first, first + count) of a plan, computed on the
 * device from the TB / PU records and written to dev_out (16 floats, device
 * memory) on `stream`:
 *   0 log2(luma samples) / 24      1 log2(1 + pictures) / 8
 *   2 max wavefront length (ctb_cols + 2 ctb_rows) / 256
 *   3 (mean luma bit depth - 8) / 4   4 4:4:4 share of the area
 *   5-8 luma TB area share of 4x4, 8x8, 16x16, 32x32 TBs
 *   9 coded luma TB area / luma area  10 intra luma TB area / luma area
 *   11 mean QpY / 51   12 std QpY / 16
 *   13 mean (nx / n) over coded luma TBs (coefficient extent)
 *   14 log2(1 + mean |mv| in luma samples) / 8   15 bi-predicted PU share */
hpvcd_status hpvcd_plan_features(hpvcd_plan* plan, uint32_t first, uint32_t count, float* dev_out,
                                 void* stream);
/* The same 16 features on the host from host-memory pictures (the same
 * integer sums, the same formulas), written to out[16]. */
hpvcd_status hpvcd_batch_features(const hpvcd_picture* host_pics, uint32_t n, float* out);
/* Exhaustive autotuning: one untimed launch, then per candidate `warmup`
 * untimed and `reps` timed launches (CUDA events on `stream`, selected
 * stages); ms[i] (host, may be NULL) = the fastest timed launch of
 * candidate i.  The fastest candidate stays set on the plan, its index in
 * *best (may be NULL). */
hpvcd_status hpvcd_plan_autotune(hpvcd_plan* plan, const hpvcd_sched* cands, uint32_t n,
                                 uint32_t stages, uint32_t reps, uint32_t warmup, void* stream,
                                 float* ms, uint32_t* best);

/* The selector network: y = W3 relu(W2 relu(W1 x + b1) + b2) + b3, bf16
 * parameters, fp32 accumulation; y[k] predicts log(time of variant k / time
 * of the fastest variant) and the pick is argmin y.  Parameters are one flat
 * vector: W1 [64][16], b1 [64], W2 [64][64], b2 [64], W3 [K][64], b3 [K]
 * (row-major [out][in]).  Training keeps an fp32 master copy (Adam). */
typedef struct hpvcd_mlp hpvcd_mlp;
hpvcd_status hpvcd_mlp_create(uint32_t n_variants, uint64_t seed, hpvcd_mlp** out);
hpvcd_status hpvcd_mlp_destroy(hpvcd_mlp* mlp);
uint32_t hpvcd_mlp_param_count(const hpvcd_mlp* mlp);
uint32_t hpvcd_mlp_variants(const hpvcd_mlp* mlp);
/* Host copy of the parameters: master != 0 -> fp32 master copy, else the
 * bf16 values the forward pass uses (widened to fp32). */
hpvcd_status hpvcd_mlp_get_params(hpvcd_mlp* mlp, float* host, int master);
/* Feature domain (host lo[16], hi[16]; both NULL clears it): rows whose
 * features leave it are not picked for (HPVCD_MLP_NO_PICK), and
 * hpvcd_plan_select then runs the first (default) candidate. */
hpvcd_status hpvcd_mlp_set_domain(hpvcd_mlp* mlp, const float* lo, const float* hi);
/* Set the master copy (and its bf16 rounding) from host fp32; resets Adam. */
hpvcd_status hpvcd_mlp_set_params(hpvcd_mlp* mlp, const float* host);
/* y [B][K] = forward(x [B][16]); device pointers. */
hpvcd_status hpvcd_mlp_forward(hpvcd_mlp* mlp, const float* dev_x, uint32_t B, float* dev_y,
                               void* stream);
/* Gradient of L = mean over B*K of (forward(x) - t)^2 with respect to the
 * parameters (dev_grad, param_count floats, may be NULL) and L (dev_loss,
 * may be NULL); the gradient is also kept for hpvcd_mlp_adam_step. */
hpvcd_status hpvcd_mlp_grad(hpvcd_mlp* mlp, const float* dev_x, const float* dev_t, uint32_t B,
                            float* dev_grad, float* dev_loss, void* stream);
/* One Adam step (beta 0.9 / 0.999) with the last gradient. */
hpvcd_status hpvcd_mlp_adam_step(hpvcd_mlp* mlp, float lr, void* stream);
/* Mini-batch Adam for `epochs` seeded shuffled passes over n rows. */
hpvcd_status hpvcd_mlp_train(hpvcd_mlp* mlp, const float* dev_x, const float* dev_t, uint32_t n,
                             uint32_t batch, uint32_t epochs, float lr, uint64_t seed, void* stream,
                             float* final_loss);
/* argmin forward(x) of B feature rows (device) into host_variant[B]
 * (HPVCD_MLP_NO_PICK for rows outside the domain, when one is set). */
hpvcd_status hpvcd_mlp_pick(hpvcd_mlp* mlp, const float* dev_x, uint32_t B, void* stream,
                            uint32_t* host_variant);
/* Choose the plan's schedule among n candidates: the network's pick from
 * the plan's features when mlp has n outputs (candidate 0 when the features
 * leave the network's domain: *chosen = HPVCD_MLP_NO_PICK), else exhaustive
 * autotuning (the fallback).  *chosen = the candidate index. */
hpvcd_status hpvcd_plan_select(hpvcd_plan* plan, hpvcd_mlp* mlp, const hpvcd_sched* cands,
                               uint32_t n, void* stream, uint32_t* chosen);

/* ------------------------------------------------------------------------ */
/* Decoding one picture without allocating.  No counterpart in the          */
/* reference (its decoder allocates every plane it reconstructs).  For       */
/* callers that may not allocate while decoding: an application that gives  */
/* the decoder a fixed share of HBM, or a frame loop in which a cudaMalloc / */
/* cudaFree (which synchronise the device) would stall other streams.       */
/* ------------------------------------------------------------------------ */
/* Bytes of the fixed scratch array each device holds for this entry point:
 * enough for every picture up to 1024x1024 luma samples (any chroma format,
 * bit depth, deblocking and SAO). */
#define HPVCD_NOALLOC_SCRATCH_BYTES (12u * 1024u * 1024u + 256u * 1024u)
/* Reconstruct, deblock and SAO-filter one intra / residual picture whose
 * descriptor (a host struct) points at device-resident inputs, writing its
 * planes into caller-owned device memory: planes[0..2] = Y, Cb, Cr (Cb/Cr
 * unused for 4:0:0), each 256-byte aligned, unpadded (luma stride = width *
 * bytes per sample, as hpvcd_plan_planes).  Enqueues its kernels on `stream`
 * and returns; allocates no memory of any kind.  Its scratch (work counter,
 * error word, wavefront progress words, picture record, CTU list, residual and
 * pre-SAO planes) is one fixed array in the library's device memory; the
 * call itself zeroes the counter, error word and progress words on `stream`
 * before use, and nothing else needs to start at zero.
 *   - The first call on a device does the set-up (looks up the array's
 *     address, sets the kernel's shared-memory limit) with that device
 *     current; make it before any stream capture.
 *   - Calls ordered on one stream are safe.  Two calls whose work overlaps
 *     on one device (different streams, different host threads) share the
 *     array and race.
 *   - dev_status (device memory, may be NULL) receives the device error word
 *     when the call's work completes: 0 = OK, bit 0 = a wavefront wait gave
 *     up (HPVCD_ERR_TIMEOUT), bit 1 = malformed TB record (HPVCD_ERR_BITSTREAM).
 *   - HPVCD_ERR_LIMIT (message in hpvcd_last_error_string) when the picture
 *     needs more scratch than HPVCD_NOALLOC_SCRATCH_BYTES;
 *     HPVCD_ERR_UNSUPPORTED for inter pictures (their references belong to
 *     the same launch: use a plan) and for pictures flagged
 *     HPVCD_PIC_STORE_DPB(e) (stores into a decoded-picture buffer belong to
 *     a context's submits). */
hpvcd_status hpvcd_decode_noalloc(const hpvcd_picture* dev_pic, void* const planes[3],
                                  uint32_t* dev_status, void* stream);

/* ------------------------------------------------------------------------ */
/* Serving loop: continuous batching of decode requests.  No reference      */
/* counterpart (the reference decodes one `decode_heic` call at a time, or  */
/* several on caller threads, decoder.rs:224); this is the service a        */
/* request router puts in front of the drop-in.                             */
/* ------------------------------------------------------------------------ */
typedef struct hpvcd_server hpvcd_server;

typedef struct hpvcd_server_cfg {
    int32_t device;
    uint32_t max_inflight;       /* batches on the GPU at once, 0 -> 3           */
    uint32_t max_batch_pictures; /* pictures fused into one launch, 0 -> 4096    */
    uint64_t max_batch_bytes;    /* bytes of one batch, 0 -> 128 MiB (smaller     */
                                 /* batches pipeline copies with decoding)      */
    uint64_t hbm_budget;         /* context HBM budget, 0 -> 80% of free memory  */
    uint32_t batching;           /* 1: fuse queued requests; 0: one per launch   */
    uint32_t batch_window_us;    /* a free slot waits until the oldest queued     */
                                 /* request is this old (or a batch is full)      */
} hpvcd_server_cfg;

/* One decode request: the tiles of one image and where its RGB8 goes. */
typedef struct hpvcd_request {
    const hpvcd_picture* pics;  /* host buffers, copied during submit          */
    uint32_t n_pics;
    const hpvcd_tile_place* place; /* per picture (the canvas index is ignored) */
    hpvcd_canvas canvas;
    void* dst;                  /* receives width*height*3 bytes on completion */
    uint64_t dst_bytes;
    uint64_t user;              /* caller tag returned in the completion       */
    uint32_t flags;             /* HPVCD_REQ_*                                 */
} hpvcd_request;

/* hpvcd_request.flags */
#define HPVCD_REQ_ZERO_COPY 0x1u /* inputs packed by hpvcd_gpu_pack_inputs in  */
                                 /* page-locked memory and dst page-locked;     */
                                 /* both must stay valid until completion, and  */
                                 /* nothing is copied on the host               */

typedef struct hpvcd_completion {
    uint64_t user;
    int32_t status;             /* hpvcd_status of the request                 */
    uint32_t batch_pictures;    /* pictures of the launch that decoded it      */
    double latency_ms;          /* submit -> output in dst                     */
    double queue_ms;            /* submit -> batch launch                      */
} hpvcd_completion;

hpvcd_status hpvcd_server_create(const hpvcd_server_cfg* cfg, hpvcd_server** out);
/* Enqueue a request (non-blocking; the request's host buffers may be
 * released when this returns). */
hpvcd_status hpvcd_server_submit(hpvcd_server* srv, const hpvcd_request* req);
/* Up to `max` completions, waiting at most timeout_ms for the first one
 * (negative: forever).  Returns the number written. */
uint32_t hpvcd_server_poll(hpvcd_server* srv, hpvcd_completion* out, uint32_t max, int32_t timeout_ms);
/* Requests submitted and not yet returned by hpvcd_server_poll. */
uint32_t hpvcd_server_pending(hpvcd_server* srv);
hpvcd_status hpvcd_server_destroy(hpvcd_server* srv);
/* Schedule of the fused batches: the selector network's pick per batch
 * (hpvcd_plan_select) among n candidates; mlp NULL -> default schedule.  The
 * network must outlive the server (or be removed first). */
hpvcd_status hpvcd_server_set_selector(hpvcd_server* srv, struct hpvcd_mlp* mlp, const hpvcd_sched* cands,
                                       uint32_t n);
/* How often each candidate was picked since the selector was set;
 * counts[K] (n > K) = batches outside the network's domain. */
hpvcd_status hpvcd_server_selector_picks(hpvcd_server* srv, uint64_t* counts, uint32_t n);

/* ------------------------------------------------------------------------ */
/* Utilities (no reference counterpart).                                    */
/* ------------------------------------------------------------------------ */
/* Copy `bytes` between host and/or device pointers on `stream` and wait for
 * it (the direction is inferred from the pointers). */
hpvcd_status hpvcd_copy(void* dst, const void* src, uint64_t bytes, void* stream);
/* sizeof() of an ABI struct by name ("hpvcd_tu", ...), 0 if unknown; lets a
 * binding check its layout against this library. */
uint64_t hpvcd_abi_sizeof(const char* name);

#ifdef __cplusplus
}
#endif

#endif /* HPVCD_GPU_H */
