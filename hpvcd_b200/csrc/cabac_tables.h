// cabac_tables.h -- normative CABAC data of H.265 shared by the host syntax
// decoder (syntax.cpp) and the seeded bitstream writer (synth.cpp).
//
// Everything here is data the standard fixes: the LPS range table and the
// state transitions of the arithmetic coder (H.265 Tables 9-52 / 9-53, as the
// reference's engine.rs:35-71 holds them), the initValues of the I-slice
// (initType 0) context variables (Tables 9-5..9-37; the reference's
// contexts.rs:147-230), the context initialisation formula (9.3.2.2,
// contexts.rs:48-60), the 4x4 sig_coeff_flag context map (9.3.4.2.5) and the
// up-right diagonal / horizontal / vertical scan orders (6.5.3-6.5.5).
#pragma once

#include <stdint.h>

namespace hpvcd_cabac {

static const uint8_t kRangeLps[64][4] = {
    {128, 176, 208, 240}, {128, 167, 197, 227}, {128, 158, 187, 216}, {123, 150, 178, 205}, {116, 142, 169, 195},
    {111, 135, 160, 185}, {105, 128, 152, 175}, {100, 122, 144, 166}, {95, 116, 137, 158},  {90, 110, 130, 150},
    {85, 104, 123, 142},  {81, 99, 117, 135},   {77, 94, 111, 128},   {73, 89, 105, 122},   {69, 85, 100, 116},
    {66, 80, 95, 110},    {62, 76, 90, 104},    {59, 72, 86, 99},     {56, 69, 81, 94},     {53, 65, 77, 89},
    {51, 62, 73, 85},     {48, 59, 69, 80},     {46, 56, 66, 76},     {43, 53, 63, 72},     {41, 50, 59, 69},
    {39, 48, 56, 65},     {37, 45, 54, 62},     {35, 43, 51, 59},     {33, 41, 48, 56},     {32, 39, 46, 53},
    {30, 37, 43, 50},     {29, 35, 41, 48},     {27, 33, 39, 45},     {26, 31, 37, 43},     {24, 30, 35, 41},
    {23, 28, 33, 39},     {22, 27, 32, 37},     {21, 26, 30, 35},     {20, 24, 29, 33},     {19, 23, 27, 31},
    {18, 22, 26, 30},     {17, 21, 25, 28},     {16, 20, 23, 27},     {15, 19, 22, 25},     {14, 18, 21, 24},
    {14, 17, 20, 23},     {13, 16, 19, 22},     {12, 15, 18, 21},     {12, 14, 17, 20},     {11, 14, 16, 19},
    {11, 13, 15, 18},     {10, 12, 15, 17},     {10, 12, 14, 16},     {9, 11, 13, 15},      {9, 11, 12, 14},
    {8, 10, 12, 14},      {8, 9, 11, 13},       {7, 9, 11, 12},       {7, 9, 10, 12},       {7, 8, 10, 11},
    {6, 8, 9, 11},        {6, 7, 9, 10},        {6, 7, 8, 9},         {2, 2, 2, 2},
};

static const uint8_t kNextMps[64] = {1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16,
                                     17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32,
                                     33, 34, 35, 36, 37, 38, 39, 40, 41, 42, 43, 44, 45, 46, 47, 48,
                                     49, 50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 60, 61, 62, 62, 63};

static const uint8_t kNextLps[64] = {0,  0,  1,  2,  2,  4,  4,  5,  6,  7,  8,  9,  9,  11, 11, 12,
                                     13, 13, 15, 15, 16, 16, 18, 18, 19, 19, 21, 21, 22, 22, 23, 24,
                                     24, 25, 26, 26, 27, 27, 28, 29, 29, 30, 30, 30, 31, 32, 32, 33,
                                     33, 33, 34, 34, 35, 35, 35, 36, 36, 36, 37, 37, 37, 38, 38, 63};

// Context variables of an I slice, one flat array.  Offsets of each syntax
// element's contexts:
enum Ctx : int {
    kSaoMerge = 0,       // sao_merge_left_flag / sao_merge_up_flag (1)
    kSaoType = 1,        // first bin of sao_type_idx_luma / _chroma (1)
    kSplitCu = 2,        // split_cu_flag (3)
    kTqBypass = 5,       // cu_transquant_bypass_flag (1)
    kPartMode = 6,       // part_mode, intra (1)
    kPrevIntra = 7,      // prev_intra_luma_pred_flag (1)
    kChromaMode = 8,     // first bin of intra_chroma_pred_mode (1)
    kSplitTf = 9,        // split_transform_flag (3): 5 - log2TrafoSize
    kCbfLuma = 12,       // cbf_luma (2): trafoDepth == 0
    kCbfChroma = 14,     // cbf_cb / cbf_cr (5): trafoDepth
    kQpDelta = 19,       // cu_qp_delta_abs prefix (2)
    kTskip = 21,         // transform_skip_flag (2): luma / chroma
    kLastX = 23,         // last_sig_coeff_x_prefix (18)
    kLastY = 41,         // last_sig_coeff_y_prefix (18)
    kCsbf = 59,          // coded_sub_block_flag (4)
    kSig = 63,           // sig_coeff_flag (44: 27 luma + 15 chroma + 2 transform-skip)
    kGt1 = 107,          // coeff_abs_level_greater1_flag (24)
    kGt2 = 131,          // coeff_abs_level_greater2_flag (6)
    kCtxCount = 137,
};

static const uint8_t kInitI[kCtxCount] = {
    153,                                                                                   // sao merge
    200,                                                                                   // sao type
    139, 141, 157,                                                                         // split_cu
    154,                                                                                   // tq bypass
    184,                                                                                   // part_mode
    184,                                                                                   // prev intra
    63,                                                                                    // chroma mode
    153, 138, 138,                                                                         // split tf
    111, 141,                                                                              // cbf luma
    94,  138, 182, 154, 154,                                                               // cbf chroma
    154, 154,                                                                              // qp delta
    139, 139,                                                                              // transform skip
    110, 110, 124, 125, 140, 153, 125, 127, 140, 109, 111, 143, 127, 111, 79,  108, 123, 63,  // last x
    110, 110, 124, 125, 140, 153, 125, 127, 140, 109, 111, 143, 127, 111, 79,  108, 123, 63,  // last y
    91,  171, 134, 141,                                                                    // csbf
    111, 111, 125, 110, 110, 94,  124, 108, 124, 107, 125, 141, 179, 153, 125, 107, 125, 141,  // sig
    179, 153, 125, 107, 125, 141, 179, 153, 125, 140, 139, 182, 182, 152, 136, 152, 136, 153,
    136, 139, 111, 136, 139, 111, 141, 111,
    140, 92,  137, 138, 140, 152, 138, 139, 153, 74,  149, 92,  139, 107, 122, 152, 140, 179,  // gt1
    166, 182, 140, 227, 122, 197,
    138, 153, 136, 167, 152, 152,  // gt2
};

// 9.3.2.2: pStateIdx | valMps << 6 of a context with initValue iv at SliceQpY qp.
inline uint8_t init_state(int iv, int qp) {
    const int m = (iv >> 4) * 5 - 45, n = ((iv & 15) << 3) - 16;
    const int q = qp < 0 ? 0 : (qp > 51 ? 51 : qp);
    int pre = ((m * q) >> 4) + n;
    pre = pre < 1 ? 1 : (pre > 126 ? 126 : pre);
    return pre <= 63 ? (uint8_t)(63 - pre) : (uint8_t)((pre - 64) | 64);
}

// 9.3.4.2.5: sig_coeff_flag context of a 4x4 TB by raster position (y*4+x).
static const uint8_t kSigCtx4x4[16] = {0, 1, 4, 5, 2, 3, 4, 5, 6, 6, 8, 8, 7, 7, 8, 8};

// Scan positions (x, y) of a (1 << log2) square block for scanIdx 0 (up-right
// diagonal), 1 (horizontal), 2 (vertical), log2 in 0..3.
struct Scans {
    uint8_t pos[4][3][64][2];
    Scans() {
        for (int l = 0; l < 4; ++l) {
            const int n = 1 << l;
            int i = 0;
            for (int s = 0; s <= 2 * (n - 1); ++s)  // diagonal: anti-diagonals, bottom-left first
                for (int y = n - 1; y >= 0; --y) {
                    const int x = s - y;
                    if (x >= 0 && x < n) {
                        pos[l][0][i][0] = (uint8_t)x;
                        pos[l][0][i][1] = (uint8_t)y;
                        ++i;
                    }
                }
            for (int k = 0; k < n * n; ++k) {
                pos[l][1][k][0] = (uint8_t)(k % n);
                pos[l][1][k][1] = (uint8_t)(k / n);
                pos[l][2][k][0] = (uint8_t)(k / n);
                pos[l][2][k][1] = (uint8_t)(k % n);
            }
        }
    }
};

inline const Scans& scans() {
    static const Scans s;
    return s;
}

// 7.4.9.11 scanIdx of an intra TB of size 1 << log2 (component's own size).
inline int scan_idx(bool intra, int log2, int comp, int chroma_idc, int mode) {
    if (!intra) return 0;
    if (!(log2 == 2 || (log2 == 3 && (comp == 0 || chroma_idc == 3)))) return 0;
    if (mode >= 6 && mode <= 14) return 2;
    if (mode >= 22 && mode <= 30) return 1;
    return 0;
}

// 8.4.2 candidate list of the luma intra mode from the left (a) and above (b)
// neighbours' modes (DC when unavailable).
inline void mpm_list(int a, int b, int out[3]) {
    if (a == b) {
        if (a < 2) {
            out[0] = 0;
            out[1] = 1;
            out[2] = 26;
        } else {
            out[0] = a;
            out[1] = 2 + ((a + 29) % 32);
            out[2] = 2 + ((a - 2 + 1) % 32);
        }
    } else {
        out[0] = a;
        out[1] = b;
        out[2] = (a != 0 && b != 0) ? 0 : ((a != 1 && b != 1) ? 1 : 26);
    }
}

// Table 8-2: chroma mode from intra_chroma_pred_mode (0..4) and the luma mode.
inline int chroma_mode(int icpm, int luma) {
    static const int cand[4] = {0, 26, 10, 1};
    if (icpm == 4) return luma;
    return cand[icpm] == luma ? 34 : cand[icpm];
}

}  // namespace hpvcd_cabac
