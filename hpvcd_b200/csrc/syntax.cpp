// syntax.cpp -- host syntax decode of an H.265 I slice (include/hpvcd_syntax.h).
//
// CABAC arithmetic decoding (H.265 9.3.4.3) and the slice_segment_data()
// syntax of an I slice (7.3.8) into the flat buffers of hpvcd_gpu.h.  The
// parse follows the order of the reference's FullDecoder: per CTB the SAO
// parameters (decode.rs:1507 parse_sao), then the coding quadtree
// (decode.rs:2495), coding units (decode.rs:2585), transform tree and units
// (decode.rs:3315, :3478) and residual_coding (cabac/residual_full.rs:392).
// Where the reference calls its reconstruction kernels per TB, this emits a
// TB record; the QP derivation (decode.rs:5868 qp_prime, 8.6.1), the intra
// mode candidates (8.4.2) and the deblocking edge / boundary-strength maps
// (decode.rs:2955-3050) are resolved here as the host side of the boundary.
//
// Every index into the picture's maps is derived from positions inside the
// picture and every loop is bounded by the syntax, so malformed data ends in
// HPVCD_ERR_BITSTREAM, never in an access outside the buffers.
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "cabac_tables.h"
#include "hpvcd_syntax.h"

#define HPVCD_API extern "C" __attribute__((visibility("default")))

void hpvcd_note_error(const char* msg);  // runtime.cu: thread's last error string

namespace {

using namespace hpvcd_cabac;

// Bits of the RBSP, most significant first, through a 64-bit window.  Reads
// past the end return zero bits and are counted.
struct Bits {
    const uint8_t* begin = nullptr;
    const uint8_t* p = nullptr;
    const uint8_t* end = nullptr;
    uint64_t win = 0;
    int avail = 0;
    uint32_t past_end = 0;

    void refill() {
        while (avail <= 56) {
            uint64_t b = 0;
            if (p < end)
                b = *p++;
            else
                ++past_end;
            win |= b << (56 - avail);
            avail += 8;
        }
    }
    uint32_t get(int n) {  // 0 <= n <= 32
        if (n == 0) return 0;
        if (avail < n) refill();
        const uint32_t v = (uint32_t)(win >> (64 - n));
        win <<= n;
        avail -= n;
        return v;
    }
    // bits consumed beyond the end of the data
    int64_t overrun() const {
        const int64_t used = (int64_t)((p - begin) + past_end) * 8 - avail;
        return used - (int64_t)(end - begin) * 8;
    }
};

struct Engine {
    Bits bits;
    uint32_t range = 510, offset = 0;
    uint64_t bins = 0;
    uint8_t ctx[kCtxCount];

    void start(const uint8_t* data, size_t n, int slice_qp) {
        bits.begin = bits.p = data;
        bits.end = data + n;
        for (int i = 0; i < kCtxCount; ++i) ctx[i] = init_state(kInitI[i], slice_qp);
        range = 510;
        offset = bits.get(9);
    }
    int decision(int ci) {
        ++bins;
        const uint8_t s = ctx[ci];
        const int st = s & 63, mps = s >> 6;
        const uint32_t lps = kRangeLps[st][(range >> 6) & 3];
        range -= lps;
        if (offset >= range) {  // least probable symbol
            offset -= range;
            range = lps;
            ctx[ci] = (uint8_t)(kNextLps[st] | ((st == 0 ? mps ^ 1 : mps) << 6));
            const int sh = __builtin_clz(range) - 23;  // range < 256: back to 9 bits
            range <<= sh;
            offset = (offset << sh) | bits.get(sh);
            return mps ^ 1;
        }
        ctx[ci] = (uint8_t)(kNextMps[st] | (mps << 6));
        if (range < 256) {
            range <<= 1;
            offset = (offset << 1) | bits.get(1);
        }
        return mps;
    }
    int bypass() {
        ++bins;
        offset = (offset << 1) | bits.get(1);
        if (offset >= range) {
            offset -= range;
            return 1;
        }
        return 0;
    }
    uint32_t bypass_bits(int n) {
        uint32_t v = 0;
        for (int i = 0; i < n; ++i) v = (v << 1) | (uint32_t)bypass();
        return v;
    }
    int terminate() {
        ++bins;
        range -= 2;
        if (offset >= range) return 1;
        if (range < 256) {
            range <<= 1;
            offset = (offset << 1) | bits.get(1);
        }
        return 0;
    }
};

struct Fail {};  // thrown inside the parse, caught at the entry point

struct Decoder {
    const hpvcd_slice_params& sp;
    Engine E;
    char msg[160] = "";

    int w, h, idc, sub_w, sub_h, log2ctb, ctb, cols, rows, gw, gh;
    int min_cb, min_tb, max_tb, bd_y, bd_c, qp_off_y, log2_min_qg;
    bool qp_delta_on;

    // per 4x4 luma cell: coding-tree depth, luma intra mode, QpY, TU edges
    std::vector<uint8_t> depth, lmode, edge_v, edge_h;
    std::vector<int8_t> qpmap;

    // outputs
    std::vector<hpvcd_tu> tus;
    std::vector<uint32_t> ctu_start;
    std::vector<int16_t> coeffs;
    std::vector<hpvcd_cell> cells;
    std::vector<hpvcd_sao_ctb> sao;
    hpvcd_scaling scaling{};
    bool has_scaling = false;

    // QP state (8.6.1)
    int qp_last = 0;   // QpY of the last coding unit decoded
    int qp_pred = 0;   // qPY_PRED of the current quantization group
    int qp_delta = 0;  // CuQpDeltaVal
    bool delta_coded = false;

    // current coding unit
    int cu_x = 0, cu_y = 0, cu_log2 = 0;
    bool cu_tqb = false, cu_nxn = false;
    int cu_lm[4] = {0, 0, 0, 0}, cu_cm[4] = {0, 0, 0, 0};

    explicit Decoder(const hpvcd_slice_params& p) : sp(p) {}

    [[noreturn]] void fail(const char* what) {
        snprintf(msg, sizeof(msg), "slice data: %s", what);
        throw Fail{};
    }

    size_t cell(int x, int y) const { return (size_t)(y >> 2) * gw + (x >> 2); }

    void fill(std::vector<uint8_t>& m, int x0, int y0, int size, uint8_t v) {
        const int x1 = std::min(x0 + size, w), y1 = std::min(y0 + size, h);
        for (int y = y0; y < y1; y += 4)
            for (int x = x0; x < x1; x += 4) m[cell(x, y)] = v;
    }

    hpvcd_status setup() {
        w = (int)sp.width;
        h = (int)sp.height;
        idc = sp.chroma_idc;
        log2ctb = sp.log2_ctb;
        min_cb = sp.log2_min_cb;
        min_tb = sp.log2_min_tb;
        max_tb = sp.log2_max_tb;
        bd_y = sp.bit_depth_y;
        bd_c = sp.bit_depth_c;
        if (idc == 2) {
            snprintf(msg, sizeof(msg), "4:2:2 slices are not handled by the host syntax decode");
            return HPVCD_ERR_UNSUPPORTED;
        }
        if (idc > 3 || log2ctb < 4 || log2ctb > 6 || min_cb < 3 || min_cb > log2ctb || min_tb < 2 ||
            max_tb > 5 || min_tb > max_tb || max_tb > log2ctb || min_tb >= min_cb || bd_y < 8 || bd_y > 12 ||
            (idc && (bd_c < 8 || bd_c > 12)) || sp.log2_max_tskip < 2 || sp.log2_max_tskip > 5 ||
            sp.max_th_depth_intra > log2ctb - min_tb || sp.diff_cu_qp_delta_depth > log2ctb - min_cb) {
            snprintf(msg, sizeof(msg), "slice parameters out of range");
            return HPVCD_ERR_INVALID_ARG;
        }
        if (w <= 0 || h <= 0 || w > 16384 || h > 16384 || (w & ((1 << min_cb) - 1)) || (h & ((1 << min_cb) - 1))) {
            snprintf(msg, sizeof(msg), "picture size %dx%d is not a multiple of the minimum CB", w, h);
            return HPVCD_ERR_INVALID_ARG;
        }
        const int qp_min = -6 * (bd_y - 8);
        if (sp.slice_qp < qp_min || sp.slice_qp > 51) {
            snprintf(msg, sizeof(msg), "SliceQpY %d outside [%d, 51]", sp.slice_qp, qp_min);
            return HPVCD_ERR_INVALID_ARG;
        }
        sub_w = idc == 1 ? 2 : 1;
        sub_h = idc == 1 ? 2 : 1;
        ctb = 1 << log2ctb;
        cols = (w + ctb - 1) / ctb;
        rows = (h + ctb - 1) / ctb;
        gw = (w + 3) / 4;
        gh = (h + 3) / 4;
        qp_off_y = 6 * (bd_y - 8);
        qp_delta_on = (sp.flags & HPVCD_SLICE_CU_QP_DELTA) != 0;
        log2_min_qg = log2ctb - sp.diff_cu_qp_delta_depth;
        const size_t nc = (size_t)gw * gh;
        depth.assign(nc, 0);
        lmode.assign(nc, 1);
        edge_v.assign(nc, 0);
        edge_h.assign(nc, 0);
        qpmap.assign(nc, 0);
        cells.assign(nc, hpvcd_cell{});
        ctu_start.assign((size_t)cols * rows + 1, 0);
        if (sp.flags & (HPVCD_SLICE_SAO_LUMA | HPVCD_SLICE_SAO_CHROMA)) sao.assign((size_t)cols * rows, hpvcd_sao_ctb{});
        if (sp.scaling) {
            scaling = *sp.scaling;
            has_scaling = true;
        }
        tus.reserve((size_t)w * h / 32);
        coeffs.reserve((size_t)w * h);
        return HPVCD_OK;
    }

    // ---- SAO (7.3.8.3) ----
    void parse_sao(int rx, int ry) {
        hpvcd_sao_ctb s{};
        const size_t at = (size_t)ry * cols + rx;
        bool merge = false;
        if (rx > 0 && E.decision(kSaoMerge)) {
            s = sao[at - 1];
            merge = true;
        } else if (ry > 0 && E.decision(kSaoMerge)) {
            s = sao[at - cols];
            merge = true;
        }
        if (!merge) {
            for (int c = 0; c < (idc ? 3 : 1); ++c) {
                const bool on = c == 0 ? (sp.flags & HPVCD_SLICE_SAO_LUMA) : (sp.flags & HPVCD_SLICE_SAO_CHROMA);
                if (!on) continue;
                hpvcd_sao_comp& sc = s.comp[c];
                if (c == 2) {
                    sc.type_idx = s.comp[1].type_idx;
                    sc.eo_class = s.comp[1].eo_class;
                } else {
                    sc.type_idx = 0;
                    if (E.decision(kSaoType)) sc.type_idx = E.bypass() ? 2 : 1;
                }
                if (!sc.type_idx) continue;
                const int bd = c ? bd_c : bd_y;
                const int cmax = (1 << (std::min(bd, 10) - 5)) - 1;
                int abs_v[4];
                for (int i = 0; i < 4; ++i) {
                    int v = 0;
                    while (v < cmax && E.bypass()) ++v;
                    abs_v[i] = v;
                }
                if (sc.type_idx == 1) {
                    for (int i = 0; i < 4; ++i) sc.offsets[i] = (int16_t)(abs_v[i] && E.bypass() ? -abs_v[i] : abs_v[i]);
                    sc.band_pos = (uint8_t)E.bypass_bits(5);
                } else {
                    sc.offsets[0] = (int16_t)abs_v[0];
                    sc.offsets[1] = (int16_t)abs_v[1];
                    sc.offsets[2] = (int16_t)-abs_v[2];
                    sc.offsets[3] = (int16_t)-abs_v[3];
                    if (c < 2) sc.eo_class = (uint8_t)E.bypass_bits(2);
                }
            }
        }
        sao[at] = s;
    }

    // ---- quantization groups (8.6.1) ----
    void start_qg(int x0, int y0) {
        const int mask = ctb - 1;
        const int qa = (x0 & mask) ? qpmap[cell(x0 - 1, y0)] : qp_last;
        const int qb = (y0 & mask) ? qpmap[cell(x0, y0 - 1)] : qp_last;
        qp_pred = (qa + qb + 1) >> 1;
        qp_delta = 0;
        delta_coded = false;
    }

    void parse_qp_delta() {
        int v = 0;
        while (v < 5 && E.decision(kQpDelta + (v ? 1 : 0))) ++v;
        if (v == 5) {  // EG0 suffix
            int k = 0;
            uint32_t add = 0;
            while (E.bypass()) {
                add += 1u << k;
                if (++k > 16) fail("cu_qp_delta_abs too long");
            }
            v += (int)(add + E.bypass_bits(k));
        }
        int d = v;
        if (v && E.bypass()) d = -v;
        const int lim = 26 + qp_off_y / 2;
        if (d < -lim || d > lim - 1) fail("CuQpDeltaVal out of range");
        qp_delta = d;
        delta_coded = true;
    }

    // ---- coding quadtree / unit (7.3.8.4, 7.3.8.5) ----
    void coding_quadtree(int x0, int y0, int log2, int cqt_depth) {
        const int size = 1 << log2;
        bool split;
        if (x0 + size <= w && y0 + size <= h && log2 > min_cb) {
            int inc = 0;
            if (x0 > 0 && depth[cell(x0 - 1, y0)] > cqt_depth) ++inc;
            if (y0 > 0 && depth[cell(x0, y0 - 1)] > cqt_depth) ++inc;
            split = E.decision(kSplitCu + inc);
        } else {
            split = log2 > min_cb;
        }
        if (qp_delta_on && log2 >= log2_min_qg) start_qg(x0, y0);
        if (split) {
            const int half = size >> 1;
            for (int b = 0; b < 4; ++b) {
                const int x = x0 + (b & 1) * half, y = y0 + (b >> 1) * half;
                if (x < w && y < h) coding_quadtree(x, y, log2 - 1, cqt_depth + 1);
            }
            return;
        }
        if (x0 + size > w || y0 + size > h) fail("coding unit outside the picture");
        coding_unit(x0, y0, log2, cqt_depth);
    }

    int parse_chroma_mode() { return E.decision(kChromaMode) ? (int)E.bypass_bits(2) : 4; }

    void coding_unit(int x0, int y0, int log2, int cqt_depth) {
        const int size = 1 << log2;
        cu_x = x0;
        cu_y = y0;
        cu_log2 = log2;
        cu_tqb = (sp.flags & HPVCD_SLICE_TQ_BYPASS) && E.decision(kTqBypass);
        cu_nxn = false;
        if (log2 == min_cb) cu_nxn = !E.decision(kPartMode);
        if (cu_nxn && log2 - 1 < min_tb) fail("NxN partition below the minimum TB size");
        fill(depth, x0, y0, size, (uint8_t)cqt_depth);
        const int pb = cu_nxn ? size >> 1 : size, npu = cu_nxn ? 4 : 1;
        int prev[4];
        for (int k = 0; k < npu; ++k) prev[k] = E.decision(kPrevIntra);
        for (int k = 0; k < npu; ++k) {
            const int px = x0 + (k & 1) * pb, py = y0 + (k >> 1) * pb;
            const int a = px > 0 ? lmode[cell(px - 1, py)] : 1;
            const int b = (py > 0 && ((py - 1) >> log2ctb) == (py >> log2ctb)) ? lmode[cell(px, py - 1)] : 1;
            int cand[3];
            mpm_list(a, b, cand);
            int mode;
            if (prev[k]) {
                const int idx = E.bypass() ? (E.bypass() ? 2 : 1) : 0;
                mode = cand[idx];
            } else {
                mode = (int)E.bypass_bits(5);
                std::sort(cand, cand + 3);
                for (int i = 0; i < 3; ++i)
                    if (mode >= cand[i]) ++mode;
            }
            cu_lm[k] = mode;
            fill(lmode, px, py, pb, (uint8_t)mode);
        }
        if (!cu_nxn)
            for (int k = 1; k < 4; ++k) cu_lm[k] = cu_lm[0];
        if (idc == 3) {
            for (int k = 0; k < npu; ++k) cu_cm[k] = chroma_mode(parse_chroma_mode(), cu_lm[k]);
            if (!cu_nxn)
                for (int k = 1; k < 4; ++k) cu_cm[k] = cu_cm[0];
        } else if (idc) {
            const int m = chroma_mode(parse_chroma_mode(), cu_lm[0]);
            for (int k = 0; k < 4; ++k) cu_cm[k] = m;
        }
        const size_t first_tb = tus.size();
        transform_tree(x0, y0, x0, y0, log2, 0, 0, 0, 0);
        // QpY of the coding unit (8.6.1), into its records and cells
        int qp = sp.slice_qp;
        if (qp_delta_on) qp = ((qp_pred + qp_delta + 52 + 2 * qp_off_y) % (52 + qp_off_y)) - qp_off_y;
        qp_last = qp;
        for (size_t i = first_tb; i < tus.size(); ++i) tus[i].qp_y = (int8_t)qp;
        const int x1 = std::min(x0 + size, w), y1 = std::min(y0 + size, h);
        for (int y = y0; y < y1; y += 4)
            for (int x = x0; x < x1; x += 4) {
                const size_t g = cell(x, y);
                qpmap[g] = (int8_t)qp;
                cells[g].qp_y = (int8_t)qp;
                cells[g].flags = cu_tqb ? HPVCD_CELL_EXEMPT : 0;
            }
    }

    // ---- transform tree / unit (7.3.8.8, 7.3.8.10) ----
    void transform_tree(int x0, int y0, int xb, int yb, int log2, int tdepth, int blk, int parent_cb,
                        int parent_cr) {
        const int max_depth = sp.max_th_depth_intra + (cu_nxn ? 1 : 0);
        bool split;
        if (log2 <= max_tb && log2 > min_tb && tdepth < max_depth && !(cu_nxn && tdepth == 0))
            split = E.decision(kSplitTf + 5 - log2);
        else
            split = log2 > max_tb || (cu_nxn && tdepth == 0);
        if (split && log2 - 1 < min_tb) fail("transform tree below the minimum TB size");
        int cb = 0, cr = 0;
        if ((log2 > 2 && idc) || idc == 3) {
            if (tdepth == 0 || parent_cb) cb = E.decision(kCbfChroma + tdepth);
            if (tdepth == 0 || parent_cr) cr = E.decision(kCbfChroma + tdepth);
        } else if (idc) {  // 4:2:0 4x4 luma: the parent's chroma flags apply
            cb = parent_cb;
            cr = parent_cr;
        }
        if (split) {
            const int half = 1 << (log2 - 1);
            for (int b = 0; b < 4; ++b)
                transform_tree(x0 + (b & 1) * half, y0 + (b >> 1) * half, x0, y0, log2 - 1, tdepth + 1, b, cb, cr);
            return;
        }
        const int cbf_l = E.decision(kCbfLuma + (tdepth == 0 ? 1 : 0));  // intra: always coded
        transform_unit(x0, y0, xb, yb, log2, blk, cbf_l, cb, cr);
    }

    int pu_of(int x, int y) const {  // PU index of a luma position inside the CU
        if (!cu_nxn) return 0;
        const int half = 1 << (cu_log2 - 1);
        return (x - cu_x >= half ? 1 : 0) + (y - cu_y >= half ? 2 : 0);
    }

    void transform_unit(int x0, int y0, int xb, int yb, int log2, int blk, int cbf_l, int cb, int cr) {
        const bool chroma_here = idc && (log2 > 2 || idc == 3);
        const bool chroma_blk3 = idc && !chroma_here && blk == 3;
        const int cbf_c = idc ? (cb | cr) : 0;  // 4:2:0 4x4: the parent's flags, for every blkIdx
        if ((cbf_l || cbf_c) && qp_delta_on && !delta_coded) parse_qp_delta();
        const uint8_t base = HPVCD_TU_INTRA | (cu_tqb ? HPVCD_TU_TQB : 0);
        edge(x0, y0, 1 << log2);
        tb(0, x0, y0, log2, base, cbf_l, cu_lm[pu_of(x0, y0)]);
        if (chroma_here) {
            const int clog2 = idc == 3 ? log2 : log2 - 1;
            const int m = cu_cm[pu_of(x0, y0)];
            tb(1, x0 / sub_w, y0 / sub_h, clog2, base, cb, m);
            tb(2, x0 / sub_w, y0 / sub_h, clog2, base, cr, m);
        } else if (chroma_blk3) {
            tb(1, xb / sub_w, yb / sub_h, 2, base, cb, cu_cm[0]);
            tb(2, xb / sub_w, yb / sub_h, 2, base, cr, cu_cm[0]);
        }
    }

    void edge(int x0, int y0, int size) {
        if (x0 > 0)
            for (int y = y0; y < std::min(y0 + size, h); y += 4) edge_v[cell(x0, y)] = 1;
        if (y0 > 0)
            for (int x = x0; x < std::min(x0 + size, w); x += 4) edge_h[cell(x, y0)] = 1;
    }

    void tb(int comp, int x, int y, int log2, uint8_t flags, int cbf, int mode) {
        hpvcd_tu t{};
        t.x = (uint16_t)x;
        t.y = (uint16_t)y;
        t.log2n = (uint8_t)log2;
        t.comp = (uint8_t)comp;
        t.mode = (uint8_t)mode;
        t.cqp_off = (int8_t)(comp == 1 ? sp.slice_cb_qp_offset : comp == 2 ? sp.slice_cr_qp_offset : 0);
        if (cbf) {
            flags |= HPVCD_TU_CBF;
            bool tskip = false;
            t.coeff_off = (uint32_t)coeffs.size();
            t.nx = residual_coding(log2, comp, mode, &tskip);
            if (tskip) flags |= HPVCD_TU_TSKIP;
        }
        t.flags = flags;
        tus.push_back(t);
    }

    // ---- residual_coding (7.3.8.11; contexts 9.3.4.2.3-9.3.4.2.7) ----
    int remaining(int rice) {
        int u = 0;
        while (u < 4 && E.bypass()) ++u;
        if (u < 4) return (u << rice) + (int)E.bypass_bits(rice);
        int k = rice + 1;
        uint32_t v = 0;
        while (E.bypass()) {
            v += 1u << k;
            if (++k > 20) fail("coeff_abs_level_remaining too long");
        }
        v += E.bypass_bits(k);
        return (4 << rice) + (int)v;
    }

    uint8_t residual_coding(int log2, int comp, int mode, bool* tskip_out) {
        const int n = 1 << log2;
        const size_t off = coeffs.size();
        coeffs.resize(off + (size_t)n * n, 0);
        bool tskip = false;
        if ((sp.flags & HPVCD_SLICE_TSKIP) && !cu_tqb && log2 <= sp.log2_max_tskip)
            tskip = E.decision(kTskip + (comp ? 1 : 0));
        *tskip_out = tskip;
        int ctx_off, ctx_shift;
        if (comp == 0) {
            ctx_off = 3 * (log2 - 2) + ((log2 - 1) >> 2);
            ctx_shift = (log2 + 1) >> 2;
        } else {
            ctx_off = 15;
            ctx_shift = log2 - 2;
        }
        const int cmax = (log2 << 1) - 1;
        int px = 0, py = 0;
        while (px < cmax && E.decision(kLastX + ctx_off + (px >> ctx_shift))) ++px;
        while (py < cmax && E.decision(kLastY + ctx_off + (py >> ctx_shift))) ++py;
        int lx = px, ly = py;
        if (px > 3) {
            const int nb = (px >> 1) - 1;
            lx = (1 << nb) * (2 + (px & 1)) + (int)E.bypass_bits(nb);
        }
        if (py > 3) {
            const int nb = (py >> 1) - 1;
            ly = (1 << nb) * (2 + (py & 1)) + (int)E.bypass_bits(nb);
        }
        const int scan = scan_idx(true, log2, comp, idc, mode);
        if (scan == 2) std::swap(lx, ly);
        if (lx >= n || ly >= n) fail("last significant position outside the TB");
        const Scans& S = scans();
        const int sbl = log2 - 2, nsb = 1 << sbl;
        int last_sb = nsb * nsb - 1, last_pos = 16;
        for (;;) {  // scan position of (lx, ly)
            if (last_pos == 0) {
                last_pos = 16;
                --last_sb;
            }
            --last_pos;
            const int xc = (S.pos[sbl][scan][last_sb][0] << 2) + S.pos[2][scan][last_pos][0];
            const int yc = (S.pos[sbl][scan][last_sb][1] << 2) + S.pos[2][scan][last_pos][1];
            if (xc == lx && yc == ly) break;
        }
        int16_t* out = coeffs.data() + off;
        uint8_t csbf[8][8];
        memset(csbf, 0, sizeof(csbf));
        int c1 = 1;  // greater1Ctx carried from the previous coded sub-block
        int max_x = 0;
        const bool hiding_on = (sp.flags & HPVCD_SLICE_SIGN_HIDING) && !cu_tqb;
        for (int i = last_sb; i >= 0; --i) {
            const int xs = S.pos[sbl][scan][i][0], ys = S.pos[sbl][scan][i][1];
            bool infer_dc = false;
            if (i < last_sb && i > 0) {
                int inc = 0;
                if (xs < nsb - 1) inc += csbf[xs + 1][ys];
                if (ys < nsb - 1) inc += csbf[xs][ys + 1];
                csbf[xs][ys] = (uint8_t)E.decision(kCsbf + std::min(inc, 1) + (comp ? 2 : 0));
                infer_dc = true;
            } else {
                csbf[xs][ys] = 1;
            }
            int sig[16], nsig = 0;  // scan positions of the significant levels, high to low
            if (i == last_sb) sig[nsig++] = last_pos;
            if (csbf[xs][ys]) {
                int prev = 0;
                if (xs < nsb - 1) prev |= csbf[xs + 1][ys];
                if (ys < nsb - 1) prev |= csbf[xs][ys + 1] << 1;
                for (int k = (i == last_sb ? last_pos - 1 : 15); k >= 0; --k) {
                    const int xp = S.pos[2][scan][k][0], yp = S.pos[2][scan][k][1];
                    if (k == 0 && infer_dc) {
                        sig[nsig++] = 0;
                        break;
                    }
                    const int xc = (xs << 2) + xp, yc = (ys << 2) + yp;
                    int sc;
                    if (log2 == 2) {
                        sc = kSigCtx4x4[(yc << 2) + xc];
                    } else if (xc + yc == 0) {
                        sc = 0;
                    } else {
                        if (prev == 0)
                            sc = xp + yp == 0 ? 2 : (xp + yp < 3 ? 1 : 0);
                        else if (prev == 1)
                            sc = yp == 0 ? 2 : (yp == 1 ? 1 : 0);
                        else if (prev == 2)
                            sc = xp == 0 ? 2 : (xp == 1 ? 1 : 0);
                        else
                            sc = 2;
                        if (comp == 0) {
                            if (xs > 0 || ys > 0) sc += 3;
                            sc += log2 == 3 ? (scan == 0 ? 9 : 15) : 21;
                        } else {
                            sc += log2 == 3 ? 9 : 12;
                        }
                    }
                    if (E.decision(kSig + (comp ? 27 + sc : sc))) {
                        sig[nsig++] = k;
                        infer_dc = false;
                    }
                }
            }
            if (!nsig) continue;
            int ctx_set = (i == 0 || comp > 0) ? 0 : 2;
            if (c1 == 0) ++ctx_set;
            c1 = 1;
            int gt1[16] = {0};
            int first_gt1 = -1;
            const int ng1 = std::min(nsig, 8);
            for (int k = 0; k < ng1; ++k) {
                gt1[k] = E.decision(kGt1 + ctx_set * 4 + std::min(c1, 3) + (comp ? 16 : 0));
                if (gt1[k]) {
                    c1 = 0;
                    if (first_gt1 < 0) first_gt1 = k;
                } else if (c1 > 0 && c1 < 3) {
                    ++c1;
                }
            }
            const int gt2 = first_gt1 >= 0 ? E.decision(kGt2 + ctx_set + (comp ? 4 : 0)) : 0;
            const bool hidden = hiding_on && sig[0] - sig[nsig - 1] > 3;
            int sign[16];
            for (int k = 0; k < nsig; ++k) sign[k] = (hidden && k == nsig - 1) ? 0 : E.bypass();
            int rice = 0, sum = 0;
            for (int k = 0; k < nsig; ++k) {
                const int base = 1 + (k < 8 ? gt1[k] : 0) + (k == first_gt1 ? gt2 : 0);
                const int thresh = k < 8 ? (k == first_gt1 ? 3 : 2) : 1;
                int a = base;
                if (base == thresh) {
                    a = base + remaining(rice);
                    if (a > 3 * (1 << rice)) rice = std::min(rice + 1, 4);
                }
                if (a > 32768) fail("level outside the 16-bit range");
                sum += a;
                int v = sign[k] ? -a : a;
                if (hidden && k == nsig - 1 && (sum & 1)) v = -v;
                if (v > 32767) fail("level outside the 16-bit range");
                const int xc = (xs << 2) + S.pos[2][scan][sig[k]][0], yc = (ys << 2) + S.pos[2][scan][sig[k]][1];
                out[yc * n + xc] = (int16_t)v;
                max_x = std::max(max_x, xc);
            }
        }
        return (uint8_t)(max_x + 1);
    }

    // ---- slice data (7.3.8.1) ----
    void run(const uint8_t* data, size_t bytes) {
        E.start(data, bytes, sp.slice_qp);
        qp_last = sp.slice_qp;
        qp_pred = sp.slice_qp;
        const bool sao_on = !sao.empty();
        for (int ry = 0; ry < rows; ++ry)
            for (int rx = 0; rx < cols; ++rx) {
                ctu_start[(size_t)ry * cols + rx] = (uint32_t)tus.size();
                if (sao_on) parse_sao(rx, ry);
                coding_quadtree(rx << log2ctb, ry << log2ctb, log2ctb, 0);
                const bool last = ry == rows - 1 && rx == cols - 1;
                if (E.terminate() != (last ? 1 : 0))
                    fail(last ? "no end_of_slice_segment_flag after the last CTB" : "slice ends before the last CTB");
                if (E.bits.overrun() > 0) fail("slice data ends early");
            }
        ctu_start[(size_t)cols * rows] = (uint32_t)tus.size();
        // boundary strengths: every TB edge of an intra picture is 2
        for (int gy = 0; gy < gh; ++gy)
            for (int gx = 0; gx < gw; ++gx) {
                const size_t g = (size_t)gy * gw + gx;
                cells[g].bs_v = (gx > 0 && edge_v[g]) ? 2 : 0;
                cells[g].bs_h = (gy > 0 && edge_h[g]) ? 2 : 0;
            }
        // maps only the parse needs
        std::vector<uint8_t>().swap(depth);
        std::vector<uint8_t>().swap(lmode);
        std::vector<uint8_t>().swap(edge_v);
        std::vector<uint8_t>().swap(edge_h);
        std::vector<int8_t>().swap(qpmap);
    }
};

// Removes emulation_prevention_three_byte (7.4.2): 0x000003 -> 0x0000.
std::vector<uint8_t> unescape(const uint8_t* d, size_t n) {
    std::vector<uint8_t> o;
    o.reserve(n);
    int zeros = 0;
    for (size_t i = 0; i < n; ++i) {
        if (zeros >= 2 && d[i] == 3) {
            zeros = 0;
            continue;
        }
        zeros = d[i] == 0 ? zeros + 1 : 0;
        o.push_back(d[i]);
    }
    return o;
}

}  // namespace

struct hpvcd_syntax_pic {
    std::unique_ptr<Decoder> d;
    hpvcd_picture desc{};
    uint64_t bins = 0;
};

namespace {

hpvcd_status decode_one(const hpvcd_slice_params* sp, const uint8_t* data, uint64_t bytes, hpvcd_syntax_pic** out,
                        char* msg, size_t msg_len) {
    *out = nullptr;
    std::unique_ptr<hpvcd_syntax_pic> p(new (std::nothrow) hpvcd_syntax_pic());
    if (!p) return HPVCD_ERR_ALLOC;
    try {
        p->d.reset(new Decoder(*sp));
        Decoder& D = *p->d;
        const hpvcd_status st = D.setup();
        if (st != HPVCD_OK) {
            snprintf(msg, msg_len, "%s", D.msg);
            return st;
        }
        if (sp->flags & HPVCD_SLICE_EBSP) {
            const std::vector<uint8_t> rbsp = unescape(data, (size_t)bytes);
            D.run(rbsp.data(), rbsp.size());
        } else {
            D.run(data, (size_t)bytes);
        }
        p->bins = D.E.bins;
    } catch (const Fail&) {
        snprintf(msg, msg_len, "%s", p->d->msg);
        return HPVCD_ERR_BITSTREAM;
    } catch (const std::bad_alloc&) {
        snprintf(msg, msg_len, "out of host memory in the syntax decode");
        return HPVCD_ERR_ALLOC;
    }
    const Decoder& D = *p->d;
    hpvcd_picture& d = p->desc;
    d.width = sp->width;
    d.height = sp->height;
    d.chroma_idc = sp->chroma_idc;
    d.bit_depth_y = sp->bit_depth_y;
    d.bit_depth_c = sp->bit_depth_c;
    d.log2_ctb = sp->log2_ctb;
    d.flags = (sp->flags & HPVCD_SLICE_STRONG_SMOOTHING ? HPVCD_PIC_STRONG_SMOOTHING : 0) |
              (sp->flags & HPVCD_SLICE_DEBLOCK ? HPVCD_PIC_DEBLOCK : 0) |
              (sp->flags & HPVCD_SLICE_SAO_LUMA ? HPVCD_PIC_SAO_LUMA : 0) |
              (sp->flags & HPVCD_SLICE_SAO_CHROMA ? HPVCD_PIC_SAO_CHROMA : 0);
    d.beta_offset_div2 = sp->beta_offset_div2;
    d.tc_offset_div2 = sp->tc_offset_div2;
    d.pps_cb_qp_offset = sp->pps_cb_qp_offset;
    d.pps_cr_qp_offset = sp->pps_cr_qp_offset;
    d.n_tus = (uint32_t)D.tus.size();
    d.n_pus = 0;
    d.n_coeffs = D.coeffs.size();
    d.tus = D.tus.data();
    d.ctu_tu_start = D.ctu_start.data();
    d.coeffs = D.coeffs.empty() ? nullptr : D.coeffs.data();
    d.cells = D.cells.data();
    d.sao = D.sao.empty() ? nullptr : D.sao.data();
    for (int l = 0; l < 2; ++l)
        for (int r = 0; r < HPVCD_MAX_REFS; ++r) d.ref_slot[l][r] = -1;
    d.scaling = D.has_scaling ? &D.scaling : nullptr;
    *out = p.release();
    return HPVCD_OK;
}

}  // namespace

HPVCD_API hpvcd_status hpvcd_syntax_decode(const hpvcd_slice_params* params, const uint8_t* data, uint64_t bytes,
                                           hpvcd_syntax_pic** out) {
    if (!params || !out || (!data && bytes)) return HPVCD_ERR_INVALID_ARG;
    char msg[200] = "";
    const hpvcd_status st = decode_one(params, data, bytes, out, msg, sizeof(msg));
    if (st != HPVCD_OK) hpvcd_note_error(msg);
    return st;
}

HPVCD_API hpvcd_status hpvcd_syntax_decode_batch(uint32_t n, const hpvcd_slice_params* params,
                                                 const uint8_t* const* data, const uint64_t* bytes, uint32_t threads,
                                                 hpvcd_syntax_pic** out, hpvcd_status* st) {
    if (!params || !data || !bytes || !out || (n && !out)) return HPVCD_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; ++i) out[i] = nullptr;
    unsigned hw = std::thread::hardware_concurrency();
    uint32_t nt = threads ? threads : (hw ? hw : 1);
    nt = std::max<uint32_t>(1, std::min<uint32_t>(nt, n));
    std::vector<hpvcd_status> res(n, HPVCD_OK);
    std::vector<std::string> msgs(n);
    std::atomic<uint32_t> next{0};
    auto work = [&]() {
        char m[200];
        for (uint32_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) {
            m[0] = 0;
            res[i] = data[i] || !bytes[i] ? decode_one(&params[i], data[i], bytes[i], &out[i], m, sizeof(m))
                                          : HPVCD_ERR_INVALID_ARG;
            if (res[i] != HPVCD_OK) msgs[i] = m;
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (std::thread& t : pool) t.join();
    hpvcd_status first = HPVCD_OK;
    for (uint32_t i = 0; i < n; ++i) {
        if (st) st[i] = res[i];
        if (res[i] != HPVCD_OK && first == HPVCD_OK) {
            first = res[i];
            char m[256];
            snprintf(m, sizeof(m), "slice %u: %s", i, msgs[i].c_str());
            hpvcd_note_error(m);
        }
    }
    return first;
}

HPVCD_API hpvcd_status hpvcd_syntax_picture(const hpvcd_syntax_pic* p, hpvcd_picture* out) {
    if (!p || !out) return HPVCD_ERR_INVALID_ARG;
    *out = p->desc;
    return HPVCD_OK;
}

HPVCD_API uint64_t hpvcd_syntax_bins(const hpvcd_syntax_pic* p) { return p ? p->bins : 0; }

HPVCD_API void hpvcd_syntax_free(hpvcd_syntax_pic* p) { delete p; }
