// synth.cpp -- seeded generator of flat per-picture reconstruction buffers.
// It plays the role of the host-side syntax decode of hpvcd: it emits the
// same records decode.rs fills while parsing (TB list in decode order,
// per-4x4 deblocking maps, per-CTB SAO parameters, PUs), drawn from seeded
// distributions instead of a bitstream.
#include "hpvcd_synth.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace {

struct Rng {  // splitmix64
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x1234567ull) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uni() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    bool bern(double p) { return uni() < p; }
    int range(int lo, int hi) {  // inclusive
        return lo + (int)(next() % (uint64_t)(hi - lo + 1));
    }
    double gauss() {
        double u1 = uni(), u2 = uni();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct CellMeta {
    bool tu_v = false, tu_h = false, pu_v = false, pu_h = false;
    bool intra = false, nz = false;
    uint8_t pred = 0;  // bit0 L0, bit1 L1
    int8_t ref[2] = {-1, -1};
    int16_t mv[2][2] = {{0, 0}, {0, 0}};
};

struct Picture {
    hpvcd_picture desc{};
    std::vector<hpvcd_tu> tus;
    std::vector<uint32_t> ctu_start;
    std::vector<int16_t> coeffs;
    std::vector<hpvcd_cell> cells;
    std::vector<hpvcd_sao_ctb> sao;
    std::vector<hpvcd_pu> pus;
    hpvcd_wp_table wp{};
    bool has_wp = false;
    hpvcd_scaling scaling{};
    bool has_scaling = false;
    std::vector<uint16_t> ctb_region;
    std::vector<int8_t> slice_deblock;  // 256 x {beta, tc} div2
    std::vector<uint8_t> pred8[3];
    std::vector<uint16_t> pred16[3];
};

struct Gen {
    const hpvcd_synth_cfg& c;
    Rng rng;
    Picture& P;
    int w, h, idc, sub_w, sub_h, gw, gh, bd, log2_ctb;
    int pic_index;
    std::vector<CellMeta> meta;

    Gen(const hpvcd_synth_cfg& cfg, Picture& pic, int index)
        : c(cfg), rng(cfg.seed), P(pic), pic_index(index) {
        w = (int)c.width;
        h = (int)c.height;
        idc = (int)c.chroma_idc;
        sub_w = idc == 1 || idc == 2 ? 2 : 1;  // SubWidthC
        sub_h = idc == 1 ? 2 : 1;              // SubHeightC
        gw = (w + 3) / 4;
        gh = (h + 3) / 4;
        bd = (int)c.bit_depth;
        log2_ctb = (int)c.log2_ctb;
        meta.assign((size_t)gw * gh, CellMeta());
    }

    CellMeta& cell(int x, int y) { return meta[(size_t)(y / 4) * gw + x / 4]; }

    int16_t level() {
        // Non-zero magnitude: 1 + floor(Exp(scale)), i.e. a rounded Laplacian
        // conditioned on being non-zero; random sign; int16 range.
        double u = rng.uni();
        if (u < 1e-12) u = 1e-12;
        double mag = 1.0 + std::floor(-std::log(u) * c.laplace_scale);
        if (mag > 32767.0) mag = 32767.0;
        int v = (int)mag;
        return (int16_t)(rng.bern(0.5) ? -v : v);
    }

    // Coefficients of one coded TB: last significant position uniform in
    // raster order, zero_frac zeros before it.  Returns nx = max_x + 1.
    uint8_t make_levels(int n, uint32_t* off) {
        *off = (uint32_t)P.coeffs.size();
        P.coeffs.resize(P.coeffs.size() + (size_t)n * n, 0);
        int16_t* lv = P.coeffs.data() + *off;
        const int last = rng.range(0, n * n - 1);
        int max_x = 0;
        for (int i = 0; i <= last; ++i) {
            if (i == last || !rng.bern(c.zero_frac)) {
                lv[i] = level();
                max_x = std::max(max_x, i % n);
            }
        }
        return (uint8_t)(max_x + 1);
    }

    void push_tb(int comp, int x, int y, int log2n, uint8_t flags, int mode, int qp, int cqp_off,
                 int res_scale = 0) {
        hpvcd_tu t{};
        t.res_scale = (int8_t)res_scale;
        t.x = (uint16_t)x;
        t.y = (uint16_t)y;
        t.log2n = (uint8_t)log2n;
        t.comp = (uint8_t)comp;
        t.mode = (uint8_t)mode;
        t.qp_y = (int8_t)qp;
        t.cqp_off = (int8_t)cqp_off;
        const int n = 1 << log2n;
        const int ts_max = c.tskip_log2_max > 2 ? (int)c.tskip_log2_max : 2;
        if ((flags & HPVCD_TU_CBF) && log2n <= ts_max && !(flags & HPVCD_TU_TQB) && rng.bern(c.tskip_p))
            flags |= HPVCD_TU_TSKIP;
        // decode.rs:4356-4374 rext_post_ops, resolved here as the host does
        if (c.rext && (flags & HPVCD_TU_CBF) && (flags & (HPVCD_TU_TSKIP | HPVCD_TU_TQB))) {
            const bool inter = !(flags & HPVCD_TU_INTRA);
            if ((c.rext & 1) && (flags & HPVCD_TU_TSKIP) && !(flags & HPVCD_TU_TQB) && log2n == 2 && !inter)
                flags |= HPVCD_TU_ROTATE;
            if (inter) {
                if (c.rext & 4) {
                    const int d = rng.range(0, 2);
                    if (d) flags |= d == 1 ? HPVCD_TU_RDPCM_H : HPVCD_TU_RDPCM_V;
                }
            } else if ((c.rext & 2) && (mode == 10 || mode == 26)) {
                flags |= mode == 26 ? HPVCD_TU_RDPCM_V : HPVCD_TU_RDPCM_H;
            }
        }
        t.flags = flags;
        if (flags & HPVCD_TU_CBF) {
            t.nx = make_levels(n, &t.coeff_off);
        } else {
            t.nx = 0;
            t.coeff_off = 0;
        }
        P.tus.push_back(t);
    }

    void mark_tu_edges(int x0, int y0, int size) {
        if (x0 > 0 && x0 < w)
            for (int y = y0; y < std::min(y0 + size, h); y += 4) cell(x0, y).tu_v = true;
        if (y0 > 0 && y0 < h)
            for (int x = x0; x < std::min(x0 + size, w); x += 4) cell(x, y0).tu_h = true;
    }
    void mark_pu_edges(int x0, int y0, int pw, int ph) {
        if (x0 > 0 && x0 < w)
            for (int y = y0; y < std::min(y0 + ph, h); y += 4) cell(x0, y).pu_v = true;
        if (y0 > 0 && y0 < h)
            for (int x = x0; x < std::min(x0 + pw, w); x += 4) cell(x, y0).pu_h = true;
    }
    void fill_cells(int x0, int y0, int size, int qp, bool exempt, bool intra) {
        for (int y = y0; y < std::min(y0 + size, h); y += 4)
            for (int x = x0; x < std::min(x0 + size, w); x += 4) {
                hpvcd_cell& cl = P.cells[(size_t)(y / 4) * gw + x / 4];
                cl.qp_y = (int8_t)qp;
                cl.flags = (exempt ? HPVCD_CELL_EXEMPT : 0) | (intra ? 0 : HPVCD_CELL_INTER);
                cell(x, y).intra = intra;
            }
    }

    // TU split probability at a level: tu_split_p, or the conditional
    // probability that a TB of this size splits given the target area mix.
    float split_p(int log2) const {
        const float* m = c.tu_mix;
        const float tot = m[0] + m[1] + m[2] + m[3];
        if (!(tot > 0.f)) return c.tu_split_p;
        float below = 0.f;  // mass of the sizes smaller than this level
        for (int k = 0; k < log2 - 2; ++k) below += m[k];
        const float here = m[log2 - 2];
        return below + here > 0.f ? below / (below + here) : 1.f;
    }

    // Transform tree of an intra or inter CU (decode.rs:3315 transform_tree,
    // :3478 transform_unit ordering: luma TB, then Cb TB(s), then Cr TB(s);
    // for 4:2:0 4x4 luma TBs the chroma TB follows the fourth one).
    void transform_tree(int x0, int y0, int xbase, int ybase, int log2, int depth, int blk,
                        bool intra, bool nxn, const int* lmodes, const int* cmodes, int cu_x,
                        int cu_y, int cu_size, int qp, bool tqb) {
        if (x0 >= w || y0 >= h) return;
        const int size = 1 << log2;
        bool split = log2 > 5 || (nxn && depth == 0);
        if (!split && log2 > 2 && rng.bern(split_p(log2))) split = true;
        if (split) {
            const int half = size / 2;
            for (int b = 0; b < 4; ++b)
                transform_tree(x0 + (b & 1) * half, y0 + (b >> 1) * half, x0, y0, log2 - 1, depth + 1,
                               b, intra, nxn, lmodes, cmodes, cu_x, cu_y, cu_size, qp, tqb);
            return;
        }
        const int pu = nxn ? cu_size / 2 : cu_size;
        const int q = nxn ? ((x0 - cu_x) >= pu ? 1 : 0) + ((y0 - cu_y) >= pu ? 2 : 0) : 0;
        uint8_t base = (intra ? HPVCD_TU_INTRA : 0) | (tqb ? HPVCD_TU_TQB : 0);
        const bool cbf_l = rng.bern(c.cbf_p);
        if (intra || cbf_l)
            push_tb(0, x0, y0, log2, base | (cbf_l ? HPVCD_TU_CBF : 0), lmodes[q], qp, 0);
        mark_tu_edges(x0, y0, size);
        if (cbf_l && !intra)
            for (int y = y0; y < std::min(y0 + size, h); y += 4)
                for (int x = x0; x < std::min(x0 + size, w); x += 4) cell(x, y).nz = true;
        if (idc == 0) return;
        int cx, cy, clog2;
        if (log2 > 2 || idc == 3) {
            cx = x0 / sub_w;
            cy = y0 / sub_h;
            clog2 = idc == 3 ? log2 : log2 - 1;
        } else if (blk == 3) {
            cx = xbase / sub_w;
            cy = ybase / sub_h;
            clog2 = 2;
        } else {
            return;
        }
        const int cmode = idc == 3 ? cmodes[q] : cmodes[0];
        const bool ccp_on = c.ccp_p > 0.f && idc == 3 && cbf_l;
        // 4:2:2: two square chroma TBs stacked per component, all Cb then all
        // Cr (decode.rs:5034-5060), each with its own cbf
        const int n_tb = idc == 2 ? 2 : 1;
        for (int comp = 1; comp <= 2; ++comp)
            for (int t = 0; t < n_tb; ++t) {
                const bool cbf = rng.bern(c.cbf_p);
                int rs = 0;  // cross_comp_pred ResScaleVal
                if (ccp_on && rng.bern(c.ccp_p)) rs = (rng.bern(0.5) ? -1 : 1) * (1 << rng.range(0, 3));
                if (!intra && !cbf && !rs) continue;
                push_tb(comp, cx, cy + (t << clog2), clog2, base | (cbf ? HPVCD_TU_CBF : 0), cmode, qp, 0, rs);
            }
    }

    int chroma_mode_for(int lmode) {  // H.265 Table 8-2 (intra_chroma_pred_mode 0..4)
        static const int cand[4] = {0, 26, 10, 1};
        const int sel = rng.range(0, 4);
        if (sel == 4) return lmode;
        return cand[sel] == lmode ? 34 : cand[sel];
    }

    void intra_cu(int x0, int y0, int log2, int qp, bool tqb) {
        const int size = 1 << log2;
        const bool nxn = log2 == 3 && rng.bern(0.5);
        int lmodes[4], cmodes[4];
        for (int i = 0; i < 4; ++i) lmodes[i] = rng.range(0, 34);
        if (!nxn)
            for (int i = 1; i < 4; ++i) lmodes[i] = lmodes[0];
        for (int i = 0; i < 4; ++i) cmodes[i] = chroma_mode_for(lmodes[i]);
        if (!nxn || idc != 3)
            for (int i = 1; i < 4; ++i) cmodes[i] = cmodes[0];
        fill_cells(x0, y0, size, qp, tqb, true);
        transform_tree(x0, y0, x0, y0, log2, 0, 0, true, nxn, lmodes, cmodes, x0, y0, size, qp, tqb);
    }

    void inter_cu(int x0, int y0, int log2, int qp, bool tqb) {
        const int size = 1 << log2;
        fill_cells(x0, y0, size, qp, tqb, false);
        // Partition: 2Nx2N, 2NxN or Nx2N (PUs of at least 8x8).
        int part = 0;
        if (log2 >= 4) {
            const double u = rng.uni();
            part = u < 0.6 ? 0 : (u < 0.8 ? 1 : 2);
        }
        const int np = part == 0 ? 1 : 2;
        const int nref = std::min<int>((int)c.n_refs, pic_index);
        for (int k = 0; k < np; ++k) {
            hpvcd_pu u{};
            u.w = (uint16_t)(part == 2 ? size / 2 : size);
            u.h = (uint16_t)(part == 1 ? size / 2 : size);
            u.x = (uint16_t)(x0 + (part == 2 ? k * size / 2 : 0));
            u.y = (uint16_t)(y0 + (part == 1 ? k * size / 2 : 0));
            const bool bi = nref > 0 && rng.bern(c.bi_p);
            const int l_first = rng.bern(0.5) ? 0 : 1;
            for (int l = 0; l < 2; ++l) {
                const bool use = bi || l == l_first;
                if (!use || nref == 0) continue;
                u.flags |= l ? HPVCD_PU_L1 : HPVCD_PU_L0;
                u.ref_idx[l] = (int8_t)rng.range(0, nref - 1);
                for (int d = 0; d < 2; ++d) {
                    const double sd = c.mv_sd * 4.0;  // quarter-pel
                    int mv = (int)std::lround(rng.gauss() * sd);
                    const int pos = d == 0 ? u.x : u.y;
                    const int ext = d == 0 ? u.w : u.h;
                    const int lim = d == 0 ? w : h;
                    const int lo = (int)(-(pos + c.mv_pad) * 4);
                    const int hi = (int)((lim + c.mv_pad - pos - ext) * 4);
                    mv = std::min(std::max(mv, lo), hi);
                    mv = std::min(std::max(mv, -32768), 32767);
                    u.mv[l][d] = (int16_t)mv;
                }
            }
            if (u.flags == 0) {  // no reference available: fall back to intra
                intra_cu(x0, y0, log2, qp, tqb);
                return;
            }
            P.pus.push_back(u);
            mark_pu_edges(u.x, u.y, u.w, u.h);
            for (int y = u.y; y < std::min<int>(u.y + u.h, h); y += 4)
                for (int x = u.x; x < std::min<int>(u.x + u.w, w); x += 4) {
                    CellMeta& m = cell(x, y);
                    m.pred = u.flags & 3;
                    for (int l = 0; l < 2; ++l) {
                        m.ref[l] = (u.flags >> l) & 1 ? (int8_t)P.desc.ref_slot[l][u.ref_idx[l]] : -1;
                        m.mv[l][0] = u.mv[l][0];
                        m.mv[l][1] = u.mv[l][1];
                    }
                }
        }
        int dummy[4] = {0, 0, 0, 0};
        transform_tree(x0, y0, x0, y0, log2, 0, 0, false, false, dummy, dummy, x0, y0, size, qp, tqb);
        // decode.rs:6546-6548 finish_inter_cu marks the CU decoded.
        hpvcd_tu t{};
        t.x = (uint16_t)x0;
        t.y = (uint16_t)y0;
        t.log2n = (uint8_t)log2;
        t.comp = 0;
        t.flags = 0;
        t.qp_y = (int8_t)qp;
        P.tus.push_back(t);
    }

    void coding_quadtree(int x0, int y0, int log2) {
        if (x0 >= w || y0 >= h) return;
        const int size = 1 << log2;
        const bool in_pic = x0 + size <= w && y0 + size <= h;
        const bool split = log2 > 3 && (!in_pic || rng.bern(c.cu_split_p));
        if (split) {
            const int half = size / 2;
            for (int b = 0; b < 4; ++b) coding_quadtree(x0 + (b & 1) * half, y0 + (b >> 1) * half, log2 - 1);
            return;
        }
        const int qp = rng.range(c.qp_min, c.qp_max);
        const bool tqb = rng.bern(c.tqb_p);
        const bool inter = c.kind == HPVCD_SYNTH_INTER && !rng.bern(c.intra_cu_p);
        if (inter)
            inter_cu(x0, y0, log2, qp, tqb);
        else if (c.pcm_p > 0.f && log2 >= 3 && log2 <= 5 && rng.bern(c.pcm_p))
            pcm_cu(x0, y0, log2, qp);
        else
            intra_cu(x0, y0, log2, qp, tqb);
    }

    // I_PCM CU (decode.rs:2768-2839): one record per component whose levels
    // are the samples, pcm_sample << (BitDepth - PcmBitDepth).
    void pcm_cu(int x0, int y0, int log2, int qp) {
        const int size = 1 << log2;
        fill_cells(x0, y0, size, qp, rng.bern(0.5), true);  // exempt: pcm_loop_filter_disabled
        mark_tu_edges(x0, y0, size);
        const int pbd = rng.range(std::max(1, bd - 4), bd);
        auto push_pcm = [&](int comp, int x, int y, int lg) {
            hpvcd_tu t{};
            t.x = (uint16_t)x;
            t.y = (uint16_t)y;
            t.log2n = (uint8_t)lg;
            t.comp = (uint8_t)comp;
            t.flags = HPVCD_TU_CBF | HPVCD_TU_INTRA | HPVCD_TU_PCM;
            t.mode = 1;
            t.qp_y = (int8_t)qp;
            const int n = 1 << lg;
            t.nx = (uint8_t)n;
            t.coeff_off = (uint32_t)P.coeffs.size();
            for (int i = 0; i < n * n; ++i) P.coeffs.push_back((int16_t)(rng.range(0, (1 << pbd) - 1) << (bd - pbd)));
            P.tus.push_back(t);
        };
        push_pcm(0, x0, y0, log2);
        if (idc == 0) return;
        const int clog2 = idc == 3 ? log2 : log2 - 1, n_tb = idc == 2 ? 2 : 1;
        for (int comp = 1; comp <= 2; ++comp)
            for (int t = 0; t < n_tb; ++t) push_pcm(comp, x0 / sub_w, y0 / sub_h + (t << clog2), clog2);
    }

    // Residual-only picture: quadtree of TBs from 32x32 down to 4x4, each
    // coded (PRED_IN_PLANE: planes hold a seeded uniform prediction).
    void residual_ctu(int x0, int y0, int log2, int xbase, int ybase, int blk) {
        if (x0 >= w || y0 >= h) return;
        const int size = 1 << log2;
        if (log2 > 5 || (log2 > 2 && rng.bern(split_p(log2)))) {
            for (int b = 0; b < 4; ++b)
                residual_ctu(x0 + (b & 1) * size / 2, y0 + (b >> 1) * size / 2, log2 - 1, x0, y0, b);
            return;
        }
        const int qp = rng.range(c.qp_min, c.qp_max);
        push_tb(0, x0, y0, log2, HPVCD_TU_CBF | HPVCD_TU_INTRA, 0, qp, 0);
        mark_tu_edges(x0, y0, size);
        fill_cells(x0, y0, size, qp, false, true);
        if (idc == 0) return;
        int cx, cy, clog2;
        if (log2 > 2 || idc == 3) {
            cx = x0 / sub_w;
            cy = y0 / sub_h;
            clog2 = idc == 3 ? log2 : log2 - 1;
        } else if (blk == 3) {
            cx = xbase / sub_w;
            cy = ybase / sub_h;
            clog2 = 2;
        } else {
            return;
        }
        // 4:2:2: two square chroma TBs stacked per component (decode.rs:5034)
        const int n_tb = idc == 2 ? 2 : 1;
        for (int comp = 1; comp <= 2; ++comp)
            for (int t = 0; t < n_tb; ++t)
                push_tb(comp, cx, cy + (t << clog2), clog2, HPVCD_TU_CBF | HPVCD_TU_INTRA, 0, qp, 0);
    }

    static bool motion_differs(const CellMeta& a, const CellMeta& b) {
        const int na = __builtin_popcount(a.pred), nb = __builtin_popcount(b.pred);
        if (na != nb) return true;
        auto far = [](const int16_t* u, const int16_t* v) {
            return std::abs(u[0] - v[0]) >= 4 || std::abs(u[1] - v[1]) >= 4;
        };
        if (na == 1) {
            const int la = (a.pred & 1) ? 0 : 1, lb = (b.pred & 1) ? 0 : 1;
            return a.ref[la] != b.ref[lb] || far(a.mv[la], b.mv[lb]);
        }
        if (a.ref[0] == b.ref[0] && a.ref[1] == b.ref[1])
            return far(a.mv[0], b.mv[0]) || far(a.mv[1], b.mv[1]);
        if (a.ref[0] == b.ref[1] && a.ref[1] == b.ref[0])
            return far(a.mv[0], b.mv[1]) || far(a.mv[1], b.mv[0]);
        return true;
    }

    // Boundary strengths per 4x4 cell (decode.rs:2955-3020 finalize_coeff_bs
    // and :3022-3050 mark_block_edges): 2 when either side is intra, 1 for a
    // transform edge with coefficients or a motion discontinuity.
    void finalize_bs() {
        for (int gy = 0; gy < gh; ++gy)
            for (int gx = 0; gx < gw; ++gx) {
                const size_t g = (size_t)gy * gw + gx;
                const CellMeta& m = meta[g];
                hpvcd_cell& cl = P.cells[g];
                cl.bs_v = cl.bs_h = 0;
                if (gx > 0 && (m.tu_v || m.pu_v)) {
                    const CellMeta& o = meta[g - 1];
                    if (m.intra || o.intra)
                        cl.bs_v = 2;
                    else if (m.tu_v && (m.nz || o.nz))
                        cl.bs_v = 1;
                    else if (motion_differs(m, o))
                        cl.bs_v = 1;
                }
                if (gy > 0 && (m.tu_h || m.pu_h)) {
                    const CellMeta& o = meta[g - gw];
                    if (m.intra || o.intra)
                        cl.bs_h = 2;
                    else if (m.tu_h && (m.nz || o.nz))
                        cl.bs_h = 1;
                    else if (motion_differs(m, o))
                        cl.bs_h = 1;
                }
            }
    }

    void sao_params() {
        const int ctb = 1 << log2_ctb;
        const int cols = (w + ctb - 1) / ctb, rows = (h + ctb - 1) / ctb;
        P.sao.assign((size_t)cols * rows, hpvcd_sao_ctb{});
        const int lim = 7;
        for (int ry = 0; ry < rows; ++ry)
            for (int rx = 0; rx < cols; ++rx) {
                hpvcd_sao_ctb& s = P.sao[(size_t)ry * cols + rx];
                if (rx > 0 && rng.bern(0.15)) {  // sao_merge_left
                    s = P.sao[(size_t)ry * cols + rx - 1];
                    continue;
                }
                if (ry > 0 && rng.bern(0.15)) {  // sao_merge_up
                    s = P.sao[(size_t)(ry - 1) * cols + rx];
                    continue;
                }
                for (int comp = 0; comp < 3; ++comp) {
                    hpvcd_sao_comp& sc = s.comp[comp];
                    if (comp == 2) {  // Cr shares Cb's type and EO class
                        sc.type_idx = s.comp[1].type_idx;
                        sc.eo_class = s.comp[1].eo_class;
                    } else {
                        sc.type_idx = rng.bern(c.sao_p) ? (uint8_t)rng.range(1, 2) : 0;
                        sc.eo_class = (uint8_t)rng.range(0, 3);
                    }
                    if (sc.type_idx == 1) {
                        sc.band_pos = (uint8_t)rng.range(0, 31);
                        for (int k = 0; k < 4; ++k) sc.offsets[k] = (int16_t)rng.range(-lim, lim);
                    } else if (sc.type_idx == 2) {
                        sc.band_pos = 0;
                        sc.offsets[0] = (int16_t)rng.range(0, lim);
                        sc.offsets[1] = (int16_t)rng.range(0, lim);
                        sc.offsets[2] = (int16_t)-rng.range(0, lim);
                        sc.offsets[3] = (int16_t)-rng.range(0, lim);
                    }
                }
            }
    }

    void run() {
        hpvcd_picture& d = P.desc;
        d.width = (uint32_t)w;
        d.height = (uint32_t)h;
        d.chroma_idc = (uint8_t)idc;
        d.bit_depth_y = d.bit_depth_c = (uint8_t)bd;
        d.log2_ctb = (uint8_t)log2_ctb;
        d.flags = c.pic_flags;
        if (c.ccp_p > 0.f && idc == 3) d.flags |= HPVCD_PIC_CROSS_COMPONENT;
        if (c.pcm_p > 0.f) d.flags |= HPVCD_PIC_PCM;
        d.beta_offset_div2 = (int8_t)c.beta_offset_div2;
        d.tc_offset_div2 = (int8_t)c.tc_offset_div2;
        d.pps_cb_qp_offset = (int8_t)c.cb_qp_offset;
        d.pps_cr_qp_offset = (int8_t)c.cr_qp_offset;
        for (int l = 0; l < 2; ++l)
            for (int r = 0; r < HPVCD_MAX_REFS; ++r)
                d.ref_slot[l][r] = r < pic_index ? pic_index - 1 - r : -1;
        if (c.scaling) {
            P.has_scaling = true;
            Rng sr(c.seed ^ 0x5CA1E5ull);
            for (int s = 0; s < 4; ++s)
                for (int m = 0; m < 6; ++m) {
                    const int used = s ? 8 : 4;
                    const int slope = sr.range(0, 12);
                    for (int y = 0; y < used; ++y)
                        for (int x = 0; x < used; ++x) {
                            const int v = 16 + slope * (x + y) + (int)std::lround(sr.gauss() * 6.0);
                            P.scaling.m[s][m][y * used + x] = (uint8_t)std::clamp(v, 1, 255);
                        }
                    P.scaling.dc[s][m] = (uint8_t)sr.range(1, 255);
                }
        }
        if (c.regions) {  // own seeded stream: the rest of the picture is unchanged
            Rng rr(c.seed ^ 0x7E61045ull);
            const int ctbz = 1 << log2_ctb;
            const int cols = (w + ctbz - 1) / ctbz, rows = (h + ctbz - 1) / ctbz, n = cols * rows;
            P.ctb_region.assign((size_t)n, 0);
            if (c.regions == 1 && n >= 3) {
                int a = rr.range(1, n - 2), b = rr.range(1, n - 1);
                if (a > b) std::swap(a, b);
                if (a == b) b = std::min(n - 1, b + 1);
                for (int i = 0; i < n; ++i) P.ctb_region[(size_t)i] = (uint16_t)((i >= a) + (i >= b)) << 8;
                P.slice_deblock.assign(512, 0);
                for (int k = 0; k < 3; ++k) {  // each slice its own offsets
                    P.slice_deblock[(size_t)2 * k] = (int8_t)rr.range(-6, 6);
                    P.slice_deblock[(size_t)2 * k + 1] = (int8_t)rr.range(-6, 6);
                }
            } else if (c.regions == 2) {
                for (int y = 0; y < rows; ++y)
                    for (int x = 0; x < cols; ++x) {
                        const int tile = (x >= (cols + 1) / 2) + 2 * (y >= (rows + 1) / 2);
                        P.ctb_region[(size_t)y * cols + x] = (uint16_t)(tile << 8 | tile);
                    }
            }
        }
        P.cells.assign((size_t)gw * gh, hpvcd_cell{});
        const int ctb = 1 << log2_ctb;
        const int cols = (w + ctb - 1) / ctb, rows = (h + ctb - 1) / ctb;
        P.ctu_start.assign((size_t)cols * rows + 1, 0);
        if (c.kind == HPVCD_SYNTH_INTER) {
            d.flags |= HPVCD_PIC_INTER;
            if (c.weighted && pic_index > 0) {
                P.has_wp = true;
                hpvcd_wp_table& t = P.wp;
                t.luma_log2_denom = (uint8_t)rng.range(0, 7);
                t.chroma_log2_denom = (uint8_t)rng.range(0, 7);
                const int sh = bd - 8;
                for (int l = 0; l < 2; ++l)
                    for (int r = 0; r < HPVCD_MAX_REFS; ++r) {
                        hpvcd_wp_entry& e = t.e[l][r];
                        e.luma_w = (int16_t)rng.range(0, 127);
                        e.luma_o = (int16_t)(rng.range(-20, 20) * (1 << sh));
                        e.cb_w = (int16_t)rng.range(0, 127);
                        e.cb_o = (int16_t)(rng.range(-20, 20) * (1 << sh));
                        e.cr_w = (int16_t)rng.range(0, 127);
                        e.cr_o = (int16_t)(rng.range(-20, 20) * (1 << sh));
                    }
            }
        }
        for (int ry = 0; ry < rows; ++ry)
            for (int rx = 0; rx < cols; ++rx) {
                P.ctu_start[(size_t)ry * cols + rx] = (uint32_t)P.tus.size();
                if (c.kind == HPVCD_SYNTH_RESIDUAL)
                    residual_ctu(rx * ctb, ry * ctb, log2_ctb, rx * ctb, ry * ctb, 0);
                else
                    coding_quadtree(rx * ctb, ry * ctb, log2_ctb);
            }
        P.ctu_start[(size_t)cols * rows] = (uint32_t)P.tus.size();
        finalize_bs();
        if (c.sao_p > 0) sao_params();
        if (c.kind == HPVCD_SYNTH_RESIDUAL) {
            d.flags |= HPVCD_PIC_PRED_IN_PLANE;
            const int cw = idc ? (w + sub_w - 1) / sub_w : 0, ch = idc ? (h + sub_h - 1) / sub_h : 0;
            for (int comp = 0; comp < (idc ? 3 : 1); ++comp) {
                const size_t cnt = comp == 0 ? (size_t)w * h : (size_t)cw * ch;
                if (bd <= 8) {
                    P.pred8[comp].resize(cnt);
                    for (size_t k = 0; k < cnt; ++k) P.pred8[comp][k] = (uint8_t)(rng.next() & 255);
                } else {
                    P.pred16[comp].resize(cnt);
                    const uint32_t mx = (1u << bd) - 1;
                    for (size_t k = 0; k < cnt; ++k) P.pred16[comp][k] = (uint16_t)(rng.next() % (mx + 1));
                }
            }
        }
    }
};

}  // namespace

struct hpvcd_synth {
    std::vector<std::unique_ptr<Picture>> pics;
};

extern "C" {

void hpvcd_synth_default_cfg(hpvcd_synth_cfg* c) {
    std::memset(c, 0, sizeof(*c));
    c->seed = 0;
    c->width = 512;
    c->height = 512;
    c->kind = HPVCD_SYNTH_RESIDUAL;
    c->chroma_idc = 1;
    c->bit_depth = 8;
    c->log2_ctb = 6;
    c->cu_split_p = 0.5f;
    c->tu_split_p = 0.5f;
    c->cbf_p = 1.0f;
    c->zero_frac = 0.85f;
    c->laplace_scale = 8.0f;
    c->tskip_p = 0.0f;
    c->tqb_p = 0.0f;
    c->sao_p = 0.0f;
    c->qp_min = 22;
    c->qp_max = 37;
    c->intra_cu_p = 0.1f;
    c->bi_p = 0.4f;
    c->mv_sd = 16.0f;
    c->mv_pad = 80.0f;
    c->n_refs = 4;
}

hpvcd_synth* hpvcd_synth_new(void) { return new (std::nothrow) hpvcd_synth(); }
void hpvcd_synth_free(hpvcd_synth* s) { delete s; }

int32_t hpvcd_synth_add(hpvcd_synth* s, const hpvcd_synth_cfg* cfg) {
    if (!s || !cfg) return -HPVCD_ERR_INVALID_ARG;
    if (cfg->width == 0 || cfg->height == 0 || (cfg->width & 7) || (cfg->height & 7) ||
        cfg->width > 16384 || cfg->height > 16384)
        return -HPVCD_ERR_INVALID_ARG;
    if (cfg->chroma_idc > 3 || cfg->bit_depth < 8 || cfg->bit_depth > 12 ||
        cfg->log2_ctb < 4 || cfg->log2_ctb > 6 || cfg->qp_min > cfg->qp_max)
        return -HPVCD_ERR_INVALID_ARG;
    auto pic = std::make_unique<Picture>();
    const int index = (int)s->pics.size();
    Gen g(*cfg, *pic, index);
    g.run();
    hpvcd_picture& d = pic->desc;
    d.n_tus = (uint32_t)pic->tus.size();
    d.tus = pic->tus.data();
    d.ctu_tu_start = pic->ctu_start.data();
    d.n_coeffs = pic->coeffs.size();
    d.coeffs = pic->coeffs.data();
    d.cells = pic->cells.data();
    d.sao = pic->sao.empty() ? nullptr : pic->sao.data();
    d.n_pus = (uint32_t)pic->pus.size();
    d.pus = pic->pus.empty() ? nullptr : pic->pus.data();
    d.wp = pic->has_wp ? &pic->wp : nullptr;
    d.scaling = pic->has_scaling ? &pic->scaling : nullptr;
    d.ctb_region = pic->ctb_region.empty() ? nullptr : pic->ctb_region.data();
    d.slice_deblock = pic->slice_deblock.empty() ? nullptr : pic->slice_deblock.data();
    for (int c = 0; c < 3; ++c)
        d.pred[c] = !pic->pred8[c].empty() ? (const void*)pic->pred8[c].data()
                    : !pic->pred16[c].empty() ? (const void*)pic->pred16[c].data()
                                              : nullptr;
    s->pics.push_back(std::move(pic));
    return index;
}

uint32_t hpvcd_synth_count(const hpvcd_synth* s) { return s ? (uint32_t)s->pics.size() : 0; }

int32_t hpvcd_synth_get(const hpvcd_synth* s, uint32_t i, hpvcd_picture* out) {
    if (!s || !out || i >= s->pics.size()) return HPVCD_ERR_INVALID_ARG;
    *out = s->pics[i]->desc;
    return HPVCD_OK;
}

}  // extern "C"
