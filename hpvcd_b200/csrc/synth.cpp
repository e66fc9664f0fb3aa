// synth.cpp -- seeded generator of flat per-picture reconstruction buffers.
// It plays the role of the host-side syntax decode of hpvcd: it emits the
// same records decode.rs fills while parsing (TB list in decode order,
// per-4x4 deblocking maps, per-CTB SAO parameters, PUs), drawn from seeded
// distributions instead of a bitstream.
#include "hpvcd_synth.h"

#include "cabac_tables.h"

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
    // bitstream mode: the slice data written for this picture, and the
    // parameters it was written with
    std::vector<uint8_t> slice;
    hpvcd_slice_params slice_params{};
};

// Coding units of an intra picture as generated, for the bitstream writer:
// transform-tree leaves in decode order with the range of TB records each
// produced.
struct TtLeaf {
    int x, y, log2;
    uint32_t tb_first, tb_end;
};
struct CuRec {
    int x, y, log2;
    bool tqb, nxn;
    int lm[4], cm[4];
    int qp;
    uint32_t tb_first, tb_end;
    std::vector<TtLeaf> leaves;
};

struct Gen {
    const hpvcd_synth_cfg& c;
    Rng rng;
    Picture& P;
    int w, h, idc, sub_w, sub_h, gw, gh, bd, log2_ctb;
    int pic_index;
    std::vector<CellMeta> meta;
    std::vector<CuRec> cus;  // bitstream mode: intra CUs in decode order

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
        const uint32_t tb0 = (uint32_t)P.tus.size();
        leaf_tbs(x0, y0, xbase, ybase, log2, blk, intra, nxn, lmodes, cmodes, cu_x, cu_y, cu_size, qp, tqb);
        if (c.bitstream && intra && !cus.empty())
            cus.back().leaves.push_back(TtLeaf{x0, y0, log2, tb0, (uint32_t)P.tus.size()});
    }

    void leaf_tbs(int x0, int y0, int xbase, int ybase, int log2, int blk, bool intra, bool nxn,
                  const int* lmodes, const int* cmodes, int cu_x, int cu_y, int cu_size, int qp, bool tqb) {
        const int size = 1 << log2;
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
        if (c.bitstream) {
            CuRec r{x0, y0, log2, tqb, nxn, {}, {}, qp, (uint32_t)P.tus.size(), 0, {}};
            for (int i = 0; i < 4; ++i) {
                r.lm[i] = lmodes[i];
                r.cm[i] = cmodes[i];
            }
            cus.push_back(std::move(r));
        }
        transform_tree(x0, y0, x0, y0, log2, 0, 0, true, nxn, lmodes, cmodes, x0, y0, size, qp, tqb);
        if (c.bitstream) cus.back().tb_end = (uint32_t)P.tus.size();
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

// ---------------------------------------------------------------------------
// Seeded CABAC writer: the generated intra picture as the slice_segment_data()
// of one H.265 I slice.  The arithmetic coder is the standard's encoder
// (H.265 9.3.4.3 decoding, inverted as in the informative encoding process:
// low / range registers, outstanding bits, flush); the syntax is written in
// the order the decoder reads it (7.3.8).  It shares only the normative tables
// (cabac_tables.h) with the decoder in syntax.cpp, so a round trip checks one
// against the other.
// ---------------------------------------------------------------------------

struct CabacWriter {
    std::vector<uint8_t> out;
    uint32_t cur = 0;
    int nbits = 0;
    uint32_t low = 0, range = 510;
    int outstanding = 0;
    bool first = true;
    uint8_t ctx[hpvcd_cabac::kCtxCount];

    void init(int qp) {
        for (int i = 0; i < hpvcd_cabac::kCtxCount; ++i) ctx[i] = hpvcd_cabac::init_state(hpvcd_cabac::kInitI[i], qp);
    }
    void raw(int b) {
        cur = (cur << 1) | (uint32_t)(b & 1);
        if (++nbits == 8) {
            out.push_back((uint8_t)cur);
            cur = 0;
            nbits = 0;
        }
    }
    void put(int b) {
        if (first)
            first = false;
        else
            raw(b);
        for (; outstanding > 0; --outstanding) raw(1 - b);
    }
    void renorm() {
        while (range < 256) {
            if (low < 256) {
                put(0);
            } else if (low >= 512) {
                low -= 512;
                put(1);
            } else {
                low -= 256;
                ++outstanding;
            }
            range <<= 1;
            low <<= 1;
        }
    }
    void bin(int ci, int b) {
        const int st = ctx[ci] & 63, mps = ctx[ci] >> 6;
        const uint32_t lps = hpvcd_cabac::kRangeLps[st][(range >> 6) & 3];
        range -= lps;
        if (b != mps) {
            low += range;
            range = lps;
            ctx[ci] = (uint8_t)(hpvcd_cabac::kNextLps[st] | ((st == 0 ? 1 - mps : mps) << 6));
        } else {
            ctx[ci] = (uint8_t)(hpvcd_cabac::kNextMps[st] | (mps << 6));
        }
        renorm();
    }
    void bypass(int b) {
        low <<= 1;
        if (b) low += range;
        if (low >= 1024) {
            put(1);
            low -= 1024;
        } else if (low < 512) {
            put(0);
        } else {
            low -= 512;
            ++outstanding;
        }
    }
    void bypass_bits(uint32_t v, int n) {
        for (int i = n - 1; i >= 0; --i) bypass((int)((v >> i) & 1));
    }
    void terminate(int b) {
        range -= 2;
        if (b) {
            low += range;
            range = 2;  // flush
            renorm();
            put((int)((low >> 9) & 1));
            raw((int)((low >> 8) & 1));
            raw(1);  // rbsp_stop_one_bit
            while (nbits) raw(0);
        } else {
            renorm();
        }
    }
};

struct SliceWriter {
    Gen& G;
    Picture& P;
    const hpvcd_synth_cfg& c;
    hpvcd_slice_params sp{};
    CabacWriter E;
    int w, h, idc, log2ctb, ctb, cols, rows, gw, qp_off;
    std::vector<uint8_t> depth, lmode;
    std::vector<int8_t> qpmap;
    size_t ci = 0;
    int qp_last = 0, qp_pred = 0;
    bool delta_coded = false;

    explicit SliceWriter(Gen& g) : G(g), P(g.P), c(g.c) {}

    size_t cell(int x, int y) const { return (size_t)(y >> 2) * gw + (x >> 2); }
    void fill(std::vector<uint8_t>& m, int x0, int y0, int size, uint8_t v) {
        for (int y = y0; y < std::min(y0 + size, h); y += 4)
            for (int x = x0; x < std::min(x0 + size, w); x += 4) m[cell(x, y)] = v;
    }

    void params() {
        w = G.w;
        h = G.h;
        idc = G.idc;
        log2ctb = G.log2_ctb;
        ctb = 1 << log2ctb;
        cols = (w + ctb - 1) / ctb;
        rows = (h + ctb - 1) / ctb;
        gw = G.gw;
        qp_off = 6 * (G.bd - 8);
        sp.width = (uint32_t)w;
        sp.height = (uint32_t)h;
        sp.chroma_idc = (uint8_t)idc;
        sp.bit_depth_y = sp.bit_depth_c = (uint8_t)G.bd;
        sp.log2_ctb = (uint8_t)log2ctb;
        sp.log2_min_cb = 3;
        sp.log2_min_tb = 2;
        sp.log2_max_tb = (uint8_t)std::min(5, log2ctb);
        sp.max_th_depth_intra = (uint8_t)(log2ctb - 2);
        sp.diff_cu_qp_delta_depth = (uint8_t)(log2ctb - 3);  // one quantization group per CU
        sp.log2_max_tskip = (uint8_t)std::max<uint32_t>(2, c.tskip_log2_max);
        sp.pps_cb_qp_offset = (int8_t)c.cb_qp_offset;
        sp.pps_cr_qp_offset = (int8_t)c.cr_qp_offset;
        sp.slice_qp = (int8_t)std::clamp((c.qp_min + c.qp_max + 1) / 2, -qp_off, 51);
        sp.beta_offset_div2 = (int8_t)c.beta_offset_div2;
        sp.tc_offset_div2 = (int8_t)c.tc_offset_div2;
        const uint32_t pf = P.desc.flags;
        sp.flags = HPVCD_SLICE_CU_QP_DELTA | HPVCD_SLICE_EBSP | (c.tskip_p > 0.f ? HPVCD_SLICE_TSKIP : 0) |
                   (c.tqb_p > 0.f ? HPVCD_SLICE_TQ_BYPASS : 0) | (c.sign_hiding ? HPVCD_SLICE_SIGN_HIDING : 0) |
                   (pf & HPVCD_PIC_DEBLOCK ? HPVCD_SLICE_DEBLOCK : 0) |
                   (pf & HPVCD_PIC_STRONG_SMOOTHING ? HPVCD_SLICE_STRONG_SMOOTHING : 0) |
                   (pf & HPVCD_PIC_SAO_LUMA ? HPVCD_SLICE_SAO_LUMA : 0) |
                   (pf & HPVCD_PIC_SAO_CHROMA && idc ? HPVCD_SLICE_SAO_CHROMA : 0);
        sp.scaling = nullptr;  // the caller points it at the picture's lists
    }

    // SAO fields the syntax does not carry are zero; components whose slice
    // flag is off are off; no SAO array without a slice flag.
    void normalise_sao() {
        const bool luma = sp.flags & HPVCD_SLICE_SAO_LUMA, chroma = sp.flags & HPVCD_SLICE_SAO_CHROMA;
        if (!luma && !chroma) {
            P.sao.clear();
            P.desc.flags &= ~(uint32_t)(HPVCD_PIC_SAO_LUMA | HPVCD_PIC_SAO_CHROMA);
            return;
        }
        P.desc.flags &= ~(uint32_t)(HPVCD_PIC_SAO_LUMA | HPVCD_PIC_SAO_CHROMA);
        P.desc.flags |= (luma ? HPVCD_PIC_SAO_LUMA : 0) | (chroma ? HPVCD_PIC_SAO_CHROMA : 0);
        if (P.sao.empty()) P.sao.assign((size_t)cols * rows, hpvcd_sao_ctb{});
        for (hpvcd_sao_ctb& s : P.sao)
            for (int k = 0; k < 3; ++k) {
                hpvcd_sao_comp& sc = s.comp[k];
                const bool on = k == 0 ? luma : (chroma && idc);
                if (!on || sc.type_idx == 0) {
                    sc = hpvcd_sao_comp{};
                    continue;
                }
                sc.rsvd = 0;
                if (sc.type_idx == 1) sc.eo_class = 0;
                if (sc.type_idx == 2) sc.band_pos = 0;
            }
        if (idc && chroma)
            for (hpvcd_sao_ctb& s : P.sao) {  // Cr takes Cb's type and class
                s.comp[2].type_idx = s.comp[1].type_idx;
                s.comp[2].eo_class = s.comp[1].eo_class;
                if (!s.comp[2].type_idx) s.comp[2] = hpvcd_sao_comp{};
            }
    }

    void write_sao(int rx, int ry) {
        const size_t at = (size_t)ry * cols + rx;
        const hpvcd_sao_ctb& s = P.sao[at];
        if (rx > 0) {
            const bool m = memcmp(&s, &P.sao[at - 1], sizeof(s)) == 0;
            E.bin(hpvcd_cabac::kSaoMerge, m);
            if (m) return;
        }
        if (ry > 0) {
            const bool m = memcmp(&s, &P.sao[at - cols], sizeof(s)) == 0;
            E.bin(hpvcd_cabac::kSaoMerge, m);
            if (m) return;
        }
        for (int k = 0; k < (idc ? 3 : 1); ++k) {
            const bool on = k == 0 ? (sp.flags & HPVCD_SLICE_SAO_LUMA) : (sp.flags & HPVCD_SLICE_SAO_CHROMA);
            if (!on) continue;
            const hpvcd_sao_comp& sc = s.comp[k];
            if (k < 2) {
                E.bin(hpvcd_cabac::kSaoType, sc.type_idx != 0);
                if (sc.type_idx) E.bypass(sc.type_idx == 2);
            }
            if (!sc.type_idx) continue;
            const int cmax = (1 << (std::min(G.bd, 10) - 5)) - 1;
            for (int i = 0; i < 4; ++i) {
                const int a = std::abs((int)sc.offsets[i]);
                for (int b = 0; b < a; ++b) E.bypass(1);
                if (a < cmax) E.bypass(0);
            }
            if (sc.type_idx == 1) {
                for (int i = 0; i < 4; ++i)
                    if (sc.offsets[i]) E.bypass(sc.offsets[i] < 0);
                E.bypass_bits(sc.band_pos, 5);
            } else if (k < 2) {
                E.bypass_bits(sc.eo_class, 2);
            }
        }
    }

    // cbf of component `comp` over the leaves of `cu` inside a square
    bool cbf_in(const CuRec& cu, int x0, int y0, int log2, int comp) const {
        const int size = 1 << log2;
        for (const TtLeaf& l : cu.leaves)
            if (l.x >= x0 && l.x < x0 + size && l.y >= y0 && l.y < y0 + size)
                for (uint32_t t = l.tb_first; t < l.tb_end; ++t)
                    if (P.tus[t].comp == comp && (P.tus[t].flags & HPVCD_TU_CBF)) return true;
        return false;
    }
    bool leaf_cbf(const TtLeaf& l, int comp) const {
        for (uint32_t t = l.tb_first; t < l.tb_end; ++t)
            if (P.tus[t].comp == comp && (P.tus[t].flags & HPVCD_TU_CBF)) return true;
        return false;
    }
    // cbf_luma || cbfChroma of a leaf as transform_unit sees them
    bool leaf_codes(const CuRec& cu, const TtLeaf& l) const {
        if (leaf_cbf(l, 0)) return true;
        if (!idc) return false;
        if (l.log2 > 2 || idc == 3) return leaf_cbf(l, 1) || leaf_cbf(l, 2);
        const int px = l.x & ~7, py = l.y & ~7;  // 4:2:0 4x4: the parent's chroma flags
        return cbf_in(cu, px, py, 3, 1) || cbf_in(cu, px, py, 3, 2);
    }

    void write_qp_delta(int d) {
        const int a = std::abs(d);
        for (int b = 0; b < std::min(a, 5); ++b) E.bin(hpvcd_cabac::kQpDelta + (b ? 1 : 0), 1);
        if (a < 5) {
            E.bin(hpvcd_cabac::kQpDelta + (a ? 1 : 0), 0);
        } else {  // EG0 suffix
            uint32_t v = (uint32_t)(a - 5);
            int k = 0;
            while (v >= (1u << k)) {
                E.bypass(1);
                v -= 1u << k;
                ++k;
            }
            E.bypass(0);
            E.bypass_bits(v, k);
        }
        if (a) E.bypass(d < 0);
    }

    void write_remaining(int v, int rice) {
        const int u = v >> rice;
        if (u < 4) {
            for (int i = 0; i < u; ++i) E.bypass(1);
            E.bypass(0);
            E.bypass_bits((uint32_t)v & ((1u << rice) - 1), rice);
            return;
        }
        for (int i = 0; i < 4; ++i) E.bypass(1);
        uint32_t r = (uint32_t)(v - (4 << rice));
        int k = rice + 1;
        while (r >= (1u << k)) {
            E.bypass(1);
            r -= 1u << k;
            ++k;
        }
        E.bypass(0);
        E.bypass_bits(r, k);
    }

    void write_last(int v, int base_ctx, int ctx_off, int ctx_shift, int cmax, int* suffix, int* nb) {
        int p = v;
        *nb = 0;
        *suffix = 0;
        if (v >= 4)
            for (p = 4; p <= cmax; ++p) {
                const int n = (p >> 1) - 1, b = (1 << n) * (2 + (p & 1));
                if (v >= b && v < b + (1 << n)) {
                    *nb = n;
                    *suffix = v - b;
                    break;
                }
            }
        for (int b = 0; b < p; ++b) E.bin(base_ctx + ctx_off + (b >> ctx_shift), 1);
        if (p < cmax) E.bin(base_ctx + ctx_off + (p >> ctx_shift), 0);
    }

    void write_residual(hpvcd_tu& t, bool tqb) {
        using namespace hpvcd_cabac;
        const int log2 = t.log2n, n = 1 << log2, comp = t.comp;
        int16_t* lv = P.coeffs.data() + t.coeff_off;
        if ((sp.flags & HPVCD_SLICE_TSKIP) && !tqb && log2 <= sp.log2_max_tskip)
            E.bin(kTskip + (comp ? 1 : 0), (t.flags & HPVCD_TU_TSKIP) != 0);
        const int scan = scan_idx(true, log2, comp, idc, t.mode);
        const Scans& S = scans();
        const int sbl = log2 - 2, nsb = 1 << sbl;
        auto at = [&](int i, int k) -> int16_t& {
            const int x = (S.pos[sbl][scan][i][0] << 2) + S.pos[2][scan][k][0];
            const int y = (S.pos[sbl][scan][i][1] << 2) + S.pos[2][scan][k][1];
            return lv[y * n + x];
        };
        int last_sb = -1, last_pos = -1;
        for (int i = nsb * nsb - 1; i >= 0 && last_sb < 0; --i)
            for (int k = 15; k >= 0; --k)
                if (at(i, k)) {
                    last_sb = i;
                    last_pos = k;
                    break;
                }
        int lx = (S.pos[sbl][scan][last_sb][0] << 2) + S.pos[2][scan][last_pos][0];
        int ly = (S.pos[sbl][scan][last_sb][1] << 2) + S.pos[2][scan][last_pos][1];
        if (scan == 2) std::swap(lx, ly);
        int ctx_off, ctx_shift;
        if (comp == 0) {
            ctx_off = 3 * (log2 - 2) + ((log2 - 1) >> 2);
            ctx_shift = (log2 + 1) >> 2;
        } else {
            ctx_off = 15;
            ctx_shift = log2 - 2;
        }
        const int cmax = (log2 << 1) - 1;
        int sx, nbx, sy, nby;
        write_last(lx, kLastX, ctx_off, ctx_shift, cmax, &sx, &nbx);
        write_last(ly, kLastY, ctx_off, ctx_shift, cmax, &sy, &nby);
        E.bypass_bits((uint32_t)sx, nbx);
        E.bypass_bits((uint32_t)sy, nby);
        uint8_t csbf[8][8];
        memset(csbf, 0, sizeof(csbf));
        int c1 = 1;
        const bool hiding_on = (sp.flags & HPVCD_SLICE_SIGN_HIDING) && !tqb;
        for (int i = last_sb; i >= 0; --i) {
            const int xs = S.pos[sbl][scan][i][0], ys = S.pos[sbl][scan][i][1];
            bool any = false;
            for (int k = 0; k < 16; ++k) any |= at(i, k) != 0;
            bool infer_dc = false;
            if (i < last_sb && i > 0) {
                int inc = 0;
                if (xs < nsb - 1) inc += csbf[xs + 1][ys];
                if (ys < nsb - 1) inc += csbf[xs][ys + 1];
                csbf[xs][ys] = any;
                E.bin(kCsbf + std::min(inc, 1) + (comp ? 2 : 0), any);
                infer_dc = true;
            } else {
                csbf[xs][ys] = 1;
            }
            int sig[16], nsig = 0;
            if (i == last_sb) sig[nsig++] = last_pos;
            if (csbf[xs][ys]) {
                int prev = 0;
                if (xs < nsb - 1) prev |= csbf[xs + 1][ys];
                if (ys < nsb - 1) prev |= csbf[xs][ys + 1] << 1;
                for (int k = (i == last_sb ? last_pos - 1 : 15); k >= 0; --k) {
                    if (k == 0 && infer_dc) {
                        sig[nsig++] = 0;  // inferred: the only level of the sub-block
                        break;
                    }
                    const int xp = S.pos[2][scan][k][0], yp = S.pos[2][scan][k][1];
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
                    const bool sg = at(i, k) != 0;
                    E.bin(kSig + (comp ? 27 + sc : sc), sg);
                    if (sg) {
                        sig[nsig++] = k;
                        infer_dc = false;
                    }
                }
            }
            if (!nsig) continue;
            const bool hidden = hiding_on && sig[0] - sig[nsig - 1] > 3;
            if (hidden) {  // the sign of the lowest-position level follows the parity of the sum
                int sum = 0;
                for (int k = 0; k < nsig; ++k) sum += std::abs((int)at(i, sig[k]));
                int16_t& f = at(i, sig[nsig - 1]);
                const int a = std::abs((int)f);
                f = (int16_t)((sum & 1) ? -a : a);
            }
            int ctx_set = (i == 0 || comp > 0) ? 0 : 2;
            if (c1 == 0) ++ctx_set;
            c1 = 1;
            int a[16], gt1[16] = {0}, first_gt1 = -1;
            for (int k = 0; k < nsig; ++k) a[k] = std::abs((int)at(i, sig[k]));
            for (int k = 0; k < std::min(nsig, 8); ++k) {
                gt1[k] = a[k] > 1;
                E.bin(kGt1 + ctx_set * 4 + std::min(c1, 3) + (comp ? 16 : 0), gt1[k]);
                if (gt1[k]) {
                    c1 = 0;
                    if (first_gt1 < 0) first_gt1 = k;
                } else if (c1 > 0 && c1 < 3) {
                    ++c1;
                }
            }
            int gt2 = 0;
            if (first_gt1 >= 0) {
                gt2 = a[first_gt1] > 2;
                E.bin(kGt2 + ctx_set + (comp ? 4 : 0), gt2);
            }
            for (int k = 0; k < nsig; ++k)
                if (!(hidden && k == nsig - 1)) E.bypass(at(i, sig[k]) < 0);
            int rice = 0;
            for (int k = 0; k < nsig; ++k) {
                const int base = 1 + (k < 8 ? gt1[k] : 0) + (k == first_gt1 ? gt2 : 0);
                const int thresh = k < 8 ? (k == first_gt1 ? 3 : 2) : 1;
                if (base == thresh) {
                    write_remaining(a[k] - base, rice);
                    if (a[k] > 3 * (1 << rice)) rice = std::min(rice + 1, 4);
                }
            }
        }
    }

    void write_tt(CuRec& cu, int x0, int y0, int log2, int tdepth, int parent_cb, int parent_cr, size_t& li) {
        using namespace hpvcd_cabac;
        const TtLeaf& l = cu.leaves[li];
        const bool split = !(l.x == x0 && l.y == y0 && l.log2 == log2);
        const int max_depth = sp.max_th_depth_intra + (cu.nxn ? 1 : 0);
        if (log2 <= sp.log2_max_tb && log2 > 2 && tdepth < max_depth && !(cu.nxn && tdepth == 0))
            E.bin(kSplitTf + 5 - log2, split);
        int cb = 0, cr = 0;
        if ((log2 > 2 && idc) || idc == 3) {
            cb = cbf_in(cu, x0, y0, log2, 1);
            cr = cbf_in(cu, x0, y0, log2, 2);
            if (tdepth == 0 || parent_cb) E.bin(kCbfChroma + tdepth, cb);
            if (tdepth == 0 || parent_cr) E.bin(kCbfChroma + tdepth, cr);
        } else if (idc) {
            cb = parent_cb;
            cr = parent_cr;
        }
        if (split) {
            const int half = 1 << (log2 - 1);
            for (int b = 0; b < 4; ++b)
                write_tt(cu, x0 + (b & 1) * half, y0 + (b >> 1) * half, log2 - 1, tdepth + 1, cb, cr, li);
            return;
        }
        const bool cbf_l = leaf_cbf(l, 0);
        E.bin(kCbfLuma + (tdepth == 0 ? 1 : 0), cbf_l);
        if ((cbf_l || cb || cr) && !delta_coded) {
            // QpY wraps modulo 52 + QpBdOffsetY (8.6.1): any QP is one delta
            // inside [-(26 + QpBdOffsetY / 2), 25 + QpBdOffsetY / 2] away
            int d = cu.qp - qp_pred;
            while (d > 25 + qp_off / 2) d -= 52 + qp_off;
            while (d < -(26 + qp_off / 2)) d += 52 + qp_off;
            write_qp_delta(d);
            delta_coded = true;
        }
        for (uint32_t t = l.tb_first; t < l.tb_end; ++t)
            if (P.tus[t].flags & HPVCD_TU_CBF) write_residual(P.tus[t], cu.tqb);
        ++li;
    }

    void write_cu(CuRec& cu, int cqt_depth) {
        using namespace hpvcd_cabac;
        const int size = 1 << cu.log2;
        // QpY: a coding unit without coded residual has no cu_qp_delta and
        // takes the prediction
        bool codes = false;
        for (const TtLeaf& l : cu.leaves) codes |= leaf_codes(cu, l);
        if (!codes) {
            cu.qp = qp_pred;
            for (uint32_t t = cu.tb_first; t < cu.tb_end; ++t) P.tus[t].qp_y = (int8_t)cu.qp;
            for (int y = cu.y; y < std::min(cu.y + size, h); y += 4)
                for (int x = cu.x; x < std::min(cu.x + size, w); x += 4) P.cells[cell(x, y)].qp_y = (int8_t)cu.qp;
        }
        if (sp.flags & HPVCD_SLICE_TQ_BYPASS) E.bin(kTqBypass, cu.tqb);
        if (cu.log2 == 3) E.bin(kPartMode, !cu.nxn);
        fill(depth, cu.x, cu.y, size, (uint8_t)cqt_depth);
        const int pb = cu.nxn ? size >> 1 : size, npu = cu.nxn ? 4 : 1;
        int prev[4], idx[4];
        for (int k = 0; k < npu; ++k) {
            const int px = cu.x + (k & 1) * pb, py = cu.y + (k >> 1) * pb;
            const int a = px > 0 ? lmode[cell(px - 1, py)] : 1;
            const int b = (py > 0 && ((py - 1) >> log2ctb) == (py >> log2ctb)) ? lmode[cell(px, py - 1)] : 1;
            int cand[3];
            mpm_list(a, b, cand);
            const int m = cu.lm[k];
            prev[k] = 0;
            for (int i = 0; i < 3; ++i)
                if (cand[i] == m) {
                    prev[k] = 1;
                    idx[k] = i;
                }
            if (!prev[k]) {
                int r = m;
                for (int i = 0; i < 3; ++i) r -= cand[i] < m;
                idx[k] = r;
            }
            fill(lmode, px, py, pb, (uint8_t)m);
        }
        for (int k = 0; k < npu; ++k) E.bin(kPrevIntra, prev[k]);
        for (int k = 0; k < npu; ++k) {
            if (prev[k]) {
                E.bypass(idx[k] > 0);
                if (idx[k] > 0) E.bypass(idx[k] > 1);
            } else {
                E.bypass_bits((uint32_t)idx[k], 5);
            }
        }
        auto icpm = [&](int cm, int lm) {
            static const int cand[4] = {0, 26, 10, 1};
            if (cm == lm) return 4;
            for (int k = 0; k < 4; ++k)
                if (cand[k] == cm || (cm == 34 && cand[k] == lm)) return k;
            return 4;
        };
        auto write_icpm = [&](int v) {
            E.bin(kChromaMode, v != 4);
            if (v != 4) E.bypass_bits((uint32_t)v, 2);
        };
        if (idc == 3)
            for (int k = 0; k < npu; ++k) write_icpm(icpm(cu.cm[k], cu.lm[k]));
        else if (idc)
            write_icpm(icpm(cu.cm[0], cu.lm[0]));
        size_t li = 0;
        write_tt(cu, cu.x, cu.y, cu.log2, 0, 0, 0, li);
        qp_last = cu.qp;
        for (int y = cu.y; y < std::min(cu.y + size, h); y += 4)
            for (int x = cu.x; x < std::min(cu.x + size, w); x += 4) qpmap[cell(x, y)] = (int8_t)cu.qp;
    }

    void write_cqt(int x0, int y0, int log2, int cqt_depth) {
        const int size = 1 << log2;
        const CuRec& cu = G.cus[ci];
        const bool split = !(cu.x == x0 && cu.y == y0 && cu.log2 == log2);
        if (x0 + size <= w && y0 + size <= h && log2 > 3) {
            int inc = 0;
            if (x0 > 0 && depth[cell(x0 - 1, y0)] > cqt_depth) ++inc;
            if (y0 > 0 && depth[cell(x0, y0 - 1)] > cqt_depth) ++inc;
            E.bin(hpvcd_cabac::kSplitCu + inc, split);
        }
        if (log2 >= log2ctb - sp.diff_cu_qp_delta_depth) {  // quantization group
            const int mask = ctb - 1;
            const int qa = (x0 & mask) ? qpmap[cell(x0 - 1, y0)] : qp_last;
            const int qb = (y0 & mask) ? qpmap[cell(x0, y0 - 1)] : qp_last;
            qp_pred = (qa + qb + 1) >> 1;
            delta_coded = false;
        }
        if (split) {
            const int half = size >> 1;
            for (int b = 0; b < 4; ++b) {
                const int x = x0 + (b & 1) * half, y = y0 + (b >> 1) * half;
                if (x < w && y < h) write_cqt(x, y, log2 - 1, cqt_depth + 1);
            }
            return;
        }
        write_cu(G.cus[ci++], cqt_depth);
    }

    void run() {
        params();
        normalise_sao();
        depth.assign((size_t)gw * G.gh, 0);
        lmode.assign((size_t)gw * G.gh, 1);
        qpmap.assign((size_t)gw * G.gh, 0);
        E.init(sp.slice_qp);
        qp_last = qp_pred = sp.slice_qp;
        for (int ry = 0; ry < rows; ++ry)
            for (int rx = 0; rx < cols; ++rx) {
                if (!P.sao.empty()) write_sao(rx, ry);
                write_cqt(rx << log2ctb, ry << log2ctb, log2ctb, 0);
                E.terminate(ry == rows - 1 && rx == cols - 1);
            }
        // emulation prevention (7.4.2): 0x0000 followed by 0..3 gets a 0x03
        P.slice.clear();
        P.slice.reserve(E.out.size() + E.out.size() / 64);
        int zeros = 0;
        for (const uint8_t b : E.out) {
            if (zeros >= 2 && b <= 3) {
                P.slice.push_back(3);
                zeros = 0;
            }
            P.slice.push_back(b);
            zeros = b == 0 ? zeros + 1 : 0;
        }
        P.slice_params = sp;
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
    if (cfg->bitstream && (cfg->kind != HPVCD_SYNTH_INTRA || cfg->chroma_idc == 2 || cfg->pcm_p > 0.f ||
                           cfg->rext || cfg->ccp_p > 0.f || cfg->regions || cfg->tskip_log2_max > 5 ||
                           cfg->qp_min < -6 * ((int)cfg->bit_depth - 8) || cfg->qp_max > 51))
        return -HPVCD_ERR_UNSUPPORTED;
    auto pic = std::make_unique<Picture>();
    const int index = (int)s->pics.size();
    Gen g(*cfg, *pic, index);
    g.run();
    if (cfg->bitstream) SliceWriter(g).run();
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

int32_t hpvcd_synth_slice(const hpvcd_synth* s, uint32_t i, hpvcd_slice_params* params, const uint8_t** data,
                          uint64_t* bytes) {
    if (!s || !params || !data || !bytes || i >= s->pics.size() || s->pics[i]->slice.empty())
        return HPVCD_ERR_INVALID_ARG;
    const Picture& P = *s->pics[i];
    *params = P.slice_params;
    params->scaling = P.has_scaling ? &P.scaling : nullptr;
    *data = P.slice.data();
    *bytes = P.slice.size();
    return HPVCD_OK;
}

int32_t hpvcd_synth_get(const hpvcd_synth* s, uint32_t i, hpvcd_picture* out) {
    if (!s || !out || i >= s->pics.size()) return HPVCD_ERR_INVALID_ARG;
    *out = s->pics[i]->desc;
    return HPVCD_OK;
}

}  // extern "C"
