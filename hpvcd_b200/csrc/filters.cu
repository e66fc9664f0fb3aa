// filters.cu -- in-loop filters and output conversion.
//
// Deblocking (deblock.rs + the serial driver decode.rs:1774-2146): every
// 4-line edge segment is independent within a pass, so one thread owns one
// segment; the vertical-edge pass runs to completion before the
// horizontal-edge pass.  Samples of exempt cells (transquant bypass, or PCM
// with pcm_loop_filter_disabled) are never written, which equals the
// reference's filter-then-restore (decode.rs:1831-1880).
//
// SAO (sao.rs + decode.rs:2258-2493): out-of-place, every sample reads the
// deblocked picture (the reference's snapshot) and writes the final plane;
// four samples per thread with vector loads and stores.
//
// RGB (yuv.rs:187-393 Q13 matrix, lib.rs:1964-1978 rgb8 narrowing,
// lib.rs:1610-1660 tile placement and cropping on the canvas).
#include <mutex>
#include <algorithm>
#include <type_traits>

#include "common.cuh"

namespace hpvcd {

// deblock.rs:34-50 (H.265 Table 8-12)
__constant__ uint8_t c_beta[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  6,  7,
                                   8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 20, 22, 24, 26, 28, 30, 32,
                                   34, 36, 38, 40, 42, 44, 46, 48, 50, 52, 54, 56, 58, 60, 62, 64};
__constant__ uint8_t c_tc[54] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,
                                 1, 1, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2,  3,  3,  3,  3,  4,
                                 4, 4, 5, 5, 6, 6, 7, 8, 9, 10, 11, 13, 14, 16, 18, 20, 22, 24};

__device__ __forceinline__ const hpvcd_cell& cell_at(const DevPic& P, int px, int py) {
    return P.cells[(size_t)(py >> 2) * P.gw + (px >> 2)];
}
__device__ __forceinline__ int qp_at(const DevPic& P, int px, int py) {
    const int gx = min(px >> 2, P.gw - 1), gy = min(py >> 2, P.gh - 1);
    return P.cells[(size_t)gy * P.gw + gx].qp_y;
}
__device__ __forceinline__ bool exempt_at(const DevPic& P, int lx, int ly) {
    return (cell_at(P, lx, ly).flags & HPVCD_CELL_EXEMPT) != 0;
}

// Deblocking offsets (div2) of the slice holding luma sample (qx, qy)
// (decode.rs:1762 slice_deblock_at: the q sample's slice).
__device__ __forceinline__ void slice_offsets(const DevPic& P, int qx, int qy, int* beta_div2, int* tc_div2) {
    *beta_div2 = P.beta_offset_div2;
    *tc_div2 = P.tc_offset_div2;
    if (P.slice_deblock && P.ctb_region) {
        const int s = P.ctb_region[(size_t)(qy >> P.log2_ctb) * P.ctb_cols + (qx >> P.log2_ctb)] >> 8;
        *beta_div2 = P.slice_deblock[2 * s];
        *tc_div2 = P.slice_deblock[2 * s + 1];
    }
}

// Cell (4x4 luma block) lookups of the filters, by cell coordinates: the
// picture's map in global memory, or the cells around a tile staged in
// shared memory (global memory outside them).
struct GCells {
    const hpvcd_cell* g;
    int gw;
    __device__ hpvcd_cell at(int gx, int gy) const { return g[(size_t)gy * gw + gx]; }
};
struct SCells {
    const hpvcd_cell* s;
    int gx0, gy0, sw, sh;  // staged cells [gx0, gx0 + sw) x [gy0, gy0 + sh)
    const hpvcd_cell* g;
    int gw;
    __device__ hpvcd_cell at(int gx, int gy) const {
        const int lx = gx - gx0, ly = gy - gy0;
        return (lx >= 0 && ly >= 0 && lx < sw && ly < sh) ? s[ly * sw + lx] : g[(size_t)gy * gw + gx];
    }
};
// QP of luma sample (px, py), positions past the picture clamped to its last cell.
template <class Cl>
__device__ __forceinline__ int qp_of(const DevPic& P, const Cl& cl, int px, int py) {
    return cl.at(min(px >> 2, P.gw - 1), min(py >> 2, P.gh - 1)).qp_y;
}
template <class Cl>
__device__ __forceinline__ bool exempt_of(const Cl& cl, int lx, int ly) {
    return (cl.at(lx >> 2, ly >> 2).flags & HPVCD_CELL_EXEMPT) != 0;
}

// Sample accessors of the deblocking segments, in plane coordinates: a
// plane in global memory, or a region of it staged in shared memory.
struct GPlane {
    void* p;
    int w, bps;
    __device__ int ld(int x, int y) const { return load_sample(p, bps, (size_t)y * w + x); }
    __device__ void st(int x, int y, int v) const { store_sample(p, bps, (size_t)y * w + x, v); }
};
struct SPlane {
    uint16_t* s;
    int x0, y0, rw;  // plane coordinates of region entry 0, region row length
    __device__ int ld(int x, int y) const { return s[(y - y0) * rw + (x - x0)]; }
    __device__ void st(int x, int y, int v) const { s[(y - y0) * rw + (x - x0)] = (uint16_t)v; }
};

// The lines of one deblocking segment: sample `tap` (negative: the P side)
// of line `line`, positioned once per segment (lines across the edge run
// along x for a vertical edge, along y for a horizontal one).
struct GLines {
    void* p;
    int bps;
    int base;    // sample index of (line 0, tap 0): planes hold fewer than 2^31 samples
    int ls, ts;  // line stride, tap stride in samples
    __device__ GLines(const GPlane& g, bool vertical, int edge, int scan)
        : p(g.p), bps(g.bps), base(vertical ? scan * g.w + edge : edge * g.w + scan),
          ls(vertical ? g.w : 1), ts(vertical ? 1 : g.w) {}
    __device__ int ld(int line, int tap) const { return load_sample(p, bps, (size_t)(base + line * ls + tap * ts)); }
    __device__ void st(int line, int tap, int v) const { store_sample(p, bps, (size_t)(base + line * ls + tap * ts), v); }
};
struct SLines {
    uint16_t* p;
    int ls, ts;
    __device__ SLines(const SPlane& r, bool vertical, int edge, int scan)
        : p(r.s + (vertical ? (scan - r.y0) * r.rw + (edge - r.x0) : (edge - r.y0) * r.rw + (scan - r.x0))),
          ls(vertical ? r.rw : 1), ts(vertical ? 1 : r.rw) {}
    __device__ int ld(int line, int tap) const { return p[line * ls + tap * ts]; }
    __device__ void st(int line, int tap, int v) const { p[line * ls + tap * ts] = (uint16_t)v; }
};
__device__ __forceinline__ GLines lines_of(const GPlane& g, bool vertical, int edge, int scan) {
    return GLines(g, vertical, edge, scan);
}
__device__ __forceinline__ SLines lines_of(const SPlane& r, bool vertical, int edge, int scan) {
    return SLines(r, vertical, edge, scan);
}

// Luma segment: 8 taps x 4 lines around the edge (tap -4..3 = p3..p0,
// q0..q3).  The decision reads lines 0 and 3; each line is then loaded,
// filtered and stored on its own, so only one line's taps are live at a time.
template <class Pl, class Cl>
__device__ __forceinline__ void luma_segment(const DevPic& P, bool vertical, int edge, int scan, const Pl& pl,
                                             const Cl& cl, bool any_exempt = true) {
    const int mid = scan + 1;
    const hpvcd_cell q = vertical ? cl.at(edge >> 2, mid >> 2) : cl.at(mid >> 2, edge >> 2);
    const int bs = vertical ? q.bs_v : q.bs_h;
    if (bs == 0) return;
    const int qp_p = vertical ? qp_of(P, cl, edge - 1, mid) : qp_of(P, cl, mid, edge - 1);
    const int qp_q = q.qp_y;
    const int avg = (qp_p + qp_q + 1) >> 1;
    const int sh = P.bd - 8;
    int bo, to;
    slice_offsets(P, vertical ? edge : mid, vertical ? mid : edge, &bo, &to);
    const int beta = c_beta[clamp3i(avg + 2 * bo, 0, 51)] << sh;
    const int tc = c_tc[clamp3i(avg + 2 * (bs - 1) + 2 * to, 0, 53)] << sh;
    if (tc == 0) return;
    const auto L = lines_of(pl, vertical, edge, scan);
    // deblock.rs:216-238 luma_decision (lines 0 and 3)
    int dp[2], dq[2], far[2], near_[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int l = 3 * k;
        const int p3 = L.ld(l, -4), p2 = L.ld(l, -3), p1 = L.ld(l, -2), p0 = L.ld(l, -1);
        const int q0 = L.ld(l, 0), q1 = L.ld(l, 1), q2 = L.ld(l, 2), q3 = L.ld(l, 3);
        dp[k] = abs(p2 - 2 * p1 + p0);
        dq[k] = abs(q2 - 2 * q1 + q0);
        far[k] = abs(p3 - p0) + abs(q0 - q3);
        near_[k] = abs(p0 - q0);
    }
    if (dp[0] + dp[1] + dq[0] + dq[1] >= beta) return;
    auto dsam = [&](int k) {
        return 2 * (dp[k] + dq[k]) < (beta >> 2) && far[k] < (beta >> 3) && near_[k] < ((5 * tc + 1) >> 1);
    };
    const bool strong = dsam(0) && dsam(1);
    const int side_thr = (beta + (beta >> 1)) >> 3;
    const bool do_p1 = dp[0] + dp[1] < side_thr, do_q1 = dq[0] + dq[1] < side_thr;
    const int maxv = (1 << P.bd) - 1;
    // exemption of the P / Q side (whole 4x4 cells)
    const bool ex_p = any_exempt && (vertical ? exempt_of(cl, edge - 1, mid) : exempt_of(cl, mid, edge - 1));
    const bool ex_q = (q.flags & HPVCD_CELL_EXEMPT) != 0;
    const int tc2 = tc >> 1;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const int p0 = L.ld(l, -1), p1 = L.ld(l, -2), p2 = L.ld(l, -3);
        const int q0 = L.ld(l, 0), q1 = L.ld(l, 1), q2 = L.ld(l, 2);
        if (strong) {  // deblock.rs:605-616
            const int p3 = L.ld(l, -4), q3 = L.ld(l, 3);
            auto c = [&](int o, int x) { return clamp3i(clamp3i(x, o - 2 * tc, o + 2 * tc), 0, maxv); };
            if (!ex_p) {
                L.st(l, -1, c(p0, (p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3));
                L.st(l, -2, c(p1, (p2 + p1 + p0 + q0 + 2) >> 2));
                L.st(l, -3, c(p2, (2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3));
            }
            if (!ex_q) {
                L.st(l, 0, c(q0, (p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3));
                L.st(l, 1, c(q1, (p0 + q0 + q1 + q2 + 2) >> 2));
                L.st(l, 2, c(q2, (p0 + q0 + q1 + 3 * q2 + 2 * q3 + 4) >> 3));
            }
        } else {  // deblock.rs:617-631
            const int delta0 = (9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4;
            if (abs(delta0) < tc * 10) {
                const int delta = clamp3i(delta0, -tc, tc);
                if (!ex_p) {
                    L.st(l, -1, clamp3i(p0 + delta, 0, maxv));
                    if (do_p1) {
                        const int dp1 = clamp3i((((p2 + p0 + 1) >> 1) - p1 + delta) >> 1, -tc2, tc2);
                        L.st(l, -2, clamp3i(p1 + dp1, 0, maxv));
                    }
                }
                if (!ex_q) {
                    L.st(l, 0, clamp3i(q0 - delta, 0, maxv));
                    if (do_q1) {
                        const int dq1 = clamp3i((((q2 + q0 + 1) >> 1) - q1 - delta) >> 1, -tc2, tc2);
                        L.st(l, 1, clamp3i(q1 + dq1, 0, maxv));
                    }
                }
            }
        }
    }
}

// Chroma segment (decode.rs:2036-2137): 4 chroma lines, both Cb and Cr.
template <class Pl, class Cl>
__device__ void chroma_segment(const DevPic& P, bool vertical, int edge, int scan, const Pl& cb, const Pl& cr,
                               const Cl& cl, bool any_exempt = true) {
    const int mid = scan + 1;
    const int lex = vertical ? edge * P.sub_w : mid * P.sub_w;
    const int ley = vertical ? mid * P.sub_h : edge * P.sub_h;
    if (lex >= P.w || ley >= P.h) return;
    const hpvcd_cell q = cl.at(lex >> 2, ley >> 2);
    const int bs = vertical ? q.bs_v : q.bs_h;
    if (bs < 2) return;
    const int lqx = min(lex, P.w - 1), lqy = min(ley, P.h - 1);
    int ppx, ppy;
    if (vertical) {
        ppx = min(max(lex - 1, 0), P.w - 1);
        ppy = min(ley, P.h - 1);
    } else {
        ppx = min(lex, P.w - 1);
        ppy = min(max(ley - 1, 0), P.h - 1);
    }
    const int avg = (qp_of(P, cl, ppx, ppy) + qp_of(P, cl, lqx, lqy) + 1) >> 1;
    int bo, to;
    slice_offsets(P, lqx, lqy, &bo, &to);
    (void)bo;
    const int sh = P.bd_c - 8;
    const int maxv = (1 << P.bd_c) - 1;
    const int scan_max = vertical ? P.ch : P.cw;
    for (int plane = 0; plane < 2; ++plane) {
        const int off = plane == 0 ? P.pps_cb_qp_offset : P.pps_cr_qp_offset;
        const int qc = qpc_map(avg + off, P.idc, P.bd_c);
        const int tc = c_tc[clamp3i(qc + 2 + 2 * to, 0, 53)] << sh;
        if (tc == 0) continue;
        const auto L = lines_of(plane == 0 ? cb : cr, vertical, edge, scan);
        for (int s = scan; s < scan + 4; ++s) {
            if (s >= scan_max) continue;
            const int l = s - scan;
            // p1, p0 | q0, q1 across the edge (taps -2, -1 | 0, 1 of line l)
            const int p0 = L.ld(l, -1), p1 = L.ld(l, -2), q0 = L.ld(l, 0), q1 = L.ld(l, 1);
            const int delta = clamp3i((((q0 - p0) * 4 + p1 - q1 + 4) >> 3), -tc, tc);
            if (delta != 0) {  // exemption by the luma positions of p0 / q0
                const int xp0 = vertical ? edge - 1 : s, yp0 = vertical ? s : edge - 1;
                const int xq0 = vertical ? edge : s, yq0 = vertical ? s : edge;
                if (!(any_exempt && exempt_of(cl, xp0 * P.sub_w, yp0 * P.sub_h))) L.st(l, -1, clamp3i(p0 + delta, 0, maxv));
                if (!(any_exempt && exempt_of(cl, xq0 * P.sub_w, yq0 * P.sub_h))) L.st(l, 0, clamp3i(q0 - delta, 0, maxv));
            }
        }
    }
}

// blockIdx.y = picture, blockIdx.z = 0 luma / 1 chroma.
__global__ void k_deblock(const DevPic* __restrict__ pics, int vertical) {
    const DevPic& P = pics[blockIdx.y];
    if (!(P.flags & HPVCD_PIC_DEBLOCK) || !P.cells) return;
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.z == 0) {
        const int edge_max = vertical ? P.w : P.h, scan_max = vertical ? P.h : P.w;
        const int n_edges = edge_max >= 12 ? (edge_max - 4) / 8 : 0;  // edges 8, 16, ... <= max - 4
        const int n_segs = scan_max / 4;
        if (id >= n_edges * n_segs) return;
        // vertical edges: neighbouring threads take neighbouring edges of the
        // same rows; horizontal edges: neighbouring segments of the same edge
        const int e = vertical ? id % n_edges : id / n_segs;
        const int s = vertical ? id / n_edges : id % n_segs;
        luma_segment(P, vertical != 0, 8 * (e + 1), 4 * s, GPlane{P.rec[0], P.w, P.bps}, GCells{P.cells, P.gw});
    } else {
        if (P.idc == 0) return;
        const int edge_max = vertical ? P.cw : P.ch, scan_max = vertical ? P.ch : P.cw;
        const int n_edges = edge_max >= 10 ? (edge_max - 2) / 8 : 0;  // edges 8, 16, ... <= max - 2
        const int n_segs = scan_max / 4;  // decode.rs:2042 `while scan + 4 <= scan_max`
        if (id >= n_edges * n_segs) return;
        const int e = vertical ? id % n_edges : id / n_segs;
        const int s = vertical ? id / n_edges : id % n_segs;
        chroma_segment(P, vertical != 0, 8 * (e + 1), 4 * s, GPlane{P.rec[1], P.cw, P.bps},
                       GPlane{P.rec[2], P.cw, P.bps}, GCells{P.cells, P.gw});
    }
}

// Four horizontally adjacent samples of a plane (x multiple of 4; plane
// widths are multiples of 4 samples, so the access is aligned and in bounds).
__device__ __forceinline__ void load4(const void* plane, int bps, size_t idx, int v[4]) {
    if (bps == 1) {
        const uint32_t w = *(const uint32_t*)((const uint8_t*)plane + idx);
#pragma unroll
        for (int i = 0; i < 4; ++i) v[i] = (w >> (8 * i)) & 0xff;
    } else {
        const uint2 w = *(const uint2*)((const uint16_t*)plane + idx);
        v[0] = w.x & 0xffff; v[1] = w.x >> 16; v[2] = w.y & 0xffff; v[3] = w.y >> 16;
    }
}
__device__ __forceinline__ void store4(void* plane, int bps, size_t idx, const int v[4]) {
    if (bps == 1)
        *(uint32_t*)((uint8_t*)plane + idx) =
            (uint32_t)v[0] | ((uint32_t)v[1] << 8) | ((uint32_t)v[2] << 16) | ((uint32_t)v[3] << 24);
    else
        *(uint2*)((uint16_t*)plane + idx) =
            make_uint2((uint32_t)v[0] | ((uint32_t)v[1] << 16), (uint32_t)v[2] | ((uint32_t)v[3] << 16));
}

// SAO: one thread per 4 horizontally adjacent samples (they share one CTB:
// CTB widths are multiples of 8 samples).  blockIdx.y = picture,
// blockIdx.z = component.  Rows y-1, y, y+1 are read over x-1 .. x+4 once.
// kGated: some picture of the launch has SAO boundaries it may not cross
// (slices / tiles); the other instantiation carries no region test.
template <bool kGated>
__global__ void k_sao(const DevPic* __restrict__ pics) {
    const DevPic& P = pics[blockIdx.y];
    const int c = blockIdx.z;
    if (P.rec[0] == P.fin[0]) return;  // no SAO for this picture
    if (c > 0 && P.idc == 0) return;
    const int pw = c ? P.cw : P.w, ph = c ? P.ch : P.h;
    const int qw = pw >> 2;
    // grid-stride over the quads of this picture and component
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < qw * ph; id += gridDim.x * blockDim.x) {
        const int x0 = (id % qw) * 4, y = id / qw;
        const void* src = P.rec[c];
        void* dst = P.fin[c];
        const int bps = P.bps;
        const size_t row = (size_t)y * pw;
        int s[4];
        load4(src, bps, row + x0, s);
        int out[4] = {s[0], s[1], s[2], s[3]};
        const bool on = c == 0 ? (P.flags & HPVCD_PIC_SAO_LUMA) != 0 : (P.flags & HPVCD_PIC_SAO_CHROMA) != 0;
        const int sw = c ? P.sub_w : 1, sh = c ? P.sub_h : 1;
        if (on && P.sao) {
            const int rx = (x0 * sw) >> P.log2_ctb, ry = (y * sh) >> P.log2_ctb;
            const hpvcd_sao_comp sc = P.sao[(size_t)ry * P.ctb_cols + rx].comp[c];
            const int bd = c ? P.bd_c : P.bd;
            const int mx = (1 << bd) - 1;
            if (sc.type_idx == 1) {  // sao.rs:205-233
    #pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const uint8_t rel = (uint8_t)((uint8_t)(s[i] >> (bd - 5)) - sc.band_pos);
                    if (rel < 4) out[i] = clamp3i(s[i] + sc.offsets[rel], 0, mx);
                }
            } else if (sc.type_idx == 2) {  // sao.rs:266-330
                int dx, dy;
                switch (sc.eo_class) {
                    case 0: dx = 1; dy = 0; break;
                    case 1: dx = 0; dy = 1; break;
                    case 2: dx = 1; dy = 1; break;
                    default: dx = 1; dy = -1; break;
                }
                // window w[r][i] = sample (x0 - 1 + i, y - 1 + r), i = 0..5
                int w[3][6];
    #pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const int yy = y - 1 + r;
                    const bool in_row = yy >= 0 && yy < ph;
                    if (r == 1) {
    #pragma unroll
                        for (int i = 0; i < 4; ++i) w[1][i + 1] = s[i];
                    } else if (in_row) {
                        int t[4];
                        load4(src, bps, (size_t)yy * pw + x0, t);
    #pragma unroll
                        for (int i = 0; i < 4; ++i) w[r][i + 1] = t[i];
                    } else {
    #pragma unroll
                        for (int i = 0; i < 4; ++i) w[r][i + 1] = 0;
                    }
                    w[r][0] = in_row && x0 > 0 ? load_sample(src, bps, (size_t)yy * pw + x0 - 1) : 0;
                    w[r][5] = in_row && x0 + 4 < pw ? load_sample(src, bps, (size_t)yy * pw + x0 + 4) : 0;
                }
                // slice / tile boundaries SAO may not cross (sao.rs:380-414):
                // bits of the CTB regions that must agree
                const uint32_t rmask = P.ctb_region ? (((P.flags & HPVCD_PIC_SAO_NO_ACROSS_SLICES) ? 0xff00u : 0u) |
                                                       ((P.flags & HPVCD_PIC_SAO_NO_ACROSS_TILES) ? 0x00ffu : 0u))
                                                    : 0u;
                auto region_ok = [&](int ax, int ay, int bx, int by) {
                    const int s = P.log2_ctb;
                    const uint32_t ra = P.ctb_region[(size_t)((ay * sh) >> s) * P.ctb_cols + ((ax * sw) >> s)];
                    const uint32_t rb = P.ctb_region[(size_t)((by * sh) >> s) * P.ctb_cols + ((bx * sw) >> s)];
                    return ((ra ^ rb) & rmask) == 0u;
                };
                // the sample loop, compiled with and without the region test
                auto eo_quad = [&](auto gated) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int x = x0 + i;
                        const int x1 = x + dx, y1 = y + dy, x2 = x - dx, y2 = y - dy;
                        bool ok = x1 >= 0 && y1 >= 0 && x1 < pw && y1 < ph && x2 >= 0 && y2 >= 0 && x2 < pw && y2 < ph;
                        if constexpr (decltype(gated)::value) ok = ok && region_ok(x, y, x1, y1) && region_ok(x, y, x2, y2);
                        if (ok) {
                            // (x + dx, y + dy) and (x - dx, y - dy) with constant window indexes
                            int n1, n2;
                            switch (sc.eo_class) {
                                case 0: n1 = w[1][i + 2]; n2 = w[1][i]; break;
                                case 1: n1 = w[2][i + 1]; n2 = w[0][i + 1]; break;
                                case 2: n1 = w[2][i + 2]; n2 = w[0][i]; break;
                                default: n1 = w[0][i + 2]; n2 = w[2][i]; break;
                            }
                            const int e = ((s[i] > n1) - (s[i] < n1)) + ((s[i] > n2) - (s[i] < n2)) + 2;
                            int o = 0;
                            if (e == 0) o = sc.offsets[0];
                            else if (e == 1) o = sc.offsets[1];
                            else if (e == 3) o = sc.offsets[2];
                            else if (e == 4) o = sc.offsets[3];
                            if (o) out[i] = clamp3i(s[i] + o, 0, mx);
                        }
                    }
                };
                if constexpr (kGated) {
                    if (rmask)
                        eo_quad(std::true_type{});
                    else
                        eo_quad(std::false_type{});
                } else {
                    (void)rmask;
                    eo_quad(std::false_type{});
                }
            }
            if (P.cells) {  // exempt cells keep the deblocked samples
    #pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (exempt_at(P, (x0 + i) * sw, y * sh)) out[i] = s[i];
            }
        }
        store4(dst, bps, row + x0, out);
    }
}

// Q13 YCbCr -> RGB8 onto the canvas, four pixels per thread.  blockIdx.y =
// picture.  Every product and sum stays below 2^31 for bit depths up to 12
// (|k_y (Y - black)| < 2^26, |coefficient x (C - neutral)| < 2^26), so the
// 32-bit arithmetic equals the reference's 64-bit one.
struct RgbCoef {
    int k_y, k_uv, cr_to_r, cb_to_g, cr_to_g, cb_to_b, y_black, c_black, neutral, cmax, sh, matrix, full;
};

__device__ __forceinline__ RgbCoef rgb_coef(const DevPic& P) {
    RgbCoef k;
    const int Q13 = 13, ONE = 1 << 13, ROUND = 1 << 12;
    const int bd = P.bd;
    const int scale = 1 << (bd - 8);
    k.full = P.full_range != 0;
    k.matrix = P.matrix;
    k.k_y = k.full ? ONE : 9539;
    k.k_uv = k.full ? ONE : 9326;
    int cr_r0, cb_g0, cr_g0, cb_b0;
    switch (P.matrix) {
        case HPVCD_MATRIX_BT470BG:
        case HPVCD_MATRIX_SMPTE170M: cr_r0 = 11485; cb_g0 = -2819; cr_g0 = -5851; cb_b0 = 14516; break;
        case HPVCD_MATRIX_BT2020NCL: cr_r0 = 12080; cb_g0 = -1348; cr_g0 = -4681; cb_b0 = 17546; break;
        case HPVCD_MATRIX_IDENTITY: cr_r0 = cb_g0 = cr_g0 = cb_b0 = 0; break;
        default: cr_r0 = 12901; cb_g0 = -1534; cr_g0 = -3835; cb_b0 = 15201; break;
    }
    k.cr_to_r = (cr_r0 * k.k_uv + ROUND) >> Q13;
    k.cb_to_g = (cb_g0 * k.k_uv + ROUND) >> Q13;
    k.cr_to_g = (cr_g0 * k.k_uv + ROUND) >> Q13;
    k.cb_to_b = (cb_b0 * k.k_uv + ROUND) >> Q13;
    k.cmax = (1 << bd) - 1;
    k.y_black = k.full ? 0 : 16 * scale;
    k.c_black = k.y_black;
    k.neutral = 128 * scale;
    k.sh = bd - 8;
    return k;
}

__device__ __forceinline__ uint32_t rgb_px(const RgbCoef& k, int idc, int luma, int cb, int cr) {
    const int Q13 = 13, ROUND = 1 << 12;
    int r, g, b;
    if (idc == 0) {
        r = g = b = (k.k_y * (luma - k.y_black) + ROUND) >> Q13;
    } else if (k.matrix == HPVCD_MATRIX_IDENTITY) {
        if (k.full) {
            r = cr; g = luma; b = cb;
        } else {
            r = (k.k_uv * (cr - k.c_black) + ROUND) >> Q13;
            g = (k.k_y * (luma - k.y_black) + ROUND) >> Q13;
            b = (k.k_uv * (cb - k.c_black) + ROUND) >> Q13;
        }
    } else if (k.matrix == HPVCD_MATRIX_YCGCO) {
        const int cg = cb - k.neutral, co = cr - k.neutral, t = luma - cg;
        r = t + co; g = luma + cg; b = t - co;
    } else {
        const int yv = k.k_y * (luma - k.y_black), cbc = cb - k.neutral, crc = cr - k.neutral;
        r = (yv + k.cr_to_r * crc + ROUND) >> Q13;
        g = (yv + k.cb_to_g * cbc + k.cr_to_g * crc + ROUND) >> Q13;
        b = (yv + k.cb_to_b * cbc + ROUND) >> Q13;
    }
    r = clamp3i(r, 0, k.cmax) >> k.sh;
    g = clamp3i(g, 0, k.cmax) >> k.sh;
    b = clamp3i(b, 0, k.cmax) >> k.sh;
    return (uint32_t)r | ((uint32_t)g << 8) | ((uint32_t)b << 16);
}

// Index in the oriented W x H image (stored layout) of stored sample (x, y)
// (lib.rs:2065-2110 rotate_luma, :2112-2200 rotate_buf; TRANSPOSE /
// TRANSVERSE keep their place there).
__device__ __forceinline__ size_t oriented_index(int x, int y, int W, int H, int o) {
    switch (o) {
        case HPVCD_ORIENT_FLIP_H: return (size_t)y * W + (W - 1 - x);
        case HPVCD_ORIENT_ROTATE180: return (size_t)(H - 1 - y) * W + (W - 1 - x);
        case HPVCD_ORIENT_FLIP_V: return (size_t)(H - 1 - y) * W + x;
        case HPVCD_ORIENT_ROTATE90: return (size_t)x * H + (H - 1 - y);
        case HPVCD_ORIENT_ROTATE270: return (size_t)(W - 1 - x) * H + y;
        default: return (size_t)y * W + x;
    }
}

__device__ __forceinline__ bool moves_samples(int o) {
    return o == HPVCD_ORIENT_FLIP_H || o == HPVCD_ORIENT_ROTATE180 || o == HPVCD_ORIENT_FLIP_V ||
           o == HPVCD_ORIENT_ROTATE90 || o == HPVCD_ORIENT_ROTATE270;
}

__global__ void k_rgb(const DevPic* __restrict__ pics, uint8_t* __restrict__ out) {
    const DevPic& P = pics[blockIdx.y];
    if (P.matrix == (int)HPVCD_CANVAS_NATIVE) return;  // k_yuv_canvas's picture
    uint8_t* canvas = out + P.canvas_off;
    const int copy_w = min(P.crop_w, max(P.canvas_w - P.dst_x, 0));
    const int copy_h = min(P.crop_h, max(P.canvas_h - P.dst_y, 0));
    const int qw = (copy_w + 3) >> 2;
    const RgbCoef k = rgb_coef(P);
    // grid-stride over the quads of this picture
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < qw * copy_h; id += gridDim.x * blockDim.x) {
        const int x0 = (id % qw) * 4, yy = id / qw;
        const int cnt = min(4, copy_w - x0);
        // crop_w <= width (a multiple of 8) and copy_h <= height: x0 .. x0 + 3
        // and yy are inside the planes
        int luma[4], cb[4] = {0, 0, 0, 0}, cr[4] = {0, 0, 0, 0};
        load4(P.fin[0], P.bps, (size_t)yy * P.w + x0, luma);
        if (P.idc) {
            const int crow = yy / P.sub_h;
            if (P.sub_w == 2) {
                const size_t ci = (size_t)crow * P.cw + (x0 >> 1);  // two chroma samples
                int t = load_sample(P.fin[1], P.bps, ci), u = load_sample(P.fin[1], P.bps, ci + 1);
                cb[0] = cb[1] = t; cb[2] = cb[3] = u;
                t = load_sample(P.fin[2], P.bps, ci);
                u = load_sample(P.fin[2], P.bps, ci + 1);
                cr[0] = cr[1] = t; cr[2] = cr[3] = u;
            } else {
                load4(P.fin[1], P.bps, (size_t)crow * P.cw + x0, cb);
                load4(P.fin[2], P.bps, (size_t)crow * P.cw + x0, cr);
            }
        }
        uint32_t px[4];
    #pragma unroll
        for (int i = 0; i < 4; ++i) px[i] = rgb_px(k, P.idc, luma[i], cb[i], cr[i]);
        if (moves_samples(P.orientation)) {  // each pixel to its oriented place
            for (int i = 0; i < cnt; ++i) {
                uint8_t* q = canvas + oriented_index(P.dst_x + x0 + i, P.dst_y + yy, P.canvas_w, P.canvas_h,
                                                     P.orientation) * 3;
                q[0] = (uint8_t)px[i];
                q[1] = (uint8_t)(px[i] >> 8);
                q[2] = (uint8_t)(px[i] >> 16);
            }
            continue;
        }
        uint8_t* o = canvas + ((size_t)(P.dst_y + yy) * P.canvas_w + P.dst_x + x0) * 3;
        if (cnt == 4 && ((uintptr_t)o & 3) == 0) {
            uint32_t* o32 = (uint32_t*)o;
            o32[0] = px[0] | (px[1] << 24);
            o32[1] = (px[1] >> 8) | (px[2] << 16);
            o32[2] = (px[2] >> 16) | (px[3] << 8);
        } else {
            for (int i = 0; i < cnt; ++i) {
                o[3 * i] = (uint8_t)px[i];
                o[3 * i + 1] = (uint8_t)(px[i] >> 8);
                o[3 * i + 2] = (uint8_t)(px[i] >> 16);
            }
        }
    }
}

// Native YCbCr canvas (lib.rs:871-991 stitch_native_yuv_band): component
// blockIdx.z of picture blockIdx.y copied onto its canvas plane at (dst_x,
// dst_y) / subsampling, rows and columns past the picture repeating its last
// one, four samples per thread.  The canvas holds Y, then Cb, then Cr, in
// the picture's sample size.
__global__ void k_yuv_canvas(const DevPic* __restrict__ pics, uint8_t* __restrict__ out) {
    const DevPic& P = pics[blockIdx.y];
    const int c = blockIdx.z;
    if (P.matrix != (int)HPVCD_CANVAS_NATIVE) return;  // k_rgb's picture
    if (c > 0 && P.idc == 0) return;
    const int sw = c ? P.sub_w : 1, sh = c ? P.sub_h : 1;
    const int CW = (P.canvas_w + sw - 1) / sw, CH = (P.canvas_h + sh - 1) / sh;
    const int dx = P.dst_x / sw, dy = P.dst_y / sh;
    const int copy_w = min((P.crop_w + sw - 1) / sw, max(CW - dx, 0));
    const int copy_h = min((P.crop_h + sh - 1) / sh, max(CH - dy, 0));
    const int pw = c ? P.cw : P.w, ph = c ? P.ch : P.h;
    const size_t luma_bytes = (size_t)P.canvas_w * P.canvas_h * P.bps;
    const size_t chroma_bytes = (size_t)CW * CH * P.bps;
    uint8_t* plane = out + P.canvas_off + (c == 0 ? 0 : luma_bytes + (c - 1) * chroma_bytes);
    const int qw = (copy_w + 3) >> 2;
    const int o = P.orientation;
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < qw * copy_h; id += gridDim.x * blockDim.x) {
        const int x0 = (id % qw) * 4, y = id / qw;
        const size_t srow = (size_t)min(y, ph - 1) * pw;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int x = x0 + i;
            if (x < copy_w)
                store_sample(plane, P.bps, oriented_index(dx + x, dy + y, CW, CH, o),
                             load_sample(P.fin[c], P.bps, srow + min(x, pw - 1)));
        }
    }
}

// ===========================================================================
// k_filter_tile -- deblocking, SAO and the output of one 64 x 64 luma tile
// (and its chroma) per CTA, in shared memory.
//
// The tile is staged with 8 columns and 4 rows of halo on every side.  The
// vertical-edge pass runs over every 4-line segment of the staged rows whose
// edge lies in [X, X + 64], the horizontal-edge pass over every 4-column
// segment of the staged columns X - 4 .. X + 67 whose edge lies in [Y, Y + 64]:
// each segment reads and writes only samples of its own lines within 4 of
// its edge, so the staged samples the SAO of the tile reads (one ring around
// it) get exactly the values of the reference's whole-picture vertical pass
// followed by its horizontal pass (decode.rs:1774-2146).  SAO then reads
// those deblocked samples (the reference's snapshot, decode.rs:2258-2493) and
// its results replace them in place only after every thread has read its
// neighbours.  Finally the tile's final samples go to the picture's final
// planes (unless the caller asked for its canvas only) and, for an RGB8
// canvas, are converted and stored at their canvas position.  The kernel
// reads `rec` and writes `fin`, which are always different planes.
// ===========================================================================
constexpr int kTile = 64;
constexpr int kTileThreads = 256;

// Region of one component: the tile (tw x th samples at (tx, ty)) with 8
// columns and 4 rows of halo; row length tw + 16 (a multiple of 8 entries).
struct TileComp {
    int tx, ty, tw, th, pw, ph;
    SPlane sp;
    __device__ int rw() const { return tw + 16; }
    __device__ int rh() const { return th + 8; }
};

__host__ __device__ inline size_t tile_comp_entries(int tw, int th) { return (size_t)(tw + 16) * (th + 8); }
// Cells staged per tile: luma columns X - 16 .. X + 79 and rows Y - 8 ..
// Y + 71 (every cell a luma or chroma segment of the tile looks up), and the
// SAO parameters of the (up to 4 x 4) CTBs covering the tile.
constexpr int kTileCellsW = 24, kTileCellsH = 20, kTileSaoCtbs = 16;
// Shared memory of a k_filter_tile CTA for the chroma-format class cfmt
// (0 4:2:0 / 4:0:0, 1 4:4:4, 2 4:2:2): samples, then cells, then SAO.
__host__ __device__ inline size_t tile_sample_bytes(int cfmt) {
    const int tw = cfmt == 1 ? 64 : 32, th = cfmt == 0 ? 32 : 64;
    return (tile_comp_entries(64, 64) + 2 * tile_comp_entries(tw, th)) * sizeof(uint16_t);
}
// The tile's final samples (no halo), component after component.
__host__ __device__ inline size_t tile_out_bytes(int cfmt) {
    const int tw = cfmt == 1 ? 64 : 32, th = cfmt == 0 ? 32 : 64;
    return (size_t)(64 * 64 + 2 * tw * th) * sizeof(uint16_t);
}
__host__ __device__ inline size_t tile_smem_bytes(int cfmt) {
    return tile_sample_bytes(cfmt) + tile_out_bytes(cfmt) + kTileCellsW * kTileCellsH * sizeof(hpvcd_cell) +
           kTileSaoCtbs * sizeof(hpvcd_sao_ctb);
}

// SAO parameters of the CTBs covering a tile, staged in shared memory.
struct SSao {
    const hpvcd_sao_ctb* s;
    int cx0, cy0, n;  // CTBs [cx0, cx0 + n) x [cy0, cy0 + n)
    __device__ hpvcd_sao_comp at(int ctbx, int ctby, int c) const { return s[(ctby - cy0) * n + (ctbx - cx0)].comp[c]; }
};

// SAO of sample (x, y) of component c, s0 its deblocked value (sao.rs:179-330,
// the driver decode.rs:2258-2493): band offset in place, edge offset from
// the deblocked neighbours, picture-border samples and exempt cells
// unchanged; rmask: bits of the CTB regions (slice << 8 | tile) that must
// agree across an edge-offset neighbour (0: no restriction).
template <bool kGated, class Pl, class Cl>
__device__ __forceinline__ int sao_sample(const DevPic& P, int c, int x, int y, int s0, const Pl& src, const Cl& cl,
                                          const SSao& sao, uint32_t rmask) {
    const int sw = c ? P.sub_w : 1, sh = c ? P.sub_h : 1;
    if (P.cells && exempt_of(cl, x * sw, y * sh)) return s0;  // exempt cells keep the deblocked sample
    const int pw = c ? P.cw : P.w, ph = c ? P.ch : P.h;
    const hpvcd_sao_comp sc = sao.at((x * sw) >> P.log2_ctb, (y * sh) >> P.log2_ctb, c);
    const int bd = c ? P.bd_c : P.bd;
    const int mx = (1 << bd) - 1;
    if (sc.type_idx == 1) {  // sao.rs:205-233
        const uint8_t rel = (uint8_t)((uint8_t)(s0 >> (bd - 5)) - sc.band_pos);
        return rel < 4 ? clamp3i(s0 + sc.offsets[rel], 0, mx) : s0;
    }
    if (sc.type_idx != 2) return s0;
    int dx, dy;  // sao.rs:266-330
    switch (sc.eo_class) {
        case 0: dx = 1; dy = 0; break;
        case 1: dx = 0; dy = 1; break;
        case 2: dx = 1; dy = 1; break;
        default: dx = 1; dy = -1; break;
    }
    const int x1 = x + dx, y1 = y + dy, x2 = x - dx, y2 = y - dy;
    if (x1 < 0 || y1 < 0 || x1 >= pw || y1 >= ph || x2 < 0 || y2 < 0 || x2 >= pw || y2 >= ph) return s0;
    if (kGated && rmask) {  // slice / tile boundaries SAO may not cross (sao.rs:380-414)
        auto region = [&](int ax, int ay) {
            return (uint32_t)P.ctb_region[(size_t)((ay * sh) >> P.log2_ctb) * P.ctb_cols + ((ax * sw) >> P.log2_ctb)];
        };
        const uint32_t r0 = region(x, y);
        if (((r0 ^ region(x1, y1)) & rmask) || ((r0 ^ region(x2, y2)) & rmask)) return s0;
    }
    const int n1 = src.ld(x1, y1), n2 = src.ld(x2, y2);
    const int e = ((s0 > n1) - (s0 < n1)) + ((s0 > n2) - (s0 < n2)) + 2;
    const int o = e == 0 ? sc.offsets[0] : (e == 1 ? sc.offsets[1] : (e == 3 ? sc.offsets[2] : (e == 4 ? sc.offsets[3] : 0)));
    return o ? clamp3i(s0 + o, 0, mx) : s0;
}

template <bool kGated>
__device__ __noinline__ int sao_sample_slow(const DevPic& P, int c, int x, int y, int s0, const SPlane src,
                                            const SCells cl, const SSao sao, uint32_t rmask) {
    return sao_sample<kGated>(P, c, x, y, s0, src, cl, sao, rmask);
}

// SAO of four horizontally adjacent samples (x0 .. x0 + 3, x0 a multiple of
// 4, so one CTB) of component c from the staged deblocked region: the 3 x 6
// neighbourhood is read once (one 8-byte load per row), the CTB's parameters
// once; out[] receives the results (sao.rs:179-330: band offset, edge offset
// with picture-border samples unchanged).  Exempt cells and slice / tile
// boundaries, when the tile has any, go through sao_sample.
template <bool kGated, class Cl>
__device__ __forceinline__ void sao_quad(const DevPic& P, int c, const TileComp& k, int x0, int y, const SSao& sao,
                                         const Cl& cl, bool slow, uint32_t rmask, int out[4]) {
    const int sw = c ? P.sub_w : 1, sh = c ? P.sub_h : 1;
    const int rw = k.rw();
    const uint16_t* row = k.sp.s + (y - k.sp.y0) * rw + (x0 - k.sp.x0);
    int w[3][6];  // w[r][j] = sample (x0 - 1 + j, y - 1 + r)
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const uint16_t* q = row + (r - 1) * rw;
        const uint2 v = *(const uint2*)q;
        w[r][0] = q[-1];
        w[r][1] = v.x & 0xffff; w[r][2] = v.x >> 16; w[r][3] = v.y & 0xffff; w[r][4] = v.y >> 16;
        w[r][5] = q[4];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) out[i] = w[1][i + 1];
    if (slow) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (x0 + i < k.pw) out[i] = sao_sample_slow<kGated>(P, c, x0 + i, y, w[1][i + 1], k.sp, cl, sao, rmask);
        return;
    }
    const hpvcd_sao_comp sc = sao.at((x0 * sw) >> P.log2_ctb, (y * sh) >> P.log2_ctb, c);
    const int bd = c ? P.bd_c : P.bd;
    const int mx = (1 << bd) - 1;
    if (sc.type_idx == 1) {  // sao.rs:205-233
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint8_t rel = (uint8_t)((uint8_t)(out[i] >> (bd - 5)) - sc.band_pos);
            // offset of band rel (a select, not an index: the parameters stay in registers)
            const int o = rel == 0 ? sc.offsets[0] : (rel == 1 ? sc.offsets[1] : (rel == 2 ? sc.offsets[2] : sc.offsets[3]));
            if (rel < 4) out[i] = clamp3i(out[i] + o, 0, mx);
        }
    } else if (sc.type_idx == 2) {  // sao.rs:266-330
        const int dx = sc.eo_class == 1 ? 0 : 1;
        const int dy = sc.eo_class == 0 ? 0 : (sc.eo_class == 3 ? -1 : 1);
        const bool rows_ok = y - dy >= 0 && y + dy >= 0 && y - dy < k.ph && y + dy < k.ph;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int x = x0 + i;
            if (!rows_ok || x - dx < 0 || x + dx >= k.pw) continue;  // a neighbour outside the picture
            int n1, n2;  // (x + dx, y + dy) and (x - dx, y - dy)
            switch (sc.eo_class) {
                case 0: n1 = w[1][i + 2]; n2 = w[1][i]; break;
                case 1: n1 = w[2][i + 1]; n2 = w[0][i + 1]; break;
                case 2: n1 = w[2][i + 2]; n2 = w[0][i]; break;
                default: n1 = w[0][i + 2]; n2 = w[2][i]; break;
            }
            const int s0 = out[i];
            const int e = ((s0 > n1) - (s0 < n1)) + ((s0 > n2) - (s0 < n2)) + 2;
            const int o = e == 0 ? sc.offsets[0] : (e == 1 ? sc.offsets[1] : (e == 3 ? sc.offsets[2] : (e == 4 ? sc.offsets[3] : 0)));
            if (o) out[i] = clamp3i(s0 + o, 0, mx);
        }
    }
}

// SAO of one tile component whose samples all lie in one CTB (CTB 64),
// without exempt cells or region limits: the CTB's parameters, read once,
// hold for every quad.  kSel: 0..3 edge offset of that class, 4 band
// offset, 5 off (a copy).  Same arithmetic as sao_quad (sao.rs:179-330).
template <int kSel>
__device__ __forceinline__ void sao_fixed(const TileComp& k, uint16_t* to, const hpvcd_sao_comp sc, int bd, int tid) {
    const int qsh = k.tw == 64 ? 4 : 3;  // quads per row: 16 or 8
    const int nq = k.th << qsh, rw = k.rw();
    const int mx = (1 << bd) - 1;
    const int o0 = sc.offsets[0], o1 = sc.offsets[1], o2 = sc.offsets[2], o3 = sc.offsets[3];
    for (int i = tid; i < nq; i += kTileThreads) {
        const int xq = 4 * (i & ((1 << qsh) - 1)), yq = i >> qsh;
        const int x0 = k.tx + xq, y = k.ty + yq;
        if (x0 >= k.pw || y >= k.ph) continue;
        const uint16_t* row = k.sp.s + (yq + 4) * rw + (xq + 8);  // sample (x0, y) of the staged region
        const uint2 c2 = *(const uint2*)row;
        int out[4] = {(int)(c2.x & 0xffff), (int)(c2.x >> 16), (int)(c2.y & 0xffff), (int)(c2.y >> 16)};
        if (kSel == 4) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint8_t rel = (uint8_t)((uint8_t)(out[u] >> (bd - 5)) - sc.band_pos);
                const int o = rel == 0 ? o0 : (rel == 1 ? o1 : (rel == 2 ? o2 : o3));
                if (rel < 4) out[u] = clamp3i(out[u] + o, 0, mx);
            }
        } else if (kSel < 4) {
            constexpr int dx = kSel == 1 ? 0 : 1;
            constexpr int dy = kSel == 0 ? 0 : (kSel == 3 ? -1 : 1);
            // n1 = (x + dx, y + dy), n2 = (x - dx, y - dy)
            int n1[4], n2[4];
            auto six = [&](const uint16_t* q, int w[6]) {  // samples x0 - 1 .. x0 + 4 of a staged row
                const uint2 v = *(const uint2*)q;
                w[0] = q[-1];
                w[1] = v.x & 0xffff; w[2] = v.x >> 16; w[3] = v.y & 0xffff; w[4] = v.y >> 16;
                w[5] = q[4];
            };
            if (kSel == 1) {
                const uint2 a = *(const uint2*)(row + rw), b = *(const uint2*)(row - rw);
                n1[0] = a.x & 0xffff; n1[1] = a.x >> 16; n1[2] = a.y & 0xffff; n1[3] = a.y >> 16;
                n2[0] = b.x & 0xffff; n2[1] = b.x >> 16; n2[2] = b.y & 0xffff; n2[3] = b.y >> 16;
            } else {
                int wa[6], wb[6];
                six(row + dy * rw, wa);
                if (dy != 0) six(row - dy * rw, wb);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    n1[u] = wa[u + 2];
                    n2[u] = dy != 0 ? wb[u] : wa[u];
                }
            }
            const bool rows_ok = y - dy >= 0 && y + dy >= 0 && y - dy < k.ph && y + dy < k.ph;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int x = x0 + u;
                if (!rows_ok || x - dx < 0 || x + dx >= k.pw) continue;  // a neighbour outside the picture
                const int s0 = out[u];
                const int e = ((s0 > n1[u]) - (s0 < n1[u])) + ((s0 > n2[u]) - (s0 < n2[u])) + 2;
                const int o = e == 0 ? o0 : (e == 1 ? o1 : (e == 3 ? o2 : (e == 4 ? o3 : 0)));
                if (o) out[u] = clamp3i(s0 + o, 0, mx);
            }
        }
        *(uint2*)(to + yq * k.tw + xq) =
            make_uint2((uint32_t)out[0] | ((uint32_t)out[1] << 16), (uint32_t)out[2] | ((uint32_t)out[3] << 16));
    }
}

// Eight horizontally adjacent samples of a plane row at (x, y), as uint16,
// zero outside the plane.  Vector load when the whole group is inside and
// 16-byte aligned.
__device__ __forceinline__ uint4 load8(const void* plane, int bps, int pw, int ph, int x, int y) {
    uint32_t w[4] = {0u, 0u, 0u, 0u};
    if (y < 0 || y >= ph || x + 8 <= 0 || x >= pw) return make_uint4(0u, 0u, 0u, 0u);
    const size_t idx = (size_t)y * pw + x;
    if (x >= 0 && x + 8 <= pw) {
        if (bps == 2 && (idx & 7) == 0) return *(const uint4*)((const uint16_t*)plane + idx);
        if (bps == 1 && (idx & 7) == 0) {
            const uint2 b = *(const uint2*)((const uint8_t*)plane + idx);
            w[0] = (b.x & 0xffu) | ((b.x & 0xff00u) << 8);
            w[1] = ((b.x >> 16) & 0xffu) | ((b.x >> 8) & 0xff0000u);
            w[2] = (b.y & 0xffu) | ((b.y & 0xff00u) << 8);
            w[3] = ((b.y >> 16) & 0xffu) | ((b.y >> 8) & 0xff0000u);
            return make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int xx = x + i;
        const uint32_t v = (xx >= 0 && xx < pw) ? (uint32_t)load_sample(plane, bps, idx + i) : 0u;
        w[i >> 1] |= v << (16 * (i & 1));
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

template <bool kGated>
__global__ void __launch_bounds__(kTileThreads, 3)
k_filter_tile(const DevPic* __restrict__ pics, uint8_t* __restrict__ out, int rgb, int cfmt) {
    extern __shared__ __align__(16) uint16_t tsm[];
    const DevPic& P = pics[blockIdx.y];
    const int tid = threadIdx.x;
    const int tiles_x = (P.w + kTile - 1) / kTile, tiles_y = (P.h + kTile - 1) / kTile;
    const int ncomp = P.idc ? 3 : 1;
    const bool deblock = (P.flags & HPVCD_PIC_DEBLOCK) && P.cells;
    const bool do_rgb = rgb && out && P.matrix != (int)HPVCD_CANVAS_NATIVE;
    const bool sao_on = P.sao && (P.flags & (HPVCD_PIC_SAO_LUMA | HPVCD_PIC_SAO_CHROMA));
    const size_t out_off = tile_sample_bytes(cfmt);
    const size_t cells_off = out_off + tile_out_bytes(cfmt);
    const size_t sao_off = cells_off + kTileCellsW * kTileCellsH * sizeof(hpvcd_cell);
    const uint32_t rmask = (kGated && P.ctb_region) ? (((P.flags & HPVCD_PIC_SAO_NO_ACROSS_SLICES) ? 0xff00u : 0u) |
                                                       ((P.flags & HPVCD_PIC_SAO_NO_ACROSS_TILES) ? 0x00ffu : 0u))
                                                    : 0u;
    for (int t = blockIdx.x; t < tiles_x * tiles_y; t += gridDim.x) {
        const int X = (t % tiles_x) * kTile, Y = (t / tiles_x) * kTile;
        // region of component c (computed where it is used: an array of the
        // three would be indexed by a loop variable and live in local memory)
        auto tcomp = [&](int c) {
            const int sw = c ? P.sub_w : 1, sh = c ? P.sub_h : 1;
            TileComp k;
            k.tx = X / sw; k.ty = Y / sh; k.tw = kTile / sw; k.th = kTile / sh;
            k.pw = c ? P.cw : P.w; k.ph = c ? P.ch : P.h;
            const size_t off = c == 0 ? 0 : tile_comp_entries(64, 64) + (c - 1) * tile_comp_entries(k.tw, k.th);
            k.sp = SPlane{tsm + off, k.tx - 8, k.ty - 4, k.tw + 16};
            return k;
        };
        // the tile's final samples of component c (no halo)
        auto tout_of = [&](int c) {
            const int cw_ = kTile / P.sub_w, ch_ = kTile / P.sub_h;
            return (uint16_t*)((unsigned char*)tsm + out_off) + (c == 0 ? 0 : 64 * 64 + (c - 1) * cw_ * ch_);
        };
        // ---- 1. stage the tile and its halo (8 samples per copy), the cells
        // around it and the SAO parameters of its CTBs ----
        __syncthreads();  // the previous tile's readers are done
        hpvcd_cell* s_cells = (hpvcd_cell*)((unsigned char*)tsm + cells_off);
        const SCells cl{s_cells, (X - 16) >> 2, (Y - 8) >> 2, kTileCellsW, kTileCellsH, P.cells, P.gw};
        bool exempt_here = false;  // an exempt cell among the staged ones
        if (P.cells)
            for (int i = tid; i < kTileCellsW * kTileCellsH; i += kTileThreads) {
                const int gx = cl.gx0 + i % kTileCellsW, gy = cl.gy0 + i / kTileCellsW;
                const hpvcd_cell cv = (gx >= 0 && gy >= 0 && gx < P.gw && gy < P.gh)
                                          ? P.cells[(size_t)gy * P.gw + gx]
                                          : hpvcd_cell{};
                s_cells[i] = cv;
                exempt_here |= (cv.flags & HPVCD_CELL_EXEMPT) != 0;
            }
        hpvcd_sao_ctb* s_sao = (hpvcd_sao_ctb*)((unsigned char*)tsm + sao_off);
        const int nsc = max(1, kTile >> P.log2_ctb);
        const SSao sao{s_sao, X >> P.log2_ctb, Y >> P.log2_ctb, nsc};
        if (sao_on)
            for (int i = tid; i < nsc * nsc; i += kTileThreads) {
                const int cx = sao.cx0 + i % nsc, cy = sao.cy0 + i / nsc;
                if (cx < P.ctb_cols && cy < P.ctb_rows) s_sao[i] = P.sao[(size_t)cy * P.ctb_cols + cx];
            }
        for (int c = 0; c < ncomp; ++c) {
            const TileComp k = tcomp(c);
            const int chunks = k.rw() >> 3;
            for (int i = tid; i < k.rh() * chunks; i += kTileThreads) {
                const int r = i / chunks, q = i - r * chunks;
                *(uint4*)(k.sp.s + r * k.rw() + 8 * q) =
                    load8(P.rec[c], P.bps, k.pw, k.ph, k.sp.x0 + 8 * q, k.sp.y0 + r);
            }
        }
        // the SAO of the tile tests exemption and slice / tile boundaries
        // per sample only when the tile has them
        // exempt cells (tested per segment and per sample only when present)
        const bool any_exempt = __syncthreads_or(exempt_here) != 0;
        const bool sao_slow = any_exempt || (kGated && rmask);
        if (deblock) {
            // ---- 2. vertical edges, then 3. horizontal edges ----
            const TileComp Lc = tcomp(0);
            const TileComp Cb = tcomp(1);
            const SPlane Cr = tcomp(2).sp;
            const int nec_v = Cb.tw / 8 + 1, nsc_v = Cb.rh() / 4;        // chroma V: edges, segments
            const int nec_h = Cb.th / 8 + 1, nsc_h = (Cb.tw + 8) / 4;    // chroma H
            for (int pass = 0; pass < 2; ++pass) {
                const bool vertical = pass == 0;
                const int n_luma = 9 * 18;
                const int n_chroma = P.idc ? (vertical ? nec_v * nsc_v : nec_h * nsc_h) : 0;
                for (int j = tid; j < n_luma + n_chroma; j += kTileThreads) {
                    if (j < n_luma) {
                        const int e = (vertical ? X : Y) + 8 * (j % 9);
                        const int scan = (vertical ? Y - 4 : X - 4) + 4 * (j / 9);
                        const int emax = vertical ? P.w : P.h, smax = vertical ? P.h : P.w;
                        if (e >= 8 && e <= emax - 4 && scan >= 0 && scan + 4 <= smax)
                            luma_segment(P, vertical, e, scan, Lc.sp, cl, any_exempt);
                    } else {
                        const int jj = j - n_luma;
                        const int ne = vertical ? nec_v : nec_h;
                        const int e = (vertical ? Cb.tx : Cb.ty) + 8 * (jj % ne);
                        const int scan = (vertical ? Cb.ty - 4 : Cb.tx - 4) + 4 * (jj / ne);
                        const int emax = vertical ? P.cw : P.ch, smax = vertical ? P.ch : P.cw;
                        if (e >= 8 && e <= emax - 2 && scan >= 0 && scan + 4 <= smax)
                            chroma_segment(P, vertical, e, scan, Cb.sp, Cr, cl, any_exempt);
                    }
                }
                __syncthreads();
            }
        }
        // ---- 4. SAO from the deblocked samples into the tile's output
        // buffer (a copy for components without SAO) ----
        for (int c = 0; c < ncomp; ++c) {
            const TileComp k = tcomp(c);
            uint16_t* const to = tout_of(c);
            const bool on = sao_on && (P.flags & (c == 0 ? HPVCD_PIC_SAO_LUMA : HPVCD_PIC_SAO_CHROMA));
            if (!sao_slow && P.log2_ctb >= 6) {  // one CTB covers the tile component
                hpvcd_sao_comp sc{};
                if (on) sc = sao.at(X >> P.log2_ctb, Y >> P.log2_ctb, c);
                const int bd = c ? P.bd_c : P.bd;
                const int sel = sc.type_idx == 1 ? 4 : (sc.type_idx == 2 ? sc.eo_class : 5);
                switch (sel) {
                    case 0: sao_fixed<0>(k, to, sc, bd, tid); break;
                    case 1: sao_fixed<1>(k, to, sc, bd, tid); break;
                    case 2: sao_fixed<2>(k, to, sc, bd, tid); break;
                    case 3: sao_fixed<3>(k, to, sc, bd, tid); break;
                    case 4: sao_fixed<4>(k, to, sc, bd, tid); break;
                    default: sao_fixed<5>(k, to, sc, bd, tid); break;
                }
                continue;
            }
            const int qw = k.tw >> 2, nq = qw * k.th;
            for (int i = tid; i < nq; i += kTileThreads) {
                const int xq = 4 * (i % qw), yq = i / qw;
                const int x0 = k.tx + xq, y = k.ty + yq;
                if (x0 >= k.pw || y >= k.ph) continue;
                uint2 v;
                if (on) {
                    int r4[4];
                    sao_quad<kGated>(P, c, k, x0, y, sao, cl, sao_slow, rmask, r4);
                    v = make_uint2((uint32_t)r4[0] | ((uint32_t)r4[1] << 16), (uint32_t)r4[2] | ((uint32_t)r4[3] << 16));
                } else {
                    v = *(const uint2*)(k.sp.s + (y - k.sp.y0) * k.rw() + (x0 - k.sp.x0));
                }
                *(uint2*)(to + yq * k.tw + xq) = v;
            }
        }
        __syncthreads();
        // ---- 5. final planes (8 samples per store) ----
        if (P.write_fin) {
            for (int c = 0; c < ncomp; ++c) {
                const TileComp k = tcomp(c);
                const uint16_t* const to = tout_of(c);
                const int rows = min(k.th, k.ph - k.ty), cols = min(k.tw, k.pw - k.tx);
                const int chunks = (cols + 7) >> 3;
                for (int i = tid; i < rows * chunks; i += kTileThreads) {
                    const int r = i / chunks, q = i - r * chunks;
                    const int x = k.tx + 8 * q, y = k.ty + r;
                    const uint16_t* src = to + r * k.tw + 8 * q;
                    const size_t idx = (size_t)y * k.pw + x;
                    if (8 * q + 8 <= cols && (idx & 7) == 0) {
                        const uint4 v = *(const uint4*)src;
                        if (P.bps == 2) {
                            *(uint4*)((uint16_t*)P.fin[c] + idx) = v;
                        } else {
                            const uint32_t lo = (v.x & 0xffu) | ((v.x >> 8) & 0xff00u) | ((v.y & 0xffu) << 16) |
                                                ((v.y & 0xff0000u) << 8);
                            const uint32_t hi = (v.z & 0xffu) | ((v.z >> 8) & 0xff00u) | ((v.w & 0xffu) << 16) |
                                                ((v.w & 0xff0000u) << 8);
                            *(uint2*)((uint8_t*)P.fin[c] + idx) = make_uint2(lo, hi);
                        }
                    } else {
                        for (int u = 0; u < 8 && 8 * q + u < cols; ++u) store_sample(P.fin[c], P.bps, idx + u, src[u]);
                    }
                }
            }
        }
        // ---- 6. RGB8 at the canvas position (four pixels per thread) ----
        if (do_rgb) {
            uint8_t* canvas = out + P.canvas_off;
            const int copy_w = min(P.crop_w, max(P.canvas_w - P.dst_x, 0));
            const int copy_h = min(P.crop_h, max(P.canvas_h - P.dst_y, 0));
            const RgbCoef kc = rgb_coef(P);
            const TileComp B = tcomp(1);
            const uint16_t* const tl = tout_of(0);
            const uint16_t* const tb = tout_of(1);
            const uint16_t* const tr = tout_of(2);
            for (int i = tid; i < (kTile / 4) * kTile; i += kTileThreads) {
                const int x0 = X + 4 * (i % (kTile / 4)), yy = Y + i / (kTile / 4);
                if (x0 >= copy_w || yy >= copy_h) continue;
                const int cnt = min(4, copy_w - x0);
                // four luma samples (one 8-byte load) and their chroma
                const uint2 lv = *(const uint2*)(tl + (yy - Y) * kTile + (x0 - X));
                const int luma[4] = {(int)(lv.x & 0xffff), (int)(lv.x >> 16), (int)(lv.y & 0xffff), (int)(lv.y >> 16)};
                int cb[4] = {0, 0, 0, 0}, cr[4] = {0, 0, 0, 0};
                if (P.idc) {
                    const int cy = yy / P.sub_h - B.ty;
                    const uint16_t* ob = tb + (size_t)cy * B.tw;
                    const uint16_t* orr = tr + (size_t)cy * B.tw;
                    if (P.sub_w == 2) {  // two chroma samples (one 4-byte load each)
                        const int cx = (x0 >> 1) - B.tx;
                        const uint32_t b = *(const uint32_t*)(ob + cx), r = *(const uint32_t*)(orr + cx);
                        cb[0] = cb[1] = b & 0xffff; cb[2] = cb[3] = b >> 16;
                        cr[0] = cr[1] = r & 0xffff; cr[2] = cr[3] = r >> 16;
                    } else {
                        const int cx = x0 - B.tx;
                        const uint2 b = *(const uint2*)(ob + cx), r = *(const uint2*)(orr + cx);
                        cb[0] = b.x & 0xffff; cb[1] = b.x >> 16; cb[2] = b.y & 0xffff; cb[3] = b.y >> 16;
                        cr[0] = r.x & 0xffff; cr[1] = r.x >> 16; cr[2] = r.y & 0xffff; cr[3] = r.y >> 16;
                    }
                }
                uint32_t px[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) px[u] = rgb_px(kc, P.idc, luma[u], cb[u], cr[u]);
                if (moves_samples(P.orientation)) {  // each pixel to its oriented place
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        if (u >= cnt) break;
                        uint8_t* q = canvas + oriented_index(P.dst_x + x0 + u, P.dst_y + yy, P.canvas_w, P.canvas_h,
                                                             P.orientation) * 3;
                        q[0] = (uint8_t)px[u];
                        q[1] = (uint8_t)(px[u] >> 8);
                        q[2] = (uint8_t)(px[u] >> 16);
                    }
                    continue;
                }
                uint8_t* o = canvas + ((size_t)(P.dst_y + yy) * P.canvas_w + P.dst_x + x0) * 3;
                if (cnt == 4 && ((uintptr_t)o & 3) == 0) {
                    uint32_t* o32 = (uint32_t*)o;
                    o32[0] = px[0] | (px[1] << 24);
                    o32[1] = (px[1] >> 8) | (px[2] << 16);
                    o32[2] = (px[2] >> 16) | (px[3] << 8);
                } else {
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        if (u >= cnt) break;
                        o[3 * u] = (uint8_t)px[u];
                        o[3 * u + 1] = (uint8_t)(px[u] >> 8);
                        o[3 * u + 2] = (uint8_t)(px[u] >> 16);
                    }
                }
            }
        }
    }
}

}  // namespace hpvcd

extern "C" cudaError_t hpvcd_launch_deblock(const hpvcd::DevPic* pics, int n_pics, int max_segments,
                                            int vertical, cudaStream_t stream) {
    if (n_pics <= 0 || max_segments <= 0) return cudaSuccess;
    const int threads = 256;
    dim3 grid((max_segments + threads - 1) / threads, n_pics, 2);
    hpvcd::k_deblock<<<grid, threads, 0, stream>>>(pics, vertical);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

// Blocks per grid-stride filter launch: 16 per SM of a B200 (148 SMs), split
// over the (picture, component) slices, so a batch of many small pictures
// is not thousands of tiny blocks.
static int filter_blocks_x(int quads, int slices, int threads) {
    const int target = 148 * 16;
    const int need = (quads + threads - 1) / threads;
    const int share = (target + slices - 1) / slices;
    return need < share ? (need > 0 ? need : 1) : (share > 0 ? share : 1);
}

extern "C" cudaError_t hpvcd_launch_sao(const hpvcd::DevPic* pics, int n_pics, int max_samples, int gated,
                                        cudaStream_t stream) {
    if (n_pics <= 0 || max_samples <= 0) return cudaSuccess;
    const int threads = 256;
    const int quads = (max_samples + 3) / 4;
    dim3 grid(filter_blocks_x(quads, n_pics * 3, threads), n_pics, 3);
    if (gated)
        hpvcd::k_sao<true><<<grid, threads, 0, stream>>>(pics);
    else
        hpvcd::k_sao<false><<<grid, threads, 0, stream>>>(pics);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

extern "C" cudaError_t hpvcd_launch_rgb(const hpvcd::DevPic* pics, int n_pics, int max_quads, uint8_t* out,
                                        cudaStream_t stream) {
    if (n_pics <= 0 || max_quads <= 0) return cudaSuccess;
    const int threads = 256;
    dim3 grid(filter_blocks_x(max_quads, n_pics, threads), n_pics, 1);
    hpvcd::k_rgb<<<grid, threads, 0, stream>>>(pics, out);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

extern "C" cudaError_t hpvcd_launch_yuv_canvas(const hpvcd::DevPic* pics, int n_pics, int max_quads, uint8_t* out,
                                               cudaStream_t stream) {
    if (n_pics <= 0 || max_quads <= 0) return cudaSuccess;
    const int threads = 256;
    dim3 grid(filter_blocks_x(max_quads, n_pics * 3, threads), n_pics, 3);
    hpvcd::k_yuv_canvas<<<grid, threads, 0, stream>>>(pics, out);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

// One k_filter_tile launch over pictures [0, n_pics) of `pics`: max_tiles =
// the 64 x 64 tiles of the largest picture, cfmt = the largest chroma
// layout class among them, out = the plan's canvases when RGB8 canvases are
// written (else NULL).  The shared-memory limit of the 4:4:4 layout was
// raised once by hpvcd_filter_tile_setup().
extern "C" cudaError_t hpvcd_launch_filter_tile(const hpvcd::DevPic* pics, int n_pics, int max_tiles, int cfmt,
                                                int gated, uint8_t* out, cudaStream_t stream) {
    if (n_pics <= 0 || max_tiles <= 0) return cudaSuccess;
    const int target = 148 * 8;  // resident CTAs of 256 threads on a B200
    const int per_pic = std::max(1, (target + n_pics - 1) / n_pics);
    dim3 grid(std::min(max_tiles, std::max(per_pic, 1)), n_pics, 1);
    const size_t smem = hpvcd::tile_smem_bytes(cfmt);
    if (gated)
        hpvcd::k_filter_tile<true><<<grid, hpvcd::kTileThreads, smem, stream>>>(pics, out, out ? 1 : 0, cfmt);
    else
        hpvcd::k_filter_tile<false><<<grid, hpvcd::kTileThreads, smem, stream>>>(pics, out, out ? 1 : 0, cfmt);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

// The shared-memory limit of the largest layout, and the whole unified L1 /
// shared array as shared memory, like the wavefront kernel: the tile filter
// of one concurrent group runs beside another group's wavefront, and an SM
// changes its L1 / shared split only when it holds no CTA.
// Once per device (a plan build calls it for every new batch layout).
namespace {
constexpr int kTileSetupDevices = 64;
std::mutex g_tile_setup_mu;
bool g_tile_setup_done[kTileSetupDevices];
}  // namespace

static cudaError_t filter_tile_attrs();

extern "C" cudaError_t hpvcd_filter_tile_setup() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kTileSetupDevices) {
        cudaGetLastError();
        return filter_tile_attrs();
    }
    std::lock_guard<std::mutex> lock(g_tile_setup_mu);
    if (g_tile_setup_done[dev]) return cudaSuccess;
    const cudaError_t e = filter_tile_attrs();
    g_tile_setup_done[dev] = e == cudaSuccess;
    return e;
}

static cudaError_t filter_tile_attrs() {
    const int lim = (int)hpvcd::tile_smem_bytes(1);
    cudaError_t e = cudaFuncSetAttribute(hpvcd::k_filter_tile<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(hpvcd::k_filter_tile<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(hpvcd::k_filter_tile<true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(hpvcd::k_filter_tile<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    return e;
}
