// recon.cu -- reconstruction of the transform-block records of a batch of
// pictures: dequantisation + inverse DCT/DST / transform skip / transquant
// bypass (transform.rs), intra prediction (intra.rs) and residual add + clip
// (reconstruct.rs), in the decode order of decode.rs:3478-5426.
//
// One CTA reconstructs one CTU at a time; CTUs are claimed from a global
// queue sorted by wavefront index (x + 2y) across all pictures, so a CTU is
// only claimed after every CTU it depends on (left, above-left, above,
// above-right) has been claimed by a running CTA -> no deadlock for any grid
// size.  Per CTU:
//   A. all coded TBs of the CTU are inverse-transformed in parallel (one warp
//      per TB) into a shared-memory residual canvas -- this needs no
//      neighbour and overlaps the wavefront wait;
//   B. wait (bounded) for the neighbour CTUs, load their edge samples, then
//      one warp walks the records in decode order: reference gathering with
//      z-order availability, substitution, filtering, prediction, add+clip,
//      all in shared memory;
//   C. the CTU interior is written to the plane and its ready flag released.
#include <cstdio>

#include "common.cuh"

namespace hpvcd {

constexpr int kReconWarps = 4;
constexpr int kReconThreads = kReconWarps * 32;
constexpr int kScr = 33;  // padded row stride of the per-warp transform scratch

// intra.rs:30-38 (H.265 Tables 8-4 / 8-5)
__constant__ int8_t c_intra_angle[33] = {32,  26,  21,  17,  13,  9,  5,  2,  0,  -2, -5,
                                         -9,  -13, -17, -21, -26, -32, -26, -21, -17, -13, -9,
                                         -5,  -2,  0,   2,   5,   9,   13,  17,  21,  26,  32};
__constant__ int16_t c_inv_angle[15] = {-4096, -1638, -910, -630, -482, -390, -315, -256,
                                        -315,  -390,  -482, -630, -910, -1638, -4096};
// transform.rs:37
__constant__ int32_t c_dequant_scale[6] = {40, 45, 51, 57, 64, 72};
// transform.rs:30 DST4
__constant__ int8_t c_dst4[4][4] = {{29, 55, 74, 84}, {74, 74, 0, -74}, {84, -29, -74, 55}, {55, -84, 74, -29}};
// H.265 DCT basis magnitudes by angle j (units of pi/64); see dct_entry().
__constant__ int8_t c_dct_mag[33] = {64, 90, 90, 90, 89, 88, 87, 85, 83, 82, 80, 78, 75, 73, 70, 67, 64,
                                     61, 57, 54, 50, 46, 43, 38, 36, 31, 25, 22, 18, 13, 9,  4,  0};

// Shared-memory layout of one CTA.  Sizes are for the largest CTB (64) and
// the largest chroma canvas of the batch (64 for 4:4:4, 32 otherwise).
struct ReconLayout {
    int cs;          // chroma canvas side
    size_t off_dct, off_res_y, off_res_c, off_int_y, off_int_c, off_top, off_left, off_scr,
        off_misc, total;
    __host__ __device__ explicit ReconLayout(int c444) {
        cs = c444 ? 64 : 32;
        size_t o = 0;
        off_dct = o;   o += 32 * 32 * sizeof(int16_t);
        off_res_y = o; o += 64 * 64 * sizeof(int32_t);
        off_res_c = o; o += 2 * (size_t)cs * cs * sizeof(int32_t);
        off_int_y = o; o += 64 * 64 * sizeof(uint16_t);
        off_int_c = o; o += 2 * (size_t)cs * cs * sizeof(uint16_t);
        off_top = o;   o += 3 * 136 * sizeof(uint16_t);
        off_left = o;  o += 3 * 64 * sizeof(uint16_t);
        off_scr = o;   o += (size_t)kReconWarps * 2 * 32 * kScr * sizeof(int16_t);
        off_misc = o;  o += 2048;
        total = o;
    }
};

// Phase-B scratch (used by warp 0 only).
struct PredScratch {
    int32_t s[132];        // substituted reference line (4n+1), -1 = unavailable
    uint16_t above[68];    // 2n+1
    uint16_t left[68];
    uint16_t fa[68];
    uint16_t fl[68];
    int32_t refs[100];     // 3n+1 angular projection
    uint32_t decoded[16];  // 16x16 luma 4x4 cells of the CTU, bit x of word y
    uint32_t item;
    int32_t err;
};

struct Canvas {
    uint16_t* interior[3];
    uint16_t* top[3];   // x = -1 .. 2S-1 stored at [x + 1]
    uint16_t* left[3];  // y = 0 .. S-1
    int32_t* res[3];
    int side[3];        // S per component
};

__device__ __forceinline__ int dct_entry(int n, int k, int m) {
    if (k == 0) return 64;
    const int k32 = k * (32 / n);
    int j = (k32 * (2 * m + 1)) & 127;
    int sign = 1;
    if (j > 64) j = 128 - j;
    if (j > 32) {
        j = 64 - j;
        sign = -1;
    }
    return sign * c_dct_mag[j];
}

// ---------------------------------------------------------------------------
// Residual of one coded TB by one warp (transform.rs:489-858, decode.rs
// :4754-4903 luma and :5313-5417 chroma), written into `res` (stride rs).
// ---------------------------------------------------------------------------
__device__ void tb_residual_warp(const DevPic& P, const hpvcd_tu& t, int32_t* res, int rs,
                                 const int16_t* dct, int16_t* buf, int16_t* tmp, int lane) {
    const int n = 1 << t.log2n;
    const bool luma = t.comp == 0;
    const int bd = luma ? P.bd : P.bd_c;
    const bool i16s = bd <= 8;
    const int16_t* lv = P.coeffs + t.coeff_off;
    if (t.flags & HPVCD_TU_TQB) {  // decode.rs:4754-4757 / :4830-4834: residual = levels
        for (int i = lane; i < n * n; i += 32) res[(i / n) * rs + (i % n)] = lv[i];
        return;
    }
    int qpp;
    if (luma) {
        qpp = qp_prime(t.qp_y, bd);
    } else {
        const int pps_off = t.comp == 1 ? P.pps_cb_qp_offset : P.pps_cr_qp_offset;
        qpp = qp_prime(qpc_map(t.qp_y + pps_off + t.cqp_off, P.idc, bd), bd);
    }
    // transform.rs:701-725 dequant_params (non-extended precision: range 15)
    const int bd_shift = bd + t.log2n + 10 - 15;
    const int max_qpp = 51 + 6 * (bd - 8);
    const int qs = clamp3i(qpp, 0, max_qpp);
    const long long factor = (long long)c_dequant_scale[qs % 6] * (1ll << (qs / 6)) * 16;
    const long long add = 1ll << (bd_shift - 1);
    if (t.flags & HPVCD_TU_TSKIP) {  // transform.rs:728-792
        const int tr_shift = 15 - bd - t.log2n;
        const int tr_add = tr_shift > 0 ? 1 << (tr_shift - 1) : 0;
        for (int i = lane; i < n * n; i += 32) {
            long long l = lv[i];
            long long v = (l * factor + add) >> bd_shift;
            v = v < -32768 ? -32768 : (v > 32767 ? 32767 : v);
            int r = tr_shift >= 0 ? ((int)v + tr_add) >> tr_shift : (int)((unsigned)v << (-tr_shift));
            res[(i / n) * rs + (i % n)] = i16s ? (int)(int16_t)r : r;
        }
        return;
    }
    const int nx = (t.nx == 0 || t.nx > n) ? n : t.nx;
    // dequantise into buf (row-major, padded); columns >= nx are zero
    // (transform.rs:510-511: stage 1 skips them).  Track the last non-zero row.
    int my_rows = 0;
    for (int i = lane; i < n * n; i += 32) {
        const int r = i / n, c = i % n;
        int v = 0;
        if (c < nx) {
            const long long l = lv[i];
            long long d = (l * factor + add) >> bd_shift;
            v = (int)(d < -32768 ? -32768 : (d > 32767 ? 32767 : d));
        }
        buf[r * kScr + c] = (int16_t)v;
        if (v) my_rows = r + 1;
    }
    int rows = my_rows;
    for (int o = 16; o; o >>= 1) rows = max(rows, __shfl_xor_sync(0xffffffffu, rows, o));
    __syncwarp();
    const bool dst = luma && n == 4 && (t.flags & HPVCD_TU_INTRA);
    const int step = 32 / n;
    // stage 1 (columns): tmp[m][c] = clip((sum_k T[k][m] * buf[k][c] + 64) >> 7)
    for (int i = lane; i < n * n; i += 32) {
        const int m = i / n, c = i % n;
        int acc = 0;
        if (dst) {
            for (int k = 0; k < 4; ++k) acc += c_dst4[k][m] * buf[k * kScr + c];
        } else {
            for (int k = 0; k < rows; ++k) acc += dct[(k * step) * 32 + m] * buf[k * kScr + c];
        }
        tmp[m * kScr + c] = (int16_t)clamp3i((acc + 64) >> 7, -32768, 32767);
    }
    __syncwarp();
    // stage 2 (rows): out[r][m] = (sum_k T[k][m] * tmp[r][k] + add2) >> shift2
    const int shift2 = 20 - bd;
    const int add2 = 1 << (shift2 - 1);
    const int kmax = dst ? 4 : nx;
    for (int i = lane; i < n * n; i += 32) {
        const int r = i / n, m = i % n;
        int acc = 0;
        if (dst) {
            for (int k = 0; k < 4; ++k) acc += c_dst4[k][m] * tmp[r * kScr + k];
        } else {
            for (int k = 0; k < kmax; ++k) acc += dct[(k * step) * 32 + m] * tmp[r * kScr + k];
        }
        const int v = (acc + add2) >> shift2;
        res[r * rs + m] = i16s ? (int)(int16_t)v : v;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Availability and sample access for component c at CTU-relative coords.
// ---------------------------------------------------------------------------
struct CtuGeo {
    int ox[3], oy[3];  // CTU origin in component samples
    int pw[3], ph[3];  // plane size
    int S[3];
    int sub_w, sub_h;
    int w, h;
};

// decode.rs:4651-4690 luma_avail / chroma_avail with the `decoded` map
// restricted to this CTU and its (already reconstructed) neighbours.
__device__ __forceinline__ bool avail(const CtuGeo& g, const PredScratch& ps, int c, int x, int y) {
    const int ax = g.ox[c] + x, ay = g.oy[c] + y;
    if (ax < 0 || ay < 0 || ax >= g.pw[c] || ay >= g.ph[c]) return false;
    const int sw = c ? g.sub_w : 1, sh = c ? g.sub_h : 1;
    if (ax * sw >= g.w || ay * sh >= g.h) return false;
    const int S = g.S[c];
    if (y < 0) return true;          // CTU row above: fully reconstructed
    if (x < 0) return y < S;         // left CTU yes, below-left CTU not yet
    if (x >= S || y >= S) return false;
    const int lx = (x * sw) >> 2, ly = (y * sh) >> 2;
    return (ps.decoded[ly] >> lx) & 1u;
}

__device__ __forceinline__ int fetch(const Canvas& cv, int c, int x, int y) {
    if (y < 0) return cv.top[c][x + 1];
    if (x < 0) return cv.left[c][y];
    return cv.interior[c][y * cv.side[c] + x];
}

// intra.rs:84-148 substitution, :151-219 filtering, :257-372 prediction, and
// the residual add of reconstruct.rs:214-251, for one TB by one warp.
__device__ void predict_tb_warp(const DevPic& P, const hpvcd_tu& t, int c, int x0, int y0,
                                const CtuGeo& g, const Canvas& cv, PredScratch& ps, int lane,
                                bool coded) {
    const int n = 1 << t.log2n;
    const bool luma = c == 0;
    const int bd = luma ? P.bd : P.bd_c;
    const int total = 4 * n + 1;
    // gather: s[i] = left[2n-1-i] (i < 2n), s[2n] = corner, s[2n+1+i] = above[i]
    for (int i = lane; i < total; i += 32) {
        int x, y;
        if (i < 2 * n) {
            x = x0 - 1;
            y = y0 + (2 * n - 1 - i);
        } else if (i == 2 * n) {
            x = x0 - 1;
            y = y0 - 1;
        } else {
            x = x0 + (i - 2 * n - 1);
            y = y0 - 1;
        }
        ps.s[i] = avail(g, ps, c, x, y) ? fetch(cv, c, x, y) : -1;
    }
    __syncwarp();
    uint32_t mask[5];
#pragma unroll
    for (int wd = 0; wd < 5; ++wd) {
        const int i = wd * 32 + lane;
        mask[wd] = __ballot_sync(0xffffffffu, i < total && ps.s[i] >= 0);
    }
    int first = -1;
#pragma unroll
    for (int wd = 4; wd >= 0; --wd)
        if (mask[wd]) first = wd * 32 + __ffs(mask[wd]) - 1;
    const int neutral = 1 << (bd - 1);
    // substituted value of position i (last available j <= i, or `first`)
    int subst[5];
#pragma unroll
    for (int wd = 0; wd < 5; ++wd) {
        const int i = wd * 32 + lane;
        int v = neutral;
        if (i < total && first >= 0) {
            int j = -1;
            const uint32_t m0 = mask[wd] & (0xffffffffu >> (31 - lane));
            if (m0) {
                j = wd * 32 + 31 - __clz(m0);
            } else {
                for (int q = wd - 1; q >= 0; --q)
                    if (mask[q]) {
                        j = q * 32 + 31 - __clz(mask[q]);
                        break;
                    }
            }
            if (j < 0) j = first;
            v = ps.s[j];
        }
        subst[wd] = v;
    }
    __syncwarp();
#pragma unroll
    for (int wd = 0; wd < 5; ++wd) {
        const int i = wd * 32 + lane;
        if (i < total) {
            // above_out[k] = s[2n + k], left_out[k] = s[2n - k]
            if (i >= 2 * n) ps.above[i - 2 * n] = (uint16_t)subst[wd];
            if (i <= 2 * n) ps.left[2 * n - i] = (uint16_t)subst[wd];
        }
    }
    __syncwarp();
    // filtering (luma, or 4:4:4 chroma without strong smoothing)
    const int mode = t.mode;
    const uint16_t* A = ps.above;
    const uint16_t* L = ps.left;
    const bool smoothing = !(P.flags & HPVCD_PIC_SMOOTHING_DISABLED);
    const bool filt_ok = luma || P.idc == 3;
    bool do_filter = false;
    if (filt_ok && smoothing && n != 4 && mode != 1) {
        const int md = min(abs(mode - 26), abs(mode - 10));
        const int thresh = n == 8 ? 7 : (n == 16 ? 1 : (n == 32 ? 0 : 8));
        do_filter = mode == 0 || md > thresh;
    }
    if (do_filter) {
        bool strong = false;
        if (luma && (P.flags & HPVCD_PIC_STRONG_SMOOTHING) && n == 32) {
            const int thr = 1 << (bd - 5);
            const int bl = L[2 * n], tl = A[0], tr = A[2 * n], cl = L[n], ct = A[n];
            strong = abs(bl + tl - 2 * cl) < thr && abs(tr + tl - 2 * ct) < thr;
        }
        for (int i = lane; i <= 2 * n; i += 32) {
            int fa, fl;
            if (strong) {
                const int tl = A[0], tr = A[2 * n], bl = L[2 * n];
                if (i == 0 || i == 2 * n) {
                    fa = A[i];
                    fl = L[i];
                } else {
                    fa = ((2 * n - i) * tl + i * tr + n) >> 6;
                    fl = ((2 * n - i) * tl + i * bl + n) >> 6;
                }
            } else if (i == 0) {
                fa = fl = (L[1] + 2 * A[0] + A[1] + 2) >> 2;
            } else if (i == 2 * n) {
                fa = A[i];
                fl = L[i];
            } else {
                fa = (A[i - 1] + 2 * A[i] + A[i + 1] + 2) >> 2;
                fl = (L[i - 1] + 2 * L[i] + L[i + 1] + 2) >> 2;
            }
            ps.fa[i] = (uint16_t)fa;
            ps.fl[i] = (uint16_t)fl;
        }
        __syncwarp();
        A = ps.fa;
        L = ps.fl;
    }
    const int max_v = (1 << bd) - 1;
    const bool edge_filters = luma && n < 32;  // is_luma gate of predict_into
    const int log2n = t.log2n;
    const int S = cv.side[c];
    uint16_t* out = cv.interior[c];
    const int32_t* res = cv.res[c];
    const int vw = min(n, g.pw[c] - (g.ox[c] + x0)), vh = min(n, g.ph[c] - (g.oy[c] + y0));
    if (mode >= 2) {
        const int angle = c_intra_angle[mode - 2];
        const bool vertical = mode >= 18;
        const uint16_t* mainr = vertical ? A : L;
        const uint16_t* side = vertical ? L : A;
        for (int i = lane; i <= 2 * n; i += 32) ps.refs[n + i] = mainr[i];
        if (angle < 0) {
            const int inv = c_inv_angle[mode - 11];
            const int lim = (n * angle) >> 5;
            for (int k = -1 - lane; k >= lim; k -= 32) {
                const int idx = min((k * inv + 128) >> 8, 2 * n);
                ps.refs[k + n] = side[max(idx, 0)];
            }
        }
        __syncwarp();
        for (int i = lane; i < n * n; i += 32) {
            const int yy = i >> log2n, xx = i & (n - 1);
            const int a = vertical ? yy : xx;  // index whose (a+1)*angle gives the position
            const int b = vertical ? xx : yy;  // index along the main reference
            const int pos = (a + 1) * angle;
            const int iidx = pos >> 5, frac = pos & 31;
            const int r0 = ps.refs[b + iidx + 1 + n];
            int v = r0;
            if (frac) v = ((32 - frac) * r0 + frac * ps.refs[b + iidx + 2 + n] + 16) >> 5;
            v = clamp3i(v, 0, max_v);
            if (edge_filters) {
                if (mode == 26 && xx == 0) v = clamp3i(A[1] + ((L[yy + 1] - A[0]) >> 1), 0, max_v);
                if (mode == 10 && yy == 0) v = clamp3i(L[1] + ((A[xx + 1] - A[0]) >> 1), 0, max_v);
            }
            if (xx < vw && yy < vh) {
                if (coded) v = clamp3i(v + res[(y0 + yy) * S + x0 + xx], 0, max_v);
                out[(y0 + yy) * S + x0 + xx] = (uint16_t)v;
            }
        }
    } else if (mode == 1) {  // DC
        int sum = 0;
        for (int i = 1; i <= n; ++i) sum += A[i] + L[i];
        const int dc = (sum + n) >> (log2n + 1);
        for (int i = lane; i < n * n; i += 32) {
            const int yy = i >> log2n, xx = i & (n - 1);
            int v = dc;
            if (edge_filters) {
                if (xx == 0 && yy == 0)
                    v = (L[1] + 2 * dc + A[1] + 2) >> 2;
                else if (yy == 0)
                    v = (A[xx + 1] + 3 * dc + 2) >> 2;
                else if (xx == 0)
                    v = (L[yy + 1] + 3 * dc + 2) >> 2;
            }
            if (xx < vw && yy < vh) {
                if (coded) v = clamp3i(v + res[(y0 + yy) * S + x0 + xx], 0, max_v);
                out[(y0 + yy) * S + x0 + xx] = (uint16_t)v;
            }
        }
    } else {  // planar
        const int tr = A[n + 1], bl = L[n + 1];
        for (int i = lane; i < n * n; i += 32) {
            const int yy = i >> log2n, xx = i & (n - 1);
            const int hh = (n - 1 - xx) * L[yy + 1] + (xx + 1) * tr;
            const int vv = (n - 1 - yy) * A[xx + 1] + (yy + 1) * bl;
            int v = (hh + vv + n) >> (log2n + 1);
            if (xx < vw && yy < vh) {
                if (coded) v = clamp3i(v + res[(y0 + yy) * S + x0 + xx], 0, max_v);
                out[(y0 + yy) * S + x0 + xx] = (uint16_t)v;
            }
        }
    }
    __syncwarp();
}

__device__ __forceinline__ void mark_decoded(const CtuGeo& g, PredScratch& ps, int x0, int y0, int n,
                                             int lane) {
    // luma CTU-relative square; cells outside the picture stay unmarked
    // (decode.rs:3170-3189 via fill_grid_rect clipped to the grid).
    for (int i = lane; i < 16; i += 32) {
        const int cy = i;
        const int y = cy * 4;
        if (y < y0 || y >= y0 + n || g.oy[0] + y >= g.h) continue;
        uint32_t bits = 0;
        for (int x = x0; x < x0 + n && x < 64; x += 4)
            if (g.ox[0] + x < g.w) bits |= 1u << (x >> 2);
        ps.decoded[cy] |= bits;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// The kernel.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kReconThreads)
k_recon(const DevPic* __restrict__ pics, const CtuItem* __restrict__ items, uint32_t n_items,
        uint32_t* work_counter, uint32_t* dev_err, int c444, uint32_t spin_limit) {
    extern __shared__ __align__(16) unsigned char smem[];
    const ReconLayout lay(c444);
    int16_t* dct = (int16_t*)(smem + lay.off_dct);
    PredScratch& ps = *(PredScratch*)(smem + lay.off_misc);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int16_t* wbuf = (int16_t*)(smem + lay.off_scr) + (size_t)warp * 2 * 32 * kScr;
    int16_t* wtmp = wbuf + 32 * kScr;

    for (int i = tid; i < 32 * 32; i += kReconThreads) dct[i] = (int16_t)dct_entry(32, i / 32, i % 32);

    for (;;) {
        __syncthreads();
        if (tid == 0) ps.item = atomicAdd(work_counter, 1u);
        __syncthreads();
        const uint32_t item = ps.item;
        if (item >= n_items) break;
        const CtuItem it = items[item];
        const DevPic& P = pics[it.pic];
        const int ctb = 1 << P.log2_ctb;
        CtuGeo g;
        g.w = P.w;
        g.h = P.h;
        g.sub_w = P.sub_w;
        g.sub_h = P.sub_h;
        g.ox[0] = it.cx * ctb;
        g.oy[0] = it.cy * ctb;
        g.pw[0] = P.w;
        g.ph[0] = P.h;
        g.S[0] = ctb;
        for (int c = 1; c < 3; ++c) {
            g.ox[c] = g.ox[0] / P.sub_w;
            g.oy[c] = g.oy[0] / P.sub_h;
            g.pw[c] = P.cw;
            g.ph[c] = P.ch;
            g.S[c] = ctb / P.sub_w;
        }
        Canvas cv;
        cv.interior[0] = (uint16_t*)(smem + lay.off_int_y);
        cv.interior[1] = (uint16_t*)(smem + lay.off_int_c);
        cv.interior[2] = cv.interior[1] + lay.cs * lay.cs;
        cv.res[0] = (int32_t*)(smem + lay.off_res_y);
        cv.res[1] = (int32_t*)(smem + lay.off_res_c);
        cv.res[2] = cv.res[1] + lay.cs * lay.cs;
        for (int c = 0; c < 3; ++c) {
            cv.top[c] = (uint16_t*)(smem + lay.off_top) + c * 136;
            cv.left[c] = (uint16_t*)(smem + lay.off_left) + c * 64;
            cv.side[c] = g.S[c];
        }
        const int ncomp = P.idc ? 3 : 1;
        const uint32_t ci = (uint32_t)it.cy * P.ctb_cols + it.cx;
        uint32_t r0 = P.ctu_start[ci], r1 = P.ctu_start[ci + 1];
        if (r1 > P.n_tus || r0 > r1) {  // malformed CTU range: report, reconstruct nothing
            if (tid == 0) atomicOr(dev_err, DEV_ERR_BITSTREAM);
            r1 = min(r1, P.n_tus);
            r0 = min(r0, r1);
        }
        if (tid < 16) ps.decoded[tid] = 0;
        if (tid == 0) ps.err = 0;
        // Inter / prediction-in-plane pictures: the plane already holds the
        // prediction; load the CTU interior.
        const bool pred_plane = (P.flags & (HPVCD_PIC_PRED_IN_PLANE | HPVCD_PIC_INTER)) != 0;
        if (pred_plane) {
            for (int c = 0; c < ncomp; ++c) {
                const int S = g.S[c];
                for (int i = tid; i < S * S; i += kReconThreads) {
                    const int y = i / S, x = i % S;
                    const int ax = g.ox[c] + x, ay = g.oy[c] + y;
                    int v = 0;
                    if (ax < g.pw[c] && ay < g.ph[c])
                        v = load_sample(P.rec[c], P.bps, (size_t)ay * g.pw[c] + ax);
                    cv.interior[c][i] = (uint16_t)v;
                }
            }
        }
        // ---- Phase A: residuals of all coded TBs, one warp per TB ----
        {
            int k = 0;
            for (uint32_t r = r0; r < r1; ++r) {
                const hpvcd_tu t = P.tus[r];
                if (!(t.flags & HPVCD_TU_CBF)) continue;
                if ((k++ % kReconWarps) != warp) continue;
                const int c = t.comp;
                const int n = 1 << t.log2n;
                const int x = (int)t.x - g.ox[c < 3 ? c : 0], y = (int)t.y - g.oy[c < 3 ? c : 0];
                const bool bad = c >= ncomp || t.log2n < 2 || t.log2n > 5 || x < 0 || y < 0 ||
                                 x + n > g.S[c] || y + n > g.S[c] ||
                                 (uint64_t)t.coeff_off + (uint64_t)n * n > P.n_coeffs;
                if (bad) {
                    if (lane == 0) atomicOr(dev_err, DEV_ERR_BITSTREAM);
                    continue;
                }
                tb_residual_warp(P, t, cv.res[c] + y * g.S[c] + x, g.S[c], dct, wbuf, wtmp, lane);
            }
        }
        // ---- Phase B prologue: wait for the neighbours and load their edges ----
        if (P.needs_wavefront && tid == 0) {
            const int cx = it.cx, cy = it.cy;
            const int nb[4][2] = {{cx - 1, cy}, {cx - 1, cy - 1}, {cx, cy - 1}, {cx + 1, cy - 1}};
            for (int k = 0; k < 4; ++k) {
                const int nx = nb[k][0], ny = nb[k][1];
                if (nx < 0 || ny < 0 || nx >= P.ctb_cols) continue;
                const uint32_t* f = P.ready + (size_t)ny * P.ctb_cols + nx;
                uint32_t spins = 0;
                while (ld_acquire(f) == 0u) {
                    if (++spins > spin_limit) {
                        atomicOr(dev_err, DEV_ERR_TIMEOUT);
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        __syncthreads();
        if (P.needs_wavefront) {
            for (int c = 0; c < ncomp; ++c) {
                const int S = g.S[c];
                for (int i = tid; i < 2 * S + 1; i += kReconThreads) {
                    const int x = i - 1;
                    const int ax = g.ox[c] + x, ay = g.oy[c] - 1;
                    int v = 0;
                    if (ay >= 0 && ax >= 0 && ax < g.pw[c])
                        v = load_sample_cg(P.rec[c], P.bps, (size_t)ay * g.pw[c] + ax);
                    cv.top[c][i] = (uint16_t)v;
                }
                for (int i = tid; i < S; i += kReconThreads) {
                    const int ax = g.ox[c] - 1, ay = g.oy[c] + i;
                    int v = 0;
                    if (ax >= 0 && ay < g.ph[c])
                        v = load_sample_cg(P.rec[c], P.bps, (size_t)ay * g.pw[c] + ax);
                    cv.left[c][i] = (uint16_t)v;
                }
            }
        }
        __syncthreads();
        // ---- Phase B: decode-order walk by warp 0 ----
        if (warp == 0) {
            const bool intra_pred_ok = !(P.flags & HPVCD_PIC_PRED_IN_PLANE);
            for (uint32_t r = r0; r < r1; ++r) {
                const hpvcd_tu t = P.tus[r];
                const int c = t.comp;
                const int n = 1 << t.log2n;
                if (c >= ncomp || t.log2n < 2 || t.log2n > 6) continue;
                const int x = (int)t.x - g.ox[c], y = (int)t.y - g.oy[c];
                if (x < 0 || y < 0 || x + n > g.S[c] || y + n > g.S[c]) continue;
                const bool coded = (t.flags & HPVCD_TU_CBF) != 0 && t.log2n <= 5 &&
                                   (uint64_t)t.coeff_off + (uint64_t)n * n <= P.n_coeffs;
                const bool intra = (t.flags & HPVCD_TU_INTRA) != 0;
                if (intra && intra_pred_ok) {
                    if (t.log2n <= 5 && t.mode <= 34)
                        predict_tb_warp(P, t, c, x, y, g, cv, ps, lane, coded);
                    else if (lane == 0)
                        atomicOr(dev_err, DEV_ERR_BITSTREAM);
                } else if (coded) {
                    // prediction already in the canvas: add + clip (reconstruct.rs:214-251)
                    const int S = g.S[c];
                    const int bd = c ? P.bd_c : P.bd;
                    const int mx = (1 << bd) - 1;
                    const int vw = min(n, g.pw[c] - (g.ox[c] + x)), vh = min(n, g.ph[c] - (g.oy[c] + y));
                    for (int i = lane; i < n * n; i += 32) {
                        const int yy = i / n, xx = i % n;
                        if (xx < vw && yy < vh) {
                            const int idx = (y + yy) * S + x + xx;
                            cv.interior[c][idx] =
                                (uint16_t)clamp3i((int)cv.interior[c][idx] + cv.res[c][idx], 0, mx);
                        }
                    }
                    __syncwarp();
                }
                if (c == 0) mark_decoded(g, ps, x, y, n, lane);
            }
        }
        __syncthreads();
        // ---- Phase C: publish the CTU ----
        for (int c = 0; c < ncomp; ++c) {
            const int S = g.S[c];
            for (int i = tid; i < S * S; i += kReconThreads) {
                const int y = i / S, x = i % S;
                const int ax = g.ox[c] + x, ay = g.oy[c] + y;
                if (ax < g.pw[c] && ay < g.ph[c])
                    store_sample(P.rec[c], P.bps, (size_t)ay * g.pw[c] + ax, cv.interior[c][i]);
            }
        }
        __threadfence();
        __syncthreads();
        if (tid == 0 && P.needs_wavefront) st_release(P.ready + ci, 1u);
    }
}

}  // namespace hpvcd

extern "C" size_t hpvcd_recon_smem_bytes(int c444) { return hpvcd::ReconLayout(c444).total; }

extern "C" cudaError_t hpvcd_launch_recon(const hpvcd::DevPic* pics, const hpvcd::CtuItem* items,
                                          uint32_t n_items, uint32_t* work_counter, uint32_t* dev_err,
                                          int c444, int grid, cudaStream_t stream) {
    const size_t smem = hpvcd::ReconLayout(c444).total;
    static bool configured[2] = {false, false};
    if (!configured[c444 ? 1 : 0]) {
        cudaError_t e = cudaFuncSetAttribute(hpvcd::k_recon, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        configured[c444 ? 1 : 0] = true;
    }
    // 2^22 polls of >= 64 ns each bound one neighbour wait to a few hundred ms.
    hpvcd::k_recon<<<grid, hpvcd::kReconThreads, smem, stream>>>(pics, items, n_items, work_counter,
                                                                 dev_err, c444, 1u << 22);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

extern "C" int hpvcd_recon_occupancy(int c444) {
    int blocks = 0;
    const size_t smem = hpvcd::ReconLayout(c444).total;
    cudaFuncSetAttribute(hpvcd::k_recon, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, hpvcd::k_recon, hpvcd::kReconThreads, smem);
    return blocks;
}
