// hpvcd_oracle.cpp -- TEST INFRASTRUCTURE: scalar C++ restatement of the
// hpvcd (Rust) reconstruction path, used only as the checker of the CUDA
// back end and as the timed CPU baseline.  Every function names the
// reference file:line it follows.  Integer arithmetic, clipping and storage
// truncation follow the reference's scalar path exactly.
#include "hpvcd_oracle.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "cpu_simd.h"

namespace {

template <typename T>
inline T clamp3(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------------------
// transform.rs
// ---------------------------------------------------------------------------

// transform.rs:30 DST4 (HEVC 4x4 DST-VII matrix, rows = basis functions).
const int32_t kDst4[4][4] = {
    {29, 55, 74, 84}, {74, 74, 0, -74}, {84, -29, -74, 55}, {55, -84, 74, -29}};

// transform.rs:37
const int64_t kDequantScale[6] = {40, 45, 51, 57, 64, 72};

// Magnitudes of the HEVC 32-point DCT basis, indexed by the angle j in units
// of pi/64 (entry = round-ish 64*sqrt(2)*cos(j*pi/64) as fixed by H.265
// Table 8-x; j = 16 gives 64, j = 32 gives 0).  The odd-part coefficient rows
// of transform.rs:67-404 (idct_odd_8/16/32) and the 4-point core :406-413 are
// all entries of this one matrix.
const int32_t kDctMag[33] = {64, 90, 90, 90, 89, 88, 87, 85, 83, 82, 80, 78, 75, 73, 70, 67, 64,
                             61, 57, 54, 50, 46, 43, 38, 36, 31, 25, 22, 18, 13, 9,  4,  0};

// Entry T_N[k][m] of the N-point HEVC inverse-transform matrix (basis k,
// sample m).
inline int32_t dct_entry(int n, int k, int m) {
    if (k == 0) return 64;
    const int k32 = k * (32 / n);
    int j = (k32 * (2 * m + 1)) % 128;
    int sign = 1;
    if (j > 64) j = 128 - j;
    if (j > 32) {
        j = 64 - j;
        sign = -1;
    }
    return sign * kDctMag[j];
}

// transform.rs:406 idct_raw_4 and :416-449 idct_raw_8/16/32: even/odd
// partial butterfly; exact integer sums (no intermediate rounding).
void idct_raw(int n, const int32_t* c, int32_t* out) {
    if (n == 4) {
        const int32_t e0 = 64 * (c[0] + c[2]);
        const int32_t e1 = 64 * (c[0] - c[2]);
        const int32_t o0 = 83 * c[1] + 36 * c[3];
        const int32_t o1 = 36 * c[1] - 83 * c[3];
        out[0] = e0 + o0;
        out[1] = e1 + o1;
        out[2] = e1 - o1;
        out[3] = e0 - o0;
        return;
    }
    const int half = n / 2;
    int32_t even[16] = {0}, ee[16] = {0};
    for (int j = 0; j < half; ++j) even[j] = c[2 * j];
    idct_raw(half, even, ee);
    for (int k = 0; k < half; ++k) {
        int32_t oo = 0;  // idct_odd_N row k: sum over odd basis functions
        for (int j = 1; j < n; j += 2) oo += dct_entry(n, j, k) * c[j];
        out[k] = ee[k] + oo;
        out[n - 1 - k] = ee[k] - oo;
    }
}

inline int32_t store(int32_t v, bool i16_store) {
    // transform.rs:55-63: `v as i16` truncates for the 8-bit storage path.
    return i16_store ? (int32_t)(int16_t)v : v;
}

// transform.rs:489-532 inv_dct_n_into.
void inv_dct(const int32_t* coeff, int n, int bd, int max_range, int nx, bool i16s,
             int32_t* out) {
    const int shift1 = 7, add1 = 1 << (shift1 - 1);
    const int shift2 = max_range + 5 - bd, add2 = 1 << (shift2 - 1);
    const int32_t cmin = -(1 << max_range), cmax = (1 << max_range) - 1;
    int32_t tmp[32 * 32];
    std::memset(tmp, 0, sizeof(int32_t) * n * n);
    nx = std::min(nx, n);
    int32_t col[32], raw[32];
    for (int c = 0; c < nx; ++c) {
        for (int k = 0; k < n; ++k) col[k] = coeff[k * n + c];
        idct_raw(n, col, raw);
        for (int m = 0; m < n; ++m) tmp[m * n + c] = clamp3((raw[m] + add1) >> shift1, cmin, cmax);
    }
    for (int r = 0; r < n; ++r) {
        idct_raw(n, tmp + r * n, raw);
        for (int m = 0; m < n; ++m) out[r * n + m] = store((raw[m] + add2) >> shift2, i16s);
    }
}

// transform.rs:535-591 inv_transform_n_into with DST4 (4x4 only).
void inv_dst4(const int32_t* coeff, int bd, int max_range, bool i16s, int32_t* out) {
    const int shift1 = 7, add1 = 1 << (shift1 - 1);
    const int shift2 = max_range + 5 - bd, add2 = 1 << (shift2 - 1);
    const int32_t cmin = -(1 << max_range), cmax = (1 << max_range) - 1;
    int32_t tmp[16];
    for (int c = 0; c < 4; ++c) {
        int32_t acc[4] = {0, 0, 0, 0};
        for (int k = 0; k < 4; ++k) {
            const int32_t ck = coeff[k * 4 + c];
            for (int m = 0; m < 4; ++m) acc[m] += kDst4[k][m] * ck;
        }
        for (int m = 0; m < 4; ++m) tmp[m * 4 + c] = clamp3((acc[m] + add1) >> shift1, cmin, cmax);
    }
    for (int r = 0; r < 4; ++r) {
        int32_t acc[4] = {0, 0, 0, 0};
        for (int k = 0; k < 4; ++k)
            for (int m = 0; m < 4; ++m) acc[m] += kDst4[k][m] * tmp[r * 4 + k];
        for (int m = 0; m < 4; ++m) out[r * 4 + m] = store((acc[m] + add2) >> shift2, i16s);
    }
}

// transform.rs:692
int max_tr_range(int bd, bool ext) { return ext ? std::max(15, bd + 6) : 15; }

// transform.rs:701-725
orc_dequant_params dequant_params(int n, int qp_prime, int bd, bool ext) {
    int log2n = 0;
    while ((1 << log2n) < n) ++log2n;
    const int64_t max_range = max_tr_range(bd, ext);
    const int64_t bd_shift = bd + log2n + 10 - max_range;
    const int max_qp_prime = 51 + 6 * (bd - 8);
    const int64_t qps = clamp3(qp_prime, 0, max_qp_prime);
    const int64_t scale = kDequantScale[qps % 6];
    const int64_t per = (int64_t)1 << (qps / 6);
    orc_dequant_params p;
    p.factor = scale * per * 16;
    p.add = (int64_t)1 << (bd_shift - 1);
    p.shift = (int32_t)bd_shift;
    p.pad = 0;
    p.clip_min = -((int64_t)1 << max_range);
    p.clip_max = ((int64_t)1 << max_range) - 1;
    return p;
}

// transform.rs:728-752
orc_ts_params ts_params(int n, int qp_prime, int bd, bool ext) {
    orc_ts_params t;
    t.dq = dequant_params(n, qp_prime, bd, ext);
    int log2n = 0;
    while ((1 << log2n) < n) ++log2n;
    int tr_shift = max_tr_range(bd, ext) - bd - log2n;
    if (ext) tr_shift = std::max(tr_shift, 0);
    t.tr_shift = tr_shift;
    t.tr_add = tr_shift > 0 ? (1 << (tr_shift - 1)) : 0;
    return t;
}

// transform.rs:668-683 ScalingMatrix::coeff (8x8 list upsampled, DC for >=16).
inline int64_t scaling_coeff(const uint8_t* m, int dc, int n, int idx) {
    if (n == 4) return m[idx];
    if (idx == 0 && n >= 16) return dc;
    const int y = idx / n, x = idx - y * n;
    const int down = (n == 8) ? 0 : (n == 16 ? 1 : 2);
    return m[(y >> down) * 8 + (x >> down)];
}

// transform.rs:764-776 dequantize_into_scalar and :794-808 (scaled).
void dequant(const int32_t* levels, int n, const orc_dequant_params& p, const uint8_t* sc,
             int sc_dc, bool i16s, int32_t* out) {
    const int64_t base = p.factor / 16;
    for (int i = 0; i < n * n; ++i) {
        const int64_t f = sc ? base * scaling_coeff(sc, sc_dc, n, i) : p.factor;
        const int64_t l = clamp3<int64_t>(levels[i], p.clip_min, p.clip_max);
        const int64_t v = clamp3<int64_t>((l * f + p.add) >> p.shift, p.clip_min, p.clip_max);
        out[i] = store((int32_t)v, i16s);
    }
}

// transform.rs:755-761 apply_transform_skip_shift, :778-792 and :810-826.
void dequant_ts(const int32_t* levels, int n, const orc_ts_params& t, const uint8_t* sc,
                int sc_dc, bool i16s, int32_t* out) {
    const orc_dequant_params& p = t.dq;
    const int64_t base = p.factor / 16;
    for (int i = 0; i < n * n; ++i) {
        const int64_t f = sc ? base * scaling_coeff(sc, sc_dc, n, i) : p.factor;
        const int64_t l = clamp3<int64_t>(levels[i], p.clip_min, p.clip_max);
        const int32_t deq =
            (int32_t)clamp3<int64_t>((l * f + p.add) >> p.shift, p.clip_min, p.clip_max);
        const int32_t r = t.tr_shift >= 0 ? (deq + t.tr_add) >> t.tr_shift
                                          : (int32_t)((uint32_t)deq << (-t.tr_shift));
        out[i] = store(r, i16s);
    }
}

// ---------------------------------------------------------------------------
// reconstruct.rs:214-251 add_residual_generic
// ---------------------------------------------------------------------------
inline int32_t sample_max(int bd) { return bd == 0 ? 0 : (bd <= 15 ? (1 << bd) - 1 : 65535); }

void add_residual(uint16_t* dst, int stride, const uint16_t* pred, const int32_t* res, int n,
                  int valid_w, int valid_h, int bd) {
    valid_w = std::min(std::min(valid_w, n), stride);
    valid_h = std::min(valid_h, n);
    const int32_t mx = sample_max(bd);
    for (int y = 0; y < valid_h; ++y)
        for (int x = 0; x < valid_w; ++x)
            dst[y * stride + x] = (uint16_t)clamp3(pred[y * n + x] + res[y * n + x], 0, mx);
}

// ---------------------------------------------------------------------------
// intra.rs
// ---------------------------------------------------------------------------
// intra.rs:30-38 (H.265 Tables 8-4 / 8-5)
const int32_t kIntraPredAngle[33] = {32,  26,  21,  17,  13,  9,  5,  2,  0,  -2, -5,
                                     -9,  -13, -17, -21, -26, -32, -26, -21, -17, -13, -9,
                                     -5,  -2,  0,   2,   5,   9,   13,  17,  21,  26,  32};
const int32_t kInvAngle[15] = {-4096, -1638, -910, -630, -482, -390, -315, -256,
                               -315,  -390,  -482, -630, -910, -1638, -4096};

// intra.rs:84-148 substitute_refs_into.  raw_* entries < 0 are unavailable.
void intra_substitute(const int32_t* raw_above, const int32_t* raw_left, int32_t raw_corner,
                      int n, int neutral, uint16_t* above_out, uint16_t* left_out) {
    const int total = 4 * n + 1;
    uint16_t s[4 * 32 + 1] = {0};
    bool avail[4 * 32 + 1] = {false};
    for (int i = 0; i < total; ++i) {
        s[i] = 0;
        avail[i] = false;
    }
    for (int i = 0; i < 2 * n; ++i) {
        const int32_t v = raw_left[2 * n - 1 - i];
        if (v >= 0) {
            s[i] = (uint16_t)v;
            avail[i] = true;
        }
    }
    if (raw_corner >= 0) {
        s[2 * n] = (uint16_t)raw_corner;
        avail[2 * n] = true;
    }
    for (int i = 0; i < 2 * n; ++i) {
        const int32_t v = raw_above[i];
        if (v >= 0) {
            s[2 * n + 1 + i] = (uint16_t)v;
            avail[2 * n + 1 + i] = true;
        }
    }
    int first = -1;
    for (int i = 0; i < total; ++i)
        if (avail[i]) {
            first = i;
            break;
        }
    if (first < 0) {
        for (int i = 0; i < total; ++i) s[i] = (uint16_t)neutral;
    } else {
        for (int i = 0; i < first; ++i) s[i] = s[first];
        for (int i = 1; i < total; ++i)
            if (!avail[i]) s[i] = s[i - 1];
    }
    above_out[0] = s[2 * n];
    left_out[0] = s[2 * n];
    for (int i = 0; i < 2 * n; ++i) {
        above_out[1 + i] = s[2 * n + 1 + i];
        left_out[1 + i] = s[2 * n - 1 - i];
    }
}

// intra.rs:151-219 filter_refs_into
void intra_filter(const uint16_t* above, const uint16_t* left, int n, int mode, bool is_luma,
                  bool smoothing, bool strong, int bd, uint16_t* fa, uint16_t* fl) {
    const int len = 2 * n + 1;
    std::memcpy(fa, above, sizeof(uint16_t) * len);
    std::memcpy(fl, left, sizeof(uint16_t) * len);
    if (!smoothing || !is_luma || n == 4 || mode == 1) return;
    const int min_dist = std::min(std::abs(mode - 26), std::abs(mode - 10));
    const int thresh = n == 8 ? 7 : (n == 16 ? 1 : (n == 32 ? 0 : 8));
    if (!(mode == 0 || min_dist > thresh)) return;
    if (strong && n == 32) {
        const int thr = 1 << (bd - 5);
        const int bl = left[2 * n], tl = above[0], tr = above[2 * n];
        const int cl = left[n], ct = above[n];
        if (std::abs(bl + tl - 2 * cl) < thr && std::abs(tr + tl - 2 * ct) < thr) {
            for (int i = 1; i < 2 * n; ++i) {
                fa[i] = (uint16_t)(((2 * n - i) * tl + i * tr + n) >> 6);
                fl[i] = (uint16_t)(((2 * n - i) * tl + i * bl + n) >> 6);
            }
            fa[0] = above[0];
            fl[0] = left[0];
            fa[2 * n] = above[2 * n];
            fl[2 * n] = left[2 * n];
            return;
        }
    }
    const int corner = above[0];
    fa[0] = (uint16_t)((left[1] + 2 * corner + above[1] + 2) >> 2);
    fl[0] = fa[0];
    for (int i = 1; i < 2 * n; ++i) {
        fa[i] = (uint16_t)((above[i - 1] + 2 * above[i] + above[i + 1] + 2) >> 2);
        fl[i] = (uint16_t)((left[i - 1] + 2 * left[i] + left[i + 1] + 2) >> 2);
    }
    fa[2 * n] = above[2 * n];
    fl[2 * n] = left[2 * n];
}

// intra.rs:257-372 predict_into_scalar
void intra_predict(int mode, const uint16_t* above, const uint16_t* left, int n, bool is_luma,
                   int bd, uint16_t* out) {
    int log2n = 0;
    while ((1 << log2n) < n) ++log2n;
    if (mode == 0) {  // PLANAR
        const int tr = above[n + 1], bl = left[n + 1];
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                const int h = (n - 1 - x) * left[y + 1] + (x + 1) * tr;
                const int v = (n - 1 - y) * above[x + 1] + (y + 1) * bl;
                out[y * n + x] = (uint16_t)((h + v + n) >> (log2n + 1));
            }
        return;
    }
    if (mode == 1) {  // DC
        int sum = 0;
        for (int i = 1; i <= n; ++i) sum += above[i] + left[i];
        const int dc = (sum + n) >> (log2n + 1);
        for (int i = 0; i < n * n; ++i) out[i] = (uint16_t)dc;
        if (is_luma && n < 32) {
            out[0] = (uint16_t)((left[1] + 2 * dc + above[1] + 2) >> 2);
            for (int x = 1; x < n; ++x) out[x] = (uint16_t)((above[x + 1] + 3 * dc + 2) >> 2);
            for (int y = 1; y < n; ++y) out[y * n] = (uint16_t)((left[y + 1] + 3 * dc + 2) >> 2);
        }
        return;
    }
    const int angle = kIntraPredAngle[mode - 2];
    const bool vertical = mode >= 18;
    const uint16_t* main_ref = vertical ? above : left;
    const uint16_t* side = vertical ? left : above;
    int32_t refs[3 * 32 + 1];
    const int base = n;
    for (int i = 0; i <= 2 * n; ++i) refs[n + i] = main_ref[i];
    if (angle < 0) {
        const int inv = kInvAngle[mode - 11];
        const int lim = (n * angle) >> 5;
        for (int k = -1; k >= lim; --k) {
            const int idx = std::min((k * inv + 128) >> 8, 2 * n);
            refs[k + base] = side[std::max(idx, 0)];
        }
    }
    const int max_v = std::max((1 << bd) - 1, 0);
    for (int a = 0; a < n; ++a) {      // a = row (vertical) or column (horizontal)
        const int pos = (a + 1) * angle;
        const int i_idx = pos >> 5;
        const int frac = pos & 31;
        for (int b = 0; b < n; ++b) {  // b = position along the main direction
            const int r0 = refs[b + i_idx + 1 + base];
            int v = r0;
            if (frac != 0) {
                const int r1 = refs[b + i_idx + 2 + base];
                v = ((32 - frac) * r0 + frac * r1 + 16) >> 5;
            }
            v = clamp3(v, 0, max_v);
            if (vertical)
                out[a * n + b] = (uint16_t)v;
            else
                out[b * n + a] = (uint16_t)v;
        }
    }
    if (is_luma && n < 32) {
        if (mode == 26) {
            for (int y = 0; y < n; ++y) {
                const int v = above[1] + ((left[y + 1] - above[0]) >> 1);
                out[y * n] = (uint16_t)clamp3(v, 0, max_v);
            }
        } else if (mode == 10) {
            for (int x = 0; x < n; ++x) {
                const int v = left[1] + ((above[x + 1] - above[0]) >> 1);
                out[x] = (uint16_t)clamp3(v, 0, max_v);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// mc.rs
// ---------------------------------------------------------------------------
// mc.rs:30-45 (H.265 Tables 8-11 / 8-12)
const int32_t kLumaFilter[4][8] = {{0, 0, 0, 64, 0, 0, 0, 0},
                                   {-1, 4, -10, 58, 17, -5, 1, 0},
                                   {-1, 4, -11, 40, 40, -11, 4, -1},
                                   {0, 1, -5, 17, 58, -10, 4, -1}};
const int32_t kChromaFilter[8][4] = {{0, 64, 0, 0},   {-2, 58, 10, -2}, {-4, 54, 16, -2},
                                     {-6, 46, 28, -4}, {-4, 36, 36, -4}, {-4, 28, 46, -6},
                                     {-2, 16, 54, -4}, {-2, 10, 58, -2}};

struct RefPlane {  // mc.rs:300-316 (edge-clamped sample fetch)
    const uint16_t* data;
    int stride, width, height;
    int sample(int x, int y) const {
        const int xc = clamp3(x, 0, width - 1), yc = clamp3(y, 0, height - 1);
        return data[yc * stride + xc];
    }
};

// mc.rs:351-439 (taps = 8) and :442-530 (taps = 4)
void interp(const RefPlane& r, int x0, int y0, int fx, int fy, int w, int h, int bd, int taps,
            const int32_t* hf, const int32_t* vf, int16_t* dst) {
    const int s1 = bd - 8;
    const int back = taps / 2 - 1;
    if (fx == 0 && fy == 0) {
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x)
                dst[y * w + x] = (int16_t)((r.sample(x0 + x, y0 + y) << 6) >> s1);
        return;
    }
    if (fy == 0) {
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                int acc = 0;
                for (int t = 0; t < taps; ++t) acc += hf[t] * r.sample(x0 + x - back + t, y0 + y);
                dst[y * w + x] = (int16_t)(acc >> s1);
            }
        return;
    }
    if (fx == 0) {
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                int acc = 0;
                for (int t = 0; t < taps; ++t) acc += vf[t] * r.sample(x0 + x, y0 + y - back + t);
                dst[y * w + x] = (int16_t)(acc >> s1);
            }
        return;
    }
    const int th = h + taps - 1;
    std::vector<int32_t> tmp((size_t)w * th);
    for (int ty = 0; ty < th; ++ty)
        for (int x = 0; x < w; ++x) {
            int acc = 0;
            for (int t = 0; t < taps; ++t)
                acc += hf[t] * r.sample(x0 + x - back + t, y0 + ty - back);
            tmp[(size_t)ty * w + x] = acc >> s1;
        }
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            int acc = 0;
            for (int t = 0; t < taps; ++t) acc += vf[t] * tmp[(size_t)(y + t) * w + x];
            dst[y * w + x] = (int16_t)(acc >> 6);
        }
}

// mc.rs:538-577
void uni_mc(const int16_t* src, int w, int h, int vw, int vh, int bd, uint16_t* dst, int stride) {
    (void)h;
    const int shift = 14 - bd;
    const int offset = shift > 0 ? 1 << (shift - 1) : 0;
    const int mx = sample_max(bd);
    for (int y = 0; y < vh; ++y)
        for (int x = 0; x < vw; ++x)
            dst[y * stride + x] = (uint16_t)clamp3((src[y * w + x] + offset) >> shift, 0, mx);
}

// mc.rs:579-629
void bi_mc(const int16_t* a, const int16_t* b, int w, int h, int vw, int vh, int bd,
           uint16_t* dst, int stride) {
    (void)h;
    const int shift = 15 - bd;
    const int offset = 1 << (shift - 1);
    const int mx = sample_max(bd);
    for (int y = 0; y < vh; ++y)
        for (int x = 0; x < vw; ++x)
            dst[y * stride + x] =
                (uint16_t)clamp3((a[y * w + x] + b[y * w + x] + offset) >> shift, 0, mx);
}

// mc.rs:631-680
void uni_mc_w(const int16_t* src, int w, int h, int vw, int vh, int bd, int wt, int off,
              int log2_denom, uint16_t* dst, int stride) {
    (void)h;
    const int log2_wd = log2_denom + 14 - bd;
    const int mx = sample_max(bd);
    const int round = log2_wd >= 1 ? 1 << (log2_wd - 1) : 0;
    for (int y = 0; y < vh; ++y)
        for (int x = 0; x < vw; ++x) {
            const int s = src[y * w + x];
            const int v = log2_wd >= 1 ? ((s * wt + round) >> log2_wd) + off : s * wt + off;
            dst[y * stride + x] = (uint16_t)clamp3(v, 0, mx);
        }
}

// mc.rs:682-736
void bi_mc_w(const int16_t* a, const int16_t* b, int w, int h, int vw, int vh, int bd, int w0,
             int o0, int w1, int o1, int log2_denom, uint16_t* dst, int stride) {
    (void)h;
    const int log2_wd = log2_denom + 14 - bd;
    const int mx = sample_max(bd);
    const int64_t rnd = ((int64_t)o0 + o1 + 1) << log2_wd;
    for (int y = 0; y < vh; ++y)
        for (int x = 0; x < vw; ++x) {
            const int64_t v =
                ((int64_t)a[y * w + x] * w0 + (int64_t)b[y * w + x] * w1 + rnd) >> (log2_wd + 1);
            dst[y * stride + x] = (uint16_t)clamp3<int64_t>(v, 0, mx);
        }
}

// ---------------------------------------------------------------------------
// decode.rs QP helpers (:5753-5770, :5868-5871, :7599-7613)
// ---------------------------------------------------------------------------
inline int qp_bd_offset(int bd) { return 6 * (bd - 8); }
inline int qp_prime(int qp, int bd) {
    const int off = qp_bd_offset(bd);
    return clamp3(qp + off, 0, 51 + off);
}
inline int qpc(int qpi, int idc, int bd) {
    qpi = clamp3(qpi, -qp_bd_offset(bd), 57);
    if (idc != 1) return std::min(qpi, 51);
    if (qpi < 30) return qpi;
    if (qpi > 43) return qpi - 6;
    static const int t[14] = {29, 30, 31, 32, 33, 33, 34, 34, 35, 35, 36, 36, 37, 37};
    return t[qpi - 30];
}
inline int clamp_qpy(int qp, int bd) { return clamp3(qp, -qp_bd_offset(bd), 51); }

// ---------------------------------------------------------------------------
// deblock.rs
// ---------------------------------------------------------------------------
// deblock.rs:34-50 (H.265 Table 8-12)
const int32_t kBeta[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  0,  6,  7,
                           8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18, 20, 22, 24, 26, 28, 30, 32,
                           34, 36, 38, 40, 42, 44, 46, 48, 50, 52, 54, 56, 58, 60, 62, 64};
const int32_t kTc[54] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,
                         1, 1, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2,  3,  3,  3,  3,  4,
                         4, 4, 5, 5, 6, 6, 7, 8, 9, 10, 11, 13, 14, 16, 18, 20, 22, 24};

struct Seg {  // flat index of (line, tap) for a vertical or horizontal edge
    uint16_t* p;
    int stride;
    bool vertical;
    int edge, scan;
    uint16_t& at(int line, int tap) const {
        return vertical ? p[(size_t)(scan + line) * stride + (edge + tap)]
                        : p[(size_t)(edge + tap) * stride + (scan + line)];
    }
    int g(int line, int tap) const { return at(line, tap); }
};

// deblock.rs:216-238 luma_decision: 0 skip, 1 strong, 2 weak (+ do_p1/do_q1)
int luma_decision(const Seg& s, int beta, int tc, bool* do_p1, bool* do_q1) {
    const int dp0 = std::abs(s.g(0, -3) - 2 * s.g(0, -2) + s.g(0, -1));
    const int dp3 = std::abs(s.g(3, -3) - 2 * s.g(3, -2) + s.g(3, -1));
    const int dq0 = std::abs(s.g(0, 2) - 2 * s.g(0, 1) + s.g(0, 0));
    const int dq3 = std::abs(s.g(3, 2) - 2 * s.g(3, 1) + s.g(3, 0));
    if (dp0 + dp3 + dq0 + dq3 >= beta) return 0;
    auto dsam = [&](int line, int dpq) {
        return 2 * dpq < (beta >> 2) &&
               std::abs(s.g(line, -4) - s.g(line, -1)) + std::abs(s.g(line, 0) - s.g(line, 3)) <
                   (beta >> 3) &&
               std::abs(s.g(line, -1) - s.g(line, 0)) < ((5 * tc + 1) >> 1);
    };
    if (dsam(0, dp0 + dq0) && dsam(3, dp3 + dq3)) return 1;
    const int side = (beta + (beta >> 1)) >> 3;
    *do_p1 = dp0 + dp3 < side;
    *do_q1 = dq0 + dq3 < side;
    return 2;
}

// deblock.rs:582-635 apply_luma_decision
void apply_luma(const Seg& s, int dec, bool do_p1, bool do_q1, int tc, int maxv) {
    if (dec == 0) return;
    const int tc2 = tc >> 1;
    for (int line = 0; line < 4; ++line) {
        const int p0 = s.g(line, -1), p1 = s.g(line, -2), p2 = s.g(line, -3), p3 = s.g(line, -4);
        const int q0 = s.g(line, 0), q1 = s.g(line, 1), q2 = s.g(line, 2), q3 = s.g(line, 3);
        if (dec == 1) {
            auto c = [&](int orig, int v) {
                return (uint16_t)clamp3(clamp3(v, orig - 2 * tc, orig + 2 * tc), 0, maxv);
            };
            s.at(line, -1) = c(p0, (p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3);
            s.at(line, -2) = c(p1, (p2 + p1 + p0 + q0 + 2) >> 2);
            s.at(line, -3) = c(p2, (2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3);
            s.at(line, 0) = c(q0, (p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3);
            s.at(line, 1) = c(q1, (p0 + q0 + q1 + q2 + 2) >> 2);
            s.at(line, 2) = c(q2, (p0 + q0 + q1 + 3 * q2 + 2 * q3 + 4) >> 3);
        } else {
            const int delta0 = (9 * (q0 - p0) - 3 * (q1 - p1) + 8) >> 4;
            if (std::abs(delta0) < tc * 10) {
                const int delta = clamp3(delta0, -tc, tc);
                s.at(line, -1) = (uint16_t)clamp3(p0 + delta, 0, maxv);
                s.at(line, 0) = (uint16_t)clamp3(q0 - delta, 0, maxv);
                if (do_p1) {
                    const int dp1 = clamp3((((p2 + p0 + 1) >> 1) - p1 + delta) >> 1, -tc2, tc2);
                    s.at(line, -2) = (uint16_t)clamp3(p1 + dp1, 0, maxv);
                }
                if (do_q1) {
                    const int dq1 = clamp3((((q2 + q0 + 1) >> 1) - q1 - delta) >> 1, -tc2, tc2);
                    s.at(line, 1) = (uint16_t)clamp3(q1 + dq1, 0, maxv);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// sao.rs
// ---------------------------------------------------------------------------
// sao.rs:205-233 (band offset, reads src writes dst)
void sao_band(uint16_t* dst, const uint16_t* src, int w, int x0, int y0, int x_end, int y_end,
              const int32_t* off, int band_pos, int bd) {
    const int mx = (1 << bd) - 1;
    const int shift = bd - 5;
    for (int y = y0; y < y_end; ++y)
        for (int x = x0; x < x_end; ++x) {
            const int s = src[(size_t)y * w + x];
            const uint8_t band = (uint8_t)(s >> shift);
            const uint8_t rel = (uint8_t)(band - (uint8_t)band_pos);
            if (rel < 4) dst[(size_t)y * w + x] = (uint16_t)clamp3(s + off[rel], 0, mx);
        }
}

// sao.rs:266-330 (edge offset, picture-border samples untouched)
// `nb_ok(x, y, nx, ny)`: neighbour (nx, ny) may be used for the sample at
// (x, y) (sao.rs:433-497 apply_sao_edge_offset_gated; always true without
// restricted boundaries).
template <typename NbOk>
void sao_edge(uint16_t* dst, const uint16_t* src, int w, int h, int x0, int y0, int x_end,
              int y_end, const int32_t* off, int eo_class, int bd, NbOk nb_ok) {
    const int mx = (1 << bd) - 1;
    int dx, dy;
    switch (eo_class) {
        case 0: dx = 1; dy = 0; break;
        case 1: dx = 0; dy = 1; break;
        case 2: dx = 1; dy = 1; break;
        default: dx = 1; dy = -1; break;
    }
    for (int y = y0; y < y_end; ++y)
        for (int x = x0; x < x_end; ++x) {
            const int s = src[(size_t)y * w + x];
            const int x1 = x + dx, y1 = y + dy, x2 = x - dx, y2 = y - dy;
            if (x1 < 0 || y1 < 0 || x1 >= w || y1 >= h) continue;
            if (x2 < 0 || y2 < 0 || x2 >= w || y2 >= h) continue;
            if (!nb_ok(x, y, x1, y1) || !nb_ok(x, y, x2, y2)) continue;
            const int n1 = src[(size_t)y1 * w + x1], n2 = src[(size_t)y2 * w + x2];
            const int e = ((s > n1) - (s < n1)) + ((s > n2) - (s < n2)) + 2;
            int o = 0;
            switch (e) {
                case 0: o = off[0]; break;
                case 1: o = off[1]; break;
                case 3: o = off[2]; break;
                case 4: o = off[3]; break;
                default: break;
            }
            if (o != 0) dst[(size_t)y * w + x] = (uint16_t)clamp3(s + o, 0, mx);
        }
}

// ---------------------------------------------------------------------------
// yuv.rs:187-393 Cvt (Q13 fixed point)
// ---------------------------------------------------------------------------
void yuv_to_rgb16(const uint16_t* Y, const uint16_t* Cb, const uint16_t* Cr, int width,
                  int height, int idc, int bd, int dw, int dh, int crop_left, int crop_top,
                  int matrix, bool full_range, uint16_t* out) {
    const int64_t Q13 = 13, ONE = 1 << 13, ROUND = 1 << 12;
    const int64_t scale = (int64_t)1 << (bd - 8);
    const int64_t k_y = full_range ? ONE : 9539;
    const int64_t k_uv = full_range ? ONE : 9326;
    int64_t cr_r0, cb_g0, cr_g0, cb_b0;
    switch (matrix) {
        case HPVCD_MATRIX_BT470BG:
        case HPVCD_MATRIX_SMPTE170M: cr_r0 = 11485; cb_g0 = -2819; cr_g0 = -5851; cb_b0 = 14516; break;
        case HPVCD_MATRIX_BT2020NCL: cr_r0 = 12080; cb_g0 = -1348; cr_g0 = -4681; cb_b0 = 17546; break;
        case HPVCD_MATRIX_IDENTITY: cr_r0 = cb_g0 = cr_g0 = cb_b0 = 0; break;
        default: cr_r0 = 12901; cb_g0 = -1534; cr_g0 = -3835; cb_b0 = 15201; break;  // BT.709
    }
    const int64_t max_val = (1 << bd) - 1;
    const int64_t cmax = bd == 8 ? 255 : max_val;
    const int64_t y_black = full_range ? 0 : 16 * scale;
    const int64_t c_black = full_range ? 0 : 16 * scale;
    const int64_t neutral = 128 * scale;
    const int64_t cr_to_r = (cr_r0 * k_uv + ROUND) >> Q13;
    const int64_t cb_to_g = (cb_g0 * k_uv + ROUND) >> Q13;
    const int64_t cr_to_g = (cr_g0 * k_uv + ROUND) >> Q13;
    const int64_t cb_to_b = (cb_b0 * k_uv + ROUND) >> Q13;
    const int sub_w = idc == 1 || idc == 2 ? 2 : 1, sub_h = idc == 1 ? 2 : 1;
    const int cw = (width + sub_w - 1) / sub_w, ch = (height + sub_h - 1) / sub_h;
    crop_left = std::min(crop_left, width - 1);
    crop_top = std::min(crop_top, height - 1);
    for (int yy = 0; yy < dh; ++yy)
        for (int xx = 0; xx < dw; ++xx) {
            const int src_y = crop_top + yy, src_x = crop_left + xx;
            const int y_row = std::min(src_y, height - 1);
            const int x_col = std::min(src_x, width - 1);
            const int64_t luma = Y[(size_t)y_row * width + x_col];
            uint16_t* o = out + ((size_t)yy * dw + xx) * 3;
            if (idc == 0) {  // yuv.rs:327 mono_rows (replicated by rgb8 narrowing)
                const int64_t v = clamp3<int64_t>((k_y * (luma - y_black) + ROUND) >> Q13, 0, cmax);
                o[0] = o[1] = o[2] = (uint16_t)v;
                continue;
            }
            const int c_row = std::min(src_y / sub_h, ch - 1);
            const int c_col = std::min(src_x / sub_w, cw - 1);
            const int64_t cb = Cb[(size_t)c_row * cw + c_col];
            const int64_t cr = Cr[(size_t)c_row * cw + c_col];
            int64_t r, g, b;
            if (matrix == HPVCD_MATRIX_IDENTITY) {  // yuv.rs:296 gbr_rows
                if (full_range) {
                    r = cr; g = luma; b = cb;
                } else {
                    r = (k_uv * (cr - c_black) + ROUND) >> Q13;
                    g = (k_y * (luma - y_black) + ROUND) >> Q13;
                    b = (k_uv * (cb - c_black) + ROUND) >> Q13;
                }
            } else if (matrix == HPVCD_MATRIX_YCGCO) {  // yuv.rs:368 ycgco_rows
                const int64_t cg = cb - neutral, co = cr - neutral, t = luma - cg;
                r = t + co; g = luma + cg; b = t - co;
            } else {  // yuv.rs:232 pixel / :327 fast_rows
                const int64_t yv = k_y * (luma - y_black);
                const int64_t cbc = cb - neutral, crc = cr - neutral;
                r = (yv + cr_to_r * crc + ROUND) >> Q13;
                g = (yv + cb_to_g * cbc + cr_to_g * crc + ROUND) >> Q13;
                b = (yv + cb_to_b * cbc + ROUND) >> Q13;
            }
            o[0] = (uint16_t)clamp3<int64_t>(r, 0, cmax);
            o[1] = (uint16_t)clamp3<int64_t>(g, 0, cmax);
            o[2] = (uint16_t)clamp3<int64_t>(b, 0, cmax);
        }
}

// ---------------------------------------------------------------------------
// Kernel set of a decode (exec.rs:31-77 ExecContext: the reference calls its
// per-block kernels through a table of function pointers, the SIMD set
// picked by CPU feature, avx/mod.rs).  The scalar set is the restatement
// above; the AVX2 set (cpu_simd.cpp) computes the same integers and serves
// the timed CPU reference arm.  Per thread: a banded decode sets it in every
// job it runs.
// ---------------------------------------------------------------------------
struct Kernels {
    void (*inv_dct)(const int32_t*, int, int, int, int, bool, int32_t*);
    void (*add_residual)(uint16_t*, int, const uint16_t*, const int32_t*, int, int, int, int);
    void (*intra_predict)(int, const uint16_t*, const uint16_t*, int, bool, int, uint16_t*);
    void (*sao_band)(uint16_t*, const uint16_t*, int, int, int, int, int, const int32_t*, int, int);
    // edge offset without slice / tile restriction (NULL: the scalar template)
    void (*sao_edge)(uint16_t*, const uint16_t*, int, int, int, int, int, int, const int32_t*, int, int);
    bool simd_rgb;
};

void inv_dct_avx2(const int32_t* coeff, int n, int bd, int max_range, int nx, bool i16s, int32_t* out) {
    if ((n == 16 || n == 32) && max_range == 15)
        orc_simd::inv_dct(coeff, n, bd, nx, i16s, out);
    else
        inv_dct(coeff, n, bd, max_range, nx, i16s, out);
}

const Kernels kScalarKernels{inv_dct, add_residual, intra_predict, sao_band, nullptr, false};
const Kernels kAvx2Kernels{inv_dct_avx2, orc_simd::add_residual, orc_simd::intra_predict, orc_simd::sao_band,
                           orc_simd::sao_edge, true};
thread_local const Kernels* tk = &kScalarKernels;

// ---------------------------------------------------------------------------
// Picture-level state
// ---------------------------------------------------------------------------
struct Geo {
    int w, h, idc, sub_w, sub_h, cw, ch, gw, gh, bd, bd_c, log2_ctb, ctb_cols, ctb_rows;
};

Geo geo_of(const hpvcd_picture* p) {
    Geo g;
    g.w = (int)p->width;
    g.h = (int)p->height;
    g.idc = p->chroma_idc;
    g.sub_w = g.idc == 1 || g.idc == 2 ? 2 : 1;  // SubWidthC
    g.sub_h = g.idc == 1 ? 2 : 1;                  // SubHeightC
    g.cw = g.idc == 0 ? 0 : (g.w + g.sub_w - 1) / g.sub_w;
    g.ch = g.idc == 0 ? 0 : (g.h + g.sub_h - 1) / g.sub_h;
    g.gw = (g.w + 3) / 4;
    g.gh = (g.h + 3) / 4;
    g.bd = p->bit_depth_y;
    g.bd_c = p->bit_depth_c;
    g.log2_ctb = p->log2_ctb;
    const int ctb = 1 << g.log2_ctb;
    g.ctb_cols = (g.w + ctb - 1) / ctb;
    g.ctb_rows = (g.h + ctb - 1) / ctb;
    return g;
}

int validate(const hpvcd_picture* p) {
    if (!p) return HPVCD_ERR_INVALID_ARG;
    if (p->width == 0 || p->height == 0 || p->width > 16384 || p->height > 16384)
        return HPVCD_ERR_LIMIT;
    if (p->chroma_idc > 3) return HPVCD_ERR_UNSUPPORTED;
    if (p->bit_depth_y < 8 || p->bit_depth_y > 12 || p->bit_depth_c < 8 || p->bit_depth_c > 12)
        return HPVCD_ERR_UNSUPPORTED;
    if (p->log2_ctb < 4 || p->log2_ctb > 6) return HPVCD_ERR_BITSTREAM;
    if ((p->flags & HPVCD_PIC_CONSTRAINED_INTRA) && !p->cells) return HPVCD_ERR_INVALID_ARG;
    return HPVCD_OK;
}

struct PicState {
    const hpvcd_picture* pic;
    Geo g;
    orc_planes pl;
    std::vector<uint8_t> decoded;  // decode.rs `decoded` map, per 4x4 luma cell
    int cur_region = 0;            // slice / tile of the TB being predicted

    int region_at(int x, int y) const {  // luma position -> slice << 8 | tile
        const hpvcd_picture* p = pic;
        if (!p->ctb_region) return 0;
        return p->ctb_region[(size_t)(y >> g.log2_ctb) * g.ctb_cols + (x >> g.log2_ctb)];
    }
    bool constrained_ok(int x, int y) const {  // decode.rs:4641-4649
        if (!(pic->flags & HPVCD_PIC_CONSTRAINED_INTRA)) return true;
        return !(pic->cells[(size_t)(y / 4) * g.gw + x / 4].flags & HPVCD_CELL_INTER);
    }
    bool luma_avail(int x, int y) const {  // decode.rs:4651-4668 (same tile, same slice, decoded)
        if (x < 0 || y < 0 || x >= g.w || y >= g.h) return false;
        if (region_at(x, y) != cur_region) return false;
        if (!constrained_ok(x, y)) return false;
        return decoded[(size_t)(y / 4) * g.gw + x / 4] != 0;
    }
    bool chroma_avail(int cx, int cy) const {  // decode.rs:4669-4690
        if (cx < 0 || cy < 0 || cx >= g.cw || cy >= g.ch) return false;
        const int lx = cx * g.sub_w, ly = cy * g.sub_h;
        if (lx >= g.w || ly >= g.h) return false;
        if (region_at(lx, ly) != cur_region) return false;
        if (!constrained_ok(lx, ly)) return false;
        return decoded[(size_t)(ly / 4) * g.gw + lx / 4] != 0;
    }
    void mark_decoded(int x0, int y0, int n) {  // decode.rs:3170-3189
        for (int y = y0; y < std::min(y0 + n, g.h); y += 4)
            for (int x = x0; x < std::min(x0 + n, g.w); x += 4)
                decoded[(size_t)(y / 4) * g.gw + x / 4] = 1;
    }
};

// decode.rs:4693-4722 gather + :4956-5004 predict_luma_block_into, and the
// chroma counterparts :5176-5278.
void predict_block(const PicState& st, int comp, int x0, int y0, int n, int mode,
                   uint16_t* pred) {
    const hpvcd_picture* p = st.pic;
    const Geo& g = st.g;
    const bool luma = comp == 0;
    const uint16_t* plane = comp == 0 ? st.pl.y : (comp == 1 ? st.pl.cb : st.pl.cr);
    const int stride = luma ? g.w : g.cw;
    auto avail = [&](int x, int y) { return luma ? st.luma_avail(x, y) : st.chroma_avail(x, y); };
    int32_t raw_above[64], raw_left[64];
    const int32_t corner = avail(x0 - 1, y0 - 1) ? plane[(size_t)(y0 - 1) * stride + x0 - 1] : -1;
    for (int i = 0; i < 2 * n; ++i) {
        raw_above[i] = avail(x0 + i, y0 - 1) ? plane[(size_t)(y0 - 1) * stride + x0 + i] : -1;
        raw_left[i] = avail(x0 - 1, y0 + i) ? plane[(size_t)(y0 + i) * stride + x0 - 1] : -1;
    }
    const int bd = luma ? g.bd : g.bd_c;
    const int neutral = 1 << (bd - 1);
    uint16_t above[65], left[65], fa[65], fl[65];
    intra_substitute(raw_above, raw_left, corner, n, neutral, above, left);
    const bool smoothing = !(p->flags & HPVCD_PIC_SMOOTHING_DISABLED);
    if (luma) {
        const bool strong = (p->flags & HPVCD_PIC_STRONG_SMOOTHING) != 0;
        intra_filter(above, left, n, mode, true, smoothing, strong, bd, fa, fl);
        tk->intra_predict(mode, fa, fl, n, true, bd, pred);
    } else if (g.idc == 3) {
        intra_filter(above, left, n, mode, true, smoothing, false, bd, fa, fl);
        tk->intra_predict(mode, fa, fl, n, false, bd, pred);
    } else {
        tk->intra_predict(mode, above, left, n, false, bd, pred);
    }
}

// decode.rs:4441-4500 load_plane_block_clipped
void load_block_clipped(const uint16_t* plane, int stride, int width, int height, int x0, int y0,
                        int n, uint16_t* pred) {
    const int vw = std::min(std::max(width - x0, 0), n), vh = std::min(std::max(height - y0, 0), n);
    for (int i = 0; i < n * n; ++i) pred[i] = 0;
    for (int y = 0; y < vh; ++y)
        for (int x = 0; x < vw; ++x) pred[y * n + x] = plane[(size_t)(y0 + y) * stride + x0 + x];
}

// decode.rs:5874-5899 scaling_matrix_from_lists: the list of this size,
// component and prediction mode ([intra Y, Cb, Cr, inter Y, Cb, Cr]); none
// (flat) without lists and for transform skip above 4x4.
const uint8_t* scaling_select(const hpvcd_scaling* s, int comp, int n, bool inter, bool tskip, int* dc) {
    if (!s || (tskip && n != 4)) return nullptr;
    int size_id = 0;
    while ((4 << size_id) < n) ++size_id;
    size_id = std::min(size_id, 3);
    const int matrix_id = std::min(comp, 2) + (inter ? 3 : 0);
    *dc = s->dc[size_id][matrix_id];
    return s->m[size_id][matrix_id];
}

// decode.rs:8418-8446 apply_rext_residual_ops: reverse the block, then
// accumulate down the columns (dir 1) or along the rows (dir 0).  With i16
// storage the reference adds in i16, wrapping (release arithmetic).
void rext_residual_ops(int32_t* res, int n, bool rotate, int dir, bool i16s) {
    if (rotate)
        for (int i = 0; i < n * n / 2; ++i) std::swap(res[i], res[n * n - 1 - i]);
    auto add = [i16s](int32_t a, int32_t b) -> int32_t {
        return i16s ? (int32_t)(int16_t)(uint16_t)((uint32_t)a + (uint32_t)b) : a + b;
    };
    if (dir == 1) {
        for (int y = 1; y < n; ++y)
            for (int x = 0; x < n; ++x) res[y * n + x] = add(res[y * n + x], res[(y - 1) * n + x]);
    } else if (dir == 0) {
        for (int y = 0; y < n; ++y)
            for (int x = 1; x < n; ++x) res[y * n + x] = add(res[y * n + x], res[y * n + x - 1]);
    }
}

int rdpcm_dir(const hpvcd_tu& t) {
    return (t.flags & HPVCD_TU_RDPCM_V) ? 1 : ((t.flags & HPVCD_TU_RDPCM_H) ? 0 : -1);
}

// Residual of one TB: decode.rs:4754-4802 (8-bit i16 path) and :4835-4903
// (i32 path) for luma, :5313-5417 for chroma.
// `allow16` false: i32 storage at 8 bits (chroma TBs with cross-component
// prediction, decode.rs:5313-5316).
void tb_residual(const hpvcd_picture* p, const Geo& g, const hpvcd_tu& t, int32_t* res, bool allow16 = true) {
    const int n = 1 << t.log2n;
    const bool luma = t.comp == 0;
    const int bd = luma ? g.bd : g.bd_c;
    const bool i16s = bd <= 8 && allow16;
    int32_t lv[32 * 32];
    // the pool holds int16 levels, or int8 ones when the host narrowed it
    // (HPVCD_PIC_COEFF8: a transport format only, the levels are the same)
    const bool c8 = (p->flags & HPVCD_PIC_COEFF8) != 0;
    for (int i = 0; i < n * n; ++i)
        lv[i] = c8 ? ((const int8_t*)p->coeffs)[(size_t)t.coeff_off + i] : p->coeffs[(size_t)t.coeff_off + i];
    if (t.flags & (HPVCD_TU_TQB | HPVCD_TU_PCM)) {  // lossless / I_PCM: levels verbatim (saturated for i16 storage)
        for (int i = 0; i < n * n; ++i) res[i] = i16s ? clamp3(lv[i], -32768, 32767) : lv[i];
        rext_residual_ops(res, n, (t.flags & HPVCD_TU_ROTATE) != 0, rdpcm_dir(t), i16s);
        return;
    }
    int qpp;
    if (luma) {
        qpp = qp_prime(t.qp_y, bd);
    } else {
        const int pps_off = t.comp == 1 ? p->pps_cb_qp_offset : p->pps_cr_qp_offset;
        qpp = qp_prime(qpc(t.qp_y + pps_off + t.cqp_off, g.idc, bd), bd);
    }
    int sc_dc = 16;
    const uint8_t* sc = scaling_select(p->scaling, t.comp, n, !(t.flags & HPVCD_TU_INTRA),
                                       (t.flags & HPVCD_TU_TSKIP) != 0, &sc_dc);
    if (t.flags & HPVCD_TU_TSKIP) {
        const orc_ts_params tp = ts_params(n, qpp, bd, false);
        dequant_ts(lv, n, tp, sc, sc_dc, i16s, res);
        rext_residual_ops(res, n, (t.flags & HPVCD_TU_ROTATE) != 0, rdpcm_dir(t), i16s);
        return;
    }
    int32_t deq[32 * 32];
    dequant(lv, n, dequant_params(n, qpp, bd, false), sc, sc_dc, i16s, deq);
    if (luma && n == 4 && (t.flags & HPVCD_TU_INTRA))
        inv_dst4(deq, bd, 15, i16s, res);
    else
        tk->inv_dct(deq, n, bd, 15, t.nx ? t.nx : n, i16s, res);
}

int recon_picture(const hpvcd_picture* p, orc_planes* pl) {
    int rc = validate(p);
    if (rc) return rc;
    PicState st;
    st.pic = p;
    st.g = geo_of(p);
    st.pl = *pl;
    st.decoded.assign((size_t)st.g.gw * st.g.gh, 0);
    const Geo& g = st.g;
    const bool pred_in_plane = (p->flags & HPVCD_PIC_PRED_IN_PLANE) != 0;
    uint16_t pred[64 * 64];
    int32_t res[32 * 32];
    int32_t cc_luma[32 * 32];  // decode.rs:279 cross_comp_luma: the last coded luma residual
    const bool ccp_pic = (p->flags & HPVCD_PIC_CROSS_COMPONENT) != 0;
    for (uint32_t i = 0; i < p->n_tus; ++i) {
        const hpvcd_tu& t = p->tus[i];
        const int n = 1 << t.log2n;
        if (t.comp > 2 || (t.comp > 0 && g.idc == 0)) return HPVCD_ERR_BITSTREAM;
        const bool ccp = ccp_pic && t.comp > 0 && t.res_scale != 0;
        const bool coded = (t.flags & HPVCD_TU_CBF) != 0;
        const bool intra = (t.flags & HPVCD_TU_INTRA) != 0;
        if (t.log2n < 2 || t.log2n > 6 || ((coded || ccp) && t.log2n > 5)) return HPVCD_ERR_BITSTREAM;
        if (coded && (uint64_t)t.coeff_off + (uint64_t)n * n > p->n_coeffs) return HPVCD_ERR_BITSTREAM;
        if (ccp) {  // the TU's coded luma TB is among the three records before
            bool found = false;
            for (uint32_t k = 1; k <= 3 && k <= i && !found; ++k) {
                const hpvcd_tu& l = p->tus[i - k];
                found = l.comp == 0 && l.x == t.x && l.y == t.y && l.log2n == t.log2n &&
                        (l.flags & HPVCD_TU_CBF);
            }
            if (!found || g.idc != 3) return HPVCD_ERR_BITSTREAM;
        }
        const bool luma = t.comp == 0;
        uint16_t* plane = luma ? pl->y : (t.comp == 1 ? pl->cb : pl->cr);
        const int pw = luma ? g.w : g.cw, ph = luma ? g.h : g.ch;
        const int bd = luma ? g.bd : g.bd_c;
        if (!coded && !intra && !ccp) {  // end of an inter CU / residual-free inter TB
            if (luma) st.mark_decoded(t.x, t.y, n);
            continue;
        }
        if (t.flags & HPVCD_TU_PCM) {  // decode.rs:2768-2839: the samples replace the block
            for (int k = 0; k < n * n; ++k) pred[k] = 0;
        } else if (intra && !pred_in_plane) {
            st.cur_region = luma ? st.region_at(t.x, t.y) : st.region_at(t.x * g.sub_w, t.y * g.sub_h);
            predict_block(st, t.comp, t.x, t.y, n, t.mode, pred);
        }
        else
            load_block_clipped(plane, pw, pw, ph, t.x, t.y, n, pred);
        const int vw = std::min(std::max(pw - (int)t.x, 0), n);
        const int vh = std::min(std::max(ph - (int)t.y, 0), n);
        if (coded) {
            tb_residual(p, g, t, res, !ccp);
        } else {
            for (int k = 0; k < n * n; ++k) res[k] = 0;  // predict_only: copy (add zero)
        }
        if (ccp_pic && t.comp == 0 && coded)
            for (int k = 0; k < n * n; ++k) cc_luma[k] = res[k];
        if (ccp) {  // decode.rs:5488-5504 apply_cross_comp_residual
            for (int k = 0; k < n * n; ++k) {
                const int64_t sy = ((int64_t)cc_luma[k] << g.bd_c) >> g.bd;
                const int64_t v = (int64_t)res[k] + ((t.res_scale * sy) >> 3);
                res[k] = (int32_t)clamp3<int64_t>(v, INT32_MIN, INT32_MAX);
            }
        }
        if (vw > 0 && vh > 0)
            tk->add_residual(plane + (size_t)t.y * pw + t.x, pw, pred, res, n, vw, vh, bd);
        if (luma) st.mark_decoded(t.x, t.y, n);
    }
    return HPVCD_OK;
}

int mc_picture(const hpvcd_picture* p, const orc_planes* refs, int n_refs, orc_planes* pl) {
    int rc = validate(p);
    if (rc) return rc;
    const Geo g = geo_of(p);
    std::vector<int16_t> p0, p1;
    for (uint32_t i = 0; i < p->n_pus; ++i) {
        const hpvcd_pu& u = p->pus[i];
        const int x0 = u.x, y0 = u.y, w = u.w, h = u.h;
        const orc_planes* r[2] = {nullptr, nullptr};
        for (int l = 0; l < 2; ++l) {
            if (!(u.flags & (l ? HPVCD_PU_L1 : HPVCD_PU_L0))) continue;
            if (u.ref_idx[l] < 0 || u.ref_idx[l] >= HPVCD_MAX_REFS) return HPVCD_ERR_BITSTREAM;
            const int slot = p->ref_slot[l][u.ref_idx[l]];
            if (slot >= 0 && slot < n_refs) r[l] = &refs[slot];
        }
        const hpvcd_wp_table* wt = p->wp;
        for (int c = 0; c < (g.idc ? 3 : 1); ++c) {
            const bool luma = c == 0;
            const int sw = luma ? 1 : g.sub_w, sh = luma ? 1 : g.sub_h;
            const int bw = w / sw, bh = h / sh;
            if (bw * bh == 0) continue;
            const int bx = x0 / sw, by = y0 / sh;
            const int pw = luma ? g.w : g.cw, ph = luma ? g.h : g.ch;
            const int bd = luma ? g.bd : g.bd_c;
            p0.assign((size_t)bw * bh, 0);
            p1.assign((size_t)bw * bh, 0);
            bool have[2] = {false, false};
            for (int l = 0; l < 2; ++l) {
                if (!r[l]) continue;
                const uint16_t* data = luma ? r[l]->y : (c == 1 ? r[l]->cb : r[l]->cr);
                RefPlane rp{data, pw, pw, ph};
                int16_t* dst = l ? p1.data() : p0.data();
                if (luma) {  // decode.rs:7063-7071
                    const int ix = x0 + (u.mv[l][0] >> 2), iy = y0 + (u.mv[l][1] >> 2);
                    const int fx = u.mv[l][0] & 3, fy = u.mv[l][1] & 3;
                    interp(rp, ix, iy, fx, fy, bw, bh, bd, 8, kLumaFilter[fx], kLumaFilter[fy], dst);
                } else {  // decode.rs:7282-7287 (Rust `/` truncates toward zero)
                    const int mvcx = u.mv[l][0] * 2 / g.sub_w, mvcy = u.mv[l][1] * 2 / g.sub_h;
                    const int ix = bx + (mvcx >> 3), iy = by + (mvcy >> 3);
                    const int fx = mvcx & 7, fy = mvcy & 7;
                    interp(rp, ix, iy, fx, fy, bw, bh, bd, 4, kChromaFilter[fx], kChromaFilter[fy],
                           dst);
                }
                have[l] = true;
            }
            if (bx >= pw || by >= ph) continue;
            const int vw = std::min(bw, pw - bx), vh = std::min(bh, ph - by);
            uint16_t* plane = luma ? pl->y : (c == 1 ? pl->cb : pl->cr);
            uint16_t* dst = plane + (size_t)by * pw + bx;
            auto wpair = [&](int l, int* wgt, int* off) {
                const hpvcd_wp_entry& e = wt->e[l][std::max<int>(u.ref_idx[l], 0)];
                *wgt = luma ? e.luma_w : (c == 1 ? e.cb_w : e.cr_w);
                *off = luma ? e.luma_o : (c == 1 ? e.cb_o : e.cr_o);
            };
            const int denom = wt ? (luma ? wt->luma_log2_denom : wt->chroma_log2_denom) : 0;
            if (have[0] && have[1]) {
                if (wt) {
                    int w0, o0, w1, o1;
                    wpair(0, &w0, &o0);
                    wpair(1, &w1, &o1);
                    bi_mc_w(p0.data(), p1.data(), bw, bh, vw, vh, bd, w0, o0, w1, o1, denom, dst, pw);
                } else {
                    bi_mc(p0.data(), p1.data(), bw, bh, vw, vh, bd, dst, pw);
                }
            } else if (have[0] || have[1]) {
                const int l = have[0] ? 0 : 1;
                const int16_t* src = l ? p1.data() : p0.data();
                if (wt) {
                    int wg, of;
                    wpair(l, &wg, &of);
                    uni_mc_w(src, bw, bh, vw, vh, bd, wg, of, denom, dst, pw);
                } else {
                    uni_mc(src, bw, bh, vw, vh, bd, dst, pw);
                }
            } else {  // decode.rs:7206-7216 missing reference -> mid-grey
                for (int yy = 0; yy < vh; ++yy)
                    for (int xx = 0; xx < vw; ++xx) dst[(size_t)yy * pw + xx] = (uint16_t)(1 << (bd - 1));
            }
        }
    }
    return HPVCD_OK;
}

// slice_deblocking_filter_disabled_flag per slice index (decode.rs:1762
// SliceDeblock.disabled; slice 0 stands for the picture when it has no
// slice map).  The flat buffers carry no such flag: a host folds it into the
// boundary strengths.  The oracle keeps the reference's own test so that the
// fold can be checked against it; orc_set_disabled_slices sets it.
static uint8_t g_slice_disabled[256];
static bool g_any_slice_disabled = false;

// decode.rs:1774-2146 apply_deblocking (single slice, PPS-level parameters):
// luma vertical, luma horizontal, chroma vertical, chroma horizontal, in
// that order.  Within a pass the segments of different CTB-row bands touch
// disjoint rows (a vertical segment its own 4 rows; a horizontal edge e rows
// e - 4 .. e + 3 of band [r0 - 4, r1 - 4)), so `run(count, body)` may run a
// pass's bands in any order or at once: serially for apply_deblocking, on
// the pool for the reference's banded driver (deblock.rs:1118
// apply_deblocking_parallel).  Exempt samples are restored band by band.
template <class Run>
int deblock_picture_t(const hpvcd_picture* p, orc_planes* pl, Run run) {
    int rc = validate(p);
    if (rc) return rc;
    if (!(p->flags & HPVCD_PIC_DEBLOCK) || !p->cells) return HPVCD_OK;
    const Geo g = geo_of(p);
    const hpvcd_cell* cells = p->cells;
    const int bd_shift = g.bd - 8, bd_shift_c = g.bd_c - 8;
    // decode.rs:1762 slice_deblock_at: the offsets of the slice holding the
    // q sample, else the picture's
    auto offsets_at = [&](int qx, int qy, int* beta_offset, int* tc_offset) {
        int b = p->beta_offset_div2, t = p->tc_offset_div2;
        if (p->slice_deblock && p->ctb_region) {
            const int s = p->ctb_region[(size_t)(qy >> g.log2_ctb) * g.ctb_cols + (qx >> g.log2_ctb)] >> 8;
            b = p->slice_deblock[2 * s];
            t = p->slice_deblock[2 * s + 1];
        }
        *beta_offset = 2 * b;
        *tc_offset = 2 * t;
    };
    // decode.rs:1934, :1979, :2060: a segment whose q sample lies in a slice
    // with deblocking disabled is skipped
    auto disabled_at = [&](int qx, int qy) {
        if (!g_any_slice_disabled) return false;
        const int s = p->ctb_region ? p->ctb_region[(size_t)(qy >> g.log2_ctb) * g.ctb_cols + (qx >> g.log2_ctb)] >> 8 : 0;
        return g_slice_disabled[s] != 0;
    };
    auto qp_at = [&](int px, int py) {
        const int gx = std::min(px / 4, g.gw - 1), gy = std::min(py / 4, g.gh - 1);
        return (int)cells[(size_t)gy * g.gw + gx].qp_y;
    };
    auto bs_v = [&](int px, int py) -> int {  // decode.rs:1660-1676
        if (px == 0 || px >= g.w || py >= g.h) return 0;
        return cells[(size_t)(py / 4) * g.gw + px / 4].bs_v;
    };
    auto bs_h = [&](int px, int py) -> int {  // decode.rs:1679-1694
        if (py == 0 || px >= g.w || py >= g.h) return 0;
        return cells[(size_t)(py / 4) * g.gw + px / 4].bs_h;
    };
    bool any_exempt = false;
    for (size_t i = 0; i < (size_t)g.gw * g.gh; ++i) any_exempt |= (cells[i].flags & HPVCD_CELL_EXEMPT) != 0;
    std::vector<uint16_t> sy, scb, scr;
    if (any_exempt) {
        sy.assign(pl->y, pl->y + (size_t)g.w * g.h);
        if (g.idc) {
            scb.assign(pl->cb, pl->cb + (size_t)g.cw * g.ch);
            scr.assign(pl->cr, pl->cr + (size_t)g.cw * g.ch);
        }
    }
    auto exempt = [&](int lx, int ly) {
        return (cells[(size_t)(ly / 4) * g.gw + lx / 4].flags & HPVCD_CELL_EXEMPT) != 0;
    };
    auto restore_luma = [&](int y0, int y1) {
        for (int y = std::max(y0, 0); y < std::min(y1, g.h); ++y)
            for (int x = 0; x < g.w; ++x)
                if (exempt(x, y)) pl->y[(size_t)y * g.w + x] = sy[(size_t)y * g.w + x];
    };
    auto restore_chroma = [&](int y0, int y1) {
        for (int cy = std::max(y0, 0); cy < std::min(y1, g.ch); ++cy)
            for (int cx = 0; cx < g.cw; ++cx)
                if (exempt(cx * g.sub_w, cy * g.sub_h)) {
                    pl->cb[(size_t)cy * g.cw + cx] = scb[(size_t)cy * g.cw + cx];
                    pl->cr[(size_t)cy * g.cw + cx] = scr[(size_t)cy * g.cw + cx];
                }
    };
    const int ctb = 1 << g.log2_ctb;
    // band b of a pass over `rows` rows with bands `bh` high: rows [r0, r1)
    // of its vertical segments / horizontal edges, and the rows it restores
    auto bands_of = [](int rows, int bh) { return (rows + bh - 1) / bh; };
    const int maxv = (1 << g.bd) - 1;
    const int nbl = bands_of(g.h, ctb);
    for (int pass = 0; pass < 2; ++pass) {
        const int edge_max = pass == 0 ? g.w : g.h, scan_max = pass == 0 ? g.h : g.w;
        run(nbl, [&](int band) {
        const int r0 = band * ctb, r1 = std::min((band + 1) * ctb, g.h);
        for (int edge = pass == 0 ? 8 : std::max(8, r0); edge <= edge_max - 4 && (pass == 0 || edge < r1); edge += 8) {
            for (int scan = pass == 0 ? r0 : 0; scan + 4 <= scan_max && (pass == 1 || scan < r1); scan += 4) {
                const int mid = scan + 1;
                const int bs = pass == 0 ? bs_v(edge, mid) : bs_h(mid, edge);
                if (bs == 0) continue;
                if (pass == 0 ? disabled_at(edge, mid) : disabled_at(mid, edge)) continue;
                const int qp_p = pass == 0 ? qp_at(edge - 1, mid) : qp_at(mid, edge - 1);
                const int qp_q = pass == 0 ? qp_at(edge, mid) : qp_at(mid, edge);
                const int avg = (qp_p + qp_q + 1) >> 1;
                int beta_offset, tc_offset;
                offsets_at(pass == 0 ? edge : mid, pass == 0 ? mid : edge, &beta_offset, &tc_offset);
                const int beta = kBeta[clamp3(avg + beta_offset, 0, 51)] << bd_shift;
                const int tc = kTc[clamp3(avg + 2 * (bs - 1) + tc_offset, 0, 53)] << bd_shift;
                if (tc == 0) continue;
                if (pass == 1 && !(edge + 4 <= g.h)) continue;
                Seg s{pl->y, g.w, pass == 0, edge, scan};
                bool dp1 = false, dq1 = false;
                const int dec = luma_decision(s, beta, tc, &dp1, &dq1);
                apply_luma(s, dec, dp1, dq1, tc, maxv);
            }
        }
        if (any_exempt) {
            if (pass == 0)
                restore_luma(r0, r1);
            else
                restore_luma(r0 - 4, band == nbl - 1 ? g.h : r1 - 4);
        }
        });
    }
    if (g.idc == 0) return HPVCD_OK;
    const int maxv_c = (1 << g.bd_c) - 1;
    const int cband = std::max(ctb / g.sub_h, 8);
    const int nbc = bands_of(g.ch, cband);
    for (int pass = 0; pass < 2; ++pass) {
        const int scan_max = pass == 0 ? g.ch : g.cw;
        const int cedge_max = pass == 0 ? g.cw : g.ch;
        run(nbc, [&](int band) {
        const int r0 = band * cband, r1 = std::min((band + 1) * cband, g.ch);
        for (int edge = pass == 0 ? 8 : std::max(8, r0); edge <= cedge_max - 2 && (pass == 0 || edge < r1); edge += 8) {
            for (int scan = pass == 0 ? r0 : 0; scan + 4 <= scan_max && (pass == 1 || scan < r1); scan += 4) {
                const int mid = scan + 1;
                const int lex = pass == 0 ? edge * g.sub_w : mid * g.sub_w;
                const int ley = pass == 0 ? mid * g.sub_h : edge * g.sub_h;
                const int bs = pass == 0 ? bs_v(lex, ley) : bs_h(lex, ley);
                if (bs < 2) continue;
                const int lqx = std::min(lex, g.w - 1), lqy = std::min(ley, g.h - 1);
                if (disabled_at(lqx, lqy)) continue;
                int ppx, ppy;
                if (pass == 0) {
                    ppx = std::min(std::max(lex - 1, 0), g.w - 1);
                    ppy = std::min(ley, g.h - 1);
                } else {
                    ppx = std::min(lex, g.w - 1);
                    ppy = std::min(std::max(ley - 1, 0), g.h - 1);
                }
                const int avg = (qp_at(ppx, ppy) + qp_at(lqx, lqy) + 1) >> 1;
                int beta_offset, tc_offset;
                offsets_at(lqx, lqy, &beta_offset, &tc_offset);
                (void)beta_offset;
                for (int plane = 0; plane < 2; ++plane) {
                    const int coff = plane == 0 ? p->pps_cb_qp_offset : p->pps_cr_qp_offset;
                    const int qpcv = qpc(avg + coff, g.idc, g.bd_c);
                    const int tc_c = kTc[clamp3(qpcv + 2 + tc_offset, 0, 53)] << bd_shift_c;
                    if (tc_c == 0) continue;
                    uint16_t* pix = plane == 0 ? pl->cb : pl->cr;
                    for (int s = scan; s < scan + 4; ++s) {
                        if (s >= scan_max) continue;
                        size_t ip0, ip1, iq0, iq1;
                        if (pass == 0) {
                            ip0 = (size_t)s * g.cw + edge - 1; ip1 = ip0 - 1;
                            iq0 = (size_t)s * g.cw + edge; iq1 = iq0 + 1;
                        } else {
                            ip0 = (size_t)(edge - 1) * g.cw + s; ip1 = (size_t)(edge - 2) * g.cw + s;
                            iq0 = (size_t)edge * g.cw + s; iq1 = (size_t)(edge + 1) * g.cw + s;
                        }
                        const int p0 = pix[ip0], p1 = pix[ip1], q0 = pix[iq0], q1 = pix[iq1];
                        const int delta = clamp3((((q0 - p0) * 4 + p1 - q1 + 4) >> 3), -tc_c, tc_c);
                        if (delta != 0) {
                            pix[ip0] = (uint16_t)clamp3(p0 + delta, 0, maxv_c);
                            pix[iq0] = (uint16_t)clamp3(q0 - delta, 0, maxv_c);
                        }
                    }
                }
            }
        }
        if (any_exempt) {
            if (pass == 0)
                restore_chroma(r0, r1);
            else
                restore_chroma(r0 - 4, band == nbc - 1 ? g.ch : r1 - 4);
        }
        });
    }
    return HPVCD_OK;
}

int deblock_picture(const hpvcd_picture* p, orc_planes* pl) {
    return deblock_picture_t(p, pl, [](int count, const std::function<void(int)>& body) {
        for (int b = 0; b < count; ++b) body(b);
    });
}


// decode.rs:2258-2493 apply_sao (serial, boundary-unrestricted path).
// Every CTB row reads the pre-SAO snapshot and writes its own rows, so
// `run(count, body)` may run the CTB rows in any order or at once (sao.rs:807
// apply_sao_parallel: CTB-row bands on the pool).
template <class Run>
int sao_picture_t(const hpvcd_picture* p, orc_planes* pl, Run run) {
    int rc = validate(p);
    if (rc) return rc;
    if (!p->sao) return HPVCD_OK;
    const bool sao_luma = (p->flags & HPVCD_PIC_SAO_LUMA) != 0;
    const bool sao_chroma = (p->flags & HPVCD_PIC_SAO_CHROMA) != 0 && p->chroma_idc != 0;
    if (!sao_luma && !sao_chroma) return HPVCD_OK;
    const Geo g = geo_of(p);
    const int ctb = 1 << g.log2_ctb;
    const bool no_slices = (p->flags & HPVCD_PIC_SAO_NO_ACROSS_SLICES) != 0;
    const bool no_tiles = (p->flags & HPVCD_PIC_SAO_NO_ACROSS_TILES) != 0;
    auto region_of = [&](int lx, int ly) -> int {
        return p->ctb_region[(size_t)(ly >> g.log2_ctb) * g.ctb_cols + (lx >> g.log2_ctb)];
    };
    const std::vector<uint16_t> oy(pl->y, pl->y + (size_t)g.w * g.h);
    std::vector<uint16_t> ocb, ocr;
    if (g.idc) {
        ocb.assign(pl->cb, pl->cb + (size_t)g.cw * g.ch);
        ocr.assign(pl->cr, pl->cr + (size_t)g.cw * g.ch);
    }
    run(g.ctb_rows, [&](int ry) {
        for (int rx = 0; rx < g.ctb_cols; ++rx) {
            const hpvcd_sao_ctb& s = p->sao[(size_t)ry * g.ctb_cols + rx];
            const int x0 = rx * ctb, y0 = ry * ctb;
            for (int c = 0; c < 3; ++c) {
                if (c == 0 && !sao_luma) continue;
                if (c > 0 && !sao_chroma) continue;
                const hpvcd_sao_comp& sc = s.comp[c];
                if (sc.type_idx == 0) continue;
                int32_t off[4] = {sc.offsets[0], sc.offsets[1], sc.offsets[2], sc.offsets[3]};
                const bool luma = c == 0;
                const int sw = luma ? 1 : g.sub_w, sh = luma ? 1 : g.sub_h;
                const int pw = luma ? g.w : g.cw, ph = luma ? g.h : g.ch;
                const int cx0 = x0 / sw, cy0 = y0 / sh;
                const int cx1 = std::min((x0 + ctb) / sw, pw), cy1 = std::min((y0 + ctb) / sh, ph);
                uint16_t* dst = luma ? pl->y : (c == 1 ? pl->cb : pl->cr);
                const uint16_t* src = luma ? oy.data() : (c == 1 ? ocb.data() : ocr.data());
                const int bd = luma ? g.bd : g.bd_c;
                if (sc.type_idx == 1)
                    tk->sao_band(dst, src, pw, cx0, cy0, cx1, cy1, off, sc.band_pos, bd);
                else if (!p->ctb_region && tk->sao_edge)
                    tk->sao_edge(dst, src, pw, ph, cx0, cy0, cx1, cy1, off, sc.eo_class, bd);
                else
                    sao_edge(dst, src, pw, ph, cx0, cy0, cx1, cy1, off, sc.eo_class, bd,
                             [&](int x, int y, int nx, int ny) {  // sao.rs:380-425 (slice / tile part)
                                 if (!p->ctb_region) return true;
                                 const int ra = region_of(x * sw, y * sh), rb = region_of(nx * sw, ny * sh);
                                 if (no_slices && (ra >> 8) != (rb >> 8)) return false;
                                 if (no_tiles && (ra & 0xff) != (rb & 0xff)) return false;
                                 return true;
                             });
            }
        }
        // decode.rs:2444-2485: exempt samples keep their pre-SAO value.
        if (!p->cells) return;
        for (int y = ry * ctb; y < std::min((ry + 1) * ctb, g.h); ++y)
            for (int x = 0; x < g.w; ++x)
                if (p->cells[(size_t)(y / 4) * g.gw + x / 4].flags & HPVCD_CELL_EXEMPT)
                    pl->y[(size_t)y * g.w + x] = oy[(size_t)y * g.w + x];
        for (int cy = ry * ctb / g.sub_h; cy < std::min((ry + 1) * ctb / g.sub_h, g.ch); ++cy)
            for (int cx = 0; cx < g.cw; ++cx) {
                const int lx = cx * g.sub_w, ly = cy * g.sub_h;
                if (p->cells[(size_t)(ly / 4) * g.gw + lx / 4].flags & HPVCD_CELL_EXEMPT) {
                    pl->cb[(size_t)cy * g.cw + cx] = ocb[(size_t)cy * g.cw + cx];
                    pl->cr[(size_t)cy * g.cw + cx] = ocr[(size_t)cy * g.cw + cx];
                }
            }
    });
    return HPVCD_OK;
}

int sao_picture(const hpvcd_picture* p, orc_planes* pl) {
    return sao_picture_t(p, pl, [](int count, const std::function<void(int)>& body) {
        for (int b = 0; b < count; ++b) body(b);
    });
}

// ---------------------------------------------------------------------------
// Work-stealing pool (threadpool.rs:300-520): one job deque per worker; a
// worker runs its own newest job, or steals the oldest job of another; a
// thread waiting for the jobs of a parallel_for runs jobs meanwhile, so a
// job may itself run a parallel_for (the grid rows' tile decodes run their
// banded filters on the same pool).
// ---------------------------------------------------------------------------
class StealPool {
public:
    explicit StealPool(int threads) : q_((size_t)std::max(threads, 1)) {
        for (auto& q : q_) q = std::make_unique<Deque>();
        for (int i = 1; i < (int)q_.size(); ++i) th_.emplace_back([this, i] { worker(i); });
    }
    ~StealPool() {
        stop_.store(true);
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    // body(i) for i in [0, count), on the pool; returns when all have run.
    void parallel_for(int count, const std::function<void(int)>& body) {
        if (count <= 0) return;
        if (count == 1 || q_.size() == 1) {
            for (int i = 0; i < count; ++i) body(i);
            return;
        }
        std::atomic<int> left{count};
        const int me = tls_id_ >= 0 ? tls_id_ : 0;
        {
            std::lock_guard<std::mutex> lk(q_[(size_t)me]->mu);
            for (int i = count - 1; i >= 0; --i) q_[(size_t)me]->d.push_back(Job{&body, i, &left});
        }
        queued_.fetch_add(count);
        cv_.notify_all();
        while (left.load() > 0)
            if (!run_one(me)) std::this_thread::yield();
    }

private:
    struct Job {
        const std::function<void(int)>* body;
        int index;
        std::atomic<int>* left;
    };
    struct Deque {
        std::mutex mu;
        std::deque<Job> d;
    };
    bool run_one(int me) {
        Job j{};
        bool got = false;
        {
            std::lock_guard<std::mutex> lk(q_[(size_t)me]->mu);
            if (!q_[(size_t)me]->d.empty()) {
                j = q_[(size_t)me]->d.back();
                q_[(size_t)me]->d.pop_back();
                got = true;
            }
        }
        for (size_t k = 1; !got && k < q_.size(); ++k) {
            Deque& o = *q_[(me + k) % q_.size()];
            std::lock_guard<std::mutex> lk(o.mu);
            if (!o.d.empty()) {
                j = o.d.front();
                o.d.pop_front();
                got = true;
            }
        }
        if (!got) return false;
        queued_.fetch_sub(1);
        (*j.body)(j.index);
        j.left->fetch_sub(1);
        return true;
    }
    void worker(int id) {
        tls_id_ = id;
        while (!stop_.load()) {
            if (run_one(id)) continue;
            std::unique_lock<std::mutex> lk(wait_mu_);
            cv_.wait_for(lk, std::chrono::milliseconds(1), [&] { return queued_.load() > 0 || stop_.load(); });
        }
    }
    std::vector<std::unique_ptr<Deque>> q_;
    std::vector<std::thread> th_;
    std::mutex wait_mu_;
    std::condition_variable cv_;
    std::atomic<int> queued_{0};
    std::atomic<bool> stop_{false};
    static thread_local int tls_id_;
};
thread_local int StealPool::tls_id_ = -1;

// Q13 YCbCr -> RGB8 of rows [y0, y1) of a tile's crop onto its canvas
// (yuv.rs:232 / :327 rows, lib.rs:1964-1978 >> (bd - 8), lib.rs:1610-1660
// placement with cropping); the AVX2 row kernel for the matrices it covers.
void tile_rgb_rows(const orc_planes& pl, const Geo& g, int matrix, bool full, int tw, int y0, int y1, uint8_t* canvas,
                   int canvas_w, int dst_x, int dst_y, int copy_w) {
    std::vector<uint16_t> buf((size_t)tw * 3);
    const int shift = g.bd - 8;
    const bool simd_ok = tk->simd_rgb && g.idc != 0 && g.bd <= 12 && matrix != HPVCD_MATRIX_IDENTITY &&
                         matrix != HPVCD_MATRIX_YCGCO && g.sub_h <= 2;
    int64_t cr_r0, cb_g0, cr_g0, cb_b0;
    switch (matrix) {
        case HPVCD_MATRIX_BT470BG:
        case HPVCD_MATRIX_SMPTE170M: cr_r0 = 11485; cb_g0 = -2819; cr_g0 = -5851; cb_b0 = 14516; break;
        case HPVCD_MATRIX_BT2020NCL: cr_r0 = 12080; cb_g0 = -1348; cr_g0 = -4681; cb_b0 = 17546; break;
        default: cr_r0 = 12901; cb_g0 = -1534; cr_g0 = -3835; cb_b0 = 15201; break;
    }
    const int32_t k_y = full ? 8192 : 9539, k_uv = full ? 8192 : 9326;
    const int32_t scale = 1 << (g.bd - 8);
    const int32_t y_black = full ? 0 : 16 * scale, neutral = 128 * scale;
    const int32_t cmax = g.bd == 8 ? 255 : (1 << g.bd) - 1;
    for (int y = y0; y < y1; ++y) {
        if (simd_ok) {
            const int yr = std::min(y, g.h - 1), cr = std::min(y / g.sub_h, g.ch - 1);
            orc_simd::rgb_row(pl.y + (size_t)yr * g.w, pl.cb + (size_t)cr * g.cw, pl.cr + (size_t)cr * g.cw, 0, tw, g.w,
                              g.cw, g.sub_w, g.bd, k_y, y_black, neutral, (int32_t)((cr_r0 * k_uv + 4096) >> 13),
                              (int32_t)((cb_g0 * k_uv + 4096) >> 13), (int32_t)((cr_g0 * k_uv + 4096) >> 13),
                              (int32_t)((cb_b0 * k_uv + 4096) >> 13), cmax, buf.data());
        } else {
            yuv_to_rgb16(pl.y, pl.cb, pl.cr, g.w, g.h, g.idc, g.bd, tw, 1, 0, y, matrix, full, buf.data());
        }
        uint8_t* o = canvas + ((size_t)(dst_y + y) * canvas_w + dst_x) * 3;
        for (int x = 0; x < copy_w * 3; ++x) o[x] = (uint8_t)(buf[x] >> shift);
    }
}

// The reference's grid decode (lib.rs:1724 decode_grid -> :1680
// fill_grid_bands): one job per grid row of tiles on the pool, each decoding
// its tiles one after another; per tile the reconstruction (serial: no
// wavefront parallel processing in these streams), the banded deblocking
// and SAO drivers, and the banded RGB conversion into the canvas.  Intra /
// residual pictures onto RGB8 canvases.
int decode_grid_reference(const hpvcd_picture* pics, uint32_t n, const hpvcd_output* out, uint8_t* rgb, int threads,
                          bool simd) {
    if (!out || out->kind != HPVCD_OUT_RGB8 || !out->place || !rgb) return HPVCD_ERR_INVALID_ARG;
    const uint32_t nc = out->n_canvases ? out->n_canvases : 1;
    std::vector<hpvcd_canvas> cvs;
    std::vector<size_t> offs;
    size_t acc = 0;
    for (uint32_t k = 0; k < nc; ++k) {
        const hpvcd_canvas cv = out->n_canvases ? out->canvases[k]
                                                : hpvcd_canvas{out->canvas_w, out->canvas_h, out->matrix,
                                                               out->full_range, out->orientation};
        if (cv.matrix == HPVCD_CANVAS_NATIVE || (cv.orientation > 1)) return HPVCD_ERR_UNSUPPORTED;
        cvs.push_back(cv);
        offs.push_back(acc);
        acc += (size_t)cv.width * cv.height * 3;
    }
    for (uint32_t i = 0; i < n; ++i) {
        const int rc = validate(&pics[i]);
        if (rc) return rc;
        if ((pics[i].flags & HPVCD_PIC_INTER) || out->place[i].canvas >= nc) return HPVCD_ERR_UNSUPPORTED;
    }
    // grid rows: tiles sharing a canvas and a top row, in submission order
    std::map<std::pair<uint32_t, uint32_t>, std::vector<uint32_t>> row_of;
    for (uint32_t i = 0; i < n; ++i) row_of[{out->place[i].canvas, out->place[i].dst_y}].push_back(i);
    std::vector<std::vector<uint32_t>> rows;
    for (auto& kv : row_of) rows.push_back(kv.second);
    const Kernels* kset = simd ? &kAvx2Kernels : &kScalarKernels;
    const Kernels* caller_set = tk;  // the calling thread runs jobs too: restored below
    StealPool pool(threads);
    std::atomic<int> err{0};
    auto on_pool = [&](int count, const std::function<void(int)>& body) {
        pool.parallel_for(count, [&](int b) {
            tk = kset;
            body(b);
        });
    };
    pool.parallel_for((int)rows.size(), [&](int r) {
        tk = kset;
        for (const uint32_t i : rows[(size_t)r]) {
            const hpvcd_picture* p = &pics[i];
            const Geo g = geo_of(p);
            std::vector<uint16_t> y((size_t)g.w * g.h), cb((size_t)std::max(g.cw * g.ch, 1)),
                cr((size_t)std::max(g.cw * g.ch, 1));
            orc_planes pl{y.data(), cb.data(), cr.data()};
            if (p->flags & HPVCD_PIC_PRED_IN_PLANE)
                for (int c = 0; c < (g.idc ? 3 : 1); ++c) {
                    const size_t cnt = c == 0 ? (size_t)g.w * g.h : (size_t)g.cw * g.ch;
                    uint16_t* dst = c == 0 ? pl.y : (c == 1 ? pl.cb : pl.cr);
                    if (!p->pred[c]) continue;
                    if ((c == 0 ? g.bd : g.bd_c) <= 8)
                        for (size_t k = 0; k < cnt; ++k) dst[k] = ((const uint8_t*)p->pred[c])[k];
                    else
                        std::memcpy(dst, p->pred[c], cnt * 2);
                }
            int rc = recon_picture(p, &pl);
            if (!rc) rc = deblock_picture_t(p, &pl, on_pool);
            if (!rc) rc = sao_picture_t(p, &pl, on_pool);
            if (rc) {
                err.store(rc);
                continue;
            }
            const hpvcd_tile_place& tp = out->place[i];
            const hpvcd_canvas& cv = cvs[tp.canvas];
            const int tw = (int)std::min<uint32_t>(tp.crop_w, (uint32_t)g.w);
            const int th = (int)std::min<uint32_t>(tp.crop_h, (uint32_t)g.h);
            const int copy_w = std::min(tw, std::max((int)cv.width - (int)tp.dst_x, 0));
            const int copy_h = std::min(th, std::max((int)cv.height - (int)tp.dst_y, 0));
            if (copy_w <= 0 || copy_h <= 0) continue;
            const int band = 64;  // yuv.rs:393 banded: rows per band
            on_pool((copy_h + band - 1) / band, [&](int b) {
                tile_rgb_rows(pl, g, (int)cv.matrix, cv.full_range != 0, copy_w, b * band, std::min(copy_h, (b + 1) * band),
                              rgb + offs[tp.canvas], (int)cv.width, (int)tp.dst_x, (int)tp.dst_y, copy_w);
            });
        }
    });
    tk = caller_set;
    return err.load();
}

}  // namespace

// ---------------------------------------------------------------------------
// C exports
// ---------------------------------------------------------------------------
extern "C" {

// The reference's CPU decode of a grid of intra / residual tiles onto RGB8
// canvases (its parallel structure: grid-row jobs, banded filters and
// colour conversion on a work-stealing pool), with the scalar kernels or the
// AVX2 set (simd != 0); `threads` pool threads including the caller.
int32_t orc_decode_grid_reference(const hpvcd_picture* pics, uint32_t n, const hpvcd_output* out, uint8_t* rgb,
                                  int32_t threads, int32_t simd) {
    if (simd && !orc_simd::available()) return HPVCD_ERR_UNSUPPORTED;
    return decode_grid_reference(pics, n, out, rgb, threads, simd != 0);
}

// Slices whose deblocking is disabled (flags[256], one per slice index;
// NULL clears them all).  Test input of the oracle only.
void orc_set_disabled_slices(const uint8_t* flags) {
    g_any_slice_disabled = false;
    for (int i = 0; i < 256; ++i) {
        g_slice_disabled[i] = flags ? flags[i] : 0;
        g_any_slice_disabled = g_any_slice_disabled || g_slice_disabled[i];
    }
}


int32_t orc_max_log2_tr_range(int32_t bd, int32_t ext) { return max_tr_range(bd, ext != 0); }
void orc_dequant_params_get(int32_t n, int32_t qp, int32_t bd, int32_t ext, orc_dequant_params* o) {
    *o = dequant_params(n, qp, bd, ext != 0);
}
void orc_ts_params_get(int32_t n, int32_t qp, int32_t bd, int32_t ext, orc_ts_params* o) {
    *o = ts_params(n, qp, bd, ext != 0);
}
void orc_dequant(const int32_t* levels, int32_t n, const orc_dequant_params* p,
                 const uint8_t* scaling, int32_t dc, int32_t i16s, int32_t* out) {
    dequant(levels, n, *p, scaling, dc, i16s != 0, out);
}
void orc_rext_residual_ops(int32_t* res, int32_t n, int32_t rotate, int32_t dir, int32_t i16s) {
    rext_residual_ops(res, n, rotate != 0, dir, i16s != 0);
}

int32_t orc_scaling_select(const hpvcd_scaling* s, int32_t comp, int32_t n, int32_t inter, int32_t tskip,
                           int32_t* first, int32_t* dc) {
    int d = 16;
    const uint8_t* m = scaling_select(s, comp, n, inter != 0, tskip != 0, &d);
    if (!m) return 0;
    *first = m[0];
    *dc = d;
    return 1;
}

void orc_dequant_ts(const int32_t* levels, int32_t n, const orc_ts_params* p,
                    const uint8_t* scaling, int32_t dc, int32_t i16s, int32_t* out) {
    dequant_ts(levels, n, *p, scaling, dc, i16s != 0, out);
}
void orc_inv_dct(const int32_t* coeff, int32_t n, int32_t bd, int32_t max_range, int32_t nx,
                 int32_t i16s, int32_t* out) {
    inv_dct(coeff, n, bd, max_range, nx, i16s != 0, out);
}
void orc_inv_dst4(const int32_t* coeff, int32_t bd, int32_t max_range, int32_t i16s, int32_t* out) {
    inv_dst4(coeff, bd, max_range, i16s != 0, out);
}
int32_t orc_dct_matrix_entry(int32_t n, int32_t k, int32_t m) { return dct_entry(n, k, m); }
void orc_add_residual(uint16_t* dst, int32_t stride, const uint16_t* pred, const int32_t* res,
                      int32_t n, int32_t vw, int32_t vh, int32_t bd) {
    add_residual(dst, stride, pred, res, n, vw, vh, bd);
}
// reconstruct.rs:125-129
void orc_narrow_i32_to_i16(const int32_t* src, int16_t* dst, int32_t count) {
    for (int i = 0; i < count; ++i) dst[i] = (int16_t)clamp3(src[i], -32768, 32767);
}
void orc_intra_substitute(const int32_t* ra, const int32_t* rl, int32_t rc, int32_t n,
                          int32_t neutral, uint16_t* ao, uint16_t* lo) {
    intra_substitute(ra, rl, rc, n, neutral, ao, lo);
}
void orc_intra_filter(const uint16_t* a, const uint16_t* l, int32_t n, int32_t mode,
                      int32_t is_luma, int32_t sm, int32_t strong, int32_t bd, uint16_t* fa,
                      uint16_t* fl) {
    intra_filter(a, l, n, mode, is_luma != 0, sm != 0, strong != 0, bd, fa, fl);
}
void orc_intra_predict(int32_t mode, const uint16_t* a, const uint16_t* l, int32_t n,
                       int32_t is_luma, int32_t bd, uint16_t* out) {
    intra_predict(mode, a, l, n, is_luma != 0, bd, out);
}
void orc_luma_interp(const uint16_t* ref, int32_t stride, int32_t width, int32_t height,
                     int32_t x0, int32_t y0, int32_t fx, int32_t fy, int32_t w, int32_t h,
                     int32_t bd, int16_t* dst) {
    RefPlane r{ref, stride, width, height};
    interp(r, x0, y0, fx, fy, w, h, bd, 8, kLumaFilter[fx], kLumaFilter[fy], dst);
}
void orc_chroma_interp(const uint16_t* ref, int32_t stride, int32_t width, int32_t height,
                       int32_t x0, int32_t y0, int32_t fx, int32_t fy, int32_t w, int32_t h,
                       int32_t bd, int16_t* dst) {
    RefPlane r{ref, stride, width, height};
    interp(r, x0, y0, fx, fy, w, h, bd, 4, kChromaFilter[fx], kChromaFilter[fy], dst);
}
void orc_uni_mc(const int16_t* s, int32_t w, int32_t h, int32_t vw, int32_t vh, int32_t bd,
                uint16_t* d, int32_t st) {
    uni_mc(s, w, h, vw, vh, bd, d, st);
}
void orc_bi_mc(const int16_t* a, const int16_t* b, int32_t w, int32_t h, int32_t vw, int32_t vh,
               int32_t bd, uint16_t* d, int32_t st) {
    bi_mc(a, b, w, h, vw, vh, bd, d, st);
}
void orc_uni_mc_weighted(const int16_t* s, int32_t w, int32_t h, int32_t vw, int32_t vh,
                         int32_t bd, int32_t wt, int32_t off, int32_t dn, uint16_t* d, int32_t st) {
    uni_mc_w(s, w, h, vw, vh, bd, wt, off, dn, d, st);
}
void orc_bi_mc_weighted(const int16_t* a, const int16_t* b, int32_t w, int32_t h, int32_t vw,
                        int32_t vh, int32_t bd, int32_t w0, int32_t o0, int32_t w1, int32_t o1,
                        int32_t dn, uint16_t* d, int32_t st) {
    bi_mc_w(a, b, w, h, vw, vh, bd, w0, o0, w1, o1, dn, d, st);
}
// inter.rs:18-58
int32_t orc_normalize_luma_offset(int32_t offset, int32_t bd, int32_t hp) {
    const int32_t range = hp ? 1 << (bd - 1) : 128;
    const int32_t scale = hp ? 1 : 1 << (bd - 8);
    return clamp3(offset, -range, range - 1) * scale;
}
int32_t orc_derive_chroma_offset(int32_t delta, int32_t weight, int32_t log2_denom, int32_t bd,
                                 int32_t hp) {
    const int64_t range = hp ? (int64_t)1 << (bd - 1) : 128;
    const int32_t scale = hp ? 1 : 1 << (bd - 8);
    const int64_t pred = range - ((range * weight) >> log2_denom);
    const int32_t off = (int32_t)clamp3<int64_t>(delta + pred, -range, range - 1);
    return off * scale;
}
int32_t orc_qp_prime(int32_t qp, int32_t bd) { return qp_prime(qp, bd); }
int32_t orc_qpc(int32_t qpi, int32_t idc, int32_t bd) { return qpc(qpi, idc, bd); }
int32_t orc_clamp_qpy(int32_t qp, int32_t bd) { return clamp_qpy(qp, bd); }

int32_t orc_deblock_luma_segment(uint16_t* plane, int32_t stride, int32_t vertical, int32_t edge,
                                 int32_t scan, int32_t beta, int32_t tc, int32_t maxv) {
    Seg s{plane, stride, vertical != 0, edge, scan};
    bool dp1 = false, dq1 = false;
    const int dec = luma_decision(s, beta, tc, &dp1, &dq1);
    apply_luma(s, dec, dp1, dq1, tc, maxv);
    return dec;
}
void orc_apply_luma_decision(uint16_t* plane, int32_t stride, int32_t vertical, int32_t edge,
                             int32_t scan, int32_t decision, int32_t tc, int32_t maxv) {
    Seg s{plane, stride, vertical != 0, edge, scan};
    if (decision <= 0) return;
    if (decision == 1) {
        apply_luma(s, 1, false, false, tc, maxv);
        return;
    }
    const int d = decision - 2;
    apply_luma(s, 2, ((d >> 1) & 1) != 0, (d & 1) != 0, tc, maxv);
}
void orc_sao_edge(uint16_t* dst, const uint16_t* src, int32_t w, int32_t h, int32_t x0, int32_t y0,
                  int32_t x_end, int32_t y_end, const int32_t* off, int32_t eo, int32_t bd) {
    sao_edge(dst, src, w, h, x0, y0, x_end, y_end, off, eo, bd, [](int, int, int, int) { return true; });
}
void orc_sao_band(uint16_t* dst, const uint16_t* src, int32_t w, int32_t x0, int32_t y0,
                  int32_t x_end, int32_t y_end, const int32_t* off, int32_t bp, int32_t bd) {
    sao_band(dst, src, w, x0, y0, x_end, y_end, off, bp, bd);
}
void orc_yuv_to_rgb16(const uint16_t* y, const uint16_t* cb, const uint16_t* cr, int32_t width,
                      int32_t height, int32_t idc, int32_t bd, int32_t dw, int32_t dh,
                      int32_t crop_left, int32_t crop_top, int32_t matrix, int32_t full_range,
                      uint16_t* out) {
    yuv_to_rgb16(y, cb, cr, width, height, idc, bd, dw, dh, crop_left, crop_top, matrix,
                 full_range != 0, out);
}

void orc_load_block_clipped(const uint16_t* plane, int32_t stride, int32_t width, int32_t height,
                            int32_t x0, int32_t y0, int32_t n, uint16_t* pred) {
    load_block_clipped(plane, stride, width, height, x0, y0, n, pred);
}
int32_t orc_recon_picture(const hpvcd_picture* pic, orc_planes* planes) {
    return recon_picture(pic, planes);
}
int32_t orc_mc_picture(const hpvcd_picture* pic, const orc_planes* refs, int32_t n_refs,
                       orc_planes* planes) {
    return mc_picture(pic, refs, n_refs, planes);
}
int32_t orc_deblock_picture(const hpvcd_picture* pic, orc_planes* planes) {
    return deblock_picture(pic, planes);
}
int32_t orc_sao_picture(const hpvcd_picture* pic, orc_planes* planes) {
    return sao_picture(pic, planes);
}

// lib.rs:2065-2110 rotate_luma and :2112-2200 rotate_buf on a w x h image of
// `esz`-byte elements: FlipH / Rotate180 / FlipV / Rotate90 / Rotate270 move
// the elements (Rotate90: row r, column c -> row c, column h - 1 - r of the
// h-wide result; Rotate270: -> row w - 1 - c, column r); Normal, Transpose
// and Transverse leave them in place.
static void orient_samples(uint8_t* img, int w, int h, int esz, uint32_t o) {
    if (o != HPVCD_ORIENT_FLIP_H && o != HPVCD_ORIENT_ROTATE180 && o != HPVCD_ORIENT_FLIP_V &&
        o != HPVCD_ORIENT_ROTATE90 && o != HPVCD_ORIENT_ROTATE270)
        return;
    const std::vector<uint8_t> src(img, img + (size_t)w * h * esz);
    for (int r = 0; r < h; ++r)
        for (int c = 0; c < w; ++c) {
            size_t d;
            switch (o) {
                case HPVCD_ORIENT_FLIP_H: d = (size_t)r * w + (w - 1 - c); break;
                case HPVCD_ORIENT_ROTATE180: d = (size_t)(h - 1 - r) * w + (w - 1 - c); break;
                case HPVCD_ORIENT_FLIP_V: d = (size_t)(h - 1 - r) * w + c; break;
                case HPVCD_ORIENT_ROTATE90: d = (size_t)c * h + (h - 1 - r); break;
                default: d = (size_t)(w - 1 - c) * h + r; break;  // Rotate270
            }
            std::memcpy(img + d * esz, &src[((size_t)r * w + c) * esz], (size_t)esz);
        }
}

int32_t orc_decode_batch(const hpvcd_picture* pics, uint32_t n, const hpvcd_output* out,
                         orc_planes* planes_out, uint8_t* rgb, int32_t threads) {
    if (!pics && n) return HPVCD_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; ++i) {
        const int rc = validate(&pics[i]);
        if (rc) return rc;
    }
    // Per-picture plane storage (16-bit, as the reference keeps it).
    std::vector<std::vector<uint16_t>> py(n), pcb(n), pcr(n);
    std::vector<orc_planes> pl(n);
    bool has_inter = false;
    for (uint32_t i = 0; i < n; ++i) {
        const Geo g = geo_of(&pics[i]);
        py[i].assign((size_t)g.w * g.h, 0);
        pcb[i].assign((size_t)std::max(g.cw * g.ch, 1), 0);
        pcr[i].assign((size_t)std::max(g.cw * g.ch, 1), 0);
        pl[i] = {py[i].data(), pcb[i].data(), pcr[i].data()};
        if (pics[i].flags & HPVCD_PIC_INTER) has_inter = true;
    }
    std::atomic<int> err{0};
    auto decode_one = [&](uint32_t i) {
        const hpvcd_picture* p = &pics[i];
        const Geo g = geo_of(p);
        if (p->flags & HPVCD_PIC_PRED_IN_PLANE) {
            for (int c = 0; c < (g.idc ? 3 : 1); ++c) {
                const size_t cnt = c == 0 ? (size_t)g.w * g.h : (size_t)g.cw * g.ch;
                const int bd = c == 0 ? g.bd : g.bd_c;
                uint16_t* dst = c == 0 ? pl[i].y : (c == 1 ? pl[i].cb : pl[i].cr);
                if (!p->pred[c]) continue;
                if (bd <= 8) {
                    const uint8_t* s = (const uint8_t*)p->pred[c];
                    for (size_t k = 0; k < cnt; ++k) dst[k] = s[k];
                } else {
                    std::memcpy(dst, p->pred[c], cnt * 2);
                }
            }
        }
        int rc = HPVCD_OK;
        if (p->flags & HPVCD_PIC_INTER) rc = mc_picture(p, pl.data(), (int)i, &pl[i]);
        if (!rc) rc = recon_picture(p, &pl[i]);
        if (!rc) rc = deblock_picture(p, &pl[i]);
        if (!rc) rc = sao_picture(p, &pl[i]);
        if (rc) err.store(rc);
    };
    if (threads > 1 && !has_inter && n > 1) {
        std::atomic<uint32_t> next{0};
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t)
            pool.emplace_back([&]() {
                for (uint32_t i; (i = next.fetch_add(1)) < n;) decode_one(i);
            });
        for (auto& th : pool) th.join();
    } else {
        for (uint32_t i = 0; i < n; ++i) decode_one(i);
    }
    if (err.load()) return err.load();
    if (planes_out) {
        for (uint32_t i = 0; i < n; ++i) {
            const Geo g = geo_of(&pics[i]);
            if (planes_out[i].y) std::memcpy(planes_out[i].y, pl[i].y, (size_t)g.w * g.h * 2);
            if (g.idc && planes_out[i].cb) std::memcpy(planes_out[i].cb, pl[i].cb, (size_t)g.cw * g.ch * 2);
            if (g.idc && planes_out[i].cr) std::memcpy(planes_out[i].cr, pl[i].cr, (size_t)g.cw * g.ch * 2);
        }
    }
    if (out && (out->kind == HPVCD_OUT_RGB8 || out->kind == HPVCD_OUT_YUV_CANVAS) && rgb && out->place) {
        // Canvases: one (canvas_w x canvas_h) or out->canvases[] (lib.rs:1724
        // decode_grid per output image).  An RGB8 canvas holds packed RGB8; a
        // native one (every canvas of a YUV canvas output, HPVCD_CANVAS_NATIVE
        // ones of an RGB8 output) Y then Cb then Cr in the format of its
        // pictures (8-bit 4:0:0 without pictures).
        const uint32_t nc = out->n_canvases ? out->n_canvases : 1;
        for (uint32_t i = 0; i < n; ++i)
            if (out->place[i].canvas >= nc) return HPVCD_ERR_INVALID_ARG;
        struct Cv {
            bool native;
            int w, h, idc, bps, sw, sh, cw, ch;
            uint32_t matrix, full_range, orientation;
            size_t off;
        };
        std::vector<Cv> cvs;
        size_t acc = 0;
        for (uint32_t k = 0; k < nc; ++k) {
            const hpvcd_canvas cv = out->n_canvases ? out->canvases[k]
                                                    : hpvcd_canvas{out->canvas_w, out->canvas_h, out->matrix,
                                                                   out->full_range, out->orientation};
            Cv c{};
            c.orientation = cv.orientation;
            c.native = out->kind == HPVCD_OUT_YUV_CANVAS || cv.matrix == HPVCD_CANVAS_NATIVE;
            c.w = (int)cv.width;
            c.h = (int)cv.height;
            c.matrix = cv.matrix;
            c.full_range = cv.full_range;
            c.idc = 0;
            c.bps = 1;
            for (uint32_t i = 0; i < n; ++i)
                if (out->place[i].canvas == k) {
                    c.idc = pics[i].chroma_idc;
                    c.bps = geo_of(&pics[i]).bd > 8 || geo_of(&pics[i]).bd_c > 8 ? 2 : 1;
                    break;
                }
            c.sw = c.idc == 1 || c.idc == 2 ? 2 : 1;
            c.sh = c.idc == 1 ? 2 : 1;
            c.cw = c.idc ? (c.w + c.sw - 1) / c.sw : 0;
            c.ch = c.idc ? (c.h + c.sh - 1) / c.sh : 0;
            c.off = acc;
            acc += c.native ? ((size_t)c.w * c.h + 2 * (size_t)c.cw * c.ch) * c.bps : (size_t)c.w * c.h * 3;
            cvs.push_back(c);
        }
        // native canvases: lib.rs:993-1091 fill_native_grid_yuv and :871-991
        // stitch_native_yuv_band: each tile's visible part copied onto the
        // image planes at its grid position (chroma at position / subsampling),
        // rows past the tile repeating its last row, columns its last sample.
        for (uint32_t i = 0; i < n; ++i) {
            const Geo g = geo_of(&pics[i]);
            const hpvcd_tile_place& tp = out->place[i];
            const Cv& c = cvs[tp.canvas];
            if (!c.native) continue;
            if (c.idc != g.idc || c.bps != (g.bd > 8 || g.bd_c > 8 ? 2 : 1)) return HPVCD_ERR_INVALID_ARG;
            for (int comp = 0; comp < (g.idc ? 3 : 1); ++comp) {
                const int sw = comp ? c.sw : 1, sh = comp ? c.sh : 1;
                const int CW = comp ? c.cw : c.w, CH = comp ? c.ch : c.h;
                const int pw = comp ? g.cw : g.w, ph = comp ? g.ch : g.h;
                const int dx = (int)tp.dst_x / sw, dy = (int)tp.dst_y / sh;
                const int copy_w = std::min(((int)tp.crop_w + sw - 1) / sw, std::max(CW - dx, 0));
                const int copy_h = std::min(((int)tp.crop_h + sh - 1) / sh, std::max(CH - dy, 0));
                const uint16_t* src = comp == 0 ? pl[i].y : (comp == 1 ? pl[i].cb : pl[i].cr);
                uint8_t* base = rgb + c.off +
                                (comp == 0 ? 0 : ((size_t)c.w * c.h + (size_t)(comp - 1) * c.cw * c.ch) * c.bps);
                for (int y = 0; y < copy_h; ++y)
                    for (int x = 0; x < copy_w; ++x) {
                        const uint16_t v = src[(size_t)std::min(y, ph - 1) * pw + std::min(x, pw - 1)];
                        const size_t o = (size_t)(dy + y) * CW + dx + x;
                        if (c.bps == 1) {
                            base[o] = (uint8_t)v;
                        } else {
                            base[2 * o] = (uint8_t)v;
                            base[2 * o + 1] = (uint8_t)(v >> 8);
                        }
                    }
            }
        }
        // RGB8 canvases: lib.rs:1610-1660 per-tile RGB then row copy with
        // cropping; lib.rs:1964-1978 rgb8 narrowing by >> (bit_depth - 8).
        std::atomic<uint32_t> next{0};
        auto convert = [&](uint32_t i) {
            const hpvcd_picture* p = &pics[i];
            const Geo g = geo_of(p);
            const hpvcd_tile_place& tp = out->place[i];
            const Cv& c = cvs[tp.canvas];
            if (c.native) return;
            const int tw = (int)tp.crop_w, th = (int)tp.crop_h;
            if (tw <= 0 || th <= 0) return;
            std::vector<uint16_t> buf((size_t)tw * th * 3);
            yuv_to_rgb16(pl[i].y, pl[i].cb, pl[i].cr, g.w, g.h, g.idc, g.bd, tw, th, 0, 0, (int)c.matrix,
                         c.full_range != 0, buf.data());
            const int shift = g.bd - 8;
            uint8_t* base = rgb + c.off;
            const int copy_w = std::min(tw, std::max(c.w - (int)tp.dst_x, 0));
            const int copy_h = std::min(th, std::max(c.h - (int)tp.dst_y, 0));
            for (int y = 0; y < copy_h; ++y)
                for (int x = 0; x < copy_w * 3; ++x)
                    base[((size_t)(tp.dst_y + y) * c.w + tp.dst_x) * 3 + x] =
                        (uint8_t)(buf[(size_t)y * tw * 3 + x] >> shift);
        };
        if (threads > 1 && n > 1) {
            std::vector<std::thread> pool;
            for (int t = 0; t < threads; ++t)
                pool.emplace_back([&]() {
                    for (uint32_t i; (i = next.fetch_add(1)) < n;) convert(i);
                });
            for (auto& th : pool) th.join();
        } else {
            for (uint32_t i = 0; i < n; ++i) convert(i);
        }
        // lib.rs:2017-2110 apply_orientation on each finished canvas
        for (const Cv& c : cvs) {
            if (c.native) {
                uint8_t* p0 = rgb + c.off;
                orient_samples(p0, c.w, c.h, c.bps, c.orientation);
                if (c.idc) {
                    uint8_t* p1 = p0 + (size_t)c.w * c.h * c.bps;
                    orient_samples(p1, c.cw, c.ch, c.bps, c.orientation);
                    orient_samples(p1 + (size_t)c.cw * c.ch * c.bps, c.cw, c.ch, c.bps, c.orientation);
                }
            } else {
                orient_samples(rgb + c.off, c.w, c.h, 3, c.orientation);
            }
        }
    }
    return HPVCD_OK;
}

}  // extern "C"
