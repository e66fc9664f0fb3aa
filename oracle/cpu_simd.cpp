// cpu_simd.cpp -- AVX2 kernels of the CPU reference arm (test
// infrastructure; see cpu_simd.h).  Every kernel computes the same integers
// as its scalar counterpart in hpvcd_oracle.cpp.
#include "cpu_simd.h"

#include <immintrin.h>

#include <algorithm>
#include <cstring>

namespace orc_simd {

bool available() { return __builtin_cpu_supports("avx2"); }

namespace {

// H.265 DCT basis magnitudes by angle j (units of pi/64): entry (k, m) of the
// n-point basis is +-mag[j] for j = k (32 / n) (2m + 1) folded into [0, 32].
constexpr int8_t kMag[33] = {64, 90, 90, 90, 89, 88, 87, 85, 83, 82, 80, 78, 75, 73, 70, 67, 64,
                             61, 57, 54, 50, 46, 43, 38, 36, 31, 25, 22, 18, 13, 9,  4,  0};

int basis(int n, int k, int m) {
    if (k == 0) return 64;
    int j = (k * (32 / n) * (2 * m + 1)) & 127;
    int sign = 1;
    if (j > 64) j = 128 - j;
    if (j > 32) {
        j = 64 - j;
        sign = -1;
    }
    return sign * kMag[j];
}

// Per transform size: the basis as int16 rows T[k][m], and the stage-1
// multipliers (T[2p][m], T[2p+1][m]) packed as one int32 per (m, p).
struct Basis {
    alignas(32) int16_t t[32][32];
    int32_t pair[32][16];
    void init(int n) {
        for (int k = 0; k < n; ++k)
            for (int m = 0; m < n; ++m) t[k][m] = (int16_t)basis(n, k, m);
        for (int m = 0; m < n; ++m)
            for (int p = 0; p < n / 2; ++p)
                pair[m][p] = (int32_t)(uint16_t)t[2 * p][m] | ((int32_t)(uint16_t)t[2 * p + 1][m] << 16);
    }
};

const Basis& basis_of(int n) {
    static Basis b16, b32;
    static bool ready = [] {
        b16.init(16);
        b32.init(32);
        return true;
    }();
    (void)ready;
    return n == 16 ? b16 : b32;
}

inline __m256i bcast_pair(int16_t a, int16_t b) {
    return _mm256_set1_epi32((int32_t)(uint16_t)a | ((int32_t)(uint16_t)b << 16));
}

}  // namespace

// Stage 1 (columns): tmp[m][c] = clip16((sum_k T[k][m] D[k][c] + 64) >> 7),
// 16 columns per vector: rows k, k+1 interleaved (unpack) and multiplied by
// the packed pair (T[k][m], T[k+1][m]) with madd, eight sums per half.  The
// pack of the two halves saturates to int16 (the reference's clip) and puts
// the columns back in order.  Stage 2 (rows): out[r][m] = (sum_k tmp[r][k]
// T[k][m] + add2) >> shift2, 16 outputs m per vector pair, the broadcast
// pair (tmp[r][k], tmp[r][k+1]) against interleaved basis rows.
void inv_dct(const int32_t* coeff, int n, int bd, int nx, bool i16s, int32_t* out) {
    const Basis& B = basis_of(n);
    const int shift2 = 20 - bd, add2 = 1 << (shift2 - 1);
    alignas(32) int16_t d[32][32];
    alignas(32) int16_t tmp[32][32];
    int rows = 0;
    for (int k = 0; k < n; ++k) {
        bool any = false;
        for (int c = 0; c < n; ++c) {
            d[k][c] = (int16_t)coeff[k * n + c];
            any |= d[k][c] != 0;
        }
        if (any) rows = k + 1;
    }
    const int pairs1 = (rows + 1) / 2;
    const __m256i r64 = _mm256_set1_epi32(64);
    for (int cg = 0; cg < n / 16; ++cg) {
        __m256i lo[16], hi[16];
        for (int p = 0; p < pairs1; ++p) {
            const __m256i a = _mm256_load_si256((const __m256i*)&d[2 * p][16 * cg]);
            const __m256i b = _mm256_load_si256((const __m256i*)&d[2 * p + 1][16 * cg]);
            lo[p] = _mm256_unpacklo_epi16(a, b);
            hi[p] = _mm256_unpackhi_epi16(a, b);
        }
        for (int m = 0; m < n; ++m) {
            __m256i al = _mm256_setzero_si256(), ah = _mm256_setzero_si256();
            for (int p = 0; p < pairs1; ++p) {
                const __m256i w = _mm256_set1_epi32(B.pair[m][p]);
                al = _mm256_add_epi32(al, _mm256_madd_epi16(lo[p], w));
                ah = _mm256_add_epi32(ah, _mm256_madd_epi16(hi[p], w));
            }
            al = _mm256_srai_epi32(_mm256_add_epi32(al, r64), 7);
            ah = _mm256_srai_epi32(_mm256_add_epi32(ah, r64), 7);
            _mm256_store_si256((__m256i*)&tmp[m][16 * cg], _mm256_packs_epi32(al, ah));
        }
    }
    const int pairs2 = (std::min(nx, n) + 1) / 2;  // columns >= nx of tmp are zero
    const __m256i radd = _mm256_set1_epi32(add2);
    for (int r = 0; r < n; ++r) {
        for (int mg = 0; mg < n / 16; ++mg) {
            __m256i al = _mm256_setzero_si256(), ah = _mm256_setzero_si256();
            for (int p = 0; p < pairs2; ++p) {
                const __m256i w = bcast_pair(tmp[r][2 * p], tmp[r][2 * p + 1]);
                const __m256i a = _mm256_load_si256((const __m256i*)&B.t[2 * p][16 * mg]);
                const __m256i b = _mm256_load_si256((const __m256i*)&B.t[2 * p + 1][16 * mg]);
                al = _mm256_add_epi32(al, _mm256_madd_epi16(_mm256_unpacklo_epi16(a, b), w));
                ah = _mm256_add_epi32(ah, _mm256_madd_epi16(_mm256_unpackhi_epi16(a, b), w));
            }
            al = _mm256_srai_epi32(_mm256_add_epi32(al, radd), shift2);
            ah = _mm256_srai_epi32(_mm256_add_epi32(ah, radd), shift2);
            if (i16s) {  // the 8-bit path keeps the residual as i16 (wrapping)
                al = _mm256_srai_epi32(_mm256_slli_epi32(al, 16), 16);
                ah = _mm256_srai_epi32(_mm256_slli_epi32(ah, 16), 16);
            }
            // al = m 0-3 | 8-11, ah = m 4-7 | 12-15 of the group
            int32_t* o = out + r * n + 16 * mg;
            _mm256_storeu_si256((__m256i*)o, _mm256_permute2x128_si256(al, ah, 0x20));
            _mm256_storeu_si256((__m256i*)(o + 8), _mm256_permute2x128_si256(al, ah, 0x31));
        }
    }
}

void add_residual(uint16_t* dst, int stride, const uint16_t* pred, const int32_t* res, int n, int valid_w,
                  int valid_h, int bd) {
    valid_w = std::min(std::min(valid_w, n), stride);
    valid_h = std::min(valid_h, n);
    const int mx = bd == 0 ? 0 : (bd <= 15 ? (1 << bd) - 1 : 65535);
    const __m256i vmx = _mm256_set1_epi32(mx), zero = _mm256_setzero_si256();
    for (int y = 0; y < valid_h; ++y) {
        int x = 0;
        for (; x + 8 <= valid_w; x += 8) {
            const __m256i p = _mm256_cvtepu16_epi32(_mm_loadu_si128((const __m128i*)(pred + y * n + x)));
            const __m256i r = _mm256_loadu_si256((const __m256i*)(res + y * n + x));
            const __m256i v = _mm256_min_epi32(_mm256_max_epi32(_mm256_add_epi32(p, r), zero), vmx);
            const __m256i pk = _mm256_permute4x64_epi64(_mm256_packus_epi32(v, v), 0x08);
            _mm_storeu_si128((__m128i*)(dst + y * stride + x), _mm256_castsi256_si128(pk));
        }
        for (; x < valid_w; ++x) {
            const int v = pred[y * n + x] + res[y * n + x];
            dst[y * stride + x] = (uint16_t)(v < 0 ? 0 : (v > mx ? mx : v));
        }
    }
}

namespace {
constexpr int kAngle[33] = {32,  26,  21,  17,  13,  9,  5,  2,  0,  -2, -5,  -9,  -13, -17, -21, -26, -32,
                            -26, -21, -17, -13, -9,  -5, -2, 0,  2,  5,  9,   13,  17,  21,  26,  32};
constexpr int kInv[15] = {-4096, -1638, -910, -630, -482, -390, -315, -256,
                          -315,  -390,  -482, -630, -910, -1638, -4096};

inline __m128i pack8(__m256i v) {  // 8 int32 in [0, 65535] -> 8 uint16
    return _mm256_castsi256_si128(_mm256_permute4x64_epi64(_mm256_packus_epi32(v, v), 0x08));
}
}  // namespace

void intra_predict(int mode, const uint16_t* above, const uint16_t* left, int n, bool is_luma, int bd,
                   uint16_t* out) {
    int log2n = 0;
    while ((1 << log2n) < n) ++log2n;
    const int max_v = std::max((1 << bd) - 1, 0);
    if (mode == 0) {  // planar
        const int tr = above[n + 1], bl = left[n + 1];
        for (int y = 0; y < n; ++y) {
            int x = 0;
            if (n >= 8) {
                const __m256i ly = _mm256_set1_epi32(left[y + 1]), trv = _mm256_set1_epi32(tr);
                const __m256i wy = _mm256_set1_epi32(n - 1 - y), by = _mm256_set1_epi32((y + 1) * bl);
                for (; x + 8 <= n; x += 8) {
                    const __m256i xs = _mm256_add_epi32(_mm256_set1_epi32(x), _mm256_setr_epi32(0, 1, 2, 3, 4, 5, 6, 7));
                    const __m256i ab = _mm256_cvtepu16_epi32(_mm_loadu_si128((const __m128i*)(above + x + 1)));
                    const __m256i h = _mm256_add_epi32(
                        _mm256_mullo_epi32(_mm256_sub_epi32(_mm256_set1_epi32(n - 1), xs), ly),
                        _mm256_mullo_epi32(_mm256_add_epi32(xs, _mm256_set1_epi32(1)), trv));
                    const __m256i v = _mm256_add_epi32(_mm256_mullo_epi32(wy, ab), by);
                    const __m256i s = _mm256_srai_epi32(_mm256_add_epi32(_mm256_add_epi32(h, v), _mm256_set1_epi32(n)),
                                                        log2n + 1);
                    _mm_storeu_si128((__m128i*)(out + y * n + x), pack8(s));
                }
            }
            for (; x < n; ++x) {
                const int h = (n - 1 - x) * left[y + 1] + (x + 1) * tr;
                const int v = (n - 1 - y) * above[x + 1] + (y + 1) * bl;
                out[y * n + x] = (uint16_t)((h + v + n) >> (log2n + 1));
            }
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
    const int angle = kAngle[mode - 2];
    const bool vertical = mode >= 18;
    const uint16_t* main_ref = vertical ? above : left;
    const uint16_t* side = vertical ? left : above;
    alignas(32) int32_t refs[3 * 32 + 8];
    const int base = n;
    for (int i = 0; i <= 2 * n; ++i) refs[n + i] = main_ref[i];
    if (angle < 0) {
        const int inv = kInv[mode - 11];
        const int lim = (n * angle) >> 5;
        for (int k = -1; k >= lim; --k) {
            const int idx = std::min((k * inv + 128) >> 8, 2 * n);
            refs[k + base] = side[std::max(idx, 0)];
        }
    }
    alignas(32) uint16_t blk[32 * 32];  // [a][b]: a = row (vertical) or column (horizontal)
    const __m256i vmax = _mm256_set1_epi32(max_v), zero = _mm256_setzero_si256(), r16 = _mm256_set1_epi32(16);
    for (int a = 0; a < n; ++a) {
        const int pos = (a + 1) * angle;
        const int i_idx = pos >> 5, frac = pos & 31;
        uint16_t* row = (vertical ? out : blk) + a * n;
        int b = 0;
        for (; b + 8 <= n; b += 8) {
            const __m256i r0 = _mm256_loadu_si256((const __m256i*)(refs + b + i_idx + 1 + base));
            __m256i v = r0;
            if (frac) {
                const __m256i r1 = _mm256_loadu_si256((const __m256i*)(refs + b + i_idx + 2 + base));
                v = _mm256_srai_epi32(_mm256_add_epi32(_mm256_add_epi32(_mm256_mullo_epi32(r0, _mm256_set1_epi32(32 - frac)),
                                                                        _mm256_mullo_epi32(r1, _mm256_set1_epi32(frac))),
                                                       r16),
                                      5);
            }
            v = _mm256_min_epi32(_mm256_max_epi32(v, zero), vmax);
            _mm_storeu_si128((__m128i*)(row + b), pack8(v));
        }
        for (; b < n; ++b) {
            const int r0 = refs[b + i_idx + 1 + base];
            int v = r0;
            if (frac) v = ((32 - frac) * r0 + frac * refs[b + i_idx + 2 + base] + 16) >> 5;
            row[b] = (uint16_t)std::min(std::max(v, 0), max_v);
        }
    }
    if (!vertical)
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b) out[b * n + a] = blk[a * n + b];
    if (is_luma && n < 32) {
        if (mode == 26) {
            for (int y = 0; y < n; ++y) {
                const int v = above[1] + ((left[y + 1] - above[0]) >> 1);
                out[y * n] = (uint16_t)std::min(std::max(v, 0), max_v);
            }
        } else if (mode == 10) {
            for (int x = 0; x < n; ++x) {
                const int v = left[1] + ((above[x + 1] - above[0]) >> 1);
                out[x] = (uint16_t)std::min(std::max(v, 0), max_v);
            }
        }
    }
}

// Offset of edge index e (0..4, 2 = none) or band index rel (0..3) by
// comparisons; samples are below 2^15, so int16 lanes hold them.
void sao_band(uint16_t* dst, const uint16_t* src, int w, int x0, int y0, int x_end, int y_end,
              const int32_t* off, int band_pos, int bd) {
    const int mx = (1 << bd) - 1;
    const int shift = bd - 5;
    const __m256i vmx = _mm256_set1_epi16((int16_t)mx), zero = _mm256_setzero_si256();
    const __m256i bp = _mm256_set1_epi16((int16_t)band_pos);
    const __m256i o0 = _mm256_set1_epi16((int16_t)off[0]), o1 = _mm256_set1_epi16((int16_t)off[1]);
    const __m256i o2 = _mm256_set1_epi16((int16_t)off[2]), o3 = _mm256_set1_epi16((int16_t)off[3]);
    for (int y = y0; y < y_end; ++y) {
        int x = x0;
        for (; x + 16 <= x_end; x += 16) {
            const __m256i s = _mm256_loadu_si256((const __m256i*)(src + (size_t)y * w + x));
            const __m256i rel = _mm256_sub_epi16(_mm256_srli_epi16(s, shift), bp);  // |rel| < 32
            __m256i o = _mm256_and_si256(_mm256_cmpeq_epi16(rel, _mm256_set1_epi16(0)), o0);
            o = _mm256_or_si256(o, _mm256_and_si256(_mm256_cmpeq_epi16(rel, _mm256_set1_epi16(1)), o1));
            o = _mm256_or_si256(o, _mm256_and_si256(_mm256_cmpeq_epi16(rel, _mm256_set1_epi16(2)), o2));
            o = _mm256_or_si256(o, _mm256_and_si256(_mm256_cmpeq_epi16(rel, _mm256_set1_epi16(3)), o3));
            const __m256i in_band = _mm256_and_si256(_mm256_cmpgt_epi16(rel, _mm256_set1_epi16(-1)),
                                                     _mm256_cmpgt_epi16(_mm256_set1_epi16(4), rel));
            const __m256i v = _mm256_min_epi16(_mm256_max_epi16(_mm256_add_epi16(s, o), zero), vmx);
            const __m256i old = _mm256_loadu_si256((const __m256i*)(dst + (size_t)y * w + x));
            _mm256_storeu_si256((__m256i*)(dst + (size_t)y * w + x), _mm256_blendv_epi8(old, v, in_band));
        }
        for (; x < x_end; ++x) {
            const int s = src[(size_t)y * w + x];
            const uint8_t rel = (uint8_t)((uint8_t)(s >> shift) - (uint8_t)band_pos);
            if (rel < 4) {
                const int v = s + off[rel];
                dst[(size_t)y * w + x] = (uint16_t)(v < 0 ? 0 : (v > mx ? mx : v));
            }
        }
    }
}

void sao_edge(uint16_t* dst, const uint16_t* src, int w, int h, int x0, int y0, int x_end, int y_end,
              const int32_t* off, int eo_class, int bd) {
    const int mx = (1 << bd) - 1;
    int dx, dy;
    switch (eo_class) {
        case 0: dx = 1; dy = 0; break;
        case 1: dx = 0; dy = 1; break;
        case 2: dx = 1; dy = 1; break;
        default: dx = 1; dy = -1; break;
    }
    const __m256i vmx = _mm256_set1_epi16((int16_t)mx), zero = _mm256_setzero_si256();
    const __m256i o0 = _mm256_set1_epi16((int16_t)off[0]), o1 = _mm256_set1_epi16((int16_t)off[1]);
    const __m256i o2 = _mm256_set1_epi16((int16_t)off[2]), o3 = _mm256_set1_epi16((int16_t)off[3]);
    const __m256i one = _mm256_set1_epi16(1);
    auto scalar = [&](int x, int y) {
        const int s = src[(size_t)y * w + x];
        const int x1 = x + dx, y1 = y + dy, x2 = x - dx, y2 = y - dy;
        if (x1 < 0 || y1 < 0 || x1 >= w || y1 >= h || x2 < 0 || y2 < 0 || x2 >= w || y2 >= h) return;
        const int n1 = src[(size_t)y1 * w + x1], n2 = src[(size_t)y2 * w + x2];
        const int e = ((s > n1) - (s < n1)) + ((s > n2) - (s < n2)) + 2;
        const int o = e == 0 ? off[0] : (e == 1 ? off[1] : (e == 3 ? off[2] : (e == 4 ? off[3] : 0)));
        if (o) {
            const int v = s + o;
            dst[(size_t)y * w + x] = (uint16_t)(v < 0 ? 0 : (v > mx ? mx : v));
        }
    };
    for (int y = y0; y < y_end; ++y) {
        if (y + dy < 0 || y + dy >= h || y - dy < 0 || y - dy >= h) continue;  // picture border rows
        const int xa = std::max(x0, dx), xb = std::min(x_end, w - dx);  // columns with both neighbours
        int x = x0;
        for (; x < std::min(xa, x_end); ++x) scalar(x, y);
        for (; x + 16 <= xb; x += 16) {
            const __m256i s = _mm256_loadu_si256((const __m256i*)(src + (size_t)y * w + x));
            const __m256i n1 = _mm256_loadu_si256((const __m256i*)(src + (size_t)(y + dy) * w + x + dx));
            const __m256i n2 = _mm256_loadu_si256((const __m256i*)(src + (size_t)(y - dy) * w + x - dx));
            // sign(s - n) = (s > n) - (s < n): cmpgt gives -1 / 0
            const __m256i e = _mm256_add_epi16(
                _mm256_add_epi16(_mm256_sub_epi16(_mm256_cmpgt_epi16(n1, s), _mm256_cmpgt_epi16(s, n1)),
                                 _mm256_sub_epi16(_mm256_cmpgt_epi16(n2, s), _mm256_cmpgt_epi16(s, n2))),
                _mm256_set1_epi16(2));
            __m256i o = _mm256_and_si256(_mm256_cmpeq_epi16(e, zero), o0);
            o = _mm256_or_si256(o, _mm256_and_si256(_mm256_cmpeq_epi16(e, one), o1));
            o = _mm256_or_si256(o, _mm256_and_si256(_mm256_cmpeq_epi16(e, _mm256_set1_epi16(3)), o2));
            o = _mm256_or_si256(o, _mm256_and_si256(_mm256_cmpeq_epi16(e, _mm256_set1_epi16(4)), o3));
            const __m256i v = _mm256_min_epi16(_mm256_max_epi16(_mm256_add_epi16(s, o), zero), vmx);
            const __m256i keep = _mm256_cmpeq_epi16(o, zero);
            const __m256i old = _mm256_loadu_si256((const __m256i*)(dst + (size_t)y * w + x));
            _mm256_storeu_si256((__m256i*)(dst + (size_t)y * w + x), _mm256_blendv_epi8(v, old, keep));
        }
        for (; x < x_end; ++x) scalar(x, y);
    }
}

void rgb_row(const uint16_t* Y, const uint16_t* Cb, const uint16_t* Cr, int x_first, int count, int width, int cw,
             int sub_w, int bd, int32_t k_y, int32_t y_black, int32_t neutral, int32_t cr_to_r, int32_t cb_to_g,
             int32_t cr_to_g, int32_t cb_to_b, int32_t cmax, uint16_t* out) {
    (void)bd;
    auto pixel = [&](int i) {
        const int sx = x_first + i;
        const int xc = std::min(sx, width - 1), cc = std::min(sx / sub_w, cw - 1);
        const int yv = k_y * (Y[xc] - y_black), cbc = Cb[cc] - neutral, crc = Cr[cc] - neutral;
        int r = (yv + cr_to_r * crc + 4096) >> 13;
        int g = (yv + cb_to_g * cbc + cr_to_g * crc + 4096) >> 13;
        int b = (yv + cb_to_b * cbc + 4096) >> 13;
        out[3 * i] = (uint16_t)std::min(std::max(r, 0), cmax);
        out[3 * i + 1] = (uint16_t)std::min(std::max(g, 0), cmax);
        out[3 * i + 2] = (uint16_t)std::min(std::max(b, 0), cmax);
    };
    const __m256i ky = _mm256_set1_epi32(k_y), yb = _mm256_set1_epi32(y_black), nt = _mm256_set1_epi32(neutral);
    const __m256i cr_r = _mm256_set1_epi32(cr_to_r), cb_g = _mm256_set1_epi32(cb_to_g);
    const __m256i cr_g = _mm256_set1_epi32(cr_to_g), cb_b = _mm256_set1_epi32(cb_to_b);
    const __m256i rnd = _mm256_set1_epi32(4096), zero = _mm256_setzero_si256(), vmax = _mm256_set1_epi32(cmax);
    const __m256i dup = _mm256_setr_epi32(0, 0, 1, 1, 2, 2, 3, 3);
    int i = 0;
    for (; i + 8 <= count; i += 8) {
        const int sx = x_first + i;
        if (sx + 7 >= width || (sx + 7) / sub_w >= cw || (sub_w == 2 && (sx & 1))) break;  // edge or odd start
        const __m256i yl = _mm256_cvtepu16_epi32(_mm_loadu_si128((const __m128i*)(Y + sx)));
        __m256i cb, cr;
        if (sub_w == 2) {
            cb = _mm256_permutevar8x32_epi32(_mm256_cvtepu16_epi32(_mm_loadl_epi64((const __m128i*)(Cb + sx / 2))), dup);
            cr = _mm256_permutevar8x32_epi32(_mm256_cvtepu16_epi32(_mm_loadl_epi64((const __m128i*)(Cr + sx / 2))), dup);
        } else {
            cb = _mm256_cvtepu16_epi32(_mm_loadu_si128((const __m128i*)(Cb + sx)));
            cr = _mm256_cvtepu16_epi32(_mm_loadu_si128((const __m128i*)(Cr + sx)));
        }
        const __m256i yv = _mm256_mullo_epi32(ky, _mm256_sub_epi32(yl, yb));
        const __m256i cbc = _mm256_sub_epi32(cb, nt), crc = _mm256_sub_epi32(cr, nt);
        __m256i r = _mm256_srai_epi32(_mm256_add_epi32(_mm256_add_epi32(yv, _mm256_mullo_epi32(cr_r, crc)), rnd), 13);
        __m256i g = _mm256_srai_epi32(
            _mm256_add_epi32(_mm256_add_epi32(_mm256_add_epi32(yv, _mm256_mullo_epi32(cb_g, cbc)), _mm256_mullo_epi32(cr_g, crc)),
                             rnd),
            13);
        __m256i b = _mm256_srai_epi32(_mm256_add_epi32(_mm256_add_epi32(yv, _mm256_mullo_epi32(cb_b, cbc)), rnd), 13);
        r = _mm256_min_epi32(_mm256_max_epi32(r, zero), vmax);
        g = _mm256_min_epi32(_mm256_max_epi32(g, zero), vmax);
        b = _mm256_min_epi32(_mm256_max_epi32(b, zero), vmax);
        alignas(32) int32_t rr[8], gg[8], bb[8];
        _mm256_store_si256((__m256i*)rr, r);
        _mm256_store_si256((__m256i*)gg, g);
        _mm256_store_si256((__m256i*)bb, b);
        for (int k = 0; k < 8; ++k) {
            out[3 * (i + k)] = (uint16_t)rr[k];
            out[3 * (i + k) + 1] = (uint16_t)gg[k];
            out[3 * (i + k) + 2] = (uint16_t)bb[k];
        }
    }
    for (; i < count; ++i) pixel(i);
}

}  // namespace orc_simd
