// recon.cu -- reconstruction of the transform-block records of a batch of
// pictures: dequantisation + inverse DCT/DST / transform skip / transquant
// bypass (transform.rs), intra prediction (intra.rs) and residual add + clip
// (reconstruct.rs), in the decode order of decode.rs:3478-5426.
//
// Two kernels:
//
//  k_residual -- every coded TB of every picture, fully parallel (one warp
//     per TB).  TBs whose prediction is already in the plane (inter TBs,
//     prediction-in-plane pictures) are added and clipped into the plane
//     right away; intra TBs leave an int16 residual in a residual plane.
//     (int16 is exact: for 8-bit the reference itself truncates to i16,
//     transform.rs:55-63; above 8 bits a residual outside +-32767 saturates
//     the clip to [0, 2^bd - 1] exactly as the unsaturated one does.)
//
//  k_recon -- the intra wavefront.  One CTA reconstructs one CTU at a time;
//     CTUs are claimed from a global queue sorted by wavefront index
//     (x + 2y) across all pictures, so a CTU is only claimed after every CTU
//     it depends on (left, above-left, above, above-right) was claimed by a
//     running CTA: no deadlock for any grid size.  Per CTU the residuals and
//     records are staged with cp.async, then luma, Cb and Cr are walked by
//     three warps in parallel (chroma availability only depends on the luma
//     `decoded` map, which each warp replays from the records), all in
//     shared memory.  Neighbours synchronise per component and quadrant:
//     each walking warp releases how many quadrants of its CTU are done once
//     their right-column / bottom-row samples are in the plane, and reads a
//     neighbour's edge segment only when a TB on its own top or left edge
//     needs it (waits bounded), so a CTU starts while its left and
//     above-right neighbours are still being walked.  Finally the whole CTU
//     is written out for the filters.
#include <mutex>
#include <climits>

#include "common.cuh"

namespace hpvcd {

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

constexpr int kScr = 33;  // padded row stride of the transform scratch
// Inverse-transform variants of k_residual (schedule knob; pixels identical).
constexpr int kIdctMatrix = 0;     // matrix product, all-zero rows / columns skipped
constexpr int kIdctButterfly = 1;  // even-odd butterflies for 16x16 and 32x32 TBs
constexpr int kIdctTensor = 2;     // integer tensor-core products (int8 halves) for 16x16 and 32x32 TBs

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

__device__ __forceinline__ int sat16(int v) { return v < -32768 ? -32768 : (v > 32767 ? 32767 : v); }

// The same basis entry as a compile-time constant, for fully unrolled
// butterflies (the multiplier becomes an immediate operand).
__host__ __device__ constexpr int dct_c(int n, int k, int m) {
    constexpr int8_t mag[33] = {64, 90, 90, 90, 89, 88, 87, 85, 83, 82, 80, 78, 75, 73, 70, 67, 64,
                                61, 57, 54, 50, 46, 43, 38, 36, 31, 25, 22, 18, 13, 9,  4,  0};
    if (k == 0) return 64;
    int j = (k * (32 / n) * (2 * m + 1)) & 127;
    int sign = 1;
    if (j > 64) j = 128 - j;
    if (j > 32) {
        j = 64 - j;
        sign = -1;
    }
    return sign * mag[j];
}

// Even-odd (partial butterfly) N-point inverse: out[m] = sum_{k < KMAX}
// T_N[k][m] * in[k * S].  Rows of the basis are symmetric for even k and
// antisymmetric for odd k, and T_N[2j][m] = T_{N/2}[j][m], so the even
// coefficients form an N/2-point inverse and out[N-1-m] = E[m] - O[m].
// Integer sums in any order are identical, so the result equals the matrix
// product bit for bit (the clip follows the complete sum in both forms).
template <int N, int S, int KMAX>
__device__ __forceinline__ void inv_butterfly(const int* in, int* out) {
    if constexpr (N == 1) {
        out[0] = KMAX > 0 ? 64 * in[0] : 0;
    } else {
        int e[N / 2];
        inv_butterfly<N / 2, 2 * S, (KMAX + 1) / 2>(in, e);
#pragma unroll
        for (int m = 0; m < N / 2; ++m) {
            int o = 0;
#pragma unroll
            for (int k = 1; k < KMAX && k < N; k += 2) o += dct_c(N, k, m) * in[k * S];
            out[m] = e[m] + o;
            out[N - 1 - m] = e[m] - o;
        }
    }
}

// One stage of a 16- or 32-point inverse by butterflies, lane = line:
// line l reads in[k] = src[l * ls + k * ks] for k < KMAX (the rest are zero)
// and writes dst[l * ld + m * md] = fin(out[m]).
template <int N, int KMAX, typename Fin>
__device__ __forceinline__ void bf_stage(const int16_t* src, int ls, int ks, int16_t* dst, int ld, int md, int lane,
                                         Fin fin) {
    if (lane >= N) return;
    int in[KMAX], out[N];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) in[k] = src[lane * ls + k * ks];
    inv_butterfly<N, 1, KMAX>(in, out);
#pragma unroll
    for (int m = 0; m < N; ++m) dst[lane * ld + m * md] = (int16_t)fin(out[m]);
}

template <int N, typename Fin>
__device__ __forceinline__ void bf_stage_k(int kcount, const int16_t* src, int ls, int ks, int16_t* dst, int ld,
                                           int md, int lane, Fin fin) {
    if (kcount <= 4)
        bf_stage<N, 4>(src, ls, ks, dst, ld, md, lane, fin);
    else if (kcount <= 8)
        bf_stage<N, 8>(src, ls, ks, dst, ld, md, lane, fin);
    else if (N == 16 || kcount <= 16)
        bf_stage<N, (N < 16 ? N : 16)>(src, ls, ks, dst, ld, md, lane, fin);
    else
        bf_stage<N, N>(src, ls, ks, dst, ld, md, lane, fin);
}

// ===========================================================================
// Integer tensor-core inverse transform of 16x16 and 32x32 TBs.
//
// Both stages are products with the H.265 basis T (entries in [-90, 90], an
// s8 value): stage 1 tmp = T^T * D over the dequantised coefficients D,
// stage 2 out = tmp * T.  The int16 operand X of each product is split
// exactly into a signed high byte and an unsigned low byte, X = 256 * hi +
// lo, and the product is 256 * (T * hi) + (T * lo): two mma.sync products
// with s32 accumulation.  No sum overflows (|sum| <= 32 * 90 * 32768 <
// 2^31), so the result is the reference's integer sum bit for bit; the
// rounding, shift and clip of each stage are applied to it unchanged.
// Fragments follow the PTX layouts of mma.m16n8k32 (32x32 TBs) and
// mma.m16n8k16 (16x16 TBs) with 8-bit operands: lane = 4 * group + t; an A
// register holds four consecutive K entries of one row (row group or group
// + 8), a B register four consecutive K entries of one column (group), a
// C/D register pair two adjacent columns (2t, 2t + 1) of one row.
// ===========================================================================
__device__ __forceinline__ void mma32(int (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1, bool a_u8,
                                      bool b_u8) {
    // D += A * B, A 16x32 (row), B 32x8 (col), 8-bit operands, s32 accumulation
    if (!a_u8 && !b_u8)
        asm volatile("mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                     "{%0,%1,%2,%3};"
                     : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
                     : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    else if (!a_u8)
        asm volatile("mma.sync.aligned.m16n8k32.row.col.s32.s8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                     "{%0,%1,%2,%3};"
                     : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
                     : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    else
        asm volatile("mma.sync.aligned.m16n8k32.row.col.s32.u8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                     "{%0,%1,%2,%3};"
                     : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
                     : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ void mma16(int (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0, bool a_u8, bool b_u8) {
    // D += A * B, A 16x16 (row), B 16x8 (col), 8-bit operands, s32 accumulation
    if (!a_u8 && !b_u8)
        asm volatile("mma.sync.aligned.m16n8k16.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                     : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
                     : "r"(a0), "r"(a1), "r"(b0));
    else if (!a_u8)
        asm volatile("mma.sync.aligned.m16n8k16.row.col.s32.s8.u8.s32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                     : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
                     : "r"(a0), "r"(a1), "r"(b0));
    else
        asm volatile("mma.sync.aligned.m16n8k16.row.col.s32.u8.s8.s32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                     : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
                     : "r"(a0), "r"(a1), "r"(b0));
}

// Basis fragments, per lane, in shared memory (index [entry][lane]):
//   s1a32: T^T as the A operand of stage 1, 32x32: 2 row tiles x 4 registers
//   s2b32: T as the B operand of stage 2, 32x32: 4 column tiles x 2 registers
//   s1a16: T^T, 16x16: 2 registers;  s2b16: T, 16x16: 2 column tiles x 1 register
constexpr int kFragS1A32 = 0, kFragS2B32 = 8, kFragS1A16 = 16, kFragS2B16 = 18, kFragEntries = 20;

__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
    return (uint32_t)(a & 0xff) | ((uint32_t)(b & 0xff) << 8) | ((uint32_t)(c & 0xff) << 16) | ((uint32_t)(d & 0xff) << 24);
}

__device__ void build_basis_frags(uint32_t* frags, int tid, int nthreads) {
    for (int e = tid; e < kFragEntries * 32; e += nthreads) {
        const int entry = e >> 5, lane = e & 31, g = lane >> 2, t = lane & 3;
        int v[4];
        if (entry < kFragS2B32) {  // A of stage 1, n = 32: A[m][k] = T[k][m]
            const int mt = entry >> 2, reg = entry & 3;
            const int m = mt * 16 + g + (reg & 1) * 8, k0 = (reg >> 1) * 16 + 4 * t;
            for (int i = 0; i < 4; ++i) v[i] = dct_entry(32, k0 + i, m);
        } else if (entry < kFragS1A16) {  // B of stage 2, n = 32: B[k][m] = T[k][m]
            const int nt = (entry - kFragS2B32) >> 1, reg = (entry - kFragS2B32) & 1;
            const int m = nt * 8 + g, k0 = reg * 16 + 4 * t;
            for (int i = 0; i < 4; ++i) v[i] = dct_entry(32, k0 + i, m);
        } else if (entry < kFragS2B16) {  // A of stage 1, n = 16
            const int reg = entry - kFragS1A16;
            const int m = g + reg * 8, k0 = 4 * t;
            for (int i = 0; i < 4; ++i) v[i] = dct_entry(16, k0 + i, m);
        } else {  // B of stage 2, n = 16
            const int nt = entry - kFragS2B16;
            const int m = nt * 8 + g, k0 = 4 * t;
            for (int i = 0; i < 4; ++i) v[i] = dct_entry(16, k0 + i, m);
        }
        frags[e] = pack4(v[0], v[1], v[2], v[3]);
    }
}

// Four int16 values split into their high bytes (s8) and low bytes (u8).
__device__ __forceinline__ void split4(int a, int b, int c, int d, uint32_t& hi, uint32_t& lo) {
    hi = pack4(a >> 8, b >> 8, c >> 8, d >> 8);
    lo = pack4(a, b, c, d);
}

// Both stages of an n x n (16 or 32) inverse DCT by one warp: buf holds the
// dequantised coefficients (row k, column c, stride kScr), tmp receives
// stage 1; emit(r, m, v) gets every output with the reference's storage.
template <int N, typename Emit>
__device__ __forceinline__ void idct_tensor(const int16_t* buf, int16_t* tmp, const uint32_t* frags, int bd, bool i16s,
                                            int lane, Emit emit) {
    constexpr int MT = N / 16, NT = N / 8;  // row tiles, column tiles
    const int g = lane >> 2, t = lane & 3;
    // ---- stage 1: tmp[m][c] = clip((sum_k T[k][m] D[k][c] + 64) >> 7) ----
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
        const int c = nt * 8 + g;
        uint32_t bh[2], bl[2];
#pragma unroll
        for (int reg = 0; reg < (N == 32 ? 2 : 1); ++reg) {
            const int k0 = reg * 16 + 4 * t;
            split4(buf[k0 * kScr + c], buf[(k0 + 1) * kScr + c], buf[(k0 + 2) * kScr + c], buf[(k0 + 3) * kScr + c],
                   bh[reg], bl[reg]);
        }
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            int dh[4] = {0, 0, 0, 0}, dl[4] = {0, 0, 0, 0};
            if constexpr (N == 32) {
                const uint32_t a[4] = {frags[(kFragS1A32 + mt * 4 + 0) * 32 + lane], frags[(kFragS1A32 + mt * 4 + 1) * 32 + lane],
                                       frags[(kFragS1A32 + mt * 4 + 2) * 32 + lane], frags[(kFragS1A32 + mt * 4 + 3) * 32 + lane]};
                mma32(dh, a, bh[0], bh[1], false, false);
                mma32(dl, a, bl[0], bl[1], false, true);
            } else {
                const uint32_t a0 = frags[(kFragS1A16 + 0) * 32 + lane], a1 = frags[(kFragS1A16 + 1) * 32 + lane];
                mma16(dh, a0, a1, bh[0], false, false);
                mma16(dl, a0, a1, bl[0], false, true);
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int m = mt * 16 + g + (e >> 1) * 8, cc = nt * 8 + 2 * t + (e & 1);
                const int acc = dh[e] * 256 + dl[e];
                tmp[m * kScr + cc] = (int16_t)clamp3i((acc + 64) >> 7, -32768, 32767);
            }
        }
    }
    __syncwarp();
    // ---- stage 2: out[r][m] = (sum_k tmp[r][k] T[k][m] + add2) >> shift2 ----
    const int shift2 = 20 - bd;
    const int add2 = 1 << (shift2 - 1);
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
        uint32_t ah[4], al[4];
#pragma unroll
        for (int reg = 0; reg < (N == 32 ? 4 : 2); ++reg) {
            const int r = mt * 16 + g + (reg & 1) * 8, k0 = (reg >> 1) * 16 + 4 * t;
            const int16_t* row = tmp + r * kScr + k0;
            split4(row[0], row[1], row[2], row[3], ah[reg], al[reg]);
        }
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            int dh[4] = {0, 0, 0, 0}, dl[4] = {0, 0, 0, 0};
            if constexpr (N == 32) {
                const uint32_t b0 = frags[(kFragS2B32 + nt * 2 + 0) * 32 + lane], b1 = frags[(kFragS2B32 + nt * 2 + 1) * 32 + lane];
                mma32(dh, ah, b0, b1, false, false);
                mma32(dl, al, b0, b1, true, false);
            } else {
                const uint32_t b0 = frags[(kFragS2B16 + nt) * 32 + lane];
                mma16(dh, ah[0], ah[1], b0, false, false);
                mma16(dl, al[0], al[1], b0, true, false);
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = mt * 16 + g + (e >> 1) * 8, m = nt * 8 + 2 * t + (e & 1);
                const int v = (dh[e] * 256 + dl[e] + add2) >> shift2;
                emit(r, m, i16s ? (int)(int16_t)v : v);
            }
        }
    }
    __syncwarp();
}

// ===========================================================================
// k_residual
// ===========================================================================
constexpr int kResWarps = 8;

// Residual of one coded TB by one warp (transform.rs:489-858, decode.rs
// :4754-4903 luma, :5313-5417 chroma).  `emit(r, m, v)` receives every
// residual sample (row r, column m) in the reference's storage semantics.
// `allow16` false keeps 8-bit residuals in i32 storage (the reference's
// path for chroma TBs with cross-component prediction, decode.rs:5313-5316).
template <int kIdct, typename Emit>
__device__ void tb_residual_warp(const DevPic& P, const hpvcd_tu& t, const int16_t* dct, int16_t* buf,
                                 int16_t* tmp, int lane, Emit emit, bool allow16 = true,
                                 const uint32_t* frags = nullptr) {
    const int n = 1 << t.log2n;
    const bool luma = t.comp == 0;
    const int bd = luma ? P.bd : P.bd_c;
    const bool i16s = bd <= 8 && allow16;
    // levels: int16, or int8 when the host narrowed the picture's pool
    const bool c8 = (P.flags & HPVCD_PIC_COEFF8) != 0;
    const int16_t* lv16 = P.coeffs + t.coeff_off;
    const int8_t* lv8 = (const int8_t*)P.coeffs + t.coeff_off;
    auto lv = [&](int i) -> int { return c8 ? (int)lv8[i] : (int)lv16[i]; };
    const uint32_t rext = t.flags & (HPVCD_TU_ROTATE | HPVCD_TU_RDPCM_H | HPVCD_TU_RDPCM_V);
    // decode.rs:4754-4757 / :4830-4834: residual = levels (transquant bypass);
    // an I_PCM record's levels are its samples (decode.rs:2768-2839)
    if ((t.flags & (HPVCD_TU_TQB | HPVCD_TU_PCM)) && !rext) {
        for (int i = lane; i < n * n; i += 32) emit(i / n, i % n, (int)lv(i));
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
    const int qs = clamp3i(qpp, 0, 51 + 6 * (bd - 8));
    const long long base = (long long)c_dequant_scale[qs % 6] * (1ll << (qs / 6));
    const long long add = 1ll << (bd_shift - 1);
    // Scaling lists (decode.rs:5874-5899, transform.rs:668-683): the factor
    // of coefficient (r, c) is base * m(r, c) instead of base * 16; 4x4
    // lists index the 4x4 raster, larger TBs the 8x8 list upsampled, with
    // the DC entry for 16x16 and 32x32.  Transform-skip TBs above 4x4 stay
    // flat.
    const uint8_t* sm = nullptr;
    int sdc = 16;
    if (P.scaling && (!(t.flags & HPVCD_TU_TSKIP) || n == 4)) {
        const int size_id = t.log2n - 2;
        const int matrix_id = min((int)t.comp, 2) + ((t.flags & HPVCD_TU_INTRA) ? 0 : 3);
        sm = P.scaling->m[size_id][matrix_id];
        sdc = P.scaling->dc[size_id][matrix_id];
    }
    const int down = t.log2n > 3 ? t.log2n - 3 : 0;
    auto factor_at = [&](int r, int c) -> long long {
        if (!sm) return base * 16;
        if (n == 4) return base * sm[r * 4 + c];
        if (n >= 16 && r == 0 && c == 0) return base * sdc;
        return base * sm[(r >> down) * 8 + (c >> down)];
    };
    if (rext && (t.flags & (HPVCD_TU_TSKIP | HPVCD_TU_TQB))) {
        // RExt residual modification (decode.rs:8418-8446): the TS / TQB
        // residual goes to int32 scratch (rotated: sample i from n*n-1-i),
        // then one lane per column (vertical RDPCM) or row (horizontal)
        // accumulates it.  At 8 bits the reference adds in wrapping i16;
        // the int32 sums wrapped once at the end are the same values.
        int32_t* r32 = reinterpret_cast<int32_t*>(buf);  // buf + tmp: 32 * kScr int32
        const int tr_shift = 15 - bd - t.log2n;
        const int tr_add = tr_shift > 0 ? 1 << (tr_shift - 1) : 0;
        const bool rot = (rext & HPVCD_TU_ROTATE) != 0;
        for (int i = lane; i < n * n; i += 32) {
            int r;
            if (t.flags & HPVCD_TU_TQB) {
                r = lv(i);
            } else {
                long long v = ((long long)lv(i) * factor_at(i / n, i % n) + add) >> bd_shift;
                v = v < -32768 ? -32768 : (v > 32767 ? 32767 : v);
                r = tr_shift >= 0 ? ((int)v + tr_add) >> tr_shift : (int)((unsigned)v << (-tr_shift));
            }
            r32[rot ? n * n - 1 - i : i] = r;
        }
        __syncwarp();
        if (lane < n) {
            if (rext & HPVCD_TU_RDPCM_V) {
                int acc = 0;
                for (int y = 0; y < n; ++y) r32[y * n + lane] = acc += r32[y * n + lane];
            } else if (rext & HPVCD_TU_RDPCM_H) {
                int acc = 0;
                for (int x = 0; x < n; ++x) r32[lane * n + x] = acc += r32[lane * n + x];
            }
        }
        __syncwarp();
        for (int i = lane; i < n * n; i += 32) {
            const int r = r32[i];
            emit(i / n, i % n, i16s ? (int)(int16_t)r : r);
        }
        __syncwarp();
        return;
    }
    if (t.flags & HPVCD_TU_TSKIP) {  // transform.rs:728-792
        const int tr_shift = 15 - bd - t.log2n;
        const int tr_add = tr_shift > 0 ? 1 << (tr_shift - 1) : 0;
        for (int i = lane; i < n * n; i += 32) {
            long long v = ((long long)lv(i) * factor_at(i / n, i % n) + add) >> bd_shift;
            v = v < -32768 ? -32768 : (v > 32767 ? 32767 : v);
            const int r = tr_shift >= 0 ? ((int)v + tr_add) >> tr_shift : (int)((unsigned)v << (-tr_shift));
            emit(i / n, i % n, i16s ? (int)(int16_t)r : r);
        }
        return;
    }
    const int nx = (t.nx == 0 || t.nx > n) ? n : t.nx;
    if (n == 4) {
        // 4x4 in registers: lane l < 16 holds coefficient (l / 4, l % 4); both
        // stages gather their four inputs by shuffles.  The same integer sums
        // as the shared-memory path, clipped after the complete sum.
        const bool dst = luma && (t.flags & HPVCD_TU_INTRA);
        const int l = lane & 15, r = l >> 2, c = l & 3;
        int d = 0;
        if (lane < 16 && c < nx) {
            const long long v = ((long long)lv(l) * factor_at(r, c) + add) >> bd_shift;
            d = (int)(v < -32768 ? -32768 : (v > 32767 ? 32767 : v));
        }
        // basis entry T[k][m] of the 4-point DCT (rows 64 / 83,36 / 64 / 36,83
        // with the H.265 signs) or of the DST
        auto basis = [dst](int k, int m) -> int {
            if (dst) return c_dst4[k][m];
            switch (k) {  // dct_c(4, k, m) without a lookup table
                case 0: return 64;
                case 1: return m == 0 ? 83 : (m == 1 ? 36 : (m == 2 ? -36 : -83));
                case 2: return (m == 0 || m == 3) ? 64 : -64;
                default: return m == 0 ? 36 : (m == 1 ? -83 : (m == 2 ? 83 : -36));
            }
        };
        // stage 1: tmp[r][c] = clip((sum_k T[k][r] d[k][c] + 64) >> 7)
        int acc = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) acc += basis(k, r) * __shfl_sync(0xffffffffu, d, k * 4 + c);
        const int tmp = clamp3i((acc + 64) >> 7, -32768, 32767);
        // stage 2: out[r][c] = (sum_k T[k][c] tmp[r][k] + add2) >> shift2
        const int shift2 = 20 - bd;
        int acc2 = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) acc2 += basis(k, c) * __shfl_sync(0xffffffffu, tmp, r * 4 + k);
        const int v = (acc2 + (1 << (shift2 - 1))) >> shift2;
        if (lane < 16) emit(r, c, i16s ? (int)(int16_t)v : v);
        __syncwarp();
        return;
    }
    // dequantise into buf; columns >= nx are zero (transform.rs:510-511);
    // track the last non-zero row so stage 1 skips all-zero rows.
    int my_rows = 0;
    for (int i = lane; i < n * n; i += 32) {
        const int r = i / n, c = i % n;
        int v = 0;
        if (c < nx) {
            const long long d = ((long long)lv(i) * factor_at(r, c) + add) >> bd_shift;
            v = (int)(d < -32768 ? -32768 : (d > 32767 ? 32767 : d));
        }
        buf[r * kScr + c] = (int16_t)v;
        if (v) my_rows = r + 1;
    }
    int rows = my_rows;
#pragma unroll
    for (int o = 16; o; o >>= 1) rows = max(rows, __shfl_xor_sync(0xffffffffu, rows, o));
    __syncwarp();
    const bool dst = luma && n == 4 && (t.flags & HPVCD_TU_INTRA);
    if (kIdct == kIdctTensor && n >= 16) {
        if (n == 16)
            idct_tensor<16>(buf, tmp, frags, bd, i16s, lane, emit);
        else
            idct_tensor<32>(buf, tmp, frags, bd, i16s, lane, emit);
        return;
    }
    if (kIdct == kIdctButterfly && n >= 16) {
        // stage 1, lane = column: rows >= `rows` are zero
        auto st1 = [](int acc) { return clamp3i((acc + 64) >> 7, -32768, 32767); };
        // stage 2, lane = row: columns >= nx are zero.  The output is kept
        // as int16 in buf: wrapped at 8 bits (the reference's i16 storage),
        // saturated above 8 bits (exact: a saturated residual clips a
        // sample to the same bound as the full value).
        const int shift2 = 20 - bd;
        const int add2 = 1 << (shift2 - 1);
        auto st2 = [=](int acc) {
            const int v = (acc + add2) >> shift2;
            return i16s ? (int)(int16_t)v : sat16(v);
        };
        if (n == 16) {
            bf_stage_k<16>(rows, buf, 1, kScr, tmp, 1, kScr, lane, st1);
            __syncwarp();
            bf_stage_k<16>(nx, tmp, kScr, 1, buf, kScr, 1, lane, st2);
        } else {
            bf_stage_k<32>(rows, buf, 1, kScr, tmp, 1, kScr, lane, st1);
            __syncwarp();
            bf_stage_k<32>(nx, tmp, kScr, 1, buf, kScr, 1, lane, st2);
        }
        __syncwarp();
        for (int i = lane; i < n * n; i += 32) {
            const int r = i / n, m = i % n;
            emit(r, m, (int)buf[r * kScr + m]);
        }
        __syncwarp();
        return;
    }
    const int step = 32 / n;
    // stage 1 (columns): tmp[m][c] = clip((sum_k T[k][m] * buf[k][c] + 64) >> 7)
    for (int i = lane; i < n * n; i += 32) {
        const int m = i / n, c = i % n;
        int acc = 0;
        if (dst) {
#pragma unroll
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
#pragma unroll
            for (int k = 0; k < 4; ++k) acc += c_dst4[k][m] * tmp[r * kScr + k];
        } else {
            for (int k = 0; k < kmax; ++k) acc += dct[(k * step) * 32 + m] * tmp[r * kScr + k];
        }
        const int v = (acc + add2) >> shift2;
        emit(r, m, i16s ? (int)(int16_t)v : v);
    }
    __syncwarp();
}

// Records per warp step of k_residual: a warp loads 32 consecutive records
// at once (one per lane, coalesced), finds their pictures in parallel and
// prefetches their coefficients into L2, then transforms them one by one.
constexpr int kResChunk = 32;

// Dequantisation scale m_levelScale[qs % 6] (transform.rs:701-725) without a
// table: lanes of one warp index it differently, which a constant-bank read
// would serialise.
__device__ __forceinline__ int level_scale(int r) {
    return r == 0 ? 40 : (r == 1 ? 45 : (r == 2 ? 51 : (r == 3 ? 57 : (r == 4 ? 64 : 72))));
}

// One 4-point inverse transform, DST-VII (kDst) or DCT, with the basis as
// immediates: o[m] = sum_k T[k][m] * in[k] (transform.rs:535-603 for the
// DST, :406-533 for the DCT; the H.265 matrices).
template <bool kDst>
__device__ __forceinline__ void inv4(int i0, int i1, int i2, int i3, int& o0, int& o1, int& o2, int& o3) {
    if (kDst) {
        o0 = 29 * i0 + 74 * i1 + 84 * i2 + 55 * i3;
        o1 = 55 * i0 + 74 * i1 - 29 * i2 - 84 * i3;
        o2 = 74 * i0 - 74 * i2 + 74 * i3;
        o3 = 84 * i0 - 74 * i1 + 55 * i2 - 29 * i3;
    } else {
        const int e0 = 64 * (i0 + i2), e1 = 64 * (i0 - i2);
        const int q0 = 83 * i1 + 36 * i3, q1 = 36 * i1 - 83 * i3;
        o0 = e0 + q0;
        o1 = e1 + q1;
        o2 = e1 - q1;
        o3 = e0 - q0;
    }
}

// Both stages of a 4x4 inverse transform in one thread's registers: d is
// the dequantised block (row k, column c at d[4k + c]); on return d holds
// the residual before the storage wrap.  Stage 1 (columns) clips
// (sum + 64) >> 7 to int16, stage 2 (rows) adds 2^(shift2 - 1) and shifts
// by shift2, the same sums as the warp path of tb_residual_warp.
template <bool kDst>
__device__ __forceinline__ void idct4_thread(int (&d)[16], int shift2) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        int o0, o1, o2, o3;
        inv4<kDst>(d[c], d[4 + c], d[8 + c], d[12 + c], o0, o1, o2, o3);
        d[c] = clamp3i((o0 + 64) >> 7, -32768, 32767);
        d[4 + c] = clamp3i((o1 + 64) >> 7, -32768, 32767);
        d[8 + c] = clamp3i((o2 + 64) >> 7, -32768, 32767);
        d[12 + c] = clamp3i((o3 + 64) >> 7, -32768, 32767);
    }
    const int add2 = 1 << (shift2 - 1);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        int o0, o1, o2, o3;
        inv4<kDst>(d[4 * r], d[4 * r + 1], d[4 * r + 2], d[4 * r + 3], o0, o1, o2, o3);
        d[4 * r] = (o0 + add2) >> shift2;
        d[4 * r + 1] = (o1 + add2) >> shift2;
        d[4 * r + 2] = (o2 + add2) >> shift2;
        d[4 * r + 3] = (o3 + add2) >> shift2;
    }
}

// A record k_residual's per-lane paths take: a coded, valid TB of size
// 2^log2n with a transform (no transform skip, bypass, I_PCM or RExt residual
// tool) whose residual is not k_ccp's.
__device__ __forceinline__ bool tb_lanes_ok(const DevPic& P, const hpvcd_tu& t, int log2n) {
    constexpr uint32_t kOther = HPVCD_TU_TSKIP | HPVCD_TU_TQB | HPVCD_TU_ROTATE | HPVCD_TU_RDPCM_H |
                                HPVCD_TU_RDPCM_V | HPVCD_TU_PCM;
    if (!(t.flags & HPVCD_TU_CBF) || (t.flags & kOther) || t.log2n != log2n) return false;
    if ((P.flags & HPVCD_PIC_CROSS_COMPONENT) && t.comp && t.res_scale) return false;
    const int ncomp = P.idc ? 3 : 1;
    if (t.comp >= ncomp) return false;
    const int pw = t.comp ? P.cw : P.w, ph = t.comp ? P.ch : P.h;
    return (int)t.x < pw && (int)t.y < ph && (uint64_t)t.coeff_off + (1u << (2 * log2n)) <= P.n_coeffs;
}

// Residual of one such 4x4 TB by one thread (the 4x4 case of
// tb_residual_warp: dequantisation transform.rs:764-858 with the same
// per-coefficient factor, then idct4_thread), stored where the warp path
// stores it: added to the plane and clipped for TBs predicted in the
// plane, else into the int16 residual plane.
__device__ void tb4_thread(const DevPic& P, const hpvcd_tu& t) {
    const int c = t.comp;
    const bool luma = c == 0;
    const int bd = luma ? P.bd : P.bd_c;
    int qpp;
    if (luma) {
        qpp = qp_prime(t.qp_y, bd);
    } else {
        const int pps_off = c == 1 ? P.pps_cb_qp_offset : P.pps_cr_qp_offset;
        qpp = qp_prime(qpc_map(t.qp_y + pps_off + t.cqp_off, P.idc, bd), bd);
    }
    const int bd_shift = bd + 2 + 10 - 15;
    const int qs = clamp3i(qpp, 0, 51 + 6 * (bd - 8));
    const long long base = (long long)level_scale(qs % 6) * (1ll << (qs / 6));
    const long long add = 1ll << (bd_shift - 1);
    const uint8_t* sm = nullptr;
    if (P.scaling) sm = P.scaling->m[0][min(c, 2) + ((t.flags & HPVCD_TU_INTRA) ? 0 : 3)];
    const int nx = (t.nx == 0 || t.nx > 4) ? 4 : t.nx;
    int d[16];
    const bool c8 = (P.flags & HPVCD_PIC_COEFF8) != 0;
    if (c8) {
        const int8_t* lv = (const int8_t*)P.coeffs + t.coeff_off;
        if (((uintptr_t)lv & 15) == 0) {
            const int4 w = *(const int4*)lv;
            const int ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int i = 0; i < 16; ++i) d[i] = (int)(int8_t)(ws[i >> 2] >> (8 * (i & 3)));
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) d[i] = lv[i];
        }
    } else {
        const int16_t* lv = P.coeffs + t.coeff_off;
        if (((uintptr_t)lv & 15) == 0) {
            const int4 w0 = *(const int4*)lv, w1 = *(const int4*)(lv + 8);
            const int ws[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
            for (int i = 0; i < 16; ++i) d[i] = (int)(int16_t)(ws[i >> 1] >> (16 * (i & 1)));
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) d[i] = lv[i];
        }
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const long long f = sm ? base * sm[i] : base * 16;
        const long long v = ((long long)d[i] * f + add) >> bd_shift;
        d[i] = (i & 3) < nx ? (int)(v < -32768 ? -32768 : (v > 32767 ? 32767 : v)) : 0;
    }
    const int shift2 = 20 - bd;
    if (luma && (t.flags & HPVCD_TU_INTRA))
        idct4_thread<true>(d, shift2);
    else
        idct4_thread<false>(d, shift2);
    const bool i16s = bd <= 8;
    const int pw = c ? P.cw : P.w, ph = c ? P.ch : P.h;
    const int x0 = t.x, y0 = t.y;
    const bool in_plane = (P.flags & HPVCD_PIC_PRED_IN_PLANE) || !(t.flags & HPVCD_TU_INTRA);
    if (in_plane) {  // reconstruct.rs:214-251: add and clip into the plane
        void* pl = P.rec[c];
        const int mx = (1 << bd) - 1;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int x = x0 + (i & 3), y = y0 + (i >> 2);
            if (x < pw && y < ph) {
                const int v = i16s ? (int)(int16_t)d[i] : d[i];
                const size_t idx = (size_t)y * pw + x;
                store_sample(pl, P.bps, idx, clamp3i(load_sample(pl, P.bps, idx) + v, 0, mx));
            }
        }
    } else {  // the int16 residual plane k_recon adds to its prediction
        int16_t* rp = P.res[c];
        const int rs = P.res_stride[c];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int y = y0 + r;
            if (y >= ph) break;
            int16_t* row = rp + (size_t)y * rs + x0;
            int16_t v4[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) v4[m] = (int16_t)sat16(i16s ? (int)(int16_t)d[4 * r + m] : d[4 * r + m]);
            if (x0 + 4 <= pw && ((uintptr_t)row & 7) == 0) {
                *(uint2*)row = make_uint2((uint32_t)(uint16_t)v4[0] | ((uint32_t)(uint16_t)v4[1] << 16),
                                          (uint32_t)(uint16_t)v4[2] | ((uint32_t)(uint16_t)v4[3] << 16));
            } else {
#pragma unroll
                for (int m = 0; m < 4; ++m)
                    if (x0 + m < pw) row[m] = v4[m];
            }
        }
    }
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// 8-point inverse DCT with the basis as immediates, even-odd form:
// o[m] = sum_k T8[k][m] * in[k] (transform.rs:406-533, the H.265 matrix).
__device__ __forceinline__ void inv8(const int (&in)[8], int (&o)[8]) {
    const int ee0 = 64 * (in[0] + in[4]), ee1 = 64 * (in[0] - in[4]);
    const int eo0 = 83 * in[2] + 36 * in[6], eo1 = 36 * in[2] - 83 * in[6];
    const int e0 = ee0 + eo0, e3 = ee0 - eo0, e1 = ee1 + eo1, e2 = ee1 - eo1;
    const int o0 = 89 * in[1] + 75 * in[3] + 50 * in[5] + 18 * in[7];
    const int o1 = 75 * in[1] - 18 * in[3] - 89 * in[5] - 50 * in[7];
    const int o2 = 50 * in[1] - 89 * in[3] + 18 * in[5] + 75 * in[7];
    const int o3 = 18 * in[1] - 50 * in[3] + 75 * in[5] - 89 * in[7];
    o[0] = e0 + o0; o[7] = e0 - o0;
    o[1] = e1 + o1; o[6] = e1 - o1;
    o[2] = e2 + o2; o[5] = e2 - o2;
    o[3] = e3 + o3; o[4] = e3 - o3;
}

// Stage 1 of a plain coded 8x8 TB by lane q (0..7) of its group of eight:
// column q dequantised (the 8x8 case of tb_residual_warp: factor
// base * m[r][q] or base * 16, columns >= nx zero) and inverse transformed,
// (sum + 64) >> 7 clipped to int16 into the group's scratch S[m * 9 + q].
__device__ void tb8_cols(const DevPic& P, const hpvcd_tu& t, int q, int16_t* S) {
    const int c = t.comp;
    const int bd = c ? P.bd_c : P.bd;
    int qpp;
    if (c == 0) {
        qpp = qp_prime(t.qp_y, bd);
    } else {
        const int pps_off = c == 1 ? P.pps_cb_qp_offset : P.pps_cr_qp_offset;
        qpp = qp_prime(qpc_map(t.qp_y + pps_off + t.cqp_off, P.idc, bd), bd);
    }
    const int bd_shift = bd + 3 + 10 - 15;
    const int qs = clamp3i(qpp, 0, 51 + 6 * (bd - 8));
    const long long base = (long long)level_scale(qs % 6) * (1ll << (qs / 6));
    const long long add = 1ll << (bd_shift - 1);
    const uint8_t* sm = nullptr;
    if (P.scaling) sm = P.scaling->m[1][min(c, 2) + ((t.flags & HPVCD_TU_INTRA) ? 0 : 3)];
    const int nx = (t.nx == 0 || t.nx > 8) ? 8 : t.nx;
    const bool c8 = (P.flags & HPVCD_PIC_COEFF8) != 0;
    int in[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = r * 8 + q;
        const int l = c8 ? (int)((const int8_t*)P.coeffs + t.coeff_off)[i] : (int)(P.coeffs + t.coeff_off)[i];
        const long long f = sm ? base * sm[i] : base * 16;
        const long long v = ((long long)l * f + add) >> bd_shift;
        in[r] = q < nx ? (int)(v < -32768 ? -32768 : (v > 32767 ? 32767 : v)) : 0;
    }
    int o[8];
    inv8(in, o);
#pragma unroll
    for (int m = 0; m < 8; ++m) S[m * 9 + q] = (int16_t)clamp3i((o[m] + 64) >> 7, -32768, 32767);
}

// Stage 2 of the same TB by lane q: row q of the stage-1 result, inverse
// transformed, + 2^(shift2 - 1) >> shift2, stored as tb4_thread stores
// (added to the plane, or into the int16 residual plane).
__device__ void tb8_rows(const DevPic& P, const hpvcd_tu& t, int q, const int16_t* S) {
    const int c = t.comp;
    const int bd = c ? P.bd_c : P.bd;
    const int shift2 = 20 - bd, add2 = 1 << (shift2 - 1);
    const bool i16s = bd <= 8;
    int in[8], o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) in[k] = S[q * 9 + k];
    inv8(in, o);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int v = (o[m] + add2) >> shift2;
        o[m] = i16s ? (int)(int16_t)v : v;
    }
    const int pw = c ? P.cw : P.w, ph = c ? P.ch : P.h;
    const int x0 = t.x, y = t.y + q;
    if (y >= ph) return;
    const bool in_plane = (P.flags & HPVCD_PIC_PRED_IN_PLANE) || !(t.flags & HPVCD_TU_INTRA);
    if (in_plane) {  // reconstruct.rs:214-251: add and clip into the plane
        void* pl = P.rec[c];
        const int mx = (1 << bd) - 1;
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            if (x0 + m >= pw) break;
            const size_t idx = (size_t)y * pw + x0 + m;
            store_sample(pl, P.bps, idx, clamp3i(load_sample(pl, P.bps, idx) + o[m], 0, mx));
        }
    } else {
        int16_t* row = P.res[c] + (size_t)y * P.res_stride[c] + x0;
        if (x0 + 8 <= pw && ((uintptr_t)row & 15) == 0) {
            uint32_t w[4];
#pragma unroll
            for (int h = 0; h < 4; ++h)
                w[h] = (uint32_t)(uint16_t)sat16(o[2 * h]) | ((uint32_t)(uint16_t)sat16(o[2 * h + 1]) << 16);
            *(uint4*)row = make_uint4(w[0], w[1], w[2], w[3]);
        } else {
#pragma unroll
            for (int m = 0; m < 8; ++m)
                if (x0 + m < pw) row[m] = (int16_t)sat16(o[m]);
        }
    }
}

template <int kIdct>
__global__ void __launch_bounds__(kResWarps * 32)
k_residual(const DevPic* __restrict__ pics, const uint32_t* __restrict__ rec_prefix, uint32_t n_pics,
           uint32_t* dev_err) {
    __shared__ int16_t dct[32 * 32];
    __shared__ __align__(16) int16_t scr[kResWarps][2][32 * kScr];  // per warp: buf, tmp (contiguous)
    __shared__ uint32_t frags[kIdct == kIdctTensor ? kFragEntries * 32 : 1];
    for (int i = threadIdx.x; i < 32 * 32; i += blockDim.x) dct[i] = (int16_t)dct_entry(32, i / 32, i % 32);
    if (kIdct == kIdctTensor) build_basis_frags(frags, threadIdx.x, blockDim.x);
    __syncthreads();
    constexpr unsigned kAll = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t first = rec_prefix[0], total = rec_prefix[n_pics];
    const uint32_t n_chunks = (total - first + kResChunk - 1) / kResChunk;
    for (uint32_t ch = blockIdx.x * kResWarps + warp; ch < n_chunks; ch += gridDim.x * kResWarps) {
        const uint32_t g0 = first + ch * kResChunk;
        // ---- this lane's record: its picture (binary search in the prefix),
        // the record, and an L2 prefetch of its coefficients ----
        const uint32_t gl = g0 + lane;
        uint32_t pic = 0;
        uint4 r4 = make_uint4(0u, 0u, 0u, 0u);
        bool mine4 = false;  // a plain coded 4x4 TB: this lane transforms it on its own
        bool mine8 = false;  // a plain coded 8x8 TB: a group of eight lanes transforms it
        if (gl < total) {
            uint32_t lo = 0, hi = n_pics;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (rec_prefix[mid] <= gl) lo = mid; else hi = mid;
            }
            pic = lo;
            const DevPic& P = pics[lo];
            r4 = *(const uint4*)(P.tus + (gl - rec_prefix[lo]));  // records are 16-byte aligned
            hpvcd_tu t;
            memcpy(&t, &r4, sizeof(t));
            if (tb_lanes_ok(P, t, 2)) {
                mine4 = true;
            } else if (tb_lanes_ok(P, t, 3)) {
                mine8 = true;
            } else if ((t.flags & HPVCD_TU_CBF) && t.log2n >= 2 && t.log2n <= 5) {
                const uint32_t esz = (P.flags & HPVCD_PIC_COEFF8) ? 1u : 2u;
                const uint64_t n2 = 1ull << (2 * t.log2n);
                if ((uint64_t)t.coeff_off + n2 <= P.n_coeffs) {
                    const char* b = (const char*)P.coeffs + (uint64_t)t.coeff_off * esz;
                    const char* e = b + n2 * esz;
                    for (const char* q = (const char*)((uintptr_t)b & ~(uintptr_t)127); q < e; q += 128) prefetch_l2(q);
                }
            }
        }
        // ---- the plain coded 4x4 TBs (most coded TBs): one per lane, in
        // registers ----
        if (mine4) {
            hpvcd_tu t;
            memcpy(&t, &r4, sizeof(t));
            tb4_thread(pics[pic], t);
        }
        const uint32_t done4 = __ballot_sync(kAll, mine4);
        // ---- the plain coded 8x8 TBs: four per pass, eight lanes each
        // (lane q of a group takes column q, then row q; the transpose goes
        // through the warp's scratch) ----
        const uint32_t done8 = __ballot_sync(kAll, mine8);
        for (uint32_t mask8 = done8; mask8;) {
            const int grp = lane >> 3, q = lane & 7;
            uint32_t m = mask8;
            for (int i = 0; i < grp; ++i) m &= m - 1u;
            const int src = m ? __ffs(m) - 1 : 0;
            const uint32_t pj = __shfl_sync(kAll, pic, src);
            uint4 w4;
            w4.x = __shfl_sync(kAll, r4.x, src);
            w4.y = __shfl_sync(kAll, r4.y, src);
            w4.z = __shfl_sync(kAll, r4.z, src);
            w4.w = __shfl_sync(kAll, r4.w, src);
            hpvcd_tu t;
            memcpy(&t, &w4, sizeof(t));
            int16_t* S = scr[warp][0] + grp * 72;
            if (m) tb8_cols(pics[pj], t, q, S);
            __syncwarp();
            if (m) tb8_rows(pics[pj], t, q, S);
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 4; ++i) mask8 &= mask8 - 1u;
        }
        // ---- the chunk's other records one by one ----
        const uint32_t nrec = min((uint32_t)kResChunk, total - g0);
        for (uint32_t j = 0; j < nrec; ++j) {
            if (((done4 | done8) >> j) & 1u) continue;
            const uint32_t pj = __shfl_sync(kAll, pic, j);
            uint4 w4;
            w4.x = __shfl_sync(kAll, r4.x, j);
            w4.y = __shfl_sync(kAll, r4.y, j);
            w4.z = __shfl_sync(kAll, r4.z, j);
            w4.w = __shfl_sync(kAll, r4.w, j);
            hpvcd_tu t;
            memcpy(&t, &w4, sizeof(t));
            const DevPic& P = pics[pj];
            if (!(t.flags & HPVCD_TU_CBF)) continue;
            if ((P.flags & HPVCD_PIC_CROSS_COMPONENT) && t.comp && t.res_scale) continue;  // k_ccp's
            const int c = t.comp;
            const int ncomp = P.idc ? 3 : 1;
            const int n = 1 << t.log2n;
            const int pw = c < 3 && c ? P.cw : P.w, ph = c < 3 && c ? P.ch : P.h;
            if (c >= ncomp || t.log2n < 2 || t.log2n > 5 || (int)t.x >= pw || (int)t.y >= ph ||
                (uint64_t)t.coeff_off + (uint64_t)n * n > P.n_coeffs) {
                if (lane == 0) atomicOr(dev_err, DEV_ERR_BITSTREAM);
                continue;
            }
            const int x0 = t.x, y0 = t.y;
            const bool in_plane = (P.flags & HPVCD_PIC_PRED_IN_PLANE) || !(t.flags & HPVCD_TU_INTRA);
            if (in_plane) {  // prediction already in the plane: add + clip (reconstruct.rs:214-251)
                void* pl = P.rec[c];
                const int mx = (1 << (c ? P.bd_c : P.bd)) - 1;
                const int keep = (t.flags & HPVCD_TU_PCM) ? 0 : 1;  // I_PCM samples replace the plane's
                tb_residual_warp<kIdct>(
                    P, t, dct, scr[warp][0], scr[warp][1], lane,
                    [&](int r, int m, int v) {
                        const int x = x0 + m, y = y0 + r;
                        if (x < pw && y < ph) {
                            const size_t idx = (size_t)y * pw + x;
                            store_sample(pl, P.bps, idx, clamp3i(keep * load_sample(pl, P.bps, idx) + v, 0, mx));
                        }
                    },
                    true, frags);
            } else {
                int16_t* rp = P.res[c];
                const int rs = P.res_stride[c];
                tb_residual_warp<kIdct>(
                    P, t, dct, scr[warp][0], scr[warp][1], lane,
                    [&](int r, int m, int v) {
                        const int x = x0 + m, y = y0 + r;
                        if (x < pw && y < ph) rp[(size_t)y * rs + x] = (int16_t)sat16(v);
                    },
                    true, frags);
            }
        }
    }
}

// ===========================================================================
// k_ccp -- chroma TBs with cross-component prediction (RExt 4:4:4)
// ===========================================================================
// One warp per chroma TB with res_scale != 0 of a HPVCD_PIC_CROSS_COMPONENT
// picture: it recomputes its TU's luma residual rY (the matrix inverse
// transform, which keeps i32 values above 8 bits), then the chroma residual
// in i32 storage (decode.rs:5286-5426; zero without coded residual,
// :5428-5466), adds (res_scale * ((rY << BitDepthC) >> BitDepthY)) >> 3
// (decode.rs:5488-5504) and writes it where k_residual would.
constexpr int kCcpWarps = 4;

__global__ void __launch_bounds__(kCcpWarps * 32)
k_ccp(const DevPic* __restrict__ pics, const uint32_t* __restrict__ rec_prefix, uint32_t n_pics,
      uint32_t* dev_err) {
    __shared__ int16_t dct[32 * 32];
    __shared__ __align__(16) int16_t scr[kCcpWarps][2][32 * kScr];
    __shared__ int32_t ry_all[kCcpWarps][32 * 32];
    for (int i = threadIdx.x; i < 32 * 32; i += blockDim.x) dct[i] = (int16_t)dct_entry(32, i / 32, i % 32);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t* ry = ry_all[warp];
    const uint32_t total = rec_prefix[n_pics];
    for (uint32_t g = rec_prefix[0] + blockIdx.x * kCcpWarps + warp; g < total; g += gridDim.x * kCcpWarps) {
        uint32_t lo = 0, hi = n_pics;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (rec_prefix[mid] <= g) lo = mid; else hi = mid;
        }
        const DevPic& P = pics[lo];
        if (!(P.flags & HPVCD_PIC_CROSS_COMPONENT)) continue;
        const uint32_t gl = g - rec_prefix[lo];
        const hpvcd_tu t = P.tus[gl];
        if (t.comp == 0 || t.res_scale == 0) continue;
        const int n = 1 << t.log2n;
        bool bad = P.idc != 3 || t.comp > 2 || t.log2n < 2 || t.log2n > 5 || (int)t.x >= P.cw ||
                   (int)t.y >= P.ch ||
                   ((t.flags & HPVCD_TU_CBF) && (uint64_t)t.coeff_off + (uint64_t)n * n > P.n_coeffs);
        // the TU's luma TB: same place and size, among the three records before
        hpvcd_tu lt{};
        bool found = false;
        for (uint32_t k = 1; k <= 3 && k <= gl && !found; ++k) {
            lt = P.tus[gl - k];
            found = lt.comp == 0 && lt.x == t.x && lt.y == t.y && lt.log2n == t.log2n;
        }
        bad = bad || !found || !(lt.flags & HPVCD_TU_CBF) ||
              (uint64_t)lt.coeff_off + (uint64_t)n * n > P.n_coeffs;
        if (bad) {
            if (lane == 0) atomicOr(dev_err, DEV_ERR_BITSTREAM);
            continue;
        }
        tb_residual_warp<kIdctMatrix>(P, lt, dct, scr[warp][0], scr[warp][1], lane,
                                      [&](int r, int m, int v) { ry[r * n + m] = v; });
        __syncwarp();
        const int c = t.comp, x0 = t.x, y0 = t.y, pw = P.cw, ph = P.ch;
        const int bdy = P.bd, bdc = P.bd_c, rs = t.res_scale;
        const bool in_plane = (P.flags & HPVCD_PIC_PRED_IN_PLANE) || !(t.flags & HPVCD_TU_INTRA);
        const int mx = (1 << bdc) - 1;
        auto out = [&](int r, int m, long long v) {
            const long long sy = ((long long)ry[r * n + m] << bdc) >> bdy;
            v += (rs * sy) >> 3;
            const int vv = (int)(v < INT_MIN ? INT_MIN : (v > INT_MAX ? INT_MAX : v));
            const int x = x0 + m, y = y0 + r;
            if (x >= pw || y >= ph) return;
            if (in_plane) {
                const size_t idx = (size_t)y * pw + x;
                const long long s = (long long)load_sample(P.rec[c], P.bps, idx) + vv;
                store_sample(P.rec[c], P.bps, idx, (int)(s < 0 ? 0 : (s > mx ? mx : s)));
            } else {
                P.res[c][(size_t)y * P.res_stride[c] + x] = (int16_t)sat16(vv);
            }
        };
        if (t.flags & HPVCD_TU_CBF)
            tb_residual_warp<kIdctMatrix>(P, t, dct, scr[warp][0], scr[warp][1], lane,
                                          [&](int r, int m, int v) { out(r, m, v); }, false);
        else
            for (int i = lane; i < n * n; i += 32) out(i / n, i % n, 0);
        __syncwarp();
    }
}

// ===========================================================================
// k_recon
// ===========================================================================
constexpr unsigned kFull = 0xffffffffu;

// Per-warp scratch of the decode-order walk (reference samples fit in 16 bits).
struct WalkScratch {
    int16_t s[132];     // substituted reference line: s[2n+q] = above[q], s[2n-q] = left[q]
    int16_t f[132];     // filtered line (same layout); also holds available values before substitution
    int16_t refs[100];  // angular projection, refs[n + k] for k in [-n, 2n]
    int32_t dc;         // DC value of the current TB
};
constexpr size_t kWsBytes = (sizeof(WalkScratch) + 15) & ~(size_t)15;

// One bordered canvas per component of a CTU S x Sh: the row above the CTU
// first (x = -1 .. 2S-1 at index x + 8), then the CTU's Sh rows of S + 8
// entries (index 7 = the column left of the CTU, x at x + 8).  Both row
// lengths are multiples of 8 entries, so every interior row starts 16-byte
// aligned.
__host__ __device__ __forceinline__ int can_top(int S) { return 2 * S + 8; }
__host__ __device__ __forceinline__ int can_row(int S) { return S + 8; }
__host__ __device__ __forceinline__ int can_size(int S, int Sh) { return can_top(S) + Sh * can_row(S); }
__device__ __forceinline__ int can_at(int S, int x, int y) {
    return y < 0 ? x + 8 : can_top(S) + y * can_row(S) + x + 8;
}
// The same index for a sample of the CTU's own rows (y >= 0), without the
// test for the row above.
__device__ __forceinline__ int can_in(int S, int x, int y) { return can_top(S) + y * can_row(S) + x + 8; }

// Shared-memory layout of one CTA: the canvases, one walk scratch per warp,
// the CTU's staged records, the 16x16 stamp map, the three TB lists.
// Records of one CTU staged at once: up to 256 luma TBs, one "mark decoded"
// record per inter CU (64 at most) and the chroma TBs (64 per component at
// 4:2:0, 128 at 4:2:2, 256 at 4:4:4).  A CTU with more records is malformed.
// Chroma formats of a layout: kFmt420 (also 4:0:0), kFmt444, kFmt422; the
// 4:4:4 layout holds every format, the 4:2:2 one also 4:2:0.
constexpr int kFmt420 = 0, kFmt444 = 1, kFmt422 = 2;
constexpr int kRecCap420 = 256 + 64 + 2 * 64;
constexpr int kRecCap422 = 256 + 64 + 2 * 128;
constexpr int kRecCap444 = 256 + 64 + 2 * 256;
constexpr int kListCap = 256;  // intra TBs of luma in one CTU (all 4x4)
// list entry: record index (< 1024) | kListEvent for a wavefront event
constexpr uint32_t kListRec = 0x3ffu, kListEvent = 0x8000u;
constexpr uint32_t kNoStamp = 0xffffffffu;

struct ReconLayout {
    int cs_w, cs_h;  // chroma canvas width and height (CTU interior)
    int rec_cap;     // staged records
    int list_c;      // list entries per chroma component
    size_t off_can_y, off_can_c, off_ws, off_recs, off_stamp, off_lists, off_misc, total;
    __host__ __device__ ReconLayout(int cfmt, int warps) {
        cs_w = cfmt == kFmt444 ? 64 : 32;
        cs_h = cfmt == kFmt420 ? 32 : 64;
        rec_cap = cfmt == kFmt444 ? kRecCap444 : (cfmt == kFmt422 ? kRecCap422 : kRecCap420);
        list_c = cfmt == kFmt444 ? 256 : (cfmt == kFmt422 ? 128 : 64);
        size_t o = 0;
        off_can_y = o; o += (size_t)can_size(64, 64) * sizeof(uint16_t);
        o = (o + 15) & ~(size_t)15;
        off_can_c = o; o += 2 * (size_t)can_size(cs_w, cs_h) * sizeof(uint16_t);
        o = (o + 15) & ~(size_t)15;
        off_ws = o;    o += (size_t)warps * kWsBytes;
        off_recs = o;  o += (size_t)rec_cap * sizeof(hpvcd_tu);
        off_stamp = o; o += 256 * sizeof(uint32_t);
        off_lists = o; o += (size_t)(kListCap + 2 * list_c) * sizeof(uint16_t);
        o = (o + 15) & ~(size_t)15;
        off_misc = o;  o += 128;  // claimed item, list counts, edge masks, neighbour levels
        total = o;
    }
    __host__ __device__ int list_off(int c) const { return c == 0 ? 0 : kListCap + (c - 1) * list_c; }
    __host__ __device__ int list_cap(int c) const { return c == 0 ? kListCap : list_c; }
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Everything one warp needs about one component of the current CTU.
struct Comp {
    int ox, oy;   // CTU origin in component samples
    int pw, ph;   // plane size
    int S, Sh;    // CTU width and height in component samples
    int sw, sh;   // luma samples per component sample (1 or 2)
    uint32_t nb_ok;  // neighbour CTUs of the same slice and tile: 1 left, 2 above-left, 4 above, 8 above-right
    const hpvcd_cell* ci_cells;  // constrained intra prediction: cells whose INTER samples are unusable
    int gw;                      // cells per row
    bool restricted;             // nb_ok != 0xf or ci_cells: gather_ref runs restricted_ok
    bool ccp;                    // chroma of a cross-component picture: res_scale gives a residual
    int bd, max_v;
    bool luma, filt, smoothing, strong;
    uint16_t* can;       // bordered canvas
    const int16_t* res;  // int16 residual plane (k_residual) at the CTU origin
    int rs;              // its row stride in samples (a multiple of 16)
};

__device__ __forceinline__ int cidx(const Comp& k, int x, int y) { return can_at(k.S, x, y); }
__device__ __forceinline__ int cin(const Comp& k, int x, int y) { return can_in(k.S, x, y); }

// Reference sample i of the line (i < 2n: left column bottom-up, 2n: the
// corner, > 2n: above row) with its availability (decode.rs:4651-4690
// luma_avail / chroma_avail restricted to this CTU and its already
// reconstructed neighbours of the same slice and tile).  Inside the
// CTU a sample is available when the luma record that marked its 4x4 cell
// decoded comes before the current record `jrec` in decode order: `stamp`
// holds, per cell, the index of the first luma record covering it
// (decode.rs:3170-3189 marks cells as records complete).
// Slices, tiles and constrained intra prediction: a sample of a neighbour CTU
// of another slice or tile (decode.rs:4651-4690 same_slice / same_tile) or
// of an inter cell under constrained_intra_pred (decode.rs:4641-4649) is not
// available.  (x, y) relative to the CTU, (ax, ay) in the plane.
__device__ __forceinline__ bool restricted_ok(const Comp& k, int x, int y, int ax, int ay) {
    uint32_t bit = 0;  // 1 left, 2 above-left, 4 above, 8 above-right, 0 this CTU
    if (x < 0)
        bit = y < 0 ? 2u : 1u;
    else if (y < 0)
        bit = x < k.S ? 4u : 8u;
    if (bit && !(k.nb_ok & bit)) return false;
    if (k.ci_cells && (k.ci_cells[(size_t)((ay * k.sh) >> 2) * k.gw + ((ax * k.sw) >> 2)].flags & HPVCD_CELL_INTER))
        return false;
    return true;
}

__device__ __forceinline__ bool gather_ref(const Comp& k, const uint32_t* stamp, uint32_t jrec, int n2, int x0,
                                           int y0, int i, int* v) {
    const bool left_side = i < n2;
    const int x = left_side ? x0 - 1 : x0 + (i - n2 - 1);
    const int y = left_side ? y0 + (n2 - 1 - i) : y0 - 1;
    const int ax = k.ox + x, ay = k.oy + y;
    // both loads from clamped (always valid) positions, issued together;
    // the availability test picks the result
    const int ys = min(max(y, 0), k.Sh - 1), xs = min(max(x, 0), k.S - 1);
    const uint32_t st = stamp[((ys * k.sh) >> 2) * 16 + ((xs * k.sw) >> 2)];
    const int cv = k.can[cidx(k, y < 0 ? x : min(x, k.S - 1), min(y, k.Sh - 1))];
    bool a = ax >= 0 && ay >= 0 && ax < k.pw && ay < k.ph;
    if (y >= 0) {
        if (x < 0)
            a = a && y < k.Sh;  // left CTU (below-left CTU is not reconstructed yet)
        else
            a = a && x < k.S && y < k.Sh && st < jrec;
    }
    if (k.restricted && a) a = restricted_ok(k, x, y, ax, ay);  // warp-uniform branch
    *v = a ? cv : 0;
    return a;
}

// The angular reference projection of intra.rs:305-318: position in the
// reference line of refs[k] (k in [-n, 2n]).
__device__ __forceinline__ int ref_pos(int k, bool vertical, int n2, int inv) {
    if (k >= 0) return vertical ? n2 + k : n2 - k;
    const int idx = max(min((k * inv + 128) >> 8, n2), 0);
    return vertical ? n2 - idx : n2 + idx;
}

// 4x4 intra TB entirely in registers: the 17 reference samples live in
// lanes 0..16 (intra.rs:84-148 substitution via shuffles; no filtering for
// n = 4, intra.rs:174), prediction (intra.rs:257-372) by lanes 0..15.
// I_PCM block (decode.rs:2768-2839): its samples, written to the residual
// plane by k_residual, go to the canvas unchanged.
__device__ __forceinline__ void pcm_tb(const Comp& k, int log2n, int x0, int y0, int lane) {
    const int n = 1 << log2n;
    const int vw = min(n, k.pw - (k.ox + x0)), vh = min(n, k.ph - (k.oy + y0));
    for (int i = lane; i < n * n; i += 32) {
        const int yy = i >> log2n, xx = i & (n - 1);
        if (xx < vw && yy < vh)
            k.can[cin(k, x0 + xx, y0 + yy)] =
                (uint16_t)clamp3i(k.res[(size_t)(y0 + yy) * k.rs + x0 + xx], 0, k.max_v);
    }
    __syncwarp();
}

__device__ __forceinline__ void intra_tb4(const Comp& k, int mode, int x0, int y0, bool coded,
                                          const uint32_t* stamp, uint32_t jrec, int lane) {
    constexpr int n = 4, n2 = 8, total = 17;
    const int yy = lane >> 2, xx = lane & 3;
    const int vw = min(n, k.pw - (k.ox + x0)), vh = min(n, k.ph - (k.oy + y0));
    const bool mine = lane < 16 && xx < vw && yy < vh;
    // the residual staged in the TB's canvas area (stage_residual)
    const int rv = coded && mine ? (int)(int16_t)k.can[cin(k, x0 + xx, y0 + yy)] : 0;
    int v = 0;
    // lanes past the line repeat the last position and drop it
    bool a = gather_ref(k, stamp, jrec, n2, x0, y0, min(lane, total - 1), &v);
    a = a && lane < total;
    const uint32_t mask = __ballot_sync(kFull, a);
    int sv;
    if (!mask) {
        sv = 1 << (k.bd - 1);
    } else {
        const uint32_t m0 = mask & ((2u << lane) - 1u);
        const int j = m0 ? 31 - __clz(m0) : __ffs(mask) - 1;
        sv = __shfl_sync(kFull, v, j);
    }
    // sv in lane i = s[i]
    int pred;
    if (mode >= 2) {
        const int angle = c_intra_angle[mode - 2];
        const bool vertical = mode >= 18;
        const int inv = angle < 0 ? c_inv_angle[mode - 11] : 0;
        const int a_ = vertical ? yy : xx, b = vertical ? xx : yy;
        const int pos = (a_ + 1) * angle;
        const int iidx = pos >> 5, frac = pos & 31;
        const int r0 = __shfl_sync(kFull, sv, ref_pos(b + iidx + 1, vertical, n2, inv));
        const int r1 = __shfl_sync(kFull, sv, ref_pos(min(b + iidx + 2, 2 * n), vertical, n2, inv));
        pred = clamp3i(frac ? ((32 - frac) * r0 + frac * r1 + 16) >> 5 : r0, 0, k.max_v);
        if (k.luma) {  // DC / vertical / horizontal edge filters (n < 32)
            const int c0 = __shfl_sync(kFull, sv, n2);
            const int a0 = __shfl_sync(kFull, sv, vertical ? n2 + 1 : n2 - 1);
            const int e = __shfl_sync(kFull, sv, mode == 26 ? n2 - (yy + 1) : n2 + xx + 1);
            if ((mode == 26 && xx == 0) || (mode == 10 && yy == 0)) pred = clamp3i(a0 + ((e - c0) >> 1), 0, k.max_v);
        }
    } else if (mode == 1) {  // DC
        int part = ((lane >= n2 - n && lane < n2) || (lane > n2 && lane <= n2 + n)) ? sv : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
        const int dc = (part + n) >> 3;
        const int l1 = __shfl_sync(kFull, sv, n2 - 1), a1 = __shfl_sync(kFull, sv, n2 + 1);
        const int e = __shfl_sync(kFull, sv, yy == 0 ? n2 + xx + 1 : n2 - yy - 1);
        pred = dc;
        if (k.luma) {
            if (xx == 0 && yy == 0)
                pred = (l1 + 2 * dc + a1 + 2) >> 2;
            else if (yy == 0 || xx == 0)
                pred = (e + 3 * dc + 2) >> 2;
        }
    } else {  // planar
        const int lft = __shfl_sync(kFull, sv, n2 - yy - 1), abv = __shfl_sync(kFull, sv, n2 + xx + 1);
        const int tr = __shfl_sync(kFull, sv, n2 + n + 1), bl = __shfl_sync(kFull, sv, n2 - n - 1);
        pred = ((n - 1 - xx) * lft + (xx + 1) * tr + (n - 1 - yy) * abv + (yy + 1) * bl + n) >> 3;
    }
    if (mine) {
        if (coded) pred = clamp3i(pred + rv, 0, k.max_v);
        k.can[cin(k, x0 + xx, y0 + yy)] = (uint16_t)pred;
    }
    __syncwarp();
}

// Whether the reference line of an n x n intra TB is filtered
// (intra.rs:151-219: luma, or 4:4:4 chroma, with smoothing on and a mode
// far enough from the horizontal / vertical).
__device__ __forceinline__ bool ref_filtered(const Comp& k, int n, int mode) {
    if (!(k.filt && k.smoothing && mode != 1)) return false;
    const int md = min(abs(mode - 26), abs(mode - 10));
    const int thresh = n == 8 ? 7 : (n == 16 ? 1 : 0);
    return mode == 0 || md > thresh;
}

// 8x8 intra TB in registers: the 33-sample reference line is s[lane] in
// `lo` and s[32] in `hi` (the same in every lane); substitution
// (intra.rs:84-148) by ballots, [1 2 1] filtering (intra.rs:151-219; no
// strong filter below 32x32) and prediction (intra.rs:257-372) by shuffles,
// two samples per lane.  Same arithmetic as the shared-memory path.
__device__ __forceinline__ void intra_tb8(const Comp& k, int mode, int x0, int y0, bool coded,
                                          const uint32_t* stamp, uint32_t jrec, int lane) {
    constexpr int n = 8, n2 = 16, log2n = 3;
    const int vw = min(n, k.pw - (k.ox + x0)), vh = min(n, k.ph - (k.oy + y0));
    int rv[2];  // residuals of this lane's two samples, staged in the TB's canvas area
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        const int yy = i >> log2n, xx = i & (n - 1);
        rv[h] = coded && xx < vw && yy < vh ? (int)(int16_t)k.can[cin(k, x0 + xx, y0 + yy)] : 0;
    }
    int v_lo = 0, v_hi = 0;
    const bool a_lo = gather_ref(k, stamp, jrec, n2, x0, y0, lane, &v_lo);
    const bool a_hi = gather_ref(k, stamp, jrec, n2, x0, y0, 2 * n2, &v_hi);  // uniform
    const uint32_t mask = __ballot_sync(kFull, a_lo);
    // ---- substitution: an unavailable sample takes the nearest available
    // one below it in the line, or the first available one ----
    const int first = mask ? __ffs(mask) - 1 : 0;
    const int first_lo = __shfl_sync(kFull, v_lo, first);
    const uint32_t m0 = mask & ((2u << lane) - 1u);
    const int below = __shfl_sync(kFull, v_lo, m0 ? 31 - __clz(m0) : 0);
    const int top = __shfl_sync(kFull, v_lo, mask ? 31 - __clz(mask) : 0);
    int s_lo, s_hi;
    if (!mask && !a_hi) {
        s_lo = s_hi = 1 << (k.bd - 1);
    } else {
        const int first_val = mask ? first_lo : v_hi;
        s_lo = a_lo ? v_lo : (m0 ? below : first_val);
        s_hi = a_hi ? v_hi : (mask ? top : first_val);
    }
    // ---- filtering ----
    int r_lo = s_lo;
    const int r_hi = s_hi;
    if (ref_filtered(k, n, mode)) {
        const int up = __shfl_up_sync(kFull, s_lo, 1);
        const int dn = __shfl_down_sync(kFull, s_lo, 1);
        const int nxt = lane == 31 ? s_hi : dn;
        r_lo = lane == 0 ? s_lo : (up + 2 * s_lo + nxt + 2) >> 2;
    }
    // R(idx), idx in [0, 32]; every lane must call it
    auto R = [&](int idx) {
        const int t = __shfl_sync(kFull, r_lo, idx & 31);
        return idx >= 32 ? r_hi : t;
    };
    const int max_v = k.max_v;
    const bool edge = k.luma;  // edge filters of luma TBs below 32x32
    int out[2];
    if (mode >= 2) {
        const int angle = c_intra_angle[mode - 2];
        const bool vertical = mode >= 18;
        const int inv = angle < 0 ? c_inv_angle[mode - 11] : 0;
        const int c0 = R(n2);
        const int a0 = R(vertical ? n2 + 1 : n2 - 1);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = lane + 32 * h;
            const int yy = i >> log2n, xx = i & (n - 1);
            const int a = vertical ? yy : xx, b = vertical ? xx : yy;
            const int pos = (a + 1) * angle;
            const int iidx = pos >> 5, frac = pos & 31;
            const int r0 = R(ref_pos(b + iidx + 1, vertical, n2, inv));
            const int r1 = R(ref_pos(min(b + iidx + 2, 2 * n), vertical, n2, inv));
            int v = clamp3i(frac ? ((32 - frac) * r0 + frac * r1 + 16) >> 5 : r0, 0, max_v);
            const int e = R(mode == 26 ? n2 - (yy + 1) : n2 + xx + 1);
            if (edge && ((mode == 26 && xx == 0) || (mode == 10 && yy == 0))) v = clamp3i(a0 + ((e - c0) >> 1), 0, max_v);
            out[h] = v;
        }
    } else if (mode == 1) {  // DC
        int part = ((lane >= n2 - n && lane < n2) || (lane > n2 && lane <= n2 + n)) ? r_lo : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
        const int dc = (part + n) >> (log2n + 1);
        const int l1 = R(n2 - 1), a1 = R(n2 + 1);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = lane + 32 * h;
            const int yy = i >> log2n, xx = i & (n - 1);
            const int e = R(yy == 0 ? n2 + xx + 1 : n2 - yy - 1);
            int v = dc;
            if (edge) {
                if (xx == 0 && yy == 0)
                    v = (l1 + 2 * dc + a1 + 2) >> 2;
                else if (yy == 0 || xx == 0)
                    v = (e + 3 * dc + 2) >> 2;
            }
            out[h] = v;
        }
    } else {  // planar
        const int tr = R(n2 + n + 1), bl = R(n2 - n - 1);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = lane + 32 * h;
            const int yy = i >> log2n, xx = i & (n - 1);
            const int lft = R(n2 - yy - 1), abv = R(n2 + xx + 1);
            out[h] = ((n - 1 - xx) * lft + (xx + 1) * tr + (n - 1 - yy) * abv + (yy + 1) * bl + n) >> (log2n + 1);
        }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int i = lane + 32 * h;
        const int yy = i >> log2n, xx = i & (n - 1);
        if (xx < vw && yy < vh) {
            int v = out[h];
            if (coded) v = clamp3i(v + rv[h], 0, max_v);
            k.can[cin(k, x0 + xx, y0 + yy)] = (uint16_t)v;
        }
    }
    __syncwarp();
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}

// Stages the visible part of a coded n x n TB's residual (written by
// k_residual) into the TB's own canvas area with asynchronous copies issued
// by one lane: 16 bytes per copy, 8 for 4x4 TBs.  Every coded TB of a CTU is
// staged before its walk starts (the lanes of the walking warp take the
// list entries in turn).  The area of a TB not yet reconstructed is never an
// available reference sample of an earlier TB (its stamp is later), so the
// staged values are never read as samples; each lane predicting a sample
// reads its residual in place.
__device__ __forceinline__ void stage_residual(const Comp& k, int log2n, int x0, int y0) {
    const int n = 1 << log2n;
    const int vw = min(n, k.pw - (k.ox + x0)), vh = min(n, k.ph - (k.oy + y0));
    const int16_t* src = k.res + (size_t)y0 * k.rs + x0;
    uint16_t* dst = k.can + cin(k, x0, y0);
    const int cr = can_row(k.S);
    if (n == 4) {
        for (int r = 0; r < vh; ++r) cp_async8(dst + r * cr, src + (size_t)r * k.rs);
        return;
    }
    const int chunks = (vw + 7) >> 3;
    for (int r = 0; r < vh; ++r)
        for (int q = 0; q < chunks; ++q) cp_async16(dst + r * cr + 8 * q, src + (size_t)r * k.rs + 8 * q);
}

// Intra TB of size 16 or 32, first part, by one warp through shared memory:
// gather, substitution (intra.rs:84-148), filtering (:151-219) and the
// per-mode set-up of the prediction (the angular projection into ws.refs,
// the DC value into ws.dc).
__device__ __forceinline__ void intra_tb_prep(const Comp& k, int log2n, int mode, int x0, int y0,
                                              const uint32_t* stamp, uint32_t jrec, WalkScratch& ws, int lane) {
    const int n = 1 << log2n;
    const int total = 4 * n + 1;
    const int n2 = 2 * n;
    // The line's words (32 positions each: 3 for n = 16, 5 for n = 32) are
    // walked in rolled loops, so the code stays small.  Gather: available
    // samples go to ws.f; lane w keeps the availability word of word w.
    const int nw = (total + 31) >> 5;
    uint32_t my_mask = 0u;
    int first = -1;  // first available position
#pragma unroll 1
    for (int wd = 0; wd < nw; ++wd) {
        const int i = wd * 32 + lane;
        int v = 0;
        bool a = gather_ref(k, stamp, jrec, n2, x0, y0, min(i, total - 1), &v);
        a = a && i < total;
        if (a) ws.f[i] = (int16_t)v;
        const uint32_t m = __ballot_sync(kFull, a);
        if (lane == wd) my_mask = m;
        if (first < 0 && m) first = wd * 32 + __ffs(m) - 1;
    }
    __syncwarp();
    // ---- substitution: an unavailable sample takes the nearest available
    // one below it in the line, or the first available one ----
    const int neutral = 1 << (k.bd - 1);
    int run = -1;  // last available position of the words before
#pragma unroll 1
    for (int wd = 0; wd < nw; ++wd) {
        const int i = wd * 32 + lane;
        const uint32_t m = __shfl_sync(kFull, my_mask, wd);
        if (i < total) {
            int v = neutral;
            if (first >= 0) {
                const uint32_t m0 = m & ((2u << lane) - 1u);
                int j = m0 ? wd * 32 + 31 - __clz(m0) : run;
                if (j < 0) j = first;
                v = ws.f[j];
            }
            ws.s[i] = (int16_t)v;
        }
        if (m) run = wd * 32 + 31 - __clz(m);
    }
    __syncwarp();
    // ---- filtering (luma, or 4:4:4 chroma without strong smoothing) ----
    const bool do_filter = ref_filtered(k, n, mode);
    const int16_t* R = ws.s;
    if (do_filter) {
        bool strong = false;
        const int tl = ws.s[n2], tr = ws.s[2 * n2], bl = ws.s[0];
        if (k.luma && k.strong && n == 32) {
            const int thr = 1 << (k.bd - 5);
            strong = abs(bl + tl - 2 * ws.s[n2 - n]) < thr && abs(tr + tl - 2 * ws.s[n2 + n]) < thr;
        }
        for (int i = lane; i < total; i += 32) {
            int v;
            if (i == 0 || i == 2 * n2) {
                v = ws.s[i];
            } else if (strong) {
                if (i == n2) {
                    v = ws.s[i];
                } else if (i > n2) {
                    const int q = i - n2;  // above[q]
                    v = ((n2 - q) * tl + q * tr + n) >> 6;
                } else {
                    const int q = n2 - i;  // left[q]
                    v = ((n2 - q) * tl + q * bl + n) >> 6;
                }
            } else {
                v = (ws.s[i - 1] + 2 * ws.s[i] + ws.s[i + 1] + 2) >> 2;
            }
            ws.f[i] = v;
        }
        __syncwarp();
        R = ws.f;
    }
    // A(q) = R[n2 + q], L(q) = R[n2 - q]
    if (mode >= 2) {
        const int angle = c_intra_angle[mode - 2];
        const bool vertical = mode >= 18;
        for (int q = lane; q <= n2; q += 32) ws.refs[n + q] = vertical ? R[n2 + q] : R[n2 - q];
        if (angle < 0) {
            const int inv = c_inv_angle[mode - 11];
            const int lim = (n * angle) >> 5;
            for (int q = -1 - lane; q >= lim; q -= 32) {
                const int idx = max(min((q * inv + 128) >> 8, n2), 0);
                ws.refs[q + n] = vertical ? R[n2 - idx] : R[n2 + idx];  // side(idx)
            }
        }
    } else if (mode == 1) {
        int part = lane < n ? R[n2 + 1 + lane] + R[n2 - 1 - lane] : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
        if (lane == 0) ws.dc = (part + n) >> (log2n + 1);
    }
    __syncwarp();
}

// Intra TB of size 16 or 32, second part: prediction (intra.rs:257-372) and
// residual add + clip (reconstruct.rs:214-251), lane l of one warp taking
// samples l, l + 32, ...  A coded TB's residual is in its canvas area
// (stage_residual).  The loops stay compact: the kernel's code competes for
// the instruction cache with the other walks resident on the SM.
__device__ __forceinline__ void intra_tb_predict(const Comp& k, int log2n, int mode, int x0, int y0, bool coded,
                                                 const WalkScratch& ws, int lane) {
    const int tl = lane, ts = 32;
    const int n = 1 << log2n;
    const int n2 = 2 * n;
    const int16_t* R = ref_filtered(k, n, mode) ? ws.f : ws.s;
    const int max_v = k.max_v;
    const bool edge_filters = k.luma && n < 32;  // is_luma gate of predict_into
    const int vw = min(n, k.pw - (k.ox + x0)), vh = min(n, k.ph - (k.oy + y0));
    auto res_at = [&](int xx, int yy) { return (int)(int16_t)k.can[cin(k, x0 + xx, y0 + yy)]; };
    if (mode >= 2) {
        const int angle = c_intra_angle[mode - 2];
        const bool vertical = mode >= 18;
        const int a0 = vertical ? R[n2 + 1] : R[n2 - 1];  // above[1] / left[1]
        const int c0 = R[n2];
#pragma unroll 1
        for (int i = tl; i < n * n; i += ts) {
            const int yy = i >> log2n, xx = i & (n - 1);
            const int a = vertical ? yy : xx;
            const int b = vertical ? xx : yy;
            const int pos = (a + 1) * angle;
            const int iidx = pos >> 5, frac = pos & 31;
            const int r0 = ws.refs[b + iidx + 1 + n];
            const int r1 = ws.refs[min(b + iidx + 2, 2 * n) + n];
            int v = frac ? ((32 - frac) * r0 + frac * r1 + 16) >> 5 : r0;
            v = clamp3i(v, 0, max_v);
            if (edge_filters) {
                if (mode == 26 && xx == 0) v = clamp3i(a0 + ((R[n2 - (yy + 1)] - c0) >> 1), 0, max_v);
                if (mode == 10 && yy == 0) v = clamp3i(a0 + ((R[n2 + xx + 1] - c0) >> 1), 0, max_v);
            }
            if (xx < vw && yy < vh) {
                if (coded) v = clamp3i(v + res_at(xx, yy), 0, max_v);
                k.can[cin(k, x0 + xx, y0 + yy)] = (uint16_t)v;
            }
        }
    } else if (mode == 1) {  // DC
        const int dc = ws.dc;
#pragma unroll 1
        for (int i = tl; i < n * n; i += ts) {
            const int yy = i >> log2n, xx = i & (n - 1);
            int v = dc;
            if (edge_filters) {
                if (xx == 0 && yy == 0)
                    v = (R[n2 - 1] + 2 * dc + R[n2 + 1] + 2) >> 2;
                else if (yy == 0)
                    v = (R[n2 + xx + 1] + 3 * dc + 2) >> 2;
                else if (xx == 0)
                    v = (R[n2 - yy - 1] + 3 * dc + 2) >> 2;
            }
            if (xx < vw && yy < vh) {
                if (coded) v = clamp3i(v + res_at(xx, yy), 0, max_v);
                k.can[cin(k, x0 + xx, y0 + yy)] = (uint16_t)v;
            }
        }
    } else {  // planar
        const int tr = R[n2 + n + 1], bl = R[n2 - n - 1];
#pragma unroll 1
        for (int i = tl; i < n * n; i += ts) {
            const int yy = i >> log2n, xx = i & (n - 1);
            const int hh = (n - 1 - xx) * R[n2 - yy - 1] + (xx + 1) * tr;
            const int vv = (n - 1 - yy) * R[n2 + xx + 1] + (yy + 1) * bl;
            int v = (hh + vv + n) >> (log2n + 1);
            if (xx < vw && yy < vh) {
                if (coded) v = clamp3i(v + res_at(xx, yy), 0, max_v);
                k.can[cin(k, x0 + xx, y0 + yy)] = (uint16_t)v;
            }
        }
    }
}

// Intra TB of size 16 or 32 by one warp.
__device__ __forceinline__ void intra_tb_big(const Comp& k, int log2n, int mode, int x0, int y0, bool coded,
                                             const uint32_t* stamp, uint32_t jrec, WalkScratch& ws, int lane) {
    intra_tb_prep(k, log2n, mode, x0, y0, stamp, jrec, ws, lane);
    intra_tb_predict(k, log2n, mode, x0, y0, coded, ws, lane);
    __syncwarp();
}

// ---- wavefront progress between neighbouring CTUs ----
// Every CTU publishes, per component, a level: how many of its quadrants
// (z-order: top-left, top-right, bottom-left, bottom-right) are
// reconstructed with their edge samples in the plane.  Other CTUs only read
// a CTU's right column and bottom row, so the levels that matter are 2 (top
// half of the right column), 3 (left half of the bottom row) and 4 (all).
// A CTU reads seven edge segments of its neighbours, each needing one level
// of one neighbour (0 left, 1 above-left, 2 above, 3 above-right):
//   bit 0 above-left corner        above-left  >= 4
//   bit 1 above row, left half      above       >= 3
//   bit 2 above row, right half     above       >= 4
//   bit 3 above-right, left half    above-right >= 3
//   bit 4 above-right, right half   above-right >= 4
//   bit 5 left column, top half     left        >= 2
//   bit 6 left column, bottom half  left        >= 4
constexpr int kSegs = 7;
constexpr uint32_t kSegMask = (1u << kSegs) - 1u;

__device__ __forceinline__ int seg_nb(int s) { return s == 0 ? 1 : (s <= 2 ? 2 : (s <= 4 ? 3 : 0)); }
__device__ __forceinline__ uint32_t seg_level(int s) { return s == 5 ? 2u : ((s == 1 || s == 3) ? 3u : 4u); }
__device__ __forceinline__ int seg_len(int s, int S, int Sh) { return s == 0 ? 1 : (s <= 4 ? S >> 1 : Sh >> 1); }

// Segments of neighbour nb readable once it has reached level v.
__device__ __forceinline__ uint32_t segs_at(int nb, uint32_t v) {
    uint32_t m = 0;
#pragma unroll
    for (int s = 0; s < kSegs; ++s)
        if (seg_nb(s) == nb && seg_level(s) <= v) m |= 1u << s;
    return m;
}

// Edge segments an n x n TB at (x, y) of a component CTU S x Sh reads from
// its neighbours: the row above spans x - 1 .. x + 2n - 1 (intra.rs:84-148),
// the left column y - 1 .. y + 2n - 1, below-left never past the CTU.
__device__ __forceinline__ uint32_t segs_needed(int x, int y, int n, int S, int Sh) {
    uint32_t m = 0;
    const int hs = S >> 1, hh = Sh >> 1;
    if (y == 0) {
        if (x == 0) m |= 1u;
        const int lo = max(x - 1, 0), hi = min(x + 2 * n, S);
        if (lo < hs) m |= 2u;
        if (hi > hs) m |= 4u;
        if (x + 2 * n > S) m |= 8u;
        if (x + 2 * n > S + hs) m |= 16u;
    }
    if (x == 0) {
        const int lo = max(y - 1, 0), hi = min(y + 2 * n, Sh);
        if (lo < hh) m |= 32u;
        if (hi > hh) m |= 64u;
    }
    return m;
}

// One component's neighbour edges as the canvas holds them: row 0 is the
// row above (x = -1 at index 7, x at 8 + x), column 7 the left column.
struct EdgeGeo {
    void* plane;
    uint16_t* can;
    int ox, oy, S, Sh, pw, ph;
};

// Loads the segments m of one component into its canvas, thread t of nt
// taking samples t, t + nt, ... (a rolled loop: this runs inside the walk,
// whose code competes for the instruction cache).  Samples outside the
// picture read as 0 (they are never available).
__device__ __forceinline__ void fetch_edges(const EdgeGeo& e, uint32_t m, int bps, int t, int nt) {
    int total = 0;
#pragma unroll 1
    for (int s = 0; s < kSegs; ++s)
        if (m >> s & 1u) total += seg_len(s, e.S, e.Sh);
#pragma unroll 1
    for (int i = t; i < total; i += nt) {
        int j = i, s = 0;
#pragma unroll 1
        for (; s < kSegs; ++s) {
            if (!(m >> s & 1u)) continue;
            const int L = seg_len(s, e.S, e.Sh);
            if (j < L) break;
            j -= L;
        }
        if (s >= kSegs) break;  // unreachable: i < total
        int dx, dy;
        if (s == 0) {
            dx = -1, dy = -1;
        } else if (s <= 4) {
            dx = (s - 1) * (e.S >> 1) + j, dy = -1;
        } else {
            dx = -1, dy = (s - 5) * (e.Sh >> 1) + j;
        }
        const int ax = e.ox + dx, ay = e.oy + dy;
        int v = 0;
        if (ax >= 0 && ay >= 0 && ax < e.pw && ay < e.ph) v = load_sample_cg(e.plane, bps, (size_t)ay * e.pw + ax);
        e.can[can_at(e.S, dx, dy)] = (uint16_t)v;
    }
}

// Writes the edge samples of quadrants [from, to) of one component to the
// plane (lanes of one warp) and releases level `to`: the warp barrier orders
// every lane's stores before lane 0's release store, which is cumulative.
__device__ __forceinline__ void publish_level(const EdgeGeo& e, int bps, int from, int to, uint32_t* level,
                                              int lane) {
    const int rows = min(e.Sh, e.ph - e.oy), cols = min(e.S, e.pw - e.ox);
    const int hs = e.S >> 1, hh = e.Sh >> 1;
    const bool right = cols == e.S, bottom = rows == e.Sh;  // a neighbour exists on that side
    // right column rows [r0, r1), bottom row cols [b0, b1)
    const int r0 = from < 2 ? 0 : hh, r1 = to >= 4 ? e.Sh : (to >= 2 ? hh : 0);
    const int b0 = from < 3 ? 0 : hs, b1 = to >= 4 ? e.S : (to >= 3 ? hs : 0);
    const int nr = right ? max(0, min(r1, rows) - r0) : 0;
    const int nb = bottom ? max(0, min(b1, cols) - b0) : 0;
    __syncwarp();
    for (int i = lane; i < nr + nb; i += 32) {
        int x, y;
        if (i < nr)
            x = e.S - 1, y = r0 + i;
        else
            x = b0 + i - nr, y = e.Sh - 1;
        store_sample(e.plane, bps, (size_t)(e.oy + y) * e.pw + e.ox + x, e.can[can_in(e.S, x, y)]);
    }
    __syncwarp();
    if (lane == 0) st_release(level, (uint32_t)to);
}

// Edge geometry of component c of CTU (cx, cy) of picture P.
__device__ __forceinline__ EdgeGeo edge_geo(const DevPic& P, uint16_t* can, int c, int cx, int cy) {
    const int ctb = 1 << P.log2_ctb;
    EdgeGeo e;
    e.plane = P.rec[c];
    e.can = can;
    e.S = c ? ctb / P.sub_w : ctb;
    e.Sh = c ? ctb / P.sub_h : ctb;
    e.ox = cx * e.S;
    e.oy = cy * e.Sh;
    e.pw = c ? P.cw : P.w;
    e.ph = c ? P.ch : P.h;
    return e;
}

// The walk's rare step, taken only by TBs flagged when the lists were built
// (a per-TB test in the loop itself costs the walk about 10 %): release the
// quadrants before this TB's (edge samples of quadrants from `prog` on go to
// the plane), then make sure the canvas holds every neighbour segment the
// n x n TB at (x, y) reads: with a courier warp (s_have_c) by waiting for its
// bits, else lanes 0..3 wait (bounded) for one neighbour each and the warp
// loads every segment the levels seen release.  Returns segments held |
// (quadrants done << 8).
__device__ __forceinline__ uint32_t walk_event(const DevPic& P, uint16_t* can, int c, int cx, int cy, int x, int y,
                                            int n, int prog, uint32_t have, uint32_t spin_limit, uint32_t* dev_err,
                                            int lane) {
    const EdgeGeo e = edge_geo(P, can, c, cx, cy);
    const int q = (x >= (e.S >> 1) ? 1 : 0) + (y >= (e.Sh >> 1) ? 2 : 0);
    if (q > prog) {
        if (q >= 2) publish_level(e, P.bps, prog, q, P.ready + ((size_t)cy * P.ctb_cols + cx) * 4 + c, lane);
        prog = q;
    }
    const uint32_t miss = (x == 0 || y == 0) ? segs_needed(x, y, n, e.S, e.Sh) & ~have : 0u;
    if (miss) {
        uint32_t lv = 0u;  // level seen (0: not polled)
        if (lane < 4) {
            uint32_t need = 0;
            for (int s = 0; s < kSegs; ++s)
                if ((miss >> s & 1u) && seg_nb(s) == lane) need = max(need, seg_level(s));
            const int nx = cx + (lane == 3 ? 1 : (lane == 2 ? 0 : -1));
            const int ny = cy - (lane == 0 ? 0 : 1);
            if (nx < 0 || ny < 0 || nx >= P.ctb_cols) {
                lv = 4u;  // outside the picture: nothing to wait for
            } else if (need) {
                const uint32_t* f = P.ready + ((size_t)ny * P.ctb_cols + nx) * 4 + c;
                uint32_t spins = 0;
                while ((lv = ld_acquire(f)) < need) {
                    if (++spins > spin_limit) {
                        atomicOr(dev_err, DEV_ERR_TIMEOUT);
                        lv = need;
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        __syncwarp();  // orders the acquires before every lane's loads
        uint32_t got = 0;
#pragma unroll
        for (int nb = 0; nb < 4; ++nb) got |= segs_at(nb, __shfl_sync(kFull, lv, nb));
        got = (got | miss) & ~have;
        fetch_edges(e, got, P.bps, lane, 32);
        have |= got;
        __syncwarp();
    }
    return have | ((uint32_t)prog << 8);
}

// Warps of a k_recon CTA: warp 0 walks luma, chroma is walked by warp 1
// (Cb, then Cr: kCW = 1) or by warps 1 and 2 (one component each: kCW = 2).
// Two warps keep eight CTU walks resident per SM at 4:2:0 (shared memory
// and registers both allow it); the third warp shortens a CTU whose chroma
// walk is as long as its luma walk (4:4:4).
// Register-capped build (kDense, three warps only): at most 80 registers
// per thread so that eight CTAs of three warps fit an SM instead of five.
// Each walk is a few percent slower, which costs a single picture whose
// wavefront holds few CTUs at a time; a batch with thousands of CTUs ready
// at once is bound by the walks resident per SM instead (a fused batch of
// 256 mixed-size images: reconstruction 73 -> 61 ms).
__host__ __device__ constexpr int recon_warps(int kCW) { return 1 + kCW; }

// kFeat: some picture of the launch has slices / tiles, constrained intra
// prediction, cross-component prediction or I_PCM blocks; without them the
// availability, coded and PCM tests compile to the plain form.  fine: the
// quadrant-level wavefront; otherwise a CTU waits for its neighbours' last
// level before its walk and releases only its last level.
template <int kCW, bool kFeat, bool kDense = false>
__global__ void __launch_bounds__(32 * recon_warps(kCW), kDense ? 8 : (kCW == 1 ? 8 : 5))
k_recon(const DevPic* __restrict__ pics, const CtuItem* __restrict__ items, uint32_t n_items,
        uint32_t* work_counter, uint32_t* dev_err, int cfmt, uint32_t spin_limit, int fine) {
    static_assert(kCW == 1 || kCW == 2, "one or two chroma warps");
    static_assert(!kDense || kCW == 2, "the register-capped build has three warps");
    constexpr int kWarps = recon_warps(kCW), kThreads = 32 * kWarps;
    extern __shared__ __align__(16) unsigned char smem[];
    const ReconLayout lay(cfmt, kWarps);
    uint32_t* s_item = (uint32_t*)(smem + lay.off_misc);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // components walked (and listed) by this warp: [c_lo, c_hi]
    const int c_lo = warp == 0 ? 0 : (kCW == 1 ? 1 : warp), c_hi = warp == 0 ? 0 : (kCW == 1 ? 2 : warp);
    for (;;) {
        __syncthreads();
        if (tid == 0) *s_item = atomicAdd(work_counter, 1u);
        __syncthreads();
        const uint32_t item = *s_item;
        if (item >= n_items) break;
        const CtuItem it = items[item];
        const DevPic& P = pics[it.pic];
        const int ctb = 1 << P.log2_ctb;
        const int ncomp = P.idc ? 3 : 1;
        const int oxl = it.cx * ctb, oyl = it.cy * ctb;
        // chroma CTU: Scw x Sch samples (4:2:2: half as wide as tall)
        const int ocx = oxl / P.sub_w, ocy = oyl / P.sub_h, Scw = ctb / P.sub_w, Sch = ctb / P.sub_h;
        const uint32_t ci = (uint32_t)it.cy * P.ctb_cols + it.cx;
        uint32_t r0 = P.ctu_start[ci], r1 = P.ctu_start[ci + 1];
        if (r1 > P.n_tus || r0 > r1) {  // malformed CTU range: report, reconstruct nothing
            if (tid == 0) atomicOr(dev_err, DEV_ERR_BITSTREAM);
            r1 = min(r1, P.n_tus);
            r0 = min(r0, r1);
        }
        uint32_t nrec = r1 - r0;
        if (nrec > (uint32_t)lay.rec_cap) {  // more records than a CTU can hold
            if (tid == 0) atomicOr(dev_err, DEV_ERR_BITSTREAM);
            nrec = (uint32_t)lay.rec_cap;
        }
        uint4* recs = (uint4*)(smem + lay.off_recs);
        uint32_t* stamp = (uint32_t*)(smem + lay.off_stamp);
        uint16_t* lists = (uint16_t*)(smem + lay.off_lists);
        uint32_t* counts = (uint32_t*)(smem + lay.off_misc) + 1;
        auto can_of = [&](int c) -> uint16_t* {
            return c == 0 ? (uint16_t*)(smem + lay.off_can_y)
                          : (uint16_t*)(smem + lay.off_can_c) + (size_t)(c - 1) * can_size(lay.cs_w, lay.cs_h);
        };
        // the CTU's records (16 bytes each; the record array is 16-byte aligned)
        for (uint32_t i = tid; i < nrec; i += kThreads) cp_async16(recs + i, P.tus + r0 + i);
        asm volatile("cp.async.commit_group;" ::: "memory");
        for (int i = tid; i < 256; i += kThreads) stamp[i] = kNoStamp;
        // the CTU's own records have arrived: the decode-order build below
        // runs before the neighbour wait, off the critical path
        cp_async_wait_all();
        __syncthreads();
        // ---- decode order, in parallel: every luma record stamps the 4x4
        // cells it marks decoded (decode.rs:3170-3189; cells outside the
        // picture stay unmarked), and each warp lists the intra TBs of its
        // components in decode order ----
        const int vis_w = min(64, P.w - oxl), vis_h = min(64, P.h - oyl);
        const bool intra_pred_ok = !(P.flags & HPVCD_PIC_PRED_IN_PLANE);
        // validity of record i for component tc: -1 skip silently, 0 invalid
        // (reported), 1 usable; (x, y) relative to the CTU
        auto rec_check = [&](const hpvcd_tu& t, int& x, int& y) -> int {
            const int tc = t.comp;
            if (tc >= ncomp || t.log2n < 2 || t.log2n > 6) return -1;
            const int n = 1 << t.log2n;
            x = (int)t.x - (tc ? ocx : oxl);
            y = (int)t.y - (tc ? ocy : oyl);
            const int Sw = tc ? Scw : ctb, Sh = tc ? Sch : ctb;
            return (x < 0 || y < 0 || x + n > Sw || y + n > Sh) ? 0 : 1;
        };
        for (uint32_t i = tid; i < nrec; i += kThreads) {
            hpvcd_tu t;
            memcpy(&t, &recs[i], sizeof(t));
            int x, y;
            const int ok = rec_check(t, x, y);
            if (ok == 0) atomicOr(dev_err, DEV_ERR_BITSTREAM);
            if (ok != 1 || t.comp != 0) continue;
            const int n = 1 << t.log2n;
            const int x1 = min(x + n, vis_w), y1 = min(y + n, vis_h);
            for (int cy = y >> 2; cy < (y1 + 3) >> 2; ++cy)
                for (int cx = x >> 2; cx < (x1 + 3) >> 2; ++cx) atomicMin(&stamp[cy * 16 + cx], i);
        }
        for (int c = c_lo; c <= c_hi && c < ncomp; ++c) {
            const int hs = (c ? Scw : ctb) >> 1, hh = (c ? Sch : ctb) >> 1;
            const uint32_t cap = (uint32_t)lay.list_cap(c);
            uint16_t* list = lists + lay.list_off(c);
            uint32_t cnt = 0;
            int qmax = 0;  // quadrant of the entries listed so far (z-order: never decreases)
            for (uint32_t base = 0; base < nrec; base += 32) {
                const uint32_t i = base + lane;
                bool mine = false;
                int q = -1;
                bool edge = false;
                if (i < nrec) {
                    hpvcd_tu t;
                    memcpy(&t, &recs[i], sizeof(t));
                    int x, y;
                    if (t.comp == c && (t.flags & HPVCD_TU_INTRA) && intra_pred_ok && rec_check(t, x, y) == 1) {
                        if (t.mode > 34 || t.log2n > 5) {
                            atomicOr(dev_err, DEV_ERR_BITSTREAM);
                        } else {
                            mine = true;
                            q = (x >= hs ? 1 : 0) + (y >= hh ? 2 : 0);
                            edge = x == 0 || y == 0;
                        }
                    }
                }
                // running maximum of q over the list order: an entry that opens
                // a later quadrant, or sits on the CTU's top / left edge, is an
                // event of the quadrant-level wavefront
                int run = q;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int o = __shfl_up_sync(kFull, run, d);
                    if (lane >= d) run = max(run, o);
                }
                int before = __shfl_up_sync(kFull, run, 1);
                before = max(lane ? before : -1, qmax);
                qmax = max(qmax, __shfl_sync(kFull, run, 31));
                const bool event = fine && (q > before || edge);
                const uint32_t m = __ballot_sync(kFull, mine);
                const uint32_t pos = cnt + __popc(m & ((1u << lane) - 1u));
                if (mine && pos < cap) list[pos] = (uint16_t)(i | (event ? kListEvent : 0u));
                cnt += __popc(m);
            }
            if (cnt > cap) {
                if (lane == 0) atomicOr(dev_err, DEV_ERR_BITSTREAM);
                cnt = cap;
            }
            if (lane == 0) counts[c] = cnt;
        }
        __syncthreads();
        // A CTU without intra TBs (inter pictures) has its final samples in the
        // plane already: it neither waits for its neighbours nor rewrites
        // anything, it only releases every component for the CTUs that
        // predict from it.
        const bool any_intra = counts[0] + (ncomp > 1 ? counts[1] + counts[2] : 0u) > 0u;
        uint32_t* level = P.ready + (size_t)ci * 4;  // per-component progress of this CTU
        if (!any_intra) {
            if (tid < ncomp) st_release(level + tid, 4u);
            continue;
        }
        // Inter pictures: the plane holds motion-compensated + residual
        // samples; load the CTU interior so intra TBs can predict from it.
        if (P.flags & HPVCD_PIC_INTER) {
            for (int c = 0; c < ncomp; ++c) {
                const int S = c ? Scw : ctb, Sh = c ? Sch : ctb, ox = c ? ocx : oxl, oy = c ? ocy : oyl;
                const int pw = c ? P.cw : P.w, ph = c ? P.ch : P.h;
                uint16_t* can = can_of(c);
                for (int i = tid; i < S * Sh; i += kThreads) {
                    const int y = i / S, x = i % S;
                    const int ax = ox + x, ay = oy + y;
                    int v = 0;
                    if (ax < pw && ay < ph) v = load_sample(P.rec[c], P.bps, (size_t)ay * pw + ax);
                    can[can_in(S, x, y)] = (uint16_t)v;
                }
            }
        }
        // neighbour CTUs that intra prediction may read: same slice and tile
        // (decode.rs:4651-4690)
        uint32_t nb_ok = 0xfu;
        if (kFeat && P.ctb_region) {
            const uint16_t me = P.ctb_region[ci];
            const int cx = it.cx, cy = it.cy;
            auto same = [&](int nx, int ny) {
                return nx >= 0 && ny >= 0 && nx < P.ctb_cols && P.ctb_region[(size_t)ny * P.ctb_cols + nx] == me;
            };
            nb_ok = (same(cx - 1, cy) ? 1u : 0u) | (same(cx - 1, cy - 1) ? 2u : 0u) | (same(cx, cy - 1) ? 4u : 0u) |
                    (same(cx + 1, cy - 1) ? 8u : 0u);
        }
        // ---- neighbour edges available now: one level read per neighbour
        // and component, then every segment already released is loaded ----
        auto geo = [&](int c) { return edge_geo(P, can_of(c), c, it.cx, it.cy); };
        uint32_t* s_have = (uint32_t*)(smem + lay.off_misc) + 4;
        uint32_t* s_lvl = (uint32_t*)(smem + lay.off_misc) + 8;
        // neighbour nb of this CTU: its level words, or null outside the picture
        auto nb_level = [&](int nb) -> const uint32_t* {
            const int nx = it.cx + (nb == 3 ? 1 : (nb == 2 ? 0 : -1));
            const int ny = it.cy - (nb == 0 ? 0 : 1);
            if (nx < 0 || ny < 0 || nx >= P.ctb_cols) return nullptr;
            return P.ready + ((size_t)ny * P.ctb_cols + nx) * 4;
        };
        if (tid < 4 * ncomp) {
            const uint32_t* f = nb_level(tid & 3);
            uint32_t v = 4u;
            if (f) {
                v = ld_acquire(f + (tid >> 2));
                uint32_t spins = 0;
                while (!fine && v < 4u) {  // whole-CTU wavefront: wait (bounded) for the last level
                    if (++spins > spin_limit) {
                        atomicOr(dev_err, DEV_ERR_TIMEOUT);
                        v = 4u;
                        break;
                    }
                    __nanosleep(64);
                    v = ld_acquire(f + (tid >> 2));
                }
            }
            s_lvl[tid] = v;
        }
        __syncthreads();
        // Everything one walking warp needs about component c of this CTU.
        auto comp_of = [&](int c) -> Comp {
            Comp k;
            k.S = c ? Scw : ctb;
            k.Sh = c ? Sch : ctb;
            k.ox = c ? ocx : oxl;
            k.oy = c ? ocy : oyl;
            k.pw = c ? P.cw : P.w;
            k.ph = c ? P.ch : P.h;
            k.sw = c ? P.sub_w : 1;
            k.sh = c ? P.sub_h : 1;
            k.nb_ok = nb_ok;
            k.ci_cells = kFeat && (P.flags & HPVCD_PIC_CONSTRAINED_INTRA) ? P.cells : nullptr;
            k.gw = P.gw;
            k.restricted = kFeat && (nb_ok != 0xfu || k.ci_cells != nullptr);
            k.ccp = kFeat && c && (P.flags & HPVCD_PIC_CROSS_COMPONENT);
            k.bd = c ? P.bd_c : P.bd;
            k.max_v = (1 << k.bd) - 1;
            k.luma = c == 0;
            k.filt = c == 0 || P.idc == 3;
            k.smoothing = !(P.flags & HPVCD_PIC_SMOOTHING_DISABLED);
            k.strong = (P.flags & HPVCD_PIC_STRONG_SMOOTHING) != 0;
            k.can = can_of(c);
            k.rs = P.res_stride[c];
            k.res = P.res[c] + (size_t)k.oy * k.rs + k.ox;
            return k;
        };
        // ---- residuals into the canvas, before the walk: the copies overlap
        // the neighbour edge loads below.  In an intra picture every sample
        // of the CTU comes from the walk, so the whole visible residual block
        // of each component is copied by all threads (the areas of uncoded
        // TBs are never read); in an inter picture the canvas holds inter
        // samples, so only the areas of coded intra TBs are staged (one lane
        // of the walking warp per list entry) ----
        if (!(P.flags & HPVCD_PIC_INTER)) {
            for (int c = 0; c < ncomp; ++c) {
                const int S = c ? Scw : ctb, Sh = c ? Sch : ctb, ox = c ? ocx : oxl, oy = c ? ocy : oyl;
                const int rows = min(Sh, (c ? P.ch : P.h) - oy), cols = min(S, (c ? P.cw : P.w) - ox);
                const int chunks = (cols + 7) >> 3;
                const int rs = P.res_stride[c];
                const int16_t* res = P.res[c] + (size_t)oy * rs + ox;
                uint16_t* can = can_of(c);
                for (int i = tid; i < rows * chunks; i += kThreads) {
                    const int r = i / chunks, q = i - r * chunks;
                    cp_async16(can + can_in(S, 8 * q, r), res + (size_t)r * rs + 8 * q);
                }
            }
        } else {
            for (int c = c_lo; c <= c_hi && c < ncomp; ++c) {
                const Comp k = comp_of(c);
                const uint32_t cnt = counts[c];
                const uint16_t* list = lists + lay.list_off(c);
                for (uint32_t e = lane; e < cnt; e += 32) {
                    hpvcd_tu t;
                    const uint4 w4 = recs[list[e] & kListRec];
                    memcpy(&t, &w4, sizeof(t));
                    const bool coded = (t.flags & HPVCD_TU_CBF) != 0 || (k.ccp && t.res_scale);
                    if (coded && !(kFeat && (t.flags & HPVCD_TU_PCM)))
                        stage_residual(k, t.log2n, (int)t.x - k.ox, (int)t.y - k.oy);
                }
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        if (tid < ncomp) {
            uint32_t h = 0;
            for (int nb = 0; nb < 4; ++nb) h |= segs_at(nb, s_lvl[tid * 4 + nb]);
            s_have[tid] = h;
        }
        __syncthreads();
        for (int c = 0; c < ncomp; ++c) fetch_edges(geo(c), s_have[c], P.bps, tid, kThreads);
        cp_async_wait_all();  // this thread's residual copies; the barrier publishes them
        __syncthreads();
        // ---- decode-order walk: each warp reconstructs its components ----
        WalkScratch& ws = *(WalkScratch*)(smem + lay.off_ws + (size_t)warp * kWsBytes);
        for (int c = c_lo; c <= c_hi && c < ncomp; ++c) {
            const Comp k = comp_of(c);
            const uint32_t cnt = counts[c];
            const uint16_t* list = lists + lay.list_off(c);
            // edge segments in the canvas, quadrants released
            uint32_t have = s_have[c];
            int prog = 0;
            // the next record is fetched while the current TB is reconstructed
            uint32_t jn = cnt ? list[0] : 0u;
            uint4 wn = cnt ? recs[jn & kListRec] : make_uint4(0u, 0u, 0u, 0u);
            for (uint32_t e = 0; e < cnt; ++e) {
                const uint32_t j = jn & kListRec;
                const bool event = (jn & kListEvent) != 0u;
                hpvcd_tu t;
                memcpy(&t, &wn, sizeof(t));
                if (e + 1 < cnt) {
                    jn = list[e + 1];
                    wn = recs[jn & kListRec];
                }
                const int x = (int)t.x - k.ox, y = (int)t.y - k.oy;
                if (event) {
                    const uint32_t r = walk_event(P, k.can, c, it.cx, it.cy, x, y, 1 << t.log2n, prog, have, spin_limit,
                                                  dev_err, lane);
                    have = r & kSegMask;
                    prog = (int)(r >> 8);
                }
                // a chroma TB with cross-component prediction has a residual
                // (written by k_ccp) even without coded coefficients
                const bool coded = (t.flags & HPVCD_TU_CBF) != 0 || (k.ccp && t.res_scale);
                if (kFeat && (t.flags & HPVCD_TU_PCM)) {
                    pcm_tb(k, t.log2n, x, y, lane);
                } else if (t.log2n == 2) {
                    intra_tb4(k, t.mode, x, y, coded, stamp, j, lane);
                } else if (t.log2n == 3) {
                    intra_tb8(k, t.mode, x, y, coded, stamp, j, lane);
                } else {
                    intra_tb_big(k, t.log2n, t.mode, x, y, coded, stamp, j, ws, lane);
                }
            }
            publish_level(geo(c), P.bps, prog, 4, level + c, lane);
        }
        __syncthreads();
        // ---- write the CTU out for the filters (8 samples per store when
        // rows allow); the kernel boundary orders it before them ----
        for (int c = 0; c < ncomp; ++c) {
            const int S = c ? Scw : ctb, Sh = c ? Sch : ctb, ox = c ? ocx : oxl, oy = c ? ocy : oyl;
            const int pw = c ? P.cw : P.w, ph = c ? P.ch : P.h;
            const uint16_t* can = can_of(c);
            const int rows = min(Sh, ph - oy), cols = min(S, pw - ox);
            if ((pw & 7) == 0 && (cols & 7) == 0) {
                const int chunks = cols >> 3;
                for (int i = tid; i < rows * chunks; i += kThreads) {
                    const int y = i / chunks, q = i % chunks;
                    const uint4 v = *(const uint4*)(can + can_in(S, 8 * q, y));
                    const size_t off = (size_t)(oy + y) * pw + ox + 8 * q;
                    if (P.bps == 2) {
                        *(uint4*)((uint16_t*)P.rec[c] + off) = v;
                    } else {
                        const uint32_t lo = (v.x & 0xffu) | ((v.x >> 8) & 0xff00u) | ((v.y & 0xffu) << 16) |
                                            ((v.y & 0xff0000u) << 8);
                        const uint32_t hi = (v.z & 0xffu) | ((v.z >> 8) & 0xff00u) | ((v.w & 0xffu) << 16) |
                                            ((v.w & 0xff0000u) << 8);
                        *(uint2*)((uint8_t*)P.rec[c] + off) = make_uint2(lo, hi);
                    }
                }
            } else {
                for (int i = tid; i < rows * cols; i += kThreads) {
                    const int y = i / cols, x = i % cols;
                    store_sample(P.rec[c], P.bps, (size_t)(oy + y) * pw + ox + x, can[can_in(S, x, y)]);
                }
            }
        }
    }
}

}  // namespace hpvcd

extern "C" size_t hpvcd_recon_smem_bytes(int cfmt, int chroma_warps) {
    return hpvcd::ReconLayout(cfmt, hpvcd::recon_warps(chroma_warps == 1 ? 1 : 2)).total;
}

extern "C" cudaError_t hpvcd_launch_residual(const hpvcd::DevPic* pics, const uint32_t* rec_prefix,
                                             uint32_t n_pics, uint32_t total_records, uint32_t* dev_err,
                                             int sms, int idct, cudaStream_t stream) {
    if (total_records == 0) return cudaSuccess;
    const uint32_t chunks = (total_records + hpvcd::kResChunk - 1) / hpvcd::kResChunk;
    const uint32_t blocks_needed = (chunks + hpvcd::kResWarps - 1) / hpvcd::kResWarps;
    const uint32_t cap = (uint32_t)sms * 8u;
    const int grid = (int)(blocks_needed < cap ? blocks_needed : cap);
    // schedule value: 0 integer tensor cores (the default), 1 butterflies, 2 matrix product
    if (idct == 0)
        hpvcd::k_residual<hpvcd::kIdctTensor><<<grid, hpvcd::kResWarps * 32, 0, stream>>>(pics, rec_prefix, n_pics,
                                                                                        dev_err);
    else if (idct == 1)
        hpvcd::k_residual<hpvcd::kIdctButterfly><<<grid, hpvcd::kResWarps * 32, 0, stream>>>(pics, rec_prefix,
                                                                                          n_pics, dev_err);
    else
        hpvcd::k_residual<hpvcd::kIdctMatrix><<<grid, hpvcd::kResWarps * 32, 0, stream>>>(pics, rec_prefix, n_pics,
                                                                                       dev_err);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

extern "C" cudaError_t hpvcd_launch_ccp(const hpvcd::DevPic* pics, const uint32_t* rec_prefix, uint32_t n_pics,
                                        uint32_t total_records, uint32_t* dev_err, int sms, cudaStream_t stream) {
    if (total_records == 0) return cudaSuccess;
    const uint32_t blocks_needed = (total_records + hpvcd::kCcpWarps - 1) / hpvcd::kCcpWarps;
    const uint32_t cap = (uint32_t)sms * 8u;
    const int grid = (int)(blocks_needed < cap ? blocks_needed : cap);
    hpvcd::k_ccp<<<grid, hpvcd::kCcpWarps * 32, 0, stream>>>(pics, rec_prefix, n_pics, dev_err);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

extern "C" cudaError_t hpvcd_launch_recon(const hpvcd::DevPic* pics, const hpvcd::CtuItem* items,
                                          uint32_t n_items, uint32_t* work_counter, uint32_t* dev_err,
                                          int cfmt, int grid, int chroma_warps, int feat, int fine, uint32_t spin,
                                          cudaStream_t stream) {
    if (n_items == 0) return cudaSuccess;
    // the dynamic shared-memory limit was raised by hpvcd_recon_occupancy()
    // when the plan was built (no non-stream API call here, so launches can
    // be captured into CUDA graphs)
    // build: 1 one chroma warp (Cb, then Cr), 2 one warp per chroma
    // component, 3 the same in the register-capped build
    const int cw = chroma_warps == 1 ? 1 : 2;
    const size_t smem = hpvcd::ReconLayout(cfmt, hpvcd::recon_warps(cw)).total;
    const int threads = 32 * hpvcd::recon_warps(cw);
    // default: 2^22 polls of >= 64 ns each bound one neighbour wait to a few
    // hundred ms
    if (spin == 0) spin = 1u << 22;
    if (chroma_warps == 3 && feat)
        hpvcd::k_recon<2, true, true><<<grid, threads, smem, stream>>>(pics, items, n_items, work_counter, dev_err,
                                                                       cfmt, spin, fine);
    else if (chroma_warps == 3)
        hpvcd::k_recon<2, false, true><<<grid, threads, smem, stream>>>(pics, items, n_items, work_counter, dev_err,
                                                                        cfmt, spin, fine);
    else if (cw == 2 && feat)
        hpvcd::k_recon<2, true><<<grid, threads, smem, stream>>>(pics, items, n_items, work_counter, dev_err, cfmt,
                                                                 spin, fine);
    else if (cw == 2)
        hpvcd::k_recon<2, false><<<grid, threads, smem, stream>>>(pics, items, n_items, work_counter, dev_err, cfmt,
                                                                  spin, fine);
    else if (feat)
        hpvcd::k_recon<1, true><<<grid, threads, smem, stream>>>(pics, items, n_items, work_counter, dev_err, cfmt,
                                                                 spin, fine);
    else
        hpvcd::k_recon<1, false><<<grid, threads, smem, stream>>>(pics, items, n_items, work_counter, dev_err, cfmt,
                                                                  spin, fine);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}

namespace {
// Every instantiation: the shared-memory limit of the 4:4:4 layout of three
// warps (the largest) and the whole unified L1 / shared array as shared
// memory.  The common carveout matters when waves of different layouts
// (4:2:0 and 4:4:4, one stream per concurrent group of a batch) follow each
// other on the SMs: an SM changes its L1 / shared split only when it holds
// no CTA, so a wave that wanted a larger split than the one running could
// start only once the other groups' waves had drained every SM.
template <int kCW, bool kFeat, bool kDense>
void recon_attrs(int lim) {
    cudaFuncSetAttribute(hpvcd::k_recon<kCW, kFeat, kDense>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(hpvcd::k_recon<kCW, kFeat, kDense>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
}

// Occupancy of one build with the layout of `cfmt` (attributes already set).
int recon_occupancy_of(int cfmt, int chroma_warps) {
    int blocks = 0;
    const int cw = chroma_warps == 1 ? 1 : 2;
    const size_t smem = hpvcd::ReconLayout(cfmt, hpvcd::recon_warps(cw)).total;
    if (chroma_warps == 3)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, hpvcd::k_recon<2, false, true>,
                                                      32 * hpvcd::recon_warps(2), smem);
    else if (cw == 2)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, hpvcd::k_recon<2, false>, 32 * hpvcd::recon_warps(2),
                                                      smem);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, hpvcd::k_recon<1, false>, 32 * hpvcd::recon_warps(1),
                                                      smem);
    return blocks;
}

// Attributes and occupancies are set up once per device: every plan build
// asks for them, and a serving loop builds a plan for every new batch
// layout (setting the attributes of every instantiation each time cost
// milliseconds per plan).  Like the no-allocation entry point's per-device
// set-up, this assumes the device's primary context lives until the process
// exits (no cudaDeviceReset while the library is in use).
constexpr int kAttrDevices = 64;
std::mutex g_attr_mu;
bool g_attr_done[kAttrDevices];
int g_attr_occ[kAttrDevices][3][3];
}  // namespace

// CTAs per SM of the wavefront kernel with the layout of `cfmt` in build
// `chroma_warps` (1 two warps, 2 three warps, 3 three warps register-capped;
// 0 counts as 2); the first call on a device sets the attributes of every
// instantiation (recon_attrs) and of the residual kernel.
extern "C" int hpvcd_recon_occupancy(int cfmt, int chroma_warps) {
    const int build = chroma_warps >= 1 && chroma_warps <= 3 ? chroma_warps : 2;
    const int cf = cfmt >= 0 && cfmt <= 2 ? cfmt : 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kAttrDevices) {
        cudaGetLastError();
        dev = -1;
    }
    std::lock_guard<std::mutex> lock(g_attr_mu);
    if (dev >= 0 && g_attr_done[dev]) return g_attr_occ[dev][cf][build - 1];
    const int lim = (int)hpvcd::ReconLayout(hpvcd::kFmt444, hpvcd::recon_warps(2)).total;
    recon_attrs<1, false, false>(lim);
    recon_attrs<2, false, false>(lim);
    recon_attrs<1, true, false>(lim);
    recon_attrs<2, true, false>(lim);
    recon_attrs<2, false, true>(lim);
    recon_attrs<2, true, true>(lim);
    // the residual pre-pass of one group runs beside another group's waves
    cudaFuncSetAttribute(hpvcd::k_residual<hpvcd::kIdctMatrix>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    cudaFuncSetAttribute(hpvcd::k_residual<hpvcd::kIdctButterfly>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    cudaFuncSetAttribute(hpvcd::k_residual<hpvcd::kIdctTensor>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    if (dev < 0) return recon_occupancy_of(cf, build);
    for (int f = 0; f < 3; ++f)
        for (int b = 1; b <= 3; ++b) g_attr_occ[dev][f][b - 1] = recon_occupancy_of(f, b);
    g_attr_done[dev] = true;
    return g_attr_occ[dev][cf][build - 1];
}
