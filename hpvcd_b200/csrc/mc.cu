// mc.cu -- motion compensation (mc.rs + decode.rs:7000-7488 motion_compensate).
//
// One CTA per PU and component; each thread produces whole output samples:
// the separable 8-tap (luma, quarter-pel) / 4-tap (chroma, eighth-pel)
// interpolation into 14-bit intermediates (mc.rs:351-530, edge-clamped
// reference fetch mc.rs:310), then the uni / bi / explicitly weighted
// combination with clipping (mc.rs:538-736), written straight into the
// current picture's plane.  Bi-prediction needs no intermediate buffer: a
// thread evaluates both lists for its sample.
#include "common.cuh"

namespace hpvcd {

// mc.rs:30-45
__constant__ int8_t c_luma_filter[4][8] = {{0, 0, 0, 64, 0, 0, 0, 0},
                                           {-1, 4, -10, 58, 17, -5, 1, 0},
                                           {-1, 4, -11, 40, 40, -11, 4, -1},
                                           {0, 1, -5, 17, 58, -10, 4, -1}};
__constant__ int8_t c_chroma_filter[8][4] = {{0, 64, 0, 0},   {-2, 58, 10, -2}, {-4, 54, 16, -2},
                                             {-6, 46, 28, -4}, {-4, 36, 36, -4}, {-4, 28, 46, -6},
                                             {-2, 16, 54, -4}, {-2, 10, 58, -2}};

struct RefView {
    const void* data;
    int bps, w, h;
    __device__ __forceinline__ int sample(int x, int y) const {
        x = clamp3i(x, 0, w - 1);
        y = clamp3i(y, 0, h - 1);
        return load_sample(data, bps, (size_t)y * w + x);
    }
};

// 14-bit intermediate of one sample (mc.rs:351-439 luma, :442-530 chroma).
template <int TAPS>
__device__ __forceinline__ int interp_sample(const RefView& r, int x, int y, int fx, int fy, int bd) {
    const int s1 = bd - 8;
    const int back = TAPS / 2 - 1;
    auto hf = [&](int t) { return TAPS == 8 ? (int)c_luma_filter[fx][t] : (int)c_chroma_filter[fx][t]; };
    auto vf = [&](int t) { return TAPS == 8 ? (int)c_luma_filter[fy][t] : (int)c_chroma_filter[fy][t]; };
    if (fx == 0 && fy == 0) return (int)(int16_t)((r.sample(x, y) << 6) >> s1);
    if (fy == 0) {
        int acc = 0;
#pragma unroll
        for (int t = 0; t < TAPS; ++t) acc += hf(t) * r.sample(x - back + t, y);
        return (int)(int16_t)(acc >> s1);
    }
    if (fx == 0) {
        int acc = 0;
#pragma unroll
        for (int t = 0; t < TAPS; ++t) acc += vf(t) * r.sample(x, y - back + t);
        return (int)(int16_t)(acc >> s1);
    }
    int acc = 0;
#pragma unroll
    for (int v = 0; v < TAPS; ++v) {
        int h = 0;
#pragma unroll
        for (int t = 0; t < TAPS; ++t) h += hf(t) * r.sample(x - back + t, y - back + v);
        acc += vf(v) * (h >> s1);  // intermediate kept in i32 (mc.rs:408-418)
    }
    return (int)(int16_t)(acc >> 6);
}

// blockIdx.x = PU, blockIdx.y = component.
__global__ void k_mc(const DevPic* __restrict__ pics, int pic_index) {
    const DevPic& P = pics[pic_index];
    const int c = blockIdx.y;
    if (c > 0 && P.idc == 0) return;
    const hpvcd_pu u = P.pus[blockIdx.x];
    const bool luma = c == 0;
    const int sw = luma ? 1 : P.sub_w, sh = luma ? 1 : P.sub_h;
    const int bw = u.w / sw, bh = u.h / sh;
    const int bx = u.x / sw, by = u.y / sh;
    const int pw = luma ? P.w : P.cw, ph = luma ? P.h : P.ch;
    if (bw <= 0 || bh <= 0 || bx >= pw || by >= ph) return;
    const int vw = min(bw, pw - bx), vh = min(bh, ph - by);
    const int bd = luma ? P.bd : P.bd_c;
    const int mx = (1 << bd) - 1;
    // reference views per list (decode.rs:7040-7120 ref_frame_for_lists)
    RefView rv[2];
    bool have[2] = {false, false};
    int ix[2], iy[2], fx[2], fy[2];
    for (int l = 0; l < 2; ++l) {
        if (!(u.flags & (l ? HPVCD_PU_L1 : HPVCD_PU_L0))) continue;
        const int ri = u.ref_idx[l];
        if (ri < 0 || ri >= HPVCD_MAX_REFS) continue;
        const int rp = P.ref_pic[l][ri];
        // the host maps references to earlier pictures of the batch (< pic_index)
        // or to DPB pictures appended after the batch's own; -1 is none
        if (rp < 0 || rp == pic_index) continue;
        const DevPic& R = pics[rp];
        rv[l] = RefView{R.fin[c], R.bps, pw, ph};
        have[l] = true;
        if (luma) {
            ix[l] = bx + (u.mv[l][0] >> 2);
            iy[l] = by + (u.mv[l][1] >> 2);
            fx[l] = u.mv[l][0] & 3;
            fy[l] = u.mv[l][1] & 3;
        } else {  // decode.rs:7282-7287, Rust `/` truncates toward zero like C
            const int mvcx = u.mv[l][0] * 2 / P.sub_w, mvcy = u.mv[l][1] * 2 / P.sub_h;
            ix[l] = bx + (mvcx >> 3);
            iy[l] = by + (mvcy >> 3);
            fx[l] = mvcx & 7;
            fy[l] = mvcy & 7;
        }
    }
    const int denom = P.has_wp ? (luma ? P.wp.luma_log2_denom : P.wp.chroma_log2_denom) : 0;
    auto wpair = [&](int l, int& wgt, int& off) {
        const hpvcd_wp_entry& e = P.wp.e[l][max((int)u.ref_idx[l], 0)];
        wgt = luma ? e.luma_w : (c == 1 ? e.cb_w : e.cr_w);
        off = luma ? e.luma_o : (c == 1 ? e.cb_o : e.cr_o);
    };
    void* dst = P.rec[c];
    for (int i = threadIdx.x; i < vw * vh; i += blockDim.x) {
        const int xx = i % vw, yy = i / vw;
        int a = 0, b = 0;
        if (have[0])
            a = luma ? interp_sample<8>(rv[0], ix[0] + xx, iy[0] + yy, fx[0], fy[0], bd)
                     : interp_sample<4>(rv[0], ix[0] + xx, iy[0] + yy, fx[0], fy[0], bd);
        if (have[1])
            b = luma ? interp_sample<8>(rv[1], ix[1] + xx, iy[1] + yy, fx[1], fy[1], bd)
                     : interp_sample<4>(rv[1], ix[1] + xx, iy[1] + yy, fx[1], fy[1], bd);
        int v;
        if (have[0] && have[1]) {
            if (P.has_wp) {  // mc.rs:682-736
                int w0, o0, w1, o1;
                wpair(0, w0, o0);
                wpair(1, w1, o1);
                const int log2_wd = denom + 14 - bd;
                const long long rnd = ((long long)o0 + o1 + 1) << log2_wd;
                const long long t = ((long long)a * w0 + (long long)b * w1 + rnd) >> (log2_wd + 1);
                v = (int)(t < 0 ? 0 : (t > mx ? mx : t));
            } else {  // mc.rs:579-629
                const int shift = 15 - bd;
                v = clamp3i((a + b + (1 << (shift - 1))) >> shift, 0, mx);
            }
        } else if (have[0] || have[1]) {
            const int s = have[0] ? a : b;
            if (P.has_wp) {  // mc.rs:631-680
                int wg, of;
                wpair(have[0] ? 0 : 1, wg, of);
                const int log2_wd = denom + 14 - bd;
                const int t = log2_wd >= 1 ? ((s * wg + (1 << (log2_wd - 1))) >> log2_wd) + of : s * wg + of;
                v = clamp3i(t, 0, mx);
            } else {  // mc.rs:538-577
                const int shift = 14 - bd;
                v = clamp3i((s + (shift > 0 ? 1 << (shift - 1) : 0)) >> shift, 0, mx);
            }
        } else {  // decode.rs:7206-7216: missing reference -> mid-grey
            v = 1 << (bd - 1);
        }
        store_sample(dst, P.bps, (size_t)(by + yy) * pw + bx + xx, v);
    }
}

}  // namespace hpvcd

extern "C" cudaError_t hpvcd_launch_mc(const hpvcd::DevPic* pics, int pic_index, int n_pus, int n_comp,
                                       cudaStream_t stream) {
    if (n_pus <= 0) return cudaSuccess;
    dim3 grid(n_pus, n_comp);
    hpvcd::k_mc<<<grid, 256, 0, stream>>>(pics, pic_index);
    hpvcd_note_launches(1);
    return cudaGetLastError();
}
