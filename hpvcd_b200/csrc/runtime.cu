// runtime.cu -- host runtime behind include/hpvcd_gpu.h: plans (device
// buffers, kernel schedule), contexts (host buffers, staging, streams,
// tickets, HBM admission) and the exported C entry points.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "common.cuh"
#include "hostcopy.h"
#include "hpvcd_syntax.h"

#define HPVCD_API extern "C" __attribute__((visibility("default")))

using hpvcd::CtuItem;
using hpvcd::DevPic;

extern "C" cudaError_t hpvcd_launch_residual(const DevPic*, const uint32_t*, uint32_t, uint32_t, uint32_t*, int,
                                             int, cudaStream_t);
extern "C" cudaError_t hpvcd_launch_ccp(const DevPic*, const uint32_t*, uint32_t, uint32_t, uint32_t*, int,
                                        cudaStream_t);
extern "C" cudaError_t hpvcd_launch_recon(const DevPic*, const CtuItem*, uint32_t, uint32_t*, uint32_t*, int, int,
                                          int, int, int, uint32_t, cudaStream_t);
extern "C" int hpvcd_recon_occupancy(int cfmt, int chroma_warps);
extern "C" hpvcd_status hpvcd_mlp_host_copy(hpvcd_mlp* M, float* params, float* lohi, int* has_domain);
extern "C" uint32_t hpvcd_mlp_pick_host(const float* w, uint32_t K, const float* x, const float* lohi,
                                        int has_domain);
extern "C" cudaError_t hpvcd_launch_deblock(const DevPic*, int, int, int, cudaStream_t);
extern "C" cudaError_t hpvcd_launch_sao(const DevPic*, int, int, int, cudaStream_t);
extern "C" cudaError_t hpvcd_launch_rgb(const DevPic*, int, int, uint8_t*, cudaStream_t);
extern "C" cudaError_t hpvcd_launch_yuv_canvas(const DevPic*, int, int, uint8_t*, cudaStream_t);
extern "C" cudaError_t hpvcd_launch_filter_tile(const DevPic*, int, int, int, int, uint8_t*, cudaStream_t);
extern "C" cudaError_t hpvcd_filter_tile_setup();
extern "C" cudaError_t hpvcd_launch_mc(const DevPic*, int, int, int, cudaStream_t);
extern "C" hpvcd_status hpvcd_mlp_pick(hpvcd_mlp*, const float*, uint32_t, void*, uint32_t*);
extern "C" uint32_t hpvcd_mlp_variants(const hpvcd_mlp*);
extern "C" cudaError_t hpvcd_launch_features(const DevPic*, uint32_t, uint32_t, unsigned long long*, float*, int,
                                             cudaStream_t);

static std::atomic<uint64_t> g_launches{0};
extern "C" void hpvcd_note_launches(uint32_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct Geo {
    int w, h, cw, ch, gw, gh, sub_w, sub_h, bps, ctb_cols, ctb_rows;
    size_t luma_bytes, chroma_bytes;
};

Geo geo_of(const hpvcd_picture& p) {
    Geo g;
    g.w = (int)p.width;
    g.h = (int)p.height;
    g.sub_w = p.chroma_idc == 1 || p.chroma_idc == 2 ? 2 : 1;  // SubWidthC
    g.sub_h = p.chroma_idc == 1 ? 2 : 1;                        // SubHeightC
    g.cw = p.chroma_idc ? (g.w + g.sub_w - 1) / g.sub_w : 0;
    g.ch = p.chroma_idc ? (g.h + g.sub_h - 1) / g.sub_h : 0;
    g.gw = (g.w + 3) / 4;
    g.gh = (g.h + 3) / 4;
    g.bps = p.bit_depth_y <= 8 && p.bit_depth_c <= 8 ? 1 : 2;
    const int ctb = 1 << p.log2_ctb;
    g.ctb_cols = (g.w + ctb - 1) / ctb;
    g.ctb_rows = (g.h + ctb - 1) / ctb;
    g.luma_bytes = (size_t)g.w * g.h * g.bps;
    g.chroma_bytes = (size_t)g.cw * g.ch * g.bps;
    return g;
}

hpvcd_status validate(const hpvcd_picture& p) {
    if (p.width == 0 || p.height == 0 || p.width > 16384 || p.height > 16384) return HPVCD_ERR_LIMIT;
    if ((p.width & 7) || (p.height & 7)) return HPVCD_ERR_BITSTREAM;
    if (p.chroma_idc > 3) return HPVCD_ERR_UNSUPPORTED;
    if (p.bit_depth_y < 8 || p.bit_depth_y > 12 || p.bit_depth_c < 8 || p.bit_depth_c > 12)
        return HPVCD_ERR_UNSUPPORTED;
    if ((p.bit_depth_y == 8) != (p.bit_depth_c == 8)) return HPVCD_ERR_UNSUPPORTED;
    if (p.log2_ctb < 4 || p.log2_ctb > 6) return HPVCD_ERR_BITSTREAM;
    if (p.n_tus && (!p.tus || !p.ctu_tu_start)) return HPVCD_ERR_INVALID_ARG;
    if (p.n_coeffs && !p.coeffs) return HPVCD_ERR_INVALID_ARG;
    if (p.n_pus && !p.pus) return HPVCD_ERR_INVALID_ARG;
    if (!p.ctu_tu_start) return HPVCD_ERR_INVALID_ARG;
    if ((p.flags & (HPVCD_PIC_DEBLOCK | HPVCD_PIC_CONSTRAINED_INTRA)) && !p.cells) return HPVCD_ERR_INVALID_ARG;
    if ((p.flags & HPVCD_PIC_PRED_IN_PLANE) && !p.pred[0]) return HPVCD_ERR_INVALID_ARG;
    return HPVCD_OK;
}

// Outputs written onto canvases (pictures placed by out->place).
// k_recon shared-memory layout class of a picture: 0 4:2:0 / 4:0:0, 1 4:4:4, 2 4:2:2.
int recon_class(const hpvcd_picture& p) { return p.chroma_idc == 3 ? 1 : (p.chroma_idc == 2 ? 2 : 0); }

bool canvas_kind(uint32_t kind) { return kind == HPVCD_OUT_RGB8 || kind == HPVCD_OUT_YUV_CANVAS; }

bool sao_active(const hpvcd_picture& p) {
    return p.sao && (p.flags & (HPVCD_PIC_SAO_LUMA | HPVCD_PIC_SAO_CHROMA));
}

struct Segment {
    uint32_t first_pic, n_pics;
    uint32_t wave_first, n_waves;  // the segment's wavefront launches (hpvcd_plan::waves)
    int max_dbk_v, max_dbk_h, max_sao;
    int max_rgb;  // RGB quads of the segment's largest picture
    int max_tiles = 0;  // 64 x 64 filter tiles of the segment's largest picture
    int tile_cfmt = 0;  // largest chroma layout class of its pictures (k_filter_tile shared memory)
};

// Deblocking, SAO and output requested together run as the fused tile kernel.
constexpr uint32_t kFilterStages = HPVCD_STAGE_DEBLOCK | HPVCD_STAGE_SAO | HPVCD_STAGE_OUTPUT;

// Independent pictures (no inter prediction) of a larger batch run as this
// many segments, each with its whole pipeline on its own stream, so that the
// streaming passes of one group overlap the latency-bound wavefront of another.
constexpr int kMaxGroups = 4;
constexpr uint32_t kMinPicturesPerGroup = 4;

// Streams and events of the concurrent groups.  A context slot creates one
// set and lends it to every plan it builds (no stream churn per batch
// layout); public plans own theirs.
struct GroupStreams {
    cudaStream_t aux[kMaxGroups] = {};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[kMaxGroups] = {};
    bool ready = false;
    cudaError_t create() {
        if (ready) return cudaSuccess;
        cudaError_t e = cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming);
        for (int g = 0; g < kMaxGroups && e == cudaSuccess; ++g) {
            e = cudaStreamCreateWithFlags(&aux[g], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_join[g], cudaEventDisableTiming);
        }
        ready = e == cudaSuccess;
        return e;
    }
    void destroy() {
        for (int g = 0; g < kMaxGroups; ++g) {
            if (ev_join[g]) cudaEventDestroy(ev_join[g]);
            if (aux[g]) cudaStreamDestroy(aux[g]);
            ev_join[g] = nullptr;
            aux[g] = nullptr;
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        ev_fork = nullptr;
        ready = false;
    }
};

}  // namespace

// Decoded-picture buffer kept in HBM across submits (dpb.rs:79-454 keeps
// reference pictures for later frames; here they never leave the device).
// Entry planes: Y, Cb, Cr at 256-byte aligned offsets, unpadded rows.
struct hpvcd_dpb {
    struct Entry {
        unsigned char* planes = nullptr;
        size_t bytes = 0;
        size_t luma_bytes = 0, chroma_bytes = 0;
        int w = 0, h = 0, idc = 0, bd = 0, bd_c = 0;
        bool valid = false;
        cudaEvent_t ev_write = nullptr;  // after the copy that stored the picture
        bool written = false;
        cudaEvent_t ev_read[HPVCD_DPB_MAX_READERS] = {};  // per context slot: the last batch reading it
        bool read[HPVCD_DPB_MAX_READERS] = {};
    };
    int device = 0;
    std::vector<Entry> entries;
    ~hpvcd_dpb() {
        for (Entry& e : entries) {
            if (e.ev_write) cudaEventSynchronize(e.ev_write);
            for (int k = 0; k < HPVCD_DPB_MAX_READERS; ++k)
                if (e.ev_read[k]) {
                    cudaEventSynchronize(e.ev_read[k]);
                    cudaEventDestroy(e.ev_read[k]);
                }
            if (e.ev_write) cudaEventDestroy(e.ev_write);
            cudaFree(e.planes);
        }
    }
};

struct hpvcd_plan {
    int device = 0;
    std::vector<hpvcd_picture> src;
    std::vector<DevPic> pics;
    DevPic* d_pics = nullptr;
    std::vector<CtuItem> items;
    CtuItem* d_items = nullptr;
    std::vector<Segment> segs;
    std::vector<uint32_t> rec_prefix;  // TB records of pictures [0, i)
    uint32_t* d_prefix = nullptr;
    unsigned char* d_res = nullptr;    // int16 residual planes
    uint32_t* d_scratch = nullptr;  // [seg counters][err][progress words...]
    size_t scratch_words = 0;
    unsigned char* d_planes = nullptr;
    size_t plane_bytes = 0;
    uint8_t* d_canvas = nullptr;
    size_t canvas_bytes = 0;
    unsigned long long* d_feat = nullptr;  // k_features sums (32) + the feature vector (16 floats)
    hpvcd_output out{};
    std::vector<hpvcd_tile_place> places;
    std::vector<hpvcd_canvas> canvases;   // resolved canvas list (>= 1 for RGB8)
    std::vector<uint64_t> canvas_offs;
    std::vector<size_t> canvas_sizes;  // bytes of each canvas
    bool any_rgb_canvas = false, any_native_canvas = false;  // which output kernels run
    hpvcd_sched sched{};
    bool recon_feat = false;  // k_recon with slices / tiles, constrained intra or cross-component tests
    // Wavefront launches: per segment, one per chroma-format class of its
    // pictures (k_recon shared-memory layout 0 4:2:0 / 4:0:0, 1 4:4:4, 2
    // 4:2:2), so the pictures of one class get the CTAs per SM of their own
    // layout.  item_off / n_full: the wave's range of the CTU work list;
    // n_items: entries launched (one fewer while a test drops a CTU).
    // ready: CTUs of the wave that can be walked at once (per picture, the
    // longest x + 2y diagonal of its CTB grid), which picks the build.
    struct Wave {
        uint32_t seg;
        int cfmt;
        uint32_t item_off, n_items, n_full;
        uint32_t ready;
    };
    std::vector<Wave> waves;
    // k_recon CTAs per SM by class and build (1 two warps, 2 three warps,
    // 3 three warps register-capped; index build - 1)
    int occ[3][3] = {{1, 1, 1}, {1, 1, 1}, {1, 1, 1}};
    // Build of a wave's wavefront kernel (hpvcd_sched.chroma_warps): 0 picks
    // three warps, register-capped when the wave has more CTUs ready at once
    // than the plain build's CTAs can hold (its share of them when segments
    // run concurrently).
    int build_of(const Wave& wv, int n_seg) const {
        const uint32_t cw = sched.chroma_warps;
        if (cw >= 1 && cw <= 3) return (int)cw;
        const int slots = concurrent ? sms * occ[wv.cfmt][1] / std::max(1, n_seg) : sms * occ[wv.cfmt][1];
        return wv.ready > (uint32_t)slots ? 3 : 2;
    }
    int occ_of(int cfmt, int build) const { return occ[cfmt][build - 1]; }
    int sms = 148;
    int max_rgb = 0;  // largest RGB job of one picture, in 4-pixel quads
    uint32_t launches_per_run = 0;
    // Plans owned by a context allocate from the stream-ordered pool of the
    // ticket's stream (no device-wide synchronisation when the layout of a
    // serving batch changes); public plans use plain cudaMalloc.
    cudaStream_t alloc_stream = nullptr;
    bool pooled = false;
    cudaGraphExec_t graphs[16] = {};  // captured launch sequences by stage mask
    // test hook of the bounded wavefront waits (hpvcd_plan_set_wait_test):
    // polls per wait (0 = default) and the work-list entry left out (-1 none)
    uint32_t spin_limit = 0;
    int32_t drop_item = -1;
    std::vector<int> dpb_refs;        // DPB entries the pictures predict from
    // concurrent segments (independent pictures): one stream per segment,
    // forked from and joined back into the launching stream
    bool concurrent = false;
    GroupStreams own;                  // used when the plan is not lent a set
    const GroupStreams* gs = nullptr;  // the set the launches use

    // whether SAO of a segment must respect slice / tile boundaries
    bool seg_sao_gated(const Segment& s) const {
        for (uint32_t i = s.first_pic; i < s.first_pic + s.n_pics; ++i)
            if (src[i].ctb_region && (src[i].flags & (HPVCD_PIC_SAO_NO_ACROSS_SLICES | HPVCD_PIC_SAO_NO_ACROSS_TILES)))
                return true;
        return false;
    }
    // whether a segment has cross-component pictures (k_ccp runs for it)
    bool seg_ccp(const Segment& s) const {
        for (uint32_t i = s.first_pic; i < s.first_pic + s.n_pics; ++i)
            if ((src[i].flags & HPVCD_PIC_CROSS_COMPONENT) && src[i].n_tus) return true;
        return false;
    }
    uint32_t launches_for(uint32_t stages) const {
        uint32_t L = 0;
        for (const auto& s : segs) {
            if (stages & HPVCD_STAGE_RECON) {
                for (uint32_t i = s.first_pic; i < s.first_pic + s.n_pics; ++i)
                    if ((src[i].flags & HPVCD_PIC_INTER) && src[i].n_pus) ++L;
                if (rec_prefix[s.first_pic + s.n_pics] > rec_prefix[s.first_pic]) L += 1 + seg_ccp(s);
                for (uint32_t w = s.wave_first; w < s.wave_first + s.n_waves; ++w) L += waves[w].n_items > 0;
            }
            if ((stages & kFilterStages) == kFilterStages) {
                L += s.max_tiles > 0;
                if (concurrent && canvas_kind(out.kind) && s.max_rgb > 0) L += (uint32_t)any_native_canvas;
                continue;
            }
            if (stages & HPVCD_STAGE_DEBLOCK) L += (s.max_dbk_v > 0) + (s.max_dbk_h > 0);
            if ((stages & HPVCD_STAGE_SAO) && s.max_sao > 0) ++L;
            if (concurrent && (stages & HPVCD_STAGE_OUTPUT) && canvas_kind(out.kind) && s.max_rgb > 0)
                L += (uint32_t)any_rgb_canvas + (uint32_t)any_native_canvas;
        }
        if (!concurrent && (stages & HPVCD_STAGE_OUTPUT) && canvas_kind(out.kind) && max_rgb > 0)
            L += (stages & kFilterStages) == kFilterStages
                     ? (uint32_t)any_native_canvas
                     : (uint32_t)any_rgb_canvas + (uint32_t)any_native_canvas;
        return L;
    }

    template <typename T>
    cudaError_t dmalloc(T** p, size_t bytes) {
        bytes = bytes ? bytes : 256;
        return pooled ? cudaMallocAsync((void**)p, bytes, alloc_stream) : cudaMalloc((void**)p, bytes);
    }
    void dfree(void* p) {
        if (!p) return;
        if (pooled)
            cudaFreeAsync(p, alloc_stream);
        else
            cudaFree(p);
    }
    ~hpvcd_plan() {
        for (cudaGraphExec_t& gx : graphs)
            if (gx) cudaGraphExecDestroy(gx);
        own.destroy();
        dfree(d_pics);
        dfree(d_items);
        dfree(d_scratch);
        dfree(d_prefix);
        dfree(d_res);
        dfree(d_planes);
        dfree(d_canvas);
        dfree(d_feat);
    }
};

namespace {

thread_local char t_last_error[256] = "";

hpvcd_status cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return HPVCD_OK;
    std::snprintf(t_last_error, sizeof(t_last_error), "%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return HPVCD_ERR_ALLOC;
    return HPVCD_ERR_CUDA;
}

}  // namespace

// Status mapping shared with the other translation units of the library.
extern "C" hpvcd_status hpvcd_internal_status(cudaError_t e) { return cuda_status(e); }

namespace {

// int16 residual planes of a picture, rows padded to 16 samples.
inline int res_stride_of(int w) { return (w + 15) & ~15; }
size_t res_plane_bytes(const Geo& g) {
    return align_up((size_t)res_stride_of(g.w) * g.h * 2, 256) +
           2 * align_up((size_t)res_stride_of(g.cw) * g.ch * 2, 256);
}

uint32_t n_canvases_of(const hpvcd_output* out) { return out->n_canvases ? out->n_canvases : 1; }

hpvcd_canvas canvas_of(const hpvcd_output* out, uint32_t k) {
    return out->n_canvases ? out->canvases[k]
                           : hpvcd_canvas{out->canvas_w, out->canvas_h, out->matrix, out->full_range, out->orientation};
}

// Sample format of a YUV canvas: that of the first picture placed on it
// (8-bit 4:0:0 when none is).
struct CanvasFmt {
    int idc, bps;
};
CanvasFmt canvas_fmt(const hpvcd_picture* pics, uint32_t n, const hpvcd_tile_place* place, uint32_t k) {
    for (uint32_t i = 0; i < n; ++i)
        if (place[i].canvas == k) return CanvasFmt{pics[i].chroma_idc, geo_of(pics[i]).bps};
    return CanvasFmt{0, 1};
}

// Canvas receiving native YCbCr planes (every canvas of a YUV canvas output,
// HPVCD_CANVAS_NATIVE ones of an RGB8 output).
bool native_canvas(uint32_t kind, const hpvcd_canvas& cv) {
    return kind == HPVCD_OUT_YUV_CANVAS || cv.matrix == HPVCD_CANVAS_NATIVE;
}

size_t canvas_bytes_of(uint32_t kind, const hpvcd_canvas& cv, CanvasFmt f) {
    const size_t w = cv.width, h = cv.height;
    if (!native_canvas(kind, cv)) return w * h * 3;
    const size_t sw = f.idc == 1 || f.idc == 2 ? 2 : 1, sh = f.idc == 1 ? 2 : 1;
    const size_t cw = f.idc ? (w + sw - 1) / sw : 0, ch = f.idc ? (h + sh - 1) / sh : 0;
    return (w * h + 2 * cw * ch) * (size_t)f.bps;
}

// Bytes of the output of a batch: all canvases, or all YUV planes.
size_t output_bytes(const hpvcd_picture* pics, uint32_t n, const hpvcd_output* out) {
    size_t b = 0;
    if (out && canvas_kind(out->kind)) {
        for (uint32_t k = 0; k < n_canvases_of(out); ++k)
            b += canvas_bytes_of(out->kind, canvas_of(out, k), canvas_fmt(pics, n, out->place, k));
        return b;
    }
    for (uint32_t i = 0; i < n; ++i) {
        const Geo geo = geo_of(pics[i]);
        b += geo.luma_bytes + 2 * geo.chroma_bytes;
    }
    return b;
}

// Device bytes a plan for these pictures needs (planes, scratch, canvas).
size_t plan_footprint(const hpvcd_picture* pics, uint32_t n, const hpvcd_output* out) {
    size_t bytes = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const Geo g = geo_of(pics[i]);
        const size_t one = align_up(g.luma_bytes, 256) + 2 * align_up(g.chroma_bytes, 256);
        bytes += one * (sao_active(pics[i]) ? 2 : 1);
        bytes += res_plane_bytes(g);
        bytes += (size_t)g.ctb_cols * g.ctb_rows * (4 + sizeof(CtuItem));
    }
    bytes += n * sizeof(DevPic);
    bytes += output_bytes(pics, n, out);
    return bytes;
}

// Rebuild the input-pointer fields of the device table from descriptors.
void fill_inputs(DevPic& d, const hpvcd_picture& p) {
    d.tus = p.tus;
    d.ctu_start = p.ctu_tu_start;
    d.coeffs = p.coeffs;
    d.cells = p.cells;
    d.sao = p.sao;
    d.pus = p.pus;
    d.scaling = p.scaling;
    d.ctb_region = p.ctb_region;
    d.slice_deblock = p.slice_deblock;
    d.n_tus = p.n_tus;
    d.n_pus = p.n_pus;
    d.n_coeffs = p.n_coeffs;
}

hpvcd_status plan_build(const hpvcd_picture* pics, uint32_t n, const hpvcd_output* out,
                        const hpvcd_sched* sched, const hpvcd_wp_table* host_wp, hpvcd_plan** result,
                        cudaStream_t pool_stream = nullptr, bool pooled = false,
                        GroupStreams* lend = nullptr, const hpvcd_dpb* dpb = nullptr) {
    if (!pics || n == 0 || !result) return HPVCD_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; ++i) {
        const hpvcd_status s = validate(pics[i]);
        if (s != HPVCD_OK) return s;
    }
    // Motion compensation reads a reference with the current picture's
    // geometry, so every reference of a picture with PUs has its size and
    // sample format (as in any conforming stream).
    for (uint32_t i = 0; i < n; ++i) {
        const hpvcd_picture& p = pics[i];
        if (!(p.flags & HPVCD_PIC_INTER) || !p.n_pus) continue;
        for (int l = 0; l < 2; ++l)
            for (int r = 0; r < HPVCD_MAX_REFS; ++r) {
                const int sv = p.ref_slot[l][r];
                if (sv < 0 || (uint32_t)sv >= i) continue;
                const hpvcd_picture& q = pics[sv];
                if (q.width != p.width || q.height != p.height || q.chroma_idc != p.chroma_idc ||
                    q.bit_depth_y != p.bit_depth_y || q.bit_depth_c != p.bit_depth_c) {
                    std::snprintf(t_last_error, sizeof(t_last_error),
                                  "picture %u references picture %d of another size or format", i, sv);
                    return HPVCD_ERR_BITSTREAM;
                }
            }
    }
    if (out && canvas_kind(out->kind) &&
        (!out->place || (out->n_canvases ? !out->canvases : (out->canvas_w == 0 || out->canvas_h == 0))))
        return HPVCD_ERR_INVALID_ARG;
    if (out && out->kind > HPVCD_OUT_YUV_CANVAS) return HPVCD_ERR_INVALID_ARG;
    if (out && canvas_kind(out->kind))  // every picture of a native canvas in its format
        for (uint32_t i = 0; i < n; ++i) {
            if (out->place[i].canvas >= n_canvases_of(out)) return HPVCD_ERR_INVALID_ARG;
            if (!native_canvas(out->kind, canvas_of(out, out->place[i].canvas))) continue;
            const CanvasFmt f = canvas_fmt(pics, n, out->place, out->place[i].canvas);
            if (f.idc != pics[i].chroma_idc || f.bps != geo_of(pics[i]).bps) {
                std::snprintf(t_last_error, sizeof(t_last_error),
                              "picture %u differs in chroma format or sample size from its YUV canvas", i);
                return HPVCD_ERR_INVALID_ARG;
            }
        }
    hpvcd_plan* P = new (std::nothrow) hpvcd_plan();
    if (!P) return HPVCD_ERR_ALLOC;
    P->alloc_stream = pool_stream;
    P->pooled = pooled;
    cudaGetDevice(&P->device);
    P->src.assign(pics, pics + n);
    if (out) {
        P->out = *out;
        if (canvas_kind(out->kind)) {
            P->places.assign(out->place, out->place + n);
            P->out.place = nullptr;
            for (uint32_t k = 0; k < n_canvases_of(out); ++k) P->canvases.push_back(canvas_of(out, k));
            P->out.canvases = nullptr;
            uint64_t off = 0;
            for (uint32_t k = 0; k < P->canvases.size(); ++k) {
                P->canvas_offs.push_back(off);
                P->canvas_sizes.push_back(
                    canvas_bytes_of(out->kind, P->canvases[k], canvas_fmt(pics, n, out->place, k)));
                off += P->canvas_sizes.back();
            }
            for (uint32_t i = 0; i < n; ++i)
                if (P->places[i].canvas >= P->canvases.size()) {
                    delete P;
                    return HPVCD_ERR_INVALID_ARG;
                }
        }
    } else {
        P->out.kind = HPVCD_OUT_YUV;
    }
    if (sched) {
        if (sched->idct > 2 || sched->chroma_warps > 3) {
            delete P;
            return HPVCD_ERR_INVALID_ARG;
        }
        P->sched = *sched;
    }
    bool any_inter = false;
    for (uint32_t i = 0; i < n; ++i) {
        if (pics[i].ctb_region ||
            (pics[i].flags & (HPVCD_PIC_CONSTRAINED_INTRA | HPVCD_PIC_CROSS_COMPONENT | HPVCD_PIC_PCM)))
            P->recon_feat = true;
        if (pics[i].flags & HPVCD_PIC_INTER) any_inter = true;
    }
    // ---- which pictures keep their final planes: all, unless the output is
    // RGB8 canvases only; then those that a later picture predicts from,
    // that a DPB stores, or whose canvas is a native one ----
    std::vector<char> keep_fin(n, 1);
    if (out && out->kind == HPVCD_OUT_RGB8 && (out->options & HPVCD_OUTPUT_CANVAS_ONLY)) {
        for (uint32_t i = 0; i < n; ++i)
            keep_fin[i] = (pics[i].flags & HPVCD_PIC_STORE_MASK) != 0 ||
                          native_canvas(out->kind, canvas_of(out, out->place[i].canvas));
        for (uint32_t i = 0; i < n; ++i)
            for (int l = 0; l < 2; ++l)
                for (int r = 0; r < HPVCD_MAX_REFS; ++r) {
                    const int sv = pics[i].ref_slot[l][r];
                    if (sv >= 0 && (uint32_t)sv < n) keep_fin[(size_t)sv] = 1;
                }
    }
    // ---- planes + scratch layout ----
    size_t plane_bytes = 0;
    std::vector<size_t> rec_off(n), fin_off(n);
    size_t ready_words = 0;
    std::vector<size_t> ready_off(n);
    for (uint32_t i = 0; i < n; ++i) {
        const Geo g = geo_of(pics[i]);
        const size_t one = align_up(g.luma_bytes, 256) + 2 * align_up(g.chroma_bytes, 256);
        rec_off[i] = plane_bytes;
        plane_bytes += one;
        // the final planes are separate when SAO runs (it reads the deblocked
        // planes) or when they are kept (the tile filter kernel never writes
        // the planes it reads)
        if (sao_active(pics[i]) || keep_fin[i]) {
            fin_off[i] = plane_bytes;
            plane_bytes += one;
        } else {
            fin_off[i] = rec_off[i];
        }
        ready_off[i] = ready_words;
        ready_words += (size_t)4 * g.ctb_cols * g.ctb_rows;  // one progress word per component
    }
    // segments: all pictures at once, or one per picture when any picture
    // predicts from another (its references must be final first).
    if (any_inter) {
        for (uint32_t i = 0; i < n; ++i) P->segs.push_back(Segment{i, 1, 0, 0, 0, 0, 0, 0});
    } else {
        // independent pictures: up to kMaxGroups contiguous groups of about
        // equal luma area, run concurrently
        const int groups = (int)std::min<uint32_t>((uint32_t)kMaxGroups, n / kMinPicturesPerGroup);
        if (groups <= 1) {
            P->segs.push_back(Segment{0, n, 0, 0, 0, 0, 0, 0});
        } else {
            double total = 0;
            for (uint32_t i = 0; i < n; ++i) total += (double)pics[i].width * pics[i].height;
            double acc = 0;
            uint32_t first = 0;
            for (uint32_t i = 0; i < n; ++i) {
                acc += (double)pics[i].width * pics[i].height;
                const int done = (int)P->segs.size();
                const bool last = i + 1 == n;
                if (last || (done < groups - 1 && acc >= total * (done + 1) / groups)) {
                    P->segs.push_back(Segment{first, i + 1 - first, 0, 0, 0, 0, 0, 0});
                    first = i + 1;
                }
            }
            P->concurrent = P->segs.size() > 1;
        }
    }
    // ---- wavefront schedule per segment and format class: CTUs sorted by
    // (x + 2y, picture, y) ----
    for (uint32_t si = 0; si < P->segs.size(); ++si) {
        Segment& s = P->segs[si];
        s.wave_first = (uint32_t)P->waves.size();
        int max_t = 0;
        for (uint32_t i = s.first_pic; i < s.first_pic + s.n_pics; ++i) {
            const Geo g = geo_of(pics[i]);
            max_t = std::max(max_t, g.ctb_cols + 2 * g.ctb_rows);
        }
        for (int cls = 0; cls < 3; ++cls) {
            const uint32_t off = (uint32_t)P->items.size();
            uint32_t ready = 0;
            for (uint32_t i = s.first_pic; i < s.first_pic + s.n_pics; ++i) {
                const hpvcd_picture& p = pics[i];
                if ((p.flags & HPVCD_PIC_PRED_IN_PLANE) || recon_class(p) != cls) continue;
                const Geo g = geo_of(p);
                ready += (uint32_t)std::min(g.ctb_rows, (g.ctb_cols + 1) / 2);
            }
            for (int t = 0; t <= max_t; ++t)
                for (uint32_t i = s.first_pic; i < s.first_pic + s.n_pics; ++i) {
                    const hpvcd_picture& p = pics[i];
                    if (p.flags & HPVCD_PIC_PRED_IN_PLANE) continue;  // k_residual did it all
                    if (recon_class(p) != cls) continue;
                    const Geo g = geo_of(p);
                    for (int y = 0; y < g.ctb_rows; ++y) {
                        const int x = t - 2 * y;
                        if (x >= 0 && x < g.ctb_cols) P->items.push_back(CtuItem{i, (uint16_t)x, (uint16_t)y});
                    }
                }
            const uint32_t cnt = (uint32_t)P->items.size() - off;
            if (cnt) P->waves.push_back(hpvcd_plan::Wave{si, cls, off, cnt, cnt, ready});
        }
        s.n_waves = (uint32_t)P->waves.size() - s.wave_first;
    }
    const size_t n_waves = P->waves.size();
    P->scratch_words = n_waves + 1 + ready_words;
    size_t res_bytes = 0;
    std::vector<size_t> res_off(n);
    for (uint32_t i = 0; i < n; ++i) {
        res_off[i] = res_bytes;
        res_bytes += res_plane_bytes(geo_of(pics[i]));
    }
    P->rec_prefix.assign(n + 1, 0);
    for (uint32_t i = 0; i < n; ++i) P->rec_prefix[i + 1] = P->rec_prefix[i] + pics[i].n_tus;
    cudaError_t e = P->dmalloc(&P->d_planes, plane_bytes);
    if (e == cudaSuccess) e = P->dmalloc(&P->d_res, res_bytes);
    if (e == cudaSuccess) e = P->dmalloc(&P->d_prefix, sizeof(uint32_t) * (n + 1));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->d_prefix, P->rec_prefix.data(), sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice,
                            pool_stream);
    if (e == cudaSuccess) e = P->dmalloc(&P->d_scratch, P->scratch_words * sizeof(uint32_t));
    if (e == cudaSuccess) e = P->dmalloc(&P->d_feat, 32 * sizeof(unsigned long long) + 16 * sizeof(float));
    if (e == cudaSuccess && canvas_kind(P->out.kind)) {
        P->canvas_bytes = 0;
        for (const size_t b : P->canvas_sizes) P->canvas_bytes += b;
        e = P->dmalloc(&P->d_canvas, P->canvas_bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(P->d_canvas, 0, P->canvas_bytes, pool_stream);
    }
    if (e != cudaSuccess) {
        delete P;
        cudaGetLastError();
        return cuda_status(e);
    }
    P->plane_bytes = plane_bytes;
    // ---- device picture table ----
    P->pics.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        const hpvcd_picture& p = pics[i];
        const Geo g = geo_of(p);
        DevPic& d = P->pics[i];
        std::memset(&d, 0, sizeof(d));
        d.w = g.w; d.h = g.h; d.cw = g.cw; d.ch = g.ch; d.gw = g.gw; d.gh = g.gh;
        d.idc = p.chroma_idc; d.sub_w = g.sub_w; d.sub_h = g.sub_h;
        d.bd = p.bit_depth_y; d.bd_c = p.bit_depth_c; d.bps = g.bps;
        d.log2_ctb = p.log2_ctb; d.ctb_cols = g.ctb_cols; d.ctb_rows = g.ctb_rows;
        d.flags = p.flags;
        d.beta_offset_div2 = p.beta_offset_div2;
        d.tc_offset_div2 = p.tc_offset_div2;
        d.pps_cb_qp_offset = p.pps_cb_qp_offset;
        d.pps_cr_qp_offset = p.pps_cr_qp_offset;
        fill_inputs(d, p);
        if (host_wp && p.wp) {
            d.wp = host_wp[i];
            d.has_wp = 1;
        }
        for (int l = 0; l < 2; ++l)
            for (int r = 0; r < HPVCD_MAX_REFS; ++r) {
                const int s = p.ref_slot[l][r];
                d.ref_pic[l][r] = (s >= 0 && (uint32_t)s < i) ? s : -1;
            }
        unsigned char* base = P->d_planes + rec_off[i];
        d.rec[0] = base;
        d.rec[1] = base + align_up(g.luma_bytes, 256);
        d.rec[2] = base + align_up(g.luma_bytes, 256) + align_up(g.chroma_bytes, 256);
        unsigned char* fb = P->d_planes + fin_off[i];
        d.fin[0] = fb;
        d.fin[1] = fb + align_up(g.luma_bytes, 256);
        d.fin[2] = fb + align_up(g.luma_bytes, 256) + align_up(g.chroma_bytes, 256);
        if (!p.chroma_idc) d.rec[1] = d.rec[2] = d.fin[1] = d.fin[2] = nullptr;
        d.ready = P->d_scratch + n_waves + 1 + ready_off[i];
        {
            unsigned char* rb = P->d_res + res_off[i];
            d.res_stride[0] = res_stride_of(g.w);
            d.res_stride[1] = d.res_stride[2] = res_stride_of(g.cw);
            const size_t ly = align_up((size_t)d.res_stride[0] * g.h * 2, 256);
            const size_t lc = align_up((size_t)d.res_stride[1] * g.ch * 2, 256);
            d.res[0] = (int16_t*)rb;
            d.res[1] = p.chroma_idc ? (int16_t*)(rb + ly) : nullptr;
            d.res[2] = p.chroma_idc ? (int16_t*)(rb + ly + lc) : nullptr;
        }
        d.needs_wavefront = (p.flags & HPVCD_PIC_PRED_IN_PLANE) ? 0 : 1;
        d.write_fin = keep_fin[i];
        if (canvas_kind(P->out.kind)) {
            const hpvcd_tile_place& tp = P->places[i];
            const hpvcd_canvas& cv = P->canvases[tp.canvas];
            d.canvas_off = P->canvas_offs[tp.canvas];
            d.canvas_w = (int)cv.width; d.canvas_h = (int)cv.height;
            const bool rgb = !native_canvas(P->out.kind, cv);
            d.matrix = rgb ? (int)cv.matrix : (int)HPVCD_CANVAS_NATIVE;  // selects k_rgb or k_yuv_canvas
            d.full_range = (int)cv.full_range;
            d.orientation = (int)cv.orientation;
            (rgb ? P->any_rgb_canvas : P->any_native_canvas) = true;
            d.dst_x = (int)tp.dst_x; d.dst_y = (int)tp.dst_y;
            // RGB8 crops at the picture; a native canvas repeats its last row / column
            d.crop_w = (int)(rgb ? std::min<uint32_t>(tp.crop_w, p.width) : std::min<uint32_t>(tp.crop_w, 65536));
            d.crop_h = (int)(rgb ? std::min<uint32_t>(tp.crop_h, p.height) : std::min<uint32_t>(tp.crop_h, 65536));
            P->max_rgb = std::max(P->max_rgb, (d.crop_w + 3) / 4 * d.crop_h);  // 4-pixel quads
        }
    }
    // ---- DPB references: every entry a picture predicts from becomes one
    // more device-table picture, read by motion compensation, never decoded ----
    {
        std::vector<int> ext_of(dpb ? dpb->entries.size() : 0, -1);
        for (uint32_t i = 0; i < n; ++i)
            for (int l = 0; l < 2; ++l)
                for (int r = 0; r < HPVCD_MAX_REFS; ++r) {
                    const int sv = pics[i].ref_slot[l][r];
                    if (sv > HPVCD_REF_DPB(0)) continue;
                    const int en = -2 - sv;
                    const hpvcd_dpb::Entry* E =
                        dpb && en < (int)dpb->entries.size() ? &dpb->entries[(size_t)en] : nullptr;
                    if (!E || !E->valid || E->w != (int)pics[i].width || E->h != (int)pics[i].height ||
                        E->idc != pics[i].chroma_idc || E->bd != pics[i].bit_depth_y ||
                        E->bd_c != pics[i].bit_depth_c) {
                        std::snprintf(t_last_error, sizeof(t_last_error),
                                      "picture %u references DPB entry %d, which is empty or of another format", i,
                                      en);
                        delete P;
                        return HPVCD_ERR_INVALID_ARG;
                    }
                    if (ext_of[(size_t)en] < 0) {
                        ext_of[(size_t)en] = (int)P->pics.size();
                        P->dpb_refs.push_back(en);
                        hpvcd_picture q{};
                        q.width = (uint32_t)E->w;
                        q.height = (uint32_t)E->h;
                        q.chroma_idc = (uint8_t)E->idc;
                        q.bit_depth_y = (uint8_t)E->bd;
                        q.bit_depth_c = (uint8_t)E->bd_c;
                        q.log2_ctb = 6;
                        const Geo gq = geo_of(q);
                        DevPic d{};
                        d.w = gq.w; d.h = gq.h; d.cw = gq.cw; d.ch = gq.ch; d.gw = gq.gw; d.gh = gq.gh;
                        d.idc = E->idc; d.sub_w = gq.sub_w; d.sub_h = gq.sub_h;
                        d.bd = E->bd; d.bd_c = E->bd_c; d.bps = gq.bps;
                        d.log2_ctb = 6; d.ctb_cols = gq.ctb_cols; d.ctb_rows = gq.ctb_rows;
                        for (int ll = 0; ll < 2; ++ll)
                            for (int rr = 0; rr < HPVCD_MAX_REFS; ++rr) d.ref_pic[ll][rr] = -1;
                        d.rec[0] = d.fin[0] = E->planes;
                        if (E->idc) {
                            d.rec[1] = d.fin[1] = E->planes + align_up(E->luma_bytes, 256);
                            d.rec[2] = d.fin[2] = E->planes + align_up(E->luma_bytes, 256) +
                                                  align_up(E->chroma_bytes, 256);
                        }
                        d.needs_wavefront = 0;
                        P->pics.push_back(d);
                    }
                    P->pics[i].ref_pic[l][r] = ext_of[(size_t)en];
                }
    }
    // ---- filter and output job sizes per segment ----
    for (Segment& s : P->segs) {
        for (uint32_t i = s.first_pic; i < s.first_pic + s.n_pics; ++i) {
            const DevPic& d = P->pics[i];
            const int lv = (d.w >= 12 ? (d.w - 4) / 8 : 0) * (d.h / 4);
            const int lh = (d.h >= 12 ? (d.h - 4) / 8 : 0) * (d.w / 4);
            const int cv = d.idc ? (d.cw >= 10 ? (d.cw - 2) / 8 : 0) * (d.ch / 4) : 0;
            const int ch = d.idc ? (d.ch >= 10 ? (d.ch - 2) / 8 : 0) * (d.cw / 4) : 0;
            s.max_dbk_v = std::max(s.max_dbk_v, std::max(lv, cv));
            s.max_dbk_h = std::max(s.max_dbk_h, std::max(lh, ch));
            if (d.rec[0] != d.fin[0]) s.max_sao = std::max(s.max_sao, d.w * d.h);
            s.max_tiles = std::max(s.max_tiles, ((d.w + 63) / 64) * ((d.h + 63) / 64));
            // the 4:4:4 layout holds every format, the 4:2:2 one also 4:2:0
            const int tcls = d.idc == 3 ? 1 : (d.idc == 2 ? 2 : 0);
            if (tcls == 1 || (tcls == 2 && s.tile_cfmt == 0)) s.tile_cfmt = tcls;
            if (canvas_kind(P->out.kind)) s.max_rgb = std::max(s.max_rgb, (d.crop_w + 3) / 4 * d.crop_h);
        }
    }
    e = P->dmalloc(&P->d_pics, sizeof(DevPic) * P->pics.size());
    if (e == cudaSuccess) e = P->dmalloc(&P->d_items, sizeof(CtuItem) * std::max<size_t>(P->items.size(), 1));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->d_pics, P->pics.data(), sizeof(DevPic) * P->pics.size(), cudaMemcpyHostToDevice,
                            pool_stream);
    if (e == cudaSuccess && !P->items.empty())
        e = cudaMemcpyAsync(P->d_items, P->items.data(), sizeof(CtuItem) * P->items.size(), cudaMemcpyHostToDevice,
                            pool_stream);
    // host vectors are pageable: the copies above are staged before returning,
    // but make the plan's first use ordered after them for plain plans too
    if (e == cudaSuccess && !pooled) e = cudaStreamSynchronize(pool_stream);
    if (e != cudaSuccess) {
        delete P;
        cudaGetLastError();
        return cuda_status(e);
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, P->device);
    P->sms = sms;
    for (int cls = 0; cls < 3; ++cls)
        for (int cw = 1; cw <= 3; ++cw) P->occ[cls][cw - 1] = std::max(1, hpvcd_recon_occupancy(cls, cw));
    {
        const cudaError_t fe = hpvcd_filter_tile_setup();
        if (fe != cudaSuccess) {
            delete P;
            return cuda_status(fe);
        }
    }
    if (P->concurrent) {
        GroupStreams* set = lend ? lend : &P->own;
        const cudaError_t ce = set->create();
        if (ce != cudaSuccess) {
            delete P;
            cudaGetLastError();
            return cuda_status(ce);
        }
        P->gs = set;
    }
    P->launches_per_run = P->launches_for(HPVCD_STAGE_ALL);
    *result = P;
    return HPVCD_OK;
}

hpvcd_status plan_launch(hpvcd_plan* P, uint32_t stages, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    // Work counters, the device error word and the wavefront progress words are
    // reset by every launch that reconstructs.
    if (stages & HPVCD_STAGE_RECON) {
        e = cudaMemsetAsync(P->d_scratch, 0, P->scratch_words * sizeof(uint32_t), st);
        if (e != cudaSuccess) return cuda_status(e);
    }
    const uint32_t n_seg = (uint32_t)P->segs.size();
    uint32_t* d_err = P->d_scratch + P->waves.size();
    const bool fused = (stages & kFilterStages) == kFilterStages;
    if (stages & HPVCD_STAGE_RECON) {
        for (size_t i = 0; i < P->src.size(); ++i) {
            const hpvcd_picture& p = P->src[i];
            if (!(p.flags & HPVCD_PIC_PRED_IN_PLANE)) continue;
            const Geo g = geo_of(p);
            const DevPic& d = P->pics[i];
            for (int c = 0; c < (p.chroma_idc ? 3 : 1); ++c) {
                if (!p.pred[c]) continue;
                e = cudaMemcpyAsync(d.rec[c], p.pred[c], c ? g.chroma_bytes : g.luma_bytes,
                                    cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) return cuda_status(e);
            }
        }
    }
    const cudaStream_t origin = st;
    if (P->concurrent) {  // fork: every segment's stream starts after the work above
        e = cudaEventRecord(P->gs->ev_fork, origin);
        for (uint32_t si = 0; si < n_seg && e == cudaSuccess; ++si)
            e = cudaStreamWaitEvent(P->gs->aux[si], P->gs->ev_fork, 0);
        if (e != cudaSuccess) return cuda_status(e);
    }
    for (uint32_t si = 0; si < n_seg; ++si) {
        const Segment& s = P->segs[si];
        const DevPic* dp = P->d_pics + s.first_pic;
        if (P->concurrent) st = P->gs->aux[si];
        if (stages & HPVCD_STAGE_RECON) {
            for (uint32_t i = s.first_pic; i < s.first_pic + s.n_pics; ++i)
                if ((P->src[i].flags & HPVCD_PIC_INTER) && P->src[i].n_pus) {
                    e = hpvcd_launch_mc(P->d_pics, (int)i, (int)P->src[i].n_pus, P->src[i].chroma_idc ? 3 : 1, st);
                    if (e != cudaSuccess) return cuda_status(e);
                }
            const uint32_t nrec = P->rec_prefix[s.first_pic + s.n_pics] - P->rec_prefix[s.first_pic];
            e = hpvcd_launch_residual(P->d_pics + s.first_pic, P->d_prefix + s.first_pic, s.n_pics, nrec, d_err,
                                      P->sms, (int)P->sched.idct, st);
            if (e == cudaSuccess && nrec && P->seg_ccp(s))
                e = hpvcd_launch_ccp(P->d_pics + s.first_pic, P->d_prefix + s.first_pic, s.n_pics, nrec, d_err,
                                     P->sms, st);
            if (e != cudaSuccess) return cuda_status(e);
            // the segment's format classes one after another, each wave with
            // its own layout and work counter
            for (uint32_t w = s.wave_first; w < s.wave_first + s.n_waves; ++w) {
                const hpvcd_plan::Wave& wv = P->waves[w];
                const int build = P->build_of(wv, (int)n_seg);
                int occ = P->occ_of(wv.cfmt, build);
                if (P->sched.recon_ctas_per_sm > 0) occ = std::min<int>(occ, (int)P->sched.recon_ctas_per_sm);
                // concurrent segments share the SMs: each gets its share of the CTAs
                const int share = P->concurrent ? std::max(1, P->sms * occ / (int)n_seg) : P->sms * occ;
                const int grid = std::max(1, std::min<int>(share, (int)wv.n_items));
                e = hpvcd_launch_recon(P->d_pics, P->d_items + wv.item_off, wv.n_items, P->d_scratch + w, d_err,
                                       wv.cfmt, grid, build, P->recon_feat ? 1 : 0,
                                       P->sched.wave ? 0 : 1, P->spin_limit, st);
                if (e != cudaSuccess) return cuda_status(e);
            }
        }
        if (fused) {  // deblocking, SAO and RGB8 in one pass over 64 x 64 tiles
            e = hpvcd_launch_filter_tile(dp, (int)s.n_pics, s.max_tiles, s.tile_cfmt, P->seg_sao_gated(s) ? 1 : 0,
                                         canvas_kind(P->out.kind) && P->any_rgb_canvas ? P->d_canvas : nullptr, st);
            if (e != cudaSuccess) return cuda_status(e);
        } else {
            if (stages & HPVCD_STAGE_DEBLOCK) {
                e = hpvcd_launch_deblock(dp, (int)s.n_pics, s.max_dbk_v, 1, st);
                if (e == cudaSuccess) e = hpvcd_launch_deblock(dp, (int)s.n_pics, s.max_dbk_h, 0, st);
                if (e != cudaSuccess) return cuda_status(e);
            }
            if (stages & HPVCD_STAGE_SAO) {
                e = hpvcd_launch_sao(dp, (int)s.n_pics, s.max_sao, P->seg_sao_gated(s) ? 1 : 0, st);
                if (e != cudaSuccess) return cuda_status(e);
            }
        }
        if (P->concurrent) {
            if ((stages & HPVCD_STAGE_OUTPUT) && canvas_kind(P->out.kind)) {
                if (P->any_rgb_canvas && !fused) e = hpvcd_launch_rgb(dp, (int)s.n_pics, s.max_rgb, P->d_canvas, st);
                if (e == cudaSuccess && P->any_native_canvas)
                    e = hpvcd_launch_yuv_canvas(dp, (int)s.n_pics, s.max_rgb, P->d_canvas, st);
                if (e != cudaSuccess) return cuda_status(e);
            }
            e = cudaEventRecord(P->gs->ev_join[si], st);  // join back into the launching stream
            if (e == cudaSuccess) e = cudaStreamWaitEvent(origin, P->gs->ev_join[si], 0);
            if (e != cudaSuccess) return cuda_status(e);
        }
    }
    st = origin;
    if (!P->concurrent && (stages & HPVCD_STAGE_OUTPUT) && canvas_kind(P->out.kind)) {
        if (P->any_rgb_canvas && !fused)
            e = hpvcd_launch_rgb(P->d_pics, (int)P->src.size(), P->max_rgb, P->d_canvas, st);
        if (e == cudaSuccess && P->any_native_canvas)
            e = hpvcd_launch_yuv_canvas(P->d_pics, (int)P->src.size(), P->max_rgb, P->d_canvas, st);
        if (e != cudaSuccess) return cuda_status(e);
    }
    return HPVCD_OK;
}

// Re-point the input fields of an existing plan at new device buffers of a
// batch with identical geometry (same layout key).
hpvcd_status plan_rebind(hpvcd_plan* P, const hpvcd_picture* pics, const hpvcd_wp_table* host_wp,
                         cudaStream_t st) {
    for (size_t i = 0; i < P->src.size(); ++i) {
        P->src[i] = pics[i];
        P->rec_prefix[i + 1] = P->rec_prefix[i] + pics[i].n_tus;
        fill_inputs(P->pics[i], pics[i]);
        if (host_wp && pics[i].wp) {
            P->pics[i].wp = host_wp[i];
            P->pics[i].has_wp = 1;
        } else {
            P->pics[i].has_wp = 0;
        }
    }
    cudaError_t e = cudaMemcpyAsync(P->d_prefix, P->rec_prefix.data(), sizeof(uint32_t) * P->rec_prefix.size(),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->d_pics, P->pics.data(), sizeof(DevPic) * P->pics.size(), cudaMemcpyHostToDevice, st);
    return cuda_status(e);
}

bool same_layout(const hpvcd_plan* P, const hpvcd_picture* pics, uint32_t n, const hpvcd_output* out) {
    if (P->src.size() != n || !P->dpb_refs.empty()) return false;  // DPB entries may have moved
    for (uint32_t i = 0; i < n; ++i) {
        const hpvcd_picture& a = P->src[i];
        const hpvcd_picture& b = pics[i];
        if (a.width != b.width || a.height != b.height || a.chroma_idc != b.chroma_idc ||
            a.bit_depth_y != b.bit_depth_y || a.bit_depth_c != b.bit_depth_c || a.log2_ctb != b.log2_ctb ||
            a.flags != b.flags || a.beta_offset_div2 != b.beta_offset_div2 ||
            a.tc_offset_div2 != b.tc_offset_div2 || a.pps_cb_qp_offset != b.pps_cb_qp_offset ||
            a.pps_cr_qp_offset != b.pps_cr_qp_offset || (a.sao != nullptr) != (b.sao != nullptr) ||
            (a.n_pus != 0) != (b.n_pus != 0) ||
            std::memcmp(a.ref_slot, b.ref_slot, sizeof(a.ref_slot)) != 0)
            return false;
    }
    const uint32_t kind = out ? out->kind : HPVCD_OUT_YUV;
    if (kind != P->out.kind) return false;
    if ((out ? out->options : 0u) != P->out.options) return false;
    if (canvas_kind(kind)) {
        const uint32_t nc = out->n_canvases ? out->n_canvases : 1;
        if (nc != P->canvases.size()) return false;
        for (uint32_t k = 0; k < nc; ++k) {
            const hpvcd_canvas c = canvas_of(out, k);
            if (std::memcmp(&c, &P->canvases[k], sizeof(c)) != 0) return false;
        }
        for (uint32_t i = 0; i < n; ++i)
            if (std::memcmp(&out->place[i], &P->places[i], sizeof(hpvcd_tile_place)) != 0) return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Contexts (host-buffer API)
// ---------------------------------------------------------------------------
struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    unsigned char* h_in = nullptr;  // pinned staging of the inputs
    size_t h_in_cap = 0;
    unsigned char* d_in = nullptr;  // device input arena
    size_t d_in_cap = 0;
    unsigned char* h_out = nullptr;  // pinned output
    size_t h_out_cap = 0;
    hpvcd_plan* plan = nullptr;
    uint64_t ticket = 0;  // 0 = free
    uint64_t out_bytes = 0;
    uint64_t plan_bytes = 0;  // device bytes of `plan`
    uint64_t held = 0;        // device bytes this slot holds (arena + plan)
    void* direct_out = nullptr;  // caller's pinned output buffer of the ticket, if any
    bool busy = false;
    std::vector<hpvcd_wp_table> wp;
    GroupStreams groups;  // lent to the slot's plans
};

}  // namespace

struct hpvcd_gpu {
    int device = 0;
    std::mutex mu;
    std::vector<Slot> slots;
    uint64_t next_ticket = 1;
    uint64_t budget = 0;
    uint64_t in_use = 0;
    hpvcd_dpb* dpb = nullptr;  // hpvcd_gpu_set_dpb
    // schedule selection per submitted batch (hpvcd_gpu_set_selector)
    hpvcd_mlp* sel = nullptr;
    std::vector<hpvcd_sched> sel_cands;
    hpvcd_sched fixed{};  // hpvcd_gpu_set_sched: the schedule without a selector
    // host copy of the network, read by the submit path's host-side pick
    std::vector<float> sel_w;
    float sel_lohi[2 * HPVCD_FEATURES] = {};
    int sel_has_domain = 0;
    uint64_t sel_picks[HPVCD_MLP_MAX_VARIANTS + 1] = {};  // last entry: batches outside the domain
    ~hpvcd_gpu() {
        for (Slot& s : slots) {
            if (s.stream) cudaStreamSynchronize(s.stream);
            delete s.plan;
            if (s.stream) cudaStreamSynchronize(s.stream);
            s.groups.destroy();
            cudaFreeHost(s.h_in);
            cudaFreeHost(s.h_out);
            cudaFree(s.d_in);
            if (s.done) cudaEventDestroy(s.done);
            if (s.stream) cudaStreamDestroy(s.stream);
        }
    }
};

namespace {

hpvcd_status grow_pinned(unsigned char** p, size_t* cap, size_t need) {
    if (*cap >= need) return HPVCD_OK;
    cudaFreeHost(*p);
    *p = nullptr;
    *cap = 0;
    const size_t sz = align_up(need + need / 4, 1 << 20);
    if (cudaMallocHost(p, sz) != cudaSuccess) {
        cudaGetLastError();
        return HPVCD_ERR_ALLOC;
    }
    *cap = sz;
    return HPVCD_OK;
}

hpvcd_status grow_device(unsigned char** p, size_t* cap, size_t need) {
    if (*cap >= need) return HPVCD_OK;
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    const size_t sz = align_up(need + need / 4, 1 << 20);
    if (cudaMalloc(p, sz) != cudaSuccess) {
        cudaGetLastError();
        return HPVCD_ERR_ALLOC;
    }
    *cap = sz;
    return HPVCD_OK;
}

Slot* find_ticket(hpvcd_gpu* g, hpvcd_ticket t) {
    for (Slot& s : g->slots)
        if (s.busy && s.ticket == t) return &s;
    return nullptr;
}

hpvcd_status device_status(hpvcd_plan* P, cudaStream_t st) {
    uint32_t err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, P->d_scratch + P->waves.size(), sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e);
    if (err & hpvcd::DEV_ERR_TIMEOUT) return HPVCD_ERR_TIMEOUT;
    if (err & hpvcd::DEV_ERR_BITSTREAM) return HPVCD_ERR_BITSTREAM;
    return HPVCD_OK;
}

// Layout of the inputs of a batch in one arena (256-byte aligned parts in a
// fixed order per picture: tus, ctu starts, coefficients, cells, SAO, PUs,
// scaling lists, CTB regions, slice deblocking offsets, prediction planes).  Shared by hpvcd_gpu_pack_inputs and submit.
struct InputPart {
    const void* src;
    size_t bytes;
    size_t off;
    uint32_t pic;
    int kind;  // 0..5 as above, 6..8 = prediction planes Y/Cb/Cr, 9 = scaling lists, 10 = CTB regions,
               // 11 = per-slice deblocking offsets
};

size_t input_layout(const hpvcd_picture* pics, uint32_t n, std::vector<InputPart>* parts) {
    size_t total = 0;
    auto add = [&](uint32_t i, int kind, const void* src, size_t bytes) {
        if (!src || !bytes) return;
        parts->push_back(InputPart{src, bytes, total, i, kind});
        total = align_up(total + bytes, 256);
    };
    for (uint32_t i = 0; i < n; ++i) {
        const hpvcd_picture& p = pics[i];
        const Geo geo = geo_of(p);
        const size_t ctbs = (size_t)geo.ctb_cols * geo.ctb_rows;
        add(i, 0, p.tus, (size_t)p.n_tus * sizeof(hpvcd_tu));
        add(i, 1, p.ctu_tu_start, (ctbs + 1) * sizeof(uint32_t));
        add(i, 2, p.coeffs, (size_t)p.n_coeffs * ((p.flags & HPVCD_PIC_COEFF8) ? 1 : sizeof(int16_t)));
        add(i, 3, p.cells, (size_t)geo.gw * geo.gh * sizeof(hpvcd_cell));
        add(i, 4, p.sao, ctbs * sizeof(hpvcd_sao_ctb));
        add(i, 5, p.pus, (size_t)p.n_pus * sizeof(hpvcd_pu));
        add(i, 9, p.scaling, sizeof(hpvcd_scaling));
        add(i, 10, p.ctb_region, ctbs * sizeof(uint16_t));
        add(i, 11, p.slice_deblock, 512);
        if (p.flags & HPVCD_PIC_PRED_IN_PLANE)
            for (int c = 0; c < (p.chroma_idc ? 3 : 1); ++c)
                add(i, 6 + c, p.pred[c], c ? geo.chroma_bytes : geo.luma_bytes);
    }
    return total;
}

void point_at(hpvcd_picture& d, int kind, const void* ptr) {
    switch (kind) {
        case 0: d.tus = (const hpvcd_tu*)ptr; break;
        case 1: d.ctu_tu_start = (const uint32_t*)ptr; break;
        case 2: d.coeffs = (const int16_t*)ptr; break;
        case 3: d.cells = (const hpvcd_cell*)ptr; break;
        case 4: d.sao = (const hpvcd_sao_ctb*)ptr; break;
        case 5: d.pus = (const hpvcd_pu*)ptr; break;
        case 9: d.scaling = (const hpvcd_scaling*)ptr; break;
        case 10: d.ctb_region = (const uint16_t*)ptr; break;
        case 11: d.slice_deblock = (const int8_t*)ptr; break;
        default: d.pred[kind - 6] = ptr; break;
    }
}

bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

// ===========================================================================
// Exported C ABI
// ===========================================================================
HPVCD_API uint32_t hpvcd_abi_version(void) { return HPVCD_ABI_VERSION; }

HPVCD_API const char* hpvcd_status_string(int s) {
    switch (s) {
        case HPVCD_OK: return "ok";
        case HPVCD_ERR_BITSTREAM: return "bitstream: malformed reconstruction buffers";
        case HPVCD_ERR_ALLOC: return "allocation failed (HBM budget or device memory)";
        case HPVCD_ERR_LIMIT: return "limit exceeded";
        case HPVCD_ERR_UNSUPPORTED: return "unsupported feature";
        case HPVCD_ERR_TIMEOUT: return "device-side wait timed out";
        case HPVCD_ERR_CUDA: return "CUDA runtime error";
        case HPVCD_ERR_INVALID_ARG: return "invalid argument";
        case HPVCD_ERR_BUSY: return "ticket not finished";
        default: return "unknown status";
    }
}

HPVCD_API uint64_t hpvcd_kernel_launch_count(void) { return g_launches.load(); }

HPVCD_API const char* hpvcd_last_error_string(void) { return t_last_error; }

// The calling thread's last error, for host code outside this file.
void hpvcd_note_error(const char* msg) { std::snprintf(t_last_error, sizeof(t_last_error), "%s", msg); }

HPVCD_API hpvcd_status hpvcd_copy(void* dst, const void* src, uint64_t bytes, void* stream) {
    if ((!dst || !src) && bytes) return HPVCD_ERR_INVALID_ARG;
    if (!bytes) return HPVCD_OK;
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    return cuda_status(e);
}

// sizeof of ABI structs, for the binding layout test.
HPVCD_API uint64_t hpvcd_abi_sizeof(const char* name) {
    if (!name) return 0;
    const struct {
        const char* n;
        size_t s;
    } t[] = {{"hpvcd_tu", sizeof(hpvcd_tu)},           {"hpvcd_cell", sizeof(hpvcd_cell)},
             {"hpvcd_sao_comp", sizeof(hpvcd_sao_comp)}, {"hpvcd_sao_ctb", sizeof(hpvcd_sao_ctb)},
             {"hpvcd_pu", sizeof(hpvcd_pu)},           {"hpvcd_wp_entry", sizeof(hpvcd_wp_entry)},
             {"hpvcd_wp_table", sizeof(hpvcd_wp_table)}, {"hpvcd_picture", sizeof(hpvcd_picture)},
             {"hpvcd_tile_place", sizeof(hpvcd_tile_place)}, {"hpvcd_output", sizeof(hpvcd_output)},
             {"hpvcd_canvas", sizeof(hpvcd_canvas)}, {"hpvcd_server_cfg", sizeof(hpvcd_server_cfg)},
             {"hpvcd_request", sizeof(hpvcd_request)}, {"hpvcd_completion", sizeof(hpvcd_completion)},
             {"hpvcd_gpu_cfg", sizeof(hpvcd_gpu_cfg)}, {"hpvcd_sched", sizeof(hpvcd_sched)},
             {"hpvcd_scaling", sizeof(hpvcd_scaling)}, {"hpvcd_slice_params", sizeof(hpvcd_slice_params)}};
    for (const auto& e : t)
        if (std::strcmp(e.n, name) == 0) return e.s;
    return 0;
}

HPVCD_API hpvcd_status hpvcd_plan_create(const hpvcd_picture* dev_pics, uint32_t n, const hpvcd_output* out,
                                         const hpvcd_sched* sched, hpvcd_plan** plan) {
    if (!dev_pics || !plan) return HPVCD_ERR_INVALID_ARG;
    // Device-pointer descriptors: weighted-prediction tables are read from
    // device memory once here.
    std::vector<hpvcd_wp_table> wp(n);
    bool any = false;
    for (uint32_t i = 0; i < n; ++i)
        if (dev_pics[i].wp) {
            if (cudaMemcpy(&wp[i], dev_pics[i].wp, sizeof(hpvcd_wp_table), cudaMemcpyDeviceToHost) != cudaSuccess) {
                cudaGetLastError();
                return HPVCD_ERR_INVALID_ARG;
            }
            any = true;
        }
    return plan_build(dev_pics, n, out, sched, any ? wp.data() : nullptr, plan);
}

HPVCD_API hpvcd_status hpvcd_plan_destroy(hpvcd_plan* plan) {
    if (!plan) return HPVCD_ERR_INVALID_ARG;
    cudaDeviceSynchronize();
    delete plan;
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_plan_launch(hpvcd_plan* plan, uint32_t stages, void* stream) {
    if (!plan) return HPVCD_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (!(stages & HPVCD_STAGE_GRAPH)) return plan_launch(plan, stages, st);
    if (st == nullptr || st == cudaStreamLegacy) return HPVCD_ERR_INVALID_ARG;
    const uint32_t key = stages & HPVCD_STAGE_ALL;
    cudaGraphExec_t& gx = plan->graphs[key];
    if (!gx) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_status(e);
        const uint64_t before = g_launches.load();
        const hpvcd_status ls = plan_launch(plan, key, st);
        e = cudaStreamEndCapture(st, &g);
        // captured launches did not run: do not count them
        g_launches.store(before);
        if (ls != HPVCD_OK) {
            if (g) cudaGraphDestroy(g);
            return ls;
        }
        if (e != cudaSuccess) return cuda_status(e);
        e = cudaGraphInstantiate(&gx, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            gx = nullptr;
            return cuda_status(e);
        }
    }
    const cudaError_t e = cudaGraphLaunch(gx, st);
    if (e == cudaSuccess) hpvcd_note_launches(plan->launches_for(key));
    return cuda_status(e);
}

HPVCD_API hpvcd_status hpvcd_plan_planes(hpvcd_plan* plan, uint32_t i, void** y, void** cb, void** cr) {
    if (!plan || i >= plan->src.size()) return HPVCD_ERR_INVALID_ARG;
    if (y) *y = plan->pics[i].fin[0];
    if (cb) *cb = plan->pics[i].fin[1];
    if (cr) *cr = plan->pics[i].fin[2];
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_plan_canvas(hpvcd_plan* plan, void** rgb, uint64_t* bytes) {
    if (!plan) return HPVCD_ERR_INVALID_ARG;
    if (rgb) *rgb = plan->d_canvas;
    if (bytes) *bytes = plan->canvas_bytes;
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_plan_device_status(hpvcd_plan* plan, void* stream) {
    if (!plan) return HPVCD_ERR_INVALID_ARG;
    return device_status(plan, (cudaStream_t)stream);
}

HPVCD_API uint32_t hpvcd_plan_launches_per_run(const hpvcd_plan* plan) {
    return plan ? plan->launches_per_run : 0;
}

HPVCD_API hpvcd_status hpvcd_plan_set_sched(hpvcd_plan* plan, const hpvcd_sched* sched);

// Feature vector (16 floats, include/hpvcd_gpu.h) of pictures [first, first +
// count) of the plan into dev_out (device memory), enqueued on `stream`.
HPVCD_API hpvcd_status hpvcd_plan_features(hpvcd_plan* plan, uint32_t first, uint32_t count, float* dev_out,
                                           void* stream) {
    if (!plan || !dev_out || count == 0 || first + count > plan->src.size() || first + count < first)
        return HPVCD_ERR_INVALID_ARG;
    uint32_t max_rec = 1;
    for (uint32_t i = first; i < first + count; ++i)
        max_rec = std::max(max_rec, std::max(plan->src[i].n_tus, plan->src[i].n_pus));
    return cuda_status(hpvcd_launch_features(plan->d_pics + first, count, max_rec, plan->d_feat, dev_out, plan->sms,
                                             (cudaStream_t)stream));
}

// Exhaustive autotuning: one untimed launch, then per candidate schedule
// `warmup` untimed and `reps` timed launches (CUDA events on `stream`);
// ms[i] = the fastest timed launch.  The fastest candidate stays set.
HPVCD_API hpvcd_status hpvcd_plan_autotune(hpvcd_plan* plan, const hpvcd_sched* cands, uint32_t n, uint32_t stages,
                                           uint32_t reps, uint32_t warmup, void* stream, float* ms, uint32_t* best) {
    if (!plan || !cands || n == 0 || reps == 0 || reps > 64 || warmup > 64) return HPVCD_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t ev[2];
    cudaError_t e = cudaEventCreate(&ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
    if (e != cudaSuccess) return cuda_status(e);
    hpvcd_status s = HPVCD_OK;
    uint32_t arg = 0;
    float best_ms = 0.f;
    std::vector<float> t(reps);
    s = hpvcd_plan_set_sched(plan, &cands[0]);
    if (s == HPVCD_OK) s = plan_launch(plan, stages & HPVCD_STAGE_ALL, st);
    for (uint32_t c = 0; c < n && s == HPVCD_OK; ++c) {
        s = hpvcd_plan_set_sched(plan, &cands[c]);
        for (uint32_t w = 0; w < warmup && s == HPVCD_OK; ++w) s = plan_launch(plan, stages & HPVCD_STAGE_ALL, st);
        for (uint32_t r = 0; r < reps && s == HPVCD_OK; ++r) {
            e = cudaEventRecord(ev[0], st);
            if (e == cudaSuccess) s = plan_launch(plan, stages & HPVCD_STAGE_ALL, st);
            if (s == HPVCD_OK && e == cudaSuccess) e = cudaEventRecord(ev[1], st);
            if (s == HPVCD_OK && e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
            if (s == HPVCD_OK && e == cudaSuccess) e = cudaEventElapsedTime(&t[r], ev[0], ev[1]);
            if (s == HPVCD_OK && e != cudaSuccess) s = cuda_status(e);
        }
        if (s != HPVCD_OK) break;
        const float fastest = *std::min_element(t.begin(), t.end());
        if (ms) ms[c] = fastest;
        if (c == 0 || fastest < best_ms) {
            best_ms = fastest;
            arg = c;
        }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (s != HPVCD_OK) return s;
    if (best) *best = arg;
    return hpvcd_plan_set_sched(plan, &cands[arg]);
}

HPVCD_API hpvcd_status hpvcd_plan_set_sched(hpvcd_plan* plan, const hpvcd_sched* sched) {
    if (!plan) return HPVCD_ERR_INVALID_ARG;
    const hpvcd_sched next = sched ? *sched : hpvcd_sched{};
    if (next.idct > 2 || next.chroma_warps > 3 || next.wave > 1) return HPVCD_ERR_INVALID_ARG;
    if (std::memcmp(&next, &plan->sched, sizeof(next)) == 0) return HPVCD_OK;
    plan->sched = next;
    // graphs captured with the previous schedule hold its kernels
    for (cudaGraphExec_t& gx : plan->graphs)
        if (gx) {
            cudaGraphExecDestroy(gx);
            gx = nullptr;
        }
    return HPVCD_OK;
}

// Test hook of the bounded wavefront waits: every wait of the plan's
// reconstruction kernel gives up after `spin_limit` polls (0 = the default),
// and entry `drop_ctu` of the CTU work list is left out of the launches
// (-1 restores it): that CTU is never reconstructed, so the waits of the CTUs
// predicting from it run out, set the device error word and return.
HPVCD_API hpvcd_status hpvcd_plan_set_wait_test(hpvcd_plan* plan, uint32_t spin_limit, int32_t drop_ctu) {
    if (!plan || drop_ctu < -1 || (drop_ctu >= 0 && (size_t)drop_ctu >= plan->items.size()))
        return HPVCD_ERR_INVALID_ARG;
    std::vector<CtuItem> list = plan->items;
    for (hpvcd_plan::Wave& wv : plan->waves) {
        const uint32_t end = wv.item_off + wv.n_full;
        wv.n_items = wv.n_full;
        if (drop_ctu >= 0 && (uint32_t)drop_ctu >= wv.item_off && (uint32_t)drop_ctu < end) {
            // the wave's later entries move up by one; its last slot is not launched
            list.erase(list.begin() + drop_ctu);
            list.insert(list.begin() + (end - 1), plan->items[(size_t)drop_ctu]);
            wv.n_items -= 1;
        }
    }
    if (!list.empty()) {
        const cudaError_t e =
            cudaMemcpy(plan->d_items, list.data(), sizeof(CtuItem) * list.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_status(e);
    }
    plan->spin_limit = spin_limit;
    plan->drop_item = drop_ctu;
    for (cudaGraphExec_t& gx : plan->graphs)
        if (gx) {
            cudaGraphExecDestroy(gx);
            gx = nullptr;
        }
    return HPVCD_OK;
}

// Schedule selection for a plan: with a selector network, the features of
// the whole batch are computed on the device and the network's predicted-
// fastest candidate is set; without one (or when its candidate count does
// not match) exhaustive autotuning over the candidates decides.
HPVCD_API hpvcd_status hpvcd_plan_select(hpvcd_plan* plan, hpvcd_mlp* mlp, const hpvcd_sched* cands, uint32_t n,
                                         void* stream, uint32_t* chosen) {
    if (!plan || !cands || n == 0) return HPVCD_ERR_INVALID_ARG;
    uint32_t pick = 0;
    hpvcd_status s;
    if (mlp && hpvcd_mlp_variants(mlp) == n) {
        float* fv = (float*)(plan->d_feat + 32);
        s = hpvcd_plan_features(plan, 0, (uint32_t)plan->src.size(), fv, stream);
        if (s == HPVCD_OK) s = hpvcd_mlp_pick(mlp, fv, 1, stream, &pick);
        // outside the network's training domain: the first (default) candidate
        if (s == HPVCD_OK) s = hpvcd_plan_set_sched(plan, &cands[pick == HPVCD_MLP_NO_PICK ? 0 : pick]);
    } else {
        s = hpvcd_plan_autotune(plan, cands, n, HPVCD_STAGE_ALL, 2, 1, stream, nullptr, &pick);
    }
    if (s == HPVCD_OK && chosen) *chosen = pick;
    return s;
}

HPVCD_API hpvcd_status hpvcd_gpu_create(const hpvcd_gpu_cfg* cfg, hpvcd_gpu** out) {
    if (!out) return HPVCD_ERR_INVALID_ARG;
    *out = nullptr;
    hpvcd_gpu_cfg c{};
    if (cfg) c = *cfg;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return HPVCD_ERR_CUDA;
    }
    if (c.device < 0 || c.device >= ndev) return HPVCD_ERR_INVALID_ARG;
    if (cudaSetDevice(c.device) != cudaSuccess) return HPVCD_ERR_CUDA;
    hpvcd_gpu* g = new (std::nothrow) hpvcd_gpu();
    if (!g) return HPVCD_ERR_ALLOC;
    g->device = c.device;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    g->budget = c.hbm_budget ? c.hbm_budget : (uint64_t)(free_b * 0.8);
    const uint32_t inflight = c.max_inflight ? std::min<uint32_t>(c.max_inflight, 64) : 4;
    g->slots.resize(inflight);
    {
        // keep freed plan memory in the device pool for the next batch
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, c.device) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        cudaGetLastError();
    }
    for (Slot& s : g->slots) {
        if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) {
            delete g;
            cudaGetLastError();
            return HPVCD_ERR_CUDA;
        }
    }
    *out = g;
    return HPVCD_OK;
}

namespace {

// After a batch's launch on its slot stream: mark the DPB entries it read,
// then store the pictures flagged HPVCD_PIC_STORE_DPB into their entries
// (each store waits for the batches of other slots still reading the entry).
hpvcd_status dpb_after_launch(hpvcd_gpu* g, Slot* slot, int slot_idx, const hpvcd_picture* pics, uint32_t n) {
    hpvcd_plan* P = slot->plan;
    cudaError_t e = cudaSuccess;
    for (const int en : P->dpb_refs) {
        hpvcd_dpb::Entry& E = g->dpb->entries[(size_t)en];
        if (!E.ev_read[slot_idx]) e = cudaEventCreateWithFlags(&E.ev_read[slot_idx], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(E.ev_read[slot_idx], slot->stream);
        if (e != cudaSuccess) return cuda_status(e);
        E.read[slot_idx] = true;
    }
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t tag = (pics[i].flags & HPVCD_PIC_STORE_MASK) >> 16;
        if (!tag) continue;
        if (!g->dpb || tag - 1 >= g->dpb->entries.size()) return HPVCD_ERR_INVALID_ARG;
        hpvcd_dpb::Entry& E = g->dpb->entries[tag - 1];
        for (int k = 0; k < HPVCD_DPB_MAX_READERS && e == cudaSuccess; ++k)
            if (E.read[k] && k != slot_idx) e = cudaStreamWaitEvent(slot->stream, E.ev_read[k], 0);
        const Geo geo = geo_of(pics[i]);
        const size_t need = align_up(geo.luma_bytes, 256) + 2 * align_up(geo.chroma_bytes, 256);
        if (e == cudaSuccess && E.bytes != need) {
            // a new size: the old storage is released once nothing uses it
            if (E.written) e = cudaEventSynchronize(E.ev_write);
            for (int k = 0; k < HPVCD_DPB_MAX_READERS && e == cudaSuccess; ++k)
                if (E.read[k] && k != slot_idx) e = cudaEventSynchronize(E.ev_read[k]);
            if (e == cudaSuccess && E.planes) e = cudaStreamSynchronize(slot->stream);
            if (e == cudaSuccess) {
                cudaFree(E.planes);
                E.planes = nullptr;
                E.bytes = 0;
                e = cudaMalloc((void**)&E.planes, need);
                if (e == cudaSuccess) E.bytes = need;
            }
        }
        const DevPic& d = P->pics[i];
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(E.planes, d.fin[0], geo.luma_bytes, cudaMemcpyDeviceToDevice, slot->stream);
        for (int c = 1; c < (pics[i].chroma_idc ? 3 : 1) && e == cudaSuccess; ++c)
            e = cudaMemcpyAsync(E.planes + align_up(geo.luma_bytes, 256) + (c - 1) * align_up(geo.chroma_bytes, 256),
                                d.fin[c], geo.chroma_bytes, cudaMemcpyDeviceToDevice, slot->stream);
        if (e == cudaSuccess && !E.ev_write) e = cudaEventCreateWithFlags(&E.ev_write, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(E.ev_write, slot->stream);
        if (e != cudaSuccess) return cuda_status(e);
        E.written = true;
        E.valid = true;
        E.w = (int)pics[i].width;
        E.h = (int)pics[i].height;
        E.idc = pics[i].chroma_idc;
        E.bd = pics[i].bit_depth_y;
        E.bd_c = pics[i].bit_depth_c;
        E.luma_bytes = geo.luma_bytes;
        E.chroma_bytes = geo.chroma_bytes;
    }
    return HPVCD_OK;
}

}  // namespace

HPVCD_API hpvcd_status hpvcd_dpb_create(int32_t device, uint32_t entries, hpvcd_dpb** out) {
    if (!out || entries == 0 || entries > 254) return HPVCD_ERR_INVALID_ARG;
    hpvcd_dpb* D = new (std::nothrow) hpvcd_dpb();
    if (!D) return HPVCD_ERR_ALLOC;
    D->device = device;
    D->entries.resize(entries);
    *out = D;
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_dpb_destroy(hpvcd_dpb* D) {
    if (!D) return HPVCD_ERR_INVALID_ARG;
    cudaSetDevice(D->device);
    delete D;
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_gpu_set_dpb(hpvcd_gpu* g, hpvcd_dpb* dpb) {
    if (!g || (dpb && dpb->device != g->device)) return HPVCD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g->mu);
    g->dpb = dpb;
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_gpu_set_selector(hpvcd_gpu* g, hpvcd_mlp* mlp, const hpvcd_sched* cands, uint32_t n) {
    if (!g || (mlp && (!cands || n == 0 || n != hpvcd_mlp_variants(mlp)))) return HPVCD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g->mu);
    g->sel = mlp;
    g->sel_cands.assign(cands, cands + (mlp ? n : 0));
    std::memset(g->sel_picks, 0, sizeof(g->sel_picks));
    g->sel_w.clear();
    if (mlp) {  // the network as it is now: later training needs another set_selector
        cudaSetDevice(g->device);
        g->sel_w.resize(hpvcd_mlp_param_count(mlp));
        const hpvcd_status s = hpvcd_mlp_host_copy(mlp, g->sel_w.data(), g->sel_lohi, &g->sel_has_domain);
        if (s != HPVCD_OK) {
            g->sel = nullptr;
            g->sel_cands.clear();
            return s;
        }
    }
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_gpu_set_sched(hpvcd_gpu* g, const hpvcd_sched* sched) {
    if (!g) return HPVCD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g->mu);
    g->fixed = sched ? *sched : hpvcd_sched{};
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_gpu_selector_picks(hpvcd_gpu* g, uint64_t* counts, uint32_t n) {
    if (!g || !counts) return HPVCD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g->mu);
    // counts[0 .. K-1]: picks per candidate; counts[K] (when n > K): batches
    // outside the network's domain (features out of range, or submitted
    // while other tickets ran), which ran the fixed schedule
    const uint32_t K = (uint32_t)g->sel_cands.size();
    for (uint32_t i = 0; i < n; ++i)
        counts[i] = i < K ? g->sel_picks[i] : (i == K ? g->sel_picks[HPVCD_MLP_MAX_VARIANTS] : 0);
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_gpu_destroy(hpvcd_gpu* g) {
    if (!g) return HPVCD_ERR_INVALID_ARG;
    cudaSetDevice(g->device);
    delete g;
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_gpu_submit(hpvcd_gpu* g, const hpvcd_picture* pics, uint32_t n,
                                        const hpvcd_output* out, hpvcd_ticket* ticket) {
    if (!g || !pics || n == 0 || !ticket) return HPVCD_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; ++i) {
        const hpvcd_status s = validate(pics[i]);
        if (s != HPVCD_OK) return s;
    }
    if (out && canvas_kind(out->kind) &&
        (!out->place || (out->n_canvases ? !out->canvases : (!out->canvas_w || !out->canvas_h))))
        return HPVCD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g->mu);
    for (uint32_t i = 0; i < n; ++i) {  // DPB stores need an attached DPB with that entry
        const uint32_t tag = (pics[i].flags & HPVCD_PIC_STORE_MASK) >> 16;
        if (tag && (!g->dpb || tag - 1 >= g->dpb->entries.size())) {
            std::snprintf(t_last_error, sizeof(t_last_error), "picture %u stores into DPB entry %u, which does not exist",
                          i, tag - 1);
            return HPVCD_ERR_INVALID_ARG;
        }
    }
    cudaSetDevice(g->device);
    Slot* slot = nullptr;
    for (Slot& s : g->slots)
        if (!s.busy) {
            slot = &s;
            break;
        }
    if (!slot) return HPVCD_ERR_BUSY;
    // ---- input layout in one arena ----
    std::vector<InputPart> parts;
    const size_t total = input_layout(pics, n, &parts);
    std::vector<hpvcd_picture> dev(pics, pics + n);
    for (hpvcd_picture& d : dev) {
        d.tus = nullptr; d.ctu_tu_start = nullptr; d.coeffs = nullptr; d.cells = nullptr;
        d.sao = nullptr; d.pus = nullptr; d.pred[0] = d.pred[1] = d.pred[2] = nullptr;
        d.scaling = nullptr;
        d.ctb_region = nullptr;
        d.slice_deblock = nullptr;
    }
    // Runs of parts laid out contiguously (as hpvcd_gpu_pack_inputs lays them
    // out) in page-locked memory go up by DMA straight from the caller's
    // memory, one transfer per run; everything else through the staging copy.
    struct Run {
        const unsigned char* src;
        size_t off, bytes;
        bool pinned;
    };
    std::vector<Run> runs;
    for (const InputPart& pt : parts) {
        const unsigned char* sp = (const unsigned char*)pt.src;
        if (!runs.empty()) {
            Run& r = runs.back();
            if (sp - pt.off == r.src - r.off && pt.off >= r.off + r.bytes) {
                r.bytes = pt.off + pt.bytes - r.off;
                continue;
            }
        }
        runs.push_back(Run{sp, pt.off, pt.bytes, false});
    }
    bool all_pinned = !runs.empty();
    for (Run& r : runs) {
        r.pinned = is_pinned(r.src);
        all_pinned &= r.pinned;
    }
    // ---- HBM admission ----
    const size_t out_bytes = output_bytes(pics, n, out);
    const bool reuse = slot->plan && same_layout(slot->plan, pics, n, out);
    // HBM admission: what this slot would hold after the call (input arena +
    // plan) against what it holds now; refuse when the context budget would
    // be exceeded (the caller may retry once other tickets are read).
    const uint64_t held = slot->held;
    const uint64_t plan_bytes = reuse ? slot->plan_bytes : plan_footprint(pics, n, out);
    const uint64_t need = std::max<uint64_t>(slot->d_in_cap, align_up(total + total / 4, 1 << 20)) + plan_bytes;
    if (g->in_use - held + need > g->budget) return HPVCD_ERR_ALLOC;
    const bool per_canvas_out = out && canvas_kind(out->kind) && out->n_canvases && out->canvas_dst;
    const bool direct_out = per_canvas_out ||
                            (out && out->host_dst && out->host_dst_bytes >= out_bytes && is_pinned(out->host_dst));
    hpvcd_status st = all_pinned ? HPVCD_OK : grow_pinned(&slot->h_in, &slot->h_in_cap, total);
    if (st == HPVCD_OK) st = grow_device(&slot->d_in, &slot->d_in_cap, std::max<size_t>(total, 256));
    if (st == HPVCD_OK && !direct_out) st = grow_pinned(&slot->h_out, &slot->h_out_cap, out_bytes);
    if (st != HPVCD_OK) return st;
    cudaError_t e = cudaSuccess;
    if (all_pinned) {
        for (const Run& r : runs) {
            e = cudaMemcpyAsync(slot->d_in + r.off, r.src, r.bytes, cudaMemcpyHostToDevice, slot->stream);
            if (e != cudaSuccess) break;
        }
    } else {
        // Staged through the slot's page-locked buffer in windows of
        // kStageWindow bytes: the copy pool fills window k + 1 while window
        // k's DMA runs.  Parts are laid out in ascending offsets.
        constexpr size_t kStageWindow = 8u << 20;
        std::vector<hpvcd_host::CopyTask> tasks;
        size_t w0 = 0, pi = 0, part_done = 0;
        while (w0 < total && e == cudaSuccess) {
            const size_t w1 = std::min(total, w0 + kStageWindow);
            tasks.clear();
            while (pi < parts.size() && parts[pi].off + part_done < w1) {
                const InputPart& pt = parts[pi];
                const size_t take = std::min(pt.bytes - part_done, w1 - (pt.off + part_done));
                tasks.push_back(hpvcd_host::CopyTask{slot->h_in + pt.off + part_done,
                                                     (const unsigned char*)pt.src + part_done, take});
                part_done += take;
                if (part_done == pt.bytes) {
                    ++pi;
                    part_done = 0;
                }
            }
            hpvcd_host::parallel_copy(tasks.data(), tasks.size());
            e = cudaMemcpyAsync(slot->d_in + w0, slot->h_in + w0, w1 - w0, cudaMemcpyHostToDevice, slot->stream);
            w0 = w1;
        }
    }
    if (e != cudaSuccess) return cuda_status(e);
    for (const InputPart& pt : parts) point_at(dev[pt.pic], pt.kind, slot->d_in + pt.off);
    slot->wp.assign(n, hpvcd_wp_table{});
    bool any_wp = false;
    for (uint32_t i = 0; i < n; ++i) {
        if (pics[i].wp) {
            slot->wp[i] = *pics[i].wp;
            any_wp = true;
        }
        dev[i].wp = pics[i].wp;  // only tested for NULL; the table itself is passed by value
    }
    if (reuse) {
        st = plan_rebind(slot->plan, dev.data(), any_wp ? slot->wp.data() : nullptr, slot->stream);
    } else {
        if (slot->plan) {
            delete slot->plan;  // stream-ordered frees on slot->stream
            slot->plan = nullptr;
            slot->plan_bytes = 0;
        }
        st = plan_build(dev.data(), n, out, nullptr, any_wp ? slot->wp.data() : nullptr, &slot->plan,
                        slot->stream, true, &slot->groups, g->dpb);
        slot->plan_bytes = st == HPVCD_OK ? plan_bytes : 0;
    }
    g->in_use = g->in_use - held + slot->d_in_cap + slot->plan_bytes;
    slot->held = slot->d_in_cap + slot->plan_bytes;
    if (st != HPVCD_OK) return st;
    int others = 0;  // tickets of this context already in flight
    for (const Slot& s : g->slots)
        if (s.busy && &s != slot) ++others;
    // The network was trained on batches decoded alone; with other tickets in
    // flight the batch runs the context's fixed schedule (counted with the
    // batches outside the network's domain).
    if (g->sel && others > 0) {
        st = hpvcd_plan_set_sched(slot->plan, &g->fixed);
        if (st != HPVCD_OK) return st;
        ++g->sel_picks[HPVCD_MLP_MAX_VARIANTS];
    } else if (g->sel) {  // the network picks the batch's schedule from its features
        // Up to kHostPickRecords records (a few ms of host work at most) the
        // features and the network run on the host, with no device round
        // trip; larger batches use the kernels and wait for their pick.  Both
        // give the same pick.
        constexpr uint64_t kHostPickRecords = 1u << 19;
        uint64_t records = 0;
        for (uint32_t i = 0; i < n; ++i) records += pics[i].n_tus + pics[i].n_pus;
        uint32_t pick = 0;
        if (records <= kHostPickRecords) {
            float fv[HPVCD_FEATURES];
            st = hpvcd_batch_features(pics, n, fv);
            if (st != HPVCD_OK) return st;
            pick = hpvcd_mlp_pick_host(g->sel_w.data(), (uint32_t)g->sel_cands.size(), fv, g->sel_lohi,
                                       g->sel_has_domain);
            st = hpvcd_plan_set_sched(slot->plan, pick == HPVCD_MLP_NO_PICK ? &g->fixed : &g->sel_cands[pick]);
        } else {
            st = hpvcd_plan_select(slot->plan, g->sel, g->sel_cands.data(), (uint32_t)g->sel_cands.size(),
                                   slot->stream, &pick);
            if (st == HPVCD_OK && pick == HPVCD_MLP_NO_PICK) st = hpvcd_plan_set_sched(slot->plan, &g->fixed);
        }
        if (st != HPVCD_OK) return st;
        ++g->sel_picks[pick == HPVCD_MLP_NO_PICK ? HPVCD_MLP_MAX_VARIANTS : pick];
    } else {
        st = hpvcd_plan_set_sched(slot->plan, &g->fixed);
        if (st != HPVCD_OK) return st;
    }
    // Tickets already in flight share the SMs with this one: the wavefront
    // kernel's persistent grid keeps to its share of the CTA slots (its CTAs
    // wait for their neighbour CTUs in place, holding slots the other
    // tickets' kernels need).  At three tickets in flight on the 4032x3024
    // grid the share is worth about 15 % of throughput; a ticket alone keeps
    // the full grid.  Sharing, the default build is the register-capped one:
    // eight CTAs per SM split between the tickets instead of five (at four
    // tickets in flight one CTA per SM each with the plain build, a quarter
    // of that per group of the grid, fewer than the group's ready CTUs).
    // With two CTAs per SM per ticket the quadrant-level wavefront also pays
    // while sharing (four grids in flight: 1.19 against 1.29 ms per image
    // with whole-CTU waits, same box).
    {
        if (others > 0) {
            hpvcd_sched s2 = slot->plan->sched;
            const hpvcd_plan* pl = slot->plan;
            if (s2.chroma_warps == 0) s2.chroma_warps = 3;
            const int occ = std::max(1, pl->occ_of(pl->waves.empty() ? 0 : pl->waves[0].cfmt, (int)s2.chroma_warps));
            const int share = std::max(1, occ / (others + 1));
            const int cur = s2.recon_ctas_per_sm ? (int)s2.recon_ctas_per_sm : occ;
            s2.recon_ctas_per_sm = (uint32_t)std::min(cur, share);
            st = hpvcd_plan_set_sched(slot->plan, &s2);
            if (st != HPVCD_OK) return st;
        }
    }
    const int slot_idx = (int)(slot - g->slots.data());
    // DPB entries this batch predicts from: wait for the stores that filled them
    for (const int en : slot->plan->dpb_refs) {
        hpvcd_dpb::Entry& E = g->dpb->entries[(size_t)en];
        if (E.written) {
            const cudaError_t we = cudaStreamWaitEvent(slot->stream, E.ev_write, 0);
            if (we != cudaSuccess) return cuda_status(we);
        }
    }
    st = plan_launch(slot->plan, HPVCD_STAGE_ALL, slot->stream);
    if (st != HPVCD_OK) return st;
    st = dpb_after_launch(g, slot, slot_idx, pics, n);
    if (st != HPVCD_OK) return st;
    // ---- output copy back ----
    hpvcd_plan* P = slot->plan;
    unsigned char* host_out = direct_out && !per_canvas_out ? (unsigned char*)out->host_dst : slot->h_out;
    slot->direct_out = direct_out ? (per_canvas_out ? (void*)1 : out->host_dst) : nullptr;
    if (per_canvas_out) {  // each canvas straight into its own buffer
        for (size_t k = 0; k < P->canvases.size() && e == cudaSuccess; ++k)
            e = cudaMemcpyAsync(out->canvas_dst[k], P->d_canvas + P->canvas_offs[k], P->canvas_sizes[k],
                                cudaMemcpyDeviceToHost, slot->stream);
    } else if (canvas_kind(P->out.kind)) {
        e = cudaMemcpyAsync(host_out, P->d_canvas, P->canvas_bytes, cudaMemcpyDeviceToHost, slot->stream);
    } else {
        size_t o = 0;
        for (uint32_t i = 0; i < n && e == cudaSuccess; ++i) {
            const Geo geo = geo_of(pics[i]);
            for (int c = 0; c < (pics[i].chroma_idc ? 3 : 1) && e == cudaSuccess; ++c) {
                const size_t b = c ? geo.chroma_bytes : geo.luma_bytes;
                e = cudaMemcpyAsync(host_out + o, P->pics[i].fin[c], b, cudaMemcpyDeviceToHost, slot->stream);
                o += b;
            }
        }
    }
    if (e == cudaSuccess) e = cudaEventRecord(slot->done, slot->stream);
    if (e != cudaSuccess) return cuda_status(e);
    slot->busy = true;
    slot->ticket = g->next_ticket++;
    slot->out_bytes = out_bytes;
    *ticket = slot->ticket;
    return HPVCD_OK;
}

HPVCD_API uint64_t hpvcd_gpu_packed_size(const hpvcd_picture* pics, uint32_t n) {
    if (!pics) return 0;
    std::vector<InputPart> parts;
    return input_layout(pics, n, &parts);
}

HPVCD_API hpvcd_status hpvcd_gpu_pack_inputs(const hpvcd_picture* pics, uint32_t n, void* dst, uint64_t bytes,
                                             hpvcd_picture* out_pics) {
    if (!pics || !dst || !out_pics) return HPVCD_ERR_INVALID_ARG;
    std::vector<InputPart> parts;
    const size_t total = input_layout(pics, n, &parts);
    if (bytes < total) return HPVCD_ERR_INVALID_ARG;
    std::vector<hpvcd_picture> res(pics, pics + n);
    std::vector<hpvcd_host::CopyTask> tasks;
    tasks.reserve(parts.size());
    for (const InputPart& pt : parts) {
        tasks.push_back(hpvcd_host::CopyTask{(unsigned char*)dst + pt.off, pt.src, pt.bytes});
        point_at(res[pt.pic], pt.kind, (unsigned char*)dst + pt.off);
    }
    hpvcd_host::parallel_copy(tasks.data(), tasks.size());
    std::memcpy(out_pics, res.data(), sizeof(hpvcd_picture) * n);
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_gpu_wait(hpvcd_gpu* g, hpvcd_ticket t, int32_t timeout_ms) {
    if (!g) return HPVCD_ERR_INVALID_ARG;
    cudaEvent_t ev;
    {
        std::lock_guard<std::mutex> lock(g->mu);
        Slot* s = find_ticket(g, t);
        if (!s) return HPVCD_ERR_INVALID_ARG;
        ev = s->done;
    }
    cudaSetDevice(g->device);
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return HPVCD_OK;
        if (e != cudaErrorNotReady) return cuda_status(e);
        if (timeout_ms >= 0 &&
            std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms))
            return HPVCD_ERR_BUSY;
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

HPVCD_API hpvcd_status hpvcd_gpu_output_size(hpvcd_gpu* g, hpvcd_ticket t, uint64_t* bytes) {
    if (!g || !bytes) return HPVCD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g->mu);
    Slot* s = find_ticket(g, t);
    if (!s) return HPVCD_ERR_INVALID_ARG;
    *bytes = s->out_bytes;
    return HPVCD_OK;
}

HPVCD_API hpvcd_status hpvcd_gpu_read(hpvcd_gpu* g, hpvcd_ticket t, void* dst, uint64_t bytes) {
    if (!g) return HPVCD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g->mu);
    Slot* s = find_ticket(g, t);
    if (!s) return HPVCD_ERR_INVALID_ARG;
    // outputs DMA'd to per-canvas destinations need no buffer here
    if (s->direct_out != (void*)1 && (!dst || bytes < s->out_bytes)) return HPVCD_ERR_INVALID_ARG;
    cudaSetDevice(g->device);
    cudaError_t e = cudaEventSynchronize(s->done);
    hpvcd_status st = cuda_status(e);
    if (st == HPVCD_OK) st = device_status(s->plan, s->stream);
    if (st == HPVCD_OK && s->direct_out != (void*)1 && dst != s->direct_out)
        hpvcd_host::parallel_copy(dst, s->direct_out ? (const unsigned char*)s->direct_out : s->h_out, s->out_bytes);
    s->busy = false;
    s->ticket = 0;
    return st;
}

// ---------------------------------------------------------------------------
// Decoding one picture without allocating (hpvcd_decode_noalloc).
//
// Some callers cannot allocate at decode time: an application that hands the
// decoder a fixed share of HBM and keeps every other byte in its own pool, or
// a frame loop with a latency budget where cudaMalloc/cudaFree would
// synchronise the device and stall unrelated streams.  For them the scratch of
// one picture's decode lives in one fixed array of module global memory,
// reserved when the module loads: work counter, device error word, wavefront
// wavefront progress words, the device picture record, the CTU work list, the int16
// residual planes and, when SAO runs, the pre-SAO planes.  The caller owns the
// inputs (device buffers) and the output planes.
//
// The array is reset per call by the first kernel the call enqueues, so calls
// ordered on one stream are safe; two calls whose work overlaps on a device
// (two streams, two host threads) use the same array and race.
// ---------------------------------------------------------------------------

// 12 MiB + 256 KiB: every picture up to 1024x1024 luma samples in any chroma
// format and bit depth with SAO on (int16 residual planes <= 6 MiB, pre-SAO
// planes <= 6 MiB, per-CTU records <= 48 KiB for 16x16 CTBs).
static constexpr size_t kNoAllocScratchBytes = HPVCD_NOALLOC_SCRATCH_BYTES;
static_assert(kNoAllocScratchBytes % 256 == 0, "scratch size");
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kNoAllocMaxDevices = 64;

struct NoAllocDevice {
    unsigned char* base = nullptr;  // address of g_noalloc_scratch on this device
    int sms = 0;
    int occ[3] = {0, 0, 0};         // k_recon CTAs per SM (4:2:0, 4:4:4, 4:2:2 layouts)
    bool ready = false;
};
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

// Byte offsets inside the scratch array.  Word 0 is the work counter, word 1
// the device error word; the progress words follow at byte 256.
struct NoAllocLayout {
    uint64_t ready, pic, prefix, items, res, snap, need;
};

NoAllocLayout noalloc_layout(const hpvcd_picture& p, const Geo& g) {
    NoAllocLayout L;
    const uint64_t n_ctu = (uint64_t)g.ctb_cols * g.ctb_rows;
    L.ready = 256;
    L.pic = align_up(L.ready + n_ctu * 16, 256);  // four progress words per CTU
    L.prefix = align_up(L.pic + sizeof(DevPic), 256);
    L.items = L.prefix + 256;
    L.res = align_up(L.items + n_ctu * sizeof(CtuItem), 256);
    L.snap = L.res + res_plane_bytes(g);
    L.need = L.snap + (sao_active(p) ? align_up(g.luma_bytes, 256) + 2 * align_up(g.chroma_bytes, 256) : 0);
    return L;
}

// Once per device, with that device current: the array's device address, the
// SM count and the k_recon shared-memory limit / occupancy.  None of these
// calls allocates.
hpvcd_status noalloc_setup(int dev, NoAllocDevice** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (!d.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e);
        e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return cuda_status(e);
        for (int f = 0; f < 3; ++f) d.occ[f] = std::max(1, hpvcd_recon_occupancy(f, 1));
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_status(e);
        d.base = (unsigned char*)p;
        d.ready = true;
    }
    *out = &d;
    return HPVCD_OK;
}

// Zero the counter, error word and progress words; store the picture record and
// the TB-record prefix; write the CTU work list in wavefront order (sorted by
// t = x + 2y, then y), the order in which every CTU's left, above-left, above
// and above-right neighbours come earlier.
__global__ void k_noalloc_setup(DevPic pic, uint32_t n_tus, unsigned char* base, NoAllocLayout L, int list) {
    const int cols = pic.ctb_cols, rows = pic.ctb_rows;
    const int n_ctu = cols * rows;
    uint32_t* words = (uint32_t*)base;
    uint32_t* ready = (uint32_t*)(base + L.ready);
    CtuItem* items = (CtuItem*)(base + L.items);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid < 2) words[tid] = 0u;
    if (tid == 0) {
        *(DevPic*)(base + L.pic) = pic;
        uint32_t* prefix = (uint32_t*)(base + L.prefix);
        prefix[0] = 0u;
        prefix[1] = n_tus;
    }
    for (int i = tid; i < n_ctu; i += gridDim.x * blockDim.x) {
        for (int c = 0; c < 4; ++c) ready[(size_t)i * 4 + c] = 0u;
        if (!list) continue;
        const int x = i % cols, y = i / cols, t = x + 2 * y;
        uint32_t rank = 0;
        for (int yy = 0; yy < rows && 2 * yy <= t; ++yy) {
            const int run = t - 2 * yy;  // cells of row yy with x' + 2yy < t
            rank += (uint32_t)(run < cols ? run : cols);
            if (yy < y && run < cols) ++rank;  // row yy holds a cell of this t before row y
        }
        items[rank] = CtuItem{0u, (uint16_t)x, (uint16_t)y};
    }
}

}  // namespace

HPVCD_API hpvcd_status hpvcd_decode_noalloc(const hpvcd_picture* dev_pic, void* const planes[3],
                                            uint32_t* dev_status, void* stream) {
    if (!dev_pic || !planes) return HPVCD_ERR_INVALID_ARG;
    const hpvcd_picture& p = *dev_pic;
    hpvcd_status s = validate(p);
    if (s != HPVCD_OK) return s;
    if (p.flags & HPVCD_PIC_INTER) {
        std::snprintf(t_last_error, sizeof(t_last_error),
                      "hpvcd_decode_noalloc: inter pictures predict from other pictures of one launch; "
                      "decode them with a plan");
        return HPVCD_ERR_UNSUPPORTED;
    }
    if (p.flags & HPVCD_PIC_STORE_MASK) {
        std::snprintf(t_last_error, sizeof(t_last_error),
                      "hpvcd_decode_noalloc: decoded-picture buffer stores belong to a context's submits; the "
                      "picture's planes are the caller's here");
        return HPVCD_ERR_UNSUPPORTED;
    }
    const int n_comp = p.chroma_idc ? 3 : 1;
    for (int c = 0; c < n_comp; ++c)
        if (!planes[c] || ((uintptr_t)planes[c] & 255)) {
            std::snprintf(t_last_error, sizeof(t_last_error),
                          "hpvcd_decode_noalloc: output plane %d is NULL or not 256-byte aligned", c);
            return HPVCD_ERR_INVALID_ARG;
        }
    const Geo g = geo_of(p);
    const NoAllocLayout L = noalloc_layout(p, g);
    if (L.need > kNoAllocScratchBytes) {
        std::snprintf(t_last_error, sizeof(t_last_error),
                      "hpvcd_decode_noalloc: a %ux%u picture needs %llu bytes of scratch, the fixed array holds "
                      "%llu (every picture up to 1024x1024 fits)",
                      p.width, p.height, (unsigned long long)L.need, (unsigned long long)kNoAllocScratchBytes);
        return HPVCD_ERR_LIMIT;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        std::snprintf(t_last_error, sizeof(t_last_error),
                      "hpvcd_decode_noalloc: device %d is beyond the %d devices this entry point serves", dev,
                      kNoAllocMaxDevices);
        return HPVCD_ERR_LIMIT;
    }
    NoAllocDevice* nd = nullptr;
    s = noalloc_setup(dev, &nd);
    if (s != HPVCD_OK) return s;
    unsigned char* base = nd->base;

    // device picture record (the fields plan_build fills for a YUV output)
    DevPic d;
    std::memset(&d, 0, sizeof(d));
    d.w = g.w; d.h = g.h; d.cw = g.cw; d.ch = g.ch; d.gw = g.gw; d.gh = g.gh;
    d.idc = p.chroma_idc; d.sub_w = g.sub_w; d.sub_h = g.sub_h;
    d.bd = p.bit_depth_y; d.bd_c = p.bit_depth_c; d.bps = g.bps;
    d.log2_ctb = p.log2_ctb; d.ctb_cols = g.ctb_cols; d.ctb_rows = g.ctb_rows;
    d.flags = p.flags;
    d.beta_offset_div2 = p.beta_offset_div2;
    d.tc_offset_div2 = p.tc_offset_div2;
    d.pps_cb_qp_offset = p.pps_cb_qp_offset;
    d.pps_cr_qp_offset = p.pps_cr_qp_offset;
    fill_inputs(d, p);
    for (int l = 0; l < 2; ++l)
        for (int r = 0; r < HPVCD_MAX_REFS; ++r) d.ref_pic[l][r] = -1;
    for (int c = 0; c < 3; ++c) d.fin[c] = c < n_comp ? planes[c] : nullptr;
    if (sao_active(p)) {
        unsigned char* sb = base + L.snap;
        d.rec[0] = sb;
        d.rec[1] = p.chroma_idc ? sb + align_up(g.luma_bytes, 256) : nullptr;
        d.rec[2] = p.chroma_idc ? sb + align_up(g.luma_bytes, 256) + align_up(g.chroma_bytes, 256) : nullptr;
    } else {
        for (int c = 0; c < 3; ++c) d.rec[c] = d.fin[c];
    }
    {
        unsigned char* rb = base + L.res;
        d.res_stride[0] = res_stride_of(g.w);
        d.res_stride[1] = d.res_stride[2] = res_stride_of(g.cw);
        const size_t ly = align_up((size_t)d.res_stride[0] * g.h * 2, 256);
        const size_t lc = align_up((size_t)d.res_stride[1] * g.ch * 2, 256);
        d.res[0] = (int16_t*)rb;
        d.res[1] = p.chroma_idc ? (int16_t*)(rb + ly) : nullptr;
        d.res[2] = p.chroma_idc ? (int16_t*)(rb + ly + lc) : nullptr;
    }
    d.ready = (uint32_t*)(base + L.ready);
    d.needs_wavefront = (p.flags & HPVCD_PIC_PRED_IN_PLANE) ? 0 : 1;

    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t n_ctu = (uint32_t)g.ctb_cols * g.ctb_rows;
    const DevPic* dp = (const DevPic*)(base + L.pic);
    uint32_t* work_counter = (uint32_t*)base;
    uint32_t* d_err = work_counter + 1;
    const int setup_blocks = (int)std::min<uint32_t>((n_ctu + 255) / 256, (uint32_t)nd->sms);
    k_noalloc_setup<<<std::max(1, setup_blocks), 256, 0, st>>>(d, p.n_tus, base, L, d.needs_wavefront);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e);
    hpvcd_note_launches(1);
    if (p.flags & HPVCD_PIC_PRED_IN_PLANE)
        for (int c = 0; c < n_comp; ++c) {
            if (!p.pred[c]) continue;
            e = cudaMemcpyAsync(d.rec[c], p.pred[c], c ? g.chroma_bytes : g.luma_bytes, cudaMemcpyDeviceToDevice,
                                st);
            if (e != cudaSuccess) return cuda_status(e);
        }
    const uint32_t* prefix = (const uint32_t*)(base + L.prefix);
    e = hpvcd_launch_residual(dp, prefix, 1, p.n_tus, d_err, nd->sms, 0, st);
    if (e == cudaSuccess && (p.flags & HPVCD_PIC_CROSS_COMPONENT) && p.n_tus)
        e = hpvcd_launch_ccp(dp, prefix, 1, p.n_tus, d_err, nd->sms, st);
    if (e != cudaSuccess) return cuda_status(e);
    if (d.needs_wavefront) {
        const int cfmt = p.chroma_idc == 3 ? 1 : (p.chroma_idc == 2 ? 2 : 0);
        const int grid = std::max(1, std::min<int>(nd->sms * nd->occ[cfmt], (int)n_ctu));
        e = hpvcd_launch_recon(dp, (const CtuItem*)(base + L.items), n_ctu, work_counter, d_err, cfmt, grid, 1,
                               (p.ctb_region || (p.flags & (HPVCD_PIC_CONSTRAINED_INTRA | HPVCD_PIC_CROSS_COMPONENT |
                                                           HPVCD_PIC_PCM))) ? 1 : 0,
                               1, 0, st);
        if (e != cudaSuccess) return cuda_status(e);
    }
    const int lv = (d.w >= 12 ? (d.w - 4) / 8 : 0) * (d.h / 4);
    const int lh = (d.h >= 12 ? (d.h - 4) / 8 : 0) * (d.w / 4);
    const int cv = d.idc ? (d.cw >= 10 ? (d.cw - 2) / 8 : 0) * (d.ch / 4) : 0;
    const int ch = d.idc ? (d.ch >= 10 ? (d.ch - 2) / 8 : 0) * (d.cw / 4) : 0;
    e = hpvcd_launch_deblock(dp, 1, std::max(lv, cv), 1, st);
    if (e == cudaSuccess) e = hpvcd_launch_deblock(dp, 1, std::max(lh, ch), 0, st);
    if (e == cudaSuccess && sao_active(p))
        e = hpvcd_launch_sao(dp, 1, d.w * d.h,
                             p.ctb_region && (p.flags & (HPVCD_PIC_SAO_NO_ACROSS_SLICES | HPVCD_PIC_SAO_NO_ACROSS_TILES)),
                             st);
    if (e == cudaSuccess && dev_status)
        e = cudaMemcpyAsync(dev_status, d_err, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    return cuda_status(e);
}
