"""Schedule selection: exhaustive autotuning and the learned selector.

The schedule of a batch (include/hpvcd_gpu.h `hpvcd_sched`) picks kernel
variants that never change pixels: the inverse transform of 16x16 / 32x32 TBs
in k_residual (integer tensor-core products, or even-odd butterflies), the
chroma warps of the wavefront kernel k_recon (one warp per chroma component
in a CTA of three, or one warp walking Cb then Cr in a CTA of two) and the
persistent k_recon CTAs per SM (occupancy maximum, or one).  Which is fastest depends on the batch: its TB-size mix,
coefficient density, QP, intra share, size and picture count.

* Exhaustive autotuning (`hpvcd_plan_autotune`) times every schedule on the
  batch itself: always right, but K decodes' worth of time.
* The selector network (`hpvcd_mlp_*`, 16 -> 64 -> 64 -> K, bf16 weights,
  fp32 accumulation, forward / backward / Adam as CUDA kernels in
  csrc/selector.cu) predicts log(t_k / t_best) for every schedule from the
  batch's 16 features (`hpvcd_plan_features`, computed on the device from the
  TB / PU records) and picks the argmin.  It is trained on timings that the
  autotuner measures, and autotuning stays the fallback (no network) and the
  yardstick (its timings score the network's picks).

Frames of the selector workload: 3840x2160 10-bit 4:2:0, QP uniform 17-42,
TB-size area mix Dirichlet(1, 1, 1, 1) over 4/8/16/32, coded-block fraction
5-60 %, 30 % intra frames and 70 % inter frames (intra-CU share 0-30 %, MV
standard deviation 1-32 luma samples, 40 % bi-prediction, 10 % explicit
weighted prediction), all seeded synthetic.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import abi, synth

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS_PATH = os.path.join(HERE, "selector_weights.npz")

# The candidate schedules, in output order of the network.
SCHEDULES = [abi.Sched(idct, cw, ctas, 0) for idct in (0, 1) for cw in (0, 1) for ctas in (0, 1)]
DEFAULT = 0  # (tensor-core transform, a warp per chroma component, occupancy maximum): the all-zero schedule
K = len(SCHEDULES)


def schedules_array():
    return (abi.Sched * K)(*SCHEDULES)


def _torch():
    import torch
    return torch


def _check(rc, what):
    abi.check(rc, what)


class Mlp:
    """The selector network on the GPU (hpvcd_mlp_*)."""

    def __init__(self, n_variants: int = K, seed: int = 1, device: int = 0):
        self.torch = _torch()
        self.dev = self.torch.device("cuda", device)
        self._L = abi.lib()
        h = C.c_void_p()
        _check(self._L.hpvcd_mlp_create(n_variants, seed, C.byref(h)), "hpvcd_mlp_create")
        self._h = h
        self.K = n_variants
        self.P = self._L.hpvcd_mlp_param_count(h)

    @property
    def handle(self):
        return self._h

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def _dev(self, a, width):
        t = self.torch.as_tensor(np.ascontiguousarray(a, np.float32).reshape(-1, width), device=self.dev)
        return t.contiguous()

    def params(self, master: bool = False) -> np.ndarray:
        out = np.empty(self.P, np.float32)
        _check(self._L.hpvcd_mlp_get_params(self._h, out.ctypes.data_as(C.c_void_p), int(master)),
               "hpvcd_mlp_get_params")
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.P
        _check(self._L.hpvcd_mlp_set_params(self._h, p.ctypes.data_as(C.c_void_p)), "hpvcd_mlp_set_params")

    def forward(self, x: np.ndarray) -> np.ndarray:
        X = self._dev(x, abi.FEATURES)
        Y = self.torch.empty((X.shape[0], self.K), dtype=self.torch.float32, device=self.dev)
        _check(self._L.hpvcd_mlp_forward(self._h, C.c_void_p(X.data_ptr()), X.shape[0], C.c_void_p(Y.data_ptr()),
                                         self._stream()), "hpvcd_mlp_forward")
        return Y.cpu().numpy()

    def grad(self, x: np.ndarray, t: np.ndarray):
        X = self._dev(x, abi.FEATURES)
        T = self._dev(t, self.K)
        G = self.torch.empty(self.P, dtype=self.torch.float32, device=self.dev)
        Lo = self.torch.empty(1, dtype=self.torch.float32, device=self.dev)
        _check(self._L.hpvcd_mlp_grad(self._h, C.c_void_p(X.data_ptr()), C.c_void_p(T.data_ptr()), X.shape[0],
                                      C.c_void_p(G.data_ptr()), C.c_void_p(Lo.data_ptr()), self._stream()),
               "hpvcd_mlp_grad")
        return float(Lo.item()), G.cpu().numpy()

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int = 200, batch: int = 256, lr: float = 2e-3,
              seed: int = 7) -> float:
        X = self._dev(x, abi.FEATURES)
        T = self._dev(t, self.K)
        loss = C.c_float()
        _check(self._L.hpvcd_mlp_train(self._h, C.c_void_p(X.data_ptr()), C.c_void_p(T.data_ptr()), X.shape[0],
                                       batch, epochs, lr, seed, self._stream(), C.byref(loss)), "hpvcd_mlp_train")
        return loss.value

    def pick(self, x: np.ndarray) -> np.ndarray:
        X = self._dev(x, abi.FEATURES)
        out = np.empty(X.shape[0], np.uint32)
        _check(self._L.hpvcd_mlp_pick(self._h, C.c_void_p(X.data_ptr()), X.shape[0], self._stream(),
                                      out.ctypes.data_as(C.POINTER(C.c_uint32))), "hpvcd_mlp_pick")
        return out

    def set_domain(self, lo: np.ndarray | None, hi: np.ndarray | None) -> None:
        """Feature range the network was trained on; batches outside it keep
        the default schedule (HPVCD_MLP_NO_PICK)."""
        self.domain = None if lo is None else (np.asarray(lo, np.float32), np.asarray(hi, np.float32))
        if lo is None:
            _check(self._L.hpvcd_mlp_set_domain(self._h, None, None), "hpvcd_mlp_set_domain")
        else:
            lo_, hi_ = (np.ascontiguousarray(a, np.float32) for a in self.domain)
            _check(self._L.hpvcd_mlp_set_domain(self._h, lo_.ctypes.data_as(C.c_void_p),
                                                hi_.ctypes.data_as(C.c_void_p)), "hpvcd_mlp_set_domain")

    def save(self, path: str = WEIGHTS_PATH) -> None:
        extra = {}
        if getattr(self, "domain", None) is not None:
            extra = {"domain_lo": self.domain[0], "domain_hi": self.domain[1]}
        np.savez(path, params=self.params(master=True), n_variants=self.K,
                 schedules=np.array([[s.idct, s.chroma_warps, s.recon_ctas_per_sm] for s in SCHEDULES], np.int32),
                 **extra)

    @classmethod
    def load(cls, path: str = WEIGHTS_PATH, device: int = 0) -> "Mlp":
        z = np.load(path)
        m = cls(int(z["n_variants"]), device=device)
        m.set_params(z["params"])
        if "domain_lo" in z:
            m.set_domain(z["domain_lo"], z["domain_hi"])
        return m

    def close(self):
        if getattr(self, "_h", None):
            self._L.hpvcd_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Targets and scoring
# ---------------------------------------------------------------------------

def targets(ms: np.ndarray) -> np.ndarray:
    """Network targets: log(t_k / t_best) per row of measured times."""
    ms = np.asarray(ms, np.float64)
    return np.log(ms / ms.min(axis=1, keepdims=True)).astype(np.float32)


def score(picks: np.ndarray, ms: np.ndarray) -> dict:
    """Decode time achieved by a pick per frame against the autotuned optimum
    and the fixed default schedule (all from measured times)."""
    ms = np.asarray(ms, np.float64)
    n = len(ms)
    best = ms.min(axis=1)
    chosen = ms[np.arange(n), np.asarray(picks)]
    default = ms[:, DEFAULT]
    return {
        "frames": int(n),
        "pick_accuracy": float(np.mean(np.asarray(picks) == ms.argmin(axis=1))),
        "within_1pct": float(np.mean(chosen <= best * 1.01)),
        "ms_selected": float(chosen.mean()),
        "ms_exhaustive": float(best.mean()),
        "ms_default": float(default.mean()),
        "gain_vs_default": float(default.sum() / chosen.sum() - 1.0),
        "regret_vs_exhaustive": float(chosen.sum() / best.sum() - 1.0),
    }


def best_fixed(ms: np.ndarray) -> int:
    """The single schedule with the lowest total time (the best the method
    without a network can do without timing each batch)."""
    return int(np.asarray(ms).sum(axis=0).argmin())


# ---------------------------------------------------------------------------
# Selector-workload frames and their measurement
# ---------------------------------------------------------------------------

@dataclass
class FrameSpec:
    seed: int
    intra: bool
    qp: int
    tu_mix: tuple
    cbf: float
    intra_cu: float
    mv_sd: float
    bi: float
    weighted: bool


def frame_specs(n: int, seed: int = 0) -> list[FrameSpec]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        mix = tuple(float(v) for v in rng.dirichlet([1.0, 1.0, 1.0, 1.0]))
        out.append(FrameSpec(seed=seed * 1_000_003 + i, intra=bool(rng.random() < 0.3),
                             qp=int(rng.integers(17, 43)), tu_mix=mix, cbf=float(rng.uniform(0.05, 0.6)),
                             intra_cu=float(rng.uniform(0.0, 0.3)), mv_sd=float(rng.uniform(1.0, 32.0)),
                             bi=0.4, weighted=bool(rng.random() < 0.1)))
    return out


W4K, H4K = 3840, 2160


def _frame_cfg(sp: FrameSpec, w=W4K, h=H4K) -> abi.SynthCfg:
    if sp.intra:
        c = synth.intra_cfg(sp.seed, w, h, bit_depth=10, chroma_idc=1)
    else:
        c = synth.inter_cfg(sp.seed, w, h, bit_depth=10, weighted=sp.weighted, n_refs=2,
                            intra_cu_p=sp.intra_cu, bi_p=sp.bi)
        c.mv_sd = sp.mv_sd
    c.qp_min, c.qp_max = sp.qp, min(sp.qp + 2, 51)
    c.cbf_p = sp.cbf
    c.cu_split_p = 0.25
    for k in range(4):
        c.tu_mix[k] = sp.tu_mix[k]
    return c


class RefPictures:
    """Two reference pictures for the inter frames: prediction-in-plane
    pictures with no TB records, so decoding them is only the copy of their
    planes.  Uploaded once (`resident` maps plan indices 0 and 1 to their
    device descriptors)."""

    def __init__(self, w=W4K, h=H4K, seed=99, upload: bool = True):
        self.synth = synth.SynthSet()
        for r in range(2):
            c = synth.residual_cfg(seed + r, w, h, bit_depth=10, chroma_idc=1)
            c.tu_split_p = 0.0
            self.synth.add(c)
        self.pics = []
        for p in self.synth.pictures():
            q = abi.Picture()
            C.pointer(q)[0] = p
            q.n_tus = 0
            q.n_coeffs = 0
            self.pics.append(q)
        self.resident = None
        self._plan = None
        if upload:
            from .gpu import DevicePlan
            self._plan = DevicePlan(self.pics)  # owns the device copies
            self.resident = {0: self._plan.dev_pics[0], 1: self._plan.dev_pics[1]}


def build_frame(sp: FrameSpec, refs: RefPictures | None, w=W4K, h=H4K):
    """Returns (keep-alive SynthSet, pictures of the plan, index of the frame)."""
    s = synth.SynthSet()
    if sp.intra:
        s.add(_frame_cfg(sp, w, h))
        return s, [s.picture(0)], 0
    for r in range(2):  # placeholders so the frame's reference slots are 1 and 0
        s.add(synth.residual_cfg(1 + r, 64, 64, bit_depth=10))
    s.add(_frame_cfg(sp, w, h))
    return s, [refs.pics[0], refs.pics[1], s.picture(2)], 2


def measure(plan, frame_index: int, reps: int = 2, stages: int = abi.STAGE_ALL):
    """Features of the frame and the autotuner's time of every schedule."""
    return measure_range(plan, frame_index, 1, reps, stages)


def measure_range(plan, first: int, count: int, reps: int = 2, stages: int = abi.STAGE_ALL):
    """Features of pictures [first, first + count) and the autotuner's time of
    every schedule for the whole plan."""
    torch = _torch()
    L = abi.lib()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    f = torch.empty(abi.FEATURES, dtype=torch.float32, device="cuda")
    _check(L.hpvcd_plan_features(plan._h, first, count, C.c_void_p(f.data_ptr()), st), "hpvcd_plan_features")
    ms = (C.c_float * K)()
    best = C.c_uint32()
    _check(L.hpvcd_plan_autotune(plan._h, schedules_array(), K, stages, reps, 0, st, ms, C.byref(best)),
           "hpvcd_plan_autotune")
    _check(plan.status(), "device status")
    return f.cpu().numpy(), np.array(ms[:], np.float32)


def collect(n_frames: int, seed: int = 0, out_path: str | None = None, threads: int = 8, reps: int = 2,
            log_every: int = 100, start: int = 0):
    """Generate, decode and time `n_frames` selector-workload frames; returns
    (features [n][16], ms [n][K]).  Frames are generated on `threads` host
    threads while the GPU measures earlier ones."""
    from concurrent.futures import ThreadPoolExecutor

    from .gpu import DevicePlan

    specs = frame_specs(start + n_frames, seed)[start:]
    refs = RefPictures()
    X = np.zeros((n_frames, abi.FEATURES), np.float32)
    T = np.zeros((n_frames, K), np.float32)
    done = 0
    with ThreadPoolExecutor(threads) as pool:
        futs = [pool.submit(build_frame, sp, refs) for sp in specs[:threads * 2]]
        nxt = len(futs)
        for i in range(n_frames):
            keep, pics, fi = futs[i].result()
            futs[i] = None
            if nxt < n_frames:
                futs.append(pool.submit(build_frame, specs[nxt], refs))
                nxt += 1
            plan = DevicePlan(pics, resident=refs.resident if fi else None)
            X[i], T[i] = measure(plan, fi, reps=reps)
            plan.close()
            del keep
            done = i + 1
            if out_path and (done % log_every == 0 or done == n_frames):
                np.savez(out_path, features=X[:done], ms=T[:done], seed=seed, start=start)
                print(f"[selector] {done}/{n_frames} frames", flush=True)
    return X[:done], T[:done]


def collect_batches(n_batches: int, seed: int = 0, out_path: str | None = None, threads: int = 4,
                    reps: int = 2, max_images: int = 64, log_every: int = 50, start: int = 0):
    """Serving batches as the selector sees them: 1..max_images images of
    the mixed-size serving workload (serving.make_images) fused into one
    plan with one RGB8 canvas per image; features over all pictures and the
    autotuner's time of every schedule.  Returns (features, ms)."""
    from concurrent.futures import ThreadPoolExecutor

    from . import serving
    from .gpu import DevicePlan

    rng = np.random.default_rng(seed)
    counts = rng.integers(1, max_images + 1, size=start + n_batches)[start:]

    def make(i):
        keep, imgs = serving.make_images(int(counts[i]), seed=seed * 100_003 + start + i)
        return keep, imgs

    X = np.zeros((n_batches, abi.FEATURES), np.float32)
    T = np.zeros((n_batches, K), np.float32)
    with ThreadPoolExecutor(threads) as pool:
        futs = [pool.submit(make, i) for i in range(min(threads, n_batches))]
        nxt = len(futs)
        for i in range(n_batches):
            keep, imgs = futs[i].result()
            futs[i] = None
            if nxt < n_batches:
                futs.append(pool.submit(make, nxt))
                nxt += 1
            pics, out, okeep = serving.fused_output(imgs)
            plan = DevicePlan(pics, out)
            f, ms = measure_range(plan, 0, len(pics), reps=reps)
            X[i], T[i] = f, ms
            plan.close()
            del keep, imgs, okeep
            if out_path and ((i + 1) % log_every == 0 or i + 1 == n_batches):
                np.savez(out_path, features=X[:i + 1], ms=T[:i + 1], seed=seed, start=start)
                print(f"[selector] {i + 1}/{n_batches} batches", flush=True)
    return X, T


# Photo sizes of grid-coded stills (HEIC): 12 MP in both orientations,
# 4:3 and 16:9 crops, 48 MP and 8 MP.
GRID_SIZES = [(4032, 3024), (3024, 4032), (4000, 3000), (4032, 2268), (8064, 6048), (3264, 2448)]


def collect_grids(n_grids: int, seed: int = 2, out_path: str | None = None, threads: int = 4,
                  reps: int = 2, log_every: int = 25, start: int = 0):
    """Grid-coded stills as the selector sees them: one photo (GRID_SIZES,
    10-bit in 3 of 4, else 8-bit; 4:2:0) split into 512x512 tiles, int8
    level pools where every level fits, decoded to an RGB8 canvas only;
    features over its tiles and the autotuner's time of every schedule.
    Returns (features, ms)."""
    from concurrent.futures import ThreadPoolExecutor

    from . import synth
    from .gpu import DevicePlan

    rng = np.random.default_rng(seed)
    specs = [(GRID_SIZES[int(rng.integers(len(GRID_SIZES)))], 8 if rng.random() < 0.25 else 10)
             for _ in range(start + n_grids)][start:]

    def make(i):
        (w, h), bd = specs[i]
        g = synth.make_grid(w, h, seed=seed * 100_019 + start + i, bit_depth=bd, chroma_idc=1)
        pics = g.synth.pictures()
        return g, pics, synth.narrow_coeffs(pics)

    X = np.zeros((n_grids, abi.FEATURES), np.float32)
    T = np.zeros((n_grids, K), np.float32)
    with ThreadPoolExecutor(threads) as pool:
        futs = [pool.submit(make, i) for i in range(min(threads, n_grids))]
        nxt = len(futs)
        for i in range(n_grids):
            g, pics, c8 = futs[i].result()
            futs[i] = None
            if nxt < n_grids:
                futs.append(pool.submit(make, nxt))
                nxt += 1
            out, okeep = synth.grid_output(g)
            out.options = abi.OUTPUT_CANVAS_ONLY
            plan = DevicePlan(pics, out)
            X[i], T[i] = measure_range(plan, 0, len(pics), reps=reps)
            plan.close()
            del g, pics, c8, okeep
            if out_path and ((i + 1) % log_every == 0 or i + 1 == n_grids):
                np.savez(out_path, features=X[:i + 1], ms=T[:i + 1], seed=seed, start=start)
                print(f"[selector] {i + 1}/{n_grids} grids", flush=True)
    return X, T


# ---------------------------------------------------------------------------
# Training and evaluation
# ---------------------------------------------------------------------------

def feature_domain(x: np.ndarray, margin: float = 0.05):
    """Per-feature [lo, hi] of the training rows, widened by `margin` of the
    range (at least 0.01)."""
    lo, hi = x.min(axis=0), x.max(axis=0)
    pad = np.maximum((hi - lo) * margin, 0.01)
    return (lo - pad).astype(np.float32), (hi + pad).astype(np.float32)


def train_network(x: np.ndarray, ms: np.ndarray, epochs: int = 200, batch: int = 256, lr: float = 2e-3,
                  seed: int = 1) -> Mlp:
    """Train the selector network on the GPU (hpvcd_mlp_train) on features
    and autotuner timings; its domain is the training rows' feature range."""
    m = Mlp(K, seed=seed)
    m.train(x, targets(ms), epochs=epochs, batch=batch, lr=lr, seed=seed + 1)
    m.set_domain(*feature_domain(x))
    return m


def score_with_fallback(picks: np.ndarray, ms: np.ndarray) -> dict:
    """score() where a pick outside the domain (MLP_NO_PICK) runs the default."""
    p = np.where(np.asarray(picks) == abi.MLP_NO_PICK, DEFAULT, np.asarray(picks)).astype(np.int64)
    r = score(p, ms)
    r["outside_domain"] = int(np.sum(np.asarray(picks) == abi.MLP_NO_PICK))
    return r


def evaluate_live(mlp: Mlp, n_frames: int, seed: int = 12345, reps: int = 2, log=None) -> dict:
    """Fresh frames (a seed never trained on): the network's pick, the
    default schedule and exhaustive autotuning, all timed on the GPU.  Also
    the cost of choosing (features + network forward, including the read of
    the pick by the host)."""
    import torch

    from .gpu import DevicePlan

    L = abi.lib()
    specs = frame_specs(n_frames, seed)
    refs = RefPictures()
    times, picks, choose_ms = [], [], []
    st = torch.cuda.current_stream()
    for i, sp in enumerate(specs):
        keep, pics, fi = build_frame(sp, refs)
        plan = DevicePlan(pics, resident=refs.resident if fi else None)
        _, ms = measure(plan, fi, reps=reps)
        fdev = torch.empty(abi.FEATURES, dtype=torch.float32, device="cuda")
        out = np.empty(1, np.uint32)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        _check(L.hpvcd_plan_features(plan._h, fi, 1, C.c_void_p(fdev.data_ptr()), C.c_void_p(st.cuda_stream)),
               "hpvcd_plan_features")
        _check(L.hpvcd_mlp_pick(mlp.handle, C.c_void_p(fdev.data_ptr()), 1, C.c_void_p(st.cuda_stream),
                                out.ctypes.data_as(C.POINTER(C.c_uint32))), "hpvcd_mlp_pick")
        t1.record()
        torch.cuda.synchronize()
        choose_ms.append(t0.elapsed_time(t1))
        plan.close()
        del keep
        times.append(ms)
        picks.append(int(out[0]))
        if log and (i + 1) % 20 == 0:
            log(f"[selector] evaluated {i + 1}/{n_frames}")
    ms = np.array(times)
    r = score_with_fallback(np.array(picks), ms)
    r["choose_ms_mean"] = float(np.mean(choose_ms))
    r["seed"] = seed
    return r


def _main(argv=None):
    import argparse
    import json

    ap = argparse.ArgumentParser(description="selector data collection / training / evaluation")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--frames", type=int, required=True)
    c.add_argument("--start", type=int, default=0)
    c.add_argument("--seed", type=int, default=0)
    c.add_argument("--out", required=True)
    c.add_argument("--threads", type=int, default=8)
    b = sub.add_parser("collect-batches")
    b.add_argument("--batches", type=int, required=True)
    b.add_argument("--start", type=int, default=0)
    b.add_argument("--seed", type=int, default=1)
    b.add_argument("--out", required=True)
    b.add_argument("--threads", type=int, default=4)
    gq = sub.add_parser("collect-grids")
    gq.add_argument("--grids", type=int, required=True)
    gq.add_argument("--start", type=int, default=0)
    gq.add_argument("--seed", type=int, default=2)
    gq.add_argument("--out", required=True)
    gq.add_argument("--threads", type=int, default=4)
    t = sub.add_parser("train")
    t.add_argument("--data", nargs="+", required=True)
    t.add_argument("--holdout", type=float, default=0.2)
    t.add_argument("--epochs", type=int, default=200)
    t.add_argument("--out", default=WEIGHTS_PATH)
    t.add_argument("--merged", default=None, help="write the merged data set with its train / held-out split")
    e = sub.add_parser("evaluate")
    e.add_argument("--frames", type=int, default=100)
    e.add_argument("--seed", type=int, default=12345)
    a = ap.parse_args(argv)
    if a.cmd == "collect":
        collect(a.frames, seed=a.seed, out_path=a.out, threads=a.threads, start=a.start)
    elif a.cmd == "collect-batches":
        collect_batches(a.batches, seed=a.seed, out_path=a.out, threads=a.threads, start=a.start)
    elif a.cmd == "collect-grids":
        collect_grids(a.grids, seed=a.seed, out_path=a.out, threads=a.threads, start=a.start)
    elif a.cmd == "train":
        xs, ts = [], []
        for path in a.data:
            z = np.load(path)
            xs.append(z["features"])
            ts.append(z["ms"])
        x = np.concatenate(xs)
        ms = np.concatenate(ts)
        keep = np.all(ms > 0, axis=1)
        x, ms = x[keep], ms[keep]
        perm = np.random.default_rng(2024).permutation(len(x))  # frames and batches in both splits
        x, ms = x[perm], ms[perm]
        split = int(round(len(x) * (1 - a.holdout)))
        m = train_network(x[:split], ms[:split], epochs=a.epochs)
        picks = m.pick(x[split:])
        fixed = best_fixed(ms[:split])
        hx, hms = x[split:], ms[split:]
        is_batch = hx[:, 1] > np.log2(3.0) / 8  # more than one picture
        res = {"train_rows": split, "heldout_rows": len(x) - split,
               "heldout": score_with_fallback(picks, hms),
               "heldout_frames": score_with_fallback(picks[~is_batch], hms[~is_batch]),
               "heldout_batches": score_with_fallback(picks[is_batch], hms[is_batch]) if is_batch.any() else None,
               "best_fixed": fixed, "best_fixed_heldout": score(np.full(len(hms), fixed), hms),
               "best_fixed_heldout_batches": (score(np.full(int(is_batch.sum()), fixed), hms[is_batch])
                                              if is_batch.any() else None)}
        print(json.dumps(res, indent=1))
        m.save(a.out)
        if a.merged:
            np.savez_compressed(a.merged, features=x.astype(np.float32), ms=ms.astype(np.float32),
                                train_rows=split)
    elif a.cmd == "evaluate":
        m = Mlp.load()
        print(json.dumps(evaluate_live(m, a.frames, a.seed, log=print), indent=1))


if __name__ == "__main__":
    _main()
