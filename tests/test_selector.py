"""Schedule selection: the selector network's CUDA kernels against the numpy
oracle (forward, loss, gradients), the device features against a host
restatement, autotuning / selection leaving pixels unchanged, and the gain
of the trained network over the method without it."""
from __future__ import annotations

import os

import numpy as np
import pytest

from hpvcd_b200 import abi, selector, synth
from oracle import mlp_ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TIMINGS = os.path.join(ROOT, "tests", "golden", "selector_timings.npz")


def _rand_params(K, seed):
    r = np.random.default_rng(seed)
    L = mlp_ref.layout(K)
    p = np.zeros(L["total"], np.float32)
    p[L["w1"]:L["b1"]] = r.normal(0, 0.4, L["b1"] - L["w1"])
    p[L["b1"]:L["w2"]] = r.normal(0, 0.1, L["w2"] - L["b1"])
    p[L["w2"]:L["b2"]] = r.normal(0, 0.15, L["b2"] - L["w2"])
    p[L["b2"]:L["w3"]] = r.normal(0, 0.1, L["w3"] - L["b2"])
    p[L["w3"]:L["b3"]] = r.normal(0, 0.15, L["b3"] - L["w3"])
    p[L["b3"]:] = r.normal(0, 0.1, L["total"] - L["b3"])
    return p


def features_host(pics) -> np.ndarray:
    """Host restatement of k_features / k_features_finish (selector.cu)."""
    area = bd = a444 = 0.0
    wave = 0
    tb = np.zeros(4)
    coded = intra = 0.0
    qps = []
    nx_sum = 0
    ncoded = 0
    npu = nmv = nbi = 0
    mv_sum = 0
    for p in pics:
        g = synth.geometry(p)
        a = p.width * p.height
        area += a
        bd += a * p.bit_depth_y
        a444 += a if p.chroma_idc == 3 else 0
        wave = max(wave, g["ctb_cols"] + 2 * g["ctb_rows"])
        t = synth.tus_of(p)
        m = (t["comp"] == 0) & (t["log2n"] >= 2) & (t["log2n"] <= 5)
        cb = (t["flags"] & abi.TU_CBF) != 0
        it = (t["flags"] & abi.TU_INTRA) != 0
        m &= cb | it
        ar = (1 << (2 * t["log2n"].astype(np.int64)))
        for z in range(4):
            tb[z] += ar[m & (t["log2n"] == z + 2)].sum()
        coded += ar[m & cb].sum()
        intra += ar[m & it].sum()
        qps.append(t["qp_y"][m].astype(np.int64) + 64)
        n = 1 << t["log2n"].astype(np.int64)
        nx = t["nx"].astype(np.int64)
        nx = np.where((nx == 0) | (nx > n), n, nx)
        nx_sum += (64 * nx // n)[m & cb].sum()
        ncoded += int((m & cb).sum())
        u = synth.pus_of(p)
        npu += len(u)
        for l in range(2):
            used = (u["flags"] & (1 << l)) != 0
            mv_sum += int(np.abs(u["mv"][used, l, :].astype(np.int64)).sum())
            nmv += int(used.sum())
        nbi += int(((u["flags"] & 3) == 3).sum())
    q = np.concatenate(qps) if qps else np.zeros(0)
    ntb = max(len(q), 1)
    qm = q.sum() / ntb
    qv = max((q.astype(np.float64) ** 2).sum() / ntb - qm * qm, 0.0)
    tbs = max(tb.sum(), 1.0)
    f = np.zeros(16)
    f[0] = np.log2(area) / 24
    f[1] = np.log2(1 + len(pics)) / 8
    f[2] = wave / 256
    f[3] = (bd / area - 8) / 4
    f[4] = a444 / area
    f[5:9] = tb / tbs
    f[9] = coded / area
    f[10] = intra / area
    f[11] = (qm - 64) / 51
    f[12] = np.sqrt(qv) / 16
    f[13] = nx_sum / max(ncoded, 1) / 64
    f[14] = np.log2(1 + mv_sum / max(nmv, 1) / 4) / 8
    f[15] = nbi / max(npu, 1)
    return f.astype(np.float32)


# ---------------------------------------------------------------------------
# CPU
# ---------------------------------------------------------------------------

def test_oracle_gradient_matches_finite_differences():
    K = 5
    p = _rand_params(K, 0).astype(np.float64)
    r = np.random.default_rng(1)
    x = r.random((7, 16))
    t = r.random((7, K))
    _, g = mlp_ref.loss_and_grad(p, x, t, K, dtype=np.float64)
    idx = r.choice(len(p), 60, replace=False)
    eps = 1e-6
    for i in idx:
        q = p.copy(); q[i] += eps
        lp = mlp_ref.loss(q, x, t, K, dtype=np.float64)
        q[i] -= 2 * eps
        lm = mlp_ref.loss(q, x, t, K, dtype=np.float64)
        assert abs((lp - lm) / (2 * eps) - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), i


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-3], np.float32)
    r = mlp_ref.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] + 3.140625) < 1e-6
    bits = r.view(np.uint32)
    assert np.all((bits & 0xFFFF) == 0)


def test_targets_and_score():
    ms = np.array([[10., 9., 12.], [5., 6., 5.5], [8., 8., 7.]])
    t = selector.targets(ms)
    assert np.allclose(t.min(axis=1), 0)
    s = selector.score(np.array([1, 0, 2]), ms)
    assert s["pick_accuracy"] == 1.0 and s["regret_vs_exhaustive"] == 0.0
    assert s["gain_vs_default"] > 0
    s0 = selector.score(np.zeros(3, int), ms)
    assert s0["gain_vs_default"] == 0.0
    assert selector.best_fixed(ms) in (0, 1, 2)


def test_frame_specs_follow_the_workload():
    sp = selector.frame_specs(2000, seed=3)
    qp = np.array([s.qp for s in sp])
    assert qp.min() >= 17 and qp.max() <= 42
    mix = np.array([s.tu_mix for s in sp])
    assert np.allclose(mix.sum(axis=1), 1.0)
    assert abs(mix.mean() - 0.25) < 0.02
    cbf = np.array([s.cbf for s in sp])
    assert cbf.min() >= 0.05 and cbf.max() <= 0.6
    assert 0.25 < np.mean([s.intra for s in sp]) < 0.35


def test_tu_mix_steers_tb_sizes():
    for mix, big in (((0.05, 0.05, 0.1, 0.8), True), ((0.8, 0.1, 0.05, 0.05), False)):
        s = synth.SynthSet()
        c = synth.intra_cfg(5, 512, 512, bit_depth=10)
        c.cu_split_p = 0.0
        for k in range(4):
            c.tu_mix[k] = mix[k]
        s.add(c)
        f = features_host(s.pictures())
        if big:
            assert f[8] > 0.6
        else:
            assert f[5] > 0.6


def test_host_batch_features_match_the_restatement():
    """hpvcd_batch_features (the submit path's host-side features) equals the
    restatement of k_features / k_features_finish on intra, inter and 4:4:4
    batches (no GPU needed)."""
    import ctypes as C
    L = abi.lib()
    s = synth.SynthSet()
    s.add(synth.intra_cfg(31, 512, 384, bit_depth=10, chroma_idc=1))
    c = synth.intra_cfg(32, 256, 256, bit_depth=8, chroma_idc=3, tskip_p=0.1)
    for k, v in enumerate((0.1, 0.2, 0.3, 0.4)):
        c.tu_mix[k] = v
    s.add(c)
    s.add(synth.intra_cfg(34, 256, 256, bit_depth=8, chroma_idc=1))
    s.add(synth.inter_cfg(33, 256, 256, weighted=True))
    pics = s.pictures()
    for first, count in ((0, 4), (3, 1), (1, 1), (0, 2)):
        arr = (abi.Picture * count)(*pics[first:first + count])
        f = (C.c_float * 16)()
        assert L.hpvcd_batch_features(arr, count, f) == abi.OK
        np.testing.assert_allclose(np.array(f), features_host(pics[first:first + count]), rtol=1e-6, atol=1e-7)


def test_trained_selector_gains_on_heldout_frames_cpu():
    """The committed network, evaluated with the numpy oracle forward pass on
    its bf16 weights over the held-out measured frames and batches: faster in
    total than the fixed default schedule (which is also the best single
    schedule of the training rows) and within 0.3 % of exhaustive
    autotuning."""
    if not (os.path.exists(TIMINGS) and os.path.exists(selector.WEIGHTS_PATH)):
        pytest.skip("no committed selector timings / weights")
    z = np.load(TIMINGS)
    x, ms, split = z["features"], z["ms"].astype(np.float64), int(z["train_rows"])
    w = np.load(selector.WEIGHTS_PATH)
    K = int(w["n_variants"])
    y, _, _ = mlp_ref.forward(mlp_ref.bf16_round(w["params"]), x[split:], K)
    picks = y.argmin(axis=1)
    if "domain_lo" in w:  # rows outside the training range keep the default schedule
        inside = np.all((x[split:] >= w["domain_lo"]) & (x[split:] <= w["domain_hi"]), axis=1)
        picks = np.where(inside, picks, abi.MLP_NO_PICK)
    s = selector.score_with_fallback(picks, ms[split:])
    fixed = selector.best_fixed(ms[:split])
    s_fixed = selector.score(np.full(len(ms) - split, fixed), ms[split:])
    # the default schedule is the best single one on these kernels (exhaustive
    # autotuning is 1.1 % ahead of it on the held-out rows): the network must
    # take most of that and never cost more than the default
    assert s["gain_vs_default"] > 0.007
    assert s["ms_selected"] <= s_fixed["ms_selected"]
    assert s["regret_vs_exhaustive"] < 0.003


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA GPU")
    return torch


@pytest.mark.gpu
def test_mlp_forward_matches_oracle():
    _gpu()
    m = selector.Mlp(selector.K)
    p = _rand_params(selector.K, 3)
    m.set_params(p)
    pb = m.params()                       # the bf16 values the kernel reads
    assert np.array_equal(pb, mlp_ref.bf16_round(p))
    assert np.array_equal(m.params(master=True), p)
    x = np.random.default_rng(4).random((37, 16)).astype(np.float32)
    y = m.forward(x)
    yr, _, _ = mlp_ref.forward(pb, x, selector.K)
    np.testing.assert_allclose(y, yr, rtol=1e-5, atol=1e-5)
    m.close()


@pytest.mark.gpu
def test_mlp_gradients_match_oracle():
    _gpu()
    K = selector.K
    m = selector.Mlp(K)
    p = _rand_params(K, 5)
    m.set_params(p)
    pb = m.params()
    r = np.random.default_rng(6)
    for B in (1, 16, 45, 300):
        x = r.random((B, 16)).astype(np.float32)
        t = r.random((B, K)).astype(np.float32)
        loss, g = m.grad(x, t)
        lr_, gr = mlp_ref.loss_and_grad(pb, x, t, K)
        assert abs(loss - lr_) <= 1e-5 * max(1.0, abs(lr_))
        # fp32 sums in a different order: relative 1e-4 of the largest entry
        np.testing.assert_allclose(g, gr, rtol=1e-4, atol=1e-4 * np.abs(gr).max())
    m.close()


@pytest.mark.gpu
def test_mlp_training_learns_a_crossover():
    """Synthetic costs with a crossover: variant 3 is fastest when feature 5
    (4x4 share) is high, variant 1 otherwise; the trained network must pick
    accordingly and beat the fixed default."""
    _gpu()
    K = selector.K
    r = np.random.default_rng(11)
    x = r.random((4000, 16)).astype(np.float32)
    base = 10 + 5 * x[:, 0:1]
    ms = np.repeat(base, K, axis=1) * 1.10
    small = x[:, 5] > 0.5
    ms[small, 3] = base[small, 0] * (1.0 - 0.1 * x[small, 5])
    ms[~small, 1] = base[~small, 0] * (1.0 - 0.05 * (1 - x[~small, 5]))
    ms[:, 0] = base[:, 0] * 1.02
    t = selector.targets(ms)
    m = selector.Mlp(K, seed=2)
    loss0, _ = m.grad(x[:512], t[:512])
    m.train(x[:3000], t[:3000], epochs=60, batch=256, lr=3e-3)
    loss1, _ = m.grad(x[:512], t[:512])
    assert loss1 < 0.2 * loss0
    picks = m.pick(x[3000:])
    s = selector.score(picks, ms[3000:])
    assert s["pick_accuracy"] > 0.9
    assert s["gain_vs_default"] > 0.05
    # the device picks equal argmin of the oracle forward on the bf16 weights
    yr, _, _ = mlp_ref.forward(m.params(), x[3000:], K)
    assert np.mean(yr.argmin(axis=1) == picks) > 0.99
    m.close()


@pytest.mark.gpu
def test_plan_features_match_host_restatement():
    torch = _gpu()
    import ctypes as C
    from hpvcd_b200.gpu import DevicePlan
    s = synth.SynthSet()
    s.add(synth.intra_cfg(31, 512, 384, bit_depth=10, chroma_idc=1))
    c = synth.intra_cfg(32, 256, 256, bit_depth=8, chroma_idc=3, tskip_p=0.1)
    for k, v in enumerate((0.1, 0.2, 0.3, 0.4)):
        c.tu_mix[k] = v
    s.add(c)
    s.add(synth.intra_cfg(34, 256, 256, bit_depth=8, chroma_idc=1))
    s.add(synth.inter_cfg(33, 256, 256, weighted=True, n_refs=1))
    pics = s.pictures()
    for l in range(2):            # the inter picture predicts from the one before only
        for r in range(1, abi.MAX_REFS):
            pics[3].ref_slot[l][r] = -1
    plan = DevicePlan(pics)
    L = abi.lib()
    f = torch.empty(16, dtype=torch.float32, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for first, count in ((0, 4), (3, 1), (1, 1)):
        abi.check(L.hpvcd_plan_features(plan._h, first, count, C.c_void_p(f.data_ptr()), st), "features")
        np.testing.assert_allclose(f.cpu().numpy(), features_host(pics[first:first + count]), rtol=1e-5, atol=1e-6)
    plan.close()


@pytest.mark.gpu
def test_autotune_and_selection_leave_pixels_unchanged():
    torch = _gpu()
    import ctypes as C
    from hpvcd_b200.gpu import DevicePlan
    from oracle import oracle as O
    s = synth.SynthSet()
    s.add(synth.intra_cfg(41, 512, 512, bit_depth=10))
    s.add(synth.intra_cfg(42, 320, 256, bit_depth=8, chroma_idc=3))
    pics = s.pictures()
    ref, _ = O.decode_batch(pics)
    plan = DevicePlan(pics)
    L = abi.lib()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    ms = (C.c_float * selector.K)()
    best = C.c_uint32()
    abi.check(L.hpvcd_plan_autotune(plan._h, selector.schedules_array(), selector.K, abi.STAGE_ALL, 2, 1, st, ms,
                                    C.byref(best)), "autotune")
    assert all(v > 0 for v in ms) and best.value == int(np.argmin(ms[:]))
    for mlp in (None, selector.Mlp(selector.K, seed=9)):
        chosen = C.c_uint32(99)
        abi.check(L.hpvcd_plan_select(plan._h, mlp.handle if mlp else None, selector.schedules_array(),
                                      selector.K, st, C.byref(chosen)), "select")
        assert chosen.value < selector.K
        plan.launch()
        assert plan.status() == abi.OK
        got = [plan.planes(i) for i in range(len(pics))]
        for g, r in zip(got, ref):
            for c in range(3):
                if r[c].size:
                    assert np.array_equal(g[c].astype(np.uint16), r[c])
    plan.close()


@pytest.mark.gpu
def test_trained_selector_gains_over_no_network():
    """Measured timings of held-out selector-workload frames (every schedule
    timed by the autotuner on a B200) scored against the committed network's
    picks: the network must beat the fixed default schedule and the best
    single schedule, and stay close to exhaustive autotuning."""
    _gpu()
    if not (os.path.exists(TIMINGS) and os.path.exists(selector.WEIGHTS_PATH)):
        pytest.skip("no committed selector timings / weights")
    z = np.load(TIMINGS)
    x, ms, split = z["features"], z["ms"].astype(np.float64), int(z["train_rows"])
    m = selector.Mlp.load()
    picks = m.pick(x[split:])
    s = selector.score_with_fallback(picks, ms[split:])
    fixed = selector.best_fixed(ms[:split])
    s_fixed = selector.score(np.full(len(ms) - split, fixed), ms[split:])
    # the default schedule is the best single one on these kernels (exhaustive
    # autotuning is 1.1 % ahead of it on the held-out rows): the network must
    # take most of that and never cost more than the default
    assert s["gain_vs_default"] > 0.007
    assert s["ms_selected"] <= s_fixed["ms_selected"]
    assert s["regret_vs_exhaustive"] < 0.003
    # the device picks are the oracle's argmin on the same bf16 weights
    y, _, _ = mlp_ref.forward(m.params(), x[split:], selector.K)
    inside = picks != abi.MLP_NO_PICK
    assert np.mean(y.argmin(axis=1)[inside] == picks[inside]) > 0.99
    m.close()


@pytest.mark.gpu
def test_server_with_selector_keeps_pixels():
    """Batches launched by the serving loop with the network choosing each
    batch's schedule decode exactly as the oracle does."""
    _gpu()
    from hpvcd_b200.gpu import Server
    from oracle import oracle as O
    s = synth.SynthSet()
    imgs = []
    for i, (w, h, bd, idc) in enumerate([(640, 448, 10, 1), (1024, 512, 8, 1), (512, 700, 8, 3), (256, 256, 10, 1)]):
        g = synth.make_grid(w, h, seed=300 + i, bit_depth=bd, chroma_idc=idc, synth=s)
        first = len(s) - g.cols * g.rows
        imgs.append(([s.picture(first + j) for j in range(g.cols * g.rows)], g.places, w, h))
    m = selector.Mlp(selector.K, seed=3)
    with Server(0, max_inflight=2, batching=True, batch_window_us=100000) as srv:
        srv.set_selector(m, selector.SCHEDULES)
        for k, (pics, places, w, h) in enumerate(imgs):
            srv.submit(pics, places, w, h, user=k)
        got = {}
        while len(got) < len(imgs):
            for c in srv.poll(16, timeout_ms=60000):
                assert c["status"] == abi.OK
                got[c["user"]] = c
        picks = srv.selector_picks(selector.K)
        srv.set_selector(None, selector.SCHEDULES)
    assert sum(picks) >= 1
    for k, (pics, places, w, h) in enumerate(imgs):
        out, keep = synth.grid_output(synth.Grid(w, h, 512, s, places))
        _, ref = O.decode_batch(pics, out, want_planes=False)
        assert np.array_equal(got[k]["image"], ref), k
    m.close()


@pytest.mark.gpu
def test_submit_path_host_pick_equals_device_pick():
    """A context's submit picks on the host (host features, host forward of
    the bf16 weights); the pick equals the device path's (k_features + the
    network kernels, hpvcd_plan_select) on the same batches."""
    torch = _gpu()
    import ctypes as C
    from hpvcd_b200.gpu import DevicePlan, GpuDecoder
    m = selector.Mlp.load() if os.path.exists(selector.WEIGHTS_PATH) else selector.Mlp(selector.K, seed=5)
    L = abi.lib()
    cands = (abi.Sched * selector.K)(*selector.SCHEDULES)
    batches = []
    for i in range(4):
        s = synth.SynthSet()
        g = synth.make_grid(1024 + 256 * i, 768, seed=40 + i, bit_depth=10 if i % 2 else 8, synth=s)
        batches.append((s, s.pictures()))
    with GpuDecoder(0) as d:
        d.set_selector(m, selector.SCHEDULES)
        for s, pics in batches:
            before = d.selector_picks(selector.K + 1)
            t = d.submit(pics)
            d.wait(t)
            d.read(t)
            after = d.selector_picks(selector.K + 1)
            host_pick = int(np.flatnonzero(np.array(after) - np.array(before))[0])
            plan = DevicePlan(pics)
            dev_pick = C.c_uint32()
            st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
            assert L.hpvcd_plan_select(plan._h, m.handle, cands, selector.K, st, C.byref(dev_pick)) == abi.OK
            torch.cuda.synchronize()
            dp = selector.K if dev_pick.value == abi.MLP_NO_PICK else dev_pick.value
            assert host_pick == dp
            plan.close()
        d.set_selector(None, selector.SCHEDULES)
    m.close()


@pytest.mark.gpu
def test_domain_guard_falls_back_to_default():
    _gpu()
    m = selector.Mlp(selector.K, seed=4)
    x = np.random.default_rng(8).random((6, 16)).astype(np.float32)
    lo = np.zeros(16, np.float32)
    hi = np.ones(16, np.float32)
    m.set_domain(lo, hi)
    x[2, 5] = 1.5   # outside
    x[4, 0] = -0.2  # outside
    picks = m.pick(x)
    assert picks[2] == abi.MLP_NO_PICK and picks[4] == abi.MLP_NO_PICK
    assert all(p < selector.K for i, p in enumerate(picks) if i not in (2, 4))
    m.set_domain(None, None)
    assert np.all(m.pick(x) < selector.K)
    m.close()
