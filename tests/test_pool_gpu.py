"""Detector pool (batched many-detector form) on the GPU.

Each pool detector must behave like its own NomaDetector (reference
cpp/lib/noma/noma_detector.cuh:65-75: train then detect, state kept between
calls): its soft outputs are compared with the FP32 oracle (the restatement of
apsm_train.cu / apsm_detect.cu) run detector by detector on the same inputs,
at the FP32-form tolerance 1e-4 relative to the largest soft output; the
hard decisions are compared away from decision boundaries.  The batch must
not change a detector's result: a job alone and in a mixed batch give
bit-identical outputs (one CTA per training job, one thread per sample).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _rel(a, b):
    scale = max(np.max(np.abs(b)), 1e-30)
    return float(np.max(np.abs(a - b)) / scale)


def _frame(seed, N, P, S, mod="QPSK"):
    from libapsm_b200 import synth

    f = synth.generate_frame(seed, K=2, N=N, P=P, S=S, modulation=mod, snr_db=20.0)
    return f.rx_train, f.tx_train[0], f.rx_data


def _oracle_run(oracle_mod, cfg, N, trains, rx_data):
    o = oracle_mod.OracleDetector(cfg, N, oracle_mod.F32)
    for rx, tx in trains:
        o.train(rx, tx)
    return o.detect(rx_data)


CFG = {"otype": "APSM", "windowSize": 20, "gaussianKernelVariance": 0.5, "eB": 0.01, "dictionarySize": 400}


@pytest.mark.parametrize("cfg", [
    CFG,
    dict(CFG, windowSize=80, dictionarySize=2000),
    dict(CFG, trainPasses=2),
    dict(CFG, startWithFullWindow=True),
    dict(CFG, trainingShuffle=True),
    dict(CFG, sampleStep=4),
    dict(CFG, gaussianKernelWeight=0.8, eB=0.001),
    dict(CFG, detectVersion="gram_tf32x3"),
    dict(CFG, windowSize=80, dictionarySize=2000, detectVersion="gram_tf32x3", gaussianKernelVariance=0.05,
         eB=0.001),
], ids=["w20", "w80", "passes2", "sfw", "shuffle", "step4", "wG08", "gram_tf32x3", "gram_tf32x3_narrow"])
def test_pool_matches_oracle_per_detector(native_lib, oracle_mod, cfg):
    from libapsm_b200 import DetectorPool, PoolJob

    pool = DetectorPool(cfg)
    # (24 and 28 antennas: 48 / 56 features, the widest class's 32-pair chunks at K below 64)
    specs = [(3, 120, 200), (4, 300, 96), (8, 60, 50), (16, 250, 300), (2, 31, 17), (32, 150, 128), (24, 90, 140),
             (28, 70, 61)]
    dets, jobs, frames = [], [], []
    for i, (N, P, S) in enumerate(specs):
        d = pool.add(N)
        rx, tx, rxd = _frame(100 + i, N, P, S)
        dets.append(d)
        frames.append((N, rx, tx, rxd))
        jobs.append(PoolJob(d, rx, tx))
    for d, (N, rx, tx, rxd) in zip(dets, frames):
        jobs.append(PoolJob(d, rxd))
    outs = pool.run(jobs)
    for k, (N, rx, tx, rxd) in enumerate(frames):
        est = outs[len(specs) + k]
        ref = _oracle_run(oracle_mod, cfg, N, [(rx, tx)], rxd)
        assert _rel(est, ref) < TOL, (k, N, _rel(est, ref))


# Operand precision of the pool's other tensor-core forms: the cross term y^H x
# carries ~2^-8 (bf16), ~2^-11 (tf32) or ~2^-16 (bf16x3) relative error of
# |y||x|, which reaches each Gaussian term scaled by |ew|; the single-product
# forms recompute the pairs where that bound is large exactly (2e-3 bar).
GRAM_TOL = {"gram_bf16": 2e-3, "gram_tf32": 2e-3, "gram_bf16x3": 1e-4}


@pytest.mark.parametrize("narrow", [False, True], ids=["wide", "narrow"])
@pytest.mark.parametrize("dv", sorted(GRAM_TOL))
def test_pool_gram_forms_match_oracle(native_lib, oracle_mod, dv, narrow):
    from libapsm_b200 import DetectorPool, PoolJob

    cfg = dict(CFG, detectVersion=dv)
    if narrow:
        cfg.update(windowSize=80, dictionarySize=2000, gaussianKernelVariance=0.05, eB=0.001)
    pool = DetectorPool(cfg)
    specs = [(3, 120, 200), (4, 300, 96), (8, 60, 50), (16, 250, 300), (2, 31, 17), (32, 150, 128), (24, 90, 140),
             (28, 70, 61)]
    dets, frames = [], []
    for i, (N, P, S) in enumerate(specs):
        dets.append(pool.add(N))
        frames.append((N,) + _frame(300 + i, N, P, S, "QAM16"))
    jobs = [PoolJob(d, f[1], f[2]) for d, f in zip(dets, frames)] + [PoolJob(d, f[3]) for d, f in zip(dets, frames)]
    outs = pool.run(jobs)
    for k, (N, rx, tx, rxd) in enumerate(frames):
        ref = _oracle_run(oracle_mod, cfg, N, [(rx, tx)], rxd)
        err = _rel(outs[len(specs) + k], ref)
        print(f"{dv} {'narrow' if narrow else 'wide'} N={N}: {err:.3e}")
        assert err < GRAM_TOL[dv], (k, N, err)


def test_pool_train_append_and_eviction(native_lib, oracle_mod):
    """Pilots appended to the resident dictionary over several batches; the
    dictionary (200 entries) fills and evicts its oldest entries."""
    from libapsm_b200 import DetectorPool, PoolJob

    cfg = dict(CFG, dictionarySize=200)
    pool = DetectorPool(cfg)
    N = 6
    d0, d1 = pool.add(N), pool.add(N)
    rx, tx, rxd = _frame(7, N, 330, 160)
    chunks = [(0, 90), (90, 150), (150, 230), (230, 330)]
    trains = []
    for lo, hi in chunks:
        trains.append((rx[:, lo:hi], tx[lo:hi]))
        pool.run([PoolJob(d0, rx[:, lo:hi], tx[lo:hi]), PoolJob(d1, rx[:, lo:hi], tx[lo:hi])])
        est0, est1 = pool.run([PoolJob(d0, rxd), PoolJob(d1, rxd)])
        ref = _oracle_run(oracle_mod, cfg, N, trains, rxd)
        assert _rel(est0, ref) < TOL, (hi, _rel(est0, ref))
        assert np.array_equal(est0, est1)
    rows, a, w = pool.get_state(d0)
    assert rows == 2 * 200


@pytest.mark.parametrize("dv", ["balanced", "gram_tf32x3", "gram_bf16"])
def test_pool_alone_equals_in_mix(native_lib, dv):
    from libapsm_b200 import DetectorPool, PoolJob

    cfg = dict(CFG, windowSize=80, dictionarySize=2000, detectVersion=dv)
    N, P, S = 8, 400, 256
    rx, tx, rxd = _frame(11, N, P, S)
    alone = DetectorPool(cfg)
    d = alone.add(N)
    alone.run([PoolJob(d, rx, tx)])
    (ref,) = alone.run([PoolJob(d, rxd)])

    mix = DetectorPool(cfg)
    others = []
    for i, (n2, p2, s2) in enumerate([(4, 900, 300), (16, 200, 1000), (32, 700, 64)]):
        others.append((mix.add(n2),) + _frame(50 + i, n2, p2, s2))
    dm = mix.add(N)
    jobs = [PoolJob(o[0], o[1], o[2]) for o in others] + [PoolJob(dm, rx, tx)]
    jobs += [PoolJob(o[0], o[3]) for o in others] + [PoolJob(dm, rxd)]
    outs = mix.run(jobs)
    assert np.array_equal(outs[-1], ref)


def test_pool_untrained_detect_is_zero_and_reset(native_lib):
    from libapsm_b200 import DetectorPool, PoolJob

    pool = DetectorPool(CFG)
    d = pool.add(4)
    rx, tx, rxd = _frame(3, 4, 50, 40)
    (est,) = pool.run([PoolJob(d, rxd)])
    assert np.all(est == 0)
    pool.run([PoolJob(d, rx, tx)])
    (e1,) = pool.run([PoolJob(d, rxd)])
    assert np.any(e1 != 0)
    pool.reset(d)
    (e2,) = pool.run([PoolJob(d, rxd)])
    assert np.all(e2 == 0)
    pool.run([PoolJob(d, rx, tx)])
    (e3,) = pool.run([PoolJob(d, rxd)])
    assert np.array_equal(e1, e3)


def test_pool_device_buffers_and_lanes(native_lib):
    import torch

    from libapsm_b200 import DetectorPool, PoolJob

    pool = DetectorPool(CFG, lanes=2)
    specs = [(4, 200, 100), (8, 150, 333)]
    dets = [pool.add(n) for n, _, _ in specs]
    frames = [_frame(20 + i, *s) for i, s in enumerate(specs)]
    host = DetectorPool(CFG)
    hd = [host.add(n) for n, _, _ in specs]
    refs = host.run([PoolJob(d, f[0], f[1]) for d, f in zip(hd, frames)] + [PoolJob(d, f[2]) for d, f in zip(hd, frames)])
    ests = []
    for lane, (d, f) in enumerate(zip(dets, frames)):
        rx, tx, rxd = (torch.from_numpy(x).cuda() for x in f)
        est = torch.empty(rxd.shape[1], dtype=torch.complex64, device="cuda")
        torch.cuda.synchronize()
        pool.run_device([PoolJob(d, rx, tx), PoolJob(d, rxd, est=est)], lane=lane)
        ests.append((est, rx, tx, rxd))
    for lane in range(2):
        pool.wait(lane)
    for k in range(2):
        assert np.array_equal(ests[k][0].cpu().numpy(), refs[2 + k])
    t_ms, d_ms = pool.last_ms(0)
    assert t_ms > 0 and d_ms > 0


def test_pool_budget_admission(native_lib):
    from libapsm_b200 import ApsmError, DetectorPool, PoolJob

    pool = DetectorPool(CFG, hbm_budget=600_000)
    d = pool.add(4)
    with pytest.raises(ApsmError, match="OUT_OF_MEMORY"):
        for _ in range(100):
            pool.add(32)
    rx, tx, rxd = _frame(5, 4, 2000, 10)
    job = PoolJob(d, rx, tx)
    assert pool.job_bytes(job) > 0
    with pytest.raises(ApsmError, match="OUT_OF_MEMORY"):
        pool.run([job])
    assert pool.bytes_in_use <= pool.budget


def test_pool_fresh_flag_is_reset_then_train(native_lib):
    from libapsm_b200 import DetectorPool, PoolJob

    pool = DetectorPool(CFG)
    d = pool.add(8)
    rx, tx, rxd = _frame(9, 8, 120, 64)
    pool.run([PoolJob(d, rx, tx)])
    (ref,) = pool.run([PoolJob(d, rxd)])
    for _ in range(2):  # trained state present: fresh discards it
        out = pool.run([PoolJob(d, rx, tx, fresh=True), PoolJob(d, rxd)])
        assert np.array_equal(out[1], ref)
    empty = np.zeros((8, 0), np.complex64)
    (est,) = pool.run([PoolJob(d, empty, np.zeros(0, np.complex64), fresh=True), PoolJob(d, rxd)])[1:]
    assert np.all(est == 0)


def test_pool_pinned_host_buffers_equal_pageable(native_lib):
    """Page-locked host buffers are copied directly (no staging); the results
    equal those of ordinary host buffers."""
    import torch

    from libapsm_b200 import DetectorPool, PoolJob

    pool = DetectorPool(CFG)
    specs = [(4, 90, 70), (8, 120, 33), (16, 60, 128)]
    frames = [_frame(40 + i, *s_) for i, s_ in enumerate(specs)]
    dets = [pool.add(n) for n, _, _ in specs]
    ref = pool.run([PoolJob(d, f[0], f[1], fresh=True) for d, f in zip(dets, frames)] +
                   [PoolJob(d, f[2]) for d, f in zip(dets, frames)])
    keep = []

    def pin(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        keep.append(t)
        return t.numpy()

    outs = [pin(np.zeros(f[2].shape[1], np.complex64)) for f in frames]
    pool.run([PoolJob(d, pin(f[0]), pin(f[1]), fresh=True) for d, f in zip(dets, frames)] +
             [PoolJob(d, pin(f[2]), est=o) for d, f, o in zip(dets, frames, outs)])
    for k in range(3):
        assert np.array_equal(outs[k], ref[3 + k])


@pytest.mark.parametrize("dv", ["balanced", "gram_tf32x3"])
def test_pool_autotune_changes_no_detector_and_no_result(native_lib, dv):
    """apsm_pool_autotune runs the batch once per candidate launch shape; the
    detectors it trains get their state back, and batches run with the chosen
    shapes give the same estimates as with the built-in ones."""
    from libapsm_b200 import DetectorPool, PoolJob

    cfg = dict(CFG, detectVersion=dv)
    specs = [(3, 220, 200), (8, 160, 96), (16, 250, 300), (32, 150, 128)]
    frames = [(N,) + _frame(400 + i, N, P, S) for i, (N, P, S) in enumerate(specs)]

    def setup(pool):
        ids = [pool.add(f[0]) for f in frames]
        pool.run([PoolJob(d, f[1][:, :100], f[2][:100]) for d, f in zip(ids, frames)])  # resident state to append to
        batch = ([PoolJob(d, f[1][:, 100:], f[2][100:]) for d, f in zip(ids, frames)] +
                 [PoolJob(d, f[3]) for d, f in zip(ids, frames)])
        return ids, batch

    tuned = DetectorPool(cfg)
    ids, batch = setup(tuned)
    before = [tuned.get_state(d) for d in ids]
    rep = tuned.autotune(tuned.prepare(batch))
    assert rep["trials"] and rep["sweep_ctas_per_sm"] >= 1
    after = [tuned.get_state(d) for d in ids]
    for x, y in zip(before, after):
        assert x[0] == y[0]
        np.testing.assert_array_equal(x[1], y[1])
        np.testing.assert_array_equal(x[2], y[2])
    outs = tuned.run(batch)

    plain = DetectorPool(cfg)
    _, batch2 = setup(plain)
    ref = plain.run(batch2)
    for k in range(len(specs), 2 * len(specs)):
        np.testing.assert_array_equal(outs[k], ref[k])


def test_pool_reserve_runs_nothing(native_lib):
    """apsm_pool_reserve grows a lane's buffers for a batch without running it:
    the detectors keep their state, and the batch run afterwards gives what it
    gives without the reservation."""
    from libapsm_b200 import DetectorPool, PoolJob

    frames = [(N,) + _frame(500 + i, N, P, S) for i, (N, P, S) in enumerate([(4, 120, 3000), (32, 200, 2000)])]

    def batch(pool, ids):
        return ([PoolJob(d, f[1], f[2]) for d, f in zip(ids, frames)] + [PoolJob(d, f[3]) for d, f in zip(ids, frames)])

    a = DetectorPool(dict(CFG, detectVersion="gram_tf32x3"), lanes=2)
    ids = [a.add(f[0]) for f in frames]
    b0 = batch(a, ids)
    a.reserve(a.prepare(b0), lane=1)
    for d in ids:
        assert a.get_state(d)[0] == 0  # untrained still
    outs = a.run(b0, lane=1)
    ref_pool = DetectorPool(dict(CFG, detectVersion="gram_tf32x3"), lanes=2)
    ids2 = [ref_pool.add(f[0]) for f in frames]
    ref = ref_pool.run(batch(ref_pool, ids2), lane=1)
    for k in range(2, 4):
        np.testing.assert_array_equal(outs[k], ref[k])


def test_pool_page_locked_training_inputs_read_in_place(native_lib):
    """A host-buffer batch whose training inputs (>= 4 MB) sit in page-locked
    memory has them read in place by the packing kernel; the estimates equal
    those of the same batch from pageable buffers (staged and uploaded)."""
    import torch

    from libapsm_b200 import DetectorPool, PoolJob

    specs = [(32, 1800, 600), (16, 1500, 900), (8, 1900, 300), (32, 1700, 200)]
    frames = [(N,) + _frame(600 + i, N, P, S) for i, (N, P, S) in enumerate(specs)]
    pinned = []

    def pin(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        pinned.append(t)
        return t.numpy()

    outs = {}
    for mode in ("pageable", "page-locked"):
        pool = DetectorPool(dict(CFG, windowSize=80, dictionarySize=2000, detectVersion="gram_tf32x3"))
        ids = [pool.add(f[0]) for f in frames]
        # enough detectors of the same frames for 4 MB of training inputs in one batch
        reps = 8
        more = [pool.add(f[0]) for _ in range(reps - 1) for f in frames]
        all_ids = ids + more
        all_frames = frames * reps
        conv = (lambda a: a) if mode == "pageable" else pin
        jobs = ([PoolJob(d, conv(f[1]), conv(f[2]), fresh=True) for d, f in zip(all_ids, all_frames)] +
                [PoolJob(d, conv(f[3]), est=conv(np.zeros(f[3].shape[1], np.complex64))) for d, f in zip(all_ids, all_frames)])
        res = pool.run(jobs)
        outs[mode] = [res[len(all_ids) + k] for k in range(len(all_ids))]
    for a, b in zip(outs["pageable"], outs["page-locked"]):
        np.testing.assert_array_equal(a, b)


def test_pool_pageable_detection_samples_staged_while_training(native_lib):
    """A batch that trains and detects from ordinary (pageable) buffers with >= 4 MB of
    detection samples stages and uploads them per detection segment while it trains; the
    estimates equal those of the same training and detection run as two batches (the second
    one stages everything before its upload).  The 48-antenna detectors run the CUDA-core
    detection (a segment of its own) beside the tensor-core classes."""
    from libapsm_b200 import DetectorPool, PoolJob

    frames = [(N,) + _frame(800 + i, N, 300, 6000) for i, N in enumerate([4, 8, 16, 32, 48])]
    outs = {}
    for mode in ("one batch", "two batches"):
        pool = DetectorPool(dict(CFG, detectVersion="gram_tf32x3"))
        dets = [(pool.add(f[0]), f) for _ in range(4) for f in frames]  # 20 detectors, 20.7 MB of samples
        train = [PoolJob(d, f[1], f[2], fresh=True) for d, f in dets]
        detect = [PoolJob(d, f[3]) for d, f in dets]
        if mode == "one batch":
            res = pool.run(train + detect)[len(train):]
        else:
            pool.run(train)
            res = pool.run(detect)
        outs[mode] = [np.array(r) for r in res]
    for a, b in zip(outs["one batch"], outs["two batches"]):
        np.testing.assert_array_equal(a, b)


def test_pool_page_locked_training_with_pageable_detection_samples(native_lib):
    """Training inputs (>= 4 MB) in page-locked buffers, read in place and packed per antenna
    class beside the kernel columns, with the detection samples in pageable buffers staged per
    segment while the batch trains: the estimates equal those of the same training and
    detection from pageable buffers run as two batches."""
    import torch

    from libapsm_b200 import DetectorPool, PoolJob

    frames = [(N,) + _frame(900 + i, N, 1500, 3000) for i, N in enumerate([8, 16, 32, 32])]
    keep = []

    def pin(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        keep.append(t)
        return t.numpy()

    outs = {}
    for mode in ("mixed", "two batches"):
        pool = DetectorPool(dict(CFG, windowSize=40, dictionarySize=1500, detectVersion="gram_tf32x3"))
        dets = [(pool.add(f[0]), f) for _ in range(4) for f in frames]  # 16 detectors, 4.4 MB of training inputs
        if mode == "mixed":
            train = [PoolJob(d, pin(f[1]), pin(f[2]), fresh=True) for d, f in dets]
            res = pool.run(train + [PoolJob(d, f[3]) for d, f in dets])[len(train):]
        else:
            pool.run([PoolJob(d, f[1], f[2], fresh=True) for d, f in dets])
            res = pool.run([PoolJob(d, f[3]) for d, f in dets])
        outs[mode] = [np.array(r) for r in res]
    for a, b in zip(outs["mixed"], outs["two batches"]):
        np.testing.assert_array_equal(a, b)


def test_pool_page_locked_estimates_written_in_place(native_lib):
    """Estimates (>= 4 MB) of a host-buffer batch into page-locked buffers are
    written there by the detection kernels; they equal those of the same batch
    with pageable outputs (copied back and scattered)."""
    import torch

    from libapsm_b200 import DetectorPool, PoolJob

    frames = [(N,) + _frame(700 + i, N, 200, 10000) for i, N in enumerate([4, 8, 16, 32])]
    outs = {}
    for mode in ("pageable", "page-locked"):
        pool = DetectorPool(dict(CFG, detectVersion="gram_tf32x3"))
        dets = [(pool.add(f[0]), f) for _ in range(16) for f in frames]  # 64 detectors, 5 MB of estimates
        pool.run([PoolJob(d, f[1], f[2]) for d, f in dets])
        ests = []
        for d, f in dets:
            e = np.zeros(f[3].shape[1], np.complex64)
            if mode == "page-locked":
                t = torch.from_numpy(e).pin_memory()
                ests.append(t)
                e = t.numpy()
            ests.append(e)
        arrays = [e for e in ests if isinstance(e, np.ndarray)]
        res = pool.run([PoolJob(d, f[3], est=e) for (d, f), e in zip(dets, arrays)])
        outs[mode] = [np.array(r) for r in res]
    for a, b in zip(outs["pageable"], outs["page-locked"]):
        np.testing.assert_array_equal(a, b)


NORM_CFGS = {  # bounds below every detector's unconstrained norm (the test checks that they bind)
    "norm-w10": dict(CFG, windowSize=10, normConstraint=0.01, dictionarySize=400),
    "norm-wrap": dict(CFG, windowSize=20, normConstraint=0.01, dictionarySize=60),
    "norm-w80": dict(CFG, windowSize=80, normConstraint=0.003, dictionarySize=400, detectVersion="gram_tf32x3"),
}


@pytest.mark.parametrize("name", sorted(NORM_CFGS))
def test_pool_norm_constraint_matches_oracle(native_lib, oracle_mod, name):
    """normConstraint (apsm_train.cu:142-145, 168-256: after every step the
    Gaussian part's RKHS norm is bounded by rescaling the coefficients) in the
    pool: each detector's training runs the exact sweep, the detections the
    pool's kernels; per detector the FP32 oracle (adapt_coeffs_f32 after each
    step) at 1e-4, including a dictionary that wraps (60 entries, 150
    pilots) and a second train call that appends."""
    from libapsm_b200 import DetectorPool, PoolJob

    cfg = NORM_CFGS[name]
    pool = DetectorPool(cfg)
    specs = [(3, 150, 200), (8, 120, 96), (16, 100, 130), (32, 80, 64)]
    dets, frames = [], []
    for i, (N, P, S) in enumerate(specs):
        dets.append(pool.add(N))
        frames.append((N,) + _frame(700 + i, N, P, S, "QAM16"))
    half = [(d, f[1][:, : f[1].shape[1] // 2], f[2][: f[1].shape[1] // 2]) for d, f in zip(dets, frames)]
    rest = [(d, f[1][:, f[1].shape[1] // 2:], f[2][f[1].shape[1] // 2:]) for d, f in zip(dets, frames)]
    pool.run([PoolJob(d, rx, tx) for d, rx, tx in half])
    outs = pool.run([PoolJob(d, rx, tx) for d, rx, tx in rest] + [PoolJob(d, f[3]) for d, f in zip(dets, frames)])
    for k, ((N, rx, tx, rxd), h, r) in enumerate(zip(frames, half, rest)):
        ref = _oracle_run(oracle_mod, cfg, N, [(h[1], h[2]), (r[1], r[2])], rxd)
        free = _oracle_run(oracle_mod, {k: v for k, v in cfg.items() if k != "normConstraint"}, N,
                           [(h[1], h[2]), (r[1], r[2])], rxd)
        assert _rel(free, ref) > 10 * TOL, (name, N, "the bound does not bind")
        err = _rel(outs[len(specs) + k], ref)
        print(f"{name} N={N}: {err:.3e}")
        assert err < TOL, (name, N, err)
