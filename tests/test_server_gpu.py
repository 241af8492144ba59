"""Request server (continuous batching) on the GPU.

A detector's results must not depend on which requests share its batches:
every detection result of a mixed request stream, admitted into batches on
two overlapping lanes, equals the result of the same detector's requests run
alone, one request per batch, on a second pool (bit-identical: one CTA per
training job, one thread per sample, no cross-job reductions)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = {"otype": "APSM", "windowSize": 20, "gaussianKernelVariance": 0.5, "eB": 0.01, "dictionarySize": 150}


def _streams(n_det, seed):
    from libapsm_b200 import synth

    rng = np.random.default_rng(seed)
    dets = []
    for i in range(n_det):
        N = int(rng.choice([2, 4, 8, 16]))
        f = synth.generate_frame(300 + i, K=2, N=N, P=400, S=600, snr_db=20.0)
        dets.append((N, f))
    reqs = []  # (detector, kind, lo, hi) in arrival order; each detector alternates train / detect
    cursor = [120] * n_det
    phase = [0] * n_det
    for _ in range(12 * n_det):
        d = int(rng.integers(0, n_det))
        if phase[d] == 0:
            p = int(rng.integers(8, 40))
            lo = cursor[d]
            cursor[d] = min(400, lo + p)
            if cursor[d] > lo:
                reqs.append((d, "train", lo, cursor[d]))
        else:
            s = int(rng.integers(50, 600))
            reqs.append((d, "detect", 0, s))
        phase[d] ^= 1
    return dets, reqs


def _jobs(dets, pool_ids, r):
    from libapsm_b200 import PoolJob

    d, kind, lo, hi = r
    N, f = dets[d]
    if kind == "train":
        return PoolJob(pool_ids[d], f.rx_train[:, lo:hi], f.tx_train[0, lo:hi])
    return PoolJob(pool_ids[d], f.rx_data[:, lo:hi])


@pytest.mark.parametrize("dv", ["balanced", "gram_tf32x3"])
def test_server_mixed_stream_equals_alone(native_lib, dv):
    from libapsm_b200 import DetectorPool, DetectorServer, PoolJob

    cfg = dict(CFG, detectVersion=dv)
    dets, reqs = _streams(10, seed=1)
    # served: all detectors share batches on two lanes
    pool = DetectorPool(cfg, lanes=2)
    ids = [pool.add(N) for N, _ in dets]
    pool.run([PoolJob(ids[d], f.rx_train[:, :120], f.tx_train[0, :120]) for d, (N, f) in enumerate(dets)])
    srv = DetectorServer(pool, max_batch=16)
    tickets = [srv.submit(_jobs(dets, ids, r)) for r in reqs]
    served = [srv.wait(t) for t in tickets]
    b, j = srv.stats()
    assert j == len(reqs) and b < len(reqs)  # requests really were batched together
    srv.close()
    # alone: one request per batch, in the same per-detector order
    alone_pool = DetectorPool(cfg)
    aid = [alone_pool.add(N) for N, _ in dets]
    for d, (N, f) in enumerate(dets):
        alone_pool.run([PoolJob(aid[d], f.rx_train[:, :120], f.tx_train[0, :120])])
    n_det_checked = 0
    for r, out in zip(reqs, served):
        res = alone_pool.run([_jobs(dets, aid, r)])[0]
        if r[1] == "detect":
            assert np.array_equal(out, res), r
            n_det_checked += 1
    assert n_det_checked > 20


def test_server_times_and_budget(native_lib):
    from libapsm_b200 import DetectorPool, DetectorServer, PoolJob

    dets, reqs = _streams(6, seed=2)
    pool = DetectorPool(CFG, hbm_budget=12_000_000, lanes=2)
    ids = [pool.add(N) for N, _ in dets]
    srv = DetectorServer(pool, max_batch=64)
    tickets = [srv.submit(_jobs(dets, ids, r)) for r in reqs]
    for t in tickets:
        srv.wait(t)
        s0, s1, s2 = srv.times(t)
        assert s0 <= s1 <= s2
    assert pool.bytes_in_use <= pool.budget
    srv.close()
