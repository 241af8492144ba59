"""Failure model of the detector pool and the request server.

The reference's failure model is CUDA_CHECK: print and exit(EXIT_FAILURE)
(cpp/lib/cuda/cuda_errorhandling.cuh:98-108, :113-134); its detector has no
deadlines or cancellation.  Here every served request ends with a status, and
failures are injected on the host only (no GPU fault, trap or hang):
  * malformed requests (unknown detector or kind, missing buffers) and
    requests larger than the HBM budget are rejected at submission;
  * a request not admitted into a batch by its deadline is dropped
    (APSM_ERR_DEADLINE); the requests that ran give the same estimates as the
    same surviving requests replayed alone;
  * a request that is not admitted yet can be cancelled (APSM_ERR_CANCELLED);
  * a request lost on its way into the queue (injected) ends by its deadline,
    or by a cancel, instead of hanging its client;
  * a lane whose scratch cannot grow (injected allocation failure) fails its
    batch with APSM_ERR_OUT_OF_MEMORY, and the next batch runs normally.
"""
import time

import numpy as np
import pytest

from libapsm_b200 import _native, synth

pytestmark = pytest.mark.gpu

CFG = {"otype": "APSM", "windowSize": 20, "gaussianKernelVariance": 0.5, "eB": 0.01, "dictionarySize": 600}
OK, DEADLINE, CANCELLED = _native.APSM_OK, _native.APSM_ERR_DEADLINE, _native.APSM_ERR_CANCELLED


def _frames(n, seed=0):
    out = []
    for i in range(n):
        N = (4, 8, 16)[i % 3]
        out.append((N, synth.generate_frame(seed + 40 + i, K=2, N=N, P=1600, S=2000, snr_db=20.0)))
    return out


def _setup(frames, lanes=1):
    from libapsm_b200 import DetectorPool, PoolJob

    pool = DetectorPool(CFG, lanes=lanes)
    ids = [pool.add(N) for N, _ in frames]
    pool.run([PoolJob(i, f.rx_train[:, :100], f.tx_train[0, :100]) for i, (_, f) in zip(ids, frames)])
    return pool, ids


def _job(ids, frames, req):
    from libapsm_b200 import PoolJob

    d, kind, lo, hi = req
    f = frames[d][1]
    if kind == "train":
        return PoolJob(ids[d], f.rx_train[:, lo:hi], f.tx_train[0, lo:hi])
    return PoolJob(ids[d], f.rx_data[:, lo:hi])


def test_malformed_and_oversized_requests_are_rejected_at_submission(native_lib):
    from libapsm_b200 import ApsmError, DetectorPool, DetectorServer, PoolJob
    from libapsm_b200.pool import JOB_DETECT, _CJob

    frames = _frames(2)
    pool, ids = _setup(frames)
    srv = DetectorServer(pool, max_batch=8)
    f = frames[0][1]
    rx = np.ascontiguousarray(f.rx_data[:, :50])
    bad = [_CJob(999, JOB_DETECT, 50, 0, rx.ctypes.data, None, None),   # unknown detector
           _CJob(ids[0], 7, 50, 0, rx.ctypes.data, None, None),        # unknown kind
           _CJob(ids[0], JOB_DETECT, 50, 0, rx.ctypes.data, None, None),  # no estimate buffer
           _CJob(ids[0], 0, 50, 0, rx.ctypes.data, None, None)]          # training without targets
    for cj in bad:
        with pytest.raises(ApsmError) as ei:
            srv.submit_prepared((cj, rx, None, None))
        assert ei.value.status == _native.APSM_ERR_INVALID_ARGUMENT
    assert srv.counts()[2] == len(bad)
    # the valid requests around them are unaffected
    t = srv.submit(PoolJob(ids[0], f.rx_data[:, :300]))
    est = srv.wait(t)
    ref_pool, ref_ids = _setup(frames)
    (ref,) = ref_pool.run([PoolJob(ref_ids[0], f.rx_data[:, :300])])
    np.testing.assert_array_equal(est, ref)
    srv.close()

    # a request whose scratch alone exceeds the HBM budget never joins a batch
    small = DetectorPool(CFG, hbm_budget=2_000_000)
    d = small.add(16)
    srv2 = DetectorServer(small, max_batch=4)
    big = synth.generate_frame(3, K=2, N=16, P=10, S=60000)
    with pytest.raises(ApsmError) as ei:
        srv2.submit(PoolJob(d, big.rx_data))
    assert ei.value.status == _native.APSM_ERR_OUT_OF_MEMORY
    srv2.close()


def test_deadline_drops_waiting_requests_and_survivors_match_replay(native_lib):
    from libapsm_b200 import DetectorServer

    frames = _frames(6)
    pool, ids = _setup(frames, lanes=1)
    srv = DetectorServer(pool, max_batch=2)
    rng = np.random.default_rng(3)
    reqs, cursor, phase = [], [100] * 6, [0] * 6
    for _ in range(48):
        d = int(rng.integers(0, 6))
        if phase[d] == 0 and cursor[d] < 1600:
            hi = min(1600, cursor[d] + int(rng.integers(16, 64)))
            reqs.append((d, "train", cursor[d], hi))
            cursor[d] = hi
        else:
            reqs.append((d, "detect", 0, int(rng.integers(200, 2000))))
        phase[d] ^= 1
    # a burst far above what one lane with batches of 2 can admit within 300 us (the first two
    # requests, admitted first, have a deadline no batch misses: some requests surely run even
    # when the lane's first batch is slow)
    preps = [srv.make_job(_job(ids, frames, r)) for r in reqs]
    tickets = [srv.submit_prepared(p, deadline=5.0 if k < 2 else 300e-6) for k, p in enumerate(preps)]
    sts = [srv.wait_status(t, 30.0) for t in tickets]
    assert set(sts) <= {OK, DEADLINE}, set(sts)
    assert sts.count(DEADLINE) > 0 and sts.count(OK) > 0, sts.count(DEADLINE)
    assert srv.counts()[0] == sts.count(DEADLINE)
    # a dropped request never ran: replaying only the surviving requests, one per batch,
    # gives the same estimates bit for bit
    ref_pool, ref_ids = _setup(frames, lanes=1)
    for r, st, p in zip(reqs, sts, preps):
        if st != OK:
            continue
        out = ref_pool.run([_job(ref_ids, frames, r)])
        if r[1] == "detect":
            np.testing.assert_array_equal(p[3], out[0])
    srv.close()


def test_cancel_waiting_request(native_lib):
    from libapsm_b200 import DetectorServer, PoolJob

    frames = _frames(1)
    pool, ids = _setup(frames, lanes=1)
    srv = DetectorServer(pool, max_batch=1)
    f = frames[0][1]
    # a long training request holds the only lane for milliseconds
    t1 = srv.submit(PoolJob(ids[0], f.rx_train[:, 100:1600], f.tx_train[0, 100:1600]))
    t2 = srv.submit(PoolJob(ids[0], f.rx_data[:, :500]))
    t3 = srv.submit(PoolJob(ids[0], f.rx_data[:, :700]))
    assert srv.cancel(t2) == OK
    assert srv.wait_status(t1) == OK and srv.wait_status(t3) == OK
    assert srv.status(t2) == CANCELLED
    assert srv.cancel(t2) == _native.APSM_ERR_INVALID_ARGUMENT  # finished already
    assert srv.counts()[1] == 1
    est3 = srv.wait(t3)
    ref_pool, ref_ids = _setup(frames, lanes=1)
    ref_pool.run([PoolJob(ref_ids[0], f.rx_train[:, 100:1600], f.tx_train[0, 100:1600])])
    (ref,) = ref_pool.run([PoolJob(ref_ids[0], f.rx_data[:, :700])])
    np.testing.assert_array_equal(est3, ref)
    # a request on the GPU runs to completion
    t4 = srv.submit(PoolJob(ids[0], f.rx_train[:, :1600], f.tx_train[0, :1600], fresh=True))
    while srv.times(t4)[1] == 0.0 and srv.status(t4) is None:
        time.sleep(1e-5)
    assert srv.cancel(t4) in (_native.APSM_ERR_UNSUPPORTED, _native.APSM_ERR_INVALID_ARGUMENT)
    assert srv.wait_status(t4) == OK
    srv.close()


def test_lost_request_ends_by_deadline_or_cancel(native_lib):
    from libapsm_b200 import DetectorServer, PoolJob

    frames = _frames(1)
    pool, ids = _setup(frames, lanes=1)
    srv = DetectorServer(pool, max_batch=4)
    f = frames[0][1]
    srv.inject_fault(_native.APSM_FAULT_DROP_REQUEST, 2)
    ta = srv.submit(PoolJob(ids[0], f.rx_data[:, :100]), deadline=0.02)
    tb = srv.submit(PoolJob(ids[0], f.rx_data[:, :100]), deadline=0)
    assert srv.wait_status(ta, 5.0) == DEADLINE
    assert srv.wait_status(tb, 0.1) == _native.APSM_ERR_TIMEOUT  # no deadline: the client's own wait bounds it
    assert srv.cancel(tb) == OK and srv.status(tb) == CANCELLED
    tc = srv.submit(PoolJob(ids[0], f.rx_data[:, :100]), deadline=1.0)
    assert srv.wait_status(tc, 5.0) == OK
    ref_pool, ref_ids = _setup(frames, lanes=1)
    (ref,) = ref_pool.run([PoolJob(ref_ids[0], f.rx_data[:, :100])])
    np.testing.assert_array_equal(srv.wait(tc), ref)
    srv.close()


def test_lane_growth_failure_fails_one_batch_only(native_lib):
    from libapsm_b200 import ApsmError, DetectorPool, DetectorServer, PoolJob

    frames = _frames(2)
    ref_pool, ref_ids = _setup(frames)
    (ref,) = ref_pool.run([PoolJob(ref_ids[1], frames[1][1].rx_data)])
    # direct pool use: the batch that needs the growth fails, the next one grows and runs
    pool = DetectorPool(CFG)
    ids = [pool.add(N) for N, _ in frames]
    pool.inject_fault(_native.APSM_FAULT_LANE_ALLOC, 1)
    init = [PoolJob(i, f.rx_train[:, :100], f.tx_train[0, :100]) for i, (_, f) in zip(ids, frames)]
    with pytest.raises(ApsmError) as ei:
        pool.run(init)
    assert ei.value.status == _native.APSM_ERR_OUT_OF_MEMORY
    pool.run(init)
    (est,) = pool.run([PoolJob(ids[1], frames[1][1].rx_data)])
    np.testing.assert_array_equal(est, ref)
    # served: the failing batch's requests end with the status, later requests run
    pool2, ids2 = _setup(frames)
    srv = DetectorServer(pool2, max_batch=4)
    big = synth.generate_frame(9, K=2, N=8, P=10, S=40000)
    pool2.inject_fault(_native.APSM_FAULT_LANE_ALLOC, 1)
    t1 = srv.submit(PoolJob(ids2[1], big.rx_data))  # needs a larger lane scratch: the injected failure
    assert srv.wait_status(t1) == _native.APSM_ERR_OUT_OF_MEMORY
    t2 = srv.submit(PoolJob(ids2[1], frames[1][1].rx_data))
    np.testing.assert_array_equal(srv.wait(t2), ref)
    srv.close()
