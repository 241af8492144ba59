"""The batched benchmark's largest shapes pinned against the FP32 oracle.

The 512-detector batch (antennas {4, 8, 16, 32}, 200-2000 pilots, 1000-16000
data symbols, window 80, a 2000-entry dictionary, the reference's default
kernel width 0.05 and eB 0.001) runs each training job as one chain of up to
2000 dependent steps.  The pool's batched sweep keeps the residual weights
r = w - sum_b a_b x_b and running window sums over the whole chain (its
incremental pair form), so FP32 drift over the full chain length is the risk
pinned here: full-length chains at the largest sizes, checked against the FP32
oracle (the restatement of cpp/lib/apsm/apsm_train.cu:80-166, 271-432 and
apsm_detect.cu:690-876) at 1e-4 of the largest soft output, with hard
decisions identical away from decision boundaries.  The oracle detects the
first S0 data symbols (the pool detects all of them).

The served form's train-append into a FULL dictionary is pinned too: a
detector trained on 2000 pilots (dictionary full) appends 64 new pilots
twice, every step evicting the oldest pair (the intended semantics of a second
train() call, cpp/lib/cuda/cuda_matrix_host.cu:334-365; see the oracle).
"""
import numpy as np
import pytest

from libapsm_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-4
S0 = 1500


def _check(est, ref, mod):
    scale = float(np.max(np.abs(ref)))
    err = float(np.max(np.abs(est - ref))) / scale
    e, r = mod.hard_decode_int(est), mod.hard_decode_int(ref)
    near = np.minimum(mod.boundary_distance(est), mod.boundary_distance(ref)) < 1e-4
    bad = int(np.sum((e != r) & ~near))
    return err, bad


@pytest.mark.parametrize("form", ["balanced", "gram_tf32x3"])
def test_full_length_chains_match_oracle(oracle_mod, form):
    from libapsm_b200 import DetectorPool, PoolJob

    cfg = dict(synth.CONFIG2_ALGORITHM, detectVersion=form)
    specs = [(32, 2000, 16000, "QAM16", 25.0), (4, 2000, 16000, "QPSK", 10.0), (16, 1999, 4000, "QAM16", 15.0)]
    pool = DetectorPool(cfg)
    dets, frames = [], []
    for i, (N, P, S, mod, snr) in enumerate(specs):
        dets.append(pool.add(N))
        frames.append(synth.generate_frame(900 + i, K=4, N=N, P=P, S=S, modulation=mod, snr_db=snr))
    outs = pool.run([PoolJob(d, f.rx_train, f.tx_train[0]) for d, f in zip(dets, frames)] +
                    [PoolJob(d, f.rx_data) for d, f in zip(dets, frames)])
    for k, ((N, P, S, _, _), f) in enumerate(zip(specs, frames)):
        est = outs[len(specs) + k]
        assert est.shape == (S,)
        o = oracle_mod.OracleDetector(cfg, N, oracle_mod.F32)
        o.train(f.rx_train, f.tx_train[0])
        ref = o.detect(f.rx_data[:, :S0])
        err, bad = _check(est[:S0], ref, f.modulation)
        print(f"{form} N={N} P={P}: soft error {err:.3e}, decisions differing {bad}")
        assert err < TOL and bad == 0, (N, err, bad)


def test_append_into_full_dictionary_matches_oracle(oracle_mod):
    from libapsm_b200 import DetectorPool, PoolJob

    cfg = dict(synth.CONFIG2_ALGORITHM)
    N, P = 16, 2000
    f = synth.generate_frame(950, K=4, N=N, P=P + 128, S=2000, modulation="QAM16", snr_db=20.0)
    pool = DetectorPool(cfg)
    d = pool.add(N)
    o = oracle_mod.OracleDetector(cfg, N, oracle_mod.F32)
    parts = [(0, P), (P, P + 64), (P + 64, P + 128)]
    for lo, hi in parts:
        pool.run([PoolJob(d, f.rx_train[:, lo:hi], f.tx_train[0, lo:hi])])
        o.train(f.rx_train[:, lo:hi], f.tx_train[0, lo:hi])
        (est,) = pool.run([PoolJob(d, f.rx_data)])
        ref = o.detect(f.rx_data)
        err, bad = _check(est, ref, f.modulation)
        print(f"append [{lo}, {hi}): soft error {err:.3e}, decisions differing {bad}")
        assert err < TOL and bad == 0, (lo, hi, err, bad)
    rows, _, _ = pool.get_state(d)
    assert rows == 2 * 2000
