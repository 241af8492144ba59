"""Why the reference is not a parity target once its dictionary overflows.

When one training call brings more pilot rows than the dictionary holds
(2P > 2 dictionarySize), the reference does not run a sliding dictionary:

  * pushRowsFromMatrix (cpp/lib/cuda/cuda_matrix_host.cu:327-347) writes all
    2P rows into the 2 dictionarySize-row ring in one kernel, one block per
    row, at ring slot (row mod capacity): rows that share a slot race and the
    slot keeps whichever write lands last;
  * moveWindow (:349-359) then only advances the ring; a slot reused after
    the ring is full keeps its coefficient;
  * the training kernel takes the window samples and targets from the call's
    pilots by dictionary row index (apsm_detect.cu:190-193 and
    apsm_train.cu:333-346), so once the ring is full every step re-trains on
    the pilots [capacity - window, capacity).

The fixture race_bpsk_evict.npz holds the reference's per-step history for such
a call.  This test restates that behaviour (in float64) with the slot contents
as unknowns, fits the content of each slot pair from the history of the step
that first uses it, and then requires every later step -- with nothing left to
fit -- to reproduce the reference's history.  The fitted slot contents are a
mix of pilot generations: the outcome of the race, different from run to run
and from any deterministic rule.  The B200 detector implements the sliding
dictionary the schedule describes (each pilot row enters once and evicts the
oldest row and its coefficient) and matches the reference wherever its
dictionary does not overflow."""
import itertools
import json
from pathlib import Path

import numpy as np
import pytest

FIXTURE = Path(__file__).resolve().parent / "golden" / "race_bpsk_evict.npz"


def dedup(rx):
    N, P = rx.shape
    X = np.zeros((2 * P, 2 * N))
    X[0::2, :N], X[0::2, N:] = rx.real.T, rx.imag.T
    X[1::2, :N], X[1::2, N:] = rx.imag.T, -rx.real.T
    return X


class RingModel:
    """The reference's training with its ring buffers (see the module docstring)."""

    def __init__(self, p, rx_train, tx_train, rx_val, tx_val):
        self.wL, self.wG, self.eB = p.linear_weight, p.gaussian_weight, p.eB
        self.ew = -0.5 / p.gaussian_variance
        self.q2, self.s, self.cap = 2 * p.window_size, p.sample_step, 2 * p.dictionary_size
        self.X = dedup(rx_train)
        self.Y = np.empty(self.X.shape[0])
        self.Y[0::2], self.Y[1::2] = tx_train.real, tx_train.imag
        # ring slot c holds half a row: Re (c even) or Im (c odd) of a pilot
        self.halves = np.empty((self.X.shape[0], rx_train.shape[0]))
        self.halves[0::2], self.halves[1::2] = rx_train.real.T, rx_train.imag.T
        self.Xv, self.tx_val = dedup(rx_val), tx_val
        self.H = np.zeros((self.cap, rx_train.shape[0]))
        self.C = np.zeros(self.cap)
        self.w = np.zeros(self.X.shape[1])
        self.u = self.o = 0

    def set_slot(self, slot, generation):
        self.H[slot] = self.halves[generation * self.cap + slot]

    def basis(self, used):
        rows = []
        for lrow in range(used):
            a = self.H[(lrow + self.o) % self.cap]
            b = self.H[(lrow + 1 + self.o) % self.cap] if lrow % 2 == 0 else -self.H[(lrow - 1 + self.o) % self.cap]
            rows.append(np.concatenate([a, b]))
        return np.array(rows), self.C[(np.arange(used) + self.o) % self.cap]

    def predict(self, x, used):
        B, c = self.basis(used)
        k = np.exp(self.ew * ((B[None, :, :] - x[:, None, :]) ** 2).sum(-1))
        return self.wL * x @ self.w + self.wG * k @ c

    def step(self, sidx):
        if self.u < self.cap:
            self.u += self.s
        else:
            self.o = (self.o + self.s) % self.cap
        used = min(self.u, self.cap)
        wk = min(self.q2, used)
        n = min(min(self.q2, sidx), wk)
        rows = np.arange(used - wk, used - wk + n)
        x = self.X[rows]
        e = self.Y[rows] - self.predict(x, used)
        c = np.where(e > self.eB, e - self.eB, np.where(e < -self.eB, e + self.eB, 0.0))
        c = c / wk / (self.wL * (x * x).sum(1) + self.wG)
        np.add.at(self.C, (rows + self.o) % self.cap, c)
        self.w += c @ x
        est = self.predict(self.Xv, used)
        return float(np.sqrt(np.mean(np.abs(est[0::2] + 1j * est[1::2] - self.tx_val) ** 2)))

    def copy(self):
        m = object.__new__(RingModel)
        m.__dict__ = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()}
        return m


@pytest.mark.skipif(not FIXTURE.exists(), reason="race fixture not generated")
def test_reference_overflowing_dictionary_is_a_slot_race(oracle_mod):
    d = np.load(FIXTURE)
    cfg = json.loads(str(d["config"]))
    ref = d["hist_ref"][:, 3].astype(np.float64)  # validation EVM after each step
    p = oracle_mod.reference_params(cfg, d["rx_train"].shape[0])
    model = RingModel(p, d["rx_train"], d["tx_train"], d["rx_data"], d["tx_data"])
    cap, s, rows = model.cap, model.s, model.X.shape[0]
    assert rows > cap and rows % cap == 0 and s == 2
    gens = rows // cap
    sidx = list(range(s, rows + 1, s))
    fitted = []
    for t in range(cap // 2):  # step t first uses ring slots 2t, 2t + 1
        best = None
        for g0, g1 in itertools.product(range(gens), repeat=2):
            m = model.copy()
            m.set_slot(2 * t, g0)
            m.set_slot(2 * t + 1, g1)
            err = abs(m.step(sidx[t]) - ref[t]) / ref[t]
            if best is None or err < best[0]:
                best = (err, g0, g1, m)
        assert best[0] < 2e-5, (t, best[0])
        fitted += [best[1], best[2]]
        model = best[3]
    # the ring is full: nothing is left to fit, every remaining step must match
    later = np.array([model.step(x) for x in sidx[cap // 2:]])
    np.testing.assert_allclose(later, ref[cap // 2:], rtol=2e-5)
    # the winners are not one generation: the slots' contents come from a race
    assert len(set(fitted)) > 1

    # the oracle (sliding dictionary) follows the schedule instead and differs
    from libapsm_b200.modulation import Modulation

    mod = Modulation(str(d["modulation"]))
    o = oracle_mod.OracleDetector(cfg, d["rx_train"].shape[0], oracle_mod.F32)
    h = o.train(d["rx_train"], d["tx_train"], val_set=(d["rx_data"], d["tx_data"], mod.bps, mod.scale))
    assert np.max(np.abs(h[:, 3] - ref) / ref) > 1e-2
