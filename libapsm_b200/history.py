"""NomaTrainHistory: per-step training / validation metrics of a training call.

Mirrors cpp/lib/noma/noma_train_history.cuh:64-99 (constructed from the
modulation's bits per symbol and scale; vectors evmTrain, evmVal, serTrain,
serVal, berTrain, berVal; toCsv).  The values are computed on the GPU by the
training call (apsm_train_history of include/apsm_b200.h); this class only
holds them and writes the reference's CSV (noma_train_history.cu:237-248).
"""
from __future__ import annotations

import numpy as np


class NomaTrainHistory:
    COLUMNS = ("train_evm", "train_ser", "train_ber", "val_evm", "val_ser", "val_ber")

    def __init__(self, bit_per_symbol: int, modulation_scale: float):
        self.bit_per_symbol = int(bit_per_symbol)
        self.modulation_scale = float(np.float32(modulation_scale))
        self.per_user = np.zeros((0, 0, 6), dtype=np.float32)  # users x steps x 6

    def extend(self, rows: np.ndarray) -> None:
        """Append the steps of one training call (users x steps x 6)."""
        rows = np.asarray(rows, dtype=np.float32)
        if self.per_user.size == 0:
            self.per_user = rows.copy()
        else:
            self.per_user = np.concatenate([self.per_user, rows], axis=1)

    @property
    def steps(self) -> np.ndarray:
        """(steps, 6) of user 0."""
        return self.per_user[0] if self.per_user.shape[0] else np.zeros((0, 6), dtype=np.float32)

    evm_train = property(lambda self: self.steps[:, 0])
    ser_train = property(lambda self: self.steps[:, 1])
    ber_train = property(lambda self: self.steps[:, 2])
    evm_val = property(lambda self: self.steps[:, 3])
    ser_val = property(lambda self: self.steps[:, 4])
    ber_val = property(lambda self: self.steps[:, 5])

    def to_csv(self, filename: str) -> None:
        """toCsv: header line, then "step,train_evm,...,val_ber" per step (floats as %g)."""
        lines = ["step," + ",".join(self.COLUMNS)]
        for i, row in enumerate(self.steps):
            lines.append(",".join([str(i)] + [f"{float(v):g}" for v in row]))
        with open(filename, "w") as f:
            f.write("\n".join(lines) + "\n")
