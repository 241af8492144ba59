"""apsm_b200: APSM multiuser detection on NVIDIA B200 (sm_100a).

Drop-in for the detector API of fraunhoferhhi/libapsm (NomaDetectorFactory /
NomaDetector); the compute runs in the hand-written CUDA kernels of the
in-tree libapsm_b200.so, reached through the C ABI of include/apsm_b200.h.
"""
from .detector import ApsmError, NomaDetector, NomaDetectorFactory, version
from .history import NomaTrainHistory
from .pool import DetectorPool, PoolJob
from .server import DetectorServer
from .modulation import Modulation, bit_error_rate, evm, symbol_error_rate
from . import synth

__all__ = ["ApsmError", "NomaDetector", "NomaDetectorFactory", "version", "Modulation", "bit_error_rate", "evm",
           "symbol_error_rate", "synth", "DetectorPool", "PoolJob", "DetectorServer", "NomaTrainHistory"]
