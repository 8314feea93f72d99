"""The split-FP32 constants hard-coded in the device code are the exact
float splits of their values."""
import math
import re
from pathlib import Path

import numpy as np

SRC = Path(__file__).resolve().parent.parent / "obit_b200" / "csrc" / "ds_math.cuh"


def _const(name):
    m = re.search(rf"{name}\s*=\s*([0-9.eE+-]+)f;", SRC.read_text())
    assert m, name
    return float(np.float32(float(m.group(1))))


def test_inv_two_pi_split():
    x = 1.0 / (2.0 * math.pi)
    hi, lo = _const("kInv2PiHi"), _const("kInv2PiLo")
    assert hi == float(np.float32(x))
    assert lo == float(np.float32(x - hi))
    assert abs((hi + lo) - x) / x < 1e-15
