"""The committed sensor weights: the .bin file the C ABI reads
(cbns_sensor_load_file) holds exactly the parameters and threshold of the
.npz the Python side uses, and both are well-formed."""
import json
import struct
from pathlib import Path

import numpy as np

DATA = Path(__file__).resolve().parents[1] / "cbns3d_cuda_b200" / "data"


def test_bin_matches_npz():
    w = np.load(DATA / "sensor_weights.npz")
    raw = (DATA / "sensor_weights.bin").read_bytes()
    assert raw[:8] == b"CBNSSNS1"
    n, tau = struct.unpack("<If", raw[8:16])
    assert n == 1601 and len(raw) == 16 + 4 * n
    p = np.frombuffer(raw[16:], dtype="<f4")
    assert np.array_equal(p, w["params"].astype(np.float32))
    assert tau == np.float32(w["tau"]) and 0.0 < tau < 1.0
    assert np.all(np.isfinite(p))
    summary = json.loads(str(w["summary"]))
    assert summary["label_threshold"] == 0.05 and np.float32(summary["tau"]) == np.float32(w["tau"])
