"""Pin the oracle to the reference: golden fixtures from the reference build.

tests/golden/*.npz were produced by tests/golden/make_golden.py, which runs
the unmodified reference executables (compiled from the reference sources by
`make -C oracle ref`) on a B200 and records the checkpoint they write after the
last step and the dt they print each step (6 significant digits).
"""
import json
from pathlib import Path

import numpy as np
import pytest

from cbns3d_cuda_b200 import make_params
from oracle import oracle as orc
from tests.helpers import per_var_rel_linf

GOLD = Path(__file__).resolve().parent / "golden"
INDEX = json.loads((GOLD / "index.json").read_text()) if (GOLD / "index.json").exists() else {}


def load_case(name):
    meta = INDEX[name]
    z = np.load(GOLD / f"{name}.npz")
    return meta, z


def oracle_run(meta, z):
    IM, JM, KM = meta["shape"]
    p = make_params(IM, JM, KM, **meta["params"])
    o = orc.OracleBlock(p)
    o.init_like_reference(z["x"], z["y"], z["z"], None if meta["freestream_start"] else z["Q0"])
    dts = []
    t = 0.0
    for _ in range(meta["nsteps"]):
        dt = o.calc_dt()
        t_new = min(t + dt, meta["t_end"])
        dts.append(t_new - t)
        rc, t, n = o.solve(1, meta["t_end"], t)
        assert rc == 0 and n == 1
    return o, np.array(dts), t


def test_golden_index_present():
    assert len(INDEX) >= 4, "run tests/golden/make_golden.py on a GPU to create the fixtures"


@pytest.mark.parametrize("name", sorted(INDEX))
def test_oracle_matches_reference_build(oracle_lib, name):
    meta, z = load_case(name)
    o, dts, t = oracle_run(meta, z)
    assert len(z["dt"]) == meta["nsteps"]
    # dt printed with 6 significant digits by the reference
    assert np.allclose(dts, z["dt"], rtol=1e-5, atol=0)
    assert abs(t - float(z["t"])) <= 1e-12 * abs(float(z["t"]))
    Q = o.get_conservative(0)
    err = per_var_rel_linf(Q, z["Q"])
    assert max(err) <= 1e-11, err
