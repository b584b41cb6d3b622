"""The host driver's command line, checked where no GPU is needed: bad options
and values end the program with status 2 and a message before any CUDA call
(the driver itself is built by __graft_entry__.build())."""
import subprocess
from pathlib import Path

import pytest

EXE = Path(__file__).resolve().parents[1] / "cbns3d_cuda_b200" / "bin" / "cbns3d_b200"

pytestmark = pytest.mark.skipif(not EXE.exists(), reason="driver not built (run __graft_entry__.build())")


@pytest.mark.parametrize("args, msg", [
    (["--bc", "bogus"], "unknown boundary mode bogus"),
    (["--bc"], "missing value after --bc"),
    (["--frobnicate"], "unknown option --frobnicate"),
    (["--precision"], "missing value after --precision"),
])
def test_bad_arguments(tmp_path, args, msg):
    r = subprocess.run([str(EXE), *args], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
    assert msg in r.stderr
