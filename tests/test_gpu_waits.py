"""Bounded device waits report a timeout instead of hanging.

With DMRG2_TEST_UNSIGNALLED_WAITS=1 the kernels that wait on a completion wait
on one that nothing signals, with a short poll limit: the split-BF16 tensor-core
GEMM waits for a tcgen05 commit that is never issued, and the cooperative Jacobi
SVD waits at a grid barrier that expects one block more than the grid has. Each
wait runs out, the kernel records the timeout, releases what it holds (tensor
memory) and returns, and the host reports DMRG2_ERR_NUMERIC. The hook is set in
a child process; afterwards the same calls in this process (hook off) run
normally on the same device.
"""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import dmrg2

pytestmark = pytest.mark.gpu
REPO = Path(__file__).resolve().parent.parent

CHILD = r"""
import numpy as np, dmrg2
lib = dmrg2.load_library()
rng = np.random.default_rng(0)
A = rng.standard_normal((200, 300))
B = rng.standard_normal((300, 150))
for what, call in [("gemm", lambda: dmrg2.gemm_bf16x3(A, B)),
                   ("jacobi", lambda: dmrg2.truncated_svd(A, 64, direction="R", method="jacobi"))]:
    try:
        call()
        print(what, "returned")
    except dmrg2.Dmrg2Error as e:
        print(what, "status", str(e).split("(status ")[1].split(")")[0], "timed out" in str(e))
"""


def test_unsignalled_waits_time_out_with_numeric_status():
    env = dict(os.environ, DMRG2_TEST_UNSIGNALLED_WAITS="1",
               PYTHONPATH=os.pathsep.join([str(REPO / "dmrg-implementations_b200"), str(REPO)]))
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines == [f"gemm status {dmrg2.ERR_NUMERIC} True", f"jacobi status {dmrg2.ERR_NUMERIC} True"], r.stdout
    # the device is still usable, and without the hook the same calls succeed
    rng = np.random.default_rng(0)
    A = rng.standard_normal((200, 300))
    B = rng.standard_normal((300, 150))
    C = dmrg2.gemm_bf16x3(A, B)
    assert np.abs(C - A @ B).max() <= 1e-5 * np.abs(A).max() * np.abs(B).max() * 300 ** 0.5
    U, S, Vh, _ = dmrg2.truncated_svd(A, 64, direction="R", method="jacobi")
    np.testing.assert_allclose(S[:64], np.linalg.svd(A, compute_uv=False)[:64], rtol=1e-12, atol=1e-12)
