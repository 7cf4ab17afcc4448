"""dmrg2_op_heff_noalloc: H_eff on device pointers with static scratch.

Compared through the C ABI with the host-buffer entry point dmrg2_op_heff and
with the CPU oracle's apply_heff (the reference's numpy contraction restated) on
the same inputs, for two calls in a row (the second reuses the scratch the
first left behind), tolerance 1e-12 relative to the largest output entry (the
fused two-site MPO is built on the device instead of the host, so entries may
differ in the last bit). Also checks that calls after the first leave the
device's free memory unchanged, that oversized shapes are rejected, and (on a
machine without a GPU) that shapes whose scratch size would overflow are
rejected before any device work. This file is collected last so it runs both
alone and after every other GPU test.
"""
import ctypes

import numpy as np
import pytest

import dmrg2
from oracle import dmrg2_oracle as O

RTOL = 1e-12
SCRATCH_BYTES = 64 << 20

# (cL, cR, d, Dl, Dm, Dr, complex): MPO-mixing kernel path, split-K step 3,
# the batched-GEMM mixing path (d^2 D > 32), and a ragged 1 x 2 edge bond
CASES = [
    (48, 48, 2, 5, 5, 5, False),
    (96, 80, 2, 5, 5, 5, True),
    (16, 24, 5, 4, 4, 4, True),
    (20, 12, 3, 8, 8, 8, False),
    (1, 2, 2, 1, 5, 5, False),
]


def rnd(rng, shape, cplx):
    x = rng.standard_normal(shape)
    if cplx:
        x = x + 1j * rng.standard_normal(shape)
    return x


def close(a, b, rtol=RTOL):
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max() / scale
    assert err <= rtol, f"relative error {err:.3e} > {rtol:.1e}"


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def call_noalloc(torch, lib, code, shape, Ld, Rd, WLd, WRd, thd, outd):
    cL, cR, d, Dl, Dm, Dr = shape
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    return lib.dmrg2_op_heff_noalloc(code, cL, cR, d, Dl, Dm, Dr, p(Ld), p(Rd), p(WLd), p(WRd), p(thd),
                                     p(outd), stream)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_noalloc_matches_op_heff_twice(torch_cuda, case):
    torch = torch_cuda
    cL, cR, d, Dl, Dm, Dr, cplx = case
    lib = dmrg2.load_library()
    code = dmrg2.C128 if cplx else dmrg2.F64
    rng = np.random.default_rng(2024 + cL + cR)
    L = rnd(rng, (cL, Dl, cL), cplx)
    R = rnd(rng, (cR, Dr, cR), cplx)
    WL = rnd(rng, (Dl, Dm, d, d), cplx)
    WR = rnd(rng, (Dm, Dr, d, d), cplx)
    thetas = [rnd(rng, (cL, d, d, cR), cplx) for _ in range(2)]
    Ld, Rd, WLd, WRd = (to_dev(torch, a) for a in (L, R, WL, WR))
    outs, free_after = [], []
    for th in thetas:
        thd = to_dev(torch, th)
        outd = torch.empty_like(thd)
        rc = call_noalloc(torch, lib, code, (cL, cR, d, Dl, Dm, Dr), Ld, Rd, WLd, WRd, thd, outd)
        assert rc == 0, lib.dmrg2_last_error(None)
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info()[0])
        outs.append(outd.cpu().numpy())
    for th, got in zip(thetas, outs):
        close(got, dmrg2.apply_heff(L, R, WL, WR, th))
        close(got, O.apply_heff(L, R, WL, WR, th))
    # the second call launched kernels only: the device's free memory is unchanged
    assert free_after[1] == free_after[0]


@pytest.mark.gpu
def test_noalloc_rejects_shapes_above_the_static_limit(torch_cuda):
    torch = torch_cuda
    lib = dmrg2.load_library()
    cL = cR = 512
    d, D = 2, 5
    need = 2 * cL * D * d * d * cR * 8
    assert need > SCRATCH_BYTES
    # buffers of the full size, so nothing could read out of bounds even if the check were missing
    Ld = torch.zeros((cL, D, cL), dtype=torch.float64, device="cuda")
    Rd = torch.zeros((cR, D, cR), dtype=torch.float64, device="cuda")
    Wd = torch.zeros((D, D, d, d), dtype=torch.float64, device="cuda")
    thd = torch.zeros((cL, d, d, cR), dtype=torch.float64, device="cuda")
    outd = torch.empty_like(thd)
    rc = call_noalloc(torch, lib, dmrg2.F64, (cL, cR, d, D, D, D), Ld, Rd, Wd, Wd, thd, outd)
    assert rc == 1
    assert b"static limit" in lib.dmrg2_last_error(None)
    torch.cuda.synchronize()


def test_noalloc_rejects_overflowing_shapes_before_device_work():
    """Shapes whose scratch size would wrap around size_t are refused with
    DMRG2_ERR_ARG before the entry point touches the device. Runs only where no
    CUDA device is visible: the pointers are stand-ins that nothing may read."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("runs on a machine without a CUDA device")
    lib = dmrg2.load_library()
    fake = ctypes.c_void_p(256)
    big = 1 << 30
    for shape in [(big, big, 2, 5, 5, 5), (64, 64, 65536, 5, 5, 5), (big, 4, 2, 4096, 5, 4096)]:
        cL, cR, d, Dl, Dm, Dr = shape
        rc = lib.dmrg2_op_heff_noalloc(dmrg2.F64, cL, cR, d, Dl, Dm, Dr, fake, fake, fake, fake, fake, fake,
                                       ctypes.c_void_p(0))
        assert rc == 1, shape
        assert b"static limit" in lib.dmrg2_last_error(None)
