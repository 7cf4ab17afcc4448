"""Timing of single sweep primitives on one GPU, on seeded random operands.

    python -m dmrg2.microbench heff --chi 256 [--d 2 --D 5 --complex --reps 50]
    python -m dmrg2.microbench heffref --chi 256 [--d 2 --D 5 --reps 50]
    python -m dmrg2.microbench svd  --n 512   [--keep 256 --complex --reps 5]
    python -m dmrg2.microbench gemm --m 1024 --n 4096 --k 1024 [--complex --reps 5]
    python -m dmrg2.microbench lanczos --chi 256 [--reps 3]
    python -m dmrg2.microbench env  --chi 256 [--reps 10]
    python -m dmrg2.microbench warm --n 512 [--keep 256 --reps 3]

heff runs dmrg2_op_heff_noalloc on device-resident operands (torch tensors)
and reports the device time per matvec (CUDA events) and its algorithmic
TFLOP/s; heffref times the same three steps (real FP64) as cuBLAS calls through
torch (a yardstick for the GEMM rate these shapes allow, not part of the library:
step 1 one GEMM of (cL D) x cL by cL x (d^2 cR), step 2 the D d^2 square mixing
matrix applied per row block, step 3 (cL d^2) x (D cR) by its transpose of R) and
the library's matvec beside them; svd runs the truncated split through dmrg2_op_svd (host buffers,
so the time includes the copies); gemm runs the FP64 DMMA GEMM and the
split-BF16 tcgen05 GEMM of the precision form on the same operands (host
buffers) and reports their difference. lanczos runs the
device Lanczos solver (dmrg2_op_lanczos: H_eff matvecs and the fused Krylov
vector passes) on a Heisenberg two-site problem with seeded Hermitian
environments; env runs one left environment update; warm runs the
warm-started subspace split (dmrg2_op_warm_split) of a matrix with a decaying
spectrum from a perturbed copy of its kept right singular vectors. They are the
fixed small workloads the kernel profiles are taken on.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

import dmrg2


def heff_flops(cL, cR, d, D, cplx):
    dd = d * d
    f = 2.0 * D * cL * dd * cR * cL + 2.0 * cL * dd * D * cR * D * dd + 2.0 * cL * dd * cR * D * cR
    return 4.0 * f if cplx else f


def _rnd(rng, shape, cplx):
    x = rng.standard_normal(shape)
    return x + 1j * rng.standard_normal(shape) if cplx else x


def bench_heff(chi, d, D, cplx, reps, seed=0):
    import torch

    rng = np.random.default_rng(seed)
    lib = dmrg2.load_library()
    code = dmrg2.C128 if cplx else dmrg2.F64
    host = [_rnd(rng, s, cplx) for s in ((chi, D, chi), (chi, D, chi), (D, D, d, d), (D, D, d, d), (chi, d, d, chi))]
    L, R, WL, WR, th = (torch.from_numpy(a).cuda() for a in host)
    out = torch.empty_like(th)
    stream = torch.cuda.current_stream()
    p = lambda t: ctypes.c_void_p(t.data_ptr())

    def call():
        rc = lib.dmrg2_op_heff_noalloc(code, chi, chi, d, D, D, D, p(L), p(R), p(WL), p(WR), p(th), p(out),
                                       ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(lib.dmrg2_last_error(None).decode())

    for _ in range(3):
        call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        call()
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) * 1e-3 / reps
    fl = heff_flops(chi, chi, d, D, cplx)
    return {"op": "heff", "chi": chi, "d": d, "D": D, "complex": cplx, "us_per_matvec": t * 1e6,
            "gflop_per_matvec": fl / 1e9, "tflops": fl / t / 1e12}


def bench_heff_ref(chi, d, D, reps, seed=0):
    import torch

    dd = d * d
    g = torch.Generator(device="cuda").manual_seed(seed)
    L = torch.randn(chi * D, chi, dtype=torch.float64, device="cuda", generator=g)
    th = torch.randn(chi, dd * chi, dtype=torch.float64, device="cuda", generator=g)
    W = torch.randn(D * dd, D * dd, dtype=torch.float64, device="cuda", generator=g)
    R = torch.randn(chi, D * chi, dtype=torch.float64, device="cuda", generator=g)

    def step1():
        return L @ th                                  # (cL D) x (d^2 cR): X[a][w][.]

    def step2(X):
        return torch.matmul(W, X.view(chi, D * dd, chi))  # per a: (D d^2) x cR

    def step3(Y):
        return Y.view(chi * dd, D * chi) @ R.t()       # (cL d^2) x cR

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e-3 / reps

    X = step1()
    Y = step2(X).contiguous()
    t1, t2, t3 = timed(step1), timed(lambda: step2(X)), timed(lambda: step3(Y))
    f1 = 2.0 * chi * D * chi * dd * chi
    f2 = 2.0 * chi * (D * dd) ** 2 * chi
    f3 = 2.0 * chi * dd * D * chi * chi
    ours = bench_heff(chi, d, D, False, reps)
    return {"op": "heffref", "chi": chi, "d": d, "D": D,
            "cublas_us": {"step1": t1 * 1e6, "step2": t2 * 1e6, "step3": t3 * 1e6, "total": (t1 + t2 + t3) * 1e6},
            "cublas_tflops": {"step1": f1 / t1 / 1e12, "step3": f3 / t3 / 1e12,
                              "matvec": (f1 + f2 + f3) / (t1 + t2 + t3) / 1e12},
            "library_us_per_matvec": ours["us_per_matvec"], "library_tflops": ours["tflops"]}


def bench_svd(n, keep, cplx, reps, seed=0):
    rng = np.random.default_rng(seed)
    U, _ = np.linalg.qr(_rnd(rng, (n, n), cplx))
    V, _ = np.linalg.qr(_rnd(rng, (n, n), cplx))
    s = np.exp(-0.05 * np.arange(n))
    M = (U * s) @ V.conj().T
    times = []
    for _ in range(reps + 1):
        t = time.perf_counter()
        dmrg2.truncated_svd(M, keep, 1e-12, "R")
        times.append(time.perf_counter() - t)
    return {"op": "svd", "n": n, "keep": keep, "complex": cplx, "ms_per_call_host": 1e3 * float(np.median(times[1:]))}


def bench_gemm(m, n, k, cplx, reps, seed=0):
    rng = np.random.default_rng(seed)
    A, B = _rnd(rng, (m, k), cplx), _rnd(rng, (k, n), cplx)
    out = {}
    for name, f in (("fp64_dmma", dmrg2.gemm), ("split_bf16_tcgen05", dmrg2.gemm_bf16x3)):
        f(A, B)
        t = time.perf_counter()
        for _ in range(reps):
            C = f(A, B)
        out[name] = {"ms_per_call_host": 1e3 * (time.perf_counter() - t) / reps}
        out[name]["C"] = C
    err = np.abs(out["split_bf16_tcgen05"].pop("C") - out["fp64_dmma"].pop("C")).max()
    return {"op": "gemm", "m": m, "n": n, "k": k, "complex": cplx, **out,
            "max_abs_diff": float(err), "flops": (8.0 if cplx else 2.0) * m * n * k}


def _heis_w(D=5):
    W = np.zeros((D, D, 2, 2))
    sz = np.diag([0.5, -0.5])
    sp = np.array([[0.0, 1.0], [0.0, 0.0]])
    I = np.eye(2)
    W[0, 0], W[0, 1], W[0, 2], W[0, 3] = I, 0.5 * sp, 0.5 * sp.T, sz
    W[1, 4], W[2, 4], W[3, 4], W[4, 4] = sp.T, sp, sz, I
    return W


def _herm_env(rng, chi, D):
    E = rng.standard_normal((chi, D, chi))
    return 0.5 * (E + np.transpose(E, (2, 1, 0)))


def bench_lanczos(chi, reps, seed=0):
    rng = np.random.default_rng(seed)
    W = _heis_w()
    L, R = _herm_env(rng, chi, 5), _herm_env(rng, chi, 5)
    th = rng.standard_normal((chi, 2, 2, chi))
    times = []
    for _ in range(reps + 1):
        t = time.perf_counter()
        e, _ = dmrg2.optimize_two_site(L, R, W, W, th, max_iter=30, tol=1e-12, max_restarts=0)
        times.append(time.perf_counter() - t)
    return {"op": "lanczos", "chi": chi, "energy": e, "ms_per_call_host": 1e3 * float(np.median(times[1:]))}


def bench_env(chi, reps, seed=0):
    rng = np.random.default_rng(seed)
    L = _herm_env(rng, chi, 5)
    A = rng.standard_normal((chi, 2, chi))
    t = time.perf_counter()
    for _ in range(reps):
        dmrg2.update_left_env(L, A, _heis_w())
    return {"op": "env", "chi": chi, "ms_per_call_host": 1e3 * (time.perf_counter() - t) / reps}


def bench_warm(n, keep, reps, seed=1):
    rng = np.random.default_rng(seed)
    U, _ = np.linalg.qr(rng.standard_normal((n, n)))
    V, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = np.concatenate([np.logspace(0, -7, keep), 1e-8 * np.logspace(0, -3, n - keep)])
    M = (U * s) @ V.T
    warm = np.linalg.qr(V[:, :keep] + 1e-4 * rng.standard_normal((n, keep)))[0].T.copy()
    times = []
    for _ in range(reps + 1):
        t = time.perf_counter()
        _, _, te = dmrg2.warm_split(M, warm, keep, "R")
        times.append(time.perf_counter() - t)
    return {"op": "warm", "n": n, "keep": keep, "trunc_err": te, "ms_per_call_host": 1e3 * float(np.median(times[1:]))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("op", choices=["heff", "heffref", "svd", "gemm", "lanczos", "env", "warm"])
    ap.add_argument("--m", type=int, default=1024)
    ap.add_argument("--k", type=int, default=1024)
    ap.add_argument("--chi", type=int, default=256)
    ap.add_argument("--d", type=int, default=2)
    ap.add_argument("--D", type=int, default=5)
    ap.add_argument("--n", type=int, default=0)
    ap.add_argument("--keep", type=int, default=0)
    ap.add_argument("--complex", action="store_true")
    ap.add_argument("--reps", type=int, default=0)
    a = ap.parse_args()
    if a.op == "heff":
        r = bench_heff(a.chi, a.d, a.D, a.complex, a.reps or 50)
    elif a.op == "heffref":
        r = bench_heff_ref(a.chi, a.d, a.D, a.reps or 50)
    elif a.op == "svd":
        n = a.n or 512
        r = bench_svd(n, a.keep or n // 2, a.complex, a.reps or 5)
    elif a.op == "lanczos":
        r = bench_lanczos(a.chi, a.reps or 3)
    elif a.op == "env":
        r = bench_env(a.chi, a.reps or 10)
    elif a.op == "warm":
        n = a.n or 512
        r = bench_warm(n, a.keep or n // 2, a.reps or 3)
    else:
        r = bench_gemm(a.m, a.n or 4096, a.k, a.complex, a.reps or 5)
    print(json.dumps(r))


if __name__ == "__main__":
    main()
