"""Python mirror of the reference's two-site DMRG interface over the C ABI.

``DMRG2GPU`` mirrors the C++ class ``DMRG2GPU<Scalar>`` of the reference driver
(gpu-rocm/dmrg2-gpu/src/dmrg2_gpu.h:24-203): construct, ``set_mpo``,
``initialize_mps_*`` (plus ``set_mps``), ``run``, ``get_energy``, ``get_mps``,
``chi_L``/``chi_R``. The module-level functions mirror the reference's numpy
two-site primitives (cpu/pdmrg/pdmrg/numerics/effective_ham.py:apply_heff,
eigensolver.py:optimize_two_site, accurate_svd.py:truncated_svd,
environments/update.py:update_left_env/update_right_env) with the same
argument meaning and tensor conventions, executed on the GPU.

Everything runs in ``libdmrg2_b200.so`` (CUDA, sm_100a). There is no CPU
fallback: importing works without a GPU, but every compute call raises
``Dmrg2Error`` when the library or a CUDA device is unavailable.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libdmrg2_b200.so"

F64, C128 = 0, 1
ROWMAJOR, REFERENCE = 0, 1
INIT_RANDOM, INIT_PRODUCT, INIT_NEEL = 0, 1, 2
OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NUMERIC, ERR_INTERNAL = 0, 1, 2, 3, 4, 5

EXPORTED = [
    "dmrg2_create", "dmrg2_destroy", "dmrg2_set_mpo", "dmrg2_set_mps", "dmrg2_init_mps",
    "dmrg2_run", "dmrg2_get_energy", "dmrg2_get_env_build_seconds", "dmrg2_get_bond_dims",
    "dmrg2_get_mps", "dmrg2_expect_local", "dmrg2_get_device_bytes", "dmrg2_last_error",
    "dmrg2_abi_version", "dmrg2_op_heff", "dmrg2_op_env_left", "dmrg2_op_env_right",
    "dmrg2_op_svd", "dmrg2_op_lanczos", "dmrg2_op_gemm", "dmrg2_resume", "dmrg2_pdmrg_run", "dmrg2_get_launch_count",
    "dmrg2_op_heff_noalloc", "dmrg2_server_create", "dmrg2_server_submit", "dmrg2_server_poll",
    "dmrg2_server_destroy", "dmrg2_op_gemm_bf16x3", "dmrg2_op_warm_split",
]
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3


class Dmrg2Error(RuntimeError):
    pass


class Config(ctypes.Structure):
    _fields_ = [
        ("L", ctypes.c_int), ("d", ctypes.c_int), ("chi_max", ctypes.c_int), ("dtype", ctypes.c_int),
        ("tol", ctypes.c_double), ("krylov_max", ctypes.c_int), ("lanczos_tol", ctypes.c_double),
        ("max_restarts", ctypes.c_int), ("cutoff", ctypes.c_double), ("min_sweeps", ctypes.c_int),
        ("device", ctypes.c_int), ("seed", ctypes.c_uint64), ("svd_method", ctypes.c_int),
        ("precision", ctypes.c_int), ("single_site", ctypes.c_int), ("truncation", ctypes.c_int),
    ]


class SweepReport(ctypes.Structure):
    _fields_ = [
        ("sweep", ctypes.c_int), ("chi_max", ctypes.c_int), ("energy", ctypes.c_double),
        ("trunc_err_max", ctypes.c_double), ("trunc_err_sum", ctypes.c_double),
        ("max_bond", ctypes.c_int), ("wall_s", ctypes.c_double), ("matvecs", ctypes.c_longlong),
        ("heff_s", ctypes.c_double), ("heff_flops", ctypes.c_double),
        ("lanczos_iters", ctypes.c_longlong), ("lanczos_unconverged", ctypes.c_int),
        ("svd_s", ctypes.c_double), ("jacobi_sweeps_max", ctypes.c_int), ("device_s", ctypes.c_double),
        ("lowprec_matvecs", ctypes.c_longlong), ("warm_splits", ctypes.c_int), ("warm_fallbacks", ctypes.c_int),
        ("eig_fallbacks", ctypes.c_int), ("warm_short", ctypes.c_int), ("rsvd_splits", ctypes.c_int),
        ("rsvd_fallbacks", ctypes.c_int), ("phase", ctypes.c_int), ("device_loops", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PdmrgOptions(ctypes.Structure):
    _fields_ = [("n_segments", ctypes.c_int), ("n_outer", ctypes.c_int), ("n_local", ctypes.c_int),
                ("n_warmup", ctypes.c_int), ("n_polish", ctypes.c_int), ("n_recal", ctypes.c_int),
                ("chi", ctypes.c_int)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("max_active", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_size_t)]


class Request(ctypes.Structure):
    _fields_ = [
        ("cfg", Config), ("W", ctypes.POINTER(ctypes.c_void_p)), ("Dl", ctypes.POINTER(ctypes.c_int)),
        ("Dr", ctypes.POINTER(ctypes.c_int)), ("A", ctypes.POINTER(ctypes.c_void_p)),
        ("bond_dims", ctypes.POINTER(ctypes.c_int)), ("init_kind", ctypes.c_int),
        ("schedule", ctypes.POINTER(ctypes.c_int)), ("n_sweeps", ctypes.c_int),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("state", ctypes.c_int), ("status", ctypes.c_int), ("energy", ctypes.c_double),
        ("sweeps", ctypes.c_int), ("trunc_err_max", ctypes.c_double), ("max_bond", ctypes.c_int),
        ("device_s", ctypes.c_double), ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double),
        ("t_done", ctypes.c_double), ("footprint_bytes", ctypes.c_size_t), ("message", ctypes.c_char * 256),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "message"}
        d["message"] = self.message.decode(errors="replace")
        return d


_lib = None


def load_library(path: str | os.PathLike | None = None):
    """Load (once) and return the ctypes handle of libdmrg2_b200.so."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise Dmrg2Error(f"{p} not built; run dmrg-implementations_b200/build.py")
    lib = ctypes.CDLL(str(p))
    vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    c_int, c_dbl = ctypes.c_int, ctypes.c_double
    sig = {
        "dmrg2_create": (c_int, [ctypes.POINTER(Config), ctypes.POINTER(vp)]),
        "dmrg2_destroy": (None, [vp]),
        "dmrg2_set_mpo": (c_int, [vp, ctypes.POINTER(vp), ip, ip, c_int]),
        "dmrg2_set_mps": (c_int, [vp, ctypes.POINTER(vp), ip, c_int]),
        "dmrg2_init_mps": (c_int, [vp, c_int, ctypes.c_uint64]),
        "dmrg2_run": (c_int, [vp, ip, c_int, ctypes.POINTER(SweepReport), c_int, ip]),
        "dmrg2_resume": (c_int, [vp, ip, c_int, ctypes.POINTER(SweepReport), c_int, ip]),
        "dmrg2_pdmrg_run": (c_int, [vp, ctypes.POINTER(PdmrgOptions), ctypes.POINTER(SweepReport), c_int, ip]),
        "dmrg2_get_launch_count": (ctypes.c_longlong, []),
        "dmrg2_get_energy": (c_int, [vp, dp]),
        "dmrg2_get_env_build_seconds": (c_int, [vp, dp]),
        "dmrg2_get_bond_dims": (c_int, [vp, ip]),
        "dmrg2_get_mps": (c_int, [vp, ctypes.POINTER(vp), c_int]),
        "dmrg2_expect_local": (c_int, [vp, vp, dp, dp]),
        "dmrg2_get_device_bytes": (c_int, [vp, ctypes.POINTER(ctypes.c_size_t)]),
        "dmrg2_last_error": (ctypes.c_char_p, [vp]),
        "dmrg2_abi_version": (c_int, []),
        "dmrg2_op_warm_split": (c_int, [c_int, c_int, c_int, vp, vp, c_int, ctypes.c_char, vp, vp, dp]),
        "dmrg2_op_heff": (c_int, [c_int] * 7 + [vp] * 6),
        "dmrg2_op_heff_noalloc": (c_int, [c_int] * 7 + [vp] * 7),
        "dmrg2_op_env_left": (c_int, [c_int] * 6 + [vp] * 4),
        "dmrg2_op_env_right": (c_int, [c_int] * 6 + [vp] * 4),
        "dmrg2_op_svd": (c_int, [c_int, c_int, c_int, vp, c_int, c_dbl, ctypes.c_char, dp, vp, vp, ip, dp]),
        "dmrg2_op_lanczos": (c_int, [c_int] * 7 + [vp] * 5 + [c_int, c_dbl, c_int, dp, ip]),
        "dmrg2_op_gemm": (c_int, [c_int] * 6 + [dp, vp, ctypes.c_longlong, vp, ctypes.c_longlong, dp, vp,
                                               ctypes.c_longlong]),
        "dmrg2_op_gemm_bf16x3": (c_int, [c_int] * 6 + [dp, vp, ctypes.c_longlong, vp, ctypes.c_longlong, dp,
                                                      vp, ctypes.c_longlong]),
        "dmrg2_server_create": (c_int, [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]),
        "dmrg2_server_submit": (c_int, [vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_longlong)]),
        "dmrg2_server_poll": (c_int, [vp, ctypes.c_longlong, c_int, ctypes.POINTER(Result)]),
        "dmrg2_server_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def launch_count():
    """Kernels launched by libdmrg2_b200.so in this process."""
    return int(load_library().dmrg2_get_launch_count())


def _err(handle=None):
    msg = load_library().dmrg2_last_error(handle)
    return msg.decode() if msg else "unknown error"


def _check(rc, handle=None, what=""):
    if rc != 0:
        raise Dmrg2Error(f"{what} failed (status {rc}): {_err(handle)}")


def _dtype_code(*arrays):
    return C128 if any(np.iscomplexobj(a) for a in arrays) else F64


def _prep(a, code):
    return np.ascontiguousarray(a, dtype=np.complex128 if code == C128 else np.float64)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def minimal_bonds(As):
    """The same MPS with every bond at most min(d^i, d^(L-i)) (exact QR sweeps, no truncation).

    Generators such as quimb's random MPS keep one bond dimension on every bond, above
    what the first and last sites can carry; the engine allocates the minimal bonds.
    """
    As = [np.asarray(A) for A in As]
    L = len(As)
    if L < 2:
        return As
    for i in range(L - 1):  # left to right: bond i+1 <= chi_l * d
        cl, d, cr = As[i].shape
        if cr > cl * d:
            Q, R = np.linalg.qr(As[i].reshape(cl * d, cr))
            As[i] = Q.reshape(cl, d, Q.shape[1])
            As[i + 1] = np.tensordot(R, As[i + 1], axes=(1, 0))
    for i in range(L - 1, 0, -1):  # right to left: bond i <= d * chi_r
        cl, d, cr = As[i].shape
        if cl > d * cr:
            Q, R = np.linalg.qr(As[i].reshape(cl, d * cr).T)
            As[i] = Q.T.reshape(Q.shape[1], d, cr)
            As[i - 1] = np.tensordot(As[i - 1], R.T, axes=(2, 0))
    return [np.ascontiguousarray(A) for A in As]


def _mpo4(Ws):
    """Accept boundary tensors given as 3-D arrays (npz fixture format)."""
    L = len(Ws)
    out = []
    for i, W in enumerate(Ws):
        W = np.asarray(W)
        if W.ndim == 3 and i == 0:
            W = W[None]
        elif W.ndim == 3 and i == L - 1:
            W = W[:, None]
        out.append(W)
    return out


# ----------------------------------------------------------------------------
# solver
# ----------------------------------------------------------------------------
class DMRG2GPU:
    """Two-site DMRG on one B200 (mirror of DMRG2GPU<Scalar>, dmrg2_gpu.h:24-203)."""

    def __init__(self, L, d, chi_max, D_mpo=None, tol=1e-10, dtype=np.float64, *, krylov_max=100,
                 lanczos_tol=1e-12, max_restarts=0, cutoff=1e-14, min_sweeps=2, device=0, seed=42,
                 svd_method=0, precision=0, single_site=False, truncation=0):
        lib = load_library()
        self.L, self.d, self.chi_max, self.D_mpo = int(L), int(d), int(chi_max), D_mpo
        self.dtype = np.dtype(dtype)
        self.code = C128 if self.dtype.kind == "c" else F64
        cfg = Config(L=self.L, d=self.d, chi_max=self.chi_max, dtype=self.code, tol=tol,
                     krylov_max=krylov_max, lanczos_tol=lanczos_tol, max_restarts=max_restarts,
                     cutoff=(cutoff if cutoff > 0 else -1.0), min_sweeps=min_sweeps, device=device,
                     seed=seed, svd_method=svd_method, precision=int(precision),
                     single_site=int(bool(single_site)), truncation=int(truncation))
        h = ctypes.c_void_p()
        _check(lib.dmrg2_create(ctypes.byref(cfg), ctypes.byref(h)), None, "dmrg2_create")
        self._h = h
        self._lib = lib
        self.reports = []

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dmrg2_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- inputs
    def set_mpo(self, Ws):
        """Row-major MPO tensors (Dl, Dr, d, d) = (mpo_l, mpo_r, s_in, s_out)."""
        Ws = [_prep(W, self.code) for W in _mpo4(Ws)]
        ptrs = (ctypes.c_void_p * self.L)(*[W.ctypes.data for W in Ws])
        Dl = (ctypes.c_int * self.L)(*[W.shape[0] for W in Ws])
        Dr = (ctypes.c_int * self.L)(*[W.shape[1] for W in Ws])
        self._keep_mpo = Ws
        _check(self._lib.dmrg2_set_mpo(self._h, ptrs, Dl, Dr, ROWMAJOR), self._h, "set_mpo")

    def set_mpo_reference(self, flat_tensors, D_mpo):
        """Reference-layout MPO: flat column-major W[w + s*D + sp*D*d + wp*D*d*d] per site."""
        Ws = [_prep(np.ravel(W), self.code) for W in flat_tensors]
        ptrs = (ctypes.c_void_p * self.L)(*[W.ctypes.data for W in Ws])
        Dl = (ctypes.c_int * 1)(int(D_mpo))
        _check(self._lib.dmrg2_set_mpo(self._h, ptrs, Dl, None, REFERENCE), self._h, "set_mpo")

    def set_mps(self, As):
        As = minimal_bonds([_prep(A, self.code) for A in As])
        dims = [As[0].shape[0]] + [A.shape[2] for A in As]
        ptrs = (ctypes.c_void_p * self.L)(*[A.ctypes.data for A in As])
        cd = (ctypes.c_int * (self.L + 1))(*dims)
        _check(self._lib.dmrg2_set_mps(self._h, ptrs, cd, ROWMAJOR), self._h, "set_mps")

    def initialize_mps_random(self, seed=0):
        _check(self._lib.dmrg2_init_mps(self._h, INIT_RANDOM, seed), self._h, "init_mps")

    def initialize_mps_product(self):
        _check(self._lib.dmrg2_init_mps(self._h, INIT_PRODUCT, 0), self._h, "init_mps")

    def initialize_mps_neel(self):
        _check(self._lib.dmrg2_init_mps(self._h, INIT_NEEL, 0), self._h, "init_mps")

    # -- solve
    def run(self, n_sweeps=None, schedule=None):
        """Run sweeps; returns a list of per-sweep report dicts (also in self.reports)."""
        if schedule is None:
            schedule = [self.chi_max] * int(n_sweeps if n_sweeps is not None else 10)
        schedule = [int(c) for c in schedule]
        n = len(schedule)
        sch = (ctypes.c_int * n)(*schedule)
        rep = (SweepReport * n)()
        nout = ctypes.c_int(0)
        _check(self._lib.dmrg2_run(self._h, sch, n, rep, n, ctypes.byref(nout)), self._h, "run")
        self.reports = [rep[i].as_dict() for i in range(nout.value)]
        return self.reports

    def resume(self, schedule):
        """Continue sweeping from the current state (no environment rebuild, no stop rule)."""
        schedule = [int(c) for c in schedule]
        n = len(schedule)
        sch = (ctypes.c_int * n)(*schedule)
        rep = (SweepReport * n)()
        nout = ctypes.c_int(0)
        _check(self._lib.dmrg2_resume(self._h, sch, n, rep, n, ctypes.byref(nout)), self._h, "resume")
        out = [rep[i].as_dict() for i in range(nout.value)]
        self.reports += out
        return out

    def pdmrg(self, n_segments=2, n_outer=20, n_local=2, n_warmup=1, n_polish=0, n_recal=0, chi=None):
        """Parallel (segmented) sweeps with boundary merges: PDMRGGPU::run(n_outer, n_local,
        n_warmup, n_polish, n_recal) with n_segments segments (gpu-rocm/pdmrg-gpu/src/
        pdmrg_gpu.h:24-40). Returns one report per full sweep and per outer iteration (phase
        1 warm-up, 2 outer, 3 recalibration, 4 polish); energy() is the last merge's."""
        opt = PdmrgOptions(n_segments=int(n_segments), n_outer=int(n_outer), n_local=int(n_local),
                           n_warmup=int(n_warmup), n_polish=int(n_polish), n_recal=int(n_recal),
                           chi=int(chi or 0))
        cap = int(n_warmup) + int(n_outer) * (1 + int(n_recal > 0)) + int(n_polish) + 1
        rep = (SweepReport * cap)()
        nout = ctypes.c_int(0)
        _check(self._lib.dmrg2_pdmrg_run(self._h, ctypes.byref(opt), rep, cap, ctypes.byref(nout)), self._h,
               "pdmrg")
        out = [rep[i].as_dict() for i in range(min(nout.value, cap))]
        self.reports += out
        return out

    # -- outputs
    def get_energy(self):
        e = ctypes.c_double()
        _check(self._lib.dmrg2_get_energy(self._h, ctypes.byref(e)), self._h, "get_energy")
        return e.value

    def env_build_seconds(self):
        e = ctypes.c_double()
        _check(self._lib.dmrg2_get_env_build_seconds(self._h, ctypes.byref(e)), self._h, "env")
        return e.value

    def bond_dims(self):
        b = (ctypes.c_int * (self.L + 1))()
        _check(self._lib.dmrg2_get_bond_dims(self._h, b), self._h, "get_bond_dims")
        return list(b)

    def chi_L(self, site):
        return self.bond_dims()[site]

    def chi_R(self, site):
        return self.bond_dims()[site + 1]

    def get_mps(self):
        dims = self.bond_dims()
        dt = np.complex128 if self.code == C128 else np.float64
        out = [np.empty((dims[i], self.d, dims[i + 1]), dt) for i in range(self.L)]
        ptrs = (ctypes.c_void_p * self.L)(*[A.ctypes.data for A in out])
        _check(self._lib.dmrg2_get_mps(self._h, ptrs, ROWMAJOR), self._h, "get_mps")
        return out

    def expect_local(self, op):
        op = _prep(op, self.code)
        re = np.zeros(self.L)
        im = np.zeros(self.L)
        _check(self._lib.dmrg2_expect_local(self._h, _ptr(op), re.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            im.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
               self._h, "expect_local")
        return re + 1j * im if self.code == C128 else re

    def device_bytes(self):
        b = ctypes.c_size_t()
        _check(self._lib.dmrg2_get_device_bytes(self._h, ctypes.byref(b)), self._h, "device_bytes")
        return b.value


# ----------------------------------------------------------------------------
# primitives (same signatures as the reference's numpy functions)
# ----------------------------------------------------------------------------

class PDMRGGPU(DMRG2GPU):
    """Parallel DMRG on one B200 (mirror of PDMRGGPU<Scalar>, gpu-rocm/pdmrg-gpu/src/
    pdmrg_gpu.h:24-62): the chain in n_segments segments swept concurrently (one stream and
    scratch lane each), coupled by boundary merges with V = 1/S. tol is the outer stop rule."""

    def __init__(self, L, d, chi_max, D_mpo=None, n_segments=2, tol=1e-10, dtype=np.float64, **kw):
        super().__init__(L, d, chi_max, D_mpo, tol=tol, dtype=dtype, **kw)
        self.n_segments = int(n_segments)

    def run(self, n_outer_sweeps=20, n_local_sweeps=2, n_warmup=1, n_polish=0, n_recal=0):
        """PDMRGGPU::run(n_outer_sweeps, n_local_sweeps, n_warmup, n_polish, n_recal)
        (pdmrg_gpu_impl.h:2585-2760); returns the energy."""
        self.pdmrg(self.n_segments, n_outer_sweeps, n_local_sweeps, n_warmup, n_polish, n_recal)
        return self.get_energy()


def apply_heff(L_env, R_env, W_left, W_right, theta):
    code = _dtype_code(L_env, R_env, W_left, W_right, theta)
    L_env, R_env, W_left, W_right, theta = (_prep(a, code) for a in (L_env, R_env, W_left, W_right, theta))
    cL, Dl, _ = L_env.shape
    cR, Dr, _ = R_env.shape
    d = theta.shape[1]
    Dm = W_left.shape[1]
    out = np.empty_like(theta)
    _check(load_library().dmrg2_op_heff(code, cL, cR, d, Dl, Dm, Dr, _ptr(L_env), _ptr(R_env),
                                        _ptr(W_left), _ptr(W_right), _ptr(theta), _ptr(out)),
           None, "op_heff")
    return out


def update_left_env(L_env, A, W):
    code = _dtype_code(L_env, A, W)
    L_env, A, W = (_prep(a, code) for a in (L_env, A, W))
    cL, Dl, _ = L_env.shape
    _, d, cO = A.shape
    Dr = W.shape[1]
    out = np.empty((cO, Dr, cO), L_env.dtype)
    _check(load_library().dmrg2_op_env_left(code, cL, cO, d, Dl, Dr, _ptr(L_env), _ptr(A), _ptr(W),
                                            _ptr(out)), None, "op_env_left")
    return out


def update_right_env(R_env, B, W):
    code = _dtype_code(R_env, B, W)
    R_env, B, W = (_prep(a, code) for a in (R_env, B, W))
    cI, Dr, _ = R_env.shape
    cO, d, _ = B.shape
    Dl = W.shape[0]
    out = np.empty((cO, Dl, cO), R_env.dtype)
    _check(load_library().dmrg2_op_env_right(code, cI, cO, d, Dl, Dr, _ptr(R_env), _ptr(B), _ptr(W),
                                             _ptr(out)), None, "op_env_right")
    return out


def truncated_svd(M, max_bond, cutoff=0.0, direction="R", method="eig"):
    """Truncated SVD split: returns (left, S, right, trunc_err).

    direction 'R': left = U (isometric columns), right = diag(S) @ Vh.
    direction 'L': left = U @ diag(S), right = Vh (isometric rows).
    S holds all min(m, n) singular values in descending order.
    method 'eig' (default): density-matrix eigensolver; 'jacobi': block Jacobi SVD.
    """
    if method == "jacobi":
        direction = direction.lower()
    code = _dtype_code(M)
    M = _prep(M, code)
    m, n = M.shape
    kmin = min(m, n)
    S = np.zeros(kmin)
    left = np.zeros(m * kmin, M.dtype)
    right = np.zeros(kmin * n, M.dtype)
    k = ctypes.c_int()
    te = ctypes.c_double()
    _check(load_library().dmrg2_op_svd(code, m, n, _ptr(M), int(max_bond), float(cutoff),
                                       direction.encode()[:1], S.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       _ptr(left), _ptr(right), ctypes.byref(k), ctypes.byref(te)),
           None, "op_svd")
    k = k.value
    return left[: m * k].reshape(m, k), S, right[: k * n].reshape(k, n), te.value


def warm_split(M, warm, k, direction="R"):
    """Warm-started subspace split of the real M at rank k from the orthonormal factor
    `warm` of a previous split (k x n rows for 'R', m x k columns for 'L'); returns
    (left, right, trunc_err)."""
    M = _prep(M, F64)
    warm = _prep(warm, F64)
    m, n = M.shape
    left = np.zeros((m, k))
    right = np.zeros((k, n))
    te = ctypes.c_double()
    _check(load_library().dmrg2_op_warm_split(F64, m, n, _ptr(M), _ptr(warm), int(k), direction.encode()[:1],
                                              _ptr(left), _ptr(right), ctypes.byref(te)), None, "op_warm_split")
    return left, right, te.value


def optimize_two_site(L_env, R_env, W_left, W_right, theta_init, max_iter=100, tol=1e-12,
                      max_restarts=4):
    """Lanczos ground state of H_eff; returns (energy, theta) like eigensolver.py."""
    code = _dtype_code(L_env, R_env, W_left, W_right, theta_init)
    L_env, R_env, W_left, W_right = (_prep(a, code) for a in (L_env, R_env, W_left, W_right))
    th = _prep(theta_init, code).copy()
    cL, Dl, _ = L_env.shape
    cR, Dr, _ = R_env.shape
    d = th.shape[1]
    Dm = W_left.shape[1]
    e = ctypes.c_double()
    it = ctypes.c_int()
    _check(load_library().dmrg2_op_lanczos(code, cL, cR, d, Dl, Dm, Dr, _ptr(L_env), _ptr(R_env),
                                           _ptr(W_left), _ptr(W_right), _ptr(th), int(max_iter),
                                           float(tol), int(max_restarts), ctypes.byref(e), ctypes.byref(it)),
           None, "op_lanczos")
    return e.value, th


_TRANS = {"N": 0, "T": 1, "C": 2, "R": 3}


def gemm(A, B, transA="N", transB="N", alpha=1.0, beta=0.0, C=None):
    """C = alpha * op(A) @ op(B) + beta * C on the FP64 tensor cores."""
    code = _dtype_code(A, B) if C is None else _dtype_code(A, B, C)
    A, B = _prep(A, code), _prep(B, code)
    M = A.shape[1] if transA in ("T", "C") else A.shape[0]
    K = A.shape[0] if transA in ("T", "C") else A.shape[1]
    N = B.shape[0] if transB in ("T", "C") else B.shape[1]
    C = np.zeros((M, N), A.dtype) if C is None else _prep(C, code).copy()
    al = (ctypes.c_double * 2)(complex(alpha).real, complex(alpha).imag)
    be = (ctypes.c_double * 2)(complex(beta).real, complex(beta).imag)
    _check(load_library().dmrg2_op_gemm(code, _TRANS[transA], _TRANS[transB], M, N, K, al, _ptr(A),
                                        A.shape[1], _ptr(B), B.shape[1], be, _ptr(C), C.shape[1]),
           None, "op_gemm")
    return C


def gemm_bf16x3(A, B, transA="N", transB="N", alpha=1.0, beta=0.0, C=None):
    """The same product in the precision form: three-term BF16 split of each operand,
    FP32 accumulation on the tcgen05 tensor cores, FP64 result (real alpha, beta)."""
    code = _dtype_code(A, B) if C is None else _dtype_code(A, B, C)
    A, B = _prep(A, code), _prep(B, code)
    M = A.shape[1] if transA in ("T", "C") else A.shape[0]
    K = A.shape[0] if transA in ("T", "C") else A.shape[1]
    N = B.shape[0] if transB in ("T", "C") else B.shape[1]
    C = np.zeros((M, N), A.dtype) if C is None else _prep(C, code).copy()
    al = (ctypes.c_double * 2)(float(np.real(alpha)), float(np.imag(alpha)))
    be = (ctypes.c_double * 2)(float(np.real(beta)), float(np.imag(beta)))
    _check(load_library().dmrg2_op_gemm_bf16x3(code, _TRANS[transA], _TRANS[transB], M, N, K, al, _ptr(A),
                                               A.shape[1], _ptr(B), B.shape[1], be, _ptr(C), C.shape[1]),
           None, "op_gemm_bf16x3")
    return C


# ----------------------------------------------------------------------------
# served / batched form
# ----------------------------------------------------------------------------
class Server:
    """Many independent ground-state solves on one device (dmrg2_server_*).

    Requests are admitted in arrival order while one of ``max_active`` slots is
    idle and their device footprint fits ``hbm_budget_bytes``; admitted solves run
    concurrently, each on its own CUDA stream.
    """

    def __init__(self, device=0, max_active=8, hbm_budget_bytes=0):
        self._lib = load_library()
        self._s = ctypes.c_void_p()
        cfg = ServerConfig(int(device), int(max_active), int(hbm_budget_bytes))
        _check(self._lib.dmrg2_server_create(ctypes.byref(cfg), ctypes.byref(self._s)), None, "server_create")

    def submit(self, mpo, schedule, mps=None, init=INIT_RANDOM, seed=0, dtype=None, tol=1e-10,
               krylov_max=30, lanczos_tol=1e-12, max_restarts=2, cutoff=1e-14, min_sweeps=2, chi_max=None,
               precision=0, truncation=0):
        """Queue one solve; returns its id. mpo: L tensors (Dl, Dr, d, d)."""
        Ws = _mpo4(mpo)
        L, d = len(Ws), Ws[0].shape[2]
        cplx = dtype == np.complex128 or any(np.iscomplexobj(w) for w in Ws) or (
            mps is not None and any(np.iscomplexobj(a) for a in mps))
        code = C128 if cplx else F64
        Ws = [_prep(w, code) for w in Ws]
        sched = (ctypes.c_int * len(schedule))(*[int(c) for c in schedule])
        cfg = Config()
        cfg.L, cfg.d, cfg.chi_max, cfg.dtype = L, d, int(chi_max or max(schedule)), code
        cfg.tol, cfg.krylov_max, cfg.lanczos_tol = tol, krylov_max, lanczos_tol
        cfg.max_restarts, cfg.min_sweeps, cfg.seed = max_restarts, min_sweeps, int(seed)
        cfg.cutoff = cutoff if cutoff > 0 else -1.0
        cfg.precision = int(precision)
        cfg.truncation = int(truncation)
        wp = (ctypes.c_void_p * L)(*[w.ctypes.data for w in Ws])
        Dl = (ctypes.c_int * L)(*[w.shape[0] for w in Ws])
        Dr = (ctypes.c_int * L)(*[w.shape[1] for w in Ws])
        req = Request()
        req.cfg, req.W, req.Dl, req.Dr = cfg, wp, Dl, Dr
        keep = [Ws]
        if mps is not None:
            As = minimal_bonds([_prep(a, code) for a in mps])
            keep.append(As)
            req.A = (ctypes.c_void_p * L)(*[a.ctypes.data for a in As])
            req.bond_dims = (ctypes.c_int * (L + 1))(*([1] + [a.shape[2] for a in As]))
        req.init_kind, req.schedule, req.n_sweeps = int(init), sched, len(schedule)
        rid = ctypes.c_longlong()
        _check(self._lib.dmrg2_server_submit(self._s, ctypes.byref(req), ctypes.byref(rid)), None, "server_submit")
        del keep
        return rid.value

    def poll(self, rid, wait=0.0):
        """Result dict of request rid; waits up to `wait` seconds (None: until finished)."""
        r = Result()
        ms = -1 if wait is None else int(wait * 1000)
        _check(self._lib.dmrg2_server_poll(self._s, ctypes.c_longlong(rid), ms, ctypes.byref(r)), None,
               "server_poll")
        return r.as_dict()

    def result(self, rid):
        return self.poll(rid, wait=None)

    def close(self):
        if getattr(self, "_s", None):
            self._lib.dmrg2_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
