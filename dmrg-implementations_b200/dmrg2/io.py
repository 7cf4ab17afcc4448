"""MPS / MPO file formats of the reference's benchmark data, and checkpoints.

Formats (readers and writers follow benchmarks/lib/data_loader.py:24-152 and
benchmarks/data/generate.py:23-101 of the reference):

* ``.bin`` MPS: int64 L, int64 bond_dims[L+1], int64 phys_dims[L], then per
  site int64 shape[3] = (D_left, d, D_right) and the complex128 tensor in C order.
* ``.bin`` MPO: int64 L, int64 mpo_bond_dims[L+1], int64 phys_dims[L], then per
  site int64 shape[4] = (D_left, d_up, d_down, D_right) and complex128 data.
  The up index is the operator's output (quimb's upper/ket index, the rows of
  the operator matrix), the down index its input.
* ``.npz`` MPO (benchmark_data/): ``tensor_i`` with boundary tensors (D, d, d)
  and bulk tensors (Dl, Dr, d, d) in (mpo_l, mpo_r, s_in, s_out) order.
* ``.npz`` MPS: ``tensor_i`` as (chi_l, d, chi_r) with end tensors (d, chi) and
  (chi, d); quimb-ordered files (chi_l, chi_r, d) are detected and transposed.
  A pickled ``metadata`` entry, when present, is skipped (no pickle loading).

Everything returns the engine's layout: MPS (chi_l, d, chi_r) with unit end
bonds, MPO (Dl, Dr, s_in, s_out).
"""
from __future__ import annotations

import numpy as np


# ---------------------------------------------------------------------------- .bin
def _read_header(f, count):
    a = np.fromfile(f, dtype=np.int64, count=count)
    if a.size != count:
        raise ValueError("truncated .bin header")
    return a


def load_mps_bin(path):
    """MPS from a .bin file -> list of complex128 (chi_l, d, chi_r) tensors."""
    with open(path, "rb") as f:
        L = int(_read_header(f, 1)[0])
        bonds = _read_header(f, L + 1)
        phys = _read_header(f, L)
        out = []
        for i in range(L):
            shape = tuple(int(x) for x in _read_header(f, 3))
            if shape != (bonds[i], phys[i], bonds[i + 1]):
                raise ValueError(f"site {i}: shape {shape} disagrees with the header")
            n = int(np.prod(shape))
            data = np.fromfile(f, dtype=np.complex128, count=n)
            if data.size != n:
                raise ValueError(f"site {i}: truncated tensor data")
            out.append(data.reshape(shape))
    return out


def save_mps_bin(path, mps):
    """Write MPS tensors (chi_l, d, chi_r) as a .bin file (complex128)."""
    mps = [np.asarray(a, dtype=np.complex128) for a in mps]
    with open(path, "wb") as f:
        np.array([len(mps)], np.int64).tofile(f)
        np.array([mps[0].shape[0]] + [a.shape[2] for a in mps], np.int64).tofile(f)
        np.array([a.shape[1] for a in mps], np.int64).tofile(f)
        for a in mps:
            np.array(a.shape, np.int64).tofile(f)
            np.ascontiguousarray(a).tofile(f)


def load_mpo_bin(path):
    """MPO from a .bin file -> list of complex128 (Dl, Dr, s_in, s_out) tensors."""
    with open(path, "rb") as f:
        L = int(_read_header(f, 1)[0])
        bonds = _read_header(f, L + 1)
        phys = _read_header(f, L)
        out = []
        for i in range(L):
            shape = tuple(int(x) for x in _read_header(f, 4))
            if shape != (bonds[i], phys[i], phys[i], bonds[i + 1]):
                raise ValueError(f"site {i}: shape {shape} disagrees with the header")
            n = int(np.prod(shape))
            data = np.fromfile(f, dtype=np.complex128, count=n)
            if data.size != n:
                raise ValueError(f"site {i}: truncated tensor data")
            t = data.reshape(shape)  # (Dl, s_out, s_in, Dr)
            out.append(np.ascontiguousarray(t.transpose(0, 3, 2, 1)))
    return out


def save_mpo_bin(path, mpo):
    """Write MPO tensors (Dl, Dr, s_in, s_out) as a .bin file (complex128)."""
    mpo = [np.asarray(w, dtype=np.complex128) for w in mpo]
    with open(path, "wb") as f:
        np.array([len(mpo)], np.int64).tofile(f)
        np.array([mpo[0].shape[0]] + [w.shape[1] for w in mpo], np.int64).tofile(f)
        np.array([w.shape[2] for w in mpo], np.int64).tofile(f)
        for w in mpo:
            t = np.ascontiguousarray(w.transpose(0, 3, 2, 1))  # (Dl, s_out, s_in, Dr)
            np.array(t.shape, np.int64).tofile(f)
            t.tofile(f)


# ---------------------------------------------------------------------------- .npz
def _npz_tensors(path):
    with np.load(path, allow_pickle=False) as z:
        keys = sorted((k for k in z.files if k.startswith("tensor_")), key=lambda k: int(k.split("_")[1]))
        return [np.asarray(z[k]) for k in keys]


def load_mpo_npz(path):
    """benchmark_data MPO (.npz) -> (Dl, Dr, s_in, s_out) tensors with unit end bonds."""
    ts = _npz_tensors(path)
    L = len(ts)
    out = []
    for i, t in enumerate(ts):
        if t.ndim == 3:
            t = t[None] if i == 0 else t[:, None]
        elif t.ndim != 4:
            raise ValueError(f"tensor_{i}: expected 3 or 4 axes, got {t.ndim}")
        out.append(np.ascontiguousarray(t))
    if out[0].shape[0] != 1 or out[L - 1].shape[1] != 1:
        raise ValueError("MPO end tensors must have unit outer bonds")
    return out


def load_mps_npz(path):
    """benchmark_data MPS (.npz) -> (chi_l, d, chi_r) tensors with unit end bonds.

    Bulk tensors are (chi_l, d, chi_r) (regular tier) or quimb's (chi_l, chi_r, d)
    (challenge tier); the order is the one under which consecutive bulk tensors
    chain and share one physical dimension. End tensors are 2-D.
    """
    ts = _npz_tensors(path)
    L = len(ts)
    bulk = ts[1:-1]

    def chains(perm):
        sh = [tuple(t.shape[k] for k in perm) for t in bulk]
        return all(sh[i][2] == sh[i + 1][0] for i in range(len(sh) - 1)) and len({x[1] for x in sh}) <= 1

    quimb = bool(bulk) and not chains((0, 1, 2)) and chains((0, 2, 1))
    out = [np.ascontiguousarray(t.transpose(0, 2, 1) if quimb else t) for t in bulk]
    first, last = ts[0], ts[-1]
    if L == 1:
        return [np.ascontiguousarray(first.reshape(1, -1, 1))]
    # end tensors: 3-D ones (engine checkpoints) follow the bulk order, 2-D ones are
    # (d, chi) / (chi, d) or their transposes
    nxt = out[0].shape[0] if out else None
    if first.ndim == 3:
        f3 = first.transpose(0, 2, 1) if quimb else first
    else:
        f = first.T if quimb else first  # -> (d, chi_r)
        if nxt is not None and f.shape[1] != nxt and f.shape[0] == nxt:
            f = f.T
        f3 = f[None]
    prv = out[-1].shape[2] if out else f3.shape[2]
    if last.ndim == 3:
        l3 = last.transpose(0, 2, 1) if quimb else last
    else:
        l3 = (last if last.shape[0] == prv else last.T)[:, :, None]  # (chi_l, d) -> (chi_l, d, 1)
    res = [np.ascontiguousarray(f3)] + out + [np.ascontiguousarray(l3)]
    for i in range(L - 1):
        if res[i].shape[2] != res[i + 1].shape[0]:
            raise ValueError(f"bond {i + 1}: {res[i].shape} does not chain with {res[i + 1].shape}")
    return res


def save_mps_npz(path, mps, **meta):
    """Checkpoint an MPS as .npz (tensor_i in (chi_l, d, chi_r) order, plus scalar metadata)."""
    arrays = {f"tensor_{i}": np.ascontiguousarray(a) for i, a in enumerate(mps)}
    for k, v in meta.items():
        arrays[k] = np.asarray(v)
    np.savez(path, **arrays)
