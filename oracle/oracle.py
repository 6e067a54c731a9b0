"""ctypes front-end of the CPU checkers (TEST INFRASTRUCTURE ONLY).

* ``liboracle.so``          -- FP64 restatement of the discord path (oracle.c).
* ``_ref/libpaddi_ref.so``  -- the reference's own CPU kernels
  (src/cpu_kernels/cpu_kernels.cpp) behind a C driver (ref_wrap.cpp).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module.  The product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference's source tree (only its src/cpu_kernels/cpu_kernels.cpp is
# compiled, into _ref/): PADDI_REF_SRC, else a PADDi checkout beside this
# repository.  Machines without it use the prebuilt library only.
REF_SRC = os.environ.get("PADDI_REF_SRC",
                         os.path.join(os.path.dirname(HERE), "..", "reference", "src"))
_LIB = None
_REF = None

FLT_MAX = float(np.finfo(np.float32).max)


class Discord(C.Structure):
    _fields_ = [("ind", C.c_int32), ("dist", C.c_float)]


class Attempt(C.Structure):
    _fields_ = [("m", C.c_int32), ("r", C.c_float), ("r2", C.c_float),
                ("n_cand", C.c_int64), ("n_disc", C.c_int64), ("found", C.c_int32),
                ("n_sel", C.c_int32), ("top", Discord)]

    def as_dict(self):
        return {"m": self.m, "r": self.r, "r2": self.r2, "n_cand": self.n_cand,
                "n_disc": self.n_disc, "found": self.found, "n_sel": self.n_sel,
                "top_ind": self.top.ind, "top_dist": self.top.dist}


def build() -> None:
    """Compile the checkers (the reference part only where its sources exist)."""
    target = "all" if has_ref_src() else os.path.join(HERE, "liboracle.so")
    subprocess.run(["make", "-s", "-C", HERE, target, f"REF_SRC={os.path.abspath(REF_SRC)}"],
                   check=True)


def has_ref_src() -> bool:
    return os.path.isfile(os.path.join(REF_SRC, "cpu_kernels", "cpu_kernels.cpp"))


def lib():
    global _LIB
    if _LIB is None:
        p = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(p):
            build()
        L = C.CDLL(p)
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
        u8p = np.ctypeslib.ndpointer(np.uint8, flags="C")
        L.or_window_stats.argtypes = [f32p, C.c_int64, C.c_int32, f64p, f64p, u8p]
        L.or_nn_profile.argtypes = [f32p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                    C.c_int32, f64p, i64p]
        L.or_pair_dist.argtypes = [f32p, C.c_int64, C.c_int32, C.c_int64, C.c_int64]
        L.or_pair_dist.restype = C.c_double
        L.or_window_nn.argtypes = [f32p, C.c_int64, C.c_int32, C.c_int64, C.POINTER(C.c_int64)]
        L.or_window_nn.restype = C.c_double
        L.or_select.argtypes = [f64p, C.c_int64, C.c_int32, C.c_float, C.c_int32,
                                C.POINTER(Attempt), C.POINTER(Discord)]
        L.or_palmad.argtypes = [f32p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                C.POINTER(Discord), C.POINTER(Attempt), C.c_int64, C.c_void_p]
        L.or_palmad.restype = C.c_int64
        L.or_pd3.argtypes = [f32p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                             C.POINTER(Discord), C.POINTER(Attempt), C.c_int64,
                             C.POINTER(C.c_int64), C.c_int32]
        L.or_lengths_nn.argtypes = [f32p, C.c_int64, C.c_int32, C.c_int32, i64p, f64p]
        L.or_pd3.restype = C.c_int32
        L.or_nn_profile_fast.argtypes = [f32p, C.c_int64, C.c_int32, f64p]
        L.or_windows_nn.argtypes = [f32p, C.c_int64, C.c_int32, i64p, C.c_int64, f64p, i64p]
        _LIB = L
    return _LIB


def ref():
    """The reference CPU kernels, or None when the prebuilt library is absent."""
    global _REF
    if _REF is None:
        p = os.path.join(HERE, "_ref", "libpaddi_ref.so")
        if not os.path.exists(p):
            if has_ref_src():
                build()
            else:
                return None
        R = C.CDLL(p)
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        R.ref_compute_statistics.argtypes = [f32p, f32p, f32p, C.c_uint32, C.c_uint32]
        R.ref_find_discords.argtypes = [f32p, f32p, f32p, i32p, f32p, C.c_uint32, C.c_float,
                                        C.c_uint32]
        R.ref_attempt_at.argtypes = [f32p, C.c_int64, C.c_int32, C.c_float,
                                     C.POINTER(Attempt), i32p, f32p]
        R.ref_palmad.argtypes = [f32p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                 C.POINTER(Discord), C.POINTER(Attempt), C.c_int64]
        R.ref_palmad.restype = C.c_int64
        R.ref_palmad_many.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_int64), C.c_int32,
                                      C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                      C.POINTER(Discord)]
        R.ref_palmad_many.restype = C.c_int64
        _REF = R
    return _REF


def refgpu():
    """The reference's FP32 GPU kernels (src/PD3_kernels.cuh, src/preprocessing.cuh)
    behind ref_gpu.cu, or None when the prebuilt library is absent."""
    p = os.path.join(HERE, "_ref", "libpaddi_refgpu.so")
    if not os.path.exists(p):
        if has_ref_src():
            build()
        else:
            return None
    G = C.CDLL(p)
    f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
    G.refgpu_palmad.argtypes = [f32p, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                C.POINTER(Discord), C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    G.refgpu_palmad.restype = C.c_int32
    return G


def refgpu_palmad(x, minL, maxL, max_attempts, iter_cap=200):
    """PALMAD with the reference's own FP32 GPU kernels and MERLIN schedule on
    the current CUDA device, up to the first length boundary after
    max_attempts attempts.  Returns (completed lengths' discords, attempts,
    device ms of those attempts)."""
    G = refgpu()
    if G is None:
        return None
    x = _f32(x)
    L = maxL - minL + 1
    out = (Discord * L)()
    na = C.c_int32(0)
    ms = C.c_double(0.0)
    done = G.refgpu_palmad(x, len(x), minL, maxL, iter_cap, max_attempts, out, C.byref(na),
                           C.byref(ms))
    if done < 0:
        raise RuntimeError(f"reference GPU path: CUDA error {-done}")
    return [(out[i].ind, out[i].dist) for i in range(done)], na.value, ms.value


def _f32(x):
    return np.ascontiguousarray(x, dtype=np.float32)


# ----------------------------------------------------------------- oracle
def window_stats(x, m):
    x = _f32(x)
    N = len(x) - m + 1
    mu = np.empty(N, np.float64)
    sd = np.empty(N, np.float64)
    flat = np.empty(N, np.uint8)
    lib().or_window_stats(x, len(x), m, mu, sd, flat)
    return mu, sd, flat.astype(bool)


def nn_profile(x, m, right_gap=None, left_gap=None, method=1):
    """FP64 squared nearest-neighbour distance and index of every window."""
    x = _f32(x)
    N = len(x) - m + 1
    nn = np.empty(N, np.float64)
    idx = np.empty(N, np.int64)
    rg = m - 1 if right_gap is None else right_gap
    lg = m - 1 if left_gap is None else left_gap
    lib().or_nn_profile(x, len(x), m, rg, lg, method, nn, idx)
    return nn, idx


def nn_profile_fast(x, m):
    """FP64 squared nn distance of every window (no index), for long series:
    vectorised diagonal blocks re-anchored every 8192 rows."""
    x = _f32(x)
    nn = np.empty(len(x) - m + 1, np.float64)
    lib().or_nn_profile_fast(x, len(x), m, nn)
    return nn


def windows_nn(x, m, windows):
    """FP64 nn (and nearest index) of each window in ``windows``, in parallel."""
    x = _f32(x)
    w = np.ascontiguousarray(windows, dtype=np.int64)
    out = np.empty(len(w), np.float64)
    arg = np.empty(len(w), np.int64)
    lib().or_windows_nn(x, len(x), m, w, len(w), out, arg)
    return out, arg


def lengths_nn(x, minL, maxL, windows):
    """FP64 nn at length minL + q of window windows[q], for every q, in parallel."""
    x = _f32(x)
    w = np.ascontiguousarray(windows, dtype=np.int64)
    assert len(w) == maxL - minL + 1
    out = np.empty(len(w), np.float64)
    lib().or_lengths_nn(x, len(x), minL, maxL, w, out)
    return out


def top1(nn):
    """(index, float distance) of the PALMAD top-1: the first maximum of float(nn)."""
    f = np.asarray(nn, dtype=np.float64).astype(np.float32)
    i = int(np.argmax(f))  # first occurrence of the maximum
    return i, float(f[i])


def pair_dist(x, m, i, j):
    x = _f32(x)
    return lib().or_pair_dist(x, len(x), m, i, j)


def window_nn(x, m, i):
    x = _f32(x)
    arg = C.c_int64(0)
    d = lib().or_window_nn(x, len(x), m, i, C.byref(arg))
    return d, arg.value


def select(nn, m, r2, top_k=1):
    nn = np.ascontiguousarray(nn, dtype=np.float64)
    att = Attempt()
    sel = (Discord * max(1, top_k))()
    lib().or_select(nn, len(nn), m, float(r2), top_k, C.byref(att), sel)
    return att.as_dict(), [(sel[i].ind, sel[i].dist) for i in range(att.n_sel)]


def palmad(x, minL, maxL, iter_cap=200, log_cap=100000):
    """Top-1 discord per length with the MERLIN schedule; (discords, attempts)."""
    x = _f32(x)
    L = maxL - minL + 1
    out = (Discord * L)()
    log = (Attempt * log_cap)()
    na = lib().or_palmad(x, len(x), minL, maxL, iter_cap, out, log, log_cap, None)
    if na < 0:
        raise RuntimeError("r-schedule exceeded the attempt cap")
    return ([(out[i].ind, out[i].dist) for i in range(L)],
            [log[i].as_dict() for i in range(min(na, log_cap))])


def pd3(x, m, top_k=1, iter_cap=200, log_cap=1000, fast=False):
    """Fixed-length discords with the halving schedule; (discords, attempts).
    fast: the vectorised nn profile (for long series)."""
    x = _f32(x)
    sel = (Discord * top_k)()
    log = (Attempt * log_cap)()
    na = C.c_int64(0)
    ns = lib().or_pd3(x, len(x), m, top_k, iter_cap, sel, log, log_cap, C.byref(na),
                      1 if fast else 0)
    if ns < 0:
        raise RuntimeError("r-schedule exceeded the attempt cap")
    return ([(sel[i].ind, sel[i].dist) for i in range(ns)],
            [log[i].as_dict() for i in range(min(na.value, log_cap))])


# ------------------------------------------------------- reference kernels
def ref_statistics(x, m):
    R = ref()
    x = _f32(x)
    N = len(x) - m + 1
    mu = np.zeros(len(x), np.float32)
    sd = np.zeros(len(x), np.float32)
    R.ref_compute_statistics(x, mu, sd, N, m)
    return mu[:N], sd[:N]


def ref_attempt(x, m, r):
    """One attempt of the reference CPU path at linear threshold r."""
    R = ref()
    x = _f32(x)
    N = len(x) - m + 1
    att = Attempt()
    cand = np.zeros(N, np.int32)
    nnd = np.zeros(N, np.float32)
    R.ref_attempt_at(x, len(x), m, float(r), C.byref(att), cand, nnd)
    return att.as_dict(), cand, nnd


def ref_palmad(x, minL, maxL, iter_cap=200, log_cap=100000):
    R = ref()
    x = _f32(x)
    L = maxL - minL + 1
    out = (Discord * L)()
    log = (Attempt * log_cap)()
    na = R.ref_palmad(x, len(x), minL, maxL, iter_cap, out, log, log_cap)
    if na < 0:
        raise RuntimeError("r-schedule exceeded the attempt cap")
    return ([(out[i].ind, out[i].dist) for i in range(L)],
            [log[i].as_dict() for i in range(min(na, log_cap))])


def ref_palmad_many(series, minL, maxL, threads, iter_cap=200):
    """Independent reference PALMAD runs on ``threads`` host threads."""
    R = ref()
    arrs = [_f32(s) for s in series]
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    lens = (C.c_int64 * len(arrs))(*[len(a) for a in arrs])
    L = maxL - minL + 1
    out = (Discord * (L * len(arrs)))()
    na = R.ref_palmad_many(ptrs, lens, len(arrs), minL, maxL, iter_cap, threads, out)
    if na < 0:
        raise RuntimeError("r-schedule exceeded the attempt cap")
    return na, [[(out[k * L + i].ind, out[k * L + i].dist) for i in range(L)]
                for k in range(len(arrs))]
