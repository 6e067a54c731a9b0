"""paddi_b200 -- B200-native discord discovery (PD3 / PALMAD hot path of PADDi).

Python mirror of the C ABI in ``include/paddi.h`` (ctypes over the in-tree
``libpaddi.so``).  The compute always runs in the CUDA library; there is no
CPU path.  If the shared library is missing or no sm_100 device is present,
the calls raise.

Reference entry points and their counterparts here:

=====================================================  ============================
reference (PADDi src/)                                 paddi_b200
=====================================================  ============================
``main`` PALMAD loop, main.cu:136-233                   :func:`palmad`
``do_PD3`` + refine + ``find_top1_discord``             :func:`pd3`
``do_PD3`` flags / nnDist on device, PD3.cuh:15         :meth:`Context.do_pd3`
``compute_statistics``, preprocessing.cuh:68            :meth:`Context.compute_statistics`
``struct Discord``, PALMAD_types.hpp:7                  :class:`Discord`
fragments + all-to-all + MIN, MPI_transfers.hpp:29-84   :mod:`paddi_b200.sharded`
=====================================================  ============================
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpaddi.so")

PADDI_OK = 0
PADDI_ERR_INVALID_ARG = 1
PADDI_ERR_CUDA = 2
PADDI_ERR_OUT_OF_MEMORY = 3
PADDI_ERR_ITER_CAP = 4
PADDI_ERR_NO_DEVICE = 5
PADDI_ERR_INTERNAL_LIMIT = 6
PADDI_ERR_UNSUPPORTED = 7

DIST_AUTO, DIST_FP32, DIST_SPLIT_BF16, DIST_SPLIT_FP16 = 0, 1, 2, 3
R_MERLIN, R_LEARNED, R_BOUND = 0, 1, 2

FLT_MAX = float(np.finfo(np.float32).max)


class PaddiError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"paddi status {status}: {msg}")
        self.status = status


class _Discord(C.Structure):
    _fields_ = [("ind", C.c_int32), ("dist", C.c_float)]


class _Opts(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("device", C.c_int32),
                ("distance_kernel", C.c_int32), ("r_policy", C.c_int32),
                ("segment_len", C.c_uint32), ("phase1_chunks", C.c_uint32),
                ("iter_cap", C.c_uint32), ("guard", C.c_float), ("flags", C.c_uint32),
                ("tile_rows", C.c_uint32)]


FLAG_LOG_BOUND = 1
MODEL_NFEAT = 12
MODEL_NPARAM = 5057


class _Log(C.Structure):
    _fields_ = [("m", C.c_int32), ("r", C.c_float), ("r2", C.c_float), ("found", C.c_int32),
                ("n_cand", C.c_int64), ("n_disc", C.c_int64), ("n_phase1", C.c_int64),
                ("n_recheck", C.c_int32), ("top", _Discord), ("ms_stats", C.c_float),
                ("ms_phase1", C.c_float), ("ms_refine", C.c_float), ("ms_select", C.c_float),
                ("ms_total", C.c_float), ("refine_pairs", C.c_int64), ("n_launches", C.c_int32),
                ("refine_kernel", C.c_int32), ("r_source", C.c_int32), ("ms_guide", C.c_float),
                ("lb", C.c_float), ("flat_frac", C.c_float), ("p1_pairs", C.c_int64),
                ("refine_live_pairs", C.c_int64), ("ms_refine_kernel", C.c_float),
                ("n_fragile", C.c_int32)]

    def as_dict(self):
        return {"m": self.m, "r": self.r, "r2": self.r2, "found": self.found,
                "n_cand": self.n_cand, "n_disc": self.n_disc, "n_phase1": self.n_phase1,
                "n_recheck": self.n_recheck, "top_ind": self.top.ind, "top_dist": self.top.dist,
                "ms_stats": self.ms_stats, "ms_phase1": self.ms_phase1,
                "ms_refine": self.ms_refine, "ms_select": self.ms_select,
                "ms_total": self.ms_total, "refine_pairs": self.refine_pairs,
                "n_launches": self.n_launches, "refine_kernel": self.refine_kernel,
                "r_source": self.r_source, "ms_guide": self.ms_guide, "lb": self.lb,
                "flat_frac": self.flat_frac, "p1_pairs": self.p1_pairs,
                "refine_live_pairs": self.refine_live_pairs,
                "ms_refine_kernel": self.ms_refine_kernel, "n_fragile": self.n_fragile}


@dataclass(frozen=True)
class Discord:
    """A discord: start index and squared z-normalised nn distance."""
    ind: int
    dist: float


# Every exported function of include/paddi.h with its ctypes signature.
# per-length range-discord profile callback: (user, m, nn, N)
PROFILE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.POINTER(C.c_float), C.c_size_t)

_SIGS = {
    "paddi_abi_version": ([], C.c_int32),
    "paddi_status_string": ([C.c_int], C.c_char_p),
    "paddi_opts_default": ([C.POINTER(_Opts)], None),
    "paddi_ctx_create": ([C.POINTER(C.c_void_p), C.POINTER(_Opts)], C.c_int),
    "paddi_ctx_destroy": ([C.c_void_p], C.c_int),
    "paddi_last_error": ([C.c_void_p], C.c_char_p),
    "paddi_ctx_reserve": ([C.c_void_p, C.c_size_t, C.c_uint32], C.c_int),
    "paddi_ctx_stream": ([C.c_void_p], C.c_void_p),
    "paddi_pd3": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint32, C.c_uint32,
                   C.c_float, C.POINTER(_Discord), C.POINTER(C.c_uint32), C.POINTER(_Log),
                   C.c_uint32, C.POINTER(C.c_uint32)], C.c_int),
    "paddi_palmad": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint32,
                      C.POINTER(_Discord), C.POINTER(_Log), C.c_uint32,
                      C.POINTER(C.c_uint32)], C.c_int),
    "paddi_palmad_device": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint32,
                             C.POINTER(_Discord), C.POINTER(_Log), C.c_uint32,
                             C.POINTER(C.c_uint32)], C.c_int),
    "paddi_compute_statistics": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                  C.c_uint32, C.c_void_p], C.c_int),
    "paddi_do_pd3": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint32, C.c_float, C.c_void_p,
                      C.c_void_p, C.POINTER(C.c_int64), C.c_void_p], C.c_int),
    "paddi_compute_statistics_noalloc": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                          C.c_uint32, C.c_void_p], C.c_int),
    "paddi_palmad_profiled": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint32,
                               C.POINTER(_Discord), C.POINTER(_Log), C.c_uint32,
                               C.POINTER(C.c_uint32), PROFILE_FN, C.c_void_p], C.c_int),
    "paddi_palmad_batched": ([C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t),
                              C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                              C.POINTER(_Discord), C.c_void_p, C.c_void_p], C.c_int),
    "paddi_autotune": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint32,
                        C.POINTER(_Opts), C.c_void_p], C.c_int),
    "paddi_r_features": ([C.POINTER(_Discord), C.c_uint32, C.c_uint32, C.c_float, C.c_float,
                          C.c_uint32, C.POINTER(C.c_float)], C.c_int),
    "paddi_model_set": ([C.c_void_p, C.c_void_p, C.c_uint32, C.c_float], C.c_int),
    "paddi_model_train": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_float,
                           C.c_uint32, C.c_uint32, C.c_float, C.c_uint64, C.c_void_p,
                           C.c_void_p], C.c_int),
    "paddi_model_grad": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_float,
                          C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "paddi_model_predict": ([C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int32,
                             C.c_void_p], C.c_int),
    "paddi_shard_phase1": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint32, C.c_float,
                            C.c_size_t, C.c_size_t, C.c_void_p], C.c_int),
    "paddi_shard_refine": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint32, C.c_float,
                            C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p,
                            C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)], C.c_int),
    "paddi_shard_select": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_uint32, C.c_float,
                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                            C.POINTER(_Discord), C.POINTER(C.c_uint32), C.POINTER(_Log)], C.c_int),
    "paddi_merlin_first_r": ([C.POINTER(_Discord), C.c_uint32, C.c_uint32,
                              C.POINTER(C.c_float)], C.c_float),
    "paddi_merlin_lower": ([C.c_float, C.c_uint32, C.c_float], C.c_float),
    "paddi_debug_set": ([C.c_void_p, C.c_int32, C.c_int64], C.c_int),
    "paddi_debug_get": ([C.c_void_p, C.c_int32, C.POINTER(C.c_int64)], C.c_int),
}

# test hooks (include/paddi.h, paddi_debug_key)
DEBUG_FAIL_ALLOC, DEBUG_WAIT_CYCLES, DEBUG_WITHHOLD_STAGE, DEBUG_LAST_PASSES = 1, 2, 3, 4
DEBUG_RECHECK_CAP = 5

# Largest n - m + 1 accepted by compute_statistics_noalloc (include/paddi.h).
NOALLOC_MAX_WINDOWS = 131072

_LIB = None


def lib() -> C.CDLL:
    """Load the in-tree CUDA library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: run __graft_entry__.build() "
                          "(make -C paddi_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _LIB = L
    return _LIB


def status_string(s: int) -> str:
    return lib().paddi_status_string(s).decode()


class Context:
    """A device context (one stream, device buffers reused across calls)."""

    def __init__(self, device: int = 0, distance_kernel: int = DIST_AUTO,
                 r_policy: int = R_MERLIN, segment_len: int = 256, phase1_chunks: int = 12,
                 iter_cap: int = 200, guard: float = 0.0, flags: int = 0, model=None,
                 model_margin: float = 1.0, tile_rows: int = 0):
        """model: parameters for R_LEARNED (default: the bundled trained model)."""
        L = lib()
        o = _Opts()
        L.paddi_opts_default(C.byref(o))
        o.device = device
        o.distance_kernel = distance_kernel
        o.r_policy = r_policy
        o.segment_len = segment_len
        o.phase1_chunks = phase1_chunks
        o.iter_cap = iter_cap
        o.guard = guard
        o.flags = flags
        o.tile_rows = tile_rows
        h = C.c_void_p()
        s = L.paddi_ctx_create(C.byref(h), C.byref(o))
        if s != PADDI_OK:
            raise PaddiError(s, status_string(s))
        self._h = h
        self.opts = o
        if r_policy == R_LEARNED:
            if model is None:
                from . import learned_r
                model = learned_r.load_default()
            self.set_model(model, model_margin)

    def close(self):
        if getattr(self, "_h", None):
            lib().paddi_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return lib().paddi_ctx_stream(self._h) or 0

    def reserve(self, n: int, maxL: int):
        self._check(lib().paddi_ctx_reserve(self._h, n, maxL))

    # ------------------------------------------------------------ learned r
    def set_model(self, params, margin: float = 1.0):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(lib().paddi_model_set(self._h, p.ctypes.data, p.size, float(margin)))

    def model_train(self, X, Y, tau=0.2, epochs=100, batch=4096, lr=3e-3, seed=0, init=None):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        p = np.array(init if init is not None else init_params(seed), dtype=np.float32)
        loss = np.zeros(max(epochs, 1), np.float32)
        self._check(lib().paddi_model_train(self._h, X.ctypes.data, Y.ctypes.data, len(Y),
                                            float(tau), epochs, batch, float(lr), seed,
                                            p.ctypes.data, loss.ctypes.data))
        return p, loss[:epochs]

    def model_grad(self, X, Y, params, tau=0.2):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        p = np.ascontiguousarray(params, dtype=np.float32)
        g = np.zeros(MODEL_NPARAM, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(lib().paddi_model_grad(self._h, X.ctypes.data, Y.ctypes.data, len(Y),
                                           float(tau), p.ctypes.data, g.ctypes.data,
                                           loss.ctypes.data))
        return g, float(loss[0])

    def model_predict(self, X, params, bf16=False):
        X = np.ascontiguousarray(X, dtype=np.float32)
        p = np.ascontiguousarray(params, dtype=np.float32)
        y = np.zeros(len(X), np.float32)
        self._check(lib().paddi_model_predict(self._h, X.ctypes.data, len(X), p.ctypes.data,
                                              1 if bf16 else 0, y.ctypes.data))
        return y

    # ------------------------------------------------------------ test hooks
    def debug_set(self, key: int, value: int):
        """Failure injection (DEBUG_*): a failing allocation, a short refine wait
        limit, a withheld refine pipeline stage."""
        self._check(lib().paddi_debug_set(self._h, key, int(value)))

    def debug_get(self, key: int) -> int:
        v = C.c_int64(0)
        self._check(lib().paddi_debug_get(self._h, key, C.byref(v)))
        return v.value

    def _check(self, s):
        if s != PADDI_OK:
            raise PaddiError(s, lib().paddi_last_error(self._h).decode())

    # ------------------------------------------------------------ drivers
    def palmad(self, series, minL: int, maxL: int, log_cap: int = 100000):
        """Top-1 discord of every length minL..maxL; returns (discords, log)."""
        x = np.ascontiguousarray(series, dtype=np.float32)
        L = maxL - minL + 1
        out = (_Discord * max(L, 1))()  # the library rejects an empty range itself
        log = (_Log * log_cap)()
        nl = C.c_uint32(0)
        self._check(lib().paddi_palmad(self._h, x.ctypes.data, len(x), minL, maxL, out, log,
                                       log_cap, C.byref(nl)))
        return ([Discord(out[i].ind, out[i].dist) for i in range(L)],
                [log[i].as_dict() for i in range(min(nl.value, log_cap))])

    def palmad_profiled(self, series, minL: int, maxL: int, on_profile=None,
                        log_cap: int = 100000):
        """paddi_palmad plus the range-discord profile of every length.

        on_profile(m, nn) receives a copy (numpy float32, N = n - m + 1) of the
        length's profile; without it the profiles are returned as a list.
        Returns (discords, log, profiles or None)."""
        x = np.ascontiguousarray(series, dtype=np.float32)
        L = maxL - minL + 1
        out = (_Discord * max(L, 1))()
        log = (_Log * log_cap)()
        nl = C.c_uint32(0)
        kept = []

        def cb(_user, m, ptr, N):
            arr = np.ctypeslib.as_array(ptr, shape=(N,)).copy()
            if on_profile is not None:
                on_profile(int(m), arr)
            else:
                kept.append(arr)

        fn = PROFILE_FN(cb)
        self._check(lib().paddi_palmad_profiled(self._h, x.ctypes.data, len(x), minL, maxL, out,
                                                log, log_cap, C.byref(nl), fn, None))
        return ([Discord(out[i].ind, out[i].dist) for i in range(L)],
                [log[i].as_dict() for i in range(min(nl.value, log_cap))],
                None if on_profile is not None else kept)

    def autotune(self, series, minL: int, maxL: int):
        """Pick the refine's tile rows and phase-1 segment length and depth on
        probe lengths of this series."""
        x = np.ascontiguousarray(series, dtype=np.float32)
        o = _Opts()
        ms = np.zeros(18, np.float32)
        self._check(lib().paddi_autotune(self._h, x.ctypes.data, len(x), minL, maxL,
                                         C.byref(o), ms.ctypes.data))
        self.opts = o
        grid = [(tr, sg, ch) for tr in (0, 64) for sg in (256, 384, 512) for ch in (8, 12, 16)]
        return {"tile_rows": o.tile_rows, "segment_len": o.segment_len,
                "phase1_chunks": o.phase1_chunks, "probe_ms": dict(zip(grid, ms.tolist()))}

    def palmad_batched(self, series_list, minL: int, maxL: int, streams: int = 4):
        """PALMAD over many uneven series; returns (discords per series, attempts)."""
        arrs = [np.ascontiguousarray(x, dtype=np.float32) for x in series_list]
        k = len(arrs)
        ptrs = (C.c_void_p * k)(*[a.ctypes.data for a in arrs])
        lens = (C.c_size_t * k)(*[len(a) for a in arrs])
        L = maxL - minL + 1
        out = (_Discord * max(k * L, 1))()
        st = np.zeros(max(k, 1), np.int32)
        att = np.zeros(max(k, 1), np.uint64)
        self._check(lib().paddi_palmad_batched(self._h, ptrs, lens, k, minL, maxL, streams, out,
                                               st.ctypes.data, att.ctypes.data))
        return ([[Discord(out[s * L + i].ind, out[s * L + i].dist) for i in range(L)]
                 for s in range(k)], att[:k].tolist())

    def palmad_device(self, d_series_ptr: int, n: int, minL: int, maxL: int,
                      log_cap: int = 100000):
        """PALMAD on a series already in device memory (pointer to n floats)."""
        L = maxL - minL + 1
        out = (_Discord * max(L, 1))()
        log = (_Log * log_cap)()
        nl = C.c_uint32(0)
        self._check(lib().paddi_palmad_device(self._h, C.c_void_p(d_series_ptr), n, minL, maxL,
                                              out, log, log_cap, C.byref(nl)))
        return ([Discord(out[i].ind, out[i].dist) for i in range(L)],
                [log[i].as_dict() for i in range(min(nl.value, log_cap))])

    def pd3(self, series, m: int, top_k: int = 1, r: float = 0.0, segment_len: int = 0,
            log_cap: int = 1000):
        """Fixed-length discords; r <= 0 runs the halving schedule from 2*sqrt(m)."""
        x = np.ascontiguousarray(series, dtype=np.float32)
        out = (_Discord * max(top_k, 1))()
        n_out = C.c_uint32(0)
        log = (_Log * log_cap)()
        nl = C.c_uint32(0)
        self._check(lib().paddi_pd3(self._h, x.ctypes.data, len(x), m, segment_len, top_k,
                                    float(r), out, C.byref(n_out), log, log_cap, C.byref(nl)))
        return ([Discord(out[i].ind, out[i].dist) for i in range(n_out.value)],
                [log[i].as_dict() for i in range(min(nl.value, log_cap))])

    def compute_statistics(self, d_T: int, d_mean: int, d_std: int, n: int, m: int,
                           stream: int = 0):
        """Device pointers; reference compute_statistics (src/preprocessing.cuh:68)."""
        self._check(lib().paddi_compute_statistics(self._h, C.c_void_p(d_T), C.c_void_p(d_mean),
                                                   C.c_void_p(d_std), n, m,
                                                   C.c_void_p(stream or None)))

    def do_pd3(self, d_T: int, n: int, m: int, r2: float, d_is_cand: int, d_nnDist: int,
               stream: int = 0) -> int:
        """Device pointers; reference do_PD3 + refine (src/PD3.cuh:15-50).  Returns #cand."""
        nc = C.c_int64(0)
        self._check(lib().paddi_do_pd3(self._h, C.c_void_p(d_T), n, m, float(r2),
                                       C.c_void_p(d_is_cand), C.c_void_p(d_nnDist),
                                       C.byref(nc), C.c_void_p(stream or None)))
        return nc.value


def r_features(discords, j: int, minL: int, lb: float, flat_frac: float,
               prev_attempts: int) -> np.ndarray:
    """The learned-r model's 12 features for length minL + j (host code of the
    library, so training uses exactly what inference uses)."""
    n = max(j, 1)
    arr = (_Discord * n)()
    for i in range(min(j, len(discords))):
        arr[i].ind = int(discords[i][0] if isinstance(discords[i], tuple) else discords[i].ind)
        arr[i].dist = float(discords[i][1] if isinstance(discords[i], tuple) else discords[i].dist)
    f = (C.c_float * MODEL_NFEAT)()
    s = lib().paddi_r_features(arr, j, minL, float(lb), float(flat_frac), int(prev_attempts), f)
    if s != PADDI_OK:
        raise PaddiError(s, status_string(s))
    return np.array(f[:], dtype=np.float32)


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation of the predictor's parameters."""
    rng = np.random.default_rng(seed)
    F, H = MODEL_NFEAT, 64
    w1 = rng.normal(0, np.sqrt(2.0 / F), (H, F))
    w2 = rng.normal(0, np.sqrt(2.0 / H), (H, H))
    w3 = rng.normal(0, np.sqrt(1.0 / H), H)
    return np.concatenate([w1.ravel(), np.zeros(H), w2.ravel(), np.zeros(H), w3,
                           [0.0]]).astype(np.float32)


def compute_statistics_noalloc(d_T: int, d_mean: int, d_std: int, n: int, m: int,
                               stream: int = 0) -> None:
    """Window mean / std of length m without any device allocation.

    For callers that may not let the library allocate device memory (hosts
    that own every device byte through their own allocator, or loops that
    cannot afford an allocation's device synchronisation).  Device pointers;
    runs on the current device.  n - m + 1 must not exceed
    NOALLOC_MAX_WINDOWS.  The library keeps one fixed scratch array per
    device: calls whose GPU work overlaps race with each other, and the first
    call on a device (which looks the array up) should come before any stream
    capture.
    """
    s = lib().paddi_compute_statistics_noalloc(C.c_void_p(d_T), C.c_void_p(d_mean),
                                               C.c_void_p(d_std), n, m,
                                               C.c_void_p(stream or None))
    if s != PADDI_OK:
        limit = (f" (n - m + 1 = {n - m + 1}, limit {NOALLOC_MAX_WINDOWS})"
                 if s == PADDI_ERR_INVALID_ARG else "")
        raise PaddiError(s, status_string(s) + limit)


def palmad(series, minL: int, maxL: int, **ctx_kw):
    """One-shot PALMAD: ``[Discord]`` for lengths minL..maxL and the attempt log."""
    with Context(**ctx_kw) as c:
        return c.palmad(series, minL, maxL)


def pd3(series, m: int, top_k: int = 1, r: float = 0.0, **ctx_kw):
    """One-shot PD3 with top-k."""
    with Context(**ctx_kw) as c:
        return c.pd3(series, m, top_k=top_k, r=r)
