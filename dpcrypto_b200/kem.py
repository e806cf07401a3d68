"""Host-side mirror of the reference's batched KEM interface over libdpkem.so.

The reference exposes batched host functions (FrodoKEM976-GPU/include/cuda_kernel.cuh:7-9,
SABER-GPU/include/cuda_kernel.cuh:6-7).  This module binds the C ABI with ctypes:

* ``Engine`` wraps one ``dpkem_ctx`` and runs keypair / enc / dec over n instances.
  numpy uint8 arrays run in host-pointer mode (copy in, compute, copy out); torch
  CUDA uint8 tensors run in device-pointer mode on the current torch stream.
* ``frodoKEMKeypair`` / ``frodoKEMEncap`` / ``frodoKEMDecap`` / ``saber_enc`` /
  ``saber_dec`` call the reference-named C shims with numpy buffers.

There is no CPU fallback: if the library or a CUDA device is missing, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# DPKEM_LIB selects another build of the library (the autotuner measures its variants this way).
LIB_PATH = os.environ.get("DPKEM_LIB") or os.path.join(HERE, "libdpkem.so")

FRODO976, FRODO976AES, LIGHTSABER, SABER, FIRESABER = 0, 1, 2, 3, 4
SCHEMES = (FRODO976, FRODO976AES, LIGHTSABER, SABER, FIRESABER)
FORM_DP4A, FORM_INT32, FORM_TC = 0, 1, 2
FLAG_DEVICE_PTRS = 1
OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, EUNSUPPORTED, EAGAIN = 0, -1, -2, -3, -4, -5, -6

class Request(ctypes.Structure):
    """dpkem_request: one operation of a mixed batch (device buffers, batched-call order)."""

    _fields_ = [("scheme", ctypes.c_int32), ("op", ctypes.c_int32), ("in0", ctypes.c_void_p),
                ("in1", ctypes.c_void_p), ("out0", ctypes.c_void_p), ("out1", ctypes.c_void_p)]


class ServiceConfig(ctypes.Structure):
    """dpkem_service_config (include/dpkem.h)."""

    _fields_ = [("max_inflight", ctypes.c_uint32), ("idle_ms", ctypes.c_uint32), ("saber_ctas", ctypes.c_uint32),
                ("warp_max", ctypes.c_uint32), ("scratch_bytes", ctypes.c_uint64), ("coin_key", ctypes.c_void_p)]


EXPORTS = {
    "dpkem_ctx_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_size_t]),
    "dpkem_ctx_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dpkem_ctx_set_max_ctas": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "dpkem_ctx_reserve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t]),
    "dpkem_selftest_timeout": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "dpkem_mixed_bytes": (ctypes.c_size_t, [ctypes.c_int, ctypes.c_size_t]),
    "dpkem_sizes": (ctypes.c_int, [ctypes.c_int] + [ctypes.POINTER(ctypes.c_size_t)] * 6),
    "dpkem_max_chunk": (ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_int]),
    "dpkem_keypair_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint,
                                           ctypes.c_void_p]),
    "dpkem_enc_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_uint, ctypes.c_void_p]),
    "dpkem_dec_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint,
                                       ctypes.c_void_p]),
    "dpkem_coins": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_uint64,
                                   ctypes.c_char_p, ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]),
    "dpkem_sync": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "dpkem_mixed_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "dpkem_mixed_batch_keyed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p,
                                               ctypes.c_char_p, ctypes.c_uint64, ctypes.c_void_p]),
    "dpkem_mixed_graph_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p,
                                                ctypes.POINTER(ctypes.c_void_p)]),
    "dpkem_mixed_graph_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "dpkem_mixed_graph_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dpkem_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "dpkem_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    "dpkem_probe_int_peaks": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_double)]),
    "dpkem_probe_i8_mma_peak": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    "dpkem_frodo_expand_a": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p]),
    "dpkem_frodo_enc_shared": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p]),
    "dpkem_frodo_dec_shared": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p]),
    "dpkem_keccak_f1600_lanes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_int]),
    "dpkem_probe_keccak_chain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.POINTER(ctypes.c_double)]),
    "dpkem_saber_enc_batch_static": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_void_p]),
    "dpkem_set_tuning": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int]),
    "dpkem_get_tuning": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]),
    "dpkem_strerror": (ctypes.c_char_p, [ctypes.c_int]),
    "dpkem_last_status": (ctypes.c_int, []),
    "dpkem_set_compat_batch": (None, [ctypes.c_size_t]),
    "dpkem_set_compat_saber_level": (None, [ctypes.c_int]),
    "dpkem_set_compat_form": (None, [ctypes.c_int]),
    "frodoKEMKeypair": (None, [ctypes.c_void_p, ctypes.c_void_p]),
    "frodoKEMEncap": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "frodoKEMDecap": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "saber_enc": (None, [ctypes.c_uint8, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "saber_dec": (None, [ctypes.c_uint8, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    # KEM service: one long-lived launch that admits requests while it runs
    "dpkem_service_default_config": (ctypes.c_int, [ctypes.c_void_p]),
    "dpkem_service_open": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "dpkem_service_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                                            ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_uint64)]),
    "dpkem_service_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_size_t)]),
    "dpkem_service_drain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    "dpkem_service_stats": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_uint64)] * 3
                            + [ctypes.POINTER(ctypes.c_int)]),
    "dpkem_service_counters": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]),
    "dpkem_service_close": (ctypes.c_int, [ctypes.c_void_p]),
    # wire format and shared-memory ring (include/dpkem_wire.h)
    "dpkem_frame_bytes": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t),
                                         ctypes.POINTER(ctypes.c_size_t)]),
    "dpkem_frames_scan": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t]
                          + [ctypes.POINTER(ctypes.c_size_t)] * 3),
    "dpkem_frames_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                                        ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "dpkem_host_register": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t]),
    "dpkem_host_unregister": (ctypes.c_int, [ctypes.c_void_p]),
    "dpkem_ring_bytes": (ctypes.c_size_t, [ctypes.c_size_t]),
    "dpkem_ring_init": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t]),
    "dpkem_ring_push": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_size_t)]),
    "dpkem_ring_pop": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                      ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "dpkem_ring_acquire": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t] + [ctypes.POINTER(ctypes.c_size_t)] * 7),
    "dpkem_ring_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t]),
    "dpkem_ring_serve": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]),
}

_lib = None


class DpkemError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = load().dpkem_strerror(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: {msg} ({status})" if what else f"{msg} ({status})")


def load() -> ctypes.CDLL:
    """Load libdpkem.so (built by dpcrypto_b200.build); raise if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m dpcrypto_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in EXPORTS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        apply_tuning()
    return _lib


TUNING_PATH = os.path.join(HERE, "tuning.json")
RUNTIME_KNOBS = ("thread_block", "mixed_frodo_task", "mixed_pair_task", "mixed_thread_task", "pipe_chunks",
                 "pipe_priority", "saber_pair_max", "saber_five_max", "saber_finish_five_max", "frodo_five_max",
                 "frodo_ss_five_max", "saber_tc_ctas_per_sm", "saber_warp_max", "saber_finish_warp_max",
                 "frodo_warp_max", "frodo_ss_warp_max", "mixed_warp_max")


_tuning: dict = {}


def get_tuning() -> dict:
    """Runtime knobs set through set_tuning / apply_tuning in this process."""
    load()
    return dict(_tuning)


def apply_tuning(path: str = TUNING_PATH) -> dict:
    """Apply the runtime knobs recorded by the autotuner (dpcrypto_b200/tuning.json), if any."""
    import json

    if not os.path.exists(path):
        return {}
    with open(path) as f:
        chosen = json.load(f).get("chosen", {})
    for k in RUNTIME_KNOBS:
        if k in chosen:
            rc = _lib.dpkem_set_tuning(k.encode(), int(chosen[k]))
            if rc != OK:
                raise DpkemError(rc, f"tuning {k}={chosen[k]}")
            _tuning[k] = int(chosen[k])
    return chosen


def tuning_value(key: str) -> int:
    """The library's current value of a knob (its compiled default unless set)."""
    v = ctypes.c_int()
    rc = load().dpkem_get_tuning(key.encode(), ctypes.byref(v))
    if rc != OK:
        raise DpkemError(rc, f"get_tuning({key})")
    return v.value


class knobs:
    """Context manager: set knobs for a block, restore their previous values after."""

    def __init__(self, **values):
        self.values = values

    def __enter__(self):
        self.saved = {k: tuning_value(k) for k in self.values}
        for k, v in self.values.items():
            set_tuning(k, v)
        return self

    def __exit__(self, *exc):
        for k, v in self.saved.items():
            set_tuning(k, v)


def set_tuning(key: str, value: int) -> None:
    rc = load().dpkem_set_tuning(key.encode(), int(value))
    if rc != OK:
        raise DpkemError(rc, f"set_tuning({key}, {value})")
    _tuning[key] = int(value)


def sizes(scheme: int) -> dict:
    vals = [ctypes.c_size_t() for _ in range(6)]
    rc = load().dpkem_sizes(scheme, *[ctypes.byref(v) for v in vals])
    if rc != OK:
        raise DpkemError(rc, f"dpkem_sizes({scheme})")
    return dict(zip(("pk", "sk", "ct", "ss", "kp_coins", "enc_coins"), (v.value for v in vals)))


def _is_torch_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and x.is_cuda


def _ptr(x):
    if _is_torch_cuda(x):
        return ctypes.c_void_p(x.data_ptr())
    assert isinstance(x, np.ndarray) and x.dtype == np.uint8 and x.flags["C_CONTIGUOUS"], "uint8 C-contiguous array"
    return ctypes.c_void_p(x.ctypes.data)


class Engine:
    """One dpkem context (device scratch arena + stream) on a CUDA device."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self._lib = load()
        h = ctypes.c_void_p()
        rc = self._lib.dpkem_ctx_create(ctypes.byref(h), device, hbm_budget)
        if rc != OK:
            raise DpkemError(rc, "dpkem_ctx_create (is a CUDA device visible?)")
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dpkem_ctx_destroy(self._h)
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

    # -- helpers ---------------------------------------------------------------
    def _alloc(self, like, n: int, size: int):
        if _is_torch_cuda(like):
            import torch

            return torch.empty((n, size), dtype=torch.uint8, device=like.device)
        return np.empty((n, size), dtype=np.uint8)

    def _mode(self, *arrs):
        dev = [_is_torch_cuda(a) for a in arrs]
        if any(dev) and not all(dev):
            raise ValueError("mix of host and device buffers")
        if all(dev):
            import torch

            h = torch.cuda.current_stream(arrs[0].device).cuda_stream
            # torch's default stream is the legacy NULL stream; the C ABI reads NULL as "the
            # context's own stream", so name the legacy stream explicitly (cudaStreamLegacy).
            return FLAG_DEVICE_PTRS, ctypes.c_void_p(h if h else 1)
        return 0, None

    @staticmethod
    def _rows(x, size: int, what: str) -> int:
        shape = tuple(x.shape)
        if len(shape) != 2 or shape[1] != size:
            raise ValueError(f"{what}: expected shape (n, {size}), got {shape}")
        return shape[0]

    def _check(self, rc: int, what: str):
        if rc != OK:
            raise DpkemError(rc, what)

    # -- operations ------------------------------------------------------------
    def keypair(self, scheme: int, coins, form: int = FORM_TC, out=None):
        z = sizes(scheme)
        n = self._rows(coins, z["kp_coins"], "coins")
        pk, sk = out if out is not None else (self._alloc(coins, n, z["pk"]), self._alloc(coins, n, z["sk"]))
        flags, st = self._mode(coins, pk, sk)
        self._check(self._lib.dpkem_keypair_batch(self._h, scheme, form, n, _ptr(coins), _ptr(pk), _ptr(sk), flags,
                                                  st), "keypair")
        return pk, sk

    def enc(self, scheme: int, pk, coins, form: int = FORM_TC, out=None):
        z = sizes(scheme)
        n = self._rows(pk, z["pk"], "pk")
        if self._rows(coins, z["enc_coins"], "coins") != n:
            raise ValueError("pk and coins batch sizes differ")
        ct, ss = out if out is not None else (self._alloc(pk, n, z["ct"]), self._alloc(pk, n, z["ss"]))
        flags, st = self._mode(pk, coins, ct, ss)
        self._check(self._lib.dpkem_enc_batch(self._h, scheme, form, n, _ptr(coins), _ptr(pk), _ptr(ct), _ptr(ss),
                                              flags, st), "enc")
        return ct, ss

    def dec(self, scheme: int, ct, sk, form: int = FORM_TC, out=None):
        z = sizes(scheme)
        n = self._rows(ct, z["ct"], "ct")
        if self._rows(sk, z["sk"], "sk") != n:
            raise ValueError("ct and sk batch sizes differ")
        ss = out if out is not None else self._alloc(ct, n, z["ss"])
        flags, st = self._mode(ct, sk, ss)
        self._check(self._lib.dpkem_dec_batch(self._h, scheme, form, n, _ptr(ct), _ptr(sk), _ptr(ss), flags, st),
                    "dec")
        return ss

    def reserve(self, nbytes: int):
        """Grow this engine's device arena to nbytes now, outside any latency-critical call."""
        self._check(self._lib.dpkem_ctx_reserve(self._h, nbytes), "reserve")

    def set_max_ctas(self, max_ctas: int):
        """Cap the CTAs of this engine's persistent launches (0 = the whole GPU)."""
        self._check(self._lib.dpkem_ctx_set_max_ctas(self._h, max_ctas), "set_max_ctas")

    def coins(self, n: int, length: int, tag: str, first: int = 0, out=None):
        out = out if out is not None else np.empty((n, length), np.uint8)
        flags, st = self._mode(out)
        self._check(self._lib.dpkem_coins(self._h, n, length, first, tag.encode(), _ptr(out), flags, st), "coins")
        return out

    # -- FrodoKEM batches under one key (torch CUDA tensors, current torch stream) -------
    def expand_a(self, scheme: int, pk):
        """A of one public key pk (a 1-D uint8 CUDA tensor) as a 976 x 976 int16 tensor."""
        import torch

        amat = torch.empty((976, 976), dtype=torch.int16, device=pk.device)
        flags, st = self._mode(pk)
        self._check(self._lib.dpkem_frodo_expand_a(self._h, scheme, _ptr(pk), ctypes.c_void_p(amat.data_ptr()), st),
                    "frodo_expand_a")
        return amat

    def enc_shared(self, scheme: int, pk, coins, form: int = FORM_TC, amat=None):
        """n encapsulations to the one public key pk (1-D); coins (n, 24); returns (ct, ss)."""
        z = sizes(scheme)
        n = self._rows(coins, z["enc_coins"], "coins")
        ct, ss = self._alloc(coins, n, z["ct"]), self._alloc(coins, n, z["ss"])
        flags, st = self._mode(coins, pk, ct, ss)
        a = ctypes.c_void_p(amat.data_ptr()) if amat is not None else None
        self._check(self._lib.dpkem_frodo_enc_shared(self._h, scheme, form, n, _ptr(coins), _ptr(pk), a, _ptr(ct),
                                                    _ptr(ss), st), "frodo_enc_shared")
        return ct, ss

    def dec_shared(self, scheme: int, ct, sk, form: int = FORM_TC, amat=None):
        """n decapsulations with the one secret key sk (1-D); ct (n, 15744); returns ss."""
        z = sizes(scheme)
        n = self._rows(ct, z["ct"], "ct")
        ss = self._alloc(ct, n, z["ss"])
        flags, st = self._mode(ct, sk, ss)
        a = ctypes.c_void_p(amat.data_ptr()) if amat is not None else None
        self._check(self._lib.dpkem_frodo_dec_shared(self._h, scheme, form, n, _ptr(ct), _ptr(sk), a, _ptr(ss), st),
                    "frodo_dec_shared")
        return ss

    def sync(self, stream=None):
        self._check(self._lib.dpkem_sync(self._h, stream), "sync")

    def profile(self, enable: bool = True):
        self._check(self._lib.dpkem_profile(self._h, int(enable)), "profile")

    def stage_times(self) -> list:
        """Per-stage device times (ms) of the last batched call, when profiling is on."""
        buf = (ctypes.c_float * 8)()
        n = self._lib.dpkem_profile_read(self._h, buf, 8)
        if n < 0:
            raise DpkemError(n, "profile_read")
        return [float(buf[k]) for k in range(n)]

    def probe_i8_mma_peak(self) -> float:
        """int8 tcgen05 MMA multiply-adds per second (one CTA per SM, back-to-back MMAs)."""
        v = ctypes.c_double()
        self._check(self._lib.dpkem_probe_i8_mma_peak(self._h, ctypes.byref(v)), "probe_i8_mma_peak")
        return v.value

    def keccak_lanes(self, lanes: int, states, perms: int = 1):
        """`perms` Keccak-f[1600] permutations of each row of `states` (an n x 25 torch CUDA
        tensor of 64-bit lanes) in the given lanes-per-state layout (1, 2, 5 or 25); returns a new
        tensor.  The calling torch stream's pending work is synchronised first."""
        import torch

        torch.cuda.current_stream(states.device).synchronize()
        out = states.new_empty(states.shape)
        self._check(self._lib.dpkem_keccak_f1600_lanes(self._h, lanes, states.shape[0], ctypes.c_void_p(states.data_ptr()),
                                                      ctypes.c_void_p(out.data_ptr()), perms), "keccak_lanes")
        return out

    def probe_keccak_chain(self, lanes: int, states: int, perms: int) -> float:
        """Device ms of `perms` dependent permutations on each of `states` states."""
        v = ctypes.c_double()
        self._check(self._lib.dpkem_probe_keccak_chain(self._h, lanes, states, perms, ctypes.byref(v)), "probe_keccak_chain")
        return v.value

    def probe_int_peaks(self):
        """(32-bit LOP3/SHF ops per second in Keccak's mix, Keccak-f[1600] per second)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.dpkem_probe_int_peaks(self._h, ctypes.byref(a), ctypes.byref(b)), "probe")
        return a.value, b.value

    # -- mixed batches ---------------------------------------------------------
    @staticmethod
    def requests(items):
        """items: iterable of (scheme, op, in0, in1, out0, out1) with torch CUDA tensors (or None)."""
        items = list(items)
        arr = (Request * len(items))()
        for k, (scheme, op, a, b, c, e) in enumerate(items):
            ptr = lambda t: t.data_ptr() if t is not None else None  # noqa: E731
            arr[k] = Request(scheme, op, ptr(a), ptr(b), ptr(c), ptr(e))
        return arr

    def mixed(self, items, form: int = FORM_TC, coin_key: bytes | None = None, coin_first: int = 0):
        """Run a mixed-scheme, mixed-operation batch as one persistent launch (device buffers).
        items: (scheme, op, in0, in1, out0, out1) tuples, or a table from Engine.requests.
        With coin_key (32 bytes), keypair / encaps items whose coins are None draw them on the
        device: SHAKE256(coin_key || LE64(coin_first + position) || "kp" / "enc")."""
        import torch

        arr = items if isinstance(items, ctypes.Array) else self.requests(items)  # prebuilt table as is
        st = torch.cuda.current_stream().cuda_stream or 1
        if coin_key is None:
            rc = self._lib.dpkem_mixed_batch(self._h, form, len(arr), ctypes.cast(arr, ctypes.c_void_p),
                                             ctypes.c_void_p(st))
        else:
            if len(coin_key) != 32:
                raise ValueError("coin_key must be 32 bytes")
            rc = self._lib.dpkem_mixed_batch_keyed(self._h, form, len(arr), ctypes.cast(arr, ctypes.c_void_p),
                                                   bytes(coin_key), coin_first, ctypes.c_void_p(st))
        self._check(rc, "mixed_batch")

    def mixed_graph(self, items, form: int = FORM_TC) -> "MixedGraph":
        return MixedGraph(self, items, form)

    def max_chunk(self, scheme: int) -> int:
        return int(self._lib.dpkem_max_chunk(self._h, scheme))


class MixedGraph:
    """A mixed batch captured once as a CUDA graph; launch() replays it on the torch stream."""

    def __init__(self, engine: Engine, items, form: int = FORM_TC):
        self._lib = engine._lib
        self._engine = engine
        arr = engine.requests(items)
        h = ctypes.c_void_p()
        rc = self._lib.dpkem_mixed_graph_create(engine._h, form, len(arr), ctypes.cast(arr, ctypes.c_void_p),
                                                ctypes.byref(h))
        if rc != OK:
            raise DpkemError(rc, "mixed_graph_create")
        self._h = h

    def launch(self):
        import torch

        st = torch.cuda.current_stream().cuda_stream or 1
        rc = self._lib.dpkem_mixed_graph_launch(self._h, ctypes.c_void_p(st))
        if rc != OK:
            raise DpkemError(rc, "mixed_graph_launch")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dpkem_mixed_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Service:
    """A KEM service on an engine's device: one long-lived persistent launch that admits
    requests while it runs (dpkem_service_*).  submit() takes a prefix of the requests (device
    buffers, the mixed batches' layout) and returns (accepted, first_ticket); poll() returns
    the tickets completed since the previous poll as a numpy array."""

    def __init__(self, engine: Engine, form: int = FORM_TC, max_inflight: int | None = None,
                 idle_ms: int | None = None, saber_ctas: int | None = None, warp_max: int | None = None,
                 scratch_bytes: int | None = None, coin_key: bytes | None = None):
        self._lib = engine._lib
        self._engine = engine
        cfg = ServiceConfig()
        rc = self._lib.dpkem_service_default_config(ctypes.byref(cfg))
        if rc != OK:
            raise DpkemError(rc, "service_default_config")
        for k, v in (("max_inflight", max_inflight), ("idle_ms", idle_ms), ("saber_ctas", saber_ctas),
                     ("warp_max", warp_max), ("scratch_bytes", scratch_bytes)):
            if v is not None:
                setattr(cfg, k, int(v))
        self._key = None
        if coin_key is not None:
            if len(coin_key) != 32:
                raise ValueError("coin_key must be 32 bytes")
            self._key = ctypes.create_string_buffer(bytes(coin_key), 32)
            cfg.coin_key = ctypes.cast(self._key, ctypes.c_void_p)
        h = ctypes.c_void_p()
        rc = self._lib.dpkem_service_open(engine._h, form, ctypes.byref(cfg), ctypes.byref(h))
        if rc != OK:
            raise DpkemError(rc, "service_open")
        self._h = h
        self._buf = np.zeros(1 << 16, np.uint64)

    def submit(self, items) -> tuple:
        """items: (scheme, op, in0, in1, out0, out1) tuples, an Engine.requests table, or a numpy
        array with dpkem_request's layout.  Returns (accepted, first_ticket); EAGAIN counts as
        nothing accepted."""
        if isinstance(items, np.ndarray):
            n, ptr = len(items), items.ctypes.data
        else:
            arr = items if isinstance(items, ctypes.Array) else Engine.requests(items)
            n, ptr = len(arr), ctypes.cast(arr, ctypes.c_void_p).value
        acc, first = ctypes.c_size_t(), ctypes.c_uint64()
        rc = self._lib.dpkem_service_submit(self._h, n, ctypes.c_void_p(ptr), ctypes.byref(acc), ctypes.byref(first))
        if rc not in (OK, EAGAIN):
            raise DpkemError(rc, "service_submit")
        return acc.value, first.value

    def poll(self) -> np.ndarray:
        """Tickets completed since the previous poll."""
        got = ctypes.c_size_t()
        rc = self._lib.dpkem_service_poll(self._h, ctypes.c_void_p(self._buf.ctypes.data), len(self._buf),
                                          ctypes.byref(got))
        if rc != OK:
            raise DpkemError(rc, "service_poll")
        return self._buf[:got.value].copy()

    def drain(self, timeout_ms: int = 30000):
        rc = self._lib.dpkem_service_drain(self._h, timeout_ms)
        if rc != OK:
            raise DpkemError(rc, "service_drain")

    def stats(self) -> dict:
        a, b, c, r = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_int()
        rc = self._lib.dpkem_service_stats(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                           ctypes.byref(r))
        if rc != OK:
            raise DpkemError(rc, "service_stats")
        return {"submitted": a.value, "completed": b.value, "launches": c.value, "running": bool(r.value)}

    def counters(self, reset: bool = False) -> dict:
        """Per-queue claims / instances / warp claims / busy ms, keyed "scheme/op/stage", plus
        idle_ms, admissions, admitted and lost_claims (dpkem_service_counters)."""
        buf = np.zeros(244, np.uint64)
        rc = self._lib.dpkem_service_counters(self._h, ctypes.c_void_p(buf.ctypes.data), len(buf), int(reset))
        if rc != OK:
            raise DpkemError(rc, "service_counters")
        out = {}
        for q in range(60):
            c = buf[4 * q:4 * q + 4]
            if c[0]:
                out[f"{q // 12}/{(q >> 2) % 3}/{q & 3}"] = {"claims": int(c[0]), "instances": int(c[1]),
                                                          "warp_claims": int(c[2]), "busy_ms": float(c[3]) * 1e-6}
        out["idle_ms"] = float(buf[240]) * 1e-6
        out["admissions"], out["admitted"], out["lost_claims"] = int(buf[241]), int(buf[242]), int(buf[243])
        return out

    def close(self):
        if getattr(self, "_h", None):
            rc = self._lib.dpkem_service_close(self._h)
            self._h = None
            if rc != OK:
                raise DpkemError(rc, "service_close")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- reference-named entry points (batch from set_compat_batch, default 768) ----
def set_compat(batch: int | None = None, saber_level: int | None = None, form: int | None = None):
    lib = load()
    if batch is not None:
        lib.dpkem_set_compat_batch(batch)
    if saber_level is not None:
        lib.dpkem_set_compat_saber_level(saber_level)
    if form is not None:
        lib.dpkem_set_compat_form(form)


def _last(what: str):
    rc = load().dpkem_last_status()
    if rc != OK:
        raise DpkemError(rc, what)


def frodoKEMKeypair(h_pk: np.ndarray, h_sk: np.ndarray) -> None:
    load().frodoKEMKeypair(_ptr(h_pk), _ptr(h_sk))
    _last("frodoKEMKeypair")


def frodoKEMEncap(ct: np.ndarray, ss: np.ndarray, pk: np.ndarray) -> None:
    load().frodoKEMEncap(_ptr(ct), _ptr(ss), _ptr(pk))
    _last("frodoKEMEncap")


def frodoKEMDecap(ss: np.ndarray, ct: np.ndarray, sk: np.ndarray) -> None:
    load().frodoKEMDecap(_ptr(ss), _ptr(ct), _ptr(sk))
    _last("frodoKEMDecap")


def saber_enc(mode: int, h_k: np.ndarray, h_pk: np.ndarray, h_c: np.ndarray) -> None:
    load().saber_enc(mode, _ptr(h_k), _ptr(h_pk), _ptr(h_c))
    _last("saber_enc")


def saber_dec(mode: int, h_c: np.ndarray, h_pk: np.ndarray, h_sk: np.ndarray, h_k: np.ndarray) -> None:
    load().saber_dec(mode, _ptr(h_c), _ptr(h_pk), _ptr(h_sk), _ptr(h_k))
    _last("saber_dec")
