"""Continuous-batching KEM serving loop over the mixed-batch entry point.

Requests (encaps / decaps on FrodoKEM-976 or Saber, each with its own device buffers)
arrive over time.  The loop keeps `slots` independent engines (a dpkem context each: own
scratch arena, own CUDA stream).  Whenever a slot is free and requests are waiting, it
admits up to `max_batch` of them (bounded by the slot's HBM budget) as one persistent
mixed-batch launch on that slot's stream, so batches admitted while others run overlap
on the device.  Per-request state (scratch records, inputs, outputs) stays on the GPU.
Completion times are device times (CUDA events against a start event), arrival times are
host times on the same origin; latency = completion - arrival.

The reference has no serving path: its drivers run one fixed batch per program
(FrodoKEM976-GPU/main.cu:13-34, SABER-GPU/main.cu:12-38).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import kem as K

REQ_DTYPE = np.dtype([("scheme", "<i4"), ("op", "<i4"), ("in0", "<u8"), ("in1", "<u8"), ("out0", "<u8"),
                      ("out1", "<u8")])
assert REQ_DTYPE.itemsize == ctypes.sizeof(K.Request)


class RequestPool:
    """Pre-built encaps/decaps requests with device buffers and their expected outputs.

    mix: fraction of encaps (else decaps) and of Frodo (else Saber l=3)."""

    def __init__(self, eng: K.Engine, n: int, enc_frac: float = 0.6, frodo_frac: float = 0.5, seed: int = 0):
        rng = np.random.default_rng(seed)
        self.n = n
        is_enc = rng.random(n) < enc_frac
        is_frodo = rng.random(n) < frodo_frac
        self.table = np.zeros(n, REQ_DTYPE)
        self.expected, self.outputs = [], []
        self.kind = np.zeros(n, np.int32)  # scheme * 3 + op
        for scheme, mask in ((K.FRODO976, is_frodo), (K.SABER, ~is_frodo)):
            z = K.sizes(scheme)
            idx_enc = np.nonzero(mask & is_enc)[0]
            idx_dec = np.nonzero(mask & ~is_enc)[0]
            m = len(idx_enc) + len(idx_dec)
            if m == 0:
                continue
            kc = torch.empty((m, z["kp_coins"]), dtype=torch.uint8, device="cuda")
            ec = torch.empty((m, z["enc_coins"]), dtype=torch.uint8, device="cuda")
            eng.coins(m, z["kp_coins"], "srv-kp", first=seed * 10000000 + scheme * 1000000, out=kc)
            eng.coins(m, z["enc_coins"], "srv-enc", first=seed * 10000000 + scheme * 1000000, out=ec)
            pk, sk = eng.keypair(scheme, kc, K.FORM_TC)
            ct, ss = eng.enc(scheme, pk, ec, K.FORM_TC)
            torch.cuda.synchronize()
            ne = len(idx_enc)
            oct_ = torch.empty((max(1, ne), z["ct"]), dtype=torch.uint8, device="cuda")
            oss = torch.empty((m, z["ss"]), dtype=torch.uint8, device="cuda")
            self.outputs += [oct_, oss]
            self.expected += [(oct_[:ne], ct[:ne]), (oss, ss)]
            self._keep = getattr(self, "_keep", []) + [kc, ec, pk, sk, ct, ss]

            def rows(t, idx):
                return t.data_ptr() + np.asarray(idx, np.uint64) * np.uint64(t.shape[1])

            j_enc, j_dec = np.arange(ne), np.arange(ne, m)
            t = self.table
            t["scheme"][idx_enc], t["op"][idx_enc] = scheme, 1
            t["in0"][idx_enc], t["in1"][idx_enc] = rows(ec, j_enc), rows(pk, j_enc)
            t["out0"][idx_enc], t["out1"][idx_enc] = rows(oct_, np.arange(ne)), rows(oss, j_enc)
            t["scheme"][idx_dec], t["op"][idx_dec] = scheme, 2
            t["in0"][idx_dec], t["in1"][idx_dec] = rows(ct, j_dec), rows(sk, j_dec)
            t["out0"][idx_dec], t["out1"][idx_dec] = rows(oss, j_dec), 0
            self.kind[idx_enc] = scheme * 3 + 1
            self.kind[idx_dec] = scheme * 3 + 2

    def clear(self):
        for t in self.outputs:
            t.zero_()

    def check(self) -> bool:
        return all(torch.equal(got, ref) for got, ref in self.expected)


class Server:
    def __init__(self, device: int = 0, slots: int = 4, max_batch: int = 4096, form: int = K.FORM_TC,
                 hbm_budget: int = 1 << 30):
        self.slots = [K.Engine(device, hbm_budget=hbm_budget) for _ in range(slots)]
        self.streams = [torch.cuda.Stream(device) for _ in range(slots)]
        self.max_batch = max_batch
        self.form = form
        self.lib = K.load()

    def close(self):
        for e in self.slots:
            e.close()

    def _submit(self, k: int, table: np.ndarray):
        eng, st = self.slots[k], self.streams[k]
        rc = self.lib.dpkem_mixed_batch(eng._h, self.form, len(table), ctypes.c_void_p(table.ctypes.data),
                                        ctypes.c_void_p(st.cuda_stream))
        if rc != K.OK:
            raise K.DpkemError(rc, "mixed_batch")
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(st)
        return ev

    def run(self, pool: RequestPool, arrivals: np.ndarray) -> dict:
        """Serve pool requests 0..len(arrivals)-1 arriving at the given times (seconds)."""
        n = len(arrivals)
        done_ms = np.full(n, np.nan)
        busy = [None] * len(self.slots)  # (event, first, last)
        t_origin = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t_origin.record(self.streams[0])
        torch.cuda.synchronize()
        host0 = time.perf_counter()
        nxt = 0
        batches = []
        prev, max_gap = 0.0, 0.0  # longest pause of this loop: a host stall, not device time
        while nxt < n or any(b is not None for b in busy):
            now = time.perf_counter() - host0
            max_gap, prev = max(max_gap, now - prev), now
            for k, b in enumerate(busy):
                if b is not None and b[0].query():
                    done_ms[b[1]:b[2]] = t_origin.elapsed_time(b[0])
                    busy[k] = None
            arrived = int(np.searchsorted(arrivals, now, side="right"))
            free = [k for k, b in enumerate(busy) if b is None]
            if nxt < arrived and free:
                last = min(arrived, nxt + self.max_batch)
                k = free[0]
                busy[k] = (self._submit(k, pool.table[nxt:last]), nxt, last)
                batches.append(last - nxt)
                nxt = last
                continue
            if nxt < n and not free:
                time.sleep(20e-6)
            elif nxt < n and arrived == nxt:
                time.sleep(min(max(arrivals[nxt] - now, 0.0), 200e-6))
            else:
                time.sleep(20e-6)
        for e in self.slots:
            e.sync()
        lat = done_ms - arrivals * 1e3
        span = (np.nanmax(done_ms) - arrivals[0] * 1e3) * 1e-3
        return {"requests": n, "ops_per_s": n / span, "p50_ms": float(np.nanpercentile(lat, 50)),
                "p99_ms": float(np.nanpercentile(lat, 99)), "mean_batch": float(np.mean(batches)),
                "batches": len(batches), "host_max_gap_ms": max_gap * 1e3, "latency_ms": lat}


def poisson_arrivals(n: int, rate: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))
