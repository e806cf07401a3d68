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
        self._views = [None] * n
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
            for j, r in enumerate(idx_enc):
                self._views[r] = (scheme, 1, ec[j], pk[j], oct_[j], oss[j])
            for j, r in zip(j_dec, idx_dec):
                self._views[r] = (scheme, 2, ct[j], sk[j], oss[j], None)

    def clear(self):
        for t in self.outputs:
            t.zero_()

    def check(self) -> bool:
        return all(torch.equal(got, ref) for got, ref in self.expected)

    def items(self) -> list:
        """Request i as (scheme, op, in0, in1, out0, out1) device tensors, in the order the
        mixed entry points take them (out1 None for decaps)."""
        return list(self._views)


FRODO_CLASS, SABER_CLASS = 0, 1


class Server:
    """slots engines (a dpkem context and a CUDA stream each).  classes: None, every slot
    takes any request; or one entry per slot, FRODO_CLASS (FrodoKEM-976, both variants) or
    SABER_CLASS, and a request is admitted only to a slot of its class.  Splitting keeps a
    Saber request (a ~0.3 ms chain) from waiting for the Frodo requests admitted with it
    (a ~4 ms chain: a 348-permutation prologue sponge, then a 976-row product per CTA)."""

    def __init__(self, device: int = 0, slots: int = 4, max_batch: int = 4096, form: int = K.FORM_TC,
                 hbm_budget: int = 1 << 30, classes=None, saber_share: float = 0.25):
        self.slots = [K.Engine(device, hbm_budget=hbm_budget) for _ in range(slots)]
        self.streams = [torch.cuda.Stream(device) for _ in range(slots)]
        self.classes = list(classes) if classes is not None else [None] * slots
        if len(self.classes) != slots:
            raise ValueError("one class per slot")
        if classes is not None:
            # Each launch is a persistent kernel that holds its CTAs until its queue drains, so
            # the classes split the GPU's resident CTAs (two per SM): saber_share of them for
            # the Saber slots, the rest for the Frodo slots, each class's share divided among
            # its slots.  A Saber launch then never waits for a Frodo launch's CTAs.
            total = 2 * torch.cuda.get_device_properties(device).multi_processor_count
            n_s = self.classes.count(SABER_CLASS)
            n_f = self.classes.count(FRODO_CLASS)
            saber_ctas = max(n_s, int(round(total * saber_share))) if n_s else 0
            for k, c in enumerate(self.classes):
                share = saber_ctas // n_s if c == SABER_CLASS else (total - saber_ctas) // max(1, n_f)
                self.slots[k].set_max_ctas(max(1, share))
        self.max_batch = max_batch
        self.form = form
        self.lib = K.load()
        # size every slot's arena for a full batch of the largest requests now: growing it
        # later would wait for the whole device (all slots) in the middle of serving
        need = int(self.lib.dpkem_mixed_bytes(K.FRODO976, max_batch))
        for e in self.slots:
            e.reserve(min(need, hbm_budget))

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
        req_class = np.where(pool.kind[:n] // 3 >= 2, SABER_CLASS, FRODO_CLASS)
        keys = sorted({c for c in self.classes}, key=lambda c: -1 if c is None else c)
        queues = {c: (np.arange(n) if c is None else np.nonzero(req_class == c)[0]) for c in keys}
        q_arr = {c: arrivals[q] for c, q in queues.items()}
        q_next = {c: 0 for c in keys}
        done_ms = np.full(n, np.nan)
        busy = [None] * len(self.slots)  # (event, request indices)
        t_origin = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t_origin.record(self.streams[0])
        torch.cuda.synchronize()
        host0 = time.perf_counter()
        batches, submit_s = [], []
        prev, max_gap = 0.0, 0.0  # longest pause of this loop: a host stall, not device time
        while any(q_next[c] < len(queues[c]) for c in keys) or any(b is not None for b in busy):
            now = time.perf_counter() - host0
            max_gap, prev = max(max_gap, now - prev), now
            for k, b in enumerate(busy):
                if b is not None and b[0].query():
                    done_ms[b[1]] = t_origin.elapsed_time(b[0])
                    busy[k] = None
            submitted = False
            for c in keys:
                arrived = int(np.searchsorted(q_arr[c], now, side="right"))
                if q_next[c] >= arrived:
                    continue
                free = [k for k, b in enumerate(busy) if b is None and self.classes[k] == c]
                if not free:
                    continue
                last = min(arrived, q_next[c] + self.max_batch)
                idx = queues[c][q_next[c]:last]
                t_sub = time.perf_counter()
                busy[free[0]] = (self._submit(free[0], np.ascontiguousarray(pool.table[idx])), idx)
                submit_s.append(time.perf_counter() - t_sub)
                batches.append(len(idx))
                q_next[c] = last
                submitted = True
            if submitted:
                continue
            waits = [q_arr[c][q_next[c]] - now for c in keys if q_next[c] < len(queues[c])]
            time.sleep(min(max(min(waits), 0.0), 200e-6) if waits and min(waits) > 0 else 20e-6)
        for e in self.slots:
            e.sync()
        lat = done_ms - arrivals * 1e3
        span = (np.nanmax(done_ms) - arrivals[0] * 1e3) * 1e-3
        out = {"requests": n, "ops_per_s": n / span, "p50_ms": float(np.nanpercentile(lat, 50)),
               "p99_ms": float(np.nanpercentile(lat, 99)), "mean_batch": float(np.mean(batches)),
               "batches": len(batches), "host_max_gap_ms": max_gap * 1e3, "latency_ms": lat,
               "submit_ms_max": max(submit_s) * 1e3, "submit_ms_mean": float(np.mean(submit_s)) * 1e3}
        for c, name in ((FRODO_CLASS, "frodo"), (SABER_CLASS, "saber")):
            m = req_class == c
            if m.any():
                out[name + "_p50_ms"] = float(np.nanpercentile(lat[m], 50))
                out[name + "_p99_ms"] = float(np.nanpercentile(lat[m], 99))
        return out


class ServiceServer:
    """Serving through one KEM service (dpkem_service_*): each request is submitted to the
    running kernel as soon as it arrives (admission inside the launch, no batching window on
    the host), and its completion is the host time at which a poll first returns its
    ticket.  saber_ctas CTAs take only Saber work, so a Saber request never waits behind
    the multi-millisecond FrodoKEM stages."""

    def __init__(self, device: int = 0, form: int = K.FORM_TC, saber_ctas: int = 32, warp_max: int | None = None,
                 max_inflight: int = 16384, idle_ms: int = 200):
        self.eng = K.Engine(device)
        self.svc = K.Service(self.eng, form, max_inflight=max_inflight, idle_ms=idle_ms, saber_ctas=saber_ctas,
                             warp_max=warp_max)

    def close(self):
        self.svc.close()
        self.eng.close()

    def run(self, pool: RequestPool, arrivals: np.ndarray) -> dict:
        """Serve pool requests 0..len(arrivals)-1 arriving at the given times (seconds)."""
        n = len(arrivals)
        base = self.svc.stats()["submitted"]  # tickets of this run: base + request index
        done_s = np.full(n, np.nan)
        nxt, completed, polls, submits = 0, 0, 0, 0
        host0 = time.perf_counter()
        while completed < n:
            now = time.perf_counter() - host0
            arrived = int(np.searchsorted(arrivals, now, side="right"))
            if arrived > nxt:
                acc, first = self.svc.submit(pool.table[nxt:arrived])
                if acc:
                    assert first == base + nxt
                    nxt += acc
                    submits += 1
            got = self.svc.poll()
            polls += 1
            if len(got):
                done_s[got.astype(np.int64) - base] = time.perf_counter() - host0
                completed += len(got)
            elif nxt == arrived and nxt < n:
                wait = arrivals[nxt] - (time.perf_counter() - host0)
                if wait > 50e-6:
                    time.sleep(min(wait, 200e-6) - 20e-6)
        lat = (done_s - arrivals) * 1e3
        span = np.nanmax(done_s) - arrivals[0]
        out = {"requests": n, "ops_per_s": n / span, "p50_ms": float(np.nanpercentile(lat, 50)),
               "p99_ms": float(np.nanpercentile(lat, 99)), "latency_ms": lat, "submits": submits,
               "mean_submit": n / max(1, submits), "polls": polls}
        saber = pool.kind[:n] // 3 >= 2
        for m, name in ((~saber, "frodo"), (saber, "saber")):
            if m.any():
                out[name + "_p50_ms"] = float(np.nanpercentile(lat[m], 50))
                out[name + "_p99_ms"] = float(np.nanpercentile(lat[m], 99))
        return out


def poisson_arrivals(n: int, rate: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))
