#!/usr/bin/env python3
"""Benchmark: FrodoKEM-976-SHAKE encaps+decaps per second at batch 8192 per GPU.

One step = encaps of the batch followed by decaps of the resulting ciphertexts
(independent keypairs per instance, generated once before timing).  The headline
form is the int8 tcgen05 product; the dp4a form and Saber (l=3, batch 4096) are
measured on the same GPU and reported beside it.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU (torchrun, one rank per GPU): every rank runs its own batch (weak scaling,
no data-path collective); value = instances of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "KEM encaps+decaps/sec at batch 8192 (int8 TC vs dp4a, bit-exact); p99 latency"
UNIT = "encaps+decaps/s"
# 32-bit LOP3/SHF operations of one Keccak-f[1600] in its minimal form: per round theta
# 20 (column parities) + 10 (rot1) + 50 (3-input XOR into the lanes), rho 48, chi 50,
# iota 2 = 180; x 24 rounds.
KECCAK_INT_OPS = 4320
FRODO_ROWS, FRODO_BLOCKS = 976, 12      # A rows per instance, SHAKE128 blocks per row
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "frodo_sa_tc_traffic.json")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--batch", type=int, default=8192)
    p.add_argument("--form", default="tc", choices=["tc", "dp4a", "int32"])
    p.add_argument("--scheme", default="frodo976", choices=["frodo976", "frodo976aes"],
                   help="headline workload: FrodoKEM-976-SHAKE (default) or FrodoKEM-976-AES")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-secondary", action="store_true")
    return p.parse_args()


def dist_env():
    from dpcrypto_b200.dist import env

    return env()


SCHEME_NAMES = {"frodo976": "FrodoKEM-976-SHAKE", "frodo976aes": "FrodoKEM-976-AES"}


def config(args, world):
    name = SCHEME_NAMES[args.scheme]
    return {
        "workload": f"{name} encaps+decaps, batch {args.batch} per GPU, {args.form} product form",
        "scheme": name, "batch_per_gpu": args.batch, "global_batch": args.batch * world,
        "form": args.form, "parallelism": f"instances sharded, {world} replica(s)",
        "l2": "inputs larger than L2 (pk+sk+ct per step = %d MB per GPU)" % (args.batch * (15632 + 31296 + 15744) >> 20),
    }


# ---------------------------------------------------------------- CPU (oracle) arms
def cpu_sample(n_inst: int, threads: int):
    """Time the oracle's encaps+decaps on n_inst instances over `threads` host threads."""
    from oracle import oracle as O

    pk, sk = O.keypair(0, O.coins(n_inst, 64, "kp"), threads=threads)
    ec = O.coins(n_inst, 24, "enc")
    t0 = time.perf_counter()
    ct, ss = O.enc(0, pk, ec, threads=threads)
    ss2 = O.dec(0, ct, sk, threads=threads)
    dt = time.perf_counter() - t0
    assert (ss == ss2).all()
    return n_inst / dt, dt


def cpu_sample_saber(n_inst: int, threads: int):
    """Time the oracle's Saber l=3 encaps+decaps on n_inst instances over `threads` host threads."""
    from oracle import oracle as O

    pk, sk = O.keypair(3, O.coins(n_inst, 96, "kp"), threads=threads)
    ec = O.coins(n_inst, 32, "enc")
    t0 = time.perf_counter()
    ct, ss = O.enc(3, pk, ec, threads=threads)
    ss2 = O.dec(3, ct, sk, threads=threads)
    dt = time.perf_counter() - t0
    assert (ss == ss2).all()
    return n_inst / dt, dt


CPU_BUILD = "oracle C port built on this host with gcc -O3 -march=native (unrolled Keccak-f, vectorised products)"


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    from oracle import oracle as O

    O.use_native()
    threads = os.cpu_count() or 1
    per_step = 16 * threads
    for _ in range(args.warmup):
        cpu_sample(per_step, threads)
    times = []
    for _ in range(args.steps):
        _, dt = cpu_sample(per_step, threads)
        times.append(dt)
    total = sum(times)
    value = per_step * args.steps / total
    v1, dt1 = cpu_sample(16, 1)
    sample = f"{per_step} FrodoKEM-976 encaps+decaps per step (16 per host thread), {CPU_BUILD}, pthreads"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64/u16 (CPU)",
        "data": "synthetic (seeded SHAKE256 coins)", "config": config(args, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                         "value_1core": v1, "sample_1core": f"16 instances on 1 thread, {dt1:.2f} s wall"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU helpers
ONE_LANE = dict(saber_warp_max=0, saber_finish_warp_max=0, saber_five_max=0, saber_finish_five_max=0,
                saber_pair_max=0, frodo_warp_max=0, frodo_ss_warp_max=0, frodo_five_max=0, frodo_ss_five_max=0)


def bench_single(eng, reps: int = 7) -> dict:
    """One request alone (n = 1, tc form): per-stage device times (stage timer, median of
    `reps`) of FrodoKEM-976 and Saber l=3 encaps and decaps, the sponge stages on a warp per
    state (the default at this size) and on one thread per state."""
    import numpy as np
    import torch

    import dpcrypto_b200 as d
    from dpcrypto_b200 import kem as K

    out = {}
    for scheme, name in ((d.FRODO976, "frodo976"), (d.SABER, "saber_l3")):
        z = d.sizes(scheme)
        kc = torch.empty((1, z["kp_coins"]), dtype=torch.uint8, device="cuda")
        ec = torch.empty((1, z["enc_coins"]), dtype=torch.uint8, device="cuda")
        eng.coins(1, z["kp_coins"], "single-kp", out=kc)
        eng.coins(1, z["enc_coins"], "single-enc", out=ec)
        pk, sk = eng.keypair(scheme, kc, d.FORM_TC)
        ct = torch.empty((1, z["ct"]), dtype=torch.uint8, device="cuda")
        ss = torch.empty((1, z["ss"]), dtype=torch.uint8, device="cuda")
        res = {"enc_stages": ["prologue", "product", "final hash"] if scheme == d.FRODO976 else
               ["prologue", "product", "finish"],
               "dec_stages": ["W / decode", "prologue", "product", "final hash"] if scheme == d.FRODO976 else
               ["inner product", "prologue", "product", "finish"]}
        for layout, kv in (("warp_per_state", {}), ("one_lane", ONE_LANE)):
            with K.knobs(**kv):
                eng.enc(scheme, pk, ec, d.FORM_TC, out=(ct, ss))
                eng.dec(scheme, ct, sk, d.FORM_TC)
                torch.cuda.synchronize()
                eng.profile(True)
                es, ds = [], []
                for _ in range(reps):
                    eng.enc(scheme, pk, ec, d.FORM_TC, out=(ct, ss))
                    es.append(eng.stage_times())
                    eng.dec(scheme, ct, sk, d.FORM_TC)
                    ds.append(eng.stage_times())
                eng.profile(False)
            enc, dec = np.median(np.array(es), axis=0), np.median(np.array(ds), axis=0)
            res[layout] = {"enc_stage_ms": [round(float(x), 4) for x in enc],
                           "dec_stage_ms": [round(float(x), 4) for x in dec],
                           "enc_ms": float(enc.sum()), "dec_ms": float(dec.sum())}
        out[name] = res
    return out


def bench_frames(eng, form, n: int = 16384, reps: int = 3) -> dict:
    """dpkem_frames_run on n mixed request frames (pinned host block in, pinned block out,
    copies inside the timing), and the same block served through the ring by the frame
    server process (client push -> last response popped)."""
    import tempfile

    import numpy as np
    import torch

    import dpcrypto_b200 as d
    from dpcrypto_b200 import frames as F
    from dpcrypto_b200.workloads import mixed_frames

    blk = mixed_frames(eng, n, seed=0)
    _, _, rb = F.scan(blk)
    req = torch.from_numpy(blk).pin_memory().numpy()
    resp = torch.empty(rb, dtype=torch.uint8).pin_memory().numpy()
    F.run(eng, req, form, out=resp)
    t = time.perf_counter()
    for _ in range(reps):
        F.run(eng, req, form, out=resp)
    dt = (time.perf_counter() - t) / reps
    out = {"requests": n, "unit": "KEM ops/s", "mix": "4 schemes x 3 ops, uniform, shuffled",
           "frames_run": {"ops_per_s": n / dt, "ms_per_block": dt * 1e3, "request_bytes": int(blk.nbytes),
                          "response_bytes": int(rb)}}
    # through the ring, served by another process
    shm = "/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir()
    path = os.path.join(shm, f"dpkem-bench-{os.getpid()}.ring")
    cap = 128 << 20
    ring = F.Ring(path, capacity=cap)
    fname = {d.FORM_TC: "tc", d.FORM_DP4A: "dp4a", d.FORM_INT32: "int32"}[form]
    proc = subprocess.Popen([sys.executable, "-m", "dpcrypto_b200.frame_server", "--ring", path, "--form", fname,
                             "--max-frames", "4096", "--idle-us", "20", "--inflight", "2"], cwd=os.path.dirname(os.path.abspath(__file__)))
    try:
        popbuf = np.empty(rb, np.uint8)
        for rep in range(2):  # the first pass warms the server up
            n_got, n_bytes, pending = 0, 0, req
            t = time.perf_counter()
            deadline = t + 300
            while n_got < n:
                if time.perf_counter() > deadline or proc.poll() is not None:
                    raise RuntimeError("frame server stalled or exited")
                if len(pending):
                    pending = pending[ring.push(pending):]
                r, count = ring.pop(out=popbuf[n_bytes:])
                n_bytes += len(r)
                n_got += count
            dt = time.perf_counter() - t
        same = bool(n_bytes == rb and np.array_equal(popbuf, resp))
        out["ring_external_process"] = {"ops_per_s": n / dt, "ms_per_block": dt * 1e3, "ring_capacity": cap,
                                        "max_frames_per_batch": 4096, "batches_in_flight": 2,
                                        "bit_exact_vs_frames_run": same}
    finally:
        ring.stop()
        proc.wait(timeout=60)
        ring.close()
        os.unlink(path)
    return out


def pcie_gbs(h2d: bool, nbytes: int = 256 << 20) -> float:
    """Pinned host<->device copy bandwidth (GB/s) of one 256 MiB buffer, CUDA-event timed."""
    import torch

    h = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    g = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for k in range(4):
        if k == 1:
            a.record()
        (g.copy_(h, non_blocking=True) if h2d else h.copy_(g, non_blocking=True))
    b.record()
    b.synchronize()
    return 3 * nbytes / (a.elapsed_time(b) * 1e-3) / 1e9


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        rows = getattr(self, "rows", [])
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1])]
        smax = max((num(r[2]) for r in rows if num(r[2])), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows), "power_w_max": max((num(r[3]) or 0) for r in rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def main():
    args = parse()
    world, rank, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, world, rank)

    import numpy as np
    import torch

    import dpcrypto_b200 as d

    torch.cuda.set_device(local)
    from dpcrypto_b200 import dist as D

    pg = D.init("nccl", timeout_s=120.0, device=torch.device("cuda", local)) if world > 1 else None
    eng = d.Engine(local)
    form = {"tc": d.FORM_TC, "dp4a": d.FORM_DP4A, "int32": d.FORM_INT32}[args.form]
    FS = {"frodo976": d.FRODO976, "frodo976aes": d.FRODO976AES}[args.scheme]
    B = args.batch
    stream = torch.cuda.current_stream()

    # ---- inputs: keypairs and coins generated on the device, untimed ----
    first, _ = D.shard(B, rank)
    kc = torch.empty((B, 64), dtype=torch.uint8, device="cuda")
    ec = torch.empty((B, 24), dtype=torch.uint8, device="cuda")
    eng.coins(B, 64, "kp", first=first, out=kc)
    eng.coins(B, 24, "enc", first=first, out=ec)
    pk, sk = eng.keypair(FS, kc, d.FORM_TC)
    ct = torch.empty((B, 15744), dtype=torch.uint8, device="cuda")
    ss = torch.empty((B, 24), dtype=torch.uint8, device="cuda")
    ss2 = torch.empty((B, 24), dtype=torch.uint8, device="cuda")

    def step(f):
        eng.enc(FS, pk, ec, f, out=(ct, ss))
        eng.dec(FS, ct, sk, f, out=ss2)

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()

    def timed(f, steps, profile=False):
        """Device time of `steps` steps on torch's stream (max over ranks) + per-stage times."""
        stages = {"enc": [], "dec": []}
        eng.profile(profile)
        barrier()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(steps):
            eng.enc(FS, pk, ec, f, out=(ct, ss))
            if profile:
                stages["enc"].append(eng.stage_times())
            eng.dec(FS, ct, sk, f, out=ss2)
            if profile:
                stages["dec"].append(eng.stage_times())
        t1.record(stream)
        barrier()
        eng.profile(False)
        ms = D.max_over_ranks(t0.elapsed_time(t1), device="cuda")
        return ms, stages

    for _ in range(args.warmup):
        step(form)
    barrier()
    sampler = ClockSampler(local)
    with sampler:
        ms, stages = timed(form, args.steps, profile=True)
    clocks = sampler.summary()
    eng.sync()
    ok = bool(torch.equal(ss, ss2))
    value = world * B * args.steps / (ms * 1e-3)

    # ---- roofline of the dominant kernel (the fused A-generation + S'A product) ----
    sa_ms = [s[1] for s in stages["enc"]] + [s[2] for s in stages["dec"]]
    sa_avg = statistics.mean(sa_ms)
    ops_per_launch = B * FRODO_ROWS * FRODO_BLOCKS * KECCAK_INT_OPS
    int_peak, keccak_peak = eng.probe_int_peaks()
    achieved = ops_per_launch / (sa_avg * 1e-3) / 1e9
    traffic = None
    if os.path.exists(TRAFFIC_FILE):
        with open(TRAFFIC_FILE) as f:
            traffic = json.load(f)["dram_bytes_per_instance"] * B
    stage_names = {"enc": ["prologue", "sa_product", "final_hash"], "dec": ["w_decode", "prologue", "sa_product",
                                                                             "final_hash"]}
    stage_ms = {op: dict(zip(stage_names[op], [statistics.mean(x) for x in zip(*stages[op])])) for op in stages}
    kernel_total = sum(sum(v.values()) for v in stage_ms.values())

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {d.FORM_TC: "u8xs8->s32 (tcgen05 kind::i8), u64 Keccak lanes", d.FORM_DP4A: "s16xs8->s32 (dp2a)",
                  d.FORM_INT32: "int32 multiply-add"}[form],
        "data": "synthetic (seeded SHAKE256 coins, keypairs generated on the GPU)", "config": config(args, world),
        "bit_exact_roundtrip": ok, "gpu_launches": 7 * args.steps,
        "roofline": {
            "kernel": "sa_tc_kernel (SHAKE128 A rows in registers -> int8 tcgen05 S'A)" if form == d.FORM_TC
            else "sa_dp4a_kernel" + ("<int32>" if form == d.FORM_INT32 else ""), "bound": "int", "unit": "Gop/s",
            "achieved": achieved, "peak": int_peak / 1e9, "frac": achieved * 1e9 / int_peak,
            "peak_source": "measured in-process: LOP3/SHF issue rate in Keccak's mix (dpkem_probe_int_peaks)",
            "algorithmic": f"{KECCAK_INT_OPS} int32 ops per Keccak-f x 12 per A row x 976 rows x batch",
            "avg_launch_ms": sa_avg, "traffic": traffic,
            "keccak_per_s": B * FRODO_ROWS * FRODO_BLOCKS / (sa_avg * 1e-3),
            "keccak_peak_per_s": keccak_peak,
        },
        "stage_ms": stage_ms, "stage_share_of_step": {k: sum(v.values()) / kernel_total for k, v in stage_ms.items()},
        "clocks": clocks,
    }
    # tensor pipe: the products' algorithmic int8 MACs (two u8 limbs per 16-bit entry of A)
    # against the measured kind::i8 MMA peak; tiny for Frodo, whose kernel is Keccak-bound
    i8_peak = eng.probe_i8_mma_peak()
    frodo_macs = B * FRODO_ROWS * FRODO_ROWS * 8 * 2
    line["tensor"] = {"i8_mma_peak_macs_per_s": i8_peak, "peak_source": "measured in-process (dpkem_probe_i8_mma_peak)",
                      "frodo_sa_int8_macs_per_s": frodo_macs / (sa_avg * 1e-3),
                      "frodo_sa_frac": frodo_macs / (sa_avg * 1e-3) / i8_peak,
                      "algorithmic": "S'A: 8 x 976 x 976 MACs x 2 limbs per instance"}
    if FS == d.FRODO976AES:  # A from AES-128 T-tables: integer ALU and load/store pipes, no Keccak
        line["roofline"] = {
            "kernel": "sa_tc_kernel<AesRows> (AES-128 A rows -> int8 tcgen05 S'A)" if form == d.FORM_TC
            else "sa_dp4a_kernel<AesRows>", "bound": "int+lsu", "unit": "G AES blocks/s",
            "achieved": B * FRODO_ROWS * 126 / (sa_avg * 1e-3) / 1e9, "peak": None, "frac": None,
            "algorithmic": "126 AES-128 blocks per A row (12 x 10.5) x 976 rows x batch",
            "avg_launch_ms": sa_avg, "traffic": None,
            "note": "no single-pipe peak: ALU and LSU both ~73 % busy (profiles/frodo976aes_sa_tc_b1184.md)",
        }

    # ---- end to end through the public API with pinned host buffers (measured right after
    #      the headline, before the secondary sections leave other state behind) ----
    if not args.no_e2e:
        pin = lambda t: t.cpu().pin_memory().numpy()  # noqa: E731
        h_pk, h_sk, h_ec = pin(pk), pin(sk), pin(ec)
        h_ct = torch.empty((B, 15744), dtype=torch.uint8).pin_memory().numpy()
        h_ss = torch.empty((B, 24), dtype=torch.uint8).pin_memory().numpy()
        h_ss2 = torch.empty((B, 24), dtype=torch.uint8).pin_memory().numpy()
        for _ in range(max(1, args.warmup)):
            eng.enc(FS, h_pk, h_ec, form, out=(h_ct, h_ss))
            eng.dec(FS, h_ct, h_sk, form, out=h_ss2)
        barrier()
        t = time.perf_counter()
        for _ in range(args.steps):
            eng.enc(FS, h_pk, h_ec, form, out=(h_ct, h_ss))
            eng.dec(FS, h_ct, h_sk, form, out=h_ss2)
        el = D.max_over_ranks(time.perf_counter() - t, device="cuda")
        h2d_b, d2h_b = B * (15632 + 24 + 15744 + 31296), B * (15744 + 24 + 24)
        h2d_gbs, d2h_gbs = pcie_gbs(True), pcie_gbs(False)
        line["e2e"] = {"value": world * B * args.steps / el, "unit": UNIT,
                       "h2d_bytes_per_step": h2d_b, "d2h_bytes_per_step": d2h_b,
                       "roundtrip_ok": bool((h_ss == h_ss2).all()),
                       "pipeline_chunks": d.kem.get_tuning().get("pipe_chunks"),
                       "pipeline_stream_priorities": bool(d.kem.get_tuning().get("pipe_priority")),
                       "pcie_gbs": {"h2d": h2d_gbs, "d2h": d2h_gbs},
                       "copy_ms_per_step_if_serial": 1e3 * (h2d_b / (h2d_gbs * 1e9) + d2h_b / (d2h_gbs * 1e9))}

    # ---- the other product forms (tc / dp4a / int32) on the same GPU ----
    if not args.no_secondary:
        fnames = {d.FORM_TC: "tc", d.FORM_DP4A: "dp4a", d.FORM_INT32: "int32"}
        forms = {fnames[form]: value}
        sa_k = {fnames[form]: sa_avg}
        for other in (d.FORM_TC, d.FORM_DP4A, d.FORM_INT32):
            if other == form:
                continue
            for _ in range(2):
                step(other)
            osteps = max(3, args.steps // 2)
            oms, ostages = timed(other, osteps, profile=True)
            forms[fnames[other]] = world * B * osteps / (oms * 1e-3)
            sa_k[fnames[other]] = statistics.mean([s[1] for s in ostages["enc"]] + [s[2] for s in ostages["dec"]])
        line["forms"] = dict(forms, sa_kernel_ms=sa_k)
        line["forms"]["tc_over_dp4a"] = forms["tc"] / forms["dp4a"]
        line["forms"]["tc_over_int32"] = forms["tc"] / forms["int32"]
        line["forms"]["product_stage_tc_over_dp4a"] = sa_k["dp4a"] / sa_k["tc"]
        line["forms"]["product_stage_tc_over_int32"] = sa_k["int32"] / sa_k["tc"]
        # FrodoKEM-976-AES at the same batch: only A's generator differs (AES-128 T-tables in
        # shared memory instead of the SHAKE128 sponge)
        pk_a, sk_a = eng.keypair(d.FRODO976AES, kc, d.FORM_TC)
        ares = {}
        for name, f in (("tc", d.FORM_TC), ("dp4a", d.FORM_DP4A)):
            for _ in range(2):
                eng.enc(d.FRODO976AES, pk_a, ec, f, out=(ct, ss))
                eng.dec(d.FRODO976AES, ct, sk_a, f, out=ss2)
            eng.profile(True)
            eng.enc(d.FRODO976AES, pk_a, ec, f, out=(ct, ss))
            es = eng.stage_times()
            eng.dec(d.FRODO976AES, ct, sk_a, f, out=ss2)
            ds = eng.stage_times()
            eng.profile(False)
            barrier()
            reps = max(3, args.steps // 2)
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(reps):
                eng.enc(d.FRODO976AES, pk_a, ec, f, out=(ct, ss))
                eng.dec(d.FRODO976AES, ct, sk_a, f, out=ss2)
            t1.record(stream)
            barrier()
            ares[name] = world * B * reps / (t0.elapsed_time(t1) * 1e-3)
            ares[name + "_sa_kernel_ms"] = (es[1] + ds[2]) / 2
            ares[name + "_aes_blocks_per_s"] = B * 976 * 126 / ((es[1] + ds[2]) / 2 * 1e-3)
            ares[name + "_roundtrip_ok"] = bool(torch.equal(ss, ss2))
        ares["tc_over_shake_tc"] = ares["tc"] / value
        line["frodo976aes_batch8192"] = dict(ares, unit=UNIT, note="AES blocks = 976 rows x 126 (12 x 10.5 per row)")
        # The same batch under one key pair (a server decapsulating under its own key, clients
        # encapsulating to it): A expanded once and read from memory by every instance's S'A
        # stage, so that stage is the product alone in each form (the reference's own product
        # stage, DoDP4Av5s, also reads A from memory) and the ratio of its times is the
        # product-only tensor-core speed-up.
        pk1, sk1 = pk[0].contiguous(), sk[0].contiguous()
        amat = eng.expand_a(FS, pk1)
        shared = {}
        for name, f in (("tc", d.FORM_TC), ("dp4a", d.FORM_DP4A), ("int32", d.FORM_INT32)):
            for _ in range(2):
                c1, s1 = eng.enc_shared(FS, pk1, ec, f, amat)
                eng.dec_shared(FS, c1, sk1, f, amat)
            eng.profile(True)
            c1, s1 = eng.enc_shared(FS, pk1, ec, f, amat)
            es = eng.stage_times()
            s2 = eng.dec_shared(FS, c1, sk1, f, amat)
            ds = eng.stage_times()
            eng.profile(False)
            barrier()
            shared[name + "_roundtrip_ok"] = bool(torch.equal(s1, s2))
            reps = max(3, args.steps // 2)
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(reps):
                c1, s1 = eng.enc_shared(FS, pk1, ec, f, amat)
                eng.dec_shared(FS, c1, sk1, f, amat)
            t1.record(stream)
            barrier()
            shared[name] = world * B * reps / (t0.elapsed_time(t1) * 1e-3)
            shared[name + "_stage_ms"] = {"enc": es, "dec": ds}
            shared[name + "_product_ms"] = (es[1] + ds[2]) / 2
        shared["tc_over_dp4a"] = shared["tc"] / shared["dp4a"]
        shared["product_only_tc_over_dp4a"] = shared["dp4a_product_ms"] / shared["tc_product_ms"]
        shared["product_only_tc_over_int32"] = shared["int32_product_ms"] / shared["tc_product_ms"]
        shared["note"] = ("encaps to one pk and decaps with one sk, A expanded once (dpkem_frodo_expand_a); "
                          "product_ms = the S'A stage reading A from memory, per 8192-instance launch")
        line["frodo976_shared_key_batch8192"] = dict(shared, unit=UNIT)
        line["forms"]["product_only_tc_over_dp4a"] = shared["product_only_tc_over_dp4a"]

        # Saber l=3, batch 4096 (configs' second workload)
        SB = 4096
        skc = torch.empty((SB, 96), dtype=torch.uint8, device="cuda")
        sec = torch.empty((SB, 32), dtype=torch.uint8, device="cuda")
        eng.coins(SB, 96, "kp", first=first, out=skc)
        eng.coins(SB, 32, "enc", first=first, out=sec)
        spk, ssk = eng.keypair(d.SABER, skc, d.FORM_TC)
        sct = torch.empty((SB, 1088), dtype=torch.uint8, device="cuda")
        sss = torch.empty((SB, 32), dtype=torch.uint8, device="cuda")
        sss2 = torch.empty((SB, 32), dtype=torch.uint8, device="cuda")
        sres = {}
        for name, f in (("tc", d.FORM_TC), ("dp4a", d.FORM_DP4A), ("int32", d.FORM_INT32)):
            for _ in range(3):
                eng.enc(d.SABER, spk, sec, f, out=(sct, sss))
                eng.dec(d.SABER, sct, ssk, f, out=sss2)
            # stage times (enc: prologue, product, finish; dec: inner product, prologue, product, finish)
            eng.profile(True)
            eng.enc(d.SABER, spk, sec, f, out=(sct, sss))
            es = eng.stage_times()
            eng.dec(d.SABER, sct, ssk, f, out=sss2)
            ds = eng.stage_times()
            eng.profile(False)
            sres[name + "_stage_ms"] = {"enc": es, "dec": ds}
            sres[name + "_product_ms"] = es[1] + ds[0] + ds[2]
            barrier()
            reps = 50
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(reps):
                eng.enc(d.SABER, spk, sec, f, out=(sct, sss))
                eng.dec(d.SABER, sct, ssk, f, out=sss2)
            t1.record(stream)
            barrier()
            sres[name] = SB * reps / (t0.elapsed_time(t1) * 1e-3)
            sres[name + "_roundtrip_ok"] = bool(torch.equal(sss, sss2))
        sres["tc_over_dp4a"] = sres["tc"] / sres["dp4a"]
        sres["product_stage_tc_over_dp4a"] = sres["dp4a_product_ms"] / sres["tc_product_ms"]
        sres["tc_over_int32"] = sres["tc"] / sres["int32"]
        # int8 MACs of the product stages (enc 786,432 + dec 983,040 ring MACs, x 2 limbs)
        s_macs = SB * (786432 + 983040) * 2
        sres["tc_product_int8_macs_per_s"] = s_macs / (sres["tc_product_ms"] * 1e-3)
        sres["tc_product_tensor_frac"] = sres["tc_product_int8_macs_per_s"] / line["tensor"]["i8_mma_peak_macs_per_s"]
        sres["product_stage_tc_over_int32"] = sres["int32_product_ms"] / sres["tc_product_ms"]
        line["saber_l3_batch4096"] = dict(sres, unit=UNIT)
        line["single_request"] = bench_single(eng)

    # ---- mixed persistent batch: 16384 requests, 4 schemes x 3 ops, one CUDA-graph launch ----
    if not args.no_secondary:
        from dpcrypto_b200.workloads import MixedBatch

        mb = MixedBatch(eng, 16384, seed=0, first=rank * 1000000)
        mres = {"requests": mb.n, "unit": "KEM ops/s", "counts": mb.counts}
        for name, f in (("tc", d.FORM_TC), ("dp4a", d.FORM_DP4A), ("int32", d.FORM_INT32)):
            g = eng.mixed_graph(mb.items, f)
            for _ in range(2):
                g.launch()
            barrier()
            reps = 3
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(reps):
                g.launch()
            t1.record(stream)
            barrier()
            mres[name] = mb.n * reps / (t0.elapsed_time(t1) * 1e-3)
            mres[name + "_ms_per_launch"] = t0.elapsed_time(t1) / reps
            eng.sync()
            mres[name + "_bit_exact"] = mb.check()
            mb.clear()
            g.close()
        # eager launches (plan built per call): coins from HBM vs drawn inside the kernel
        host_tab = eng.requests(mb.items)  # request tables built once, outside the timing
        dev_tab = eng.requests([(sc, op, None if op != 2 else a, b, c, e) for (sc, op, a, b, c, e) in mb.items])
        key = bytes(range(32))
        for name, its, kw in (("tc_eager", host_tab, {}), ("tc_eager_device_coins", dev_tab,
                                                           {"coin_key": key, "coin_first": 0})):
            for _ in range(2):
                eng.mixed(its, d.FORM_TC, **kw)
            barrier()
            reps = 3
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(reps):
                eng.mixed(its, d.FORM_TC, **kw)
            t1.record(stream)
            barrier()
            eng.sync()
            mres[name] = mb.n * reps / (t0.elapsed_time(t1) * 1e-3)
        mb.clear()  # the device-coin run wrote other keys: rerun with host coins and check
        eng.mixed(mb.items, d.FORM_TC)
        eng.sync()
        mres["tc_eager_bit_exact"] = mb.check()
        mb.clear()
        mres["eager_note"] = ("one dpkem_mixed_batch call per launch: host plan build (list scheduling of "
                              "the task graph) + upload + launch, vs the graph's replay")
        mres["device_coins_note"] = "keypair/encaps coins drawn in the persistent kernel (no coin reads from HBM)"
        line["mixed_16384"] = mres

    # ---- serving loop: Poisson arrivals, 60 % encaps / 40 % decaps, 50/50 Frodo / Saber l=3 ----
    if not args.no_secondary and world == 1:
        from dpcrypto_b200.serving import FRODO_CLASS, SABER_CLASS, RequestPool, Server, poisson_arrivals

        pool = RequestPool(eng, 16384, seed=0)
        serving = {"requests_per_level": pool.n, "mix": "60% encaps / 40% decaps, 50/50 FrodoKEM-976 / Saber l=3",
                   "slots": 4, "max_batch": 4096, "unit": "KEM ops/s",
                   "modes": {"shared": "every slot takes any request",
                             "split": "2 slots for Frodo requests, 2 for Saber requests"}}
        for name, f in (("tc", d.FORM_TC), ("dp4a", d.FORM_DP4A)):
            for mode, classes in (("shared", None), ("split", [FRODO_CLASS, FRODO_CLASS, SABER_CLASS, SABER_CLASS])):
                srv = Server(slots=4, max_batch=4096, form=f, classes=classes)
                try:
                    srv.run(pool, np.zeros(2048))  # warm-up
                    peaks = []
                    for _ in range(2):  # best of two saturated runs: one host or device hiccup
                        pool.clear()    # would otherwise scale every load level down
                        peaks.append(srv.run(pool, np.zeros(pool.n))["ops_per_s"])
                    peak = max(peaks)
                    levels = []
                    for frac in (0.1, 0.25, 0.5, 0.75, 1.0):
                        pool.clear()
                        r = srv.run(pool, poisson_arrivals(pool.n, rate=frac * peak, seed=int(frac * 100)))
                        levels.append({"load": frac, "offered_per_s": frac * peak, "ops_per_s": r["ops_per_s"],
                                       "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "mean_batch": r["mean_batch"],
                                       "frodo_p50_ms": r["frodo_p50_ms"], "frodo_p99_ms": r["frodo_p99_ms"],
                                       "saber_p50_ms": r["saber_p50_ms"], "saber_p99_ms": r["saber_p99_ms"],
                                       "host_max_gap_ms": r["host_max_gap_ms"], "submit_ms_max": r["submit_ms_max"]})
                    torch.cuda.synchronize()
                    key = name if mode == "shared" else f"{name}_split"
                    serving[key] = {"peak_ops_per_s": peak, "levels": levels, "bit_exact": pool.check()}
                finally:
                    srv.close()
        # admission inside the running kernel: one long-lived service launch, each request
        # submitted as it arrives (no host batching window), 16 CTAs for Saber work only
        from dpcrypto_b200.serving import ServiceServer

        serving["service"] = {"note": "dpkem_service_*: requests admitted by the running persistent kernel into "
                                      "per-stage ready queues; 16 of its CTAs take only Saber work"}
        for name, f in (("tc", d.FORM_TC), ("dp4a", d.FORM_DP4A)):
            srv = ServiceServer(form=f, saber_ctas=16)
            try:
                srv.run(pool, np.zeros(2048))  # warm-up
                peak = max(srv.run(pool, np.zeros(pool.n))["ops_per_s"] for _ in range(2))
                levels = []
                for frac in (0.1, 0.25, 0.5, 0.75, 1.0):
                    if frac == 1.0:
                        pool.clear()  # the last level's outputs are checked against the batched calls
                    r = srv.run(pool, poisson_arrivals(pool.n, rate=frac * peak, seed=int(frac * 100) + 7))
                    levels.append({"load": frac, "offered_per_s": frac * peak, "ops_per_s": r["ops_per_s"],
                                   "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "frodo_p50_ms": r["frodo_p50_ms"],
                                   "frodo_p99_ms": r["frodo_p99_ms"], "saber_p50_ms": r["saber_p50_ms"],
                                   "saber_p99_ms": r["saber_p99_ms"], "mean_submit": r["mean_submit"]})
                torch.cuda.synchronize()
                serving["service"][name] = {"peak_ops_per_s": peak, "levels": levels, "bit_exact": pool.check()}
            finally:
                srv.close()
        line["serving"] = serving

    # ---- wire format: 16384 mixed request frames from pinned host memory, then the same
    #      frames through the shared-memory ring with the frame server in its own process ----
    if not args.no_secondary and world == 1:
        line["frames_16384"] = bench_frames(eng, form)

    # ---- CPU baseline: the oracle on the host cores, rank 0 at N=1 ----
    if world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        O.use_native()
        threads = os.cpu_count() or 1
        n_inst = 64 * threads
        cv, dt = cpu_sample(n_inst, threads)
        cv1, dt1 = cpu_sample(32, 1)
        sv, sdt = cpu_sample_saber(4096 * max(1, threads // 4), threads)
        sv1, sdt1 = cpu_sample_saber(1024, 1)
        line["cpu_baseline"] = {"value": cv, "unit": UNIT, "cores": threads, "kind": "port",
                                "value_1core": cv1, "sample_1core": f"32 instances on 1 thread, {dt1:.2f} s wall",
                                "saber_l3_value": sv, "saber_l3_sample": f"Saber l=3 encaps+decaps on {threads} threads, "
                                                                        f"{sdt:.2f} s wall",
                                "saber_l3_value_1core": sv1, "saber_l3_sample_1core": f"1024 on 1 thread, {sdt1:.2f} s wall",
                                "sample": f"{n_inst} FrodoKEM-976 encaps+decaps (64 per host thread), "
                                          f"{CPU_BUILD}, {dt:.1f} s wall",
                                "note": "reported baseline, not the target"}

    peaks, src = measured_peaks()
    line["peaks_file"] = src
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    eng.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
