"""Autotuner: pick the build- and run-time knobs of libdpkem.so on the GPU at hand.

Knobs:
  keccak_unroll      rounds per iteration of the Keccak-f[1600] round loop (compile time)
  thread_block       block size of the latency-bound thread-per-instance kernels
  mixed_frodo_task   instances per Frodo thread-level task in the persistent mixed kernel
  mixed_pair_task    instances per two-role prologue task (two threads per instance)
  mixed_thread_task  instances per other thread-level task
  pipe_chunks        chunks (one stream each) of a pipelined host-buffer batch
  pipe_priority      chunk streams with descending priorities (earlier chunks finish first)
  saber_pair_max     Keccak lanes per state in the Saber prologue: batches of up to this many
                     instances run GenMatrix on lane pairs (shorter chain while SM
                     sub-partitions idle), larger ones on one lane (fewer issue slots per
                     state); the sweep times both at 2k-16k instances and keeps the crossover
Not knobs, with the measured reason recorded in the output: the MMA tile shape (the int8
MMAs are <1 % of the tensor pipe: M = 128 is the smallest tile that keeps one TMEM lane per
output row) and Keccak lanes per state in the throughput-bound kernels (the fused S'A
stages and the persistent mixed kernel keep one state per thread: a pair costs more issue
slots per state on an integer pipe those kernels already saturate).

    python -m dpcrypto_b200.autotune --build          # build variants (CPU, nvcc)
    python -m dpcrypto_b200.autotune --measure        # on a B200: sweep, write tuning.json

Each variant library is measured in its own process (DPKEM_LIB points kem.py at it).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
VARIANTS = os.path.join(HERE, "_build", "variants")
OUT = os.path.join(HERE, "tuning.json")
UNROLLS = (1, 2, 3, 4)


def variant_lib(u: int) -> str:
    return os.path.join(VARIANTS, f"unroll{u}", "libdpkem.so")


def build_variants() -> None:
    sys.path.insert(0, ROOT)
    from dpcrypto_b200 import build as b

    for u in UNROLLS:
        t = time.time()
        b.build(out=variant_lib(u), defines=[f"-DDPKEM_KECCAK_UNROLL={u}"])
        print(f"built unroll={u} in {time.time() - t:.0f} s", flush=True)


# ---------------------------------------------------------------- child: measure one library
def _child(u: int) -> dict:
    import numpy as np
    import torch

    sys.path.insert(0, ROOT)
    import dpcrypto_b200 as d
    from dpcrypto_b200 import kem
    from dpcrypto_b200.workloads import MixedBatch

    res = {"keccak_unroll": u}
    eng = d.Engine(0)
    res["int_ops_per_s"], res["keccak_per_s"] = eng.probe_int_peaks()

    pk = sk = ec = None

    def frodo_time(B: int, reps: int = 3):
        nonlocal pk, sk, ec
        kc = torch.empty((B, 64), dtype=torch.uint8, device="cuda")
        ec = torch.empty((B, 24), dtype=torch.uint8, device="cuda")
        eng.coins(B, 64, "tune-kp", out=kc)
        eng.coins(B, 24, "tune-enc", out=ec)
        pk, sk = eng.keypair(d.FRODO976, kc, d.FORM_TC)
        ct = torch.empty((B, 15744), dtype=torch.uint8, device="cuda")
        ss = torch.empty((B, 24), dtype=torch.uint8, device="cuda")
        for _ in range(2):
            eng.enc(d.FRODO976, pk, ec, d.FORM_TC, out=(ct, ss))
            eng.dec(d.FRODO976, ct, sk, d.FORM_TC)
        torch.cuda.synchronize()
        eng.profile(True)
        stages = []
        t0 = time.perf_counter()
        for _ in range(reps):
            eng.enc(d.FRODO976, pk, ec, d.FORM_TC, out=(ct, ss))
            e = eng.stage_times()
            eng.dec(d.FRODO976, ct, sk, d.FORM_TC)
            stages.append((e, eng.stage_times()))
        torch.cuda.synchronize()
        eng.profile(False)
        wall = (time.perf_counter() - t0) / reps
        dev = float(np.mean([sum(e) + sum(x) for e, x in stages]))
        thread_ms = float(np.mean([e[0] + e[2] + x[1] + x[3] for e, x in stages]))
        return wall, dev, thread_ms

    B = 4096
    res["frodo_b4096_ms"] = frodo_time(B)[1]
    sweep = {}
    for tb in (32, 64, 128):
        kem.set_tuning("thread_block", tb)
        sweep[tb] = frodo_time(B, reps=2)[2]
    res["thread_block_ms"] = sweep
    kem.set_tuning("thread_block", min(sweep, key=sweep.get))
    # mixed batch task sizes
    mb = MixedBatch(eng, 4096, seed=7)
    msweep = {}
    for ft, stt, tt in ((256, 128, 256), (128, 128, 256), (64, 64, 128), (32, 32, 64)):
        kem.set_tuning("mixed_frodo_task", ft)
        kem.set_tuning("mixed_pair_task", stt)
        kem.set_tuning("mixed_thread_task", tt)
        eng.mixed(mb.items, d.FORM_TC)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(2):
            eng.mixed(mb.items, d.FORM_TC)
        torch.cuda.synchronize()
        msweep[f"{ft}/{stt}/{tt}"] = (time.perf_counter() - t0) / 2 * 1e3
        eng.sync()
        ok = mb.check()
        mb.clear()
        if not ok:
            raise RuntimeError("mixed batch mismatch while tuning")
    res["mixed_task_ms"] = msweep
    # host-buffer pipeline depth, measured end to end (pinned buffers, copies included) at the
    # batch of the headline workload (8,192): the best depth depends on the batch
    B = 8192
    frodo_time(B, reps=1)  # keys and coins for this batch
    h_pk, h_sk = pk.cpu().pin_memory().numpy(), sk.cpu().pin_memory().numpy()
    h_ec = ec.cpu().pin_memory().numpy()
    h_ct = torch.empty((B, 15744), dtype=torch.uint8).pin_memory().numpy()
    h_ss = torch.empty((B, 24), dtype=torch.uint8).pin_memory().numpy()
    h_ss2 = torch.empty((B, 24), dtype=torch.uint8).pin_memory().numpy()  # pinned: pageable copies serialise
    psweep = {}
    for prio in (0, 1):
        kem.set_tuning("pipe_priority", prio)
        for pc in (2, 4, 6, 8):
            kem.set_tuning("pipe_chunks", pc)
            eng.enc(d.FRODO976, h_pk, h_ec, d.FORM_TC, out=(h_ct, h_ss))
            t0 = time.perf_counter()
            for _ in range(3):
                eng.enc(d.FRODO976, h_pk, h_ec, d.FORM_TC, out=(h_ct, h_ss))
                eng.dec(d.FRODO976, h_ct, h_sk, d.FORM_TC, out=h_ss2)
            psweep[f"{pc}/{prio}"] = (time.perf_counter() - t0) / 3 * 1e3
    res["pipe_chunks_priority_ms"] = psweep
    # Keccak lanes per state in the Saber l=3 prologue, by batch size: encaps + decaps, device buffers
    def saber_time(n: int) -> float:
        kc = torch.empty((n, 96), dtype=torch.uint8, device="cuda")
        sc = torch.empty((n, 32), dtype=torch.uint8, device="cuda")
        eng.coins(n, 96, "tune-kp", out=kc)
        eng.coins(n, 32, "tune-enc", out=sc)
        spk, ssk = eng.keypair(d.SABER, kc, d.FORM_TC)
        sct = torch.empty((n, 1088), dtype=torch.uint8, device="cuda")
        sss = torch.empty((n, 32), dtype=torch.uint8, device="cuda")
        for _ in range(2):
            eng.enc(d.SABER, spk, sc, d.FORM_TC, out=(sct, sss))
            eng.dec(d.SABER, sct, ssk, d.FORM_TC)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(10):
            eng.enc(d.SABER, spk, sc, d.FORM_TC, out=(sct, sss))
            eng.dec(d.SABER, sct, ssk, d.FORM_TC)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / 10 * 1e3

    lsweep = {}
    for n in (2048, 4096, 8192, 16384):
        for name, val in (("one", 0), ("pair", 1 << 30)):
            kem.set_tuning("saber_pair_max", val)
            lsweep[f"{n}/{name}"] = saber_time(n)
    res["saber_lanes_ms"] = lsweep
    return res


def measure() -> dict:
    results = []
    for u in UNROLLS:
        lib = variant_lib(u)
        if not os.path.exists(lib):
            print(f"missing {lib}; run --build first", file=sys.stderr)
            continue
        env = dict(os.environ, DPKEM_LIB=lib)
        r = subprocess.run([sys.executable, "-m", "dpcrypto_b200.autotune", "--child", str(u)], cwd=ROOT, env=env,
                           capture_output=True, text=True, timeout=900)
        if r.returncode != 0:
            raise RuntimeError(f"variant {u} failed:\n{r.stdout}\n{r.stderr}")
        results.append(json.loads(r.stdout.strip().splitlines()[-1]))
        print(json.dumps(results[-1]), flush=True)
    best = min(results, key=lambda x: x["frodo_b4096_ms"])
    tb = min(best["thread_block_ms"], key=lambda k: best["thread_block_ms"][k])
    mk = min(best["mixed_task_ms"], key=best["mixed_task_ms"].get)
    pc, prio = (int(x) for x in min(best["pipe_chunks_priority_ms"], key=best["pipe_chunks_priority_ms"].get).split("/"))
    ft, stt, tt = (int(x) for x in mk.split("/"))
    ls = best["saber_lanes_ms"]
    pair_max = max([int(k.split("/")[0]) for k in ls if k.endswith("/pair") and ls[k] < ls[k.replace("/pair", "/one")]],
                   default=0)
    import torch

    out = {
        "device": torch.cuda.get_device_name(0),
        "chosen": {"keccak_unroll": best["keccak_unroll"], "thread_block": int(tb), "mixed_frodo_task": ft,
                   "mixed_pair_task": stt, "mixed_thread_task": tt, "pipe_chunks": pc,
                   "pipe_priority": prio, "saber_pair_max": pair_max},
        "fixed": {"mma_tile": "M=128 (N=8 Frodo, N=8/16 Saber), K=32: int8 MMA <1% of the tensor pipe",
                  "keccak_lanes_per_state_throughput_kernels": 1},
        "measurements": results,
        "command": "python -m dpcrypto_b200.autotune --measure",
        "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
    }
    if os.path.exists(OUT):  # keep the end-to-end sweeps recorded beside earlier runs
        with open(OUT) as f:
            extra = json.load(f).get("measurements_extra")
        if extra:
            out["measurements_extra"] = extra
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--build", action="store_true")
    ap.add_argument("--measure", action="store_true")
    ap.add_argument("--child", type=int)
    a = ap.parse_args()
    if a.child is not None:
        print(json.dumps(_child(a.child)))
        return
    if a.build:
        build_variants()
    if a.measure:
        print(json.dumps(measure()["chosen"]))


if __name__ == "__main__":
    main()
