"""Frame server: answers request frames that another process writes into a shared ring.

    python -m dpcrypto_b200.frame_server --ring /dev/shm/dpkem.ring [--create CAPACITY]
        [--form tc|dp4a|int32] [--device 0] [--max-frames 4096] [--budget-gib 8]

The ring (include/dpkem_wire.h) is page-locked once with dpkem_host_register, so each
batch is copied between the ring and the GPU by DMA straight from and into the shared
pages.  The loop itself is the library's dpkem_ring_serve, called without holding the
GIL: it takes contiguous request frames and response room at its own cursors, runs up to
--inflight batches at once (one dpkem context each, so one batch's copies overlap
another's kernels) and publishes the responses in request order.
It returns, and the process exits 0, when a client sets the ring's stop word.
"""
from __future__ import annotations

import argparse
import ctypes
import sys

from . import frames as F
from . import kem as K

FORMS = {"tc": K.FORM_TC, "dp4a": K.FORM_DP4A, "int32": K.FORM_INT32}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--ring", required=True)
    ap.add_argument("--create", type=int, default=None, help="create the ring with this capacity (bytes)")
    ap.add_argument("--form", default="tc", choices=sorted(FORMS))
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--max-frames", type=int, default=4096)
    ap.add_argument("--budget-gib", type=float, default=8.0)
    ap.add_argument("--idle-us", type=int, default=50)
    ap.add_argument("--inflight", type=int, default=2, help="batches in flight (one context each)")
    a = ap.parse_args(argv)

    ring = F.Ring(a.ring, a.create)
    engines = [K.Engine(a.device, hbm_budget=int(a.budget_gib * (1 << 30) / a.inflight)) for _ in range(a.inflight)]
    handles = (ctypes.c_void_p * len(engines))(*[e._h for e in engines])
    lib = K.load()
    # size the arenas for a full batch of the largest frames now (Frodo decaps requests,
    # Frodo keypair responses, Frodo records): growing one later waits for the whole GPU
    worst = int(lib.dpkem_mixed_bytes(K.FRODO976, a.max_frames)) + a.max_frames * (
        F.frame_bytes(K.FRODO976, 2)[0] + F.frame_bytes(K.FRODO976, 0)[1])
    for e in engines:
        e.reserve(min(worst, int(a.budget_gib * (1 << 30) / a.inflight)))
    rc = lib.dpkem_host_register(ring.base, ring.size)
    if rc != K.OK:
        print(f"frame_server: host_register failed: {lib.dpkem_strerror(rc).decode()}", file=sys.stderr)
        return 1
    try:
        rc = lib.dpkem_ring_serve(handles, len(engines), FORMS[a.form], ring.base, a.max_frames, a.idle_us)
    finally:
        lib.dpkem_host_unregister(ring.base)
        for e in engines:
            e.close()
    if rc != K.OK:
        print(f"frame_server: {lib.dpkem_strerror(rc).decode()}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
