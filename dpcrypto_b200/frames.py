"""Wire-format frames and the shared-memory ring (include/dpkem_wire.h), from Python.

Frames: a 32-byte header (magic "DPKF", version, scheme, op, status, id, frame_bytes) and
the payload sections of the batched API in argument order, each 16-byte aligned, the
frame padded to 32 bytes.  `encode` builds a block of same-kind request frames with numpy;
`decode` splits a response block back into arrays.

Ring: a file (normally under /dev/shm) mapped by a client process and by the frame
server (python -m dpcrypto_b200.frame_server).  All counter handling is done by the
library's dpkem_ring_* functions (release/acquire atomics), so the client side needs no
GPU: push request frames, pop response frames.
"""
from __future__ import annotations

import ctypes
import mmap
import os

import numpy as np

from . import kem as K

OP_KEYPAIR, OP_ENC, OP_DEC = 0, 1, 2
HEADER = 32
MAGIC, PAD = 0x464B5044, 0x504B5044
HDR_DTYPE = np.dtype([("magic", "<u4"), ("version", "u1"), ("scheme", "u1"), ("op", "u1"), ("status", "i1"),
                      ("id", "<u8"), ("frame_bytes", "<u4"), ("reserved", "<u4", (3,))])
assert HDR_DTYPE.itemsize == HEADER


def frame_bytes(scheme: int, op: int) -> tuple:
    """(request frame bytes, response frame bytes) of (scheme, op)."""
    rq, rs = ctypes.c_size_t(), ctypes.c_size_t()
    rc = K.load().dpkem_frame_bytes(scheme, op, ctypes.byref(rq), ctypes.byref(rs))
    if rc != K.OK:
        raise K.DpkemError(rc, f"frame_bytes({scheme}, {op})")
    return rq.value, rs.value


def _pad16(x: int) -> int:
    return (x + 15) & ~15


def sections(scheme: int, op: int, response: bool) -> list:
    """[(name, offset, length)] of the payload sections of one frame."""
    z = K.sizes(scheme)
    if not response:
        if op == OP_KEYPAIR:
            return [("coins", HEADER, z["kp_coins"])]
        if op == OP_ENC:
            return [("coins", HEADER, z["enc_coins"]), ("pk", HEADER + _pad16(z["enc_coins"]), z["pk"])]
        return [("ct", HEADER, z["ct"]), ("sk", HEADER + z["ct"], z["sk"])]
    if op == OP_KEYPAIR:
        return [("pk", HEADER, z["pk"]), ("sk", HEADER + z["pk"], z["sk"])]
    if op == OP_ENC:
        return [("ct", HEADER, z["ct"]), ("ss", HEADER + z["ct"], z["ss"])]
    return [("ss", HEADER, z["ss"])]


def encode(scheme: int, op: int, ids, **payload) -> np.ndarray:
    """Block of len(ids) request frames of one kind; payload arrays are (n, size) uint8,
    named as in `sections` (coins / pk for encaps, ct / sk for decaps, coins for keypair)."""
    ids = np.asarray(ids, dtype=np.uint64)
    n = len(ids)
    size, _ = frame_bytes(scheme, op)
    out = np.zeros((n, size), np.uint8)
    hdr = out[:, :HEADER].copy().view(HDR_DTYPE).reshape(n)
    hdr["magic"], hdr["version"], hdr["scheme"], hdr["op"] = MAGIC, 1, scheme, op
    hdr["id"], hdr["frame_bytes"] = ids, size
    out[:, :HEADER] = hdr.view(np.uint8).reshape(n, HEADER)
    for name, off, length in sections(scheme, op, response=False):
        a = np.asarray(payload[name], np.uint8).reshape(n, length)
        out[:, off:off + length] = a
    return out.reshape(-1)


def pad_frame(nbytes: int) -> np.ndarray:
    """A filler frame of nbytes (a multiple of 32) that readers skip."""
    f = np.zeros(nbytes, np.uint8)
    h = f[:HEADER].view(HDR_DTYPE)
    h["magic"], h["version"], h["frame_bytes"] = PAD, 1, nbytes
    return f


def headers(block: np.ndarray) -> np.ndarray:
    """Headers of every frame in a block (PAD frames included), in order."""
    block = np.asarray(block, np.uint8).reshape(-1)
    out, pos = [], 0
    while pos < len(block):
        h = block[pos:pos + HEADER].copy().view(HDR_DTYPE)[0]
        out.append(h)
        pos += int(h["frame_bytes"])
        if int(h["frame_bytes"]) == 0:
            raise ValueError("frame of 0 bytes")
    return np.array(out, dtype=HDR_DTYPE)


def decode(block: np.ndarray, scheme: int, op: int) -> dict:
    """Split a block of same-kind response frames into {'id', 'status', <section>: (n, size)}."""
    _, size = frame_bytes(scheme, op)
    block = np.asarray(block, np.uint8).reshape(-1)
    if len(block) % size:
        raise ValueError("block is not a whole number of frames of this kind")
    rows = block.reshape(-1, size)
    hdr = rows[:, :HEADER].copy().view(HDR_DTYPE).reshape(-1)
    if not ((hdr["magic"] == MAGIC) & (hdr["scheme"] == scheme) & (hdr["op"] == op)).all():
        raise ValueError("unexpected frame header")
    out = {"id": hdr["id"].copy(), "status": hdr["status"].copy()}
    for name, off, length in sections(scheme, op, response=True):
        out[name] = rows[:, off:off + length]
    return out


def scan(block: np.ndarray, max_frames: int = 0) -> tuple:
    """(frames, used bytes, response bytes) of a request block (library check)."""
    block = np.ascontiguousarray(block, np.uint8)
    n, used, rb = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
    rc = K.load().dpkem_frames_scan(block.ctypes.data, block.nbytes, max_frames, ctypes.byref(n),
                                    ctypes.byref(used), ctypes.byref(rb))
    if rc != K.OK:
        raise K.DpkemError(rc, "frames_scan")
    return n.value, used.value, rb.value


def run(eng: K.Engine, block: np.ndarray, form: int = K.FORM_TC, out: np.ndarray | None = None) -> np.ndarray:
    """Answer a block of request frames on the engine's GPU (dpkem_frames_run)."""
    block = np.ascontiguousarray(block, np.uint8)
    _, _, rb = scan(block)
    if out is None:
        out = np.empty(rb, np.uint8)
    wrote = ctypes.c_size_t()
    rc = K.load().dpkem_frames_run(eng._h, form, block.ctypes.data, block.nbytes, out.ctypes.data, out.nbytes,
                                   ctypes.byref(wrote))
    if rc != K.OK:
        raise K.DpkemError(rc, "frames_run")
    return out[:wrote.value]


class Ring:
    """A request/response ring in a shared file mapping (see include/dpkem_wire.h)."""

    CONTROL = 4096
    _OFF = {"req_tail": 64, "req_head": 128, "resp_tail": 192, "resp_head": 256, "stop": 320, "served": 384}

    def __init__(self, path: str, capacity: int | None = None):
        lib = K.load()
        self.path = path
        if capacity is not None:
            size = lib.dpkem_ring_bytes(capacity)
            fd = os.open(path, os.O_CREAT | os.O_RDWR | os.O_TRUNC, 0o600)
            os.ftruncate(fd, size)
        else:
            fd = os.open(path, os.O_RDWR)
            size = os.fstat(fd).st_size
        self._mm = mmap.mmap(fd, size)
        os.close(fd)
        self._buf = np.frombuffer(self._mm, np.uint8)
        self.base = self._buf.ctypes.data
        self.size = size
        if capacity is not None:
            rc = lib.dpkem_ring_init(self.base, capacity)
            if rc != K.OK:
                raise K.DpkemError(rc, "ring_init")
        self.capacity = int(self._buf[8:16].view("<u8")[0])

    def counter(self, name: str) -> int:
        o = self._OFF[name]
        return int(self._buf[o:o + 8].view("<u8")[0])

    def push(self, block: np.ndarray) -> int:
        """Append the longest prefix of whole request frames that fits; bytes taken (0: no room yet)."""
        block = np.ascontiguousarray(block, np.uint8)
        got = ctypes.c_size_t()
        rc = K.load().dpkem_ring_push(self.base, block.ctypes.data, block.nbytes, ctypes.byref(got))
        if rc == K.EAGAIN:
            return 0
        if rc != K.OK:
            raise K.DpkemError(rc, "ring_push")
        return got.value

    def pop(self, cap: int = 64 << 20, out: np.ndarray | None = None) -> tuple:
        """Take the response frames available now: (bytes as a view of `out`, frame count)."""
        if out is None:
            out = np.empty(cap, np.uint8)
        got, n = ctypes.c_size_t(), ctypes.c_size_t()
        rc = K.load().dpkem_ring_pop(self.base, out.ctypes.data, out.nbytes, ctypes.byref(got), ctypes.byref(n))
        if rc != K.OK:
            raise K.DpkemError(rc, "ring_pop")
        return out[:got.value], n.value

    def acquire(self, max_frames: int = 0):
        """Server side by hand: None, or dict of the offsets dpkem_ring_acquire returns."""
        v = [ctypes.c_size_t() for _ in range(7)]
        rc = K.load().dpkem_ring_acquire(self.base, max_frames, *[ctypes.byref(x) for x in v])
        if rc == K.EAGAIN:
            return None
        if rc != K.OK:
            raise K.DpkemError(rc, "ring_acquire")
        keys = ("req_off", "req_bytes", "req_advance", "resp_off", "resp_bytes", "resp_advance", "n_frames")
        return dict(zip(keys, (x.value for x in v)))

    def release(self, a: dict):
        rc = K.load().dpkem_ring_release(self.base, a["req_advance"], a["resp_advance"], a["n_frames"])
        if rc != K.OK:
            raise K.DpkemError(rc, "ring_release")

    def request_view(self, off: int, n: int) -> np.ndarray:
        return self._buf[self.CONTROL + off:self.CONTROL + off + n]

    def response_view(self, off: int, n: int) -> np.ndarray:
        o = self.CONTROL + self.capacity + off
        return self._buf[o:o + n]

    def stop(self):
        o = self._OFF["stop"]
        self._buf[o:o + 8].view("<u8")[0] = 1

    def close(self):
        self._buf = None
        self._mm.close()
