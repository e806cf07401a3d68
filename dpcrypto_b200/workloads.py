"""Seeded synthetic workloads shared by bench.py and the serving loop.

All randomness is the device coin stream SHAKE256(00..1F || LE64(i) || tag) (dpkem_coins),
so every run builds the same keys, ciphertexts and request order.
"""
from __future__ import annotations

import numpy as np
import torch

from . import kem as K

MIX_SCHEMES = (K.FRODO976, K.LIGHTSABER, K.SABER, K.FIRESABER)


class MixedBatch:
    """n requests drawn uniformly from 4 schemes x {keypair, encaps, decaps}, shuffled with a
    fixed seed; inputs prepared with the batched entry points (untimed); `expected` holds the
    batched results so a mixed run can be checked byte for byte."""

    def __init__(self, eng: K.Engine, n: int, seed: int = 0, first: int = 0):
        rng = np.random.default_rng(seed)
        kinds = rng.integers(0, 12, size=n)  # scheme index * 3 + op
        self.items, self.outputs, self.expected = [], [], []
        per = {k: np.nonzero(kinds == k)[0] for k in range(12)}
        slots = [None] * n
        for si, scheme in enumerate(MIX_SCHEMES):
            z = K.sizes(scheme)
            n_kp, n_enc, n_dec = (len(per[si * 3 + op]) for op in range(3))
            m = max(n_enc, n_dec)
            kc = torch.empty((n_kp + m, z["kp_coins"]), dtype=torch.uint8, device="cuda")
            ec = torch.empty((max(1, m), z["enc_coins"]), dtype=torch.uint8, device="cuda")
            eng.coins(n_kp + m, z["kp_coins"], "mix-kp", first=first + 100000 * si, out=kc)
            eng.coins(max(1, m), z["enc_coins"], "mix-enc", first=first + 100000 * si, out=ec)
            pk, sk = eng.keypair(scheme, kc, K.FORM_TC)
            ct, ss = eng.enc(scheme, pk[n_kp:n_kp + max(1, m)], ec, K.FORM_TC) if m else (None, None)
            torch.cuda.synchronize()
            # outputs
            opk = torch.empty((max(1, n_kp), z["pk"]), dtype=torch.uint8, device="cuda")
            osk = torch.empty((max(1, n_kp), z["sk"]), dtype=torch.uint8, device="cuda")
            oct_ = torch.empty((max(1, n_enc), z["ct"]), dtype=torch.uint8, device="cuda")
            oss = torch.empty((max(1, n_enc), z["ss"]), dtype=torch.uint8, device="cuda")
            dss = torch.empty((max(1, n_dec), z["ss"]), dtype=torch.uint8, device="cuda")
            self.outputs += [opk, osk, oct_, oss, dss]
            for j, r in enumerate(per[si * 3]):
                slots[r] = (scheme, 0, kc[j], None, opk[j], osk[j])
            for j, r in enumerate(per[si * 3 + 1]):
                slots[r] = (scheme, 1, ec[j], pk[n_kp + j], oct_[j], oss[j])
            for j, r in enumerate(per[si * 3 + 2]):
                slots[r] = (scheme, 2, ct[j], sk[n_kp + j], dss[j], None)
            self.expected += [(opk[:n_kp], pk[:n_kp]), (osk[:n_kp], sk[:n_kp]), (oct_[:n_enc], ct[:n_enc]),
                              (oss[:n_enc], ss[:n_enc]), (dss[:n_dec], ss[:n_dec])]
        self.items = slots
        self.n = n
        self.counts = {f"{s}/{op}": int((kinds == i * 3 + op).sum()) for i, s in enumerate(MIX_SCHEMES)
                       for op in range(3)}

    def clear(self):
        for t in self.outputs:
            t.zero_()

    def check(self) -> bool:
        return all(torch.equal(got, ref) for got, ref in self.expected)


def mixed_frames(eng: K.Engine, n: int, seed: int = 0, first: int = 0) -> np.ndarray:
    """n request frames (include/dpkem_wire.h), kinds uniform over the 4 schemes x 3 ops
    and shuffled; id = position.  Keys and ciphertexts come from the batched calls."""
    from . import frames as F

    rng = np.random.default_rng(seed)
    kinds = rng.integers(0, 12, size=n)
    rows = [None] * n
    for si, scheme in enumerate(MIX_SCHEMES):
        z = K.sizes(scheme)
        idx = [np.nonzero(kinds == si * 3 + op)[0] for op in range(3)]
        m = max(1, len(idx[1]), len(idx[2]))
        kc = eng.coins(len(idx[0]) + m, z["kp_coins"], "frm-kp", first=first + 100000 * si)
        ec = eng.coins(m, z["enc_coins"], "frm-enc", first=first + 100000 * si)
        pk, sk = eng.keypair(scheme, kc[len(idx[0]):], K.FORM_TC)
        ct, _ = eng.enc(scheme, pk, ec, K.FORM_TC)
        blocks = [F.encode(scheme, 0, idx[0], coins=kc[:len(idx[0])]),
                  F.encode(scheme, 1, idx[1], coins=ec[:len(idx[1])], pk=pk[:len(idx[1])]),
                  F.encode(scheme, 2, idx[2], ct=ct[:len(idx[2])], sk=sk[:len(idx[2])])]
        for op in range(3):
            size = F.frame_bytes(scheme, op)[0]
            b = blocks[op].reshape(-1, size)
            for j, r in enumerate(idx[op]):
                rows[r] = b[j]
    return np.concatenate(rows)
