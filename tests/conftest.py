import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def engine():
    from dpcrypto_b200 import Engine, build

    build.build()
    eng = Engine(0)
    yield eng
    eng.close()


@pytest.fixture(scope="session")
def saber_tv():
    import numpy as np

    return dict(np.load(os.path.join(ROOT, "tests", "golden", "saber_l3_tv.npz")))


@pytest.fixture(scope="session")
def oracle_check_items(oracle):
    """Checker for mixed-request tests: every `stride`-th request (scheme, op, in0, in1,
    out0, out1), as the mixed entry points take them, recomputed by the CPU oracle from its
    inputs and compared with the outputs the GPU wrote.  Returns the number checked."""
    import numpy as np

    def host(t):
        return t.detach().cpu().numpy().reshape(1, -1)

    def check(items, stride, offset=0):
        groups = {}
        for i in range(offset, len(items), stride):
            scheme, op = items[i][0], items[i][1]
            groups.setdefault((scheme, op), []).append(items[i])
        checked = 0
        for (scheme, op), rows in groups.items():
            a = np.concatenate([host(r[2]) for r in rows])
            if op == 0:
                pk, sk = oracle.keypair(scheme, a, threads=8)
                got = [(host(r[4]), host(r[5])) for r in rows]
                want = list(zip(pk, sk))
            elif op == 1:
                pk = np.concatenate([host(r[3]) for r in rows])
                ct, ss = oracle.enc(scheme, pk, a, threads=8)
                got = [(host(r[4]), host(r[5])) for r in rows]
                want = list(zip(ct, ss))
            else:
                sk = np.concatenate([host(r[3]) for r in rows])
                ss = oracle.dec(scheme, a, sk, threads=8)
                got = [(host(r[4]),) for r in rows]
                want = [(s,) for s in ss]
            for j, (g, w) in enumerate(zip(got, want)):
                for gi, wi in zip(g, w):
                    assert (gi.ravel() == wi.ravel()).all(), (scheme, op, j)
            checked += len(rows)
        return checked

    return check
