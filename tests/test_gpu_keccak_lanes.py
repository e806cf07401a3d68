"""Keccak-f[1600] in every lanes-per-state layout the sponge stages use (one thread, a
bit-interleaved lane pair, five lanes of a warp, a warp per state) against the CPU oracle's permutation, on
random and edge states, with batch sizes that leave partial warps and partial groups."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lanes", [1, 2, 5, 25])
@pytest.mark.parametrize("n,perms", [(1, 1), (7, 1), (33, 3), (601, 2)])
def test_keccak_lanes_match_oracle(engine, oracle, lanes, n, perms):
    rng = np.random.default_rng(n * 10 + lanes)
    states = rng.integers(0, 2**63, size=(n, 25), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=(n, 25), dtype=np.uint64)
    states[0] = 0
    if n > 1:
        states[1] = np.uint64(0xFFFFFFFFFFFFFFFF)
    want = states.copy()
    lib = oracle.lib()
    for s in range(n):
        row = np.ascontiguousarray(want[s])
        for _ in range(perms):
            lib.oracle_keccak_f1600(row.ctypes.data)
        want[s] = row
    got = engine.keccak_lanes(lanes, torch.from_numpy(states.view(np.int64)).cuda(), perms)
    assert (got.cpu().numpy().view(np.uint64) == want).all()


@pytest.mark.parametrize("lanes", [1, 2, 5, 25])
def test_keccak_lanes_chain_1024(engine, oracle, lanes):
    """1,024 states, 64 dependent permutations each, every layout: the profiling case for the
    per-permutation issue counts (one launch of lanes_kernel per layout), checked against the
    oracle on a stride of the states."""
    n, perms = 1024, 64
    rng = np.random.default_rng(1024 + lanes)
    states = rng.integers(0, 2**63, size=(n, 25), dtype=np.uint64)
    got = engine.keccak_lanes(lanes, torch.from_numpy(states.view(np.int64)).cuda(), perms)
    got = got.cpu().numpy().view(np.uint64)
    lib = oracle.lib()
    for s in range(0, n, 97):
        row = np.ascontiguousarray(states[s])
        for _ in range(perms):
            lib.oracle_keccak_f1600(row.ctypes.data)
        assert (got[s] == row).all(), s
