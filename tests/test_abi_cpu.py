"""C-ABI checks that need no GPU: the library loads, exports every symbol the header
declares, reports sizes, and fails loudly (no CPU fallback) without a device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    inc = os.path.join(ROOT, "include")
    text = "".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc)) if f.endswith(".h"))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*([A-Za-z_][A-Za-z_0-9]*)\s*\(", text, flags=re.M))
    return {n for n in names if n not in ("if", "defined")}


@pytest.fixture(scope="module")
def lib():
    from dpcrypto_b200 import build

    path = build.build()
    return ctypes.CDLL(path)


def test_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) >= 19
    for n in sorted(names):
        assert hasattr(lib, n), n


def test_binding_covers_header():
    from dpcrypto_b200 import EXPORTS

    assert _declared() == set(EXPORTS)


def test_sizes():
    import dpcrypto_b200 as d

    assert d.sizes(0) == dict(pk=15632, sk=31296, ct=15744, ss=24, kp_coins=64, enc_coins=24)
    assert (d.sizes(2)["pk"], d.sizes(2)["sk"], d.sizes(2)["ct"]) == (672, 1568, 736)
    assert (d.sizes(3)["pk"], d.sizes(3)["sk"], d.sizes(3)["ct"]) == (992, 2304, 1088)
    assert (d.sizes(4)["pk"], d.sizes(4)["sk"], d.sizes(4)["ct"]) == (1312, 3040, 1472)
    assert d.sizes(1) == d.sizes(0)  # FrodoKEM-976-AES: the SHAKE variant's sizes
    with pytest.raises(d.DpkemError):
        d.sizes(5)


def test_no_silent_fallback_without_device():
    import torch

    import dpcrypto_b200 as d

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(d.DpkemError):
        d.Engine(0)


def test_tuning_knobs():
    """Every knob the autotuner writes is accepted within its range; unknown keys and values
    out of range are rejected (dpkem_set_tuning is host-only)."""
    from dpcrypto_b200 import kem

    lib = kem.load()
    saved = kem.get_tuning()
    try:
        for k in kem.RUNTIME_KNOBS:
            assert lib.dpkem_set_tuning(k.encode(), 32 if k == "thread_block" else 1) == kem.OK, k
            assert kem.tuning_value(k) == (32 if k == "thread_block" else 1), k
        for k in ("saber_pair_max", "saber_five_max", "saber_finish_five_max", "frodo_five_max", "frodo_ss_five_max",
                  "saber_tc_ctas_per_sm", "saber_warp_max", "saber_finish_warp_max", "frodo_warp_max",
                  "frodo_ss_warp_max", "mixed_warp_max"):
            assert lib.dpkem_set_tuning(k.encode(), 0) == kem.OK  # 0 = never on lane pairs / five lanes
        assert lib.dpkem_set_tuning(b"pipe_priority", 0) == kem.OK
        assert lib.dpkem_set_tuning(b"thread_block", 0) == kem.EINVAL
        assert lib.dpkem_set_tuning(b"thread_block", 48) == kem.EINVAL
        assert lib.dpkem_set_tuning(b"saber_pair_max", -1) == kem.EINVAL
        assert lib.dpkem_set_tuning(b"no_such_knob", 1) == kem.EINVAL
    finally:
        defaults = {"thread_block": 64, "mixed_frodo_task": 256, "mixed_pair_task": 128, "mixed_thread_task": 256,
                    "pipe_chunks": 4, "pipe_priority": 1, "saber_pair_max": 6144, "saber_five_max": 0,
                    "saber_finish_five_max": 0, "frodo_five_max": 0, "frodo_ss_five_max": 0,
                    "saber_tc_ctas_per_sm": 0, "saber_warp_max": 512, "saber_finish_warp_max": 1024,
                    "frodo_warp_max": 1024, "frodo_ss_warp_max": 1024, "mixed_warp_max": 0}
        for k in kem.RUNTIME_KNOBS:
            lib.dpkem_set_tuning(k.encode(), saved.get(k, defaults[k]))


def test_autotune_lanes_choice():
    """Per-stage lanes-per-state thresholds from a synthetic sweep: each layout covers the
    batches up to the largest size at which it was fastest; a five-lane range shadowed by the
    warp range is dropped; the pair threshold compares pair and one lane on prologue + finish."""
    from dpcrypto_b200 import autotune as at

    def sweep(win: dict, layouts):
        return {f"{n}/{l}": (1.0 if l == w else 2.0) for n, w in win.items() for l in layouts}

    sab = ("warp", "five", "pair", "one")
    fro = ("warp", "five", "one")
    best = {
        "lanes_saber_prologue_ms": sweep({64: "warp", 512: "warp", 1024: "five", 4096: "pair", 16384: "one"}, sab),
        "lanes_saber_finish_ms": sweep({64: "warp", 512: "five", 1024: "warp", 4096: "pair", 16384: "one"}, sab),
        "lanes_frodo_prologue_ms": sweep({64: "warp", 1024: "warp", 4096: "one"}, fro),
        "lanes_frodo_ss_ms": sweep({64: "five", 1024: "one", 4096: "one"}, fro),
        "saber_tc_ctas_per_sm_ms": {"1024/0": 1.0, "1024/1": 1.2, "4096/0": 2.0, "4096/1": 1.9},
        "mixed_warp_max_ms": {"512/0": 3.0, "512/512": 2.0, "4096/0": 5.0, "4096/512": 5.1},
    }
    ch = at.lanes_choice(best)
    assert ch["saber_warp_max"] == 512 and ch["saber_five_max"] == 1024
    assert ch["saber_finish_warp_max"] == 1024 and ch["saber_finish_five_max"] == 0  # shadowed
    # pair against one lane on prologue + finish: 1 + 1 < 2 + 2 at 4096; 2 + 2 > 1 + 1 at 16384;
    # a tie where neither is fastest
    assert ch["saber_pair_max"] == 4096
    assert ch["frodo_warp_max"] == 1024 and ch["frodo_five_max"] == 0
    assert ch["frodo_ss_warp_max"] == 0 and ch["frodo_ss_five_max"] == 64
    assert ch["saber_tc_ctas_per_sm"] == 0
    assert ch["mixed_warp_max"] == 512
    from dpcrypto_b200 import kem

    assert set(ch) <= set(kem.RUNTIME_KNOBS)


def test_service_host_checks():
    """Service entry points: documented defaults, and argument errors reported before any
    device work (no GPU needed)."""
    import ctypes as C

    from dpcrypto_b200 import kem

    lib = kem.load()
    cfg = kem.ServiceConfig()
    assert lib.dpkem_service_default_config(C.byref(cfg)) == kem.OK
    assert (cfg.max_inflight, cfg.idle_ms, cfg.saber_ctas, cfg.warp_max, cfg.scratch_bytes) == (16384, 1000, 0, 32, 0)
    assert not cfg.coin_key
    assert lib.dpkem_service_default_config(None) == kem.EINVAL
    out = C.c_void_p()
    assert lib.dpkem_service_open(None, kem.FORM_TC, None, C.byref(out)) == kem.EINVAL
    acc, first = C.c_size_t(7), C.c_uint64()
    assert lib.dpkem_service_submit(None, 1, None, C.byref(acc), C.byref(first)) == kem.EINVAL
    assert acc.value == 0
    assert lib.dpkem_service_poll(None, None, 0, None) == kem.EINVAL
    assert lib.dpkem_service_drain(None, 10) == kem.EINVAL
    assert lib.dpkem_service_close(None) == kem.EINVAL


def test_build_defines_from_tuning(tmp_path, monkeypatch):
    """Both Keccak round-unroll knobs in tuning.json become compile-time defines."""
    import json

    from dpcrypto_b200 import build

    t = tmp_path / "tuning.json"
    t.write_text(json.dumps({"chosen": {"keccak_unroll": 2, "keccak_unroll_rows": 6, "thread_block": 32}}))
    monkeypatch.setattr(build, "TUNING", str(t))
    assert build.tuning_defines() == ["-DDPKEM_KECCAK_UNROLL=2", "-DDPKEM_KECCAK_UNROLL_ROWS=6"]
    t.write_text(json.dumps({"chosen": {"keccak_unroll": 1}}))
    assert build.tuning_defines() == ["-DDPKEM_KECCAK_UNROLL=1"]
