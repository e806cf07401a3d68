"""dpcrypto_b200: batched FrodoKEM-976-SHAKE and Saber KEM engine for B200 (sm_100a).

The compute path is libdpkem.so (hand-written CUDA for sm_100a behind a C ABI,
include/dpkem.h); this package only binds it (kem.py) and builds it (build.py).
"""
from .kem import (  # noqa: F401
    EXPORTS, FIRESABER, FLAG_DEVICE_PTRS, FORM_DP4A, FORM_INT32, FORM_TC, FRODO976, FRODO976AES, LIGHTSABER, SABER, SCHEMES,
    DpkemError, Engine, MixedGraph, Request, Service, ServiceConfig, frodoKEMDecap, frodoKEMEncap, frodoKEMKeypair, load, saber_dec, saber_enc, set_compat,
    sizes,
)
