"""vortexstark_b200 — the VortexSTARK Circle-STARK commitment path on NVIDIA B200.

Hand-written sm_100a CUDA (libvortex_b200.so, C ABI in include/vortex_b200.h)
for the M31 circle NTT / LDE, Blake2s Merkle commitments, FRI folds with
per-layer commitments, the Fiat-Shamir transcript and query decommitment of
the Fibonacci prover.  Python modules mirror the reference's Rust modules:
``circle``, ``ntt``, ``merkle``, ``fri``, ``channel``, ``prover``, ``verifier``,
``proof``.
"""
from ._lib import lib, VortexError  # noqa: F401

__version__ = "0.1.0"
