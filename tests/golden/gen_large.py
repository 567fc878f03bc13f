"""Generate tests/golden/large_proofs.json: the oracle's proofs of the two
largest configurations, as SHA-256 digests.

Run from the repository root, one size per process (each needs tens of GB of
host memory and minutes of CPU time):

    python tests/golden/gen_large.py 28 2
    python tests/golden/gen_large.py 30 1

Source of truth: the C oracle's memory-lean prove (``oracle.prove_lean``),
which is checked byte for byte against the full oracle prove at every smaller
size in tests/test_oracle.py.  Inputs are the ones tests/test_gpu_large.py
proves: (a, b) = fib_inputs(9000 + log_n, 1)[0], 80 queries.  Each entry
records the proof length, its SHA-256, the trace / quotient / first FRI
roots, the oracle's wall time, its thread count and its peak resident set.
"""
import hashlib
import json
import os
import resource
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from vortexstark_b200.workload import fib_inputs  # noqa: E402

OUT = os.path.join(HERE, "large_proofs.json")


def main(log_n: int, blowup: int) -> None:
    a, b = fib_inputs(9000 + log_n, 1)[0]
    t0 = time.time()
    blob = O.prove_lean(a, b, log_n, blowup, 80)
    dt = time.time() - t0
    w = [int.from_bytes(blob[4 * i:4 * i + 4], "little") for i in range(30)]
    entry = {
        "log_n": log_n, "blowup_bits": blowup, "a": a, "b": b, "n_queries": 80,
        "len": len(blob), "sha256": hashlib.sha256(blob).hexdigest(),
        "trace_root": w[5:13], "quotient_root": w[13:21], "fri_root0": w[22:30],
        "oracle_seconds": round(dt, 1), "oracle_threads": O.get_threads(),
        "oracle_peak_rss_gib": round(resource.getrusage(resource.RUSAGE_SELF).ru_maxrss / 2**20, 2),
    }
    rc, msg = O.verify(blob, blowup, 80)
    assert rc == 0, msg
    data = json.load(open(OUT)) if os.path.exists(OUT) else {}
    data[f"{log_n}_{blowup}"] = entry
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
        f.write("\n")
    print(json.dumps(entry))


if __name__ == "__main__":
    main(int(sys.argv[1]), int(sys.argv[2]))
