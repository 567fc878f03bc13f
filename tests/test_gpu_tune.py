"""The autotuner's knobs change launch shapes only: NTTs, Fibonacci proofs
and lifted commitments are identical to the oracle under every plan tried,
and after vx_autotune itself."""
import numpy as np
import pytest

from gpu_util import to_dev, to_host
from vortexstark_b200 import tune
from vortexstark_b200.workload import m31_array

pytestmark = pytest.mark.gpu
P = 0x7FFFFFFF

NTT_PLANS = [(9, 3), (9, 5), (10, 4), (10, 6), (11, 7), (12, 8), (12, 9), (12, 10), (11, 11), (12, 12),
             (13, 12), (14, 12), (14, 10), (13, 11), (13, 10), (11, 8)]


@pytest.fixture(autouse=True)
def _defaults():
    tune.reset()
    yield
    tune.reset()


@pytest.mark.parametrize("k", [11, 13, 14, 17, 20, 23, 24, 26])
def test_ntt_plans_match_oracle(oracle, k):
    from vortexstark_b200 import ntt
    from vortexstark_b200.circle import Coset
    cache = ntt.TwiddleCache(Coset.half_coset(k))
    x = m31_array(300 + k, 1 << k)
    want = oracle.ntt_evaluate(x, oracle.coset("half_coset", k))
    for bottom, upper in NTT_PLANS:
        tune.set_ntt_plan(k, bottom, upper)
        assert tune.get(tune.NTT_PLAN, k) == (bottom, upper)
        d = to_dev(x)
        ntt.evaluate(d, cache)
        assert np.array_equal(to_host(d), want), (bottom, upper)
        ntt.interpolate(d, cache)
        assert np.array_equal(to_host(d), x), (bottom, upper)


@pytest.mark.parametrize("L", [13, 16, 22])
def test_stwo_ntt_plans_match_oracle(oracle, L):
    from vortexstark_b200 import ntt
    cache = ntt.StwoNttCache(L)
    x = m31_array(77 + L, 1 << L)
    want = oracle.stwo_ntt_evaluate(x)
    for bottom, upper in NTT_PLANS:
        tune.set_ntt_plan(L, bottom, upper)
        d = to_dev(x)
        ntt.evaluate_stwo(d, cache)
        assert np.array_equal(to_host(d), want), (bottom, upper)
        ntt.interpolate_stwo(d, cache)
        assert np.array_equal(to_host(d), x), (bottom, upper)


def _proof(log_n, oracle_bytes):
    from vortexstark_b200.prover import ProverCache, prove_cached_bytes
    cache = ProverCache(log_n)  # a fresh slot: trees carved with the current knobs
    got = prove_cached_bytes(3, 5, cache)
    cache.close()
    assert got == oracle_bytes
    return got


def test_proofs_identical_under_leaf_k_and_ntt_plans(oracle):
    log_n = 16  # evaluation domain 2^17 (blowup 2): the leaf kernel runs
    from vortexstark_b200.prover import BLOWUP_BITS
    le = log_n + BLOWUP_BITS
    want = oracle.prove(3, 5, log_n)
    for k in (1, 2, 3, 4):
        for d in range(le - 4, le + 1):
            tune.set_leaf_k(d, k)
            tune.set_fold_leaf_k(d, 5 - k)
        assert tune.get(tune.LEAF_K, le)[0] == k
        assert tune.get(tune.FOLD_LEAF_K, le - 1)[0] == 5 - k
        _proof(log_n, want)
    for bottom, upper in NTT_PLANS[:3]:
        for t in range(4, le + 1):
            tune.set_ntt_plan(t, bottom, upper)
        _proof(log_n, want)


def test_lifted_identical_under_leaf_k(oracle):
    from vortexstark_b200.lifted import commit_lifted
    from vortexstark_b200 import _lib
    logs = [10] * 6 + [14] * 4 + [16] * 3   # lifted domain 2^18
    rng = np.random.default_rng(5)
    cols = [rng.integers(0, P, 1 << L, dtype=np.uint32) for L in logs]
    want = oracle.commit_lifted(cols, 2, 40)
    for k in (1, 2, 4):
        for d in range(12, 19):
            tune.set_leaf_k(d, k)
        _lib.lib().vx_lifted_release_all()  # the cached context was carved with the old knob
        assert commit_lifted(cols, 2, 40) == want, k


def test_autotune_report_and_results(oracle):
    from vortexstark_b200 import _lib
    rep = tune.autotune(19)
    assert sorted(rep["ntt"]) == list(range(13, 20))
    assert sorted(rep["leaf_k"]) == [17, 18, 19]
    assert sorted(rep["fold_leaf_k"]) == [17, 18, 19]
    for d, (k, ms) in rep["fold_leaf_k"].items():
        assert 1 <= k <= 4 and ms > 0
        assert tune.get(tune.FOLD_LEAF_K, d)[0] == k
    for t, (b, u, ms) in rep["ntt"].items():
        assert 10 <= b <= 12 and 6 <= u <= 9 and ms > 0
        assert tune.get(tune.NTT_PLAN, t) == (b, u)
    for d, (k, ms) in rep["leaf_k"].items():
        assert 1 <= k <= 4 and ms > 0
        assert tune.get(tune.LEAF_K, d)[0] == k
    _lib.lib().vx_lifted_release_all()
    _proof(17, oracle.prove(3, 5, 17))


def test_tune_set_rejects_bad_knobs():
    from vortexstark_b200 import _lib
    for args in ((0, 20, 8, 9), (0, 20, 12, 13), (0, 20, 15, 9), (0, 20, 12, 2), (1, 20, 5, 0), (2, 20, 5, 0),
                 (3, 20, 1, 0), (0, 40, 12, 9)):
        with pytest.raises(_lib.VortexError):
            _lib.check(_lib.lib().vx_tune_set(*args))


def test_fri_chain_identical_under_fold_leaf_k(oracle):
    from vortexstark_b200.fri import FriChain
    L = 19
    src = np.stack([m31_array(500 + c, 1 << L) for c in range(4)])
    state = list(range(8))
    want = oracle.fri_chain(src, state)
    cols = [to_dev(c) for c in src]
    for k in (1, 2, 3, 4):
        for d in range(17, 19):
            tune.set_fold_leaf_k(d, k)
        ch = FriChain(L)  # trees carved with the current knob
        ch.commit_async(cols, state)
        roots, alphas, last = ch.result()
        ch.close()
        assert np.array_equal(np.array(roots, np.uint32), want[0]), k
        assert np.array_equal(np.array(last, np.uint32), want[2]), k
