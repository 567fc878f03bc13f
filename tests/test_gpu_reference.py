"""The oracle and the product against the reference's own CUDA kernels.

oracle/_ref/libvxref.so is the reference's hot-path .cu sources, compiled
unmodified for sm_100a with its default features, driven through the
prove_lean_inner order (oracle/ref_driver.cu).  Equal proof bytes pin the
oracle's NTT / twiddle conventions, Blake2s trees, quotient and folds to the
reference's device code.
"""
import pytest

from vortexstark_b200 import prover
from vortexstark_b200.workload import fib_inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(oracle):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/libvxref.so not built (needs the reference sources at build time)")
    return oracle


@pytest.mark.parametrize("log_n", [4, 5, 6, 8, 10, 12, 14, 16])
def test_reference_kernels_equal_oracle_and_product(ref, log_n):
    for a, b in fib_inputs(1000 + log_n, 2) + [(1, 1)]:
        want = ref.ref_prove(a, b, log_n)
        assert ref.prove(a, b, log_n) == want, ("oracle", log_n, a, b)
        assert prover.prove_bytes(a, b, log_n) == want, ("product", log_n, a, b)


def test_reference_kernels_blowup_one(ref):
    a, b = fib_inputs(4242, 1)[0]
    want = ref.ref_prove(a, b, 10, 1)
    assert ref.prove(a, b, 10, 1) == want
    assert prover.prove_bytes(a, b, 10, 1) == want
