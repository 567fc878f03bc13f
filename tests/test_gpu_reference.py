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


@pytest.mark.parametrize("log_n", [20, 24])
def test_ntt_faster_than_reference_kernels(ref, log_n):
    """Same transform, same B200: this library's evaluate / interpolate against
    the reference's (one Forge layer kernel per layer), timed with CUDA events."""
    import torch
    from vortexstark_b200 import ntt
    from vortexstark_b200.circle import Coset
    from vortexstark_b200.workload import m31_array
    from gpu_util import to_dev

    ref_e, ref_i = ref.ref_ntt_time(log_n, 5)
    cache = ntt.TwiddleCache(Coset.half_coset(log_n))
    d = to_dev(m31_array(log_n, 1 << log_n))
    ntt.evaluate(d, cache)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    for _ in range(5):
        ntt.evaluate(d, cache)
    ev[1].record()
    for _ in range(5):
        ntt.interpolate(d, cache)
    ev[2].record()
    torch.cuda.synchronize()
    my_e, my_i = ev[0].elapsed_time(ev[1]) / 5, ev[1].elapsed_time(ev[2]) / 5
    print(f"\nNTT 2^{log_n}: evaluate {my_e:.3f} ms (reference kernels {ref_e:.3f} ms), "
          f"interpolate {my_i:.3f} ms (reference kernels {ref_i:.3f} ms)")
    assert my_e < ref_e and my_i < ref_i


def _ref_ntt(ref, name):
    from vortexstark_b200 import _lib

    fn = getattr(ref.ref_lib(), name)
    fn.argtypes = _lib._SIGS[name]
    return fn


@pytest.mark.parametrize("log_n", [20, 28])
def test_ntt_words_equal_reference_kernels(ref, log_n):
    """Every word of evaluate and interpolate on 2^log_n uniform M31 values
    over half_coset(log_n) equals the reference's own launchers
    (circle_ntt.cu:248-312, Forge layer kernels) run on the same twiddle
    tables; the round trip returns the input."""
    import torch
    from vortexstark_b200 import ntt
    from vortexstark_b200.circle import Coset
    from vortexstark_b200.ntt import _host_u32
    from vortexstark_b200.workload import m31_array
    from gpu_util import to_dev

    n = 1 << log_n
    cache = ntt.TwiddleCache(Coset.half_coset(log_n))
    x = to_dev(m31_array(7000 + log_n, n))
    mine, theirs = x.clone(), x.clone()
    offs, sizes = _host_u32(cache.layer_offsets), _host_u32(cache.layer_sizes)
    ntt.evaluate(mine, cache)
    _ref_ntt(ref, "cuda_circle_ntt_evaluate")(theirs.data_ptr(), cache.d_twiddles.data_ptr(),
                                              cache.d_circle_twids.data_ptr(), offs, sizes, log_n - 1, n)
    torch.cuda.synchronize()
    assert torch.equal(mine, theirs)
    assert not torch.equal(mine, x)
    ntt.interpolate(mine, cache)
    _ref_ntt(ref, "cuda_circle_ntt_interpolate")(theirs.data_ptr(), cache.d_itwiddles.data_ptr(),
                                                 cache.d_circle_itwids.data_ptr(), offs, sizes, log_n - 1, n)
    torch.cuda.synchronize()
    assert torch.equal(mine, theirs)
    assert torch.equal(mine, x)
    del x, mine, theirs, cache
    torch.cuda.empty_cache()
