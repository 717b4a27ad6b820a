"""GPU: rdcu_rhs_noalloc, the RHS entry point that allocates no device memory.

Some callers cannot call cudaMalloc: a process whose GPU memory is already held by
another framework's caching allocator (a raw cudaMalloc would fail or fragment it), or
a real-time loop that cannot afford the device-wide synchronisation cudaMalloc/cudaFree
may bring.  rdcu_rhs_noalloc serves them from a fixed 64 MiB device array inside the
library.  This test calls it through the C ABI several times in a row -- each call runs
on whatever the previous one left in that shared array -- and checks each result
against the allocating entry point rdcu_rhs on the same input, within the 1e-12
relative (max-norm) RHS tolerance of the other parity tests, and that the device's
free memory does not move across the calls.  It also checks a dictionary with many
inverse channels close to the array's size, and that problems too large for the array
are refused.  This file sorts last so that a run stopping at its first
failure has already run every other test.
"""
import numpy as np
import pytest

from oracle.problem import Problem, cgle_terms
from tests.helpers import rel_err, random_terms, spec_terms

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _compare(R, torch, prob, rng, calls):
    """rdcu_rhs_noalloc against rdcu_rhs on `calls` fresh random states; every device
    buffer is made before the first call, so the free device memory (cudaMemGetInfo)
    measured after the first call must not change over the later ones."""
    s = R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob))
    ys = [torch.tensor(rng.uniform(-1, 1, prob.n * prob.N), dtype=torch.float64, device="cuda")
          for _ in range(calls)]
    f_ref = [torch.empty_like(y) for y in ys]
    f_new = [torch.full_like(y, float("nan")) for y in ys]
    torch.cuda.synchronize()
    free = []
    for call in range(calls):
        s.rhs(ys[call].data_ptr(), f_ref[call].data_ptr())
        R.rhs_noalloc(prob.n, prob.Ns, prob.Ls, spec_terms(prob), ys[call].data_ptr(), f_new[call].data_ptr())
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        a, b = f_new[call].cpu().numpy(), f_ref[call].cpu().numpy()
        assert np.all(np.isfinite(a)), call
        assert rel_err(a, b) < TOL, call
    s.close()
    # the first call may load the library's device code (and with it the fixed array);
    # the calls after it allocate nothing
    assert len(set(free[1:])) == 1, free


def test_noalloc_matches_rdcu_rhs_twice(cuda):
    import rdcu_b200 as R

    rng = np.random.default_rng(2024)
    prob = Problem(2, (64, 48), (30.0, 25.0), cgle_terms(2) + random_terms(rng, 2, 2, 6))
    _compare(R, cuda, prob, rng, 3)


def _channel_terms():
    # every first and second derivative of both fields (Y 2..13 for n = 2 in 2D) times
    # u0: twelve distinct derivative factors, each an inverse transform of its own
    return [(0.1 * (k - 1), [k % 2, k, 1, 0, 1]) for k in range(2, 14)]


def test_noalloc_many_channels_near_the_limit(cuda):
    """2 fields, 12 inverse channels on 1024 x 512: (2 + 12) * 1024 * 257 * 16 B = 59 MB
    of the 64 MiB array."""
    import rdcu_b200 as R
    from oracle.problem import Term

    rng = np.random.default_rng(7)
    prob = Problem(2, (1024, 512), (60.0, 30.0), [Term(C, ints) for C, ints in _channel_terms()])
    _compare(R, cuda, prob, rng, 2)


def test_noalloc_refuses_many_channels_beyond_the_limit(cuda):
    """The same dictionary on 1200 x 512 needs 69 MB: refused; the 2-channel CGLE
    dictionary on that grid (20 MB) runs."""
    import rdcu_b200 as R

    torch = cuda
    Ns, Ls = (1200, 512), (60.0, 30.0)
    y = torch.zeros(2 * 1200 * 512, dtype=torch.float64, device="cuda")
    f = torch.zeros_like(y)
    with pytest.raises(R.RdcuError) as e:
        R.rhs_noalloc(2, Ns, Ls, _channel_terms(), y.data_ptr(), f.data_ptr())
    assert e.value.code == R.RDCU_ERR_UNSUPPORTED
    R.rhs_noalloc(2, Ns, Ls, [(t.C, t.ints) for t in cgle_terms(2)], y.data_ptr(), f.data_ptr())
    torch.cuda.synchronize()
    assert float(f.abs().max()) == 0.0  # the RHS of the zero state


def test_noalloc_refuses_oversize(cuda):
    import rdcu_b200 as R

    torch = cuda
    y = torch.zeros(16, dtype=torch.float64, device="cuda")
    f = torch.zeros(16, dtype=torch.float64, device="cuda")
    # 2 fields on 256^3 need ~0.5 GB of spectra: beyond the fixed array
    with pytest.raises(R.RdcuError) as e:
        R.rhs_noalloc(2, (256, 256, 256), (1.0, 1.0, 1.0), [(t.C, t.ints) for t in cgle_terms(3)],
                      y.data_ptr(), f.data_ptr())
    assert e.value.code == R.RDCU_ERR_UNSUPPORTED
