"""GPU: rdcu_rhs_noalloc, the RHS entry point that allocates no device memory.

Some callers cannot call cudaMalloc: a process whose GPU memory is already held by
another framework's caching allocator (a raw cudaMalloc would fail or fragment it), or
a real-time loop that cannot afford the device-wide synchronisation cudaMalloc/cudaFree
may bring.  rdcu_rhs_noalloc serves them from a fixed 64 MiB device array inside the
library.  This test calls it through the C ABI twice in a row -- the second call runs
on whatever the first left in that shared array -- and checks each result against the
allocating entry point rdcu_rhs on the same input, within the 1e-12 relative (max-norm)
RHS tolerance of the other parity tests.  It also checks that a problem too large for
the array is refused.  This file sorts last so that a run stopping at its first
failure has already run every other test.
"""
import numpy as np
import pytest

from oracle.problem import Problem, cgle_terms
from tests.helpers import rel_err, random_terms, spec_terms

pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_noalloc_matches_rdcu_rhs_twice(cuda):
    import rdcu_b200 as R

    torch = cuda
    rng = np.random.default_rng(2024)
    prob = Problem(2, (64, 48), (30.0, 25.0), cgle_terms(2) + random_terms(rng, 2, 2, 6))
    s = R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob))
    for call in range(2):
        y = torch.tensor(rng.uniform(-1, 1, prob.n * prob.N), dtype=torch.float64, device="cuda")
        f_ref = torch.empty_like(y)
        f_new = torch.full_like(y, float("nan"))
        torch.cuda.synchronize()
        s.rhs(y.data_ptr(), f_ref.data_ptr())
        R.rhs_noalloc(prob.n, prob.Ns, prob.Ls, spec_terms(prob), y.data_ptr(), f_new.data_ptr())
        torch.cuda.synchronize()
        a, b = f_new.cpu().numpy(), f_ref.cpu().numpy()
        assert np.all(np.isfinite(a)), call
        assert rel_err(a, b) < TOL, call
    s.close()


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
