"""C ABI checks that need no GPU: librdcu loads, exports every entry point that
include/rdcu.h declares, validates specifications before touching CUDA, and its
initial-condition generator reproduces the reference's glibc rand() stream."""
import ctypes
import os
import re

import numpy as np
import pytest

import rdcu_b200 as R
from oracle.problem import glibc_uniform_ic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "rdcu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rdcu_\w+)\s*\(", text)))


def test_header_declares_the_abi():
    names = declared_functions()
    for must in ("rdcu_create", "rdcu_destroy", "rdcu_rhs", "rdcu_step", "rdcu_solve", "rdcu_jac", "rdcu_eval"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(R.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(R.EXPORTS) == declared_functions()


def _spec(**kw):
    s = R.rdcu_spec()
    s.n = kw.get("n", 2)
    s.ndim = kw.get("ndim", 2)
    for a in range(3):
        s.Ns[a] = 8
        s.Ls[a] = 1.0
    s.nterms = 0
    s.method = kw.get("method", 0)
    s.rtol = s.atol = 1e-8
    return s


@pytest.mark.parametrize("bad", [dict(n=0), dict(ndim=0), dict(ndim=4), dict(method=7)])
def test_create_rejects_bad_specs(bad):
    lib = R.load_library()
    h = ctypes.c_void_p()
    rc = lib.rdcu_create(ctypes.byref(h), ctypes.byref(_spec(**bad)))
    assert rc == R.RDCU_ERR_INVALID
    assert lib.rdcu_last_error(None)


def test_create_rejects_out_of_range_terms():
    with pytest.raises(R.RdcuError) as e:
        R.Solver(2, (8, 8), (1.0, 1.0), [(1.0, [0, 14, 1])])  # 2 fields, 2D: Y indices 0..13
    assert e.value.code == R.RDCU_ERR_INVALID
    with pytest.raises(R.RdcuError):
        R.Solver(2, (8, 8), (1.0, 1.0), [(1.0, [2, 0, 1])])  # field 2 of 2


def test_error_strings():
    lib = R.load_library()
    assert lib.rdcu_error_string(R.RDCU_ERR_CUDA) == b"CUDA error"
    assert lib.rdcu_error_string(0) == b"ok"


@pytest.mark.parametrize("n,N,A,A0,seed", [(1, 7, 1e-3, 0.0, 1), (2, 50, 2.0, 0.5, 3), (3, 11, 1.0, -1.0, 12345)])
def test_random_ic_matches_glibc_stream(n, N, A, A0, seed):
    np.testing.assert_array_equal(R.random_ic(n, N, A, A0, seed), glibc_uniform_ic(n, N, A, A0, seed))


def test_no_cpu_fallback_without_gpu():
    """Without a GPU the library fails loudly (there is no CPU path)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(R.RdcuError) as e:
        R.Solver(2, (8, 8), (1.0, 1.0), [(1.0, [0, 0, 1])])
    assert e.value.code == R.RDCU_ERR_CUDA


def test_problem_coupling_lists_match_the_oracle():
    """The package's coupling lists (workload definitions) and the oracle's agree."""
    from oracle import problem as op
    from rdcu_b200 import problems as pp

    for ndim in (1, 2, 3):
        for b, c in ((2.0, 0.8), (0.7, -1.3), (-1.5, 0.0)):
            assert pp.cgle_coupling_lines(ndim, b, c) == op.cgle_coupling_lines(ndim, b, c)
            parsed = [op.parse_term(s) for s in pp.cgle_coupling_lines(ndim, b, c)]
            assert any(abs(t.C - c) < 1e-6 for t in parsed) and any(abs(t.C + b) < 1e-6 for t in parsed)
    assert pp.brusselator_coupling_lines() == op.brusselator_coupling_lines()


def test_buffer_arguments():
    """Buffers go to the C ABI as addresses, arrays or tensors; arrays and tensors must
    be contiguous; 0 and None are NULL."""
    import numpy as np
    import torch

    import rdcu_b200 as R

    a = np.zeros(4)
    assert R._addr(a).value == a.ctypes.data
    assert R._addr(0) is None and R._addr(None) is None
    assert R._addr(np.int64(16)).value == 16
    t = torch.zeros(3, dtype=torch.float64)
    assert R._addr(t).value == t.data_ptr()
    with pytest.raises(ValueError):
        R._addr(np.zeros((4, 4))[:, 1])
    with pytest.raises(ValueError):
        R._addr(torch.zeros(4, 4)[:, 1])
    with pytest.raises(TypeError):
        R._addr(True)
    with pytest.raises(TypeError):
        R._addr("0x10")
