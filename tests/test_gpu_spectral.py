"""GPU parity: the fused pseudospectral RHS and Y blocks of librdcu against the oracle.

Tolerance: 1e-12 relative in max-norm (the RHS criterion of the reference port's
acceptance), on white-noise and smooth inputs, even and odd grids, 1-3 dimensions,
random dictionaries with mixed derivatives, power-0 factors and constant terms.
"""
import numpy as np
import pytest

from oracle import spectral as osp
from oracle.problem import Problem, cgle_terms, parse_term
from tests.helpers import rel_err, random_terms, smooth_field, spec_terms

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _solver(prob, **kw):
    import rdcu_b200 as R

    return R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob), **kw)


def gpu_rhs(torch, prob, y, want_Y=False):
    s = _solver(prob)
    yd = torch.tensor(y, dtype=torch.float64, device="cuda")
    fd = torch.full_like(yd, float("nan"))
    Yd = torch.full((prob.nY * prob.n * prob.N * 2,), float("nan"), dtype=torch.float64, device="cuda") \
        if want_Y else None
    torch.cuda.synchronize()
    s.rhs(yd.data_ptr(), fd.data_ptr(), Yd.data_ptr() if want_Y else 0)
    f = fd.cpu().numpy()
    Y = Yd.cpu().numpy().view(np.complex128).reshape(prob.nY * prob.n, prob.N) if want_Y else None
    s.close()
    return f, Y


@pytest.mark.parametrize("Ns,Ls", [((16, 16), (20.0, 20.0)), ((32, 16), (100.0, 50.0)),
                                   ((64, 64), (100.0, 100.0))])
def test_cgle_2d_white_noise(cuda, Ns, Ls):
    rng = np.random.default_rng(1)
    prob = Problem(2, Ns, Ls, cgle_terms(2))
    y = rng.uniform(-1, 1, 2 * prob.N)
    f, _ = gpu_rhs(cuda, prob, y)
    fo = osp.rhs(y, prob)
    assert rel_err(f, fo) < TOL


@pytest.mark.parametrize("Ns", [(8,), (7,), (6,), (12,), (8, 6), (5, 7), (6, 5), (4, 4, 6), (6, 4, 5), (8, 8, 8),
                                (3, 5, 4), (16, 12, 10)])
def test_random_dictionary_shapes(cuda, Ns):
    rng = np.random.default_rng(sum(Ns) * 7 + len(Ns))
    ndim = len(Ns)
    n = 2
    Ls = tuple(float(rng.uniform(1, 10)) for _ in Ns)
    prob = Problem(n, Ns, Ls, random_terms(rng, n, ndim, 12))
    y = rng.uniform(-1, 1, n * prob.N)
    f, Y = gpu_rhs(cuda, prob, y, want_Y=True)
    fo, Yo = osp.rhs(y, prob, return_Y=True)
    assert rel_err(f, fo) < TOL
    # every block, real and imaginary parts (Y.dat)
    for k in range(prob.nY * n):
        scale = max(np.max(np.abs(Yo[k])), 1e-300)
        assert np.max(np.abs(Y[k] - Yo[k])) / scale < TOL, k


def test_cgle_3d(cuda):
    rng = np.random.default_rng(3)
    prob = Problem(2, (16, 8, 12), (30.0, 20.0, 25.0), cgle_terms(3))
    y = rng.uniform(-1, 1, 2 * prob.N)
    f, _ = gpu_rhs(cuda, prob, y)
    assert rel_err(f, osp.rhs(y, prob)) < TOL


def test_three_fields_mixed(cuda):
    rng = np.random.default_rng(5)
    n, Ns = 3, (12, 10)
    terms = random_terms(rng, n, 2, 20, max_factors=4)
    terms.append(parse_term("0.7,2"))      # constant term
    terms.append(parse_term("1.5,1,4"))    # odd-length list: power read as 0
    prob = Problem(n, Ns, (7.0, 9.0), terms)
    y = smooth_field(rng, prob)
    f, _ = gpu_rhs(cuda, prob, y)
    assert rel_err(f, osp.rhs(y, prob)) < TOL


def test_negative_powers(cuda):
    rng = np.random.default_rng(9)
    prob = Problem(2, (16, 8), (5.0, 3.0), [parse_term(s) for s in
                                            ["1.0,0,0,-1", "0.5,1,1,-2,0,1", "1.0,0,6,1", "-0.3,1,2,1,0,-1"]])
    y = rng.uniform(1.0, 2.0, 2 * prob.N)
    f, _ = gpu_rhs(cuda, prob, y)
    assert rel_err(f, osp.rhs(y, prob)) < TOL


@pytest.mark.parametrize("Ns", [(128, 128), (256, 256), (32, 32, 32)])
def test_plane_wave_laplacian_large(cuda, Ns):
    """Size-independent check at full sizes: a plane wave is an eigenfunction of the
    spectral Laplacian (exact up to rounding), so f = -|k|^2 u."""
    ndim = len(Ns)
    Ls = tuple(100.0 for _ in Ns)
    n = 1
    # u_aa indices: n + ndim*n + (a*ndim+a)*n
    terms = [parse_term("1.0,0,%d,1" % (1 + ndim + a * ndim + a)) for a in range(ndim)]
    prob = Problem(n, Ns, Ls, terms)
    grids = np.meshgrid(*[np.arange(N) * (L / N) for N, L in zip(Ns, Ls)], indexing="ij")
    ks = [2 * np.pi / L * m for L, m in zip(Ls, [3, 5, 2][:ndim])]
    u = np.cos(sum(k * g for k, g in zip(ks, grids)) + 0.3)
    f, _ = gpu_rhs(cuda, prob, u.ravel())
    expect = -sum(k * k for k in ks) * u.ravel()
    assert rel_err(f, expect) < 1e-11


def test_misaligned_device_input(cuda):
    """A caller's state array that is only 8-byte aligned (an offset view) takes the
    scalar load path of the length-specialised kernels: same values as an aligned one."""
    import rdcu_b200 as R

    rng = np.random.default_rng(31)
    prob = Problem(2, (64, 128), (80.0, 160.0), cgle_terms(2))
    y = rng.uniform(-1, 1, 2 * prob.N)
    s = R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob))
    big = cuda.zeros(2 * prob.N + 1, dtype=cuda.float64, device="cuda")
    big[1:] = cuda.tensor(y, dtype=cuda.float64, device="cuda")
    ya = cuda.tensor(y, dtype=cuda.float64, device="cuda")
    assert big[1:].data_ptr() % 16 == 8
    f1, f2 = cuda.empty_like(ya), cuda.empty_like(ya)
    cuda.cuda.synchronize()
    s.rhs(big[1:].data_ptr(), f1.data_ptr())
    s.rhs(ya.data_ptr(), f2.data_ptr())
    assert cuda.equal(f1, f2)
    assert rel_err(f1.cpu().numpy(), osp.rhs(y, prob)) < TOL
    s.close()


@pytest.mark.parametrize("Ns", [(64, 512), (512, 64), (128, 256), (64, 128, 256), (256, 64, 64), (96, 192), (192, 96),
                                (96, 64, 192)])
def test_length_specialised_kernels(cuda, Ns):
    """Line lengths 64..512 (powers of two, 96, 192) run kernels compiled for their length."""
    rng = np.random.default_rng(sum(Ns))
    prob = Problem(2, Ns, tuple(0.78 * N for N in Ns), cgle_terms(len(Ns)))
    y = rng.uniform(-1, 1, 2 * prob.N)
    f, _ = gpu_rhs(cuda, prob, y)
    assert rel_err(f, osp.rhs(y, prob)) < TOL


@pytest.mark.parametrize("case", ["dense3", "degree4", "derivative_product"])
def test_dictionary_forms(cuda, case):
    """Dense polynomial form (3 fields, degree <= 3) and the term list (degree 4; a
    product with a derivative block) against the oracle."""
    rng = np.random.default_rng(7)
    if case == "dense3":
        lines = ["0.5,0", "1.0,0,0,1,1,1,2,1", "-0.7,1,1,3", "0.3,2,0,2,2,1", "1.1,2,1,1", "0.2,0,3,1",
                 "-0.4,1,2,1"]
        prob = Problem(3, (32, 24), (20.0, 15.0), [parse_term(l) for l in lines])
    elif case == "degree4":
        lines = ["1.0,0,0,4", "-0.5,1,0,2,1,2", "0.25,0,1,1", "0.3,1,6,1"]
        prob = Problem(2, (64, 32), (30.0, 20.0), [parse_term(l) for l in lines])
    else:
        lines = ["1.0,0,0,1,2,1", "-0.5,1,1,2,5,1", "0.25,0,6,1", "0.3,1,13,1"]
        prob = Problem(2, (64, 32), (30.0, 20.0), [parse_term(l) for l in lines])
    y = rng.uniform(-1, 1, prob.n * prob.N)
    f, _ = gpu_rhs(cuda, prob, y)
    assert rel_err(f, osp.rhs(y, prob)) < TOL


def test_array_and_tensor_arguments(cuda):
    """Host arrays and CUDA tensors passed as buffers give the same results as integer
    addresses. A temporary passed itself is safe, because the call holds it."""
    import torch

    import rdcu_b200 as R

    prob = Problem(2, (16, 16), (20.0, 20.0), cgle_terms(2))
    y = np.random.default_rng(9).uniform(-1, 1, 2 * prob.N)
    s = R.Solver(prob.n, prob.Ns, prob.Ls, spec_terms(prob))
    f1 = np.empty_like(y)
    s.rhs(y.ctypes.data, f1.ctypes.data)
    f2 = np.empty_like(y)
    s.rhs(y, f2)
    yd = torch.tensor(y, device="cuda")
    fd = torch.empty_like(yd)
    s.rhs(yd, fd)
    torch.cuda.synchronize()
    assert np.array_equal(f1, f2) and np.array_equal(f1, fd.cpu().numpy())
    s.set_state(0.0, 1e-3, np.array(y))
    out = np.empty_like(y)
    s.get_state(out)
    assert np.array_equal(out, y)
    s.close()


# 3D grids whose lines have 128 or 256 points run the specialised passes: the axis-0
# and axis-1 passes on TMA tiles (at most two fields, no more inverse channels than
# fields) and the x pass one row per warp (dense-polynomial dictionaries); the other axes
# stay small so the oracle finishes in seconds.  Odd sizes leave a partial last tile
# (columns beyond the spectrum are zero-filled on load and clipped on store).
def _tile_terms(kind):
    if kind == "cgle":
        return 2, cgle_terms(3)
    if kind == "one_field":  # n = 1: one folded linear channel
        return 1, [parse_term(s) for s in ["1.0,0,0,1", "0.5,0,4,1", "0.7,0,8,1", "0.3,0,12,1", "-1.0,0,0,3"]]
    if kind == "axis0_pair":  # n = 2: d_0 and d_0 d_0 both in the channels (two axis-0 groups)
        return 2, [parse_term(s) for s in ["1.0,0,0,1", "0.4,0,2,1", "0.6,0,8,1", "-0.5,1,3,1", "0.3,1,9,1",
                                           "0.2,1,16,1", "-1.0,0,0,3", "0.5,1,0,1,1,2"]]
    # n = 2: a folded channel for field 0 and the derivative d_1 u0 inside a product
    # (two channels), constant and power-0 factors
    return 2, [parse_term(s) for s in ["1.0,0,0,1", "0.4,0,14,1", "-0.6,0,22,1", "0.8,1,4,1,1,1", "-0.3,1,1,3",
                                       "0.2,1", "0.5,0,1,2,0,0"]]


@pytest.mark.parametrize("Ns,kind", [((256, 6, 10), "cgle"), ((128, 12, 8), "cgle"), ((256, 4, 6), "one_field"),
                                     ((128, 7, 9), "mixed"), ((128, 3, 5), "cgle"), ((256, 5, 7), "mixed"),
                                     ((6, 256, 10), "cgle"), ((5, 128, 7), "cgle"), ((4, 6, 256), "cgle"),
                                     ((6, 5, 128), "one_field"), ((128, 128, 8), "cgle"), ((8, 128, 256), "cgle"),
                                     ((256, 6, 8), "axis0_pair"), ((128, 5, 6), "axis0_pair")])
def test_tiled_passes_3d(cuda, Ns, kind):
    rng = np.random.default_rng(sum(Ns))
    n, terms = _tile_terms(kind)
    Ls = tuple(float(rng.uniform(5, 50)) for _ in Ns)
    prob = Problem(n, Ns, Ls, terms)
    # white noise: the RHS and every Y.dat block.  The oracle's full complex transforms
    # of these 10^4-point grids leave roundoff of ~2e-12 of a block's scale in imaginary
    # parts that are exactly zero here (even-order blocks), hence 1e-11 for the blocks.
    y = rng.uniform(-1, 1, n * prob.N)
    f, Y = gpu_rhs(cuda, prob, y, want_Y=True)
    fo, Yo = osp.rhs(y, prob, return_Y=True)
    assert rel_err(f, fo) < TOL
    for k in range(prob.nY * n):
        scale = max(np.max(np.abs(Yo[k])), 1e-300)
        assert np.max(np.abs(Y[k] - Yo[k])) / scale < 1e-11, k
    # a smooth field (some of its blocks are pure roundoff): the RHS
    y = smooth_field(rng, prob)
    f, _ = gpu_rhs(cuda, prob, y)
    assert rel_err(f, osp.rhs(y, prob)) < TOL


# With RDCU_PLANE_PASSES=1, 3D grids whose x rows and axis-1 lines both have 128 or 256
# points (axis-0 lines of 128 or 256 points too) take the x passes that also transform
# along axis 1, one thread-block cluster per plane; by default the axis-1 passes on TMA
# tiles run.  Both against the oracle, and against each other to rounding ("mixed" has
# a derivative inside a product: the forward plane pass with the general inverse x pass).
@pytest.mark.parametrize("Ns,kind", [((128, 128, 128), "cgle"), ((128, 256, 128), "cgle"),
                                     ((128, 128, 256), "one_field"), ((128, 128, 128), "mixed"),
                                     ((128, 128, 128), "axis0_pair"), ((256, 128, 128), "cgle")])
def test_plane_passes_3d(cuda, monkeypatch, Ns, kind):
    rng = np.random.default_rng(sum(Ns) + len(kind))
    n, terms = _tile_terms(kind)
    Ls = tuple(float(rng.uniform(20, 80)) for _ in Ns)
    prob = Problem(n, Ns, Ls, terms)
    for y in (rng.uniform(-1, 1, n * prob.N), smooth_field(rng, prob)):
        monkeypatch.setenv("RDCU_PLANE_PASSES", "1")
        f, _ = gpu_rhs(cuda, prob, y)
        assert rel_err(f, osp.rhs(y, prob)) < TOL
        monkeypatch.delenv("RDCU_PLANE_PASSES")
        g, _ = gpu_rhs(cuda, prob, y)
        assert rel_err(f, g) < 1e-13
