"""GPU: ensembles of 2D DP45 problems (rdcu_ensemble_*) against single handles.

Every member of a batched ensemble must reproduce, bitwise, the trajectory of a single
handle with the same spec: the same accepted and rejected attempts and the same final
state -- for uneven grid sizes (powers of two and not), per-member coefficients and
tolerances, dictionaries whose channels take the general (unsorted) axis-0 path, members
that start at different times, and after the autotuner changed the tiles.
"""
import numpy as np
import pytest

from oracle.problem import cgle_coupling_lines, parse_term

pytestmark = pytest.mark.gpu


def _cgle(b, c):
    return [(t.C, list(t.ints)) for t in (parse_term(s) for s in cgle_coupling_lines(2, b, c))]


def _members(rng):
    out = []
    for k, (Ns, b, c) in enumerate([((16, 16), 2.0, 0.8), ((24, 20), 1.0, -0.5), ((32, 32), 2.5, -1.5),
                                    ((20, 15), 0.7, 0.3), ((64, 48), 1.5, -1.0), ((48, 64), 3.0, -2.0),
                                    ((96, 192), 1.2, -0.6)]):
        out.append(dict(n=2, Ns=Ns, Ls=(0.78 * Ns[0], 0.78 * Ns[1]), terms=_cgle(b, c),
                        rtol=1e-8 if k % 2 else 1e-9, atol=1e-8 if k % 2 else 1e-9))
    # products of derivative blocks (n = 2, Y index = block * 2 + field: u0_x = 2,
    # u1_y = 5, u0_xy = 8): five inverse channels, the general axis-0 path
    terms = [(0.1, [0, 6, 1]), (0.1, [0, 12, 1]), (0.1, [1, 7, 1]), (0.1, [1, 13, 1]),
             (1.0, [0, 0, 1]), (-1.0, [0, 0, 3]), (1.0, [1, 1, 1]), (-1.0, [1, 1, 3]),
             (0.05, [0, 0, 1, 2, 1]), (0.05, [1, 1, 1, 5, 1]), (0.02, [0, 2, 1, 5, 1]),
             (0.01, [1, 8, 1, 0, 1]), (0.3, [0, 1, 1]), (-0.3, [1, 0, 1])]
    out.append(dict(n=2, Ns=(24, 32), Ls=(30.0, 40.0), terms=terms, rtol=1e-8, atol=1e-8))
    return out


def _ics(members, seed):
    rng = np.random.default_rng(seed)
    return [rng.uniform(-0.5, 0.5, m["n"] * m["Ns"][0] * m["Ns"][1]) for m in members]


def _single(torch, m, y0, t0, h0, t1):
    import rdcu_b200 as R

    s = R.Solver(m["n"], m["Ns"], m["Ls"], m["terms"], rtol=m["rtol"], atol=m["atol"])
    y = torch.tensor(y0, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    s.set_state(t0, h0, y.data_ptr())
    s.solve(t1, [])
    out = torch.empty_like(y)
    t, h, _ = s.get_state(out.data_ptr())
    acc, att = s.counters()
    s.close()
    return out.cpu().numpy(), t, h, acc, att


def _run_ensemble(torch, ens, members, ys, t0s, h0, t1):
    for i, y0 in enumerate(ys):
        y = torch.tensor(y0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ens.set_state(i, t0s[i], h0, y.data_ptr())
    ens.solve(t1)
    res = []
    for i, y0 in enumerate(ys):
        out = torch.empty(y0.size, dtype=torch.float64, device="cuda")
        t, h = ens.get_state(i, out.data_ptr())
        acc, att = ens.counters(i)
        res.append((out.cpu().numpy(), t, h, acc, att))
    return res


def test_members_match_single_handles_bitwise(cuda):
    import rdcu_b200 as R

    rng = np.random.default_rng(1)
    members = _members(rng)
    ys = _ics(members, 2)
    t0s = [0.0, 0.0, 0.1, 0.0, 0.05, 0.0, 0.0, 0.0]
    ens = R.Ensemble(members)
    got = _run_ensemble(cuda, ens, members, ys, t0s, 1e-3, 2.0)
    for i, m in enumerate(members):
        ref = _single(cuda, m, ys[i], t0s[i], 1e-3, 2.0)
        y, t, h, acc, att = got[i]
        assert (acc, att) == (ref[3], ref[4]), (i, acc, att, ref[3], ref[4])
        assert t == ref[1] and h == ref[2], i
        assert np.array_equal(y, ref[0]), (i, float(np.max(np.abs(y - ref[0]))))
        assert acc > 5
    ens.close()


def test_tuned_tiles_keep_results(cuda):
    import rdcu_b200 as R

    rng = np.random.default_rng(3)
    members = _members(rng)[:5]
    ys = _ics(members, 4)
    ens = R.Ensemble(members)
    before = _run_ensemble(cuda, ens, members, ys, [0.0] * 5, 1e-3, 0.2)
    tile = ens.tune()
    assert tile in (512, 1024, 2048, 4096)
    after = _run_ensemble(cuda, ens, members, ys, [0.0] * 5, 1e-3, 0.2)
    for a, b in zip(before, after):
        assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]
    ens.close()


def test_finished_members_are_not_stepped(cuda):
    import rdcu_b200 as R

    rng = np.random.default_rng(5)
    members = _members(rng)[:3]
    ys = _ics(members, 6)
    ens = R.Ensemble(members)
    res = _run_ensemble(cuda, ens, members, ys, [0.0, 0.5, 0.0], 1e-3, 0.3)
    assert res[1][3:] == (0, 0) and np.array_equal(res[1][0], ys[1])
    assert res[0][3] > 0 and res[2][3] > 0
    # a second solve continues from where each member stopped
    ens.solve(0.6)
    acc1, _ = ens.counters(1)
    assert acc1 > 0
    ens.close()


def test_error_paths(cuda):
    import rdcu_b200 as R

    good = dict(n=2, Ns=(16, 16), Ls=(12.0, 12.0), terms=_cgle(2.0, 0.8))
    with pytest.raises(R.RdcuError) as e:
        R.Ensemble([good, dict(n=2, Ns=(8, 8, 8), Ls=(5.0, 5.0, 5.0), terms=[])])
    assert e.value.code == R.RDCU_ERR_UNSUPPORTED
    ens = R.Ensemble([good])
    y = cuda.zeros(2 * 256, dtype=cuda.float64, device="cuda")
    with pytest.raises(R.RdcuError) as e:
        ens.set_state(3, 0.0, 1e-3, y.data_ptr())
    assert e.value.code == R.RDCU_ERR_INVALID
    ens.close()
