"""The reference run as several ranks (the fork-based MPI stand-in of
oracle/shim) against the same run on one rank.

GAMERA-OP's README runs it as mpirun -n N with one thread per rank; the
oracle and the timed CPU baseline do the same through the stand-in.  A
2x2x1 decomposition of the Orszag-Tang case (C1's "4 ranks") must give the
single-rank result: the decomposition changes only how the ranks compute
their own grid coordinates, which on this uniform grid gives the same bits.
Test infrastructure only (CPU).
"""
import numpy as np
import pytest

ref_run = pytest.importorskip("ref_run")

NG = 4


@pytest.mark.skipif(not ref_run.available("cart", "strict"), reason="reference binary not built")
@pytest.mark.parametrize("dims,bc", [((2, 2, 1), "pppppp"), ((2, 1, 2), "pppppp"),
                                     ((2, 2, 1), "eeppee")])
def test_ranks_match_one_rank(dims, bc):
    n = (32, 32, 8) if dims[2] == 1 else (32, 16, 16)
    env = {"GOP_BC": bc, "GOP_DOMAIN": "0,1,0,1,0,0.25"}
    one = ref_run.run(n, 12, problem="ot", env=env, timeout=600)
    many = ref_run.run(n, 12, problem="ot", env=env, dims=dims, timeout=600)
    a, b = one.state(-1), many.state(-1)
    act = tuple(slice(NG, NG + m) for m in n)
    for k in ("rho", "v1", "v2", "v3", "p"):
        np.testing.assert_array_equal(a[k][act], b[k][act], err_msg=k)
    for ax, k in enumerate(("bi", "bj", "bk")):
        s = list(act)
        s[ax] = slice(NG, NG + n[ax] + 1)
        np.testing.assert_array_equal(a[k][tuple(s)], b[k][tuple(s)], err_msg=k)
    assert a["time"] == b["time"]


@pytest.mark.skipif(not ref_run.available("cart", "strict"), reason="reference binary not built")
def test_rank_timing_line_and_failure_exit():
    """The timing line comes from rank 0, and a process grid that does not
    match the rank count fails instead of hanging."""
    r = ref_run.run((16, 16, 8), 4, problem="blast", dims=(2, 2, 2), keep_output=False,
                    timeout=300)
    assert r.wall_steps == 3 and r.wall_seconds > 0
    with pytest.raises(RuntimeError):
        ref_run.run((15, 16, 8), 2, problem="blast", dims=(2, 2, 2), keep_output=False,
                    timeout=300)
