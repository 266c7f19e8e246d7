"""The served path on the GPU: requests admitted by slots and an HBM budget,
advanced together in batched rounds while others arrive and leave, give the
same result as each request run alone (bit for bit: the same kernels and the
same arithmetic per cell), and the mixed-precision result stays within the
requested L1 tolerance of the plain FP64 path (per variable; vector
components relative to the vector's magnitude, gop.accuracy)."""
import numpy as np
import pytest


pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-5  # relative L1 per variable, mixed vs plain FP64


@pytest.fixture(scope="module")
def gop():
    import gop as g
    g.lib()
    return g


def _jobs(gop):
    from gop.workloads import Job, _domain
    rng = np.random.default_rng(77)
    grids = [(16, 16, 16), (24, 16, 16), (32, 32, 8), (20, 20, 20)]
    jobs = []
    t = 0.0
    for r in range(10):
        n = grids[rng.integers(len(grids))]
        kind = gop.PROBLEM_BLAST if r % 2 == 0 else gop.PROBLEM_LOOP_CART
        steps = int(rng.integers(20, 81))
        t += float(rng.exponential(0.02))
        jobs.append(Job(r, kind, n, steps, domain=_domain(kind, n), arrival=t))
    return jobs


def test_served_results_equal_alone_and_within_tolerance_of_fp64(gop):
    from gop import accuracy, serve, workloads
    jobs = _jobs(gop)
    eng = serve.GpuEngine(keep=lambda j: True)
    budget = 3 * max(eng.footprint(j) for j in jobs)
    rep = serve.Server(eng, budget, max_live=3, chunk=16, workers=2).run(jobs)
    assert len(rep.outcomes) == len(jobs)
    assert rep.peak_bytes <= budget and rep.peak_live <= 3
    assert rep.rounds > max(j.steps for j in jobs) // 16  # requests shared rounds
    pool = {}
    for o, j in zip(rep.outcomes, jobs):
        assert o.rid == j.rid and o.result["steps"] == j.steps
        alone = workloads.build(j, device_init=True)  # as the engine builds it
        alone.step(j.steps)
        a = serve.download_result(alone, pool, copy=True)
        alone.close()
        assert np.array_equal(o.result["gas"], a["gas"]), j
        assert np.array_equal(o.result["face_b"], a["face_b"]), j
        assert o.result["time"] == a["time"]
        ref = workloads.build(j, precision=gop.PREC_FP64, device_init=True)
        ref.step(j.steps)
        r = serve.download_result(ref, pool, copy=True)
        ref.close()
        errs = accuracy.rel_l1(j.n, o.result, r)
        assert max(errs.values()) <= TOL_MIXED, (j, errs)
        assert o.result["divb_max"] < 1e-9


def test_batch_autotune_keeps_state_and_results(gop):
    from gop import workloads
    from gop.workloads import batched_uneven
    jobs = [j for j in batched_uneven(count=12, steps=4, seed=3) if j.cells <= 64 ** 3][:5]
    for j in jobs:
        j.n = tuple(min(v, 32) for v in j.n)
        j.domain = workloads._domain(j.kind, j.n)
    alone = []
    for j in jobs:
        a = workloads.build(j)
        a.step(j.steps)
        alone.append(a.download(("gas", "face_b")))
        a.close()
    members = [workloads.build(j) for j in jobs]
    b = gop.Batch(members)
    chosen = b.autotune(reps=1)
    # candidate 14 (GOP_TUNE_SWEEP) is the tile-staged sweep of a flux or EMF launch
    assert len(chosen) == 11 and all(0 <= v <= 14 for v in chosen.values())
    b.step([j.steps for j in jobs])
    for a, m in zip(alone, members):
        d = m.download(("gas", "face_b"))
        assert np.array_equal(d["gas"], a["gas"])
        assert np.array_equal(d["face_b"], a["face_b"])
    # tuning again after steps leaves every member's state as it was
    before = [m.download(("gas", "face_b")) for m in members]
    b.autotune(reps=1)
    for m, d0 in zip(members, before):
        d = m.download(("gas", "face_b"))
        assert np.array_equal(d["gas"], d0["gas"])
        assert np.array_equal(d["face_b"], d0["face_b"])


def test_batch_autotune_with_sweep_sized_members_keeps_state_and_results(gop):
    """Members large enough for the sweep kernels: the batch autotune also
    times the batch step with and without them (restoring every member
    after each trial), and the batch still ends bit-identical to each
    member stepped alone."""
    shapes = [(96, 96, 96), (64, 64, 64), (96, 64, 32)]
    alone = []
    for n in shapes:
        a = gop.make(gop.PROBLEM_BLAST, n, b=(0.4, 0.5, 0.3))
        a.prepare()
        a.step(6)
        alone.append(a.download(("gas", "face_b")))
        a.close()
    members = [gop.make(gop.PROBLEM_BLAST, n, b=(0.4, 0.5, 0.3)) for n in shapes]
    for m in members:
        m.prepare()
    b = gop.Batch(members)
    before = [m.download(("gas", "face_b")) for m in members]
    b.autotune(reps=1)
    for m, d0 in zip(members, before):
        d = m.download(("gas", "face_b"))
        assert np.array_equal(d["gas"], d0["gas"])
        assert np.array_equal(d["face_b"], d0["face_b"])
        assert m.stats()["steps"] == 0
    b.step([6] * len(members))
    for a, m in zip(alone, members):
        d = m.download(("gas", "face_b"))
        assert np.array_equal(d["gas"], a["gas"])
        assert np.array_equal(d["face_b"], a["face_b"])
    b.close()
    for m in members:
        m.close()
