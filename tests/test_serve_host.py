"""Host logic of the request loop (gop.serve) on the CPU: admission by
slots and HBM budget, first-come-first-served order, continuous batching
(requests join and leave between rounds), exact step accounting, and the
sharded several-rank path over gloo.  A fake engine stands in for the GPU:
it advances a simulated clock by the work of each round."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, str(ROOT / "gamera-op_b200"))
from gop import serve  # noqa: E402
from gop.workloads import Job, served_stream, SERVE_GRIDS  # noqa: E402


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


class FakeEngine:
    """Device bytes = 1000 per cell; a round costs cells x steps / rate."""

    def __init__(self, clock, rate=1e9):
        self.clock, self.rate = clock, rate
        self.done_steps = {}
        self.rounds = []
        self.live = set()
        self._pending = None

    def footprint(self, job):
        return 1000 * job.cells

    def create(self, job):
        assert job.rid not in self.live
        self.live.add(job.rid)
        self.done_steps[job.rid] = 0
        return job.rid

    def prebuild(self, handles):
        assert all(h in self.live for h in handles)

    def launch(self, handles, steps):
        assert len(handles) == len(steps) and all(s > 0 for s in steps)
        assert all(h in self.live for h in handles)
        self.rounds.append(tuple(handles))
        self._pending = (handles, steps)

    def wait(self):
        handles, steps = self._pending
        work = 0
        for h, s in zip(handles, steps):
            self.done_steps[h] += s
            work += s * self.cells[h]
        self.clock.t += work / self.rate

    def finish(self, job, h):
        self.live.remove(h)
        return self.done_steps[h]


def run(jobs, budget, max_live=4, chunk=50):
    clk = Clock()
    eng = FakeEngine(clk)
    eng.cells = {j.rid: j.cells for j in jobs}
    srv = serve.Server(eng, budget, max_live=max_live, chunk=chunk, clock=clk, sleep=clk.sleep)
    return srv.run(jobs), eng


def jobs_of(specs):
    return [Job(r, 2, n, steps, arrival=t) for r, (n, steps, t) in enumerate(specs)]


def test_every_request_gets_exactly_its_steps():
    jobs = served_stream(count=40, seed=1)
    rep, eng = run(jobs, budget=10 ** 13)
    assert len(rep.outcomes) == 40
    for o, j in zip(rep.outcomes, sorted(jobs, key=lambda j: j.rid)):
        assert o.rid == j.rid and o.result == j.steps
        assert o.done >= o.arrival and o.admitted >= o.arrival
    assert not eng.live


def test_slots_and_budget_are_respected():
    jobs = served_stream(count=60, seed=2)
    big = max(1000 * j.cells for j in jobs)
    budget = 2 * big
    rep, eng = run(jobs, budget=budget, max_live=5)
    assert rep.peak_bytes <= budget
    assert rep.peak_live <= 5
    assert max(len(r) for r in eng.rounds) <= 5


def test_oversized_request_is_refused():
    jobs = jobs_of([((64, 64, 64), 10, 0.0)])
    with pytest.raises(serve.AdmissionError):
        run(jobs, budget=1000 * 64 ** 3 - 1)


def test_first_come_first_served_admission():
    # the head (large) must wait for memory; smaller later ones may not overtake it
    jobs = jobs_of([((32, 32, 32), 400, 0.0), ((64, 64, 64), 100, 0.001),
                    ((16, 16, 16), 100, 0.002)])
    budget = 1000 * (64 ** 3 + 16 ** 3)  # 64^3 cannot join while 32^3 is live
    rep, _ = run(jobs, budget=budget, max_live=8, chunk=50)
    adm = {o.rid: o.admitted for o in rep.outcomes}
    assert adm[1] <= adm[2]
    assert adm[1] >= rep.outcomes[0].done


def test_requests_join_and_leave_between_rounds():
    # a long request is live while short ones arrive, run and leave
    jobs = jobs_of([((64, 64, 64), 3000, 0.0)] + [((16, 16, 16), 60, 0.05 * k) for k in range(1, 6)])
    rep, eng = run(jobs, budget=10 ** 13, max_live=8, chunk=20)
    shared = [r for r in eng.rounds if 0 in r and len(r) > 1]
    assert shared, "short requests never shared a round with the long one"
    # short requests finish long before the long one
    done = {o.rid: o.done for o in rep.outcomes}
    assert max(done[k] for k in range(1, 6)) < done[0]
    # the member set changes over time (continuous batching, not a queue)
    assert len(set(eng.rounds)) > 3


def test_serial_baseline_is_a_fifo_queue():
    jobs = jobs_of([((8, 8, 8), 10, 0.0), ((8, 8, 8), 10, 0.0), ((8, 8, 8), 10, 5.0)])
    t = [0.0]

    def clock():
        return t[0]

    def run_one(j):
        t[0] += 1.0
        return j.rid

    rep = serve.serial(jobs, run_one, clock=clock)
    tts = [o.time_to_solution for o in rep.outcomes]
    assert tts == [1.0, 2.0, 1.0]
    assert rep.makespan == 6.0


def test_shard_covers_every_request_once():
    jobs = served_stream(count=37, seed=3)
    parts = [serve.shard(jobs, r, 3) for r in range(3)]
    ids = sorted(j.rid for p in parts for j in p)
    assert ids == list(range(37))


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jobs = served_stream(count=30, seed=4)
        mine = serve.shard(jobs, rank, world)
        clk = Clock()
        eng = FakeEngine(clk, rate=1e9 * (rank + 1))  # ranks run at different speeds
        eng.cells = {j.rid: j.cells for j in mine}
        rep = serve.Server(eng, 10 ** 13, max_live=4, chunk=100, clock=clk, sleep=clk.sleep).run(mine)
        tot = serve.combine(rep, dist)
        q.put((rank, tot, rep.cell_updates(), rep.makespan, len(rep.outcomes)))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_serving_over_gloo():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort()
    totals = [g[1] for g in got]
    assert totals[0] == totals[1]
    assert totals[0]["requests"] == 30
    assert totals[0]["cell_updates"] == sum(g[2] for g in got)
    assert totals[0]["makespan_s"] == max(g[3] for g in got)
    jobs = served_stream(count=30, seed=4)
    assert totals[0]["cell_updates"] == sum(j.cells * j.steps for j in jobs)


def test_threaded_set_up_and_copy_back_keep_the_invariants():
    jobs = served_stream(count=50, seed=6)
    clk = Clock()
    eng = FakeEngine(clk)
    eng.cells = {j.rid: j.cells for j in jobs}
    budget = 3 * max(1000 * j.cells for j in jobs)
    rep = serve.Server(eng, budget, max_live=6, chunk=40, clock=clk, sleep=clk.sleep,
                       workers=3).run(jobs)
    assert sorted(o.rid for o in rep.outcomes) == list(range(50))
    for o in rep.outcomes:
        assert o.result == next(j.steps for j in jobs if j.rid == o.rid)
    assert rep.peak_bytes <= budget and rep.peak_live <= 6
    assert not eng.live
