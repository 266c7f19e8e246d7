"""Seeded synthetic workloads of the batched and served paths.

Each request or batch member is a plain description (problem kind, grid,
physics parameters, step count); ``build`` turns one into a prepared
:class:`gop.Instance`.  The generators only use numpy's seeded
``default_rng``, so the same seed gives the same work on every machine.

* ``batched_uneven``: independent Orszag-Tang (thin grids) and blast-wave
  (cubes) grids of uneven size, gamma in [1.4, 5/3], blast overpressure
  ratio in [10, 1000] and background plasma beta in [0.01, 10] (uniform),
  field direction uniform on the sphere.
* ``served_stream``: a Poisson arrival stream of blast-wave and Cartesian
  field-loop requests with grid sizes drawn from fixed weights and step
  counts uniform in [100, 1000].
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import (COORD_CARTESIAN, PREC_FP64, PREC_MIXED, PROBLEM_BLAST, PROBLEM_LOOP_CART,
               PROBLEM_OT, Instance, grid_uniform)

BATCH_GRIDS = ((64, 64, 4), (128, 128, 4), (256, 256, 4), (64, 64, 64), (96, 96, 96),
               (128, 128, 128))
SERVE_GRIDS = ((32, 32, 32), (64, 64, 64), (96, 96, 96), (128, 128, 128), (192, 192, 192))
SERVE_WEIGHTS = (0.3, 0.3, 0.2, 0.15, 0.05)
MIXED_TOLERANCE = 1e-5  # requests asking for at least this L1 error run mixed


@dataclass
class Job:
    """One grid to advance: a batch member or a served request."""
    rid: int
    kind: int
    n: tuple
    steps: int
    gamma: float = 5.0 / 3.0
    over: dict = field(default_factory=dict)  # gop_problem fields
    domain: tuple = ()
    bc: str = "pppppp"
    tol: float = MIXED_TOLERANCE
    arrival: float = 0.0  # seconds from the stream's start

    @property
    def cells(self) -> int:
        return self.n[0] * self.n[1] * self.n[2]

    @property
    def precision(self) -> int:
        return PREC_MIXED if self.tol >= MIXED_TOLERANCE else PREC_FP64

    def coords(self):
        return [grid_uniform(self.n[a], self.domain[2 * a], self.domain[2 * a + 1])
                for a in range(3)]


def _domain(kind, n):
    """Cubic cells: the third axis spans n_k/n_i of the first."""
    zr = n[2] / n[0]
    if kind == PROBLEM_OT:
        return (0.0, 1.0, 0.0, 1.0, 0.0, zr)
    if kind == PROBLEM_BLAST:
        return (-0.5, 0.5, -0.5, 0.5, -0.5 * zr, 0.5 * zr)
    return (-2.0, 2.0, -2.0, 2.0, -2.0 * zr, 2.0 * zr)


def _unit_vector(rng):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def batched_uneven(count=96, steps=200, seed=20261203):
    """Independent grids of uneven size (uniform over BATCH_GRIDS): the thin
    n^2 x 4 grids hold an Orszag-Tang vortex, the cubes a blast wave with
    overpressure ratio ~ U[10, 1000] over p_out = 0.1, plasma beta
    2 p_out / |B|^2 ~ U[0.01, 10] and field direction uniform on the sphere;
    gamma ~ U[1.4, 5/3] for all.  Every member advances ``steps`` steps."""
    rng = np.random.default_rng(seed)
    jobs = []
    for r in range(count):
        n = BATCH_GRIDS[rng.integers(len(BATCH_GRIDS))]
        kind = PROBLEM_OT if n[2] == 4 else PROBLEM_BLAST
        gamma = float(rng.uniform(1.4, 5.0 / 3.0))
        over = {}
        if kind == PROBLEM_BLAST:
            ratio = float(rng.uniform(10.0, 1000.0))
            beta = float(rng.uniform(0.01, 10.0))
            p_out = 0.1
            bmag = math.sqrt(2.0 * p_out / beta)
            over = dict(p_out=p_out, p_in=ratio * p_out, b=tuple(bmag * _unit_vector(rng)))
        jobs.append(Job(r, kind, n, steps, gamma, over, _domain(kind, n)))
    return jobs


def served_stream(count=160, rate=50.0, seed=5150, tol=MIXED_TOLERANCE):
    """Poisson arrivals (mean ``rate`` per second) of blast-wave and
    Cartesian field-loop requests."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for r in range(count):
        t += float(rng.exponential(1.0 / rate))
        n = SERVE_GRIDS[rng.choice(len(SERVE_GRIDS), p=SERVE_WEIGHTS)]
        kind = PROBLEM_BLAST if rng.random() < 0.5 else PROBLEM_LOOP_CART
        steps = int(rng.integers(100, 1001))
        jobs.append(Job(r, kind, n, steps, 5.0 / 3.0, {}, _domain(kind, n), tol=tol, arrival=t))
    return jobs


def build(job: Job, precision=None, host=None, device_init=False) -> Instance:
    """Creates, initialises and prepares the instance of a job.  ``host``
    (a dict) keeps the host arrays of the initial state for reuse by later
    jobs of the same grid shape; ``device_init`` builds the initial state on
    the device instead (no host arrays, no upload)."""
    prec = job.precision if precision is None else precision
    inst = Instance(job.n, *job.coords(), coord=COORD_CARTESIAN, bc=job.bc, precision=prec,
                    gamma=job.gamma)
    if device_init:
        inst.init_problem_device(job.kind, **job.over)
        inst.prepare()
        return inst
    out = None
    if host is not None:
        if inst.N not in host:
            host[inst.N] = (np.zeros(inst.shape(6)), np.zeros(inst.shape(3)))
        out = host[inst.N]
    gas, fb = inst.init_problem(job.kind, out=out, **job.over)
    inst.upload(gas, fb)
    inst.prepare()
    return inst


def footprint(job: Job, precision=None) -> int:
    """Device bytes an instance of the job holds (gop_footprint)."""
    from . import footprint as fp
    return fp(job.n, COORD_CARTESIAN, job.precision if precision is None else precision)
