"""Seeded synthetic workloads of the adaptation path (no dataset exists for
them; every draw comes from a splitmix64 stream of the stated seed).

* batched boxes: `count` box meshes with grid edge n log-uniform in
  [nmin, nmax] and a uniform target size h drawn in [0.3/n, 1.5/n], each box
  perturbed by up to 0.1 h0 with its index as the perturbation seed;
* serving stream: Poisson arrivals of adaptation jobs (rate `rate` per
  second) whose tet count is log-uniform in [2e3, 2e6] (n = round((tets/6)^(1/3))),
  half with a uniform size h in [1.0/n, 1.6/n], half with the anisotropic-front
  workload's size field: the recovered Hessian of u = tanh(50(x - o - 0.1
  sin 2 pi y)) with the front offset o drawn in [0.3, 0.7], sizes between
  min_h = 0.5/n and max_h = 2/n and weight (max_h - min_h) / 2000 (the
  Frobenius norm of the exact Hessian peaks near 2000 at the front).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

MASK = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014), uniform doubles from the top 53 bits."""

    def __init__(self, seed: int):
        self.state = seed & MASK

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next() >> 11) * 2.0 ** -53


@dataclass
class BoxJob:
    index: int
    n: int             # grid edge: 6 n^3 tets
    size: float        # uniform target size h (0 = radial field below)
    seed: int          # perturbation seed
    radial: tuple | None = None   # (h0, h1, cx, cy, cz) for h0 + h1 |x - c|
    arrival: float = 0.0          # seconds from the start of a serving run
    front: tuple | None = None    # (offset, weight, min_h, max_h): tanh-front Hessian size

    @property
    def tets(self) -> int:
        return 6 * self.n ** 3

    def estimated_output_tets(self) -> float:
        """Rough size after adaptation (fit of mesh_adapt on uniform boxes:
        about 6.9 / (h n)^3 times the input); used only to plan memory."""
        if self.front is not None:
            # a band at min_h = 0.5/n in a field of up to 2/n: about the
            # output of a uniform size 1/n
            return self.tets * 6.9
        if self.radial is None:
            c = self.size * self.n
            return self.tets * max(6.9 / c ** 3, 0.5)
        h0, h1 = self.radial[:2]
        # mean size over the unit cube is about h0 + 0.5 h1
        c = (h0 + 0.5 * h1) * self.n
        return self.tets * max(6.9 / c ** 3, 0.5)


def place_jobs(jobs, nbins):
    """Whole jobs onto nbins GPUs by greedy bin packing on estimated output
    tets: largest job first (ties by index) onto the least-loaded bin (ties
    by the lower bin). Returns one ascending list of job positions per bin.
    Jobs never share data, so the bins need no exchange."""
    order = sorted(range(len(jobs)), key=lambda i: (-jobs[i].estimated_output_tets(), i))
    load = [0.0] * nbins
    bins = [[] for _ in range(nbins)]
    for i in order:
        b = min(range(nbins), key=lambda k: (load[k], k))
        bins[b].append(i)
        load[b] += jobs[i].estimated_output_tets()
    return [sorted(b) for b in bins]


def route_stream(jobs, nbins):
    """Jobs of an arrival stream routed to nbins GPUs as they arrive: each
    job, in arrival order, to the GPU that has been given the least estimated
    output tets so far (ties by the lower GPU). Returns one list of job
    positions per GPU, in arrival order."""
    load = [0.0] * nbins
    bins = [[] for _ in range(nbins)]
    for i in sorted(range(len(jobs)), key=lambda k: (jobs[k].arrival, k)):
        b = min(range(nbins), key=lambda k: (load[k], k))
        bins[b].append(i)
        load[b] += jobs[i].estimated_output_tets()
    return bins


def batched_boxes(count=512, seed=1, nmin=4, nmax=40):
    rng = SplitMix64(seed)
    out = []
    lo, hi = math.log(nmin), math.log(nmax)
    for i in range(count):
        n = int(round(math.exp(lo + rng.uniform() * (hi - lo))))
        h = (0.3 + 1.2 * rng.uniform()) / n
        out.append(BoxJob(i, n, h, i))
    return out


def serving_stream(count=200, seed=2, rate=200.0, tmin=2e3, tmax=2e6):
    rng = SplitMix64(seed)
    out = []
    t = 0.0
    lo, hi = math.log(tmin), math.log(tmax)
    for i in range(count):
        t += -math.log(1.0 - rng.uniform()) / rate
        tets = math.exp(lo + rng.uniform() * (hi - lo))
        n = max(2, int(round((tets / 6.0) ** (1.0 / 3.0))))
        if rng.uniform() < 0.5:
            h = (1.0 + 0.6 * rng.uniform()) / n
            out.append(BoxJob(i, n, h, i, None, t))
        else:
            # the front offset is the first of three draws (the other two
            # are unused; every non-uniform job takes three)
            c = tuple(0.3 + 0.4 * rng.uniform() for _ in range(3))
            min_h, max_h = 0.5 / n, 2.0 / n
            out.append(BoxJob(i, n, 0.0, i, None, t,
                              (c[0], (max_h - min_h) / 2000.0, min_h, max_h)))
    return out


def build_job_mesh(G, job: BoxJob, pert=0.1):
    """The job's classified full-topology box on the current GPU with its
    adapt_size field (input preparation)."""
    if job.front is not None:
        coords, conn, h = job_host_input(G, job, pert)
        m = G.Mesh.reduced(3, coords, conn)
        m.derive_model_full()
        m.add_field(0, "adapt_size", h)
        return m
    coords, conn, _ = G.box(job.n, job.seed, pert)
    m = G.Mesh.reduced(3, coords, conn)
    m.derive_model_full()
    nv = coords.size // 3
    if job.radial is None:
        h = np.full(nv, job.size)
    else:
        h0, h1, cx, cy, cz = job.radial
        d = coords.reshape(-1, 3) - np.array([cx, cy, cz])
        h = h0 + h1 * np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    m.add_field(0, "adapt_size", h)
    return m


def job_host_input(G, job: BoxJob, pert=0.1):
    """Host arrays of the job's input: coords, conn, h. A front job's size
    field comes from the library's size-field chain on the GPU (element
    gradients, volume recovery twice, size from Hessian)."""
    coords, conn, _ = G.box(job.n, job.seed, pert)
    nv = coords.size // 3
    if job.front is not None:
        offset, weight, min_h, max_h = job.front
        m = G.Mesh.reduced(3, coords, conn)
        m.derive_model_full()
        m.add_field(0, "dye", front_field(coords, offset))
        hessian_size_field(m, "dye", weight, min_h, max_h)
        h = next(t.data for t in m.tags(0) if t.name == "adapt_size").copy()
        m.close()
        return coords, conn, h
    if job.radial is None:
        h = np.full(nv, job.size)
    else:
        h0, h1, cx, cy, cz = job.radial
        d = coords.reshape(-1, 3) - np.array([cx, cy, cz])
        h = h0 + h1 * np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    return coords, conn, h


# ---------------------------------------------------------------------------
# the anisotropic-front workload: a tanh front, its recovered Hessian as the
# size field, and a rotation warp applied in steps

FRONT_SHARPNESS = 50.0
HESSIAN_WEIGHT = 2.5e-5     # max_h - w |H| reaches min_h across the front
MIN_H, MAX_H = 0.002, 0.05


def front_field(coords, offset=0.5):
    """u = tanh(50 (x - offset - 0.1 sin(2 pi y))) at every vertex."""
    x = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
    return np.tanh(FRONT_SHARPNESS * (x[:, 0] - offset - 0.1 * np.sin(2.0 * np.pi * x[:, 1])))


def rotation_warp(coords, angle):
    """Displacement that turns every point within 0.5 of the axis x = y = 0.5
    by angle * 2 (0.5 - r) about that axis (r: distance to it), and leaves the
    rest in place."""
    x = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
    dx, dy = x[:, 0] - 0.5, x[:, 1] - 0.5
    r = np.sqrt(dx * dx + dy * dy)
    a = np.arctan2(dy, dx)
    rot = np.where(r < 0.5, angle * 2.0 * (0.5 - r), 0.0)
    out = np.zeros_like(x)
    out[:, 0] = np.cos(a + rot) * r - dx
    out[:, 1] = np.sin(a + rot) * r - dy
    return out.ravel()


def hessian_size_field(m, dye="dye", weight=HESSIAN_WEIGHT, min_h=MIN_H, max_h=MAX_H):
    """adapt_size from the recovered Hessian of the vertex field `dye`, the
    chain the reference's warp test uses (test_warp.cpp:70-83): element
    gradients, recovery to vertices, again, then size_from_hessian. Works on
    the library's meshes and on the CPU checkers alike."""
    d = m.dim() if callable(getattr(m, "dim", None)) else m.dim
    if m.has_tag(0, "adapt_size"):
        m.free_tag(0, "adapt_size")
    m.element_gradients(dye)
    m.recover_by_volume("grad_" + dye)
    m.free_tag(d, "grad_" + dye)
    m.element_gradients("grad_" + dye)
    m.free_tag(0, "grad_" + dye)
    m.recover_by_volume("grad_grad_" + dye)
    m.free_tag(d, "grad_grad_" + dye)
    m.size_from_hessian("grad_grad_" + dye, [weight], min_h, max_h)
    m.free_tag(0, "grad_grad_" + dye)
