"""Full-size parity cases run the same way on the reference (CPU, OpenMP
build in oracle/_ref/) and on this library (GPU): the seeded 512-box set's
small boxes and its largest ones, and the 96^3 anisotropic front workload's
first mesh_adapt and first warp step.

Each flow takes a mesh factory `make(dim, coords, conn)` so one definition
drives both implementations; tests/golden/make_large_digests.py records the
reference's digests, the GPU tests compare with them."""
import numpy as np

from omega_h_v1_b200 import workloads as W

# mesh_adapt arguments of the box sets (adapt.cpp:82-94 call of the box
# workloads) and of the front workload (test_warp.cpp's floors, a pass cap
# the front needs)
BOX_ADAPT = (1.0 / 3.0, 0.3, 4, 50)
FRONT_ADAPT = (1.0 / 3.0, 0.4, 0, 500)
FRONT_N, FRONT_WARP_STEPS, FRONT_ANGLE, FRONT_WARP_FLOOR = 96, 8, 0.5, 0.1


def batched_subset(count_largest=3, nmax_small=16):
    """Jobs of the seeded 512-box set (seed 1) pinned at full size: every box
    with n <= nmax_small, then the count_largest boxes of largest n (ties by
    index)."""
    jobs = W.batched_boxes()
    small = [j for j in jobs if j.n <= nmax_small]
    large = sorted(jobs, key=lambda j: (-j.n, j.index))[:count_largest]
    return small + large


def box_job_mesh(make, box, job):
    """The job's classified box with its uniform adapt_size, from a box
    generator `box(n, seed, pert)` (the library's and the oracle's are the
    same)."""
    coords, conn, _ = box(job.n, job.seed, 0.1)
    m = make(3, coords, conn)
    m.derive_model_full()
    m.add_field(0, "adapt_size", np.full(coords.size // 3, job.size))
    return m


def _vertex_field(m, name):
    for t in m.tags(0):
        if t.name == name:
            return t.data
    raise KeyError(name)


def front_mesh(make, box):
    """The 96^3 box carrying u = tanh(50 (x - 0.5 - 0.1 sin 2 pi y)) as the
    vertex field "dye" and its recovered-Hessian size field."""
    coords, conn, _ = box(FRONT_N, 0, 0.1)
    m = make(3, coords, conn)
    m.derive_model_full()
    m.add_field(0, "dye", W.front_field(coords))
    W.hessian_size_field(m)
    return m


def front_warp_step(m):
    """One of the eight warp steps: rotate by 0.5/8 rad, warp_to_limit
    (floor 0.1), new size field and mesh_adapt, up to four tries until the
    warp is used up. Returns the number of tries."""
    m.add_field(0, "warp", W.rotation_warp(_vertex_field(m, "coordinates"),
                                           FRONT_ANGLE / FRONT_WARP_STEPS), 3)
    tries = 0
    for _ in range(4):
        ok = m.warp_to_limit(FRONT_WARP_FLOOR)
        W.hessian_size_field(m)
        m.adapt(*FRONT_ADAPT)
        tries += 1
        if ok:
            break
    m.free_tag(0, "warp")
    return tries
