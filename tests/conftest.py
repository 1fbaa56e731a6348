"""Shared test set-up: the `gpu` marker and helpers that build the same
seeded mesh in the CUDA library, the oracle and the reference."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def build_cpu(factory, n, seed=0, pert=0.1, size=None, radial=None,
              fields=False, parallel=False):
    """A classified full-topology box in a CPU checker (oracle or reference),
    built the way the reference's tests do (test_warp_3d.cpp:115-119)."""
    from oracle import oracle as O
    coords, conn, center = O.box(n, seed, pert)
    m = factory(3, coords, conn)
    m.derive_model_full()
    nv = coords.size // 3
    if radial is not None:
        h = O.radial_size(coords, center, radial[0], radial[1])
    else:
        h = np.full(nv, 0.05 if size is None else size)
    m.add_field(0, "adapt_size", h)
    if fields:
        add_fields(m, seed)
    if parallel:
        m.make_parallel()
    return m


def add_fields(m, seed):
    """A conserved, a pointwise and an untransferred field, seeded."""
    from oracle import oracle as O
    rng = np.random.default_rng(seed + 1000)
    nt, nv = m.count(3), m.count(0)
    m.add_field(3, "mass", rng.random(nt), 1, O.X_CONSERVE)
    m.add_field(3, "pointwise", rng.random(nt * 3), 3, O.X_POINTWISE)
    m.add_field(0, "dye", rng.random(nv), 1, O.X_NOT)


def build_gpu(n, seed=0, pert=0.1, size=None, radial=None, fields=False,
              parallel=False):
    import omega_h_v1_b200 as G
    coords, conn, center = G.box(n, seed, pert)
    m = G.Mesh.reduced(3, coords, conn)
    m.derive_model_full()
    nv = coords.size // 3
    if radial is not None:
        h = radial_size_np(coords, center, radial[0], radial[1])
    else:
        h = np.full(nv, 0.05 if size is None else size)
    m.add_field(0, "adapt_size", h)
    if fields:
        add_fields(m, seed)
    if parallel:
        m.make_parallel()
    return m


def radial_size_np(coords, center, h0, h1):
    """h0 + h1 |x - c|, evaluated in the oracle's operation order."""
    d = coords.reshape(-1, 3) - center
    return h0 + h1 * np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])


def vertex_field(m, name):
    for t in m.tags(0):
        if t.name == name:
            return t.data
    return None


def front_warp_run(m, steps=2, angle=0.25, weight=4e-4, min_h=0.04, max_h=0.2,
                   warp_floor=0.2, adapt=True):
    """The reference's warp-test flow (test_warp.cpp:70-98) at test sizes on
    any of the three implementations: a tanh front carried as the vertex
    field "dye", its recovered-Hessian size field, mesh_adapt, then warp
    steps (rotation field, warp_to_limit, new size field, adapt until the
    warp is used up). Returns the warp_to_limit results."""
    from omega_h_v1_b200 import workloads as W
    m.add_field(0, "dye", W.front_field(vertex_field(m, "coordinates")))
    W.hessian_size_field(m, weight=weight, min_h=min_h, max_h=max_h)
    if adapt:
        m.adapt(1 / 3., 0.3, 4, 50)
    oks = []
    for _ in range(steps):
        m.add_field(0, "warp", W.rotation_warp(vertex_field(m, "coordinates"), angle), 3)
        for _ in range(3):
            ok = m.warp_to_limit(warp_floor)
            oks.append(ok)
            W.hessian_size_field(m, weight=weight, min_h=min_h, max_h=max_h)
            if adapt:
                m.adapt(1 / 3., 0.3, 4, 50)
            if ok:
                break
        m.free_tag(0, "warp")
    return oks
