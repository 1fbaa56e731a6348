"""Regenerates the VTU fixtures (tests/golden/vtu/) with the reference's own
writer (write_mesh_vtk_opts, vtk_io.cpp:807-826), compiled into oracle/_ref/
by oracle/Makefile: `python tests/golden/make_vtu_golden.py`.

Each case is a small seeded mesh written by the reference in one format:
binary (the default build), ASCII, or zlib-compressed binary (the USE_ZLIB=1
build), plus one parallel ".pvtu" pair. The CPU tests pin the Python
restatement of the format (oracle/vtu.py) to these bytes; the GPU tests read
them with the library and write them back byte for byte.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "vtu")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from conftest import add_fields  # noqa: E402
from make_golden import Quiet  # noqa: E402
from oracle import oracle as O  # noqa: E402


def square(n, seed=0, pert=0.1):
    """n x n squares, two triangles each, interior vertices perturbed."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    xs = np.linspace(0.0, 1.0, n + 1)
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    coords = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], 1)
    inner = (X.ravel() > 0) & (X.ravel() < 1) & (Y.ravel() > 0) & (Y.ravel() < 1)
    coords[inner, :2] += rng.uniform(-pert * h, pert * h, (inner.sum(), 2))
    tris = []
    for j in range(n):
        for i in range(n):
            a, b = j * (n + 1) + i, j * (n + 1) + i + 1
            c, d = a + n + 1, b + n + 1
            tris += [(a, b, d), (a, d, c)]
    return coords.ravel(), np.array(tris, np.uint32).ravel()


def box_mesh(variant, n, seed, size, fields=False, adapt=True):
    coords, conn, _ = O.box(n, seed, 0.1)
    m = O.ReferenceVariant(3, coords, conn, variant)
    m.derive_model_full()
    m.add_field(0, "adapt_size", np.full(coords.size // 3, size))
    if fields:
        add_fields(m, seed)
    if adapt:
        with Quiet():
            m.adapt(0.3, 0.3, 4, 50)
    return m


def extra_tags(m):
    """One tag of each remaining kind: u8 on elements, u64 on edges."""
    m.add_tag(3, "region", (np.arange(m.count(3)) % 5).astype(np.uint8), O.T_U8, 1)
    m.add_tag(1, "edge_key", np.arange(m.count(1), dtype=np.uint64) * 2654435761, O.T_U64, 1)


# name -> (reference build, ascii, builder)
CASES = {
    "box2_adapt_binary.vtu": ("serial", False, lambda v: box_mesh(v, 2, 3, 0.45)),
    "box2_fields_ascii.vtu": ("serial", True, lambda v: box_mesh(v, 2, 4, 0.45, fields=True)),
    "box2_tags_zlib.vtu": ("zlib", False, lambda v: box_mesh(v, 2, 5, 0.45)),
    "box3_reduced_binary.vtu": ("serial", False, None),
    "square4_binary.vtu": ("serial", False, None),
    "square4_ascii.vtu": ("serial", True, None),
}


def build(name, variant):
    if name.startswith("box3_reduced"):
        coords, conn, _ = O.box(3, 7, 0.1)
        m = O.ReferenceVariant(3, coords, conn, variant)
        m.add_field(0, "adapt_size", np.full(coords.size // 3, 0.3))
        return m
    if name.startswith("square4"):
        coords, conn = square(4, 2)
        m = O.ReferenceVariant(2, coords, conn, variant)
        m.add_field(0, "speed", np.linspace(0.0, 1.0, coords.size // 3))
        return m
    return CASES[name][2](variant)


def main():
    os.makedirs(OUT, exist_ok=True)
    for name, (variant, ascii_, _) in CASES.items():
        m = build(name, variant)
        if name.startswith("box2_tags"):
            extra_tags(m)
        m.write_vtk(os.path.join(OUT, name), ascii=ascii_)
        print(name, os.path.getsize(os.path.join(OUT, name)))
    # a parallel mesh: "box2_parallel.pvtu" indexes the piece "box2_parallel.vtu"
    m = box_mesh("serial", 2, 6, 0.45)
    m.make_parallel()
    m.write_vtk(os.path.join(OUT, "box2_parallel.pvtu"))
    for f in ("box2_parallel.vtu", "box2_parallel.pvtu"):
        print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
