"""Tuner for the library's launch shapes (the tuning table of
libosh_b200.so: lanes per row of the long-row kernels, threads per block,
scan tile size).

    python -m omega_h_v1_b200.tune [--n 48] [--reps 5] [--out PATH]

Each key is swept in turn over its allowed values (the others held at the
best found so far) on mesh_adapt of a seeded box with a radial size field,
timed with CUDA events on the stream the library launches on; the fastest
value is kept. Every value gives the same mesh, which the run checks (the
adapted mesh's device digest must not change). The table is written as
"name value" lines to PATH (default: tuning.txt beside the library, which
the library reads when it loads).
"""
import argparse
import ctypes as C
import os
import sys


def _lib(G):
    L = G.lib()
    L.osh_b200_tuning_count.restype = C.c_uint
    L.osh_b200_tuning_name.restype = C.c_char_p
    L.osh_b200_tuning_name.argtypes = [C.c_uint]
    L.osh_b200_tuning_get.restype = C.c_int
    L.osh_b200_tuning_get.argtypes = [C.c_char_p, C.POINTER(C.c_uint)]
    L.osh_b200_tuning_set.restype = C.c_int
    L.osh_b200_tuning_set.argtypes = [C.c_char_p, C.c_uint]
    return L


# allowed values per key, as the library states them
CANDIDATES = {
    "carry_group": (4, 8, 16),
    "vert_group": (4, 8, 16),
    "indset_vert_group": (4, 8, 16),
    "indset_edge_group": (1, 2, 4, 8),
    "quality_block": (64, 128, 256, 512),
    "gather_block": (128, 256, 512),
    "scan_items": (8, 16),
    "scan_threads": (256, 512),
    "indset_blocks": (0, 1, 2, 4),
}
# keys the single-mesh sweep does not tune (they only act in the
# concurrent many-mesh driver): their allowed values
OTHER_KEYS = {
    "small_mesh_elems": (0, 25000, 50000, 100000, 200000),
}


def table(L):
    out = {}
    for i in range(L.osh_b200_tuning_count()):
        name = L.osh_b200_tuning_name(i).decode()
        v = C.c_uint()
        L.osh_b200_tuning_get(name.encode(), C.byref(v))
        out[name] = v.value
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=48, help="box edge (6 n^3 tets)")
    ap.add_argument("--reps", type=int, default=5, help="timed adapts per value")
    ap.add_argument("--out", default=None, help="table file (default: beside the library)")
    args = ap.parse_args(argv)
    import numpy as np
    import torch
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    import omega_h_v1_b200 as G
    L = _lib(G)
    torch.cuda.set_device(0)
    stream = torch.cuda.default_stream()
    coords, conn, center = G.box(args.n, 0, 0.1)
    base = G.Mesh.reduced(3, coords, conn)
    base.derive_model_full()
    d = coords.reshape(-1, 3) - center
    base.add_field(0, "adapt_size", 0.01 * 48 / args.n + 0.04 * np.sqrt((d * d).sum(1)))
    L.osh_b200_set_stream(base.h, C.c_void_p(0))

    def adapt_ms():
        hs = []
        for _ in range(args.reps + 1):
            h = L.osh_b200_clone(base.h)
            G.check()
            L.osh_b200_set_stream(h, C.c_void_p(0))
            hs.append(h)
        L.osh_adapt(hs[0], 1 / 3., 0.3, 4, 50)   # warm-up
        G.check()
        digest = L.osh_b200_digest(hs[0])
        L.osh_free(hs[0])
        times = []
        for h in hs[1:]:
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            L.osh_adapt(h, 1 / 3., 0.3, 4, 50)
            e1.record(stream)
            G.check()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            L.osh_free(h)
        return float(np.median(times)), digest

    ref_ms, ref_digest = adapt_ms()
    print("start: %.3f ms per adapt  %s" % (ref_ms, table(L)), flush=True)
    for name, values in CANDIDATES.items():
        best_v, best_ms = None, None
        for v in values:
            if L.osh_b200_tuning_set(name.encode(), v) != 0:
                continue
            ms, digest = adapt_ms()
            if digest != ref_digest:
                raise SystemExit("%s = %d changed the mesh" % (name, v))
            print("  %-18s %4d: %.3f ms" % (name, v, ms), flush=True)
            if best_ms is None or ms < best_ms:
                best_v, best_ms = v, ms
        L.osh_b200_tuning_set(name.encode(), best_v)
    final_ms, digest = adapt_ms()
    assert digest == ref_digest
    out = args.out or os.path.join(here, "tuning.txt")
    with open(out, "w") as f:
        f.write("# launch shapes for libosh_b200.so, chosen by omega_h_v1_b200/tune.py\n")
        f.write("# on %s: mesh_adapt of a %d^3 box, %.3f ms (defaults: %.3f ms)\n"
                % (torch.cuda.get_device_name(0), args.n, final_ms, ref_ms))
        for k, v in table(L).items():
            f.write("%s %d\n" % (k, v))
    print("wrote %s: %.3f ms per adapt (defaults %.3f)" % (out, final_ms, ref_ms))
    base.close()


if __name__ == "__main__":
    main()
