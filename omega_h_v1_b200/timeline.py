"""Device timeline of mesh_adapt: where the time between kernels goes.

    python -m omega_h_v1_b200.timeline [--n 48] [--trace PATH]

Adapts resident copies of a seeded n^3 box with the radial size field
h = 0.01 + 0.04 |x - c| (four warm-up adapts, then two recorded ones) on the
legacy default stream, records the device activity with torch.profiler
(CUPTI), and prints for each recorded adapt: its span, the device's busy
time, kernel count and time, and the idle gaps attributed to the operation
before each gap (a kernel, a memset, a copy; a gap after a device-to-host
read is the host waiting on its read-back), with the kernels that took the
most time. --trace also writes the Chrome trace.
"""
import argparse
import collections
import ctypes as C
import json
import os
import sys
import tempfile


def _gaps(path, top):
    d = json.load(open(path))
    ev = d["traceEvents"] if isinstance(d, dict) else d
    gpu = [e for e in ev if e.get("ph") == "X" and e.get("cat") in ("kernel", "gpu_memcpy",
                                                                    "gpu_memset")]
    gpu.sort(key=lambda e: e["ts"])
    ts = [(e["ts"], e["ts"] + e["dur"], e["name"], e["cat"]) for e in gpu]
    # the two recorded adapts, split at the marker kernel run between them
    # (a fill of torch's), else at the largest gap between operations
    marks = [i for i, t in enumerate(ts) if t[3] == "kernel" and "FillFunctor" in t[2]]
    if marks:
        parts = (ts[:marks[0]], ts[marks[0] + 1:])
    else:
        gaps = [(ts[i + 1][0] - ts[i][1], i) for i in range(len(ts) - 1)]
        cut = max(gaps)[1] + 1
        parts = (ts[:cut], ts[cut:])
    for part in parts:
        t0, t1 = part[0][0], part[-1][1]
        busy = sum(b - a for a, b, _, _ in part)
        kern = sum(b - a for a, b, _, c in part if c == "kernel")
        nk = sum(1 for p in part if p[3] == "kernel")
        print("adapt: span %.3f ms, busy %.3f ms, kernels %.3f ms in %d, %d copies/memsets"
              % ((t1 - t0) / 1e3, busy / 1e3, kern / 1e3, nk, len(part) - nk))
        after = collections.defaultdict(float)
        cnt = collections.Counter()
        for i in range(len(part) - 1):
            g = part[i + 1][0] - part[i][1]
            key = part[i][2][:30] if part[i][3] == "gpu_memcpy" else part[i][3]
            after[key] += g
            cnt[key] += 1
        for k, v in sorted(after.items(), key=lambda kv: -kv[1])[:6]:
            print("  gap after %-32s %8.3f ms over %4d (mean %.1f us)"
                  % (k, v / 1e3, cnt[k], v / cnt[k]))
        byk = collections.defaultdict(float)
        kc = collections.Counter()
        for a, b, n, c in part:
            if c == "kernel":
                name = n.split("(")[0]
                byk[name] += b - a
                kc[name] += 1
        for n, v in sorted(byk.items(), key=lambda kv: -kv[1])[:top]:
            print("    %-48s %4d %8.3f ms" % (n[:48], kc[n], v / 1e3))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=48)
    ap.add_argument("--trace", default=None, help="also keep the Chrome trace here")
    ap.add_argument("--top", type=int, default=15)
    args = ap.parse_args(argv)
    import numpy as np
    import torch
    from torch.profiler import ProfilerActivity, profile
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    import omega_h_v1_b200 as G
    L = G.lib()
    torch.cuda.set_device(0)
    coords, conn, center = G.box(args.n, 0, 0.1)
    base = G.Mesh.reduced(3, coords, conn)
    base.derive_model_full()
    dd = coords.reshape(-1, 3) - center
    base.add_field(0, "adapt_size", 0.01 + 0.04 * np.sqrt(dd[:, 0] * dd[:, 0] +
                                                           dd[:, 1] * dd[:, 1] +
                                                           dd[:, 2] * dd[:, 2]))
    hs = []
    for _ in range(6):
        h = L.osh_b200_clone(base.h)
        G.check()
        L.osh_b200_set_stream(h, C.c_void_p(0))
        hs.append(h)
    torch.cuda.synchronize()
    for i in range(4):
        L.osh_adapt(hs[i], 1 / 3., 0.3, 4, 50)
        G.check()
        L.osh_free(hs[i])
    marker = torch.zeros(1, device="cuda")
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CPU, ProfilerActivity.CUDA]) as prof:
        for i in range(4, 6):
            L.osh_adapt(hs[i], 1 / 3., 0.3, 4, 50)
            G.check()
            torch.cuda.synchronize()
            L.osh_free(hs[i])
            if i == 4:
                marker.fill_(1.0)  # the boundary between the two adapts
                torch.cuda.synchronize()
    path = args.trace or os.path.join(tempfile.mkdtemp(), "trace.json")
    prof.export_chrome_trace(path)
    _gaps(path, args.top)
    base.close()


if __name__ == "__main__":
    main()
