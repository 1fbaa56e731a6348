"""Benchmark of the B200 mesh-adaptation pass (libosh_b200.so).

Workload: the 48^3 unit-cube box (663,552 tets, 6 per hex), interior
vertices perturbed by up to 0.1 h0, isotropic size h(x) = 0.01 + 0.04 |x - c|
with c drawn from the seeded stream, adapted by mesh_adapt(1/3, 0.3, 4, 50)
to convergence. A step is one full mesh_adapt of that input.

Metric: adapted tets/s = (elements entering every pass that changed the mesh,
summed) / (time of those adapt calls). `value` times K steps back to back on
meshes already resident in HBM (one prepared copy per step), with CUDA events
on the stream the library launches on, bracketed by a barrier and a device
synchronise. `e2e` times the same work through the C ABI from pinned host
buffers: osh_new / osh_build_ents / fields / labels uploaded, osh_adapt, and
the adapted tets and coordinates read back, every step.

--impl reference times the reference's own OpenMP build (compiled from its
sources by oracle/Makefile) on the host cores, on the same workload.

Multi-GPU: one mesh per rank (replicas only; a single mesh does not shard);
value = all ranks' tets / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import signal
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "adapted tets/s per refine+coarsen+swap pass"
UNIT = "tets/s"
N_BOX = 48
H0, H1 = 0.01, 0.04
SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS = 1.0 / 3.0, 0.3, 4, 50
L2_BYTES = 126 * 2 ** 20
# DRAM bytes (read + write) per launch of a probed kernel over one adapt of
# this workload, measured by ncu and recorded with the command that measured
# them in profiles/traffic.json; None where no capture exists
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "traffic.json")


def recorded_traffic(probe):
    try:
        with open(TRAFFIC_FILE) as f:
            rec = json.load(f).get(probe)
        return (float(rec["bytes_per_launch"]), rec.get("command")) if rec else (None, None)
    except (OSError, ValueError, KeyError, TypeError):
        return None, None
# the kernel whose roofline the bench line reports: the fill of the carried
# upward rows of edges and faces, the largest single kernel of the adapt
# after the label copies (one launch per carried pair and pass)
DEFAULT_PROBE = "carry_up_fill"


def workload_config():
    return {"workload": "box48_radial_size_mesh_adapt", "box_n": N_BOX,
            "tets_in": 6 * N_BOX ** 3, "size_field": "0.01+0.04|x-c|, c~U[0.3,0.7]^3 seed 0",
            "adapt": "mesh_adapt(1/3, 0.3, 4, 50)", "parallelism": "replicas",
            "l2": "inputs larger than L2: each step adapts its own resident copy and "
                  "grows it to ~2.3M tets (>500 MB of connectivity and adjacency)"}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device):
        self.p = None
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(device),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.send_signal(signal.SIGTERM)
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)

def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(x, world, op):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, world):
    """Step times are the slowest rank's (replicas finish independently)."""
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.MAX) if world > 1 else x


def sum_over_ranks(x, world):
    """Work units add up over the replicas."""
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.SUM) if world > 1 else x


def replica_throughput(units_local, ms_local, world):
    """Whole-job throughput of independent replicas: all ranks' units over
    the slowest rank's time."""
    ms = max_over_ranks(ms_local, world)
    units = sum_over_ranks(units_local, world)
    return units / (ms / 1e3), ms, units


# ---------------------------------------------------------------------------
# our arm

def build_input(G):
    """The config's classified full-topology box with its size field, on the
    GPU (input preparation, not timed)."""
    coords, conn, center = G.box(N_BOX, 0, 0.1)
    m = G.Mesh.reduced(3, coords, conn)
    m.derive_model_full()
    d = coords.reshape(-1, 3) - center
    h = H0 + H1 * np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    m.add_field(0, "adapt_size", h)
    return m


def host_input(m):
    """Host copies of everything the C API needs to rebuild the input."""
    snap = m.snapshot()
    arrays = {"conn": {d: np.ascontiguousarray(snap.conn[d]) for d in snap.conn},
              "counts": snap.counts, "tags": {}}
    for d in range(4):
        arrays["tags"][d] = [(t.name, t.type, t.ncomps, t.transfer,
                              np.ascontiguousarray(t.data)) for t in snap.tags[d]]
    return arrays


def pin(a):
    """A page-locked copy of a numpy array (cudaHostAlloc through torch)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t


def e2e_step(G, L, inp, stream_ptr):
    """One adapt through the public C ABI from pinned host buffers: the
    uploads and the result's read-back queued on the mesh's stream
    (osh_b200_copy_to_*_async), all inside the timed region."""
    h2d = 0
    m = L.osh_new(3)
    G.check()
    L.osh_b200_set_stream(m, C.c_void_p(stream_ptr))
    G.check()
    nv = inp["counts"][0]
    L.osh_build_ents(m, 0, nv)
    for d in (1, 2, 3):
        arr = inp["pinned_conn"][d]
        p = L.osh_build_ents(m, d, inp["counts"][d])
        L.osh_b200_copy_to_device_async(m, p, C.c_void_p(arr.data_ptr()), arr.numel() * 4)
        h2d += arr.numel() * 4
    for d in range(4):
        for (name, ty, nc, tr, _), arr in zip(inp["tags"][d], inp["pinned_tags"][d]):
            if ty == G.T_F64:
                p = L.osh_new_field(m, d, name.encode(), nc, tr)
            else:
                p = L.osh_new_label(m, d, name.encode(), nc)
            nbytes = arr.numel() * arr.element_size()
            L.osh_b200_copy_to_device_async(m, p, C.c_void_p(arr.data_ptr()), nbytes)
            h2d += nbytes
    G.check()
    L.osh_adapt(m, SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS)
    G.check()
    passes, elems = C.c_uint(), C.c_double()
    L.osh_b200_adapt_stats(C.byref(passes), C.byref(elems))
    nt = L.osh_count(m, 3)
    nvo = L.osh_count(m, 0)
    # the result read into pinned host buffers (grown when a step needs more)
    import torch
    if inp.get("out_conn") is None or inp["out_conn"].numel() < nt * 4:
        inp["out_conn"] = torch.empty(nt * 4, dtype=torch.int32, pin_memory=True)
    if inp.get("out_x") is None or inp["out_x"].numel() < nvo * 3:
        inp["out_x"] = torch.empty(nvo * 3, dtype=torch.float64, pin_memory=True)
    L.osh_b200_copy_to_host_async(m, C.c_void_p(inp["out_conn"].data_ptr()),
                                  L.osh_down(m, 3, 0), nt * 4 * 4)
    L.osh_b200_copy_to_host_async(m, C.c_void_p(inp["out_x"].data_ptr()), L.osh_coords(m),
                                  nvo * 3 * 8)
    L.osh_b200_synchronize(m)
    G.check()
    d2h = nt * 4 * 4 + nvo * 3 * 8
    L.osh_free(m)
    return elems.value, h2d, d2h


def run_ours(args, world, rank, local):
    import torch
    import omega_h_v1_b200 as G
    torch.cuda.set_device(local)
    L = G.lib()
    # the library works on the legacy default stream here, so events recorded
    # on it bracket every launch and copy of the timed region
    stream = torch.cuda.default_stream()
    stream_ptr = 0
    base = build_input(G)
    tets_in = base.count(3)
    nsteps = args.warmup + args.steps
    # one resident copy per step, prepared before timing
    copies = []
    for _ in range(nsteps):
        h = L.osh_b200_clone(base.h)
        G.check()
        L.osh_b200_set_stream(h, C.c_void_p(stream_ptr))
        copies.append(h)
    torch.cuda.synchronize()
    elems = []

    def adapt(h):
        L.osh_adapt(h, SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS)
        G.check()
        passes, e = C.c_uint(), C.c_double()
        L.osh_b200_adapt_stats(C.byref(passes), C.byref(e))
        return e.value, passes.value

    for i in range(args.warmup):
        adapt(copies[i])
        L.osh_free(copies[i])
    torch.cuda.synchronize()
    # the probe of the dominant kernel runs live inside the timed region
    names = [L.osh_b200_probe_name(i).decode() for i in range(L.osh_b200_probe_count())]
    if args.probe not in names:
        raise SystemExit("unknown probe %r (have %s)" % (args.probe, ", ".join(names)))
    probe_id = names.index(args.probe)
    L.osh_b200_probe_reset()
    L.osh_b200_probe_enable(1 << probe_id)
    launches0 = L.osh_b200_launch_count()
    syncs0 = L.osh_b200_sync_count()
    clocks = Clocks(local)
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    npass = []
    for i in range(args.warmup, nsteps):
        # a step adapts its resident copy and releases the result (as the
        # warm-up steps did), so the device pool holds one step's memory
        e, p = adapt(copies[i])
        L.osh_free(copies[i])
        elems.append(e)
        npass.append(p)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    launches = L.osh_b200_launch_count() - launches0
    syncs = L.osh_b200_sync_count() - syncs0
    L.osh_b200_probe_enable(0)
    ms_local = ev0.elapsed_time(ev1)
    plaunch, pms, pbytes = C.c_uint(), C.c_double(), C.c_double()
    L.osh_b200_probe_read(probe_id, C.byref(plaunch), C.byref(pms), C.byref(pbytes))
    value, ms, units = replica_throughput(float(sum(elems)), ms_local, world)

    e2e = None
    if not args.no_e2e:
        e2e = e2e_leg(G, L, base, args, world, stream, stream_ptr)
    fp32 = None
    if not args.no_fp32:
        fp32 = fp32_leg(G, L, base, args, world, stream, stream_ptr, ms_local)
    peak, peak_kind = measured_peak()
    roof = None
    if plaunch.value:
        avg_ms = pms.value / plaunch.value
        avg_bytes = pbytes.value / plaunch.value
        achieved = avg_bytes / (avg_ms / 1e3) / 1e9
        traffic, traffic_cmd = recorded_traffic(args.probe)
        if args.traffic is not None:
            traffic, traffic_cmd = args.traffic, "--traffic"
        roof = {"bound": "hbm", "kernel": L.osh_b200_probe_name(probe_id).decode(),
                "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "launches": plaunch.value, "avg_launch_us": round(avg_ms * 1e3, 2),
                "algorithmic_bytes_per_launch": round(avg_bytes),
                "bytes_rule": "each array read once and each output written once per "
                              "launch: same_l and the old offsets 8(rows+1), the old "
                              "rows' highs and directions 8 uses, the highs' new ids "
                              "4 highs, the new offsets 4(rows+1), the kept uses "
                              "written as highs and directions 8 kept, and per use "
                              "of the entities the pass made (filled in the same "
                              "launch) its low, the row's count and the use written 20",
                "traffic": traffic,
                "dram_frac": (round(traffic / (avg_ms / 1e3) / 1e9 / peak, 4)
                              if traffic else None),
                "traffic_source": traffic_cmd}
    base.close()
    return {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 48^3 box, radial size field)",
        "config": workload_config(),
        "roofline": roof,
        "e2e": e2e,
        "fp32_filter": fp32,
        "gpu_launches": int(launches),
        "per_adapt": {"launches": round(launches / args.steps, 1),
                      "host_waits": round(syncs / args.steps, 1)},
        "clocks": clk,
        "tets_in": tets_in,
        "passes_per_step": npass[0] if npass else None,
    }


def fp32_leg(G, L, base, args, world, stream, stream_ptr, plain_ms):
    """The same adapts with the single-precision filter (candidate lengths
    and qualities decided on an FP32 estimate with an error bound, FP64
    recheck near every threshold), timed the same way after the plain leg;
    the adapted mesh's device digest must equal the plain path's."""
    import torch
    def fresh(filt):
        h = L.osh_b200_clone(base.h)
        G.check()
        L.osh_b200_set_stream(h, C.c_void_p(stream_ptr))
        L.osh_b200_set_fp32_filter(h, 1 if filt else 0)
        return h
    digests = []
    for filt in (False, True):
        h = fresh(filt)
        L.osh_adapt(h, SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS)
        G.check()
        digests.append(L.osh_b200_digest(h))
        L.osh_free(h)
    copies = [fresh(True) for _ in range(args.steps)]
    L.osh_b200_fp32_stats_reset()
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    units = 0.0
    for h in copies:
        L.osh_adapt(h, SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS)
        G.check()
        passes, e = C.c_uint(), C.c_double()
        L.osh_b200_adapt_stats(C.byref(passes), C.byref(e))
        units += e.value
        L.osh_free(h)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms_local = e0.elapsed_time(e1)
    value, ms, _ = replica_throughput(units, ms_local, world)
    fs = G.fp32_stats(reset=True)
    # one more adapt, untimed, in audit mode: every decision taken on an
    # estimate taken again in double, every estimate checked against its bound
    G.set_fp32_audit(True)
    h = fresh(True)
    L.osh_adapt(h, SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS)
    G.check()
    audited_digest = L.osh_b200_digest(h)
    L.osh_free(h)
    au = G.fp32_audit_stats()
    fa = G.fp32_stats(reset=True)
    G.set_fp32_audit(False)
    return {"value": round(value, 1), "unit": UNIT, "ms_per_step": round(ms / args.steps, 3),
            "vs_plain_fp64": round(plain_ms / ms_local, 3),
            "identical_to_plain": bool(digests[0] == digests[1] == audited_digest),
            "decided_single": fs["decided"], "rechecked_double": fs["rechecked"],
            "audit": {"decisions_audited": au["audited"], "flips": au["flips"],
                      "estimates_checked": au["checked"],
                      "bound_exceeded": fa["bound_exceeded"],
                      "max_fp32_quality_error": fa["max_error"]}}


def e2e_leg(G, L, base, args, world, stream, stream_ptr):
    """End to end through the C ABI from pinned host memory."""
    import torch
    inp = host_input(base)
    inp["pinned_conn"] = {d: pin(inp["conn"][d]) for d in (1, 2, 3)}
    inp["pinned_tags"] = {d: [pin(t[4]) for t in inp["tags"][d]] for d in range(4)}
    for _ in range(max(1, min(args.warmup, 1))):
        e2e_step(G, L, inp, stream_ptr)
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e_units, h2d, d2h = 0.0, 0, 0
    for _ in range(args.steps):
        u, a, b = e2e_step(G, L, inp, stream_ptr)
        e_units += u
        h2d, d2h = a, b
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    e_units = sum_over_ranks(e_units, world)
    return {"value": round(e_units / (e_ms / 1e3), 1), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": round(e_ms / args.steps, 3)}


# ---------------------------------------------------------------------------
# batched workload: 512 box meshes of uneven sizes

BATCH_CHUNK_EST_TETS = 60e6     # estimated output tets per adapt_batch call
BATCH_UNION_ELEMS = 1000000     # current elements per union inside a call
CONCURRENT_THREADS = 4   # host threads (streams) of the concurrent leg


def reserve_pool(G, fraction=0.5):
    """Grow the library's device memory pool up front (input preparation, not
    timed), as a long-running service would, so that growing meshes do not
    pay for pool growth inside their passes; returns the bytes reserved."""
    import torch
    free, _ = torch.cuda.mem_get_info()
    nbytes = int(fraction * free)
    G.pool_reserve(nbytes)
    G.pool_stats(reset_high=True)
    return nbytes


def batch_times(L):
    c, p, s = C.c_double(), C.c_double(), C.c_double()
    L.osh_b200_batch_times(C.byref(c), C.byref(p), C.byref(s))
    return {"concat": round(c.value, 3), "passes": round(p.value, 3), "split": round(s.value, 3)}


def batched_chunks(jobs):
    """Jobs in ascending input size, cut into calls of about
    BATCH_CHUNK_EST_TETS estimated output tets (bounds the memory held)."""
    order = sorted(range(len(jobs)), key=lambda i: (jobs[i].tets, i))
    chunks, cur, est = [], [], 0.0
    for i in order:
        e = jobs[i].estimated_output_tets()
        if cur and est + e > BATCH_CHUNK_EST_TETS:
            chunks.append(cur)
            cur, est = [], 0.0
        cur.append(i)
        est += e
    if cur:
        chunks.append(cur)
    return chunks


def run_batched(args, world, rank, local, cpu_sample=True):
    """512 meshes adapted one by one (plain FP64 path) and together
    (adapt_batch, and concurrent streams), same inputs, same call order;
    every mesh's result must have the same device digest in every leg. On N
    GPUs the meshes are placed whole by greedy bin packing on estimated
    output tets (no data-path exchange): each leg's value is all ranks'
    elements over the slowest rank's time."""
    import torch
    import omega_h_v1_b200 as G
    from omega_h_v1_b200 import workloads as W
    torch.cuda.set_device(local)
    L = G.lib()
    stream = torch.cuda.default_stream()
    all_jobs = W.batched_boxes(args.batch_count, seed=1, nmax=args.batch_nmax)
    mine = W.place_jobs(all_jobs, world)[rank] if world > 1 else list(range(len(all_jobs)))
    jobs = [all_jobs[i] for i in mine]
    reserve_pool(G)
    t0 = time.perf_counter()
    bases = [W.build_job_mesh(G, j) for j in jobs]
    prep_s = time.perf_counter() - t0
    chunks = batched_chunks(jobs)

    def clones(fp32=False):
        out = []
        for b in bases:
            h = L.osh_b200_clone(b.h)
            G.check()
            L.osh_b200_set_stream(h, C.c_void_p(0))
            L.osh_b200_set_fp32_filter(h, 1 if fp32 else 0)
            out.append(h)
        return out

    def plain_leg(hs, idx):
        digests, elems = {}, 0.0
        for i in idx:
            L.osh_adapt(hs[i], SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS)
            G.check()
            p, e = C.c_uint(), C.c_double()
            L.osh_b200_adapt_stats(C.byref(p), C.byref(e))
            elems += e.value
            digests[i] = L.osh_b200_digest(hs[i])
            L.osh_free(hs[i])
        return digests, elems

    batch_secs = {}

    def batch_leg(hs, chunk_list):
        batch_secs.clear()
        digests, elems, unions, upasses = {}, 0.0, 0, 0
        for idx in chunk_list:
            arr = (C.c_void_p * len(idx))(*[hs[i] for i in idx])
            rc = L.osh_b200_adapt_batch(arr, len(idx), SIZE_FLOOR, GOOD_QUAL, NLAYERS,
                                        MAX_OPS, BATCH_UNION_ELEMS, None, None)
            if rc:
                G.check()
            u, st, up, mp = (C.c_uint() for _ in range(4))
            e = C.c_double()
            L.osh_b200_batch_stats(C.byref(u), C.byref(st), C.byref(up), C.byref(mp),
                                   C.byref(e))
            elems += e.value
            unions += u.value
            upasses += up.value
            for k, v in batch_times(L).items():
                batch_secs[k] = round(batch_secs.get(k, 0.0) + v, 3)
            for i in idx:
                digests[i] = L.osh_b200_digest(hs[i])
                L.osh_free(hs[i])
        return digests, elems, unions, upasses

    def concurrent_leg(hs, chunk_list, nthreads=CONCURRENT_THREADS):
        digests, elems = {}, 0.0
        for idx in chunk_list:
            arr = (C.c_void_p * len(idx))(*[hs[i] for i in idx])
            rc = L.osh_b200_adapt_concurrent(arr, len(idx), SIZE_FLOOR, GOOD_QUAL, NLAYERS,
                                             MAX_OPS, nthreads, 0, None, None)
            if rc:
                G.check()
            for k, i in enumerate(idx):
                p, e = C.c_uint(), C.c_double()
                L.osh_b200_batch_mesh_stats(k, C.byref(p), C.byref(e))
                elems += e.value
                digests[i] = L.osh_b200_digest(hs[i])
                L.osh_free(hs[i])
        return digests, elems

    # warm-up on the smallest meshes through both paths (untimed)
    warm = chunks[0][:16]
    hs = clones()
    plain_leg(hs, warm)
    for i in range(len(hs)):
        if i not in warm:
            L.osh_free(hs[i])
    hs = clones()
    batch_leg(hs, [warm])
    for i in range(len(hs)):
        if i not in warm:
            L.osh_free(hs[i])
    hs = clones()
    concurrent_leg(hs, [warm])
    for i in range(len(hs)):
        if i not in warm:
            L.osh_free(hs[i])
    order = [i for c in chunks for i in c]

    def timed(fn):
        torch.cuda.synchronize()
        barrier(world)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1)

    hs = clones()
    torch.cuda.synchronize()
    launches0 = L.osh_b200_launch_count()
    (pd, pe), plain_ms = timed(lambda: plain_leg(hs, order))
    plain_launches = L.osh_b200_launch_count() - launches0
    hs = clones()
    torch.cuda.synchronize()
    (bd64, be64, _, _), batch64_ms = timed(lambda: batch_leg(hs, chunks))
    secs64 = dict(batch_secs)
    # concurrent streams, double and with the filter
    hs = clones()
    torch.cuda.synchronize()
    (cd64, ce64), conc64_ms = timed(lambda: concurrent_leg(hs, chunks))
    hs = clones(fp32=True)
    torch.cuda.synchronize()
    (cd32, ce32), conc32_ms = timed(lambda: concurrent_leg(hs, chunks))
    # the batched path with the single-precision filter (double recheck)
    hs = clones(fp32=True)
    torch.cuda.synchronize()
    L.osh_b200_fp32_stats_reset()
    clocks = Clocks(local)
    launches0 = L.osh_b200_launch_count()
    (bd, be, unions, upasses), batch_ms = timed(lambda: batch_leg(hs, chunks))
    batch_launches = L.osh_b200_launch_count() - launches0
    clk = clocks.stop()
    fs = G.fp32_stats()
    same = all(pd[i] == bd[i] == bd64[i] for i in range(len(jobs)))
    same_conc = all(pd[i] == cd64[i] == cd32[i] for i in range(len(jobs)))
    for b in bases:
        b.close()
    # whole-job figures: every rank's elements over the slowest rank's time
    # (each rank took the same collective steps, in this order)
    pe, plain_ms = sum_over_ranks(pe, world), max_over_ranks(plain_ms, world)
    be64, batch64_ms = sum_over_ranks(be64, world), max_over_ranks(batch64_ms, world)
    ce64, conc64_ms = sum_over_ranks(ce64, world), max_over_ranks(conc64_ms, world)
    ce32, conc32_ms = sum_over_ranks(ce32, world), max_over_ranks(conc32_ms, world)
    be, batch_ms = sum_over_ranks(be, world), max_over_ranks(batch_ms, world)
    same = sum_over_ranks(0.0 if same else 1.0, world) == 0.0
    same_conc = sum_over_ranks(0.0 if same_conc else 1.0, world) == 0.0
    value = be / (batch_ms / 1e3)
    plain_value = pe / (plain_ms / 1e3)
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": 1, "warmup": 1, "ms_per_step": round(batch_ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded box meshes, uniform size fields)",
        "config": {"workload": "batched_%d_boxes_n4_%d" % (len(all_jobs), args.batch_nmax),
                   "meshes": len(all_jobs),
                   "placement": ("greedy bin packing on estimated output tets, %d meshes "
                                 "on rank 0" % len(jobs)) if world > 1 else "one GPU",
                   "n": "log-uniform in [4,%d], seed 1" % args.batch_nmax,
                   "size": "U[0.3/n, 1.5/n]",
                   "tets_in": int(sum(j.tets for j in all_jobs)),
                   "adapt": "mesh_adapt(1/3, 0.3, 4, 50) of every mesh",
                   "calls": len(chunks), "union_input_elems": BATCH_UNION_ELEMS,
                   "l2": "inputs larger than L2 (26M tets in, hundreds of M out)"},
        "path": "batched, single-precision filter with double recheck",
        "plain": {"value": round(plain_value, 1), "ms": round(plain_ms, 3),
                  "gpu_launches": int(plain_launches),
                  "path": "one mesh_adapt per mesh, double"},
        "batched_fp64": {"value": round(be64 / (batch64_ms / 1e3), 1),
                         "ms": round(batch64_ms, 3), "union_secs": secs64},
        "concurrent_fp64": {"value": round(ce64 / (conc64_ms / 1e3), 1),
                            "ms": round(conc64_ms, 3), "threads": CONCURRENT_THREADS,
                            "speedup_vs_plain": round(plain_ms / conc64_ms, 3),
                            "path": "osh_b200_adapt_concurrent: unchanged mesh_adapt per "
                                    "mesh, host threads on streams of their own"},
        "concurrent_fp32": {"value": round(ce32 / (conc32_ms / 1e3), 1),
                            "ms": round(conc32_ms, 3), "threads": CONCURRENT_THREADS,
                            "speedup_vs_plain": round(plain_ms / conc32_ms, 3),
                            "path": "concurrent streams with the single-precision filter"},
        "identical_concurrent": bool(same_conc and abs(pe - ce64) < 0.5
                                     and abs(pe - ce32) < 0.5),
        "speedup_vs_plain": round(plain_ms / batch_ms, 3),
        "identical_to_plain": bool(same and abs(pe - be) < 0.5 and abs(pe - be64) < 0.5),
        "fp32": {"decided_single": fs["decided"], "rechecked_double": fs["rechecked"],
                 "max_quality_error": fs["max_error"],
                 "bound_exceeded": fs["bound_exceeded"]},
        "elems_in": be, "unions": unions, "union_passes": upasses,
        "union_secs": batch_secs,
        "gpu_launches": int(batch_launches), "clocks": clk,
        "prep_s": round(prep_s, 1),
        "device_peak_bytes": G.pool_stats()["peak"],
    }
    if cpu_sample and not args.no_cpu and rank == 0:
        out["cpu_baseline"] = batched_cpu_sample(jobs)
    return out


def batched_summary(b):
    """The 512-box legs in the headline line: whole-job tets/s of each path,
    the best many-mesh path against one mesh_adapt after another, and
    whether every mesh ended identical in every leg."""
    legs = {"plain_fp64": b["plain"]["value"], "union_fp64": b["batched_fp64"]["value"],
            "union_fp32": b["value"], "concurrent_fp64": b["concurrent_fp64"]["value"],
            "concurrent_fp32": b["concurrent_fp32"]["value"]}
    best = max((k for k in legs if k != "plain_fp64"), key=lambda k: legs[k])
    return {"workload": b["config"]["workload"], "meshes": b["config"]["meshes"],
            "tets_in": b["config"]["tets_in"], "elems_in": b["elems_in"],
            "unit": UNIT, "legs": legs,
            "ms": {"plain_fp64": b["plain"]["ms"], "union_fp64": b["batched_fp64"]["ms"],
                   "union_fp32": b["ms_per_step"], "concurrent_fp64": b["concurrent_fp64"]["ms"],
                   "concurrent_fp32": b["concurrent_fp32"]["ms"]},
            "best_path": best, "vs_plain": round(legs[best] / legs["plain_fp64"], 3),
            "union_fp32_vs_plain": b["speedup_vs_plain"],
            "identical_to_plain": bool(b["identical_to_plain"] and b["identical_concurrent"]),
            "fp32": b["fp32"], "gpu_launches_union_fp32": b["gpu_launches"],
            "placement": b["config"].get("placement"), "clocks": b["clocks"]}


def run_serving(args, world, rank, local):
    """Poisson arrivals (seed 2, args.rate per second) of box jobs with
    log-uniform tet counts, served with continuous batching; latency is each
    job's completion time minus its scheduled arrival. On N GPUs each job is
    routed on arrival to the GPU given the least estimated work so far, and
    every GPU serves its own jobs (no exchange); the latency percentiles are
    over all jobs."""
    import torch
    import omega_h_v1_b200 as G
    from omega_h_v1_b200 import workloads as W
    torch.cuda.set_device(local)
    L = G.lib()
    all_jobs = W.serving_stream(args.serve_count, seed=2, rate=args.rate)
    mine = W.route_stream(all_jobs, world)[rank] if world > 1 else list(range(len(all_jobs)))
    jobs = [all_jobs[i] for i in mine]
    inputs = [W.job_host_input(G, j) for j in jobs]
    free, total = torch.cuda.mem_get_info()
    budget = int(0.6 * free)
    reserve_pool(G)
    # warm-up: two small jobs through a throwaway server
    warm = G.Server(SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS, budget)
    small = sorted(range(len(jobs)), key=lambda i: jobs[i].tets)[:2]
    for i in small:
        warm.submit(*inputs[i])
    while warm.step() > 0:
        pass
    for i in warm.poll():
        warm.take(i).close()
    warm.close()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    launches0 = L.osh_b200_launch_count()
    sv = G.Server(SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS, budget)
    t0 = time.perf_counter() - sv.stats()["now"]   # server clock origin
    sv.start()   # the engine thread steps while this thread submits
    ids = {}
    submit_secs = 0.0
    active_samples = []
    for nxt, job in enumerate(jobs):
        wait = job.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        ts = time.perf_counter()
        ids[sv.submit(*inputs[nxt])] = nxt
        submit_secs += time.perf_counter() - ts
        active_samples.append(sv.stats()["active"])
    while sv.wait(0.05) > 0:
        active_samples.append(sv.stats()["active"])
    for j in sv.poll():
        sv.take(j).close()
    sv.stop()
    torch.cuda.synchronize()
    makespan = time.perf_counter() - t0
    clk = clocks.stop()
    launches = L.osh_b200_launch_count() - launches0
    lat, elems, tets_in = [], 0.0, 0
    for jid, i in ids.items():
        info = sv.job_info(jid)
        lat.append(info["t_done"] - jobs[i].arrival)
        elems += info["elems_in"]
        tets_in += jobs[i].tets
    st = sv.stats()
    sv.close()
    span = makespan - all_jobs[0].arrival
    if world > 1:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, lat)
        lat = [x for part in parts for x in part]
        elems = sum_over_ranks(elems, world)
        tets_in = int(sum_over_ranks(float(tets_in), world))
        span = max_over_ranks(span, world)
    lat = np.sort(np.array(lat))
    p50 = float(np.percentile(lat, 50))
    p99 = float(np.percentile(lat, 99))
    return {
        "metric": METRIC, "value": round(elems / span, 1), "unit": UNIT, "n_gpus": world,
        "steps": 1, "warmup": 1, "ms_per_step": round(span * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Poisson stream of box jobs)",
        "config": {"workload": "serving_poisson", "jobs": len(all_jobs), "rate_per_s": args.rate,
                   "routing": ("each job on arrival to the GPU given the least estimated "
                               "work so far" if world > 1 else "one GPU"),
                   "tets": "log-uniform in [2e3, 2e6] per job, seed 2",
                   "size": "half uniform U[1.0/n, 1.6/n], half the recovered Hessian of "
                           "tanh(50(x-o-0.1 sin 2 pi y)), o~U[0.3,0.7], sizes 0.5/n..2/n, "
                           "weight (2/n-0.5/n)/2000 (computed on the GPU before the stream)",
                   "tets_in": int(tets_in), "budget_bytes": budget,
                   "adapt": "mesh_adapt(1/3, 0.3, 4, 50) per job",
                   "l2": "inputs larger than L2 (hundreds of MB resident)"},
        "latency_ms": {"p50": round(p50 * 1e3, 2), "p99": round(p99 * 1e3, 2),
                       "max": round(float(lat[-1]) * 1e3, 2)},
        "mean_active_jobs": round(float(np.mean(active_samples)), 2) if active_samples else 0,
        "server_steps": st["steps"], "elems_in": elems,
        "device_peak_bytes": G.pool_stats()["peak"],
        "server_secs": {k: round(st[k], 3) for k in
                        ("secs_admit", "secs_join", "secs_passes", "secs_retire")},
        "submit_secs": round(submit_secs, 3),
        "gpu_launches": int(launches), "clocks": clk,
    }


WARP_N, WARP_STEPS, WARP_ANGLE = 96, 8, 0.5
WARP_ARGS = (1.0 / 3.0, 0.4, 0, 500)   # test_warp.cpp's floors; a pass cap the front needs
WARP_QUAL_FLOOR = 0.1


def run_warp(args, world, rank, local):
    """The anisotropic-front workload: a 96^3 box, u = tanh(50 (x - 0.5 -
    0.1 sin 2 pi y)) carried as a vertex field, adapt_size from its recovered
    Hessian (min_h 0.002, max_h 0.05), mesh_adapt, then 8 warp steps rotating
    the region within 0.5 of the axis x = y = 0.5 by 0.5 rad in total, each
    warp_to_limit (floor 0.1), new size field and mesh_adapt until the warp
    is used up. value = elements entering adapt passes / time in adapt calls."""
    import torch
    import omega_h_v1_b200 as G
    from omega_h_v1_b200 import workloads as W
    torch.cuda.set_device(local)
    L = G.lib()
    stream = torch.cuda.default_stream()
    reserve_pool(G)
    coords, conn, _ = G.box(WARP_N, 0, 0.1)
    m = G.Mesh.reduced(3, coords, conn)
    m.derive_model_full()
    L.osh_b200_set_stream(m.h, C.c_void_p(0))
    m.add_field(0, "dye", W.front_field(coords))
    tets_in = m.count(3)
    ev = []

    def adapt():
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.adapt(*WARP_ARGS)
        e1.record(stream)
        p, e = C.c_uint(), C.c_double()
        L.osh_b200_adapt_stats(C.byref(p), C.byref(e))
        ev.append((e0, e1, e.value, p.value))

    def field_xyz(name):
        p = L.osh_get_field(m.h, 0, name.encode())
        G.check()
        out = np.empty(m.count(0) * 3, np.float64)
        L.osh_b200_copy_to_host(out.ctypes.data_as(C.c_void_p), p, out.nbytes)
        return out

    clocks = Clocks(local)
    launches0 = L.osh_b200_launch_count()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    W.hessian_size_field(m)
    adapt()
    tries = []
    for _ in range(WARP_STEPS):
        m.add_field(0, "warp", W.rotation_warp(field_xyz("coordinates"),
                                               WARP_ANGLE / WARP_STEPS), 3)
        for k in range(4):
            ok = m.warp_to_limit(WARP_QUAL_FLOOR)
            W.hessian_size_field(m)
            adapt()
            if ok:
                break
        tries.append(k + 1)
        m.free_tag(0, "warp")
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    launches = L.osh_b200_launch_count() - launches0
    adapt_ms = sum(a.elapsed_time(b) for a, b, _, _ in ev)
    elems = sum(e for _, _, e, _ in ev)
    passes = sum(p for _, _, _, p in ev)
    out = {
        "metric": METRIC, "value": round(elems / (adapt_ms / 1e3), 1), "unit": UNIT,
        "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": round(adapt_ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 96^3 box, tanh front, rotation warp)",
        "config": {"workload": "front_warp_box96", "box_n": WARP_N, "tets_in": tets_in,
                   "field": "tanh(50(x-0.5-0.1 sin 2 pi y)), Hessian weight %g" %
                            W.HESSIAN_WEIGHT,
                   "min_h": W.MIN_H, "max_h": W.MAX_H, "warp_steps": WARP_STEPS,
                   "rotation_rad": WARP_ANGLE, "warp_floor": WARP_QUAL_FLOOR,
                   "adapt": "mesh_adapt(1/3, 0.4, 0, 500) after each warp",
                   "l2": "inputs larger than L2 (5.3M to 30M tets resident)"},
        "adapt_calls": len(ev), "passes": passes, "elems_in": elems,
        "tets_out": m.count(3), "warp_tries": tries, "procedure_s": round(wall, 3),
        "device_peak_bytes": G.pool_stats()["peak"],
        "gpu_launches": int(launches), "clocks": clk,
    }
    m.close()
    return out


def warp_cpu_sample():
    """The reference's OpenMP build on the front workload's first stage:
    the Hessian size field and the first mesh_adapt of the 96^3 box."""
    from oracle import oracle as O
    import omega_h_v1_b200 as G
    from omega_h_v1_b200 import workloads as W
    if not O.have_reference():
        return None
    lib = O._lib(O.REF_OMP_SO, "refd_").lib
    lib.refd_adapt_counted.restype = C.c_uint
    lib.refd_adapt_counted.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_uint,
                                       C.c_uint, C.POINTER(C.c_uint), C.POINTER(C.c_double)]
    coords, conn, _ = G.box(WARP_N, 0, 0.1)
    m = O.Reference(3, coords, conn)
    m.derive_model_full()
    m.add_field(0, "adapt_size", np.full(coords.size // 3, W.MAX_H))
    m.add_field(0, "dye", W.front_field(coords))
    p, e = C.c_uint(), C.c_double()
    with _Quiet():
        t0 = time.perf_counter()
        W.hessian_size_field(m)
        lib.refd_adapt_counted(m.h, *WARP_ARGS, C.byref(p), C.byref(e))
        secs = time.perf_counter() - t0
    m.close()
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": round(e.value / secs, 1), "unit": UNIT, "cores": cores,
            "kind": "reference",
            "sample": "size field and first mesh_adapt of the 96^3 front workload "
                      "(%d passes, %.0f tets in)" % (p.value, e.value)}


def batched_cpu_sample(jobs, budget_est_tets=12e6):
    """The reference's OpenMP mesh_adapt on the first jobs of the seeded list
    (up to budget_est_tets estimated output tets)."""
    from oracle import oracle as O
    import omega_h_v1_b200 as G
    from omega_h_v1_b200 import workloads as W
    if not O.have_reference():
        return None
    lib = O._lib(O.REF_OMP_SO, "refd_").lib
    lib.refd_adapt_counted.restype = C.c_uint
    lib.refd_adapt_counted.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_uint,
                                       C.c_uint, C.POINTER(C.c_uint), C.POINTER(C.c_double)]
    elems, secs, used, est = 0.0, 0.0, 0, 0.0
    for j in jobs:
        if est > budget_est_tets:
            break
        est += j.estimated_output_tets()
        coords, conn, h = W.job_host_input(G, j)
        m = O.Reference(3, coords, conn)
        m.derive_model_full()
        m.add_field(0, "adapt_size", h)
        p, e = C.c_uint(), C.c_double()
        with _Quiet():
            t0 = time.perf_counter()
            lib.refd_adapt_counted(m.h, SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS,
                                   C.byref(p), C.byref(e))
            secs += time.perf_counter() - t0
        m.close()
        elems += e.value
        used += 1
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": round(elems / secs, 1), "unit": UNIT, "cores": cores,
            "kind": "reference",
            "sample": "mesh_adapt of the first %d jobs of the seeded list (%.0f tets in "
                      "over their passes)" % (used, elems)}


# ---------------------------------------------------------------------------
# CPU arms (reference build of the same path)

class _Quiet:
    """Silence the reference's printf output on fd 1 while it runs."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def cpu_reference_run(nsteps_total, ntimed):
    """Times the reference's OpenMP build of mesh_adapt on the workload:
    returns (tets/s, cores, sample description, ms per step)."""
    from oracle import oracle as O
    if not O.have_reference():
        return None
    coords, conn, center = O.box(N_BOX, 0, 0.1)
    h = O.radial_size(coords, center, H0, H1)
    lib = O._lib(O.REF_OMP_SO, "refd_").lib
    lib.refd_adapt_counted.restype = C.c_uint
    lib.refd_adapt_counted.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_uint,
                                       C.c_uint, C.POINTER(C.c_uint), C.POINTER(C.c_double)]

    def fresh():
        m = O.Reference(3, coords, conn)
        m.derive_model_full()
        m.add_field(0, "adapt_size", h)
        return m

    # pass count and elements entering them (untimed)
    m = fresh()
    passes, elems = C.c_uint(), C.c_double()
    with _Quiet():
        lib.refd_adapt_counted(m.h, SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS,
                               C.byref(passes), C.byref(elems))
    m.close()
    times = []
    for i in range(nsteps_total):
        m = fresh()
        with _Quiet():
            t0 = time.perf_counter()
            m.adapt(SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS)
            t1 = time.perf_counter()
        m.close()
        if i >= nsteps_total - ntimed:
            times.append(t1 - t0)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    t = float(sum(times))
    return (elems.value * len(times) / t, cores,
            "%d full mesh_adapt runs of the 48^3 workload (%d passes, %.0f tets in)"
            % (len(times), passes.value, elems.value), 1e3 * t / len(times))


def gpu_reference_run(nadapts=2):
    """Times the reference built in its own CUDA loop mode (loop_cuda.hpp
    and Thrust, compiled for sm_100a from its sources into
    oracle/_ref/libosh_ref_cuda.so) on the same workload: returns a dict, or
    None when that build or a GPU is missing."""
    from oracle import oracle as O
    so = os.path.join(os.path.dirname(O.__file__), "_ref", "libosh_ref_cuda.so")
    if not os.path.exists(so):
        return None
    try:
        import torch
        if not torch.cuda.is_available():
            return None
    except Exception:
        return None
    L = C.CDLL(so)
    vp = C.c_void_p
    if L.refc_ready() != 0:
        return None
    L.refc_new_reduced.restype = vp
    L.refc_new_reduced.argtypes = [C.c_uint, C.c_uint, O._f64p, C.c_uint, O._u32p]
    L.refc_derive_model_full.argtypes = [vp]
    L.refc_free.argtypes = [vp]
    L.refc_add_vertex_field.argtypes = [vp, C.c_char_p, O._f64p]
    L.refc_adapt.restype = C.c_uint
    L.refc_adapt.argtypes = [vp, C.c_double, C.c_double, C.c_uint, C.c_uint]
    L.refc_adapt_counted.restype = C.c_uint
    L.refc_adapt_counted.argtypes = [vp, C.c_double, C.c_double, C.c_uint, C.c_uint,
                                     C.POINTER(C.c_uint), C.POINTER(C.c_double)]
    L.refc_count.restype = C.c_uint
    L.refc_count.argtypes = [vp, C.c_uint]
    coords, conn, center = O.box(N_BOX, 0, 0.1)
    h = O.radial_size(coords, center, H0, H1)

    def fresh():
        m = L.refc_new_reduced(3, coords.size // 3, coords, conn.size // 4, conn)
        L.refc_derive_model_full(m)
        L.refc_add_vertex_field(m, b"adapt_size", h)
        return m

    m = fresh()
    passes, elems = C.c_uint(), C.c_double()
    with _Quiet():
        L.refc_adapt_counted(m, SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS,
                             C.byref(passes), C.byref(elems))
    tets_out = L.refc_count(m, 3)
    L.refc_free(m)
    times = []
    for _ in range(nadapts):
        m = fresh()
        with _Quiet():
            t0 = time.perf_counter()
            L.refc_adapt(m, SIZE_FLOOR, GOOD_QUAL, NLAYERS, MAX_OPS)
            t1 = time.perf_counter()
        L.refc_free(m)
        times.append(t1 - t0)
    t = float(sum(times))
    return {"value": round(elems.value * len(times) / t, 1), "unit": UNIT,
            "ms_per_step": round(1e3 * t / len(times), 1), "tets_out": int(tets_out),
            "passes": passes.value,
            "build": "the reference's CUDA loop mode (loop_cuda.hpp, Thrust) compiled for "
                     "sm_100a from its own sources, NDEBUG",
            "sample": "%d full mesh_adapt runs of the 48^3 workload on one B200" % len(times)}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    r = cpu_reference_run(args.warmup + args.steps, args.steps)
    if r is None:
        return {"impl": "reference", "unavailable": "reference library not built "
                "(oracle/_ref missing; run __graft_entry__.build() where the reference is)"}
    value, cores, sample, ms = r
    return {"impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded 48^3 box, radial size field)",
            "config": workload_config(),
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "reference_gpu": None if args.no_ref_gpu else gpu_reference_run()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--probe", default=os.environ.get("OSH_BENCH_PROBE", DEFAULT_PROBE),
                    help="probe name of the kernel whose roofline is reported")
    ap.add_argument("--traffic", type=float, default=None,
                    help="DRAM bytes per launch of that kernel from an ncu capture")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling)")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own CUDA build")
    ap.add_argument("--no-fp32", action="store_true",
                    help="skip the single-precision filter leg of the box48 workload")
    ap.add_argument("--no-batched", action="store_true",
                    help="box48 workload: skip the 512-box legs (batched_cfg4 in the line)")
    ap.add_argument("--workload", default="box48",
                    choices=["box48", "batched", "serving", "warp"],
                    help="box48: the 48^3 radial-size adapt; batched: 512 uneven boxes, "
                         "plain one-by-one path against adapt_batch; serving: Poisson "
                         "stream of jobs through the continuous-batching server; warp: "
                         "96^3 tanh-front Hessian size field with 8 warp steps")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--batch-nmax", type=int, default=40,
                    help="largest grid edge of the batched boxes (40 = the full workload)")
    ap.add_argument("--serve-count", type=int, default=200)
    ap.add_argument("--rate", type=float, default=200.0)
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        out = run_reference(args, world, rank)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.workload == "batched":
        out = run_batched(args, world, rank, local)
    elif args.workload == "serving":
        out = run_serving(args, world, rank, local)
    elif args.workload == "warp":
        out = run_warp(args, world, rank, local)
    else:
        out = run_ours(args, world, rank, local)
        if not args.no_batched:
            # the many-mesh set the single-precision batched target is stated
            # on; the headline stays the 48^3 adapt, the largest workload the
            # reference arm can time step by step
            out["batched_cfg4"] = batched_summary(
                run_batched(args, world, rank, local, cpu_sample=False))
    if rank == 0:
        if not args.no_cpu and args.workload == "serving":
            from omega_h_v1_b200 import workloads as W
            out["cpu_baseline"] = batched_cpu_sample(
                W.serving_stream(args.serve_count, seed=2, rate=args.rate), 20e6)
        elif not args.no_cpu and args.workload == "warp":
            out["cpu_baseline"] = warp_cpu_sample()
        elif not args.no_cpu and args.workload == "box48":
            r = cpu_reference_run(1, 1)
            if r is not None:
                v, cores, sample, _ = r
                out["cpu_baseline"] = {"value": round(v, 1), "unit": UNIT, "cores": cores,
                                       "kind": "reference", "sample": sample}
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
