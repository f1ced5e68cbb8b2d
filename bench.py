"""Benchmark of the packed-Pauli hot path (one JSON line on rank 0).

Default workload (N=1): config 2 of the reference's benchmark set --
A (32,768 terms) x B (16,384 terms) on 100 qubits, k-local weight {2,3,4},
then simplify (atol=1e-12): 536,870,912 products.  Metric: products simplified
per second ("terms/s").  Other workloads: --workload commutation (config 3,
bit-packed 262,144^2 matrix), grouping (config 3, group_commuting qwc or
full), expectation (config 4, forward + gradient), batched (config 5).
Config 1 (the CPU-runnable sequence) is a parity case of the tests.

* value      device-resident throughput; each step is timed with CUDA events on
             the stream the library launches on, L2 flushed between steps;
* e2e        the same metric through the public API (wolfgang_quantum.PauliSum
             host objects: host->device upload of the operands, device->host
             read of the result inside the timed region);
* roofline   the dominant kernel of the step, from CUDA events recorded around
             each launch by the library's profiler during the timed steps;
* cpu_baseline  the reference's own C++ core (oracle/_ref, compiled from its
             sources) on a bounded sample of the same workload, 1 core.
`--impl reference` times that reference core alone as the reference arm.
Multi-GPU (torchrun): every rank runs an independent replica (the path has no
exchange step); value = all ranks' work / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def load_workloads():
    """The seeded workload generators (numpy only), loaded by file path:
    importing them as wolfgang_b200.workloads would run the package's
    __init__, which loads its native libraries -- the reference arm must not
    map any of them."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("wg_bench_workloads", ROOT / "wolfgang_b200" / "workloads.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def host_cpu() -> dict:
    """CPU model and the cores this process may run on (for every CPU baseline)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count()
    return {"cpu_model": model, "nproc": usable}


def peaks() -> tuple[float, str]:
    try:
        return float(json.loads(PEAKS_FILE.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs.  A region
    shorter than the first sample gets one sample taken right after it (the
    record then says so): a leftover clock lock or a throttle reason still
    shows there."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int) -> None:
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.after_region = False

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            if not self.lines:
                self.after_region = True
                deadline = time.time() + 2.0
                while not self.lines and time.time() < deadline and self.proc.poll() is None:
                    time.sleep(0.02)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "sampled_after_region": self.after_region}


# ---------------------------------------------------------------- distributed

def dist_setup(gpus: int, backend: str | None = None):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE / MASTER_*).

    The group only carries the barriers and the max-over-ranks timing: NCCL on
    GPU boxes, gloo where no GPU is visible (the CPU tests of this path)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    on_gpu = dist.get_backend() == "nccl"
    t = torch.tensor([value], dtype=torch.float64, device="cuda" if on_gpu else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def host_available_bytes() -> int | None:
    """MemAvailable of /proc/meminfo in bytes (None where it cannot be read)."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return None


def shard(items: list, rank: int, world: int) -> list:
    """This rank's share of independent work units (round robin): the path has
    no exchange step, so ranks split units and never communicate data."""
    return items[rank::world]


# ---------------------------------------------------------------- helpers

def pinned_d2h_bandwidth(torch, nbytes: int = 1 << 30) -> float:
    """Device-to-pinned-host copy bandwidth of this box in GB/s (best of 3
    copies of 1 GiB, CUDA events): the link that bounds an end-to-end call
    whose result comes back to the host."""
    src = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    dst = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    best = float("inf")
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del src, dst
    return nbytes / (best * 1e-3) / 1e9


def flush_l2(torch, buf):
    buf.add_(1.0)  # 512 MiB write, larger than the 126 MB L2


def dev(torch, a):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).cuda()
    return torch.from_numpy(a).cuda()


def roofline(prof: dict, bytes_per_launch: dict, peak: float, peak_kind: str, traffic: dict | None = None) -> dict:
    """Dominant kernel by total time; achieved = its algorithmic bytes per launch / mean launch time.

    traffic: measured DRAM bytes (read + write) per launch of a kernel, where an
    ncu capture exists for this workload family (scaled per item)."""
    if not prof:
        return {}
    name, (count, total_ms) = max(prof.items(), key=lambda kv: kv[1][1])
    per_launch_ms = total_ms / count
    algo_bytes = bytes_per_launch.get(name)
    out = {"kernel": name, "bound": "hbm", "unit": "GB/s", "peak": peak, "peak_source": peak_kind,
           "launches": count, "ms_per_launch": per_launch_ms, "traffic": (traffic or {}).get(name),
           "share": total_ms / sum(v[1] for v in prof.values())}
    if algo_bytes:
        achieved = algo_bytes / (per_launch_ms * 1e-3) / 1e9
        out.update(achieved=achieved, frac=achieved / peak, algorithmic_bytes=algo_bytes)
    return out


# ---------------------------------------------------------------- products (config 2)

def reference_products_sample(A, B, rows: int) -> tuple[float, int]:
    """Reference PauliSum::matmul(simplify=True) on A[:rows] x B; returns (seconds, products)."""
    from oracle import Reference

    ref = Reference()
    n, ax, az, ac = A
    _, bx, bz, bc = B
    t0 = time.perf_counter()
    ref.matmul(n, (ax[:rows], az[:rows], ac[:rows]), (bx, bz, bc), simplify=True,
               max_intermediate_terms=rows * len(bc))
    return time.perf_counter() - t0, rows * len(bc)


def products_parity(torch, L, A, B, W, ax, az, ac, bx, bz, bc, sh, span: int = 1 << 20) -> dict:
    """One more device call of the products workload, checked against the
    oracle on the key ranges of its first and last `span` survivors: those
    survivors must equal the oracle's matmul + simplify over the same ranges
    bit for bit (keys, order, coefficient bits)."""
    import ctypes as ct

    from oracle import Oracle
    from wolfgang_b200 import capi

    nl, nr = len(A[3]), len(B[3])
    dv = torch.cuda.current_device()
    ox, oz, oc, Uc = ct.c_void_p(), ct.c_void_p(), ct.c_void_p(), ct.c_size_t()
    capi.check(L.wg_pauli_products(dv, W, ax.data_ptr(), az.data_ptr(), ac.data_ptr(), nl, bx.data_ptr(),
                                   bz.data_ptr(), bc.data_ptr(), nr, capi.WG_PRODUCTS_SIMPLIFY, 1e-12, 0.0,
                                   ct.byref(ox), ct.byref(oz), ct.byref(oc), ct.byref(Uc), sh))
    U = Uc.value

    def fetch(p0, p1):
        x = np.empty((p1 - p0, W), np.uint64)
        z = np.empty((p1 - p0, W), np.uint64)
        c = np.empty(p1 - p0, np.complex128)
        for arr, ptr, size in ((x, ox, 8 * W), (z, oz, 8 * W), (c, oc, 16)):
            capi.check(L.wg_memcpy_dtoh(dv, arr.ctypes.data, ptr.value + p0 * size, arr.nbytes, sh))
        return x, z, c

    def key(x, z, i):
        k = np.zeros(2 * W, np.uint64)
        k[0::2], k[1::2] = x[i], z[i]
        return k

    orc = Oracle()
    checked, exact, worst = 0, True, 0.0
    t0 = time.perf_counter()
    for p0 in (0, max(0, U - span - 1)):
        p1 = min(U, p0 + span + 1)
        x, z, c = fetch(p0, p1)
        lo, hi = key(x, z, 0), key(x, z, len(c) - 1)  # [first, last): the range's last survivor bounds it
        want = orc.matmul_keyrange(A[0], A[1:], B[1:], lo, hi, cap=len(c))
        got = (x[:-1], z[:-1], c[:-1])
        exact = exact and all(np.ascontiguousarray(g).tobytes() == np.ascontiguousarray(w).tobytes()
                              for g, w in zip(got, want))
        if len(want[2]) == len(got[2]):
            worst = max(worst, float(np.max(np.abs(got[2] - want[2]))) if len(got[2]) else 0.0)
        checked += len(got[2])
    for q in (ox, oz, oc):
        capi.check(L.wg_free(dv, q, sh))
    return {"survivors_checked": checked, "survivors": U, "bit_exact": bool(exact), "max_abs_err": worst,
            "how": f"oracle matmul+simplify over the key ranges of the first and last {span} survivors "
                   f"({time.perf_counter() - t0:.1f} s); the whole result is checked range by range by "
                   "tests/test_gpu_fullsize.py"}


def bench_products(args, world, rank, torch) -> dict:
    from wolfgang_b200 import capi
    from wolfgang_b200.workloads import klocal_pair_100q

    A, B = klocal_pair_100q(args.lhs_terms, args.rhs_terms)
    n = A[0]
    W = 2
    nl, nr = len(A[3]), len(B[3])
    P = nl * nr
    ax, az, ac = dev(torch, A[1]), dev(torch, A[2]), dev(torch, A[3])
    bx, bz, bc = dev(torch, B[1]), dev(torch, B[2]), dev(torch, B[3])
    stream = torch.cuda.current_stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    L = capi.lib()
    l2 = torch.empty(128 * 1024 * 1024, dtype=torch.float32, device="cuda")
    U_last = [0]

    def step():
        ox, oz, oc = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        U = ctypes.c_size_t()
        capi.check(L.wg_pauli_products(0 if world == 1 else torch.cuda.current_device(), W, ax.data_ptr(),
                                       az.data_ptr(), ac.data_ptr(), nl, bx.data_ptr(), bz.data_ptr(), bc.data_ptr(),
                                       nr, capi.WG_PRODUCTS_SIMPLIFY, 1e-12, 0.0, ctypes.byref(ox), ctypes.byref(oz),
                                       ctypes.byref(oc), ctypes.byref(U), sh))
        U_last[0] = U.value
        for p in (ox, oz, oc):
            capi.check(L.wg_free(torch.cuda.current_device(), p, sh))

    for _ in range(args.warmup):
        step()
        flush_l2(torch, l2)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = capi.kernel_launches()
    capi.profile_enable(True)
    capi.profile_report()
    total_ms = 0.0
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            flush_l2(torch, l2)
        torch.cuda.synchronize()
    capi.profile_enable(False)
    prof = capi.profile_report()
    launches = capi.kernel_launches() - launches0
    barrier(world)
    torch.cuda.synchronize()
    t_max = max_over_ranks(total_ms, world)
    ms_per_step = t_max / args.steps
    value = world * P / (ms_per_step * 1e-3)
    U = U_last[0]

    # roofline: algorithmic bytes per launch of each kernel (the bytes a launch
    # must move at minimum): keys are 2W words + a 4-byte index per item.
    rec = 8 * 2 * W + 4
    per_launch = {
        "products_kernel": P * (rec + 16),                    # write keys+index+coefficient
        "radix_scatter_kernel": P * 2 * rec,                  # read + write keys and index
        "radix_hist_kernel": P * 8,                           # read one key word
        "seg_head_kernel": P * (8 * 2 * W + 4),               # read keys, write flag
        "seg_reduce_kernel": P * (4 + 16) + U * 20,           # idx + gathered coefficient, sums
        "write_out_kernel": U * (8 * 2 * W + 16),
        # bucketed path: an item is a 4-byte product index; codes are 8 bytes;
        # operand gathers hit L2 and are not counted
        "bucket_coarse_kernel": P * 4,                         # write the item index
        "bucket_fine_kernel": P * (4 + 8 + 4),                 # idx in, code + idx out (one pass)
        "bucket_final_kernel": P * (8 + 4) + U * (4 + 16),     # code + idx in; survivors' idx + sum out
        "bucket_output_kernel": U * (4 + 16) + U * (8 * 2 * W + 16),  # survivors in, the U terms out
    }
    peak, peak_kind = peaks()
    out = {
        "metric": "H@H+simplify terms/s",
        "value": value,
        "unit": "terms/s",
        "ms_per_step": ms_per_step,
        "config": {"workload": f"config2: A({nl})xB({nr}) terms, 100 qubits, k-local w in {{2,3,4}}, "
                               "matmul+simplify(atol=1e-12)",
                   "products": P, "survivors": U, "words": W,
                   "l2": "intermediates >> L2 (126 MB); 512 MiB L2 flush between steps",
                   "byte_model_bytes_per_step": 2 * P * 48 + U * 48,
                   "byte_model_GBps": (2 * P * 48 + U * 48) / (ms_per_step * 1e-3) / 1e9},
        # DRAM bytes per item of bucket_final_kernel measured by ncu (read + write,
        # 1015.0 MB for a 33,554,432-product case of this workload)
        "roofline": roofline(prof, per_launch, peak, peak_kind,
                             traffic={"bucket_final_kernel": int(P * 1015.0e6 / 33554432)}),
        "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }

    # end to end through the public API (host PauliSum in, host PauliSum out)
    if args.e2e_steps > 0:
        import wolfgang_quantum as wq

        hA = wq.PauliSum._from_packed(n, A[1], A[2], A[3])
        hB = wq.PauliSum._from_packed(n, B[1], B[2], B[3])
        # Every rank's host result is U * (16W + 16) bytes (24 GB here).  When
        # the node's free memory cannot hold one per local rank at once, the
        # ranks make their end-to-end calls one after another, each timing its
        # own, and the line says so.
        result_bytes = U * (16 * W + 16)
        local_ranks = int(os.environ.get("LOCAL_WORLD_SIZE", str(world)))
        avail = host_available_bytes()
        fits = avail is None or avail >= local_ranks * result_bytes * 1.3
        concurrent = max_over_ranks(0.0 if fits else 1.0, world) == 0.0

        step_s: list[float] = []

        def e2e_calls() -> tuple[float, int]:
            r = hA.matmul(hB, max_intermediate_terms=P)  # warm
            t0 = time.perf_counter()
            for _ in range(args.e2e_steps):
                # each step is one call: the previous step's result is released
                # first (inside the timed region), so that a call does not run
                # beside another 24 GB result
                ts = time.perf_counter()
                r = None
                r = hA.matmul(hB, max_intermediate_terms=P)
                step_s.append(time.perf_counter() - ts)
            dt_, terms_ = (time.perf_counter() - t0) / args.e2e_steps, r.num_terms
            del r
            return dt_, terms_

        if concurrent:
            barrier(world)
            dt, terms = e2e_calls()
        else:
            dt, terms = 0.0, 0
            for turn in range(world):
                barrier(world)
                if turn == rank:
                    dt, terms = e2e_calls()
            barrier(world)
        dt = max_over_ranks(dt, world)
        out["e2e"] = {"value": world * P / dt, "unit": "terms/s", "s_per_step": dt,
                      "steps": args.e2e_steps, "s_per_step_min": min(step_s) if step_s else None,
                      "s_per_step_max": max(step_s) if step_s else None,
                      "pinned_d2h_GBps": pinned_d2h_bandwidth(torch),
                      "h2d_bytes_per_step": (nl + nr) * (16 * W + 16),
                      "d2h_bytes_per_step": terms * (16 * W + 16),
                      "api": "wolfgang_quantum.PauliSum.matmul (host operands and result)",
                      "ranks_concurrent": concurrent}
        if not concurrent:
            out["e2e"]["note"] = (f"{local_ranks} host results of {result_bytes / 1e9:.1f} GB did not fit in "
                                  f"{avail / 1e9:.0f} GB of free host memory at once: the ranks made their calls "
                                  "one after another; value = all ranks' products / the slowest rank's call")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["parity"] = products_parity(torch, L, A, B, W, ax, az, ac, bx, bz, bc, sh)
        secs, prods = reference_products_sample(A, B, args.cpu_rows)
        out["cpu_baseline"] = {"value": prods / secs, "unit": "terms/s", "cores": 1, "kind": "reference",
                               "extrapolated": True, **host_cpu(),
                               "sample": f"A[:{args.cpu_rows}] x B = {prods} products, reference PauliSum::matmul"
                                         f"(simplify=True) compiled from its sources, {secs:.1f} s; products/s of "
                                         "the row sample stand for the full A x B (every lhs row meets the same "
                                         "rhs); the reference's matmul and simplify are single-threaded"}
    return out


# ---------------------------------------------------------------- other workloads

def timed_steps(torch, steps, warmup, fn, flush=None):
    """Per-step CUDA-event timing on the current stream; returns (total ms, profile, launches)."""
    from wolfgang_b200 import capi

    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        fn()
        if flush is not None:
            flush()
    torch.cuda.synchronize()
    launches0 = capi.kernel_launches()
    capi.profile_enable(True)
    capi.profile_report()
    total = 0.0
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
            if flush is not None:
                flush()
        torch.cuda.synchronize()
    capi.profile_enable(False)
    return total, capi.profile_report(), capi.kernel_launches() - launches0, clocks.summary()


def bench_commutation(args, world, rank, torch) -> dict:
    """Config 3: bit-packed 262,144^2 commutation matrix (128 qubits)."""
    from wolfgang_b200 import capi
    from wolfgang_b200.workloads import sparse_operator_128q

    n, x, z, _ = sparse_operator_128q(args.terms)
    T = len(x)
    pitch = (T + 31) // 32
    dx, dz = dev(torch, x), dev(torch, z)
    bits = torch.empty(T * pitch, dtype=torch.int32, device="cuda")
    L = capi.lib()
    sh = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def step():
        capi.check(L.wg_commutation_bits(torch.cuda.current_device(), 2, dx.data_ptr(), dz.data_ptr(), T,
                                         dx.data_ptr(), dz.data_ptr(), T, bits.data_ptr(), pitch, args.algo, sh))

    total, prof, launches, clocks = timed_steps(torch, args.steps, args.warmup, step)
    t = max_over_ranks(total, world) / args.steps
    pairs = T * T
    out_bytes = T * pitch * 4
    peak, kind = peaks()
    rl = roofline(prof, {"commute_plane_kernel": out_bytes, "commute_ballot_kernel": out_bytes}, peak, kind)
    rl["pairs_per_s"] = pairs / (t * 1e-3)
    out = {"metric": "commutation pairs/s", "value": world * pairs / (t * 1e-3), "unit": "pairs/s", "ms_per_step": t,
           "config": {"workload": f"config3: {T} terms x {T} terms, 128 qubits, p=0.05, bit-packed matrix",
                      "output_bytes": out_bytes, "algo": args.algo},
           "roofline": rl, "gpu_launches": launches, "clocks": clocks,
           "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import Reference

        ref = Reference()
        rows = args.cpu_rows
        t0 = time.perf_counter()
        ref.commutes(n, (x[:rows], z[:rows]), (x, z))
        dt = time.perf_counter() - t0
        got = np.unpackbits(bits.view(T, pitch)[:rows].cpu().numpy().view(np.uint8).reshape(rows, -1), axis=1,
                            bitorder="little")[:, :T]
        from oracle import Oracle

        want = Oracle().commutes(n, (x[:rows], z[:rows]), (x, z))
        out["parity"] = {"rows_checked": rows, "pairs_checked": rows * T, "bit_exact": bool(np.array_equal(got, want)),
                         "how": "the first rows of the device bit matrix against the oracle's flags"}
        out["cpu_baseline"] = {"value": rows * T / dt, "unit": "pairs/s", "cores": 1, "kind": "reference",
                               "extrapolated": True, **host_cpu(), "sample": f"{rows} rows x {T} terms via reference PauliSum::commutes_with "
                                         f"(auto CPU dispatch: {ref.cpu_backend()}), {dt:.1f} s"}
    return out


def bench_grouping(args, world, rank, torch) -> dict:
    """Config 3, second half: group_commuting of the 262,144-term operator (mode qwc, or full)."""
    from wolfgang_b200 import capi
    from wolfgang_b200.workloads import sparse_operator_128q

    n, x, z, c = sparse_operator_128q(args.terms)
    T = len(x)
    dx, dz = dev(torch, x), dev(torch, z)
    order = np.zeros(T, np.uintp)
    sizes = np.zeros(T, np.uintp)
    psz = ctypes.POINTER(ctypes.c_size_t)
    ng = ctypes.c_size_t()
    L = capi.lib()
    sh = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    full = 1 if args.group_mode == "full" else 0

    def step():
        capi.check(L.wg_group_commuting(torch.cuda.current_device(), 2, T, dx.data_ptr(), dz.data_ptr(), full,
                                        order.ctypes.data_as(psz), sizes.ctypes.data_as(psz), ctypes.byref(ng), sh))

    total, prof, launches, clocks = timed_steps(torch, args.steps, args.warmup, step)
    t = max_over_ranks(total, world) / args.steps
    out = {"metric": "group_commuting terms/s", "value": world * T / (t * 1e-3), "unit": "terms/s", "ms_per_step": t,
           "config": {"workload": f"config3: group_commuting(mode={args.group_mode!r}) of {T} terms, 128 qubits, "
                                  "p=0.05", "groups": int(ng.value)},
           "roofline": {"bound": "latency", "note": "sequential first-fit: one CTA examines every open group per "
                                                   "term, terms in the deterministic order"},
           "gpu_launches": launches, "clocks": clocks,
           "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import Reference

        rows = min(T, args.cpu_group_terms)
        t0 = time.perf_counter()
        groups = Reference().group_commuting(n, x[:rows], z[:rows], c[:rows], mode=args.group_mode)
        dt = time.perf_counter() - t0
        sx, sz = dev(torch, x[:rows]), dev(torch, z[:rows])
        o2 = np.zeros(rows, np.uintp)
        s2 = np.zeros(rows, np.uintp)
        n2 = ctypes.c_size_t()
        capi.check(L.wg_group_commuting(torch.cuda.current_device(), 2, rows, sx.data_ptr(), sz.data_ptr(), full,
                                        o2.ctypes.data_as(psz), s2.ctypes.data_as(psz), ctypes.byref(n2), sh))
        same = [int(v) for v in s2[: n2.value]] == [len(g[2]) for g in groups] and np.array_equal(
            x[:rows][o2.astype(np.int64)], np.concatenate([g[0] for g in groups]))
        out["parity"] = {"terms_checked": rows, "groups_equal": bool(same),
                         "how": "device group_commuting of the reference's sample against the reference core's "
                                "groups (sizes, members in order); 262,144 terms: tests/test_gpu_fullsize.py"}
        out["cpu_baseline"] = {"value": rows / dt, "unit": "terms/s", "cores": 1, "kind": "reference",
                               "extrapolated": rows < T, **host_cpu(), "sample": f"reference PauliSum::group_commuting(mode={args.group_mode!r}) on the first "
                                         f"{rows} terms ({len(groups)} groups, {dt:.1f} s); the greedy's cost grows "
                                         "with the number of open groups, so the full operator runs slower per term"}
    return out


def bench_expectation(args, world, rank, torch) -> dict:
    """Config 4: 26 qubits (1 GiB psi), 20,000 Hermitian terms in 2,000 x-groups; E + dE/dc + dE/dpsi*."""
    from wolfgang_b200.expectation import ExpectationPlan
    from wolfgang_b200.workloads import xpattern_operator

    n = args.qubits
    op = xpattern_operator(n=n)
    g = torch.Generator(device="cuda")
    g.manual_seed(20261207)
    psi = torch.randn(1 << n, dtype=torch.complex128, device="cuda", generator=g)
    psi /= torch.linalg.vector_norm(psi)
    if args.c64:
        psi = psi.to(torch.complex64)
    plan = ExpectationPlan(op)
    res = torch.empty(2, dtype=torch.float64, device="cuda")

    def step():
        plan.run(psi, terms=True, hpsi=not args.forward_only)

    total, prof, launches, clocks = timed_steps(torch, args.steps, args.warmup, step)
    t = max_over_ranks(total, world) / args.steps
    amp = 16 if psi.dtype == torch.complex128 else 8
    G = plan.n_groups
    psi_bytes = (1 << n) * amp
    peak, kind = peaks()
    rl = roofline(prof, {"expect_forward_kernel": G * psi_bytes,
                         "expect_adjoint_kernel": G * psi_bytes + (1 << n) * 16}, peak, kind)
    del res
    out_cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # reference expectation_statevector_complex128 (forward only: the
        # reference has no gradient) on the first k terms, scaled to all T
        from oracle import Reference

        k = args.cpu_terms
        hpsi = psi.to(torch.complex128).cpu().numpy() if not args.c64 else psi.cpu().numpy()
        x, z, c = op[1][:k], op[2][:k], op[3][:k]
        t0 = time.perf_counter()
        Reference().expectation(n, x, z, c, hpsi)
        per_term = (time.perf_counter() - t0) / k
        from oracle import Oracle

        _, ev, _ = plan.run(psi, terms=True)
        ev = ev.cpu().numpy()
        sample = np.random.default_rng(4).choice(len(op[3]), size=16, replace=False)
        err = float(np.max(np.abs(ev[sample] - Oracle().term_expectations(n, op[1][sample], op[2][sample], hpsi))))
        parity = {"terms_checked": 16, "max_abs_err": err, "tolerance": 1e-12,
                  "how": "dE/dc_k = <psi|P_k|psi> of 16 random terms against the FP64 oracle on the same stored "
                         "amplitudes; 64 terms, H psi and finite differences: tests/test_gpu_fullsize.py"}
        out_cpu = {"value": 1.0 / (per_term * len(op[3])), "unit": "evals/s", "cores": 1, "kind": "reference",
                   "extrapolated": True, **host_cpu(), "sample": f"reference expectation_statevector_complex128 on the first {k} of {len(op[3])} terms "
                             f"({per_term:.3f} s per term), scaled to all terms; forward only (no gradient in "
                             f"the reference)"}
    return {"metric": "E+grad evals/s" if not args.forward_only else "E evals/s", "value": world * 1e3 / t,
            "unit": "evals/s", "ms_per_step": t, "cpu_baseline": out_cpu, "parity": parity,
            "config": {"workload": f"config4: {n} qubits, {len(op[3])} terms, {G} x-groups, "
                                   f"{'c64' if args.c64 else 'c128'} psi, forward{'' if args.forward_only else '+adjoint'}",
                       "byte_model_bytes_per_step": G * psi_bytes + (0 if args.forward_only else 2 * psi_bytes + G * psi_bytes)},
            "roofline": rl, "gpu_launches": launches, "clocks": clocks,
            "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()}}


def bench_batched(args, world, rank, torch) -> dict:
    """Config 5: 512 uneven (H, psi) pairs, forward + gradient, batched vs per-call."""
    from wolfgang_b200.expectation import ExpectationBatch, ExpectationPlan
    from wolfgang_b200.workloads import uneven_pair_operator, uneven_pairs

    pairs = uneven_pairs(args.pairs, n_min=args.min_qubits, n_max=args.max_qubits)
    if world > 1:
        pairs = shard(pairs, rank, world)
    plans, psis = [], []
    dtype = torch.complex64 if args.c64 else torch.complex128
    for n, T, seed in pairs:
        plans.append(ExpectationPlan(uneven_pair_operator(n, T, seed)))
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        p = torch.randn(1 << n, dtype=torch.complex128, device="cuda", generator=gen)
        psis.append((p / torch.linalg.vector_norm(p)).to(dtype))
    from wolfgang_b200 import capi

    amp = 8 if args.c64 else 16
    fwd_bytes = sum(pl.n_groups * (1 << pl.n) * amp for pl in plans)  # G_x |psi| per pair
    adj_bytes = fwd_bytes + sum((1 << pl.n) * 16 for pl in plans)      # + H psi written
    batch = ExpectationBatch(plans, psis, gradients=True)
    l0 = capi.kernel_launches()
    batch.capture()  # one direct run, then the captured one
    per_run = (capi.kernel_launches() - l0) // 2

    total, _, _, clocks = timed_steps(torch, args.steps, args.warmup, batch.replay)
    t = max_over_ranks(total, world) / args.steps
    launches = per_run * args.steps  # kernels each replay launches, times the timed replays
    # per-kernel times: a replay records no library events, so one run is
    # launched directly with the profiler on (outside the timed region)
    _, prof, _, _ = timed_steps(torch, 1, 0, batch.run)
    # the same batch without gradients (E and dE/dc only), for the E-only
    # per-call comparison below
    fwd = ExpectationBatch(plans, psis, gradients=False)
    fwd.capture()
    fwd_total, _, _, _ = timed_steps(torch, max(1, args.steps // 2), 1, fwd.replay)
    fwd_ms = fwd_total / max(1, args.steps // 2)
    fwd.close()

    def per_call():
        for pl, ps in zip(plans, psis):
            pl.run(ps, terms=True, hpsi=True)

    pc_total, _, _, _ = timed_steps(torch, max(1, args.steps // 2), 1, per_call)
    pc = pc_total / max(1, args.steps // 2)

    # the plain per-call drop-in: wg_expectation (the path behind
    # DevicePauliSum.expectation_statevector) builds its plan on every call and
    # returns E only -- no gradient, so it does less than a batched evaluation
    import ctypes as ct

    from wolfgang_b200.workloads import uneven_pair_operator as _upo

    L = capi.lib()
    dv = torch.cuda.current_device()
    dops = []
    for n, T, seed in pairs:
        _, x, z, c = _upo(n, T, seed)
        dops.append((n, T, dev(torch, x), dev(torch, z), dev(torch, c)))
    val = (ct.c_double * 2)()

    def one_shot():
        for (n, T, dx, dz, dc), ps in zip(dops, psis):
            capi.check(L.wg_expectation(dv, n, T, dx.data_ptr(), dz.data_ptr(), dc.data_ptr(), ps.data_ptr(),
                                        capi.WG_DTYPE_C64 if args.c64 else capi.WG_DTYPE_C128, val, None))

    one_shot()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    one_shot()
    torch.cuda.synchronize()
    os_ms = 1e3 * (time.perf_counter() - t0)
    npairs = len(pairs) * world
    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # parity: E and dE/dc of the 16 smallest pairs against the FP64 oracle
        # (all 512 pairs: tests/test_gpu_fullsize.py)
        from oracle import Oracle

        orc = Oracle()
        batch.run()
        torch.cuda.synchronize()
        small = sorted(range(len(pairs)), key=lambda i: pairs[i][1] << pairs[i][0])[:16]
        e_err = t_err = 0.0
        for i in small:
            n, T, seed = pairs[i]
            _, x, z, c = uneven_pair_operator(n, T, seed)
            ps = psis[i].cpu().numpy()
            E = complex(batch.values[i, 0].item(), batch.values[i, 1].item())
            e_err = max(e_err, abs(E - orc.expectation(n, x, z, c, ps)) / max(1.0, abs(E)))
            ev = batch.term_values[i][:T].cpu().numpy()
            t_err = max(t_err, float(np.max(np.abs(ev - orc.term_expectations(n, x, z, ps)))))
        parity = {"pairs_checked": 16, "max_rel_err_E": e_err, "max_abs_err_dE_dc": t_err, "tolerance_rel": 1e-10,
                  "how": f"{'complex64' if args.c64 else 'complex128'} states, FP64 oracle on the same stored "
                         "amplitudes"}
        # reference expectation (forward only) per term measured at a few qubit
        # counts on this config's own operators; every pair's time estimated
        # as T * 2^n * (time per amplitude at the nearest probed size)
        from oracle import Reference

        from wolfgang_b200.workloads import uneven_pair_state

        ref = Reference()
        probe = {}
        for n_probe in (12, 16, 20, 24):
            op = uneven_pair_operator(n_probe, 64, 7 + n_probe)
            st = uneven_pair_state(n_probe, 7 + n_probe)
            k = 64 if n_probe <= 20 else 4
            t0 = time.perf_counter()
            ref.expectation(n_probe, op[1][:k], op[2][:k], op[3][:k], st)
            probe[n_probe] = (time.perf_counter() - t0) / k / (1 << n_probe)
        def per_amp(n):
            return probe[min(probe, key=lambda q: abs(q - n))]

        est = sum(T * per_amp(n) * (1 << n) for n, T, _ in pairs)
        cpu = {"value": len(pairs) / est, "unit": "evals/s", "cores": 1, "kind": "reference",
               "extrapolated": True, **host_cpu(), "sample": "reference expectation_statevector_complex128 timed per term at 12/16/20/24 qubits "
                         f"({', '.join(f'{q}: {v * 1e9:.2f} ns/amp' for q, v in probe.items())}); every pair "
                         "estimated as T * 2^n * (ns per amplitude at the nearest probed size); forward only (no gradient in the "
                         f"reference); {est:.0f} s estimated for the batch"}
    return {"metric": "batched E+grad evals/s", "value": npairs / (t * 1e-3), "unit": "evals/s", "ms_per_step": t,
            "config": {"workload": f"config5: {npairs} uneven (H, psi) pairs, n in [{args.min_qubits},{args.max_qubits}], T log-uniform "
                                   f"[100,50000], {'c64' if args.c64 else 'c128'}, forward+gradient, one CUDA graph",
                       "per_call_evals_per_s": len(pairs) / (pc * 1e-3), "per_call_ms": pc,
                       "batched_over_per_call": pc / t,
                       "per_call_path": "one ExpectationPlan.run(terms, H psi) per pair, plans built once",
                       "one_shot_ms": os_ms, "batched_forward_ms": fwd_ms,
                       "batched_forward_over_one_shot": os_ms / fwd_ms,
                       "one_shot_path": "wg_expectation per pair (DevicePauliSum.expectation_statevector's path: "
                                        "plan built per call, E only), against the batch without gradients",
                       "qubits": f"{args.min_qubits}..{args.max_qubits}"},
            "roofline": roofline(prof, {"expect_forward_kernel": fwd_bytes, "expect_adjoint_kernel": adj_bytes},
                                 *peaks()),
            "parity": parity,
            "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clocks,
            "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()}}


def bench_products_batch(args, world, rank, torch) -> dict:
    """Batched uneven products: 256 products A_p * B_p (64 qubits, 16-4,096
    terms a side) prepared once and replayed from a CUDA graph, against the
    plain per-call GPU path (one wg_pauli_products per pair)."""
    import ctypes as ct

    from wolfgang_b200 import capi
    from wolfgang_b200.products import ProductsBatch
    from wolfgang_b200.workloads import uneven_product_operands, uneven_product_pairs

    descs = uneven_product_pairs(args.pairs if args.pairs != 512 else 256)
    if world > 1:
        descs = shard(descs, rank, world)
    pairs = [uneven_product_operands(*d) for d in descs]
    P = sum(len(A[3]) * len(B[3]) for A, B in pairs)
    dv = torch.cuda.current_device()
    L = capi.lib()
    ops = [([dev(torch, v) for v in A[1:]], [dev(torch, v) for v in B[1:]]) for A, B in pairs]
    w = (pairs[0][0][0] + 63) // 64

    def per_call():
        for (A, B), (a, b) in zip(pairs, ops):
            ox, oz, oc, U = ct.c_void_p(), ct.c_void_p(), ct.c_void_p(), ct.c_size_t()
            capi.check(L.wg_pauli_products(dv, w, a[0].data_ptr(), a[1].data_ptr(), a[2].data_ptr(), len(A[3]),
                                           b[0].data_ptr(), b[1].data_ptr(), b[2].data_ptr(), len(B[3]),
                                           capi.WG_PRODUCTS_SIMPLIFY, 1e-12, 0.0, ct.byref(ox), ct.byref(oz),
                                           ct.byref(oc), ct.byref(U), None))
            for q in (ox, oz, oc):
                capi.check(L.wg_free(dv, q, None))

    per_call()  # warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    per_call()
    torch.cuda.synchronize()
    per_call_ms = 1e3 * (time.perf_counter() - t0)

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch = ProductsBatch([((A[0], a[0], a[1], a[2]), (B[0], b[0], b[1], b[2])) for (A, B), (a, b) in zip(pairs, ops)])
    torch.cuda.synchronize()
    create_ms = 1e3 * (time.perf_counter() - t0)
    l0 = capi.kernel_launches()
    batch.capture()  # one direct run, then the captured one
    per_run = (capi.kernel_launches() - l0) // 2
    total, _, _, clocks = timed_steps(torch, args.steps, args.warmup, batch.replay)
    t = max_over_ranks(total, world) / args.steps
    launches = per_run * args.steps  # kernels each replay launches, times the timed replays
    # per-kernel times: a replay records no library events, so the same run is
    # launched directly with the profiler on (outside the timed region)
    _, prof, _, _ = timed_steps(torch, max(1, args.steps // 2), 1, batch.run)
    peak, kind = peaks()
    rl = roofline(prof, {"pbatch_sums_kernel": 4 * batch.n_products + 24 * batch.n_keys,
                         "pbatch_write_kernel": batch.n_keys * 12 + batch.n_keys * (16 * w + 16)}, peak, kind)
    out = {"metric": "batched products terms/s", "value": world * P / (t * 1e-3), "unit": "terms/s",
           "ms_per_step": t,
           "config": {"workload": f"{len(pairs) * world} uneven products A_p*B_p, 64 qubits, 16-4096 terms a side, "
                                  "k-local w in 1..6, matmul+simplify(atol=1e-12), one CUDA graph replay",
                      "products": P, "keys": batch.n_keys, "per_call_ms": per_call_ms,
                      "per_call_path": "wg_pauli_products per pair (plan-free drop-in, synchronising)",
                      "create_ms": create_ms, "batched_over_per_call": per_call_ms / t,
                      "first_use_over_per_call": per_call_ms / (create_ms + t),
                      "note": "create sorts every product's key once (the symbolic pass); a replay forms, sums and "
                              "culls the coefficients"},
           "roofline": rl, "gpu_launches": launches, "clocks": clocks,
           "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import Oracle, Reference

        # parity: every pair's result bit for bit against the oracle, on the
        # smallest pairs and every 16th pair
        orc = Oracle()
        got = batch.results()
        check = sorted(range(len(pairs)), key=lambda i: len(pairs[i][0][3]) * len(pairs[i][1][3]))[:8]
        check += list(range(0, len(pairs), 16))
        exact = True
        for i in sorted(set(check)):
            A, B = pairs[i]
            raw = orc.matmul(A[0], A[1:], B[1:], simplify=False)
            want = orc.simplify(A[0], *raw, 1e-12, 0.0)
            exact = exact and all(np.ascontiguousarray(g).tobytes() == np.ascontiguousarray(wv).tobytes()
                                  for g, wv in zip(got[i], want))
        out["parity"] = {"pairs_checked": len(set(check)), "bit_exact": bool(exact), "max_abs_err": 0.0 if exact else None}
        ref = Reference()
        sample = list(range(0, len(pairs), 8))
        t0 = time.perf_counter()
        prods = 0
        for i in sample:
            A, B = pairs[i]
            ref.matmul(A[0], A[1:], B[1:], simplify=True, max_intermediate_terms=max(1, len(A[3]) * len(B[3])))
            prods += len(A[3]) * len(B[3])
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": prods / dt, "unit": "terms/s", "cores": 1, "kind": "reference",
                               "extrapolated": True, **host_cpu(),
                               "sample": f"reference PauliSum::matmul(simplify=True) on every 8th pair "
                                         f"({len(sample)} pairs, {prods} products, {dt:.1f} s)"}
    batch.close()
    return out


# ---------------------------------------------------------------- per-op comparison with the reference GPU path

# Device-resident operations timed on both sides (this repository: --workload
# ops; the reference's own CUDA path: --impl reference-gpu), each on seeded
# inputs both arms regenerate identically:
#   hh_simplify      config 1: H @ H with simplify (4,096 x 4,096 terms, 20 qubits)
#   simplify_5e6     simplify of 5,000,000 terms on 20 qubits drawn from 100,000
#                    distinct keys (98 % duplicates)
#   commute_4096     config 1: the 4,096 x 4,096 commutation flags (uint8 output)
#   commute_16384    config 3's first 16,384 terms: the 16,384^2 flags (uint8)
#   expect_20q       config 1: <psi|H|psi>, 2^20 amplitudes, 4,096 terms
#   products_config2 config 2: 32,768 x 16,384 products + simplify (5.4e8 products)
#   expect_26q       config 4: <psi|H|psi>, 2^26 amplitudes, 20,000 terms
OPS = ("hh_simplify", "simplify_5e6", "commute_4096", "commute_16384", "expect_20q", "products_config2",
       "expect_26q")


def ops_input(W, op):
    """Seeded inputs of one comparison operation (numpy; both arms)."""
    if op in ("hh_simplify", "commute_4096", "expect_20q"):
        (n, x, z, c), psi = W.hamiltonian_20q_and_state()
        return n, x, z, c, psi
    if op == "simplify_5e6":
        rng = np.random.default_rng(W.SEED_BASE + 11)
        n, px, pz, _ = W.bernoulli_operator(rng, 20, 100_000, 0.25)
        pick = rng.integers(0, 100_000, size=5_000_000)
        c = (rng.normal(size=5_000_000) + 1j * rng.normal(size=5_000_000)).astype(np.complex128)
        return n, px[pick], pz[pick], c, None
    if op == "commute_16384":
        n, x, z, c = W.sparse_operator_128q()
        return n, x[:16384], z[:16384], c[:16384], None
    if op == "products_config2":
        return W.klocal_pair_100q()
    if op == "expect_26q":
        n, x, z, c = W.xpattern_operator(n=26)
        return n, x, z, c, W.state_26q()
    raise ValueError(op)


def _host_timed(warmup, reps, call):
    for _ in range(warmup):
        call()
    t0 = time.perf_counter()
    for _ in range(reps):
        call()
    return 1e3 * (time.perf_counter() - t0) / max(reps, 1)


def bench_ops(args, world, rank, torch) -> dict:
    """This repository's side of the per-op comparison (device-resident: the
    operands are on the device before timing; each call synchronises)."""
    import ctypes as ct

    from wolfgang_b200 import capi

    W = load_workloads()
    L = capi.lib()
    dv = torch.cuda.current_device()
    res = {}
    for op in [o for o in args.ops.split(",") if o]:
        reps = 1 if op in ("expect_26q", "products_config2") else args.steps
        inp = ops_input(W, op)
        if op in ("hh_simplify", "products_config2"):
            if op == "hh_simplify":
                n, x, z, c, _ = inp
                A = B = (n, x, z, c)
            else:
                A, B = inp
            n, w = A[0], (A[0] + 63) // 64
            a = [dev(torch, v) for v in A[1:]]
            b = [dev(torch, v) for v in B[1:]]
            out = {}

            def call():
                ox, oz, oc, U = ct.c_void_p(), ct.c_void_p(), ct.c_void_p(), ct.c_size_t()
                capi.check(L.wg_pauli_products(dv, w, a[0].data_ptr(), a[1].data_ptr(), a[2].data_ptr(), len(A[3]),
                                               b[0].data_ptr(), b[1].data_ptr(), b[2].data_ptr(), len(B[3]),
                                               capi.WG_PRODUCTS_SIMPLIFY, 1e-12, 0.0, ct.byref(ox), ct.byref(oz),
                                               ct.byref(oc), ct.byref(U), None))
                out["terms"] = U.value
                for q in (ox, oz, oc):
                    capi.check(L.wg_free(dv, q, None))

            ms = _host_timed(1, reps, call)
            res[op] = {"ms": ms, "terms": out["terms"], "products": len(A[3]) * len(B[3])}
        elif op == "simplify_5e6":
            n, x, z, c, _ = inp
            d = [dev(torch, v) for v in (x, z, c)]
            out = {}

            def call():
                ox, oz, oc, U = ct.c_void_p(), ct.c_void_p(), ct.c_void_p(), ct.c_size_t()
                capi.check(L.wg_simplify(dv, 1, len(c), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), 1e-12,
                                         0.0, ct.byref(ox), ct.byref(oz), ct.byref(oc), ct.byref(U), None))
                out["terms"] = U.value
                for q in (ox, oz, oc):
                    capi.check(L.wg_free(dv, q, None))

            res[op] = {"ms": _host_timed(1, reps, call), "terms": out["terms"], "input_terms": len(c)}
        elif op.startswith("commute"):
            n, x, z, _, _ = inp
            T = len(x)
            w = (n + 63) // 64
            d = [dev(torch, v) for v in (x, z)]
            pitch = (T + 31) // 32
            bits = torch.empty(T * pitch, dtype=torch.int32, device="cuda")
            flags = torch.empty(T * T, dtype=torch.uint8, device="cuda")

            def bits_call():
                capi.check(L.wg_commutation_bits(dv, w, d[0].data_ptr(), d[1].data_ptr(), T, d[0].data_ptr(),
                                                 d[1].data_ptr(), T, bits.data_ptr(), pitch, 0, None))
                torch.cuda.synchronize()

            def u8_call():
                capi.check(L.wg_commutation_bits(dv, w, d[0].data_ptr(), d[1].data_ptr(), T, d[0].data_ptr(),
                                                 d[1].data_ptr(), T, bits.data_ptr(), pitch, 0, None))
                capi.check(L.wg_bits_to_u8(dv, bits.data_ptr(), T, T, pitch, flags.data_ptr(), None))
                torch.cuda.synchronize()

            ms_bits = _host_timed(1, reps, bits_call)
            ms_u8 = _host_timed(1, reps, u8_call)
            res[op] = {"ms": ms_u8, "ms_bits_only": ms_bits, "commuting": int(flags.sum(dtype=torch.int64).item())}
        else:  # expectation: the one-shot drop-in (plan built per call) and a reused plan
            from wolfgang_b200.expectation import ExpectationPlan

            n, x, z, c, psi = inp
            dx, dz, dc, dpsi = (dev(torch, v) for v in (x, z, c, psi))
            val = (ct.c_double * 2)()

            def one_shot():
                capi.check(L.wg_expectation(dv, n, len(c), dx.data_ptr(), dz.data_ptr(), dc.data_ptr(),
                                            dpsi.data_ptr(), capi.WG_DTYPE_C128, val, None))

            plan = ExpectationPlan((n, x, z, c))

            def reuse():
                r, _, _ = plan.run(dpsi)
                torch.cuda.synchronize()

            res[op] = {"ms": _host_timed(1, reps, one_shot), "ms_plan_reused": _host_timed(1, reps, reuse),
                       "value": [val[0], val[1]]}
            plan.close()
        torch.cuda.empty_cache()
    return {"metric": "device-resident ms per call (sum over ops)", "value": sum(v["ms"] for v in res.values()),
            "unit": "ms", "higher_is_better": False, "ms_per_step": sum(v["ms"] for v in res.values()),
            "config": {"workload": "per-op comparison set (bench.OPS): " + args.ops,
                       "timing": "host clock around each synchronising call, operands resident on the device",
                       "sort": args.sort, "ops": res},
            "gpu_launches": None}


def reference_gpu_arm(args) -> dict:
    """The reference's own CUDA path (its DevicePauliSum, src/cuda/*.cu built
    for sm_100a, oracle/_ref/libwgref_cuda.so) on the same operations and
    GPU, device-resident, timed by the host clock around each of its
    synchronising calls.  Loads no library of this repository."""
    from oracle import ReferenceGPU

    if not ReferenceGPU.available():
        return {"impl": "reference-gpu", "unavailable": "oracle/_ref/libwgref_cuda.so was not built"}
    ref = ReferenceGPU()
    W = load_workloads()
    res = {}
    for op in [o for o in args.ops.split(",") if o]:
        reps = 1 if op in ("expect_26q", "products_config2") else args.steps
        inp = ops_input(W, op)
        try:
            if op in ("hh_simplify", "products_config2"):
                if op == "hh_simplify":
                    n, x, z, c, _ = inp
                    A = B = (n, x, z, c)
                else:
                    A, B = inp
                P = len(A[3]) * len(B[3])
                ms, terms = ref.matmul(A[0], A[1:], B[1:], True, max(P, 50_000_000), 1, reps)
                res[op] = {"ms": ms, "terms": terms, "products": P}
            elif op == "simplify_5e6":
                n, x, z, c, _ = inp
                ms, terms = ref.simplify(n, x, z, c, 1e-12, 0.0, 1, reps)
                res[op] = {"ms": ms, "terms": terms, "input_terms": len(c)}
            elif op.startswith("commute"):
                n, x, z, _, _ = inp
                ms, count = ref.commutes_device(n, (x, z), (x, z), 1, reps)
                res[op] = {"ms": ms, "commuting": count}
            else:
                n, x, z, c, psi = inp
                ms, v = ref.expectation(n, x, z, c, psi, 1 if reps > 1 else 0, reps)
                res[op] = {"ms": ms, "value": [v.real, v.imag]}
        except Exception as exc:  # the reference's own refusal (e.g. out of memory) is reported, not hidden
            res[op] = {"error": str(exc)}
    return {"impl": "reference-gpu", "metric": "device-resident ms per call (sum over ops)",
            "value": sum(v.get("ms", 0.0) for v in res.values()), "unit": "ms", "higher_is_better": False,
            "config": {"workload": "per-op comparison set (bench.OPS): " + args.ops,
                       "timing": "host clock around each synchronising call of the reference's DevicePauliSum, "
                                 "operands uploaded once beforehand",
                       "build": "reference src/cuda/*.cu, nvcc 12.9 -O2 -gencode arch=compute_100a,code=sm_100a",
                       "ops": res}}


def reference_arm(args, world, rank) -> dict:
    """Times the reference's own CPU core on bounded samples of the same workload.

    Only oracle/_ref/libwgref.so (the reference core compiled from its sources)
    is loaded: the generators come in by file path, not through the package."""
    A, B = load_workloads().klocal_pair_100q()
    for _ in range(args.warmup):
        reference_products_sample(A, B, 16)
    total, prods = 0.0, 0
    for _ in range(args.steps):
        s, p = reference_products_sample(A, B, args.ref_rows)
        total += s
        prods += p
    v = prods / total
    return {
        "metric": "H@H+simplify terms/s", "value": v, "unit": "terms/s", "impl": "reference",
        "ms_per_step": 1e3 * total / args.steps,
        "config": {"workload": "config2: A(32768)xB(16384) terms, 100 qubits, k-local w in {2,3,4}, matmul+simplify(atol=1e-12)",
                   "sample_rows": args.ref_rows},
        "extrapolated": True,
        "cpu_baseline": {"value": v, "unit": "terms/s", "cores": 1, "kind": "reference", "extrapolated": True,
                         **host_cpu(),
                         "sample": f"A[:{args.ref_rows}] x B per step ({args.ref_rows * len(B[3])} products), "
                                   "reference PauliSum::matmul(simplify=True), scalar path; products/s of the row "
                                   "sample stand for the full A(32768) x B(16384) (every lhs row meets the same "
                                   "rhs); the reference's matmul and simplify are single-threaded, so 1 core of "
                                   "nproc is used"},
        "e2e": {"value": v, "unit": "terms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def build_parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-gpu"], default="ours")
    ap.add_argument("--workload", choices=["products", "commutation", "grouping", "expectation", "batched",
                                           "products_batch", "ops"], default="products")
    ap.add_argument("--ops", default=",".join(OPS), help="operations of --workload ops / --impl reference-gpu")
    ap.add_argument("--group-mode", choices=["qwc", "full"], default="qwc", help="grouping mode (config 3)")
    ap.add_argument("--cpu-group-terms", type=int, default=16384, help="reference terms timed for grouping")
    ap.add_argument("--terms", type=int, default=262144, help="commutation terms (config 3)")
    ap.add_argument("--algo", type=int, default=0, help="commutation algorithm: 0 auto, 1 ballot, 2 bit-plane")
    ap.add_argument("--qubits", type=int, default=26, help="expectation qubits (config 4)")
    ap.add_argument("--c64", action="store_true", help="complex64 statevector storage")
    ap.add_argument("--forward-only", action="store_true")
    ap.add_argument("--pairs", type=int, default=512, help="batched pairs (config 5)")
    ap.add_argument("--min-qubits", type=int, default=8, help="batched pairs: smallest qubit count")
    ap.add_argument("--max-qubits", type=int, default=24, help="batched pairs: largest qubit count")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-rows", type=int, default=1024)
    ap.add_argument("--cpu-terms", type=int, default=8, help="reference terms timed for the expectation baseline")
    ap.add_argument("--ref-rows", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--autotune", choices=["off", "cached", "search"], default="cached",
                    help="autotuner mode; a search runs in the untimed warm-up and the line records the cache")
    ap.add_argument("--sort", choices=["auto", "lsd", "bucket"], default="auto",
                    help="sort-reduce algorithm of products and simplify (results identical)")
    ap.add_argument("--lhs-terms", type=int, default=32768, help="A terms (smaller values: profiling cases)")
    ap.add_argument("--rhs-terms", type=int, default=16384, help="B terms")
    return ap


def main() -> None:
    args = build_parser().parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3

    if args.impl == "reference-gpu":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        out = reference_gpu_arm(args)
        out.update(n_gpus=1, steps=args.steps, warmup=args.warmup, data="synthetic (seeded generators)")
        print(json.dumps(out), flush=True)
        return

    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return
        out = reference_arm(args, 1, 0)
        out.update(n_gpus=args.gpus, steps=args.steps, warmup=args.warmup, higher_is_better=True,
                   scaling="weak", vs_baseline=None, dtype="f64", data="synthetic (seeded generator of config 2)")
        print(json.dumps(out), flush=True)
        return

    import torch

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    if args.sort != "auto":
        from wolfgang_b200 import capi

        capi.set_sort_algorithm({"lsd": capi.WG_SORT_LSD, "bucket": capi.WG_SORT_BUCKET}[args.sort])
    if args.autotune != "cached":
        from wolfgang_b200 import capi

        capi.autotune_mode({"off": capi.WG_TUNE_OFF, "search": capi.WG_TUNE_SEARCH}[args.autotune])
    fn = {"products": bench_products, "commutation": bench_commutation, "grouping": bench_grouping,
          "expectation": bench_expectation, "batched": bench_batched, "products_batch": bench_products_batch,
          "ops": bench_ops}[args.workload]
    out = fn(args, world, rank, torch)
    out.setdefault("higher_is_better", True)
    out.update(n_gpus=world, steps=args.steps, warmup=args.warmup, scaling="weak",
               vs_baseline=None, dtype="u64" if args.workload in ("commutation", "grouping") else "f64",
               data=f"synthetic (seeded generator, workload {args.workload})")
    if args.autotune != "cached":
        from wolfgang_b200 import capi

        out.setdefault("config", {})["autotune"] = {"mode": args.autotune, "cache": capi.autotune_export()}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
