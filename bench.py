"""Benchmark of the B200-native CSR product C = A·B.

Workload (one step = one full product, symbolic + numeric, on one batch):
C = A·A for the 27-point stencil on a 128^3 grid (n = 2,097,152,
nnz(A) = 55,742,968, 1,489,355,288 intermediate products, nnz(C) =
254,840,104), fp64 values, seeded synthetic data. With N GPUs (torchrun)
the grid grows to 128 x 128 x (128 N) and rank r owns the z-slab of planes
[128 r, 128 r + 128): its rows of A times the B rows they reference (its
slab plus one halo plane each side, generated locally), so per-GPU work is
fixed (weak scaling) and no collective touches the data path.

value  = GFLOP/s (2 x intermediate products / time), inputs resident in HBM,
         C written into preallocated buffers, whole job (sum over ranks of
         the work / max over ranks of the time).
e2e    = the same metric through the C ABI entry nspb_spgemm_host with
         pinned host operands and a pinned host C: every step copies A (and
         B) host->device and C device->host, overlapped with the product.
--impl reference: the CPU product (OpenMP Gustavson restating the
         reference's semantics; the reference has no CPU implementation) on
         all host cores, same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L = 128
SEED = 20261203
# the row-group kernels the default call runs (dominant launches of the stencil
# product): from entry maps when the call recorded them, else the staged walk
NUM_KERNEL = {True: "k_num_map", False: "k_num_rg"}
SYM_KERNEL = {True: "k_sym_map", False: "k_sym_group"}
METRIC = "SpGEMM GFLOP/s, C=A*A, 27-point stencil 128^3, fp64"
WORKLOAD = "stencil27_128^3_AxA_fp64"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="nspb", choices=["nspb", "reference"])
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--grid", type=int, default=128,
                   help="stencil edge L (default 128; smaller grids for profiler captures)")
    p.add_argument("--no-forms", action="store_true",
                   help="skip the batched / fp32c / reference-kernel lines (profiler captures)")
    p.add_argument("--form-steps", type=int, default=5,
                   help="timed steps of each form (after one warm-up step)")
    p.add_argument("--only-form", default=None, choices=["batched", "fp32c", "reference_gpu",
                                                          "powerlaw"],
                   help="run one form alone (prints its object as the JSON line)")
    p.add_argument("--fp32c-grid", type=int, default=160)
    p.add_argument("--pl-rows", type=int, default=1_000_000,
                   help="power-law matrix order (default 1M; smaller for profiler captures)")
    p.add_argument("--batch-count", type=int, default=256)
    p.add_argument("--batch-nmax", type=int, default=100_000)
    p.add_argument("--row-kernel", type=int, default=0,
                   help="opts.row_kernel of the timed calls (0 = the library default)")
    return p.parse_args()


def _timed(fn, steps, warmup):
    """Mean ms of fn() over `steps` after `warmup` calls, CUDA events on the
    current stream with a synchronize on both sides."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


class _StepTimer:
    """Device time of single calls: synchronize, event, call, event, synchronize.
    Work released after a call (freeing its outputs) happens outside the
    measured span, for every arm alike. Returns the median over the steps:
    device allocation inside the calls (cudaMalloc of C, as the reference's
    entry point does) occasionally takes several ms."""

    def __init__(self):
        import torch
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)

    def __call__(self, fn, steps, warmup, after=None):
        import torch
        for _ in range(warmup):
            fn()
            if after:
                after()
        times = []
        for _ in range(steps):
            torch.cuda.synchronize()
            self.e0.record()
            fn()
            self.e1.record()
            torch.cuda.synchronize()
            times.append(self.e0.elapsed_time(self.e1))
            if after:
                after()
        return statistics.median(times)


def form_batched(args, index):
    """Batched products against one nspb_spgemm call per product, on equal
    work: both arms run the symbolic and numeric phases and allocate C on
    every step (outputs are released outside the timed spans). Workloads: the
    6 Galerkin products of the SA-AMG hierarchy of the 27-point stencil on
    96^3, and those plus `batch-count` random products. Plan replays (the
    symbolic phase and C's allocation done once, the numeric phase replayed
    from a CUDA graph) are reported beside them."""
    import nsp_b200 as nb
    from nsp_b200 import amg
    t0 = time.time()
    pairs = amg.amg_batch(L=96, levels=4, seed=SEED)
    n_amg = len(pairs)
    pairs += amg.random_batch(args.batch_count, 1000, args.batch_nmax, 4, 32, seed=SEED)
    dA = [a.to_device() for a, _ in pairs]
    dB = [b.to_device() for _, b in pairs]
    setup_s = time.time() - t0
    ips = [nb.intprod(a, b)[1] for a, b in zip(dA, dB)]
    keep = []
    timer = _StepTimer()
    steps, warm = args.form_steps, 1
    out = {"config": {"workload": "amg96_galerkin_x6 + random products",
                      "products": len(pairs), "amg_products": n_amg,
                      "random_products": args.batch_count, "random_n": [1000, args.batch_nmax],
                      "random_degrees": [4, 32], "setup_s": round(setup_s, 1),
                      "timing": "median device time of single calls, C allocated inside both "
                                "arms, outputs freed outside the timed spans"}}
    clocks = Clocks(index)
    clocks.start()
    for name, sl in (("amg", slice(0, n_amg)), ("amg_plus_random", slice(0, len(pairs)))):
        a_s, b_s, ip = dA[sl], dB[sl], float(sum(ips[sl]))
        ms_b = timer(lambda: keep.append(nb.spgemm_batched(a_s, b_s)), steps, warm, keep.clear)
        ms_s = timer(lambda: keep.extend(nb.spgemm(a, b) for a, b in zip(a_s, b_s)), steps, warm,
                     keep.clear)
        plan = nb.Plan(a_s, b_s, check_errors=False)
        ms_p = timer(plan.execute, steps, warm)
        del plan
        out[name] = {"intprod": int(ip),
                     "batched": {"ms": ms_b, "gflops": 2 * ip / ms_b / 1e6},
                     "one_call_per_product": {"ms": ms_s, "gflops": 2 * ip / ms_s / 1e6},
                     "speedup_batched_vs_one_call": ms_s / ms_b,
                     "plan_replay": {"ms": ms_p, "gflops": 2 * ip / ms_p / 1e6,
                                     "speedup_vs_one_call": ms_s / ms_p}}
    out["clocks"] = clocks.stop()
    return out


def _fp32c_errors(c32, c64, cabs):
    """Error of the compensated result against the fp64 one: the largest
    |c32 - c64| / sum_k |a_ik b_kj| over all entries, and the largest per-entry
    relative error |c32 - c64| / |c64| over entries with |c64| above 1e-3 of
    their sum_k |a b| (away from cancellation; an entry that cancels to a
    tiny fraction of its sum|ab| carries a relative error of the scaled error
    divided by that fraction), with that entry count."""
    d = (c32.val - c64.val).abs()
    scaled = (d / cabs.val.clamp_min(1e-300)).max().item()
    mask = c64.val.abs() > 1e-3 * cabs.val
    rel = (d[mask] / c64.val.abs()[mask]).max().item() if bool(mask.any()) else 0.0
    return {"max_err_scaled_by_sum_abs": scaled, "max_rel_err": rel,
            "rel_err_entries": int(mask.sum().item()), "entries": int(c64.val.numel())}


def form_fp32c_one(args, index, which):
    """FP32 compensated against fp64 on one matrix (fp32-representable values):
    C preallocated for both paths, full products timed; errors per matrix."""
    import torch
    import nsp_b200 as nb
    from nsp_b200.csr import HostCSR
    if which == "powerlaw":
        A = nb.gen.powerlaw(args.pl_rows, alpha=2.1, mean_deg=16.0, max_deg=50_000, seed=SEED,
                            fp32=True)
        wl = f"powerlaw_{args.pl_rows}_AxA"
    else:
        A = nb.gen.stencil(args.fp32c_grid, npts=27, seed=SEED, fp32=True)
        wl = f"stencil27_{args.fp32c_grid}^3_AxA"
    d64 = A.to_device()
    d32 = HostCSR(A.nrows, A.ncols, A.rowptr, A.col, A.val.astype(np.float32)).to_device()
    ip = nb.intprod(d64, d64)[1]
    rp, nnz = nb.spgemm_symbolic(d64, d64)

    def alloc():
        return nb.DeviceCSR(A.nrows, A.ncols, torch.empty_like(rp),
                            torch.empty(nnz, dtype=torch.int32, device="cuda"),
                            torch.empty(nnz, dtype=torch.float64, device="cuda"))
    o64, o32, o32w = alloc(), alloc(), alloc()
    st = {}

    def f32():
        _, s_ = nb.spgemm(d32, d32, precision="fp32c", out=o32, check_errors=False,
                          return_stats=True)
        st.update(s_)
    clocks = Clocks(index)
    clocks.start()
    ms64 = _timed(lambda: nb.spgemm(d64, d64, out=o64, check_errors=False), args.form_steps, 1)
    ms32 = _timed(f32, args.form_steps, 1)
    ms32w = _timed(lambda: nb.spgemm(d32, d32, precision="fp32w", out=o32w, check_errors=False),
                   args.form_steps, 1)
    clk = clocks.stop()
    nb.spgemm(d32, d32, precision="fp32c", out=o32)  # checked calls
    nb.spgemm(d32, d32, precision="fp32w", out=o32w)
    nb.spgemm(d64, d64, out=o64)
    dabs = nb.DeviceCSR(d64.nrows, d64.ncols, d64.rowptr, d64.col, d64.val.abs())
    cabs = nb.spgemm(dabs, dabs)
    for o in (o32, o32w):
        assert torch.equal(o64.rowptr, o.rowptr) and torch.equal(o64.col, o.col)
    err = _fp32c_errors(o32, o64, cabs)
    errw = _fp32c_errors(o32w, o64, cabs)
    del o64, o32, o32w, cabs
    return {"workload": wl, "intprod": ip, "nnz_C": nnz,
            "fp32c": {"ms": ms32, "gflops": 2 * ip / ms32 / 1e6,
                      "what": "fp32 values, error-free fp32 products, two-sum compensated "
                              "fp32 pairs in the hash slots; rows over the bound in fp64"},
            "fp32w": {"ms": ms32w, "gflops": 2 * ip / ms32w / 1e6,
                      "what": "fp32 values, products exact in fp64, fp64 accumulation"},
            "fp64": {"ms": ms64, "gflops": 2 * ip / ms64 / 1e6},
            "speedup_fp32c_vs_fp64": ms64 / ms32, "speedup_fp32w_vs_fp64": ms64 / ms32w,
            "errors_vs_fp64": err, "errors_vs_fp64_fp32w": errw,
            "rows_in_fp64": st.get("rows_redone"),
            "a_priori_bound": st.get("max_row_err"), "clocks": clk}


def form_reference_gpu(args, index, A, dA):
    """The reference's own nsp_spgemm_kernel_hash (built for sm_100a from the
    reference sources into oracle/_ref by the oracle Makefile) against this
    library's drop-in of the same entry point, on the same device inputs.
    Both allocate C inside every call (the reference's contract, as timed by
    its loc_time, src/spspmpi.cu:288-305). The reference's bins are checked
    on the CPU first so it never reaches its unbounded chunk kernel
    (nsp/src/nsp.cu:1725-1897)."""
    import ctypes as C
    import torch
    import nsp_b200 as nb
    import oracle
    if not os.path.exists(oracle.REF_SO):
        return {"unavailable": "oracle/_ref/libnsp_ref.so not built (reference sources absent)"}
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden
    ip, tot = oracle.intprod(A, A)
    ok, why = make_golden.reference_bins_safe(A, A)
    if not ok:
        return {"unavailable": f"input reaches a reference path refused on the CPU: {why}"}
    lib = C.CDLL(oracle.REF_SO)
    lib.ref_nsp_time_device.restype = C.c_float
    lib.ref_nsp_time_device.argtypes = [C.c_int] * 3 + [C.c_void_p] * 3 + [C.c_int] + \
        [C.c_void_p] * 3 + [C.c_int] * 3 + [C.POINTER(C.c_int), C.POINTER(C.c_float)]
    nnz = C.c_int(0)
    p = (dA.rowptr.data_ptr(), dA.col.data_ptr(), dA.val.data_ptr())
    times = (C.c_float * args.form_steps)()
    clocks = Clocks(index)
    clocks.start()
    lib.ref_nsp_time_device(A.nrows, A.ncols, A.ncols, *p, A.nnz, *p, A.nnz, 1, args.form_steps,
                            C.byref(nnz), times)
    ref_ms = statistics.median(list(times))  # the same statistic as this library's arm
    torch.cuda.synchronize()
    a = nb.sfcsr_of(dA)
    cs = []

    def ours():
        c = nb.SfCSR()
        nb.nsp_spgemm_kernel_hash(a, a, c)
        cs.append(c)

    def release():
        for c in cs:
            for ptr in (c.d_rpt, c.d_col, c.d_val):
                nb.lib.nspb_free(C.c_void_p(ptr))
        cs.clear()
    ms = _StepTimer()(ours, args.form_steps, 1, release)
    clk = clocks.stop()
    flops = 2.0 * tot
    return {"entry": "nsp_spgemm_kernel_hash(sfCSR*, sfCSR*, sfCSR*), C cudaMalloc'ed inside",
            "workload": WORKLOAD, "nnz_C": nnz.value,
            "reference_nsp": {"ms": ref_ms, "gflops": flops / ref_ms / 1e6,
                              "build": "reference nsp.cu + nsp_calc_val_sort_rows.cu, "
                                       "nvcc -O3 -arch sm_100a -DDOUBLE"},
            "nspb_dropin": {"ms": ms, "gflops": flops / ms / 1e6},
            "speedup_nspb_vs_reference": ref_ms / ms, "steps": args.form_steps,
            "statistic": "median of single calls (CUDA events, device synchronised around each)",
            "clocks": clk}


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def local_problem(rank, world):
    """This rank's A row block (global columns) and the B rows it needs, with
    A's columns shifted to index them."""
    import nsp_b200 as nb
    nz = L * world
    z0, z1 = L * rank, L * (rank + 1)
    A = nb.gen.stencil_slab(L, L, nz, z0, z1, 27, SEED)
    if world == 1:
        return A, A
    h0, h1 = max(z0 - 1, 0), min(z1 + 1, nz)
    B = nb.gen.stencil_slab(L, L, nz, h0, h1, 27, SEED)
    A.col = (A.col - h0 * L * L).astype(np.int32)
    A.ncols = B.nrows
    return A, B


def alg_bytes(A, B, nnz_c):
    """Every input read once and C written once (rowptr int32, col int32,
    val fp64)."""
    return (4 * (A.nrows + 1) + 12 * A.nnz + 4 * (B.nrows + 1) + 12 * B.nnz
            + 4 * (A.nrows + 1) + 12 * nnz_c)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    (profiles/roofline_traffic.txt: 'kernel: bytes' lines)."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    try:
        for line in open(path):
            if line.startswith(kernel + ":"):
                return float(line.split(":", 1)[1].split()[0])
    except Exception:
        pass
    return None


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # the sampler takes a moment to start: wait for its first line so the
            # samples fall inside the timed region that follows
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_product_rate(A, B, rows, threads):
    """GFLOP/s of the CPU oracle on rows [0, rows) of A·B (one timed run
    after one warm-up)."""
    import oracle
    ip, _ = oracle.intprod(A, B, threads)
    flops = 2.0 * float(ip[:rows].sum())
    oracle.spgemm_rows(A, B, 0, min(rows, 2000), threads)
    t0 = time.perf_counter()
    oracle.spgemm_rows(A, B, 0, rows, threads)
    dt = time.perf_counter() - t0
    return flops / dt / 1e9, dt


def sample_rows(A, B, threads, budget_s=8.0):
    """Largest leading row block the CPU finishes in about budget_s."""
    import oracle
    probe = min(A.nrows, 65536)
    _, dt = cpu_product_rate(A, B, probe, threads)
    rows = int(probe * budget_s / max(dt, 1e-6))
    return max(1, min(A.nrows, rows))


def run_reference(args, rank, world):
    """CPU arm: the oracle (OpenMP Gustavson) on all host cores."""
    if rank != 0:
        return
    import oracle
    from oracle import gen as ogen
    # the same seeded stencil, built by the oracle's numpy restatement of the
    # generator: this arm loads no part of the product library
    A = ogen.stencil(L, 27, SEED)
    B = A
    threads = os.cpu_count() or 1
    rows = sample_rows(A, B, threads, budget_s=max(2.0, 120.0 / max(args.steps + args.warmup, 1)))
    ip, _ = oracle.intprod(A, B, threads)
    flops = 2.0 * float(ip[:rows].sum())
    for _ in range(args.warmup):
        oracle.spgemm_rows(A, B, 0, rows, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.spgemm_rows(A, B, 0, rows, threads)
        times.append(time.perf_counter() - t0)
    t = sum(times) / len(times)
    v = flops / t / 1e9
    sample = f"rows [0,{rows}) of {A.nrows} ({rows / A.nrows:.1%}), {flops / 2:.3e} products"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": f"synthetic (seeded 27-point stencil, seed {SEED})",
        "config": {"workload": WORKLOAD, "sample": sample},
        "cpu_baseline": {"value": v, "unit": "GFLOP/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def form_powerlaw(args, index):
    """C = A·A for the power-law matrix (n = 1M, Zipf alpha 2.1, mean degree
    16, max 50k), fp64, C preallocated: every bin, the long-row kernels too."""
    import torch
    import nsp_b200 as nb
    P = nb.gen.powerlaw(args.pl_rows, alpha=2.1, mean_deg=16.0, max_deg=50_000, seed=SEED)
    dP = P.to_device()
    rp, nnz = nb.spgemm_symbolic(dP, dP)
    out = nb.DeviceCSR(P.nrows, P.ncols, torch.empty_like(rp),
                       torch.empty(nnz, dtype=torch.int32, device="cuda"),
                       torch.empty(nnz, dtype=torch.float64, device="cuda"))
    ip = nb.intprod(dP, dP)[1]
    clocks = Clocks(index)
    clocks.start()
    ms = _timed(lambda: nb.spgemm(dP, dP, out=out, check_errors=False,
                                  row_kernel=args.row_kernel), args.form_steps, 1)
    clk = clocks.stop()
    _, st = nb.spgemm(dP, dP, out=out, return_stats=True, row_kernel=args.row_kernel)
    return {"workload": f"powerlaw_{args.pl_rows}_AxA_fp64", "nnz_A": P.nnz, "intprod": ip,
            "nnz_C": nnz, "ms": ms, "gflops": 2 * ip / ms / 1e6,
            "effective_gbs": alg_bytes(P, P, nnz) / (ms * 1e-3) / 1e9,
            "sym_bins": st["sym_bins"], "num_bins": st["num_bins"], "clocks": clk}


def _guarded(fn, *a):
    """A form's object, or its error: a failing form does not take the
    headline line with it (the error is in the line)."""
    import torch
    try:
        r = fn(*a)
    except Exception as ex:  # noqa: BLE001
        r = {"error": f"{type(ex).__name__}: {ex}"}
    torch.cuda.empty_cache()
    return r


def run_only_form(args, local):
    import torch
    torch.cuda.set_device(local)
    if args.only_form == "batched":
        res = form_batched(args, local)
    elif args.only_form == "fp32c":
        res = {"stencil": form_fp32c_one(args, local, "stencil"),
               "powerlaw": form_fp32c_one(args, local, "powerlaw")}
    elif args.only_form == "powerlaw":
        res = form_powerlaw(args, local)
    else:
        import nsp_b200 as nb
        A = nb.gen.stencil(L, npts=27, seed=SEED)
        res = form_reference_gpu(args, local, A, A.to_device())
    print(json.dumps({"form": args.only_form, **res}), flush=True)


def main():
    global L, METRIC, WORKLOAD
    args = parse()
    if args.grid != L:
        L = args.grid
        METRIC = f"SpGEMM GFLOP/s, C=A*A, 27-point stencil {L}^3, fp64"
        WORKLOAD = f"stencil27_{L}^3_AxA_fp64"
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.only_form:
        return run_only_form(args, local)

    import ctypes as C
    import torch
    import nsp_b200 as nb
    from nsp_b200 import _lib

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        pg = dist

    def barrier():
        if pg:
            pg.barrier()

    def max_over_ranks(x):
        if not pg:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x):
        if not pg:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.SUM)
        return float(t.item())

    Ah, Bh = local_problem(rank, world)
    dA = Ah.to_device(dev)
    dB = dA if Bh is Ah else Bh.to_device(dev)
    stream = torch.cuda.current_stream(dev)

    # size C once (symbolic), preallocate it, then time full products into it
    C0, st0 = nb.spgemm(dA, dB, return_stats=True)
    nnz_c = st0["nnz"]
    intprod = st0["intprod"]
    del C0
    out = nb.DeviceCSR(dA.nrows, dB.ncols,
                       torch.empty(dA.nrows + 1, dtype=torch.int32, device=dev),
                       torch.empty(nnz_c, dtype=torch.int32, device=dev),
                       torch.empty(nnz_c, dtype=torch.float64, device=dev))
    a_in, b_in = dA.as_in(), dB.as_in()
    c_out = _lib.CsrOut()
    c_out.rowptr, c_out.col, c_out.val = (out.rowptr.data_ptr(), out.col.data_ptr(),
                                          out.val.data_ptr())
    c_out.capacity = nnz_c
    opts = nb.make_opts(check_errors=False, stream=stream)
    opts.timing = 1
    opts.row_kernel = args.row_kernel
    stats = _lib.Stats()

    def step():
        _lib.check(nb.lib.nspb_spgemm(C.byref(a_in), C.byref(b_in), C.byref(c_out),
                                      C.byref(opts), C.byref(stats)), "nspb_spgemm")

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize(dev)
    clocks = Clocks(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    phase = {"ms_rowinfo": 0.0, "ms_symbolic": 0.0, "ms_scan": 0.0, "ms_numeric": 0.0}
    launches = 0
    barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
        for k in phase:
            phase[k] += getattr(stats, k)
        launches += stats.launches
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clk = clocks.stop()
    ms_local = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms_local)
    flops_all = sum_over_ranks(2.0 * intprod)
    value = flops_all / (ms * 1e-3) / 1e9
    for k in phase:
        phase[k] /= args.steps

    # correctness guard on the measured configuration: a final checked call
    opts.check_errors = 1
    step()
    torch.cuda.synchronize(dev)

    # ---- roofline of the dominant kernel
    peak, peak_kind = peaks()
    dominant = "numeric" if phase["ms_numeric"] >= phase["ms_symbolic"] else "symbolic"
    if dominant == "numeric":
        kbytes = alg_bytes(Ah, Bh, nnz_c)
        kms = phase["ms_numeric"]
        kname = NUM_KERNEL[bool(stats.entry_map)]
    else:
        kbytes = 4 * (Ah.nrows + 1) + 4 * Ah.nnz + 4 * (Bh.nrows + 1) + 4 * Bh.nnz + 4 * Ah.nrows
        kms = phase["ms_symbolic"]
        kname = SYM_KERNEL[bool(stats.entry_map)]
    achieved = kbytes / (kms * 1e-3) / 1e9 if kms > 0 else 0.0
    traffic = profiled_traffic(kname)

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if args.e2e_steps > 0:
        hA = [torch.from_numpy(x).pin_memory() for x in (Ah.rowptr, Ah.col, Ah.val)]
        hB = hA if Bh is Ah else [torch.from_numpy(x).pin_memory()
                                  for x in (Bh.rowptr, Bh.col, Bh.val)]
        hC = [torch.empty(dA.nrows + 1, dtype=torch.int32).pin_memory(),
              torch.empty(nnz_c, dtype=torch.int32).pin_memory(),
              torch.empty(nnz_c, dtype=torch.float64).pin_memory()]
        h2d = sum(x.numel() * x.element_size() for x in hA)
        if Bh is not Ah:
            h2d += sum(x.numel() * x.element_size() for x in hB)
        d2h = sum(x.numel() * x.element_size() for x in hC)

        class _Host:  # host CSR view over pinned tensors
            def __init__(self, m, arrs):
                self.nrows, self.ncols = m.nrows, m.ncols
                self.rowptr, self.col, self.val = arrs

        hAo = _Host(Ah, hA)
        hBo = hAo if Bh is Ah else _Host(Bh, hB)

        def e2e_step():
            # host operands in, host C out: copies overlapped with the product
            nb.spgemm_host(hAo, hBo, out=hC, stream=stream)

        e2e_step()
        torch.cuda.synchronize(dev)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        torch.cuda.synchronize(dev)
        e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.e2e_steps)
        e2e = {"value": flops_all / (e2e_ms * 1e-3) / 1e9, "unit": "GFLOP/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": e2e_ms, "steps": args.e2e_steps,
               "entry": "nspb_spgemm_host (C ABI, pinned host operands and C; structure "
                        "copied first, values in row chunks during the symbolic phase, C "
                        "copied back in row blocks under the numeric phase)"}

    # ---- CPU baseline (rank 0 at N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rows = sample_rows(Ah, Bh, threads, budget_s=10.0)
        v, dt = cpu_product_rate(Ah, Bh, rows, threads)
        cpu = {"value": v, "unit": "GFLOP/s", "cores": threads, "kind": "port",
               "sample": f"rows [0,{rows}) of {Ah.nrows} ({rows / Ah.nrows:.1%}) of the same "
                         f"product, {dt:.1f} s, OpenMP Gustavson oracle"}

    if pg:
        pg.barrier()
    if rank == 0:
        gbs = alg_bytes(Ah, Bh, nnz_c) * world / (ms * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic (seeded 27-point stencil, seed {SEED})",
            "config": {"workload": WORKLOAD, "grid": [L, L, L * world], "n_rows_per_gpu": dA.nrows,
                       "nnz_A_per_gpu": dA.nnz, "intprod_per_gpu": intprod,
                       "nnz_C_per_gpu": nnz_c,
                       "l2": f"inputs ({12 * dA.nnz / 1e6:.0f} MB) and C ({12 * nnz_c / 1e9:.2f} GB) "
                             "exceed the 126 MB L2; no flush",
                       "parallelism": "row z-slabs per GPU, halo planes generated locally, "
                                      "no collective"},
            "effective_gbs": gbs,
            "phases_ms": phase,
            "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes": kbytes,
                         "ms_per_launch": kms},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        if world == 1 and not args.no_forms:
            line["reference_gpu"] = _guarded(form_reference_gpu, args, local, Ah, dA)
            del out, dA, dB
            torch.cuda.empty_cache()
            line["forms"] = {
                "batched": _guarded(form_batched, args, local),
                "fp32c": {"stencil": _guarded(form_fp32c_one, args, local, "stencil"),
                          "powerlaw": _guarded(form_fp32c_one, args, local, "powerlaw")},
                "powerlaw_fp64": _guarded(form_powerlaw, args, local)}
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
