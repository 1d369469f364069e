"""SpMV throughput on one B200 (or N, one process per GPU): the power-law
workload (n = 4,000,000; lognormal(2.2, 1.0) row lengths; 70% of each row's
columns in a +/-1000 band, 30% uniform; seed 1), FP64.

One step = one y = A x through a plan (the format resident in HBM, x gathered
through L2).  The headline format is the compacted AXT (AXT COM, bs 128).
Inputs are larger than L2 (~0.8 GB streamed per step), so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--format COM128] [--workload powerlaw4m|poisson512|stencil160]
                    [--no-formats] [--no-cpu]

`--impl reference` times the reference's own CPU kernel (edoardoCB/int_spmv
intSpmv_main.c, compiled from its own source into oracle/_ref) for the same
format on the host cores, each step a bounded row sample of the workload.
Prints ONE JSON line on rank 0.
"""
from __future__ import annotations

import argparse
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

METRIC = "SpMV GFLOP/s"
UNIT = "GFLOP/s"
FALLBACK_HBM_GBS = 6650.0


# ------------------------------------------------------------- workloads --
def make_workload(name: str):
    from int_spmv_b200 import matrices as M
    if name == "powerlaw4m":
        row, col, val = M.powerlaw(4_000_000, seed=1)
        return dict(name="powerlaw_n4M_seed1", row=row, col=col, val=val, x=M.uniform_x(4_000_000, 1),
                    desc="power-law n=4,000,000, rl=clip(rint(lognormal(2.2,1.0)),1,5000), 70% band +/-1000, "
                         "30% uniform, N(0,1) values, x~U[-1,1], seed 1")
    if name == "powerlaw1m":
        row, col, val = M.powerlaw(1_000_000, seed=3)
        return dict(name="powerlaw_n1M_seed3", row=row, col=col, val=val, x=M.uniform_x(1_000_000, 3),
                    desc="power-law n=1,000,000 (same generator, seed 3)")
    if name == "stencil100":
        row, col, val = M.stencil27(100, seed=2)
        return dict(name="stencil27_100", row=row, col=col, val=val, x=M.uniform_x(100 ** 3, 2),
                    desc="3D 27-point stencil 100^3 (same generator, seed 2)")
    if name == "poisson512":
        row, col, val = M.poisson2d(512)
        return dict(name="poisson2d_512", row=row, col=col, val=val, x=M.uniform_x(512 * 512, 0),
                    desc="2D 5-point Poisson 512x512, natural order, x~U[-1,1] seed 0")
    if name == "stencil160":
        row, col, val = M.stencil27(160, seed=2)
        return dict(name="stencil27_160", row=row, col=col, val=val, x=M.uniform_x(160 ** 3, 2),
                    desc="3D 27-point stencil 160^3, diag 26, off -1+U[-0.1,0.1], seed 2")
    raise ValueError(name)


def build_format(F, csr, x, fmt: str):
    """fmt: CSR | AXC | K1 | K1P | NOC<th> | COM<bs>.  Returns the host format
    object (None for CSR) and the reference format name."""
    if fmt == "CSR":
        return None, "CSR"
    if fmt == "AXC":
        return F.getFormatDataAXC(0, csr, x)[1], "AXC"
    if fmt in ("K1", "K1P"):
        return F.getFormatDataK1(8, csr, x)[1], fmt
    if fmt.startswith("NOC"):
        th = int(fmt[3:])
        return F.getFormatDataAXT(0, 128, 8, th, "NOC", csr, x)[1], f"AXT_NOC_H{th}_HW8"
    if fmt.startswith("COM"):
        bs = int(fmt[3:])
        return F.getFormatDataAXT(0, bs, 8, 1, "COM", csr, x)[1], f"AXT_COM_H1_HW8_BS{bs}"
    raise ValueError(fmt)


VALUE_KIND = {"f64": "FP64 values, FP64 accumulate", "f32": "FP32 values, FP32 multiply, FP64 accumulate",
              "f32lo": "FP32 values + BF16 lo-word, FP64 accumulate"}


def run_config(wl, fmt_name: str, val: str, col: str, B: float) -> dict:
    """The workload both arms run (ours and --impl reference print the same
    dict): matrix, format, value and column form, L2 handling."""
    return {"workload": wl["name"], "format": fmt_name, "n": len(wl["row"]) - 1, "nnz": len(wl["col"]),
            "value_kind": VALUE_KIND[val] + (", u32 columns" if col == "u32" else ", 16-bit column deltas"),
            "l2": "no flush: inputs larger than L2 (%.0f MB algorithmic bytes per step)" % (B / 1e6),
            "parallelism": "replicas (one full matrix per process, no collective)"}


def format_name(fmt: str) -> str:
    """The reference's name of a bench format (getFormatData*, intSpmv_main.c:324-1381)."""
    if fmt in ("CSR", "AXC", "K1", "K1P"):
        return fmt
    if fmt.startswith("NOC"):
        return f"AXT_NOC_H{int(fmt[3:])}_HW8"
    return f"AXT_COM_H1_HW8_BS{int(fmt[3:])}"


def alg_bytes(n: int, nnz: int, bval: int = 8) -> float:
    """nnz*(b_val + b_idx) + n*(b_x + b_y) + 4*(n+1)."""
    return nnz * (bval + 4.0) + n * 16.0 + 4.0 * (n + 1)


# --------------------------------------------------------------- helpers --
def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def traffic_for(kernel_key: str):
    """dram bytes per launch from a committed ncu summary, if one exists."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    try:
        d = json.loads(p.read_text())
        return d.get(kernel_key)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled in the background."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, period_ms: int = 100):
        self.samples, self.proc, self.t = [], None, None
        self.gpu, self.period = gpu_index, period_ms

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.period)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.time(), [s.strip() for s in line.split(",")]))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, t0: float, t1: float):
        win = [s for t, s in self.samples if t0 <= t <= t1] or [s for _, s in self.samples]
        if not win:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(s[1]) for s in win if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in win if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in win for i in range(4) if len(s) > 5 + i and s[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(win),
                "power_w_max": max(float(s[3]) for s in win if s[3].replace(".", "").isdigit()) if win else None}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), ws


def max_over_ranks(v: float, ws: int, device=None) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rest(ws: int, seconds: float = 1.5):
    """Drain the device, idle `seconds`, then meet the other ranks: a
    measurement that follows starts from a rested GPU."""
    import torch
    torch.cuda.synchronize()
    time.sleep(seconds)
    barrier(ws)


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def timed(step, steps: int, warmup: int, ws: int, stream, device=None):
    """W untimed steps, then exactly K steps between barrier + synchronize,
    timed with CUDA events on `stream`; returns the max over ranks [s]."""
    import torch
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_wall0 = time.time()
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    t_wall1 = time.time()
    barrier(ws)
    sec = e0.elapsed_time(e1) / 1e3
    return max_over_ranks(sec, ws, device), (t_wall0, t_wall1)


# ------------------------------------------------------- reference (CPU) --
def reference_time(row, col, val, x, fmt: str, budget_s: float, calls: int | None = None, row_frac: float = 1.0,
                   warm: int = 1):
    """The reference's own kernel for `fmt` on the host cores: builds the
    reference format with the reference builder, then times its kernel
    (its gettimeofday timing).  Returns (sec/call, nnz of the sample, info)."""
    from oracle import Reference
    R = Reference()
    n = len(row) - 1
    nr = max(1, int(n * row_frac))
    srow = row[:nr + 1]
    snnz = int(srow[-1])
    s = R.csr(srow, col[:snnz], val[:snnz])
    s._keep[3][:] = np.diff(srow)
    cores = os.cpu_count() or 1
    kind, mat, bs, work = None, None, 0, 0
    if fmt == "CSR":
        kind, mat = "cf_CSR", s
        cores = 1  # the reference's cf_CSR is serial (intSpmv_main.c:386)
    elif fmt == "AXC":
        d = R.build_axc(s, x, ompNT=cores)
        kind, mat = "int_axc", d["struct"]
    elif fmt in ("K1", "K1P"):
        d = R.build_k1(s, x)
        kind, mat, work = ("int_k1" if fmt == "K1" else "int_k1p"), d["struct"], d["chunkNum"] * 8
    elif fmt.startswith("NOC"):
        th = int(fmt[3:])
        d = R.build_axt(s, x, 8, th, "NOC", 128, ompNT=cores)
        kind, mat = ("int_axt_noc_h1" if th == 1 else "int_axt_noc"), d["struct"]
    else:
        bs = int(fmt[3:])
        d = R.build_axt(s, x, 8, 1, "COM", bs, ompNT=cores)
        kind, mat = "int_axt_com_h1", d["struct"]
    et, _, _ = R.time_kernel(kind, mat, x, nr, work_len=work, bs=bs, iters=max(1, warm), ompNT=cores)
    if calls is None:
        calls = int(max(3, min(200, budget_s / max(et, 1e-6))))
    et, ot, _ = R.time_kernel(kind, mat, x, nr, work_len=work, bs=bs, iters=calls, ompNT=cores)
    if fmt == "K1":
        et += ot
    return et, snnz, dict(kernel=kind, calls=calls, cores=cores, rows=nr)


# ------------------------------------------------------------------ main --
def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="powerlaw4m")
    ap.add_argument("--format", default="COM128")
    ap.add_argument("--kernel", default="auto", choices=["auto", "ldg", "tma", "rows", "wide"])
    ap.add_argument("--variant", type=int, default=-1, help="kernel variant (-1: the tuned default)")
    ap.add_argument("--val", default="f64", choices=["f64", "f32", "f32lo"],
                    help="value storage: FP64, or FP32 (+ BF16 lo-word) multiplied in FP32, FP64 accumulation")
    ap.add_argument("--col", default="u32", choices=["u32", "d16"], help="column storage: u32 or 16-bit deltas")
    ap.add_argument("--mode", default="spmv", choices=["spmv", "spmm", "batch"],
                    help="spmv: one matrix (default); spmm: Y = A X for k right-hand sides; batch: many "
                         "uneven banded matrices in one graph launch vs one plan per matrix")
    ap.add_argument("--spmm-k", default="8,16,32", help="--mode spmm: right-hand-side counts, comma-separated")
    ap.add_argument("--spmm-vals", default="f64,f32", help="--mode spmm: value forms, comma-separated (f64, f32)")
    ap.add_argument("--spmm-plan", default="tuned", choices=["tuned", "com128"],
                    help="--mode spmm: the autotuner's plan per case, or AUTO on AXT COM bs128")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--batch-nmax", type=float, default=2e5, help="largest n of the batched matrices")
    ap.add_argument("--no-formats", action="store_true", help="skip the per-format table")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the SpMM and batched lines (1M-row SpMM k = 8/16/32; 512 banded matrices)")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the FP64 / FP32-value lines on the 27-point stencil 160^3")
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of reference CPU work")
    a = ap.parse_args(argv)
    rank, local_rank, ws = dist_env()
    W = max(3, a.warmup)

    if a.impl == "reference":
        return main_reference(a, rank, ws, W)
    if a.mode == "spmm":
        return main_spmm(a, rank, ws, W)
    if a.mode == "batch":
        return main_batch(a, rank, ws, W)

    import torch
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from int_spmv_b200 import _lib
    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    wl = make_workload(a.workload)
    csr = F.CSR(wl["row"], wl["col"], wl["val"])
    n, nnz = csr.n, csr.nnz
    fmt_obj, fmt_name = build_format(F, csr, wl["x"], a.format)
    plan = D.Plan(csr, fmt_obj, kernel=a.kernel, variant=max(a.variant, 0), val=a.val, col=a.col,
                  reorder=a.format != "K1")
    del fmt_obj
    stream = torch.cuda.current_stream()
    x = torch.from_numpy(wl["x"]).to(dev)
    y = torch.empty(n, dtype=torch.float64, device=dev)
    flops = 2.0 * nnz
    B = plan.info["alg_bytes"]  # nnz*(b_val + b_idx) + n*16 + 4*(n+1) for this value / column form

    l0 = _lib.launch_count()
    plan.spmv(x, y)
    per_step = _lib.launch_count() - l0  # library kernel launches in one step
    try:
        gpu_id = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        gpu_id = str(local_rank)
    sampler = ClockSampler(gpu_id)
    sampler.start()
    time.sleep(0.3)
    sec, (tw0, tw1) = timed(lambda: plan.spmv(x, y), a.steps, W, ws, stream, dev)
    # the same K steps again with an event pair around each main kernel
    plan.time_kernels(a.steps)
    sec_k, _ = timed(lambda: plan.spmv(x, y), a.steps, 3, ws, stream, dev)
    kms, klaunches = plan.kernel_ms()
    plan.time_kernels(0)
    kern_ev_s = max_over_ranks(kms / 1e3 / max(klaunches, 1), ws, dev)
    # the dominant kernel's average launch duration for the roofline: five
    # chunks of at least max(K, 200)/5 launches of the main kernel back to
    # back, each between one event pair (an event pair around each launch
    # adds the event records' gaps to every launch), after 3 untimed ones;
    # the median chunk, every chunk reported; then one product restores y.
    # Measured from a rested GPU, as the HBM peak (a best-of-10 copy) is: on
    # these boxes ~100 ms of back-to-back HBM-bound work slows this kernel by
    # up to 8%, and ~2 s idle restores it
    rest(ws)
    plan.time_main(x, y, 3)
    per_chunk = max(20, max(a.steps, 200) // 5)
    chunks = [plan.time_main(x, y, per_chunk) for _ in range(5)]
    kern_s = max_over_ranks(float(np.median(chunks)) / 1e3, ws, dev)
    tw2 = time.time()
    plan.spmv(x, y)
    torch.cuda.synchronize()
    time.sleep(0.25)
    sampler.stop()
    clocks = sampler.summary(tw0, tw2)
    ms = sec / a.steps * 1e3
    value = ws * a.steps * flops / sec / 1e9
    gbs = B / (sec / a.steps) / 1e9
    kern_gbs = B / kern_s / 1e9
    kname = plan.kernel_name()
    peak, peak_src = hbm_peak()

    # end to end through the public API on pinned host buffers
    hx = torch.from_numpy(wl["x"].copy()).pin_memory()
    hy = torch.empty(n, dtype=torch.float64).pin_memory()
    e2e_steps = max(3, min(a.steps, 300))
    sec_e2e, _ = timed(lambda: plan.spmv_host(hx, hy), e2e_steps, 3, ws, stream, dev)
    e2e = {"value": ws * e2e_steps * flops / sec_e2e / 1e9, "unit": UNIT, "h2d_bytes_per_step": 8 * n,
           "d2h_bytes_per_step": 8 * n, "steps": e2e_steps, "ms_per_step": sec_e2e / e2e_steps * 1e3}

    # parity of this run's y against the oracle (the checker, not the product)
    check = None
    if rank == 0:
        from oracle import Oracle
        orc = Oracle()
        plan.spmv(x, y)
        yr = orc.cf_csr(wl["row"], wl["col"], wl["val"], wl["x"])
        ab = orc.abs_csr(wl["row"], wl["col"], wl["val"], wl["x"])
        err = np.abs(y.cpu().numpy() - yr)
        tol = 1e-12 if a.val == "f64" else 1e-6
        check = {"max_componentwise": float(np.max(err / np.maximum(ab, 1e-300))), "bound": tol,
                 "pass": bool(np.all(err <= tol * ab)),
                 "normwise": float(np.linalg.norm(err) / np.linalg.norm(yr))}

    # every format and value/column form on the same matrix: time, the
    # fraction of the roofline of its own algorithmic bytes, and its error
    formats = {}
    if not a.no_formats:
        variants = [(f, "f64", "u32", "auto") for f in ["CSR", "AXC", "K1", "K1P", "NOC1", "NOC4", "NOC8",
                                                           "NOC16", "COM128", "COM256", "COM512"]]
        variants += [("CSR", "f64", "u32", "rows"), ("AXC", "f64", "u32", "rows"), ("NOC1", "f64", "u32", "ldg"),
                     ("COM128", "f64", "u32", "ldg"), ("NOC4", "f64", "u32", "ldg"), ("NOC8", "f64", "u32", "ldg"),
                     ("NOC4", "f64", "u32", "tma"), ("COM128", "f64", "u32", "tma")]
        variants += [(f, vk, ck, "auto") for f in ("COM128", "NOC1")
                     for vk, ck in (("f32", "u32"), ("f64", "d16"), ("f32", "d16"))]
        variants += [(f, vk, ck, "ldg") for f in ("COM128", "NOC1")
                     for vk, ck in (("f32", "u32"), ("f32lo", "u32"), ("f64", "d16"), ("f32", "d16"),
                                    ("f32lo", "d16"))]
        for f, vk, ck, kern in variants:
            fo, _ = build_format(F, csr, wl["x"], f)
            try:
                p = D.Plan(csr, fo, val=vk, col=ck, kernel=kern, reorder=f != "K1")
            except Exception as e:  # a form this format does not take
                formats[f"{f}/{vk}/{ck}/{kern}"] = {"unsupported": str(e)[:80]}
                continue
            finally:
                del fo
            k = max(20, min(a.steps, 400))
            s_, _ = timed(lambda: p.spmv(x, y), k, 5, ws, stream, dev)
            t = s_ / k
            # the main kernel alone (k launches back to back, from a rested
            # GPU); for K1 the rest of the step is the reorder pass, the
            # reference's ordTime (intSpmv_main.c:1001-1016)
            rest(ws, 0.5)
            p.time_main(x, y, 3)
            tk = max_over_ranks(p.time_main(x, y, k) / 1e3, ws, dev)
            bb = p.info["alg_bytes"]
            kid = {0: "auto", 1: "ldg", 2: "tma", 3: "rows", 4: "wide"}.get(p.info["kernel"], "?")
            row_ = {"ms": t * 1e3, "gflops": flops / t / 1e9, "gbs": bb / t / 1e9, "frac": bb / t / 1e9 / peak,
                    "kernel_ms": tk * 1e3, "kernel_frac": bb / tk / 1e9 / peak, "kernel": p.kernel_name()}
            if f == "K1":
                row_["ord_ms"] = max(0.0, (t - tk) * 1e3)
            if check is not None:
                p.spmv(x, y)
                yh = y.cpu().numpy()
                e_ = np.abs(yh - yr)
                row_["max_componentwise_err"] = float(np.max(e_ / np.maximum(ab, 1e-300)))
                row_["normwise_err"] = float(np.linalg.norm(e_) / np.linalg.norm(yr))
                aerr, rerr, pos = F.getErrors(yr, yh)  # the reference's own columns (intSpmv_main.c:404-425)
                row_.update(aErr=aerr, rErr=rerr, pos=int(pos))
            formats[f"{p.info['name']}/{vk}/{ck}/{kid}"] = row_
            del p
        # the vendor library on the same CSR, as a comparison row only (never
        # the product path): torch's CSR matrix-vector product, cuSPARSE SpMV
        try:
            A = torch.sparse_csr_tensor(torch.from_numpy(wl["row"].astype(np.int32)).to(dev),
                                        torch.from_numpy(wl["col"].astype(np.int32)).to(dev),
                                        torch.from_numpy(wl["val"]).to(dev), size=(n, n))
            k = max(20, min(a.steps, 400))
            s_, _ = timed(lambda: torch.mv(A, x), k, 5, ws, stream, dev)
            t = s_ / k
            row_ = {"ms": t * 1e3, "gflops": flops / t / 1e9, "gbs": B / t / 1e9, "frac": B / t / 1e9 / peak,
                    "kernel": "cuSPARSE SpMV via torch.sparse (library comparison, not the product)"}
            if check is not None:
                e_ = np.abs(torch.mv(A, x).cpu().numpy() - yr)
                row_["max_componentwise_err"] = float(np.max(e_ / np.maximum(ab, 1e-300)))
            formats["cuSPARSE_CSR/f64/i32/library"] = row_
            del A
        except Exception as e:  # the comparison row must not sink the run
            formats["cuSPARSE_CSR/f64/i32/library"] = {"unavailable": str(e)[:120]}

    # the precision target on the 27-point stencil 160^3: plain FP64 against
    # the reduced-byte forms, each with the kernel AUTO picks, its own
    # algorithmic bytes and its error against the FP64 oracle
    precision = None
    if not a.no_precision and a.workload != "stencil160":
        try:
            precision = precision_lines(a, rank, ws, stream, dev, peak)
        except Exception as e:  # the extra lines must not sink the headline
            precision = {"unavailable": str(e)[:160]}

    # multi-RHS SpMM (AUTO's plan) and the 512 batched matrices in one graph
    # launch, on one GPU (rank 0 of a single-process run)
    spmm = batched = None
    if ws == 1 and not a.no_extras:
        try:
            spmm, _ = spmm_lines(max(20, min(a.steps, 200)), 5, False, peak)
        except Exception as e:  # the extra lines must not sink the headline
            spmm = {"unavailable": str(e)[:160]}
        try:
            batched = batch_lines(a, max(20, min(a.steps, 200)), 5, peak)
        except Exception as e:
            batched = {"unavailable": str(e)[:160]}

    # format conversion: the host builder (OpenMP, the reference's layout
    # rules) against the same conversion on the GPU, for the compacted AXT
    conversion = None
    if not a.no_formats:
        try:
            fd_h, _ = F.getFormatDataAXT(0, 128, 8, 1, "COM", csr, wl["x"])
            drow, dcol, dval = D.to_device(wl["row"]), D.to_device(wl["col"]), D.to_device(wl["val"])
            dv_s = []
            for _ in range(2):  # the first call also loads the builder's kernels
                dv = D.DeviceAXT(drow, dcol, dval, x, bs=128, th=1, mode="COM")
                dv_s.append(dv.conversion_s)
                del dv
            dv_s = dv_s[-1]
            # the plan itself (the compacted AXT's lane-interleaved stream)
            # from the host CSR and from the device CSR, wall clock
            plan_s = {}
            t0 = time.perf_counter()
            ph = D.Plan(csr, None, kernel="wide", variant=4)
            plan_s["host_s"] = time.perf_counter() - t0
            del ph
            for _ in range(2):  # the first call also loads the builder's kernels
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                pdv = D.Plan.from_device_csr(drow, dcol, dval, kernel="wide", variant=4)
                plan_s["gpu_s"] = time.perf_counter() - t0
                del pdv
            del drow, dcol, dval
            conversion = {"format": "AXT_COM_H1_HW8_BS128", "host_s": fd_h.ct, "host_threads": os.cpu_count(),
                          "gpu_s": dv_s, "note": "host: getFormatDataAXT (ispmv_build_axt, wall clock); "
                                                 "gpu: ispmv_dev_build_axt on device CSR + x (CUDA events)",
                          "plan": dict(plan_s, note="plan of the lane-interleaved stream (variant 4): "
                                                    "ispmv_plan_csr from host CSR vs ispmv_plan_dev_csr from "
                                                    "device CSR, wall clock including synchronisation")}
        except Exception as e:
            conversion = {"unavailable": str(e)[:120]}

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu:
        try:
            from oracle import Reference
            if Reference.available():
                et, snnz, info = reference_time(wl["row"], wl["col"], wl["val"], wl["x"], a.format, a.cpu_budget)
                cpu = {"value": 2.0 * snnz / et / 1e9, "unit": UNIT, "cores": info["cores"], "kind": "reference",
                       "sample": f"{info['kernel']} (intSpmv_main.c) on the full workload, {info['calls']} calls, "
                                 f"{info['cores']} OpenMP threads; x is baked into ax by the reference builder"}
            else:
                cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                       "sample": "unavailable: oracle/_ref missing or host lacks AVX-512"}
        except Exception as e:  # the baseline must not sink the run
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": a.steps, "warmup": W,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"f64": "f64", "f32": "f32-mul/f64-acc", "f32lo": "f32+bf16lo-mul/f64-acc"}[a.val],
            "data": f"synthetic: {wl['desc']} (int_spmv_b200/matrices.py)",
            "config": run_config(wl, fmt_name, a.val, a.col, alg_bytes(n, nnz, {"f64": 8, "f32": 4, "f32lo": 4}[a.val])),
            "kernel": {"family": {0: "auto", 1: "ldg", 2: "tma", 3: "rows", 4: "wide"}.get(plan.info["kernel"], "?"),
                       "name": kname, "replicas": ws},
            "gb_per_s": gbs,
            "roofline": {"bound": "hbm", "achieved": kern_gbs, "peak": peak, "unit": "GB/s",
                         "frac": kern_gbs / peak, "traffic": traffic_for(f"{wl['name']}/{a.format}/{kname}"),
                         "kernel": kname, "kernel_ms": kern_s * 1e3, "kernel_launches": 5 * per_chunk,
                         "kernel_ms_chunks": chunks,
                         "kernel_ms_event_pairs": kern_ev_s * 1e3, "event_pair_launches": klaunches,
                         "step_gbs": gbs, "step_frac": gbs / peak, "peak_source": peak_src,
                         "note": "achieved = algorithmic bytes of one SpMV (nnz*(b_val+b_idx) + n*16 + 4*(n+1)) / the main "
                                 "kernel's mean duration over launches back to back between one CUDA event pair "
                                 "(ispmv_plan_time_main), the median of 5 such chunks (kernel_ms_chunks), timed "
                                 "from a rested GPU (1.5 s idle first) as the HBM peak's best-of-10 copy is; "
                                 "kernel_ms_event_pairs is the mean of an event pair around "
                                 "each main kernel inside K whole steps; step_gbs uses the whole step (main kernel + "
                                 "row fix-up, a programmatic dependent launch)"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(round(per_step * a.steps)),
            "clocks": clocks,
            "parity": check,
            "formats": formats,
            "precision": precision,
            "spmm": spmm,
            "batched": batched,
            "conversion": conversion,
        }
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def precision_lines(a, rank, ws, stream, dev, peak):
    """FP64 against the reduced-byte forms on the 3D 27-point stencil 160^3
    (n = 4,096,000, nnz = 109,215,352; diagonal 26, off-diagonal
    -1 + U[-0.1, 0.1], seed 2), compacted AXT bs 128, each form on the kernel
    AUTO picks: step and main-kernel time, GB/s of the form's own
    algorithmic bytes (b_val = 8 or 4, b_idx = 4, or 2 + the per-batch bases
    for 16-bit deltas), the fraction of the HBM peak, and the error against
    the FP64 oracle; then the speed-up of each form over FP64."""
    import torch

    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    wl = make_workload("stencil160")
    csr = F.CSR(wl["row"], wl["col"], wl["val"])
    com = F.getFormatDataAXT(0, 128, 8, 1, "COM", csr, wl["x"])[1]
    x = torch.from_numpy(wl["x"]).to(dev)
    y = torch.empty(csr.n, dtype=torch.float64, device=dev)
    yr = ab = None
    if rank == 0:
        from oracle import Oracle
        orc = Oracle()
        yr = orc.cf_csr(wl["row"], wl["col"], wl["val"], wl["x"])
        ab = orc.abs_csr(wl["row"], wl["col"], wl["val"], wl["x"])
    k = max(200, min(a.steps, 2000))
    out = {"workload": wl["name"], "n": csr.n, "nnz": csr.nnz, "format": "AXT_COM_H1_HW8_BS128", "steps": k}
    forms = [("f64", "u32", "f64/u32", {}), ("f32", "u32", "f32/u32", {}), ("f32", "d16", "f32/d16", {}),
             ("f64", "d16", "f64/d16", {}), ("f32lo", "u32", "f32lo/u32", {}),
             ("f64", "u32", "f64/u32/plain-loads", dict(kernel="wide", variant=0))]
    for vk, ck, key, kw in forms:
        p = D.Plan(csr, com, val=vk, col=ck, **kw)
        s_, _ = timed(lambda: p.spmv(x, y), k, 5, ws, stream, dev)
        rest(ws, 0.5)
        p.time_main(x, y, 3)
        t, tk = s_ / k, max_over_ranks(p.time_main(x, y, k) / 1e3, ws, dev)
        bb = p.info["alg_bytes"]
        row = {"ms": t * 1e3, "kernel_ms": tk * 1e3, "gflops": 2.0 * csr.nnz / t / 1e9, "alg_bytes": bb,
               "gbs": bb / tk / 1e9, "frac": bb / tk / 1e9 / peak, "kernel": p.kernel_name(),
               "bound": 1e-12 if vk == "f64" else 1e-6}
        if rank == 0:
            p.spmv(x, y)
            yh = y.cpu().numpy()
            e = np.abs(yh - yr)
            row["max_componentwise_err"] = float(np.max(e / np.maximum(ab, 1e-300)))
            row["normwise_err"] = float(np.linalg.norm(e) / np.linalg.norm(yr))
            row["pass"] = bool(np.all(e <= row["bound"] * ab))
            aerr, rerr, pos = F.getErrors(yr, yh)
            row.update(aErr=aerr, rErr=rerr, pos=int(pos))
        out[key] = row
        del p
    # against the FP64 plan AUTO picks (the fastest FP64 kernel on this
    # matrix), and against the same lane-interleaved plain-load kernel in FP64
    for bk, name in (("f64/u32", "speedup_vs_f64"), ("f64/u32/plain-loads", "speedup_vs_f64_plain_loads")):
        base = out[bk]
        out[name] = {f: {"step": base["ms"] / out[f]["ms"], "kernel": base["kernel_ms"] / out[f]["kernel_ms"]}
                     for f in ("f32/u32", "f32/d16", "f64/d16", "f32lo/u32")}
    out["target"] = "FP32 values / FP64 accumulate >= 1.4x plain FP64 at <= 1e-6 relative error"
    return out


def _event_time(fn, steps: int, warmup: int) -> float:
    """Seconds per call of fn, CUDA events on the current stream."""
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
    return e0.elapsed_time(e1) / 1e3 / steps


def spmm_lines(steps: int, warmup: int, tuned: bool, peak: float, ks=(8, 16, 32), vals=("f64", "f32")):
    """Y = A X on the power-law generator at n = 1,000,000 (seed 3), X n x k
    row-major U[-1, 1], k in `ks` (8, 16, 32), values in `vals` (FP64, FP32).
    The plan is the autotuner's choice (tuned) or AUTO's compacted AXT (bs 128).  Per
    (value form, k): time, GFLOP/s, GB/s and the HBM fraction of
    nnz*(b_val + 4) + n*k*16 + 4*(n+1) (A read once, X and Y once), and the
    error of every column against the oracle.  Returns (results, launches)."""
    import torch
    from int_spmv_b200 import _lib, autotune
    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from oracle import Oracle
    wl = make_workload("powerlaw1m")
    csr = F.CSR(wl["row"], wl["col"], wl["val"])
    n, nnz = csr.n, csr.nnz
    orc = Oracle()
    com = None if tuned else F.getFormatDataAXT(0, 128, 8, 1, "COM", csr, wl["x"])[1]
    res, launches = {}, 0
    for val in vals:
        for k in ks:
            if tuned:
                plan, choice = autotune.best_plan(csr, wl["x"], val=val, k=k, use_cache=False)
            else:
                plan, choice = D.Plan(csr, com, val=val), {"format": "COM128", "kwargs": {}}
            X = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, (n, k))).cuda()
            Y = torch.empty_like(X)
            l0 = _lib.launch_count()
            plan.spmm(X, Y)
            per = _lib.launch_count() - l0
            t = _event_time(lambda: plan.spmm(X, Y), steps, warmup)
            launches += per * steps
            plan.spmm(X, Y)
            Yh, Xh = Y.cpu().numpy(), X.cpu().numpy()
            err = 0.0
            for j in range(k):
                xj = np.ascontiguousarray(Xh[:, j])
                ref, ab = orc.cf_csr(wl["row"], wl["col"], wl["val"], xj), orc.abs_csr(wl["row"], wl["col"], wl["val"], xj)
                err = max(err, float(np.max(np.abs(Yh[:, j] - ref) / np.maximum(ab, 1e-300))))
            bval = 8 if val == "f64" else 4
            B = nnz * (bval + 4) + n * k * 16 + 4 * (n + 1)
            res[f"{val}/k{k}"] = {"ms": t * 1e3, "gflops": 2 * nnz * k / t / 1e9, "gbs": B / t / 1e9,
                                  "alg_bytes": B, "frac": B / t / 1e9 / peak, "kernel": plan.kernel_name(),
                                  "format": choice["format"], "kwargs": choice["kwargs"],
                                  "max_componentwise_err": err, "bound": 1e-12 if val == "f64" else 1e-6,
                                  "rhs_columns_checked": k}
            del plan, X, Y
    return dict(workload="spmm_powerlaw_n1M_seed3", n=n, nnz=nnz, steps=steps, **res), launches


def main_spmm(a, rank, ws, W):
    """The SpMM workload alone (spmm_lines with the autotuner's plans)."""
    import torch
    torch.cuda.set_device(0)
    peak, peak_src = hbm_peak()
    ks = tuple(int(k) for k in a.spmm_k.split(","))
    vals = tuple(a.spmm_vals.split(","))
    res, launches = spmm_lines(a.steps, W, a.spmm_plan == "tuned", peak, ks, vals)
    head = f"{vals[0]}/k{max(ks)}"
    best = res[head]
    out = {"metric": "SpMM GFLOP/s (2*nnz*k)", "value": best["gflops"], "unit": "GFLOP/s", "n_gpus": 1,
           "steps": a.steps, "warmup": W, "ms_per_step": best["ms"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": vals[0], "data": "synthetic: power-law n=1,000,000 seed 3, X~U[-1,1]",
           "config": {"workload": "spmm_powerlaw_n1M_seed3", "n": res["n"], "nnz": res["nnz"], "k": list(ks),
                      "choice": "autotuned per (value form, k)" if a.spmm_plan == "tuned" else "AUTO on AXT COM bs128"},
           "gpu_launches": launches,
           "roofline": {"bound": "hbm", "achieved": best["gbs"], "peak": peak, "unit": "GB/s",
                        "frac": best["frac"], "traffic": None, "kernel": best["kernel"], "peak_source": peak_src,
                        "note": f"achieved = (nnz*(b_val+4) + n*k*16 + 4*(n+1)) / step time, {head}"},
           "results": res}
    print(json.dumps(out), flush=True)


def batch_lines(a, steps: int, warmup: int, peak: float) -> dict:
    """Many uneven FEM-like banded matrices (n log-uniform in [1e3, nmax],
    rows of 7-81 entries within +/-3*rl of the diagonal; seed 4), each with
    its own x: one block-diagonal plan in one CUDA-graph launch (the
    lane-interleaved kernel, and the persistent work-queue kernel), against
    one plan per matrix launched one after the other.  Every matrix of the
    graph launch is checked against its own oracle product."""
    import torch
    from int_spmv_b200 import _lib
    from int_spmv_b200 import batch as BT
    from int_spmv_b200 import device as D
    from int_spmv_b200 import formats as F
    from int_spmv_b200 import matrices as M
    from oracle import Oracle
    t0 = time.time()
    mats = M.fem_batch_c(count=a.batch_count, seed=4, n_lo=1e3, n_hi=a.batch_nmax)
    big, off = BT.blockdiag(mats)
    n, nnz = big.n, big.nnz
    x = M.uniform_x(n, 4)
    xt = torch.from_numpy(x).cuda()
    res = {}
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    for name, kw in (("graph_wide", dict(kernel="wide")), ("graph_queue", dict(kernel="ldg", variant=16))):
        plan = D.Plan(big, None, val=a.val, **kw)
        l0 = _lib.launch_count()
        plan.spmv_graph(xt, y)  # captures the product's kernels, then launches the graph once
        in_graph = _lib.launch_count() - l0 - 1
        torch.cuda.synchronize()
        t = _event_time(lambda: plan.spmv_graph(xt, y), steps, warmup)
        bb = plan.info["alg_bytes"]
        res[name] = {"ms": t * 1e3, "gflops": 2 * nnz / t / 1e9, "gbs": bb / t / 1e9, "frac": bb / t / 1e9 / peak,
                     "kernel": plan.kernel_name(), "graph_launches_per_step": 1, "kernels_in_graph": in_graph}
        if name == "graph_wide":
            plan.spmv_graph(xt, y)
            yb = y.cpu().numpy()
        del plan
    del big
    # one plan per matrix, launched one after the other (2 launches each)
    plans, ys, xs = [], [], []
    for m, (row, col, val) in enumerate(mats):
        csr = F.CSR(row, col, val)
        plans.append(D.Plan(csr, None, kernel="wide", val=a.val))
        xs.append(xt[int(off[m]):int(off[m + 1])])
        ys.append(y[int(off[m]):int(off[m + 1])])

    def each():
        for p_, x_, y_ in zip(plans, xs, ys):
            p_.spmv(x_, y_)
    l0 = _lib.launch_count()
    each()
    per = _lib.launch_count() - l0
    t = _event_time(each, max(3, steps // 4), warmup)
    res["separate"] = {"ms": t * 1e3, "gflops": 2 * nnz / t / 1e9, "launches_per_step": per}
    del plans
    # parity: every matrix of the graph launch against the oracle
    orc, err = Oracle(), 0.0
    tol = 1e-12 if a.val == "f64" else 1e-6
    for m, (row, col, val) in enumerate(mats):
        a0, a1 = int(off[m]), int(off[m + 1])
        ref, ab = orc.cf_csr(row, col, val, x[a0:a1]), orc.abs_csr(row, col, val, x[a0:a1])
        err = max(err, float(np.max(np.abs(yb[a0:a1] - ref) / np.maximum(ab, 1e-300))))
    return {"workload": f"fem_batch_{a.batch_count}_nmax{a.batch_nmax:g}", "matrices": len(mats), "n": n, "nnz": nnz,
            "value_kind": a.val, "steps": steps, "results": res,
            "speedup_graph_vs_separate": res["separate"]["ms"] / res["graph_wide"]["ms"],
            "parity": {"max_componentwise": err, "bound": tol, "pass": err <= tol, "matrices_checked": len(mats)},
            "setup_s": time.time() - t0}


def main_batch(a, rank, ws, W):
    """The batched workload alone (batch_lines)."""
    import torch
    torch.cuda.set_device(0)
    peak, _ = hbm_peak()
    r = batch_lines(a, a.steps, W, peak)
    g = r["results"]["graph_wide"]
    out = {"metric": "batched SpMV GFLOP/s (2*sum nnz)", "value": g["gflops"], "unit": "GFLOP/s",
           "n_gpus": 1, "steps": a.steps, "warmup": W, "ms_per_step": g["ms"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64" if a.val == "f64" else "f32-mul/f64-acc",
           "data": f"synthetic: {a.batch_count} banded FEM-like matrices, n log-uniform in [1e3, {a.batch_nmax:g}], "
                   "rl U[7,81] within +/-3 rl, seed 4 (int_spmv_b200/matrices.py fem_batch_c)",
           "config": {"workload": r["workload"], "matrices": r["matrices"], "n": r["n"], "nnz": r["nnz"],
                      "value_kind": a.val},
           "gpu_launches": a.steps * g["kernels_in_graph"], **{k: r[k] for k in ("speedup_graph_vs_separate",
                                                                                 "parity", "results", "setup_s")}}
    print(json.dumps(out), flush=True)


def main_reference(a, rank, ws, W):
    """The reference's own CPU path on the host cores (rank 0 only)."""
    if rank != 0:
        return
    from oracle import Reference
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref missing or the host lacks AVX-512"}))
        return
    wl = make_workload(a.workload)
    n, nnz = len(wl["row"]) - 1, len(wl["col"])
    # size each step so warm-up + timed steps take about two minutes
    et_full, _, info = reference_time(wl["row"], wl["col"], wl["val"], wl["x"], a.format, 0.0, calls=1)
    per_step = 120.0 / (a.steps + W)
    frac = float(min(1.0, max(1.0 / 64, per_step / max(et_full, 1e-9))))
    et, snnz, info = reference_time(wl["row"], wl["col"], wl["val"], wl["x"], a.format, 0.0,
                                    calls=a.steps, row_frac=frac, warm=W)
    value = 2.0 * snnz / et / 1e9
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": a.steps,
           "warmup": W, "ms_per_step": et * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": f"synthetic: {wl['desc']}",
           "config": run_config(wl, format_name(a.format), "f64", "u32", alg_bytes(n, nnz)),
           "kernel": {"family": "reference CPU", "name": info["kernel"], "threads": info["cores"]},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["cores"], "kind": "reference",
                            "sample": f"{info['kernel']} (intSpmv_main.c) on the first {info['rows']} rows "
                                      f"({snnz} nonzeros) of the workload per step, {info['cores']} threads"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
