#!/usr/bin/env python
"""Benchmark of the B200 engine on the N = 100,000 cylinder (regularised Laplace kernel,
leaf 64, eta 2, ACA+ epsilon 1e-6, 16 right-hand sides ~ N(0, 1) seed 1).

A step is one H-matrix-vector product with 16 right-hand sides over the assembled
matrix.  The headline `value` is H-gemv GB/s of the mixed-precision engine (FP32 bulk,
FP64 truncation): algorithmic bytes (every stored leaf scalar once, x read and y
written once) over device time, inputs resident in HBM.  Also reported: ACA+ leaves/s,
the FP64 engine on the same inputs, mixed-vs-FP64 speedups with relative errors against
the exact dense product (sampled rows, FP64), the end-to-end time through the C ABI with
host buffers, the roofline of the dominant kernel and the reference's CPU build.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Multi-GPU runs are independent replicas (one matrix per GPU, weak scaling).
"""
import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "H-gemv GB/s vs HBM peak; ACA+ leaves/s; mixed vs FP64 speedup at rel.err 1e-6"
WORKLOAD = dict(name="cylinder N=100000 (250x400 grid), 1/(4pi(r+0.01)), leaf 64, eta 2, ACA+ eps 1e-6, 16 RHS",
                n_theta=250, n_z=400, leaf=64, eta=2.0, eps=1e-6, nrhs=16, seed=1, delta=0.01)


def load_module(name, path, pkg_dir=None):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=pkg_dir)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def package():
    d = os.path.join(ROOT, "hmat-oss_b200")
    return load_module("hmat_oss_b200", os.path.join(d, "__init__.py"), [d])


def workloads():
    return load_module("hmat_workloads", os.path.join(ROOT, "hmat-oss_b200", "workloads.py"))


def measured_traffic(phase):
    """DRAM bytes per launch of a gemv phase's kernel from the committed ncu capture of this
    workload (profiles/traffic_cylinder100k_mixed.json), or None."""
    p = os.path.join(ROOT, "profiles", "traffic_cylinder100k_mixed.json")
    try:
        d = json.load(open(p))["phases"][phase]
        return (d["dram_read_mb"] + d["dram_write_mb"]) * 1e6
    except (OSError, KeyError, ValueError):
        return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm = []
        mx = 0.0
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = max(mx, float(r[1]))
                for n, v in zip(names, r[3:7]):
                    if v.lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dense_rows_reference(pts, x, rows, delta):
    """Exact y[rows] = K[rows, :] x in FP64 (the dense product, sampled rows)."""
    d = pts[rows][:, None, :] - pts[None, :, :]
    r = np.sqrt((d * d).sum(-1))
    K = 1.0 / (4.0 * np.pi * (r + delta))
    return K @ x


def cpu_baseline_reference(pts, x, wl_cfg, steps=1, warmup=0, scalar="S"):
    """The reference library's own CPU build (oracle/_ref) on this workload: assembly,
    then gemv with 16 right-hand sides; OPENBLAS_NUM_THREADS=1 (the reference disables
    BLAS threading inside its calls and has no tree-level parallelism)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.have_reference():
        return None
    t0 = time.time()
    r = O.run_reference(pts, 0, wl_cfg["eps"], leaf=wl_cfg["leaf"], eta=wl_cfg["eta"], delta=wl_cfg["delta"], x=x,
                        nrhs=x.shape[1], scalar=scalar, gemv_reps=steps, gemv_warmup=warmup)
    wall = time.time() - t0
    L = r["leaves"]
    s = 4 if scalar == "S" else 8
    full = L[L[:, 4] == 0]
    rk = L[(L[:, 4] == 1) & (L[:, 5] > 0)]
    stored = int((full[:, 1].astype(np.int64) * full[:, 3]).sum() + (rk[:, 5].astype(np.int64) *
                                                                      (rk[:, 1] + rk[:, 3])).sum())
    nbytes = stored * s + 2 * len(pts) * x.shape[1] * s
    t = r["json"]["t_gemv_mean"] if steps > 0 else r["json"]["t_gemv_first"]
    return {"gbs": nbytes / t / 1e9, "t_gemv_s": t, "t_assemble_s": r["json"]["t_assemble"], "bytes": nbytes,
            "rk_count": r["json"]["rk_count"], "wall_s": wall, "scalar": scalar}


def batch_cpu_baseline(batch):
    """The reference's CPU build on every matrix of the batch, one process per matrix (the
    library has global state), as many at once as the host has cores: wall time of the whole
    batch, matrices/s and ACA+ leaves/s over it, FP32 storage as the mixed engine."""
    import concurrent.futures as cf
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.have_reference():
        return None
    cores = os.cpu_count() or 1

    def one(c):
        r = O.run_reference(c["points"], 1, c["eps"], leaf=c["leaf"], eta=c["eta"], ell=c["ell"], nugget=c["nugget"],
                            scalar="S")
        return r["json"]["rk_count"], r["json"]["t_assemble"]

    t0 = time.time()
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:  # each call runs the reference in its own process
        out = list(ex.map(one, batch))
    wall = time.time() - t0
    rk = sum(o[0] for o in out)
    return {"matrices_per_s": len(batch) / wall, "aca_leaves_per_s": rk / wall, "wall_s": wall,
            "assembly_s_sum": sum(o[1] for o in out), "cores": cores, "kind": "reference",
            "cpu": cpu_model(),
            "sample": f"all {len(batch)} matrices, one reference process each, {cores} at a time (assembly)"}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    wl = workloads()
    pts = wl.cylinder(WORKLOAD["n_theta"], WORKLOAD["n_z"])
    x = wl.rhs(len(pts), WORKLOAD["nrhs"], WORKLOAD["seed"])
    res = cpu_baseline_reference(pts, x, WORKLOAD, steps=args.steps, warmup=args.warmup)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref is missing"}))
        return 0
    line = {"impl": "reference", "metric": METRIC, "value": res["gbs"], "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["t_gemv_s"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 storage, f64 compression",
            "data": "synthetic", "config": {"workload": WORKLOAD["name"], "value_type": "HMAT_SIMPLE_PRECISION",
                                            "assembly_s": res["t_assemble_s"], "rk_leaves": res["rk_count"],
                                            "aca_leaves_per_s": res["rk_count"] / res["t_assemble_s"]},
            "cpu_baseline": {"value": res["gbs"], "unit": "GB/s", "cores": 1, "kind": "reference",
                             "sample": f"full workload: one assembly, {args.warmup} warm-up + {args.steps} timed gemv"},
            "e2e": {"value": res["gbs"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def max_over_ranks(value, dist, device="cuda"):
    """The largest per-rank value (a step time): every rank times its own replica alone, so
    the job's step time is the slowest rank's.  All ranks must call it, in the same order."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _time_device(fn, steps, warmup, stream):
    """Mean device ms of fn(stream) over `steps` calls after `warmup`, CUDA events on `stream`."""
    import torch
    for _ in range(warmup):
        fn(stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def supplementary(args):
    """One JSON line for a configuration other than the headline one (cfg0: plain FP64
    cylinder 8,000; cfg2: uneven batch of 64 covariance matrices; cfg3: complex Helmholtz
    cylinder 200,000; cfg4: adjoint of 1/2 ||H x - b||^2 on a 50,000-point cube)."""
    import torch
    hb, wl = package(), workloads()
    name = args.workload
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    out = {"workload": name, "supplementary": True, "data": "synthetic", "steps": args.steps, "warmup": args.warmup}

    def make(c, vt):
        hb.set_parameters(compressionMinLeafSize=0)
        k = hb.kernel(c["kind"], delta=c.get("delta", 0.01), ell=c.get("ell", 0.3), nugget=c.get("nugget", 0.0),
                      wavenumber=c.get("wavenumber", 0.0))
        t0 = time.time()
        h = hb.HMatrix(c["points"], k, value_type=vt, leaf_size=c["leaf"], eta=c["eta"], epsilon=c["eps"])
        torch.cuda.synchronize()
        return h, time.time() - t0

    def gemv_ms(h, x_host, dtype, trans="N"):
        xd = torch.from_numpy(np.ascontiguousarray(x_host.T)).to("cuda", dtype)
        yd = torch.zeros_like(xd)
        nr = x_host.shape[1]
        ms = _time_device(lambda s: h.gemv_device(xd.data_ptr(), yd.data_ptr(), nr, trans=trans,
                                                  stream=s.cuda_stream), args.steps, args.warmup, stream)
        return ms, yd.T.cpu().numpy()

    def asm_ms(h):
        t = h.phase_times()
        return t["full_ms"] + t["aca_ms"] + t["truncate_ms"], t

    if name in ("cfg0", "cfg3"):
        c = wl.config(name)
        cplx = c["complex"]
        x = wl.rhs(len(c["points"]), c["nrhs"], c["seed"], complex_=cplx)
        res = {}
        for label, vt, dt in ((("C", 2, torch.complex64), ("Z", 3, torch.complex128)) if cplx else
                              (("S", 0, torch.float32), ("D", 1, torch.float64))):
            h, wall = make(c, vt)
            a_ms, parts = asm_ms(h)
            ms, y = gemv_ms(h, x, dt)
            T = h.leaf_table()
            nrk = int(((T[:, 4] == 1)).sum())
            res[label] = {"assembly_device_ms": a_ms, "assembly_wall_s": wall, "phase_ms": parts,
                          "gemv_ms": ms, "gemv_gbs": h.gemv_bytes(c["nrhs"]) / (ms * 1e-3) / 1e9,
                          "rk_leaves": nrk, "aca_leaves_per_s": nrk / ((parts["aca_ms"] + parts["truncate_ms"]) * 1e-3),
                          "gemv_schedule": h.gemv_tuning(), "y": y}
            h.close()
        lo, hi = ("C", "Z") if cplx else ("S", "D")
        err = float(np.linalg.norm(res[lo]["y"] - res[hi]["y"]) / np.linalg.norm(res[hi]["y"]))
        for v in res.values():
            v.pop("y")
        out.update({"metric": "H-gemv GB/s; ACA+ leaves/s", "nrhs": c["nrhs"], "n": len(c["points"]),
                    "results": res, "mixed_rel_err_vs_fp64_hmatrix": err,
                    "gemv_speedup_mixed_vs_fp64": res[hi]["gemv_ms"] / res[lo]["gemv_ms"]})
    elif name == "cfg2":
        # the 64 matrices as one batch (hmat_b200_batch_*): one assembly and one product for all
        # of them, one launch per phase
        batch = wl.batch_config(64, seed=0)
        pts = [c["points"] for c in batch]
        kers = [hb.kernel(hb.EXP_COV, ell=c["ell"], nugget=c["nugget"]) for c in batch]
        hb.set_parameters(compressionMinLeafSize=0)
        nrhs = 1
        X = np.concatenate([wl.rhs(len(c["points"]), nrhs, c["seed"]) for c in batch], axis=0)
        res, ys = {}, {}
        for label, vt, dt in (("S", 0, torch.float32), ("D", 1, torch.float64)):
            t0 = time.time()
            b = hb.HMatrixBatch(pts, kers, value_type=vt, leaf_size=64, eta=2.0, epsilon=1e-5)
            torch.cuda.synchronize()
            wall = time.time() - t0
            a_ms, parts = asm_ms(b)
            T = b.leaf_table()
            rk = int((T[:, 4] == 1).sum())
            ms, ys[label] = gemv_ms(b, np.asfortranarray(X), dt)
            res[label] = {"matrices": len(batch), "dof": int(X.shape[0]), "leaves": int(len(T)), "rk_leaves": rk,
                          "assembly_device_ms": a_ms, "phase_ms": parts, "assembly_wall_s": wall,
                          "aca_leaves_per_s": rk / ((parts["aca_ms"] + parts["truncate_ms"]) * 1e-3),
                          "matrices_per_s": len(batch) / (a_ms * 1e-3), "gemv_ms": ms,
                          "gemv_gbs": b.gemv_bytes(nrhs) / (ms * 1e-3) / 1e9,
                          "gemv_launches": b.gemv_launches(nrhs), "gemv_schedule": b.gemv_tuning()}
            b.close()
        err = float(np.linalg.norm(ys["S"] - ys["D"]) / np.linalg.norm(ys["D"]))
        cpu = None
        if not args.no_cpu_baseline:
            cpu = batch_cpu_baseline(batch)
        out.update({"metric": "ACA+ leaves/s and matrices/s over the batch (device assembly time); batched H-gemv GB/s",
                    "nrhs": nrhs, "results": res, "mixed_rel_err_vs_fp64_hmatrix": err,
                    "assembly_speedup_mixed_vs_fp64": res["D"]["assembly_device_ms"] / res["S"]["assembly_device_ms"],
                    "gemv_speedup_mixed_vs_fp64": res["D"]["gemv_ms"] / res["S"]["gemv_ms"],
                    "cpu_baseline": cpu})
    elif name == "cfg4":
        c = wl.config(name)
        n = len(c["points"])
        x = wl.rhs(n, 1, c["seed"])
        b = wl.rhs(n, 1, c["seed"] + 1)
        h, wall = make(c, 0)
        xd = torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda", torch.float32)
        bd = torch.from_numpy(np.ascontiguousarray(b.T)).to("cuda", torch.float32)
        rd = torch.zeros_like(xd)
        dx = torch.zeros_like(xd)
        offs, total = h.payload_layout()
        g = torch.zeros(total, device="cuda", dtype=torch.float32)
        one = 1.0

        def backward(s):
            # r = H x - b, then dx = H^T r and the leaf gradients in one pass
            rd.copy_(bd)
            h.gemv_device(xd.data_ptr(), rd.data_ptr(), 1, alpha=one, beta=-1.0, stream=s.cuda_stream)
            h.gemv_adjoint(xd.data_ptr(), rd.data_ptr(), 1, dx.data_ptr(), g.data_ptr(), accumulate=False,
                           stream=s.cuda_stream)

        with torch.cuda.stream(stream):
            ms = _time_device(backward, args.steps, args.warmup, stream)
        fwd = h.gemv_bytes(1)
        payload = total * 4
        out.update({"metric": "adjoint GB/s (forward bytes + written leaf gradients)", "n": n,
                    "backward_ms": ms, "bytes": fwd + payload,
                    "gbs": (fwd + payload) / (ms * 1e-3) / 1e9, "assembly_device_ms": asm_ms(h)[0],
                    "gemv_schedule": h.gemv_tuning()})
        h.close()
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--workload", default="cfg1", choices=["cfg0", "cfg1", "cfg2", "cfg3", "cfg4"],
                    help="cfg1 is the headline line; the others print supplementary lines")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    if args.workload != "cfg1":
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            return supplementary(args)
        return 0

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    hb = package()
    wl = workloads()
    cfg = WORKLOAD
    pts = wl.cylinder(cfg["n_theta"], cfg["n_z"])
    n = len(pts)
    nrhs = cfg["nrhs"]
    x_host = wl.rhs(n, nrhs, cfg["seed"])
    hb.set_parameters(compressionMinLeafSize=0)
    kern = hb.kernel(hb.LAPLACE_REG, delta=cfg["delta"])

    def build(vt):
        t0 = time.time()
        h = hb.HMatrix(pts, kern, value_type=vt, leaf_size=cfg["leaf"], eta=cfg["eta"], epsilon=cfg["eps"])
        torch.cuda.synchronize()
        return h, time.time() - t0

    def time_gemv(h, dtype):
        xd = torch.from_numpy(np.ascontiguousarray(x_host.T)).to(device="cuda", dtype=dtype)  # column-major N x r
        yd = torch.zeros_like(xd)
        # an explicit stream: the engine launches on the stream it is given, and events
        # recorded on that same stream bracket the timed region
        stream = torch.cuda.Stream()
        sp = stream.cuda_stream
        torch.cuda.synchronize()
        for _ in range(args.warmup):
            h.gemv_device(xd.data_ptr(), yd.data_ptr(), nrhs, stream=sp)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            h.gemv_device(xd.data_ptr(), yd.data_ptr(), nrhs, stream=sp)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist)
        return ms, yd.T.cpu().numpy().astype(np.float64)

    # ---- mixed precision engine (headline) ----
    h32, wall32 = build(hb.HMAT_SIMPLE_PRECISION)
    pt32 = h32.phase_times()
    aca32 = {k: v["threads"] for k, v in h32.aca_tuning().items()}
    T32 = h32.leaf_table()
    n_rk = int((T32[:, 4] == 1).sum())
    bytes32 = h32.gemv_bytes(nrhs)
    with ClockSampler(local) as clk:
        ms32, y32 = time_gemv(h32, torch.float32)
    clocks = clk.summary()

    # roofline of the dominant kernel (y-phase) from eager per-phase event timing
    xd = torch.from_numpy(np.ascontiguousarray(x_host.T)).to(device="cuda", dtype=torch.float32)
    yd = torch.zeros_like(xd)
    prof = [h32.gemv_profile(xd.data_ptr(), yd.data_ptr(), nrhs) for _ in range(5)]
    ph_ms = {k: float(np.mean([p["ms"][k] for p in prof])) for k in prof[0]["ms"]}
    ph_bytes = prof[0]["bytes"]
    dom = max(ph_ms, key=lambda k: ph_ms[k])
    peak, peak_kind = measured_peaks()
    achieved = ph_bytes[dom] / (ph_ms[dom] * 1e-3) / 1e9

    # end to end through the C ABI gemv with pinned host buffers (copies in the timed region)
    x_pin = torch.from_numpy(np.asfortranarray(x_host, dtype=np.float32).ravel(order="F")).pin_memory()
    y_pin = torch.zeros_like(x_pin).pin_memory()
    a = np.array([1.0], np.float32)
    b = np.array([0.0], np.float32)
    for _ in range(args.warmup):
        h32.hi.gemv(b"N", a.ctypes.data, h32.m, x_pin.data_ptr(), b.ctypes.data, y_pin.data_ptr(), nrhs)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rc = h32.hi.gemv(b"N", a.ctypes.data, h32.m, x_pin.data_ptr(), b.ctypes.data, y_pin.data_ptr(), nrhs)
        assert rc == 0
    # each call is synchronous (the result is in host memory when it returns)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps, dist)

    # ---- FP64 engine on the same inputs ----
    fp64 = None
    if not args.no_fp64:
        h64, wall64 = build(hb.HMAT_DOUBLE_PRECISION)
        pt64 = h64.phase_times()
        ms64, y64 = time_gemv(h64, torch.float64)
        bytes64 = h64.gemv_bytes(nrhs)
        rows = np.random.default_rng(7).choice(n, 256, replace=False)
        yex = dense_rows_reference(pts, x_host, rows, cfg["delta"])
        err64 = float(np.linalg.norm(y64[rows] - yex) / np.linalg.norm(yex))
        err32 = float(np.linalg.norm(y32[rows] - yex) / np.linalg.norm(yex))
        err32_vs_h64 = float(np.linalg.norm(y32 - y64) / np.linalg.norm(y64))
        asm32 = pt32["full_ms"] + pt32["aca_ms"] + pt32["truncate_ms"]
        asm64 = pt64["full_ms"] + pt64["aca_ms"] + pt64["truncate_ms"]
        fp64 = {"gemv_ms": ms64, "gemv_gbs": bytes64 / (ms64 * 1e-3) / 1e9, "assembly_device_ms": asm64,
                "aca_leaves_per_s": n_rk / ((pt64["aca_ms"] + pt64["truncate_ms"]) * 1e-3),
                "rel_err_vs_dense_sampled": err64,
                "mixed_rel_err_vs_dense_sampled": err32, "mixed_rel_err_vs_fp64_hmatrix": err32_vs_h64,
                "gemv_speedup_mixed_vs_fp64": ms64 / ms32, "assembly_speedup_mixed_vs_fp64": asm64 / asm32,
                "step_speedup_mixed_vs_fp64": (asm64 + ms64) / (asm32 + ms32)}
        h64.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_reference(pts, x_host, cfg, steps=1, warmup=0)
        except Exception as e:  # reported, not fatal
            cpu = {"error": str(e)}

    if rank == 0:
        asm32 = pt32["full_ms"] + pt32["aca_ms"] + pt32["truncate_ms"]
        launches = args.steps * h32.gemv_launches(nrhs)  # gather, z-phase classes, [z-reduce], y-phase, final
        line = {
            "metric": METRIC, "value": world * bytes32 / (ms32 * 1e-3) / 1e9, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 truncation)", "data": "synthetic",
            "config": {"workload": cfg["name"], "value_type": "HMAT_SIMPLE_PRECISION", "nrhs": nrhs,
                       "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (leaf data per step "
                       f"{bytes32 / 1e9:.3f} GB)", "leaves": int(len(T32)), "rk_leaves": n_rk,
                       "bytes_per_step": bytes32, "assembly_device_ms": asm32, "assembly_wall_s": wall32,
                       "aca_leaves_per_s": n_rk / ((pt32["aca_ms"] + pt32["truncate_ms"]) * 1e-3),
                       "phase_ms": pt32, "aca_shapes": aca32, "gemv_schedule": h32.gemv_tuning()},
            "roofline": {"bound": "hbm", "kernel": f"gemv {dom}", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": measured_traffic(dom),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one capture "
                                           "(profiles/traffic_cylinder100k_mixed.json)",
                         "phase_ms": ph_ms, "phase_bytes": ph_bytes,
                         "whole_gemv_frac": bytes32 / (ms32 * 1e-3) / 1e9 / peak},
            "mixed_vs_fp64": fp64,
            "e2e": {"value": world * bytes32 / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": world * n * nrhs * 4, "d2h_bytes_per_step": world * n * nrhs * 4,
                    "path": "hmat_interface_t.gemv (C ABI), pinned host x/y"},
            "cpu_baseline": None if cpu is None or "error" in cpu else {
                "value": cpu["gbs"], "unit": "GB/s", "cores": 1, "kind": "reference",
                "sample": "reference CPU build on the full workload, FP32 storage (HMAT_SIMPLE_PRECISION): one "
                          f"assembly ({cpu['t_assemble_s']:.1f} s) and one 16-RHS gemv ({cpu['t_gemv_s']:.2f} s)"},
            "clocks": clocks,
            "gpu_launches": launches,
        }
        if cpu is not None and "error" in cpu:
            line["cpu_baseline_error"] = cpu["error"]
        print(json.dumps(line))
    h32.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
