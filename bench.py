#!/usr/bin/env python
"""Batched 4pi CCCS benchmark: dose-loading-matrix construction, beamlets/s.

Workload (one step): the 4pi torso plan -- a 200x200x160 phantom at 2.5 mm,
up to 400 candidate beams on a sphere pruned for couch/gantry clearance, 16x16
beamlets of 0.5 cm kept where they see the PTV, 48 cones (8 zenith x 6
azimuth), 12-bin spectrum -- through Terma, CCCS and the BEV->PVCS column
stage into the per-beam CSR dose-loading matrices, all beams in one call.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fd2|reference]

One JSON line on rank 0.  `value` is device-timed with the density resident in
HBM; `e2e` goes through the public API with host inputs (density volume and
beamlet descriptors copied from pinned memory every step) and the whole CSR
result read back into pinned memory, batch by batch while the next batch is
computed (DoseMatConstruction's host_out).  Multi-GPU: one process per GPU; N GPUs
take a 4pi candidate set of N x 400 beams, partitioned by beam across the
ranks by a greedy balance on the CCCS march length (fastdose_b200.sharding),
each rank building its share's matrices with no collective on the data path;
weak scaling (about 400 beams per GPU); time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CCCS beamlets/s (dose-loading matrix, batched 4pi)"
# From one ncu capture of the CCCS march on the 40-beam plan (6056 beamlets,
# 8.2 waves; profiles/cccs_kernel_4pi_torso_40beams.md):
# dram__bytes_read.sum + dram__bytes_write.sum, and smsp__inst_executed.sum
CCCS_DRAM_BYTES_PER_BEAMLET = (28.562879e9 + 9.447058e9) / 6056
CCCS_WARP_INST_PER_BEAMLET = 124.063924973e9 / 6056
UNIT = "beamlets/s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def plan_inputs(n_beams):
    from fastdose_b200 import phantoms
    from fastdose_b200.types import make_bundle

    cfg = phantoms.config2(n_beams)
    bundles = np.array([make_bundle(cfg["isocenter"], a, sad=cfg["sad"], fluence_dim=cfg["fluence_dim"],
                                    beamlet_size=cfg["beamlet_size"], sub_fluence_dim=cfg["sub_fluence_dim"],
                                    sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"])
                        for a in cfg["angles"]])
    return cfg, bundles


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
            os.unlink(self.path)
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        if sm:
            out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                   "samples": len(sm), "sm_min_mhz": min(sm)}
        return out


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def stratified_order(beamlets, every=10):
    """Beamlet order for the CPU samples: beams 0, every, 2*every, ... taken
    round-robin (one beamlet of each in turn), so consecutive samples spread
    over the sphere of beams; the plan's other beams follow."""
    groups = [list(range(sum(len(b) for b in beamlets[:i]), sum(len(b) for b in beamlets[:i + 1])))
              for i in range(len(beamlets))]
    picked = [g for i, g in enumerate(groups) if i % every == 0 and g]
    order = []
    depth = 0
    while any(depth < len(g) for g in picked):
        order += [g[depth] for g in picked if depth < len(g)]
        depth += 1
    rest = [k for i, g in enumerate(groups) if i % every != 0 for k in g]
    return np.array(order + rest, np.int64)


def cpu_baseline(cfg, beamlets, fluence, budget_s, threads, start=0, order=None):
    """The CPU restatement (single-precision build) on host threads over a
    bounded sample of the plan's beamlets, taken in `order` from position
    `start`: beamlets/s, and where the next sample should start."""
    import oracle

    flat = np.concatenate(beamlets)
    order = stratified_order(beamlets) if order is None else order
    ph = cfg["phantom"]
    done = 0
    t0 = time.perf_counter()
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(threads) as ex:
        while time.perf_counter() - t0 < budget_s and done < len(flat):
            idx = order[(start + done + np.arange(threads)) % len(flat)]
            list(ex.map(lambda b: oracle.beamlet_pipeline(b, fluence, ph.density, ph.volume, cfg["spectrum"],
                                                          cfg["kernel"], precision="float"), flat[idx]))
            done += len(idx)
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(), "kind": "port",
            "sample": f"{done} of {len(flat)} beamlets of the same plan (Terma, CCCS, column), {dt:.1f} s, "
                      f"taken round-robin from every 10th beam"}, start + done


def workload_name(n_beams, n_beamlets):
    """The bench workload, named the same by both arms (the beamlet count is
    its own config key: the reference arm flags beamlets with the host
    restatement of the texture test, which may differ in a beamlet or two)."""
    del n_beamlets
    return (f"4pi torso 200x200x160 @2.5mm, {n_beams} beams, 16x16 beamlets of 0.5 cm flagged by the PTV, "
            f"8x6 cones, 12-bin spectrum")


REFERENCE_FLAGS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "flags_c2_ref.npz")


def oracle_plan_beamlets(bundles, ptv_mask, volume):
    """The plan's beamlets without this library: beamletInit's host
    restatement in the reference's order (pixels row by row, beams in turn),
    on the PTV flags of the reference's own beamletFlagInit for this plan
    when the committed fixture holds them (the default 400-beam plan), else on
    the oracle's host restatement of the flag test.  That restatement samples
    the mask with emulated 8-bit filter weights; the texture unit's filtering
    arithmetic is not published, and on this plan the restatement flags 459
    margin pixels (0.45 %) that the reference does not.  Returns the beamlets
    and the source of the flags."""
    import oracle
    from fastdose_b200.types import BEAM_DTYPE

    flags, source = None, "the oracle's host restatement of beamletFlagInit (emulated texture weights)"
    if os.path.exists(REFERENCE_FLAGS):
        g = np.load(REFERENCE_FLAGS)
        if g["bundles"].shape == bundles.shape and np.asarray(g["bundles"], bundles.dtype).tobytes() == bundles.tobytes():
            flags = g["flags"]
            source = "the reference's own beamletFlagInit output for this plan (tests/golden/flags_c2_ref.npz)"
    if flags is None:
        beams0 = np.array([oracle.calc_range(_bundle_beam(b), volume)[1] for b in bundles])
        flags = oracle.beamlet_flags(beams0, ptv_mask, volume, tex_mode=1, precision="float")
    out = []
    for bb, fl in zip(bundles, flags):
        fx, fy = (int(v) for v in bb["fluence_dim"])
        got = []
        for j in range(fy):
            for i in range(fx):
                if fl[i + j * fx]:
                    st, b = oracle.beamlet_init(bb, i, j, volume)
                    got.append(b)
        out.append(np.array(got) if got else np.zeros((0,), BEAM_DTYPE))
    return out, source


def run_reference(args, rank):
    """--impl reference: the reference has no CPU implementation of this path;
    its algorithm is timed through the CPU restatement on all host cores.
    Only oracle/ code runs here: the plan's geometry and flags come from the
    oracle's host restatements, not from this library."""
    if rank != 0:
        return
    import oracle

    cfg, bundles = plan_inputs(args.beams * max(1, args.gpus))
    ph = cfg["phantom"]
    beamlets, flag_source = oracle_plan_beamlets(bundles, ph.masks["PTV"], ph.volume)
    n_bl = int(sum(len(b) for b in beamlets))
    fluence = oracle.beamlet_fluence(bundles[0])
    threads = os.cpu_count() or 1
    order = stratified_order(beamlets)
    steps = []
    pos = 0
    # each step a bounded sample; the whole run stays near 2.5 minutes
    per_step = min(args.cpu_seconds, max(2.0, 150.0 / (args.warmup + args.steps)))
    for i in range(args.warmup + args.steps):
        r, pos = cpu_baseline(cfg, beamlets, fluence, per_step, threads, start=pos, order=order)
        if i >= args.warmup:
            steps.append(r["value"])
    v = statistics.median(steps)
    r["sample"] += f"; {pos} beamlets over {args.warmup + args.steps} steps, median of the timed steps"
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_name(len(bundles), n_bl), "beams": len(bundles), "beamlets": n_bl,
                       "parallelism": f"CPU restatement on {threads} host threads", "flags": flag_source},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "cpu_model": r["cpu_model"], "kind": "port",
                             "sample": r["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _bundle_beam(bb):
    from fastdose_b200.types import BEAM_DTYPE

    b = np.zeros((), BEAM_DTYPE)
    b["isocenter"] = bb["isocenter"]
    b["beamlet_size"] = bb["beamlet_size"]
    b["fmap_size"] = bb["fluence_dim"]
    b["sad"] = bb["sad"]
    b["angles"] = bb["angles"]
    b["long_spacing"] = bb["long_spacing"]
    return b


def time_spmv(M, n_in, n_out, peak, reps=10, warmup=3):
    """One product M x alone: CUDA-event time per launch after warm-up, and its
    bandwidth (matrix stream + x + y) against the HBM peak."""
    import torch

    s = torch.cuda.current_stream()
    xv = torch.rand(n_in, device="cuda")
    yv = torch.empty(n_out, device="cuda")
    for _ in range(warmup):
        M.spmv(xv, yv, stream=s)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        M.spmv(xv, yv, stream=s)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    nb = M.info()["device_bytes"] + n_in * 4 + n_out * 4  # matrix stream + x + y
    return {"ms": ms, "bytes": nb, "gbs": nb / ms * 1e-6, "frac": nb / ms * 1e-6 / peak,
            "x_in_shared": M.info()["x_in_shared"]}


def spmv_leg(ctx, key, rows, seed=3, reps=10, warmup=3):
    """--only-spmv: the optimization benchmark's synthetic pair (rows x 40k) in
    one format, A x then A^T y timed alone (profiling)."""
    from fastdose_b200 import optimize

    vt, fmt = key.split("_")
    cols = 40_000
    A, AT = optimize.Matrix.synthetic(ctx, rows, cols, rows // 25, 0.5, seed=seed, value_type=vt, index_format=fmt)
    peak, _ = _peaks()
    return {"format": key, "rows": rows, "cols": cols, "nnz": A.info()["nnz"],
            "A": time_spmv(A, cols, rows, peak, reps, warmup), "AT": time_spmv(AT, rows, cols, peak, reps, warmup)}


def optimizer_leg(ctx, iters, rows=2_500_000, n_beams=400, seed=3):
    """Fluence optimization on the IMRT-scale synthetic matrix: 2.5M VOI rows
    (PTV first) x 40k beamlets (400 beams x 10x10 maps), ~2% nonzeros, D from
    the 10x10 fluence maps, weights as the optimization benchmark states.
    BOO iterations/s with the matrix in FP32 and in FP16/BF16 (per-beamlet
    scale), the objective reached by each after the same iterations, and the
    SpMV bandwidth against the HBM roofline."""
    import torch

    from fastdose_b200 import optimize

    fd = 10
    cols = n_beams * fd * fd
    window, density = rows // 25, 0.5  # each VOI row meets 2% of the beamlets
    n_ptv = rows // 10
    rng = np.random.default_rng(seed)
    n_oar = rows - n_ptv
    w = dict(max_dose=np.concatenate([np.ones(n_ptv), rng.uniform(0.3, 0.7, n_oar)]).astype(np.float32),
             max_weights=np.concatenate([np.ones(n_ptv), rng.uniform(0.1, 1.0, n_oar)]).astype(np.float32),
             min_dose=np.ones(n_ptv, np.float32), min_weights=np.ones(n_ptv, np.float32),
             oar_weights=rng.uniform(0.0, 0.1, n_oar).astype(np.float32))
    D = optimize.block_diag([optimize.fluence_grad(fd, np.ones(fd * fd, np.uint8))] * n_beams)
    Dm = optimize.Matrix.from_csr(ctx, *D[:3], cols)
    DTm = Dm.transpose()
    groups = np.arange(0, cols + 1, fd * fd, dtype=np.int64)
    peak, _ = _peaks()
    out = {"workload": f"synthetic VOI matrix {rows}x{cols} (PTV {n_ptv}), window {window}, density {density}, "
                       f"D from {n_beams} 10x10 maps, gamma 1, eta 0.1, beam weight 0.1; BOO iterations"}
    x0 = torch.full((cols,), 0.01, dtype=torch.float32, device="cuda")
    # the FP32 matrix and plan are kept to dose every format's plan exactly:
    # DVHs of the PTV and OAR rows against the FP32-optimized plan's
    A32 = x32 = dvh32 = P32 = None
    finals = {}
    structures = [np.arange(n_ptv), np.arange(n_ptv, rows)]
    n_bins = 200
    for vt, fmt in (("f32", "i32"), ("f32", "packed16"), ("f16", "packed16"), ("bf16", "packed16")):
        key = f"{vt}_{fmt}"
        A, AT = optimize.Matrix.synthetic(ctx, rows, cols, window, density, seed=seed, value_type=vt,
                                          index_format=fmt)
        info = A.info()
        P = optimize.Problem(ctx, A, AT, Dm, DTm, n_ptv, n_oar, w["max_dose"], w["max_weights"], w["min_dose"],
                             w["min_weights"], w["oar_weights"], 1.0, 0.1)
        bw = 0.1 * P.beam_weights_init(groups)
        # SpMV alone: A x and A^T y over the whole matrix
        spmv_a = time_spmv(A, cols, rows, peak)
        spmv_at = time_spmv(AT, rows, cols, peak)
        P.boo(groups, bw, x0, step_size=1e-3, iters=3, want=0, change_trigger=10 ** 9)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = P.boo(groups, bw, x0, step_size=1e-3, iters=iters, want=0, change_trigger=10 ** 9)
        dt = time.perf_counter() - t0
        if key == "f16_packed16":  # the same iterations with every trial launched kernel by kernel
            P.set_graph(False)
            P.boo(groups, bw, x0, step_size=1e-3, iters=3, want=0, change_trigger=10 ** 9)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            P.boo(groups, bw, x0, step_size=1e-3, iters=iters, want=0, change_trigger=10 ** 9)
            graph_off_it_s = r["k"] / (time.perf_counter() - t1)
            P.set_graph(True)
        out[key] = {"it_per_s": r["k"] / dt, "trials": r["trials"], "iters": r["k"], "loss": float(r["loss"][r["k"] - 1]),
                   "nnz": info["nnz"], "matrix_bytes": info["device_bytes"],
                   "exception_chunks": info["exception_chunks"],
                   "spmv": spmv_a, "spmv_transpose": spmv_at}
        if key == "f16_packed16":
            out[key]["it_per_s_without_graph"] = graph_off_it_s
        finals[key] = r["x"].clone()
        if A32 is None:
            A32, x32, P32 = A, r["x"].clone(), P
            dose32 = A32.spmv(x32)
            width = float(dose32.max().item()) / (n_bins - 1)
            _, dvh32 = optimize.dvh(ctx, dose32, structures, n_bins, width)
            out[key]["dvh"] = {"bins": n_bins, "bin_width": width, "structures": ["PTV rows", "OAR rows"]}
        else:
            _, dvh_k = optimize.dvh(ctx, A32.spmv(r["x"]), structures, n_bins, width)
            out[key]["dvh_max_abs_diff_vs_f32"] = float(np.abs(dvh_k - dvh32).max())
        if P is not P32:
            del P, AT
        if A is not A32:
            del A
        torch.cuda.empty_cache()
    # every format's plan scored on the FP32 matrix (FP32 products, FP64 sums)
    for key, xk in finals.items():
        out[key]["objective_on_f32_matrix"] = P32.eval_g(xk)
    base_obj = out["f32_i32"]["objective_on_f32_matrix"]
    for key in finals:
        out[key]["objective_on_f32_matrix_rel_diff"] = abs(out[key]["objective_on_f32_matrix"] - base_obj) / abs(base_obj)
    del A32, x32, P32, finals
    torch.cuda.empty_cache()
    out["reference_form"] = reference_form_spmv(ctx, rows // 10, cols, seed, peak)
    out["reference_cuda"] = reference_optimizer_leg(ctx, rows // 10, n_beams, fd, seed)
    base = out["f32_i32"]
    for key in ("f32_packed16", "f16_packed16", "bf16_packed16"):
        out[key]["speedup_vs_f32_i32"] = out[key]["it_per_s"] / base["it_per_s"]
        out[key]["objective_rel_diff_vs_f32"] = abs(out[key]["loss"] - base["loss"]) / abs(base["loss"])
    for key in ("f16_packed16", "bf16_packed16"):
        out[key]["speedup_vs_f32_packed16"] = out[key]["it_per_s"] / out["f32_packed16"]["it_per_s"]
    return out


def reference_optimizer_leg(ctx, rows, n_beams, fd, seed, iters=40, cpu_seconds=10.0):
    """The reference's own GPU optimizer (BOO_IMRT_L2OneHalf_gpu_QL with its
    eval_g / eval_grad / proxL2Onehalf_QL_gpu over cuSPARSE and cuBLAS,
    IMRTOptimize.cu:16-194, compiled for sm_100a in oracle/_ref/libfdref.so)
    on a tenth of the optimization matrix's rows, beside this library's BOO
    in FP32 and FP16 on the same matrix and weights; and the CPU restatement
    of the same loop (the oracle's single-precision build, one host thread,
    a bounded number of iterations) as the CPU baseline.  A baseline leg:
    nothing here is this library's product path."""
    import torch

    import oracle
    from fastdose_b200 import optimize
    from oracle import ref

    cols = n_beams * fd * fd
    window, density = rows // 25, 0.5
    n_ptv = rows // 10
    n_oar = rows - n_ptv
    rng = np.random.default_rng(seed)
    w = dict(max_dose=np.concatenate([np.ones(n_ptv), rng.uniform(0.3, 0.7, n_oar)]).astype(np.float32),
             max_weights=np.concatenate([np.ones(n_ptv), rng.uniform(0.1, 1.0, n_oar)]).astype(np.float32),
             min_dose=np.ones(n_ptv, np.float32), min_weights=np.ones(n_ptv, np.float32),
             oar_weights=rng.uniform(0.0, 0.1, n_oar).astype(np.float32))
    D = optimize.block_diag([optimize.fluence_grad(fd, np.ones(fd * fd, np.uint8))] * n_beams)
    Dm = optimize.Matrix.from_csr(ctx, *D[:3], cols)
    DTm = Dm.transpose()
    groups = np.arange(0, cols + 1, fd * fd, dtype=np.int64)
    out = {"workload": f"synthetic VOI matrix {rows}x{cols} (PTV {n_ptv}), window {window}, density {density}; "
                       f"{iters} BOO iterations from x = 0.01, beam weight 0.1, gamma 1, eta 0.1"}
    res = {}
    for vt, fmt in (("f32", "i32"), ("f16", "packed16")):
        A, AT = optimize.Matrix.synthetic(ctx, rows, cols, window, density, seed=seed, value_type=vt, index_format=fmt)
        P = optimize.Problem(ctx, A, AT, Dm, DTm, n_ptv, n_oar, w["max_dose"], w["max_weights"], w["min_dose"],
                             w["min_weights"], w["oar_weights"], 1.0, 0.1)
        bw = 0.1 * P.beam_weights_init(groups)
        x0 = np.full(cols, 0.01, np.float32)
        P.boo(groups, bw, x0, step_size=1e-3, iters=3, want=0, change_trigger=10 ** 9)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = P.boo(groups, bw, x0, step_size=1e-3, iters=iters, want=0, change_trigger=10 ** 9)
        dt = time.perf_counter() - t0
        res[f"fd2_{vt}_{fmt}"] = {"it_per_s": r["k"] / dt, "loss": float(r["loss"][r["k"] - 1])}
        if vt == "f32":
            host = [A.to_host(), AT.to_host()]
            bw32 = bw
        del P, A, AT
        torch.cuda.empty_cache()
    (a_off, a_col, a_val), (t_off, t_col, t_val) = host
    Ah = (a_off, a_col.astype(np.int64), a_val, cols)
    ATh = (t_off, t_col.astype(np.int64), t_val, rows)
    Dt = optimize.block_diag([optimize.fluence_grad(fd, np.ones(fd * fd, np.uint8))] * n_beams)
    masks = np.ones((n_beams, fd * fd), np.uint8)
    x0 = np.full(cols, 0.01, np.float32)
    if ref.available():
        R = ref.OptProblem(Ah, Dt, n_ptv, n_oar, w["max_dose"], w["max_weights"], w["min_dose"], w["min_weights"],
                           w["oar_weights"], 1.0, 0.1, AT=ATh)
        R.boo(masks, bw32, x0, x0, 1e-3, 3, want=0, change_trigger=10 ** 9)
        t0 = time.perf_counter()
        rr = R.boo(masks, bw32, x0, x0, 1e-3, iters, want=0, change_trigger=10 ** 9)
        dt = time.perf_counter() - t0
        R.close()
        res["reference_f32_i64"] = {"it_per_s": rr["k"] / dt, "loss": float(rr["loss"][rr["k"] - 1]),
                                    "note": "cuSPARSE SpMV on FP32 values with int64 indices, cuBLAS reductions "
                                            "with host scalars (about 15 host synchronisations per trial)"}
        for key in ("fd2_f32_i32", "fd2_f16_packed16"):
            res[key]["speedup_vs_reference"] = res[key]["it_per_s"] / res["reference_f32_i64"]["it_per_s"]
    else:
        res["reference_f32_i64"] = {"unavailable": "oracle/_ref/libfdref.so is not built"}
    # CPU baseline: the oracle's single-precision BOO, one host thread, bounded
    O = oracle.Problem(Ah, Dt, n_ptv, n_oar, w["max_dose"], w["max_weights"], w["min_dose"], w["min_weights"],
                       w["oar_weights"], 1.0, 0.1, precision="float", AT=ATh)
    n_cpu, t0 = 0, time.perf_counter()
    state = None
    while n_cpu < iters and time.perf_counter() - t0 < cpu_seconds:
        rc = O.boo(groups, bw32, x0 if state is None else rc["x"], 1e-3, n_cpu + 1, want=0, change_trigger=10 ** 9,
                   state=state)
        state = (rc["k"], rc["theta"], rc["t"], rc["v"])
        n_cpu = rc["k"]
    dt = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": n_cpu / dt, "unit": "BOO iterations/s", "cores": 1, "cpu_model": cpu_model(),
                           "kind": "port", "sample": f"{n_cpu} iterations of the same problem, {dt:.1f} s"}
    out.update(res)
    del Dm, DTm
    torch.cuda.empty_cache()
    return out


def reference_form_spmv(ctx, rows, cols, seed, peak):
    """A x in the reference's form -- cuSPARSE SpMV on FP32 values with int64
    row offsets and column indices (MatCSR64 through cusparseSpMV, as
    Eigen2Cusparse leaves it) -- next to this library's FP32/int32 and
    FP16/packed-16 products of the same matrix (a tenth of the optimization
    matrix's rows, still far larger than L2)."""
    import torch

    from fastdose_b200 import optimize

    window, density = rows // 25, 0.5
    s = torch.cuda.current_stream()

    def timed(fn, reps=10):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    x = torch.rand(cols, device="cuda")
    y = torch.empty(rows, device="cuda")
    res = {"rows": rows, "cols": cols}
    A, AT = optimize.Matrix.synthetic(ctx, rows, cols, window, density, seed=seed, value_type="f32", index_format="i32")
    del AT
    off, col, val = A.to_host()
    res["nnz"] = int(len(val))
    res["fd2_f32_i32_ms"] = timed(lambda: A.spmv(x, y, stream=s))
    del A
    S = torch.sparse_csr_tensor(torch.from_numpy(off).cuda(), torch.from_numpy(col.astype(np.int64)).cuda(),
                                torch.from_numpy(val).cuda(), size=(rows, cols))
    del off, col, val
    xc = x.unsqueeze(1)
    res["cusparse_f32_i64_ms"] = timed(lambda: torch.mm(S, xc))
    ref_bytes = res["nnz"] * 12 + (rows + 1) * 8 + cols * 4 + rows * 4
    res["cusparse_gbs"] = ref_bytes / res["cusparse_f32_i64_ms"] * 1e-6
    del S, xc
    A16, AT16 = optimize.Matrix.synthetic(ctx, rows, cols, window, density, seed=seed, value_type="f16",
                                          index_format="packed16")
    del AT16
    res["fd2_f16_packed16_ms"] = timed(lambda: A16.spmv(x, y, stream=s))
    res["f16_speedup_vs_cusparse_f32_i64"] = res["cusparse_f32_i64_ms"] / res["fd2_f16_packed16_ms"]
    res["f32_speedup_vs_cusparse_f32_i64"] = res["cusparse_f32_i64_ms"] / res["fd2_f32_i32_ms"]
    del A16
    torch.cuda.empty_cache()
    return res


def c4_leg(ctx, n_per_iso=300, opt_iters=20):
    """--c4: the multi-isocentre head-and-neck configuration -- 256x256x200 at
    2.5 mm, four PTV segments with their own isocentres, n_per_iso beams each
    (1200 in all) of 6..20 beamlets a side masked to the segment, one BEV grid
    per isocentre (12, 16, 20, 16 pixels a side), one dose-loading matrix per
    isocentre -- then the four matrices joined on the device and optimized
    together with the FP16 matrix (PTV union rows and a subsampled ring)."""
    import torch

    from fastdose_b200 import api, optimize, phantoms
    from fastdose_b200.types import make_bundle

    cfg = phantoms.config4(n_per_iso)
    ph = cfg["phantom"]
    dens = api.Density(ctx, ph.density, ph.volume)
    spec, kern = api.Spectrum(ctx, cfg["spectrum"]), api.Kernel(ctx, cfg["kernel"])
    plans = []
    for iso in cfg["isos"]:
        bundles = np.array([make_bundle(iso["isocenter"], a, sad=cfg["sad"], fluence_dim=int(fd),
                                        beamlet_size=cfg["beamlet_size"], sub_fluence_dim=iso["sub_fluence_dim"],
                                        sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"])
                            for a, fd in zip(iso["angles"], iso["fluence_dims"])])
        beams, flags, fds = [], [], []
        for fd in np.unique(iso["fluence_dims"]):  # one flag pass per fluence dimension
            idx = np.flatnonzero(iso["fluence_dims"] == fd)
            fl = api.beamletFlagInit(ctx, bundles[idx], iso["mask"], ph.volume)
            for j, f, b in zip(idx, fl, api.bundles_beamlets(bundles[idx], fl, ph.volume)):
                if len(b):
                    beams.append(b)
                    flags.append(np.asarray(f).reshape(-1))
                    fds.append(int(fd))
        plans.append(dict(beams=beams, flags=flags, fds=fds, fluence=api.beamlet_fluence(bundles[0])))
    n_beams = sum(len(p["beams"]) for p in plans)
    n_bl = sum(len(b) for p in plans for b in p["beams"])
    counts = [len(b) for p in plans for b in p["beams"]]
    s = torch.cuda.current_stream()
    # warm-up: the four matrices once, untimed and held together as the timed
    # pass holds them (the CCCS schedule of each batch shape is tuned, and the
    # context's buffers and memory pool reach their size), then timed
    warm = [api.DoseMatConstruction(ctx, p["beams"], p["fluence"], dens, spec, kern, stream=s) for p in plans]
    for m in warm:
        m.close()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(plans) + 1)]
    ev[0].record(s)
    parts = []
    for i, p in enumerate(plans):
        parts.append(api.DoseMatConstruction(ctx, p["beams"], p["fluence"], dens, spec, kern, stream=s))
        ev[i + 1].record(s)
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[-1])
    per_iso = [{"bev_grid": int(iso["sub_fluence_dim"]), "beamlets": int(sum(len(b) for b in p["beams"])),
                "ms": ev[i].elapsed_time(ev[i + 1])} for i, (iso, p) in enumerate(zip(cfg["isos"], plans))]
    for q in per_iso:
        q["beamlets_per_s"] = q["beamlets"] / (q["ms"] * 1e-3)
    joint = api.MatCSREnsemble.concat(ctx, parts)
    nnz = joint.info()["nnz"]
    for m in parts:
        m.close()
    # joint optimization, FP16 matrix
    nv = ph.density.size
    ptv = np.zeros(ph.density.shape, bool)
    for iso in cfg["isos"]:
        ptv |= iso["mask"].astype(bool)
    ring = (ph.density > 0.5) & ~ptv
    ptv_idx = np.flatnonzero(ptv.reshape(-1))
    ring_idx = np.flatnonzero(ring.reshape(-1))[::8]
    voxel_row = np.full(nv, -1, np.int32)
    voxel_row[ptv_idx] = np.arange(len(ptv_idx))
    voxel_row[ring_idx] = len(ptv_idx) + np.arange(len(ring_idx))
    n_ptv, n_oar = len(ptv_idx), len(ring_idx)
    t0 = time.perf_counter()
    A, AT = optimize.Matrix.voi(ctx, joint, voxel_row, n_ptv + n_oar, value_type="f16", index_format="packed16")
    torch.cuda.synchronize()
    voi_s = time.perf_counter() - t0
    joint.close()
    D = optimize.block_diag([optimize.fluence_grad(fd, f) for p in plans for fd, f in zip(p["fds"], p["flags"])])
    Dm = optimize.Matrix.from_csr(ctx, *D[:3], D[3])
    P = optimize.Problem(ctx, A, AT, Dm, Dm.transpose(), n_ptv, n_oar, np.full(n_ptv + n_oar, 1.1, np.float32),
                         np.ones(n_ptv + n_oar, np.float32), np.ones(n_ptv, np.float32), np.ones(n_ptv, np.float32),
                         np.full(n_oar, 0.05, np.float32), 1.0, 0.1)
    groups = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    bw = 0.1 * P.beam_weights_init(groups)
    x0 = np.full(A.shape[1], 0.01, np.float32)
    P.boo(groups, bw, x0, step_size=1e-3, iters=2, want=0, change_trigger=10 ** 9)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = P.boo(groups, bw, x0, step_size=1e-3, iters=opt_iters, want=0, change_trigger=10 ** 9)
    opt_s = time.perf_counter() - t0
    out = {"workload": f"multi-isocentre head and neck 256x256x200 @2.5mm, 4 isocentres, {n_beams} beams "
                       f"({min(counts)}-{max(counts)} beamlets), BEV grids 12/16/20/16, 8x6 cones",
           "beams": n_beams, "beamlets": n_bl, "nnz": int(nnz), "construction_ms": ms, "per_isocentre": per_iso,
           "beamlets_per_s": n_bl / (ms * 1e-3), "voi_rows": n_ptv + n_oar, "voi_nnz": A.info()["nnz"],
           "voi_restriction_s": voi_s, "opt_f16_it_per_s": r["k"] / opt_s,
           "opt_loss_first_last": [float(r["loss"][0]), float(r["loss"][r["k"] - 1])]}
    del P, A, AT, Dm
    torch.cuda.empty_cache()
    return out


def served_requests(ctx, n_requests, seed=11, n_phantoms=24):
    """Seeded plan requests of the served benchmark: a torso phantom whose
    sides are drawn from 96..256 voxels (2.5 mm), 1..50 beams from the 4pi
    sphere, 16x16 beamlet maps masked to the PTV.  The phantoms come from a
    pool of n_phantoms (each request draws its own beams), which keeps the
    request set cheap to build on the host."""
    from fastdose_b200 import api, phantoms
    from fastdose_b200.types import make_bundle

    rng = np.random.default_rng(seed)
    angles = phantoms.sphere_beam_angles(400)
    pool = []
    for i in range(min(n_phantoms, n_requests)):
        dim = tuple(int(v) for v in rng.integers(96, 257, size=3))
        ph = phantoms.torso_phantom(seed=100 + i, dim=dim, ptv_radius=2.5, ptv_offset=(1.5, 1.0, 0.0))
        pool.append((ph, phantoms.mask_centroid(ph.masks["PTV"], ph.voxel)))
    reqs = []
    for i in range(n_requests):
        ph, iso = pool[int(rng.integers(0, len(pool)))]
        sel = rng.choice(len(angles), size=int(rng.integers(1, 51)), replace=False)
        bundles = np.array([make_bundle(iso, angles[j], sad=100.0, fluence_dim=16, beamlet_size=0.5,
                                        sub_fluence_dim=16, sub_fluence_on=4, long_spacing=0.25) for j in sel])
        flags = api.beamletFlagInit(ctx, bundles, ph.masks["PTV"], ph.volume)
        beams = [b for b in api.bundles_beamlets(bundles, flags, ph.volume) if len(b)]
        if beams:
            reqs.append(dict(phantom=ph, beams=beams, fluence=api.beamlet_fluence(bundles[0])))
    return reqs


def _lat_stats(lat_s):
    lat = 1e3 * np.asarray(lat_s, np.float64)
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat.max()), "requests": int(lat.size)}


def served_leg(ctx, rates=(1.0, 5.0, 10.0, 20.0, 50.0), n_requests=200, seconds_per_rate=20.0, seed=11, workers=2,
               plain_requests=30, graph_rate=10.0):
    """p50/p99 plan latency (arrival -> dose-loading matrix on the device) and
    beamlets/s of the service under Poisson arrivals at each rate, over
    min(n_requests, max(30, rate * seconds_per_rate)) requests (seconds_per_rate
    0: n_requests at every rate); and of the plain form -- one request at a
    time, one beam per construction call -- run live at 1 request/s over the
    first plain_requests requests.  At higher rates the plain single server is
    overloaded (its utilisation, rate x mean service time, is reported); its
    latencies there are a FIFO replay of its service times of the same
    requests, measured live at 1/s for the first plain_requests and back to
    back for the rest.
    The service launches kernel by kernel; at graph_rate the same arrivals
    also run with each construction batch launched as one CUDA graph.  Before
    the sweep, the first 48 requests run once untimed in both forms."""
    import threading

    import torch

    from fastdose_b200 import api, phantoms, service

    spec, kern = phantoms.synthetic_spectrum(), phantoms.synthetic_kernel()
    reqs = served_requests(ctx, n_requests, seed)
    n_bl = [sum(len(b) for b in r["beams"]) for r in reqs]
    out = {"workload": f"{len(reqs)} requests: torso sides U[96,256] at 2.5 mm (a pool of 24 phantoms), 1-50 beams, "
                       f"16x16 PTV-masked beamlets ({sum(n_bl)} beamlets), 8x6 cones; Poisson arrivals",
           "beamlets": int(sum(n_bl))}
    rng = np.random.default_rng(seed + 1)

    # ---- the plain form, live: a single server, one beam per call, 1 request/s
    kk, ss = api.Kernel(ctx, kern), api.Spectrum(ctx, spec)
    st = torch.cuda.current_stream()
    n_plain = min(plain_requests, len(reqs))

    def plain_run(r):
        d = api.Density(ctx, r["phantom"].density, r["phantom"].volume)
        for b in r["beams"]:
            api.DoseMatConstruction(ctx, [b], r["fluence"], d, ss, kk, stream=st).close()
        d.close()
        torch.cuda.synchronize()

    plain_run(reqs[0])  # warm
    arrivals = np.cumsum(rng.exponential(1.0, size=n_plain))
    t0 = time.perf_counter()
    lat, service_s = [], []
    for a, r in zip(arrivals, reqs[:n_plain]):
        now = time.perf_counter() - t0
        if now < a:
            time.sleep(a - now)
        s0 = time.perf_counter()
        plain_run(r)
        end = time.perf_counter()
        service_s.append(end - s0)
        lat.append(end - t0 - a)
    plain_live = dict(_lat_stats(lat), rate_per_s=1.0, beamlets_per_s=sum(n_bl[:n_plain]) / (time.perf_counter() - t0),
                      mean_service_ms=1e3 * float(np.mean(service_s)))
    out["plain_live_1_per_s"] = plain_live
    # the plain form's service time of every other request the sweep runs,
    # back to back, so that its replay at each rate covers the same requests
    n_max = len(reqs) if seconds_per_rate <= 0 else min(len(reqs), max(30, int(max(rates) * seconds_per_rate)))
    for r in reqs[n_plain:n_max]:
        s0 = time.perf_counter()
        plain_run(r)
        service_s.append(time.perf_counter() - s0)

    svc = service.Service(device=torch.cuda.current_device(), workers=workers)
    big = int(np.argmax(n_bl))
    warmed = set()
    for _ in range(4 * workers):  # until every worker has run the largest request once
        tickets = [svc.submit(reqs[big]["phantom"], reqs[big]["beams"], reqs[big]["fluence"], spec, kern)
                   for _ in range(workers)]
        for t in tickets:
            m, s = svc.wait(t)
            m.close()
            warmed.add(int(s["worker"]))
        if len(warmed) == workers:
            break
    # one untimed pass over the request pool, kernel by kernel and with graphs,
    # so that the first rate of the sweep does not pay the workers' first-touch
    # allocations and graph instantiations that later rates no longer see
    for graph in (False, True):
        tickets = [svc.submit(r["phantom"], r["beams"], r["fluence"], spec, kern, graph=graph)
                   for r in reqs[:min(len(reqs), 48)]]
        for t in tickets:
            svc.wait(t)[0].close()
    arrivals = {}

    def run_rate(lam, n, graph):
        sub = reqs[:n]
        if lam not in arrivals:
            arrivals[lam] = np.cumsum(rng.exponential(1.0 / lam, size=n))
        arr = arrivals[lam]
        tickets = [None] * n
        t_base = svc.clock_ms()

        def submitter():
            for i, (a, r) in enumerate(zip(arr, sub)):
                delay = t_base + 1e3 * a - svc.clock_ms()
                if delay > 0:
                    time.sleep(delay * 1e-3)
                tickets[i] = svc.submit(r["phantom"], r["beams"], r["fluence"], spec, kern, graph=graph)

        with ClockSampler(torch.cuda.current_device()) as clk:
            th = threading.Thread(target=submitter)
            th.start()
            th.join()
            stats = []
            for t in tickets:
                m, s = svc.wait(t)
                m.close()
                stats.append(s)
        lat = np.array([s["end_ms"] - s["submit_ms"] for s in stats]) * 1e-3
        span_s = (max(s["end_ms"] for s in stats) - min(s["submit_ms"] for s in stats)) * 1e-3
        return arr, dict(_lat_stats(lat), beamlets_per_s=sum(n_bl[:n]) / span_s, workers=workers, graph=graph,
                         queue_p50_ms=float(np.percentile([s["start_ms"] - s["submit_ms"] for s in stats], 50)),
                         # per request (arrival order): beamlets, worker, submit ms (from the first
                         # submit), queue ms, run ms
                         timeline=[[int(s["beamlets"]), int(s["worker"]), round(s["submit_ms"] - stats[0]["submit_ms"], 1),
                                    round(s["start_ms"] - s["submit_ms"], 1), round(s["end_ms"] - s["start_ms"], 1)]
                                   for s in stats],
                         clocks=clk.summary())

    for lam in rates:
        n = len(reqs) if seconds_per_rate <= 0 else min(len(reqs), max(30, int(lam * seconds_per_rate)))
        arr, svc_stats = run_rate(lam, n, graph=False)
        # the plain single server at this rate: FIFO replay of its measured
        # service times of the same n requests
        end, rl = 0.0, []
        for a, sv in zip(arr[:n], service_s[:n]):
            end = max(end, a) + sv
            rl.append(end - a)
        key = f"rate_{lam:g}_per_s"
        out[key] = {
            "service": svc_stats,
            "plain_single_beam": dict(_lat_stats(rl), utilisation=lam * float(np.mean(service_s[:n])), requests=n,
                                      basis="live" if lam == 1.0 else
                                      f"FIFO replay at this rate of the plain form's service times of the same "
                                      f"{n} requests (the first {n_plain} timed live at 1/s, the rest back to back)"),
        }
        if lam == 1.0:
            out[key]["plain_single_beam"].update({k: plain_live[k] for k in ("p50_ms", "p99_ms", "max_ms")},
                                                 basis="live")
    if graph_rate and f"rate_{graph_rate:g}_per_s" in out:
        n = min(len(reqs), max(30, int(graph_rate * seconds_per_rate))) if seconds_per_rate > 0 else len(reqs)
        _, on = run_rate(graph_rate, n, graph=True)  # the same arrivals, one graph per construction batch
        on.pop("timeline")
        out[f"rate_{graph_rate:g}_per_s"]["service_with_graphs"] = on
    svc.close()
    return out


def single_beam_leg(ctx, beamlets, fluence, dens, spec, kern, stream, n_beams=20):
    """The plain single-beam form: the same beams one DoseMatConstruction call
    (one beam) at a time, as the reference's per-beam loop runs them."""
    import torch

    from fastdose_b200 import api

    sel = beamlets[:n_beams]
    for b in sel[:2]:
        api.DoseMatConstruction(ctx, [b], fluence, dens, spec, kern, stream=stream).close()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for b in sel:
        api.DoseMatConstruction(ctx, [b], fluence, dens, spec, kern, stream=stream).close()
    e1.record(stream)
    torch.cuda.synchronize()
    n = int(sum(len(b) for b in sel))
    return {"beams": len(sel), "beamlets": n, "value": n / (e0.elapsed_time(e1) * 1e-3), "unit": UNIT}


def reference_cuda_leg(ctx, cfg, bundles, flags, all_beamlets, fluence, dens, spec, stream, value_8x6, every=8):
    """The reference's own CUDA build on this B200 (oracle/_ref/libfdref.so:
    its sources compiled unmodified for sm_100a) beside this library, both on
    the 8x8 cone kernel of the same seed: IMRT::DoseMatConstruction's per-beam
    steps (Terma, CCCS, BEV2PVCSInterp into the dense matrix, cuSPARSE
    dense-to-CSR; one beam at a time, as its loop runs) over every
    `every`-th beam of the plan, and this library on the same beams -- batched
    in one call, and one beam per call -- and batched on the whole plan.
    The reference's march with the plan's 8x6 kernel never ends (a cone at
    phi = 90 degrees has a zero direction component in its fast-math build),
    so the comparison uses 8 azimuths.  A baseline leg: nothing here is this
    library's product path."""
    import torch

    from fastdose_b200 import api, phantoms
    from oracle import ref

    if not ref.available():
        return {"unavailable": "oracle/_ref/libfdref.so is not built (oracle/build_ref.sh needs the reference sources)"}
    ph = cfg["phantom"]
    k88 = phantoms.synthetic_kernel(n_theta=8, n_phi=8)
    sel = [i for i in range(0, len(bundles), every) if len(all_beamlets[i])]
    r = ref.dose_mat_steps(bundles[sel], flags[sel], ph.density, ph.volume, cfg["spectrum"], k88, extent=cfg["extent"])
    if r["status"] != 0:
        return {"unavailable": f"reference DoseMatConstruction steps returned {r['status']}"}
    t = r["times_ms"]
    out = {"sample": f"every {every}th beam of the plan: {len(sel)} beams, {int(r['beamlets'])} beamlets, 8x8 cones",
           "reference": {"beamlets_per_s": r["beamlets"] / (float(t[4]) * 1e-3), "ms": float(t[4]),
                         "stage_ms": {"terma": float(t[0]), "cccs": float(t[1]), "interp": float(t[2]),
                                      "dense_to_csr": float(t[3])},
                         "nnz": int(r["nnz"].sum()),
                         "note": "IMRTDoseMat.cu:183-259 run step by step by oracle/ref/ref_harness.cu; the "
                                 "supervoxel flag array gets slack (its kernel writes past it on volumes that are "
                                 "not a multiple of 32 voxels) and the BEV dose is cleared between beams"}}
    kern88 = api.Kernel(ctx, k88)
    beams_sel = [all_beamlets[i] for i in sel]

    def timed(fn, reps=1):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    n_sel = int(sum(len(b) for b in beams_sel))
    ms_b = timed(lambda: api.DoseMatConstruction(ctx, beams_sel, fluence, dens, spec, kern88, stream=stream).close(), 2)
    ms_1 = timed(lambda: [api.DoseMatConstruction(ctx, [b], fluence, dens, spec, kern88, stream=stream).close()
                          for b in beams_sel])
    n_all = int(sum(len(b) for b in all_beamlets))
    ms_all = timed(lambda: api.DoseMatConstruction(ctx, all_beamlets, fluence, dens, spec, kern88,
                                                   stream=stream).close(), 2)
    out["fd2"] = {"batched_beamlets_per_s": n_sel / (ms_b * 1e-3), "per_beam_beamlets_per_s": n_sel / (ms_1 * 1e-3),
                  "whole_plan_batched_beamlets_per_s": n_all / (ms_all * 1e-3),
                  "whole_plan_8x6_beamlets_per_s": value_8x6}
    refv = out["reference"]["beamlets_per_s"]
    out["speedup_vs_reference"] = {"batched_same_beams": out["fd2"]["batched_beamlets_per_s"] / refv,
                                   "per_beam_same_beams": out["fd2"]["per_beam_beamlets_per_s"] / refv,
                                   "whole_plan_batched": out["fd2"]["whole_plan_batched_beamlets_per_s"] / refv}
    return out


def c1_leg(ctx, stream, reps=20):
    """C1, plain CCCS of one beam: the 64^3 slab phantom, gantry 0, 10x10 open
    beamlets of 0.5 cm (16x16 sub-maps).  This library's whole construction
    (Terma, CCCS, columns) per plan with the plan's 8x6 cones and with 8x8,
    CUDA events over `reps` plans; beside it the reference's own CUDA build
    (oracle/_ref/libfdref.so) running IMRT::DoseMatConstruction's per-beam
    steps on the same beam with the 8x8 kernel (its 8x6 march never ends).
    A baseline leg: nothing here is this library's product path."""
    import torch

    from fastdose_b200 import api, phantoms
    from fastdose_b200.types import make_bundle

    cfg = phantoms.config1()
    ph = cfg["phantom"]
    bund = make_bundle(cfg["isocenter"], cfg["angles"][0], sad=cfg["sad"], fluence_dim=cfg["fluence_dim"],
                       beamlet_size=cfg["beamlet_size"], sub_fluence_dim=cfg["sub_fluence_dim"],
                       sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"])
    flags = np.ones(cfg["fluence_dim"] ** 2, np.uint8)
    beams = api.bundle_beamlets(bund, flags, ph.volume)
    fluence = api.beamlet_fluence(bund)
    dens, spec = api.Density(ctx, ph.density, ph.volume), api.Spectrum(ctx, cfg["spectrum"])
    k88 = phantoms.synthetic_kernel(n_theta=8, n_phi=8)
    out = {"workload": "64^3 slab phantom at 2.5 mm (bone and lung slabs), one beam at gantry 0, 10x10 open "
                       "beamlets of 0.5 cm, 16x16 sub-maps, 12-bin spectrum", "beamlets": int(len(beams))}
    for name, kern in (("8x6", cfg["kernel"]), ("8x8", k88)):
        kn = api.Kernel(ctx, kern)
        for _ in range(3):
            api.DoseMatConstruction(ctx, [beams], fluence, dens, spec, kn, stream=stream).close()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            api.DoseMatConstruction(ctx, [beams], fluence, dens, spec, kn, stream=stream).close()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[f"fd2_{name}"] = {"ms_per_plan": ms, "beamlets_per_s": len(beams) / (ms * 1e-3)}
    from oracle import ref

    if not ref.available():
        out["reference_8x8"] = {"unavailable": "oracle/_ref/libfdref.so is not built"}
        return out
    runs = []
    for _ in range(4):
        r = ref.dose_mat_steps(np.array([bund]), flags.reshape(1, -1), ph.density, ph.volume, cfg["spectrum"], k88,
                               extent=cfg["extent"])
        if r["status"] != 0:
            out["reference_8x8"] = {"unavailable": f"reference DoseMatConstruction steps returned {r['status']}"}
            return out
        runs.append([float(x) for x in r["times_ms"]])
    t = min(runs[1:], key=lambda x: x[4])  # the first run warms the reference's code path
    out["reference_8x8"] = {"ms_per_plan": t[4], "beamlets_per_s": r["beamlets"] / (t[4] * 1e-3),
                            "stage_ms": {"terma": t[0], "cccs": t[1], "interp": t[2], "dense_to_csr": t[3]},
                            "note": "IMRTDoseMat.cu:183-259 run step by step by oracle/ref/ref_harness.cu; the "
                                    "fastest of three runs after one warm-up"}
    out["speedup_vs_reference_8x8"] = out["fd2_8x8"]["beamlets_per_s"] / out["reference_8x8"]["beamlets_per_s"]
    return out


def run_fd2(args, rank, world):
    import torch
    import torch.distributed as dist

    from fastdose_b200 import api, sharding

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    ctx = api.Context(dev)
    # N ranks: a 4pi candidate set of N x `beams` beams, partitioned by beam
    # across the ranks (greedy balance on the CCCS march length); each rank
    # builds the dose-loading matrix of its share, with no collective
    cfg, bundles = plan_inputs(args.beams * world)
    ph = cfg["phantom"]
    flags = api.beamletFlagInit(ctx, bundles, ph.masks["PTV"], ph.volume)
    all_beamlets = api.bundles_beamlets(bundles, flags, ph.volume)
    parts = sharding.partition_beams(sharding.beam_costs(all_beamlets), world)
    beamlets = [all_beamlets[i] for i in parts[rank]]
    n_bl_total = int(sum(len(b) for b in all_beamlets))
    n_bl = int(sum(len(b) for b in beamlets))
    fluence = api.beamlet_fluence(bundles[0])
    spec = api.Spectrum(ctx, cfg["spectrum"])
    kern = api.Kernel(ctx, cfg["kernel"])
    dens = api.Density(ctx, ph.density, ph.volume)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    def step_device():
        m = api.DoseMatConstruction(ctx, beamlets, fluence, dens, spec, kern, stream=stream)
        info = m.info()
        m.close()
        return info

    # ---- device-resident timing
    for _ in range(args.warmup):
        info = step_device()
    launches0 = ctx.launch_count()
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            info = step_device()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    launches = (ctx.launch_count() - launches0) // args.steps
    # stage breakdown from one extra, instrumented step (its event waits serialise
    # the host, so it is kept out of the timed loop)
    ctx.set_timing(True)
    ctx.stage_times()
    step_device()
    stages = ctx.stage_times()
    ctx.set_timing(False)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    value = n_bl_total * args.steps / (ms * 1e-3)

    # ---- end to end through the public API: pinned host inputs, CSR read back
    dens_host = torch.from_numpy(np.ascontiguousarray(ph.density)).pin_memory()
    beams_host = torch.from_numpy(np.concatenate(beamlets).view(np.uint8).copy()).pin_memory()

    from fastdose_b200.types import BEAM_DTYPE

    hb = beams_host.numpy().view(BEAM_DTYPE)
    per, o = [], 0
    for b in beamlets:
        per.append(hb[o:o + len(b)])
        o += len(b)
    dens_np = dens_host.numpy().reshape(ph.density.shape)

    # The matrix comes back to pinned host buffers while it is built: each
    # batch's rows are copied on a copy stream during the next batch's device
    # work (host_out), so only the last batch's copy follows the construction.
    host = api.HostCSR(n_bl, info["nnz"])
    e2e_batch = args.e2e_batch if args.e2e_batch >= 0 else max(4096, -(-n_bl // 6))

    def step_e2e():
        # the library copies the density volume and the beamlet descriptors from these pinned host buffers
        dn = api.Density(ctx, dens_np, ph.volume)
        m = api.DoseMatConstruction(ctx, per, fluence, dn, spec, kern, stream=stream, host_out=host,
                                    batch_beamlets=e2e_batch)
        m.close()
        dn.close()
        return host.nbytes()

    for _ in range(max(1, min(args.warmup, 2))):
        d2h = step_e2e()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        d2h = step_e2e()
    torch.cuda.synchronize()
    barrier()
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = n_bl_total * args.steps / float(te.item())
    h2d = dens_host.numel() * 4 + beams_host.numel()

    # ---- roofline of the dominant kernel (the CCCS march)
    P = 16 * 16
    L = np.concatenate([b["long_dim"] for b in beamlets]).astype(np.float64)
    cccs_bytes = float(np.sum(4.0 * P * L * 3))  # Terma + density read, dose written, per beamlet
    # DRAM bytes the CCCS kernel moves per beamlet: dram__bytes_read.sum + dram__bytes_write.sum of one
    # ncu capture of the march on the 40-beam plan (6056 beamlets, 38.0 GB),
    # scaled by the beamlets of this step (each zenith pass re-reads its slices: traffic grows with beamlets)
    cccs_traffic = CCCS_DRAM_BYTES_PER_BEAMLET * n_bl
    cccs_ms = stages["cccs"]
    peak, peak_kind = _peaks()
    achieved = cccs_bytes / (cccs_ms * 1e-3) / 1e9 if cccs_ms > 0 else None
    # The march's special-function roof: each ray step costs 3 MUFU operations
    # (two exp2, one rsqrt) for each of the P rays; a base ray in normalised BEV
    # units (pixels laterally, slices in depth) crosses L (1 + (|dx| + |dy|) / dz)
    # voxel boundaries over the L slices of one (zenith, azimuth) pass.  Peak: 16
    # MUFU results per clock per SM (the CUDA throughput table) at the sampled clock.
    dirs = api.cone_directions(ctx, kern, np.concatenate(beamlets))  # [beamlet, theta, phi, 4]
    ratio = (np.abs(dirs[..., 0]) + np.abs(dirs[..., 1])) / np.maximum(dirs[..., 2], 1e-6)
    ray_steps = float(np.sum(L[:, None, None] * (1.0 + ratio)))
    sfu_ops = ray_steps * P * 3.0
    clk_now = clk.summary()
    sm_mhz = clk_now.get("sm_mhz") or 1965.0
    sfu_peak = 16.0 * (torch.cuda.get_device_properties(dev).multi_processor_count) * sm_mhz * 1e6
    sfu_achieved = sfu_ops / (cccs_ms * 1e-3) if cccs_ms > 0 else None
    # The march's binding roof is instruction issue: warp instructions per
    # beamlet from the ncu capture, over the CUDA-event CCCS time, against 4
    # warp instructions per clock per SM (one per sub-partition) at the sampled
    # SM clock.
    issue_inst = CCCS_WARP_INST_PER_BEAMLET * n_bl
    issue_peak = 4.0 * torch.cuda.get_device_properties(dev).multi_processor_count * sm_mhz * 1e6
    issue_achieved = issue_inst / (cccs_ms * 1e-3) if cccs_ms > 0 else None
    # The whole pipeline against HBM under the compulsory-traffic convention:
    # per beamlet Terma and density written and read, dose written and read
    # (4 P L 6), the density footprint read once (taken as its nonzero count),
    # the column's value and index written (4 + 4 per nonzero), and the offsets.
    pipe_bytes = float(np.sum(4.0 * P * L * 6)) + float(info["nnz"]) * (4 + 4 + 4) + 8.0 * (n_bl + 1)
    pipe_ms = ms / args.steps
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(len(bundles), n_bl_total), "beams": len(bundles), "beamlets": n_bl_total,
                   "beams_per_rank": [len(p) for p in parts],
                   "nnz": int(info["nnz"]), "l2": "inputs and BEV scratch larger than L2 (126 MB)",
                   "parallelism": f"beams partitioned over {world} GPU(s), no collective"},
        "stage_ms_per_step": {k: v for k, v in stages.items() if v},
        "gpu_launches": int(launches),
        "cccs_tuned": {"schedules": {str(k): v for k, v in ctx.tuned_schedules()[0].items()},
                       "tuning_runs": ctx.tuned_schedules()[1]},
        "roofline": {"bound": "hbm", "kernel": "cccs_kernel", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "traffic": cccs_traffic,
                     "peak_source": peak_kind, "algorithmic_bytes_per_step": cccs_bytes},
        "sfu_roofline": {"bound": "MUFU", "kernel": "cccs_kernel", "ops_per_step": sfu_ops, "ray_steps": ray_steps,
                         "achieved_ops_per_s": sfu_achieved, "peak_ops_per_s": sfu_peak,
                         "frac": sfu_achieved / sfu_peak if sfu_achieved else None,
                         "basis": "3 MUFU per ray step; ray steps L (1 + (|dx|+|dy|)/dz) per cone pass from the "
                                  "device's cone directions; peak 16/clk/SM at the sampled SM clock"},
        "issue_roofline": {"bound": "issue", "kernel": "cccs_kernel", "warp_instructions_per_step": issue_inst,
                           "achieved": issue_achieved, "peak": issue_peak, "unit": "warp instructions/s",
                           "frac": issue_achieved / issue_peak if issue_achieved else None,
                           "basis": "warp instructions per beamlet from one ncu capture of the 40-beam plan "
                                    "(smsp__inst_executed.sum / beamlets), scaled by this step's beamlets; "
                                    "peak 4 per clock per SM at the sampled SM clock"},
        "pipeline_roofline": {"bound": "hbm", "bytes_per_step": pipe_bytes, "ms_per_step": pipe_ms,
                              "achieved": pipe_bytes / (pipe_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                              "frac": pipe_bytes / (pipe_ms * 1e-3) / 1e9 / peak,
                              "basis": "per beamlet 4 P L 6 + 4 per footprint voxel (taken as its nonzeros) + "
                                       "8 per nonzero (value, index) + 8 per row offset"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "batch_beamlets": int(e2e_batch), "read_back": "pinned, overlapped with the next batch"},
        "clocks": clk_now,
    }
    if world > 1 and not args.no_extras:
        # the single-GPU legs (one beam per call, reference CUDA, optimizer,
        # C4, served) belong to the 1-GPU line; a multi-GPU run times the
        # sharded construction only
        line["extras"] = "single-GPU legs are reported by the 1-GPU run"
    if world == 1 and not args.no_extras:
        sb = single_beam_leg(ctx, beamlets, fluence, dens, spec, kern, stream)
        sb["batched_speedup"] = value / sb["value"]
        line["single_beam"] = sb
        line["reference_cuda"] = reference_cuda_leg(ctx, cfg, bundles, flags, all_beamlets, fluence, dens, spec,
                                                    stream, value)
        line["c1"] = c1_leg(ctx, stream)
        line["optimizer"] = optimizer_leg(ctx, args.opt_iters, args.opt_rows)
        line["c4"] = c4_leg(ctx)
        # the service's worker contexts start from a device the earlier legs
        # have handed back, as a service process would find it
        import gc

        gc.collect()
        torch.cuda.empty_cache()
        ctx.release()
        line["served"] = served_leg(ctx, rates=tuple(float(r) for r in args.served_rates.split(",")),
                                    n_requests=args.served_requests, seconds_per_rate=args.served_seconds,
                                    workers=args.served_workers)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, beamlets, fluence, args.cpu_seconds, os.cpu_count() or 1)[0]
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fd2", choices=["fd2", "reference"])
    ap.add_argument("--beams", type=int, default=400)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the single-beam and optimizer legs")
    ap.add_argument("--opt-iters", type=int, default=500)
    ap.add_argument("--opt-rows", type=int, default=2_500_000)
    ap.add_argument("--only-optimizer", action="store_true", help="run the optimizer leg alone (profiling)")
    ap.add_argument("--only-c1", action="store_true", help="time config 1 (one beam, 64^3) alone")
    ap.add_argument("--only-spmv", default=None, choices=["f32_i32", "f32_packed16", "f16_packed16", "bf16_packed16"],
                    help="time A x and A^T y of the optimization matrix in one format (profiling)")
    ap.add_argument("--spmv-reps", type=int, default=10)
    ap.add_argument("--served-workers", type=int, default=2)
    ap.add_argument("--served-requests", type=int, default=200)
    ap.add_argument("--served-seconds", type=float, default=20.0,
                    help="arrival seconds per rate (caps the requests at low rates); 0: all requests at every rate")
    ap.add_argument("--plain-requests", type=int, default=30, help="requests of the live plain-form run")
    ap.add_argument("--served-rates", default="1,5,10,20,50", help="arrival rates (requests/s) of the served leg")
    ap.add_argument("--e2e-batch", type=int, default=-1,
                    help="beamlets per construction batch of the end-to-end leg (-1: a sixth of the plan, >= 4096)")
    ap.add_argument("--c4", action="store_true", help="run the multi-isocentre configuration alone")
    ap.add_argument("--only-served", action="store_true", help="run the served leg alone")
    args = ap.parse_args()
    if args.c4:
        import torch

        from fastdose_b200 import api

        torch.cuda.set_device(0)
        print(json.dumps({"c4": c4_leg(api.Context(0))}), flush=True)
        return
    if args.only_c1:
        import torch

        from fastdose_b200 import api

        print(json.dumps({"c1": c1_leg(api.Context(0), torch.cuda.current_stream())}), flush=True)
        return
    if args.only_spmv:
        import torch

        from fastdose_b200 import api

        torch.cuda.set_device(0)
        print(json.dumps({"spmv": spmv_leg(api.Context(0), args.only_spmv, args.opt_rows, reps=args.spmv_reps)}),
              flush=True)
        return
    if args.only_optimizer or args.only_served:
        import torch

        from fastdose_b200 import api

        torch.cuda.set_device(0)
        ctx = api.Context(0)
        if args.only_optimizer:
            print(json.dumps({"optimizer": optimizer_leg(ctx, args.opt_iters, args.opt_rows)}), flush=True)
        else:
            print(json.dumps({"served": served_leg(ctx, rates=tuple(float(r) for r in args.served_rates.split(",")),
                                                   n_requests=args.served_requests,
                                                   seconds_per_rate=args.served_seconds,
                                                   workers=args.served_workers, plain_requests=args.plain_requests)}),
                  flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_fd2(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
