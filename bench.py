"""Benchmark of the surfacelet analyze/synthesize path on B200.

Workload (one step, per rank): NSSurfacelet(scales = 3, direction_levels =
[2, 2, 3]) on a batch of float32 128^3 volumes, i.i.d. N(0, 1) from a seeded
generator: analyze, synthesize, and the adjoint of synthesize, per volume.
Metric: Mvoxels/s of input volume through analyze + synthesize + adjoint,
whole job (all ranks).  Each volume's coefficients are 411 MB, larger than
the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl reference]

Under torchrun (N > 1) each rank runs its own batch (weak scaling, no
data-path collective); the elapsed time is the max over ranks.  The line
also carries: e2e (the same step through the public API with pinned host
buffers, copies inside the timed region), the roofline of the dominant kernel
(CUDA-event launch times from a profiled replay), the float64-oracle CPU
baseline, the plain unfused GPU form (cuFFT through torch, timing comparison
only), and the decimated Surfacelet 128^3 line as `secondary`.
"""

import argparse
import datetime
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "Mvoxels/s analyze+synthesize(+adjoint), fused vs plain GPU at rel.err ≤1e-5"
DIMS = (128, 128, 128)
NS_KW = dict(scales=3, direction_levels=[2, 2, 3])
DEC_KW = dict(scales=3, direction_levels=[2, 2, 3], pyramid_ratio=2)


def load_package():
    name = "surfacelets_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = os.path.join(ROOT, "surfacelets.jl_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ── clocks during the timed region ──────────────────────────────────────────


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        if not sm:
            return None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "samples": len(sm),
                "reasons": sorted(reasons)}


# ── the reference arm: the oracle port on the host cores ────────────────────


def run_reference(args, rank):
    if rank != 0:
        return
    sys.path.insert(0, ROOT)
    from oracle import ns as N
    from oracle.cpu_baseline import NSBaseline
    cores = os.cpu_count()
    base = NSBaseline(N.NSParams.make(**NS_KW), DIMS, np.float32, workers=cores)
    x = np.random.default_rng(0).standard_normal(DIMS).astype(np.float32)

    def step():
        c = base.analyze(x)
        y = base.synthesize(c)
        base.analyze(y, synth_masks=True)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    v = float(np.prod(DIMS)) / dt / 1e6
    line = {
        "metric": METRIC, "value": v, "unit": "Mvoxels/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "NSSurfacelet(scales=3, direction_levels=[2,2,3]) 128^3 float32, "
                               "analyze+synthesize+adjoint of one volume per step", "batch": 1},
        "cpu_baseline": {"value": v, "unit": "Mvoxels/s", "cores": cores, "kind": "port",
                         "sample": "one 128^3 volume analyze+synthesize+adjoint per step, scipy.fft "
                                   f"with workers={cores}, float32 masks from the float64 oracle"},
        "e2e": {"value": v, "unit": "Mvoxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ── our arm ──────────────────────────────────────────────────────────────────


def kernel_bytes(tag, P, launches_per_step, nz_total):
    """Algorithmic bytes of all launches of `tag` in one profiled step: each
    input read once and each output written once (float32 volumes: 4 B a
    voxel; spectra on the rfft grid: 8 B a bin)."""
    N = float(np.prod(DIMS))
    H = float((DIMS[0] // 2 + 1) * DIMS[1] * DIMS[2])
    per_item = {
        "ns_r2c_axis1": 4 * N + 8 * H,
        "ns_c2r_axis1": 8 * H + 4 * N,
        "ns_c2c_axis2": 16 * H,
        "ns_c2c_axis3": 16 * H,
        "ns_mask_axis3": 8 * H,
        "ns_accum_axis3": 8 * H,
    }.get(tag)
    if per_item is None:
        return None
    extra = {"ns_mask_axis3": 8 * H, "ns_accum_axis3": 32 * H}.get(tag, 0.0)
    return per_item * nz_total + extra * launches_per_step


_SGEMM = []


def sgemm_tflops():
    """Measured FP32 peak: cuBLAS SGEMM of 8192^3 with TF32 off, best of five."""
    if not _SGEMM:
        import torch
        prev = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = False
        n = 8192
        a = torch.randn(n, n, device="cuda")
        b = torch.randn(n, n, device="cuda")
        torch.matmul(a, b)
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        torch.backends.cuda.matmul.allow_tf32 = prev
        del a, b
        torch.cuda.empty_cache()
        _SGEMM.append(2.0 * n ** 3 / (best / 1e3) / 1e12)
    return _SGEMM[0]


def host64(t):
    """A column-major device volume as a float64 NumPy array (Julia axis order)."""
    return np.asfortranarray(t.permute(*reversed(range(t.dim()))).cpu().numpy().transpose()).astype(np.float64)


def oracle_errors(x, c, y, g):
    """rel. L2 against the float64 oracle of one timed volume's analysis
    coefficients c = A x, its synthesis y = S c and the adjoint g = S^T y,
    each streamed subband by subband (host threads for the FFTs)."""
    sys.path.insert(0, ROOT)
    from oracle import ns as ON
    ON.set_fft_workers(os.cpu_count() or 1)
    try:
        T = ON.make_tables(ON.NSParams.make(**NS_KW), DIMS)
        S = c.shape[-1]

        def rel_stream(gen, dev):
            e2 = r2 = 0.0
            for s, band in gen:
                e2 += float(np.sum((host64(dev[..., s - 1]) - band) ** 2))
                r2 += float(np.sum(band ** 2))
            return float(np.sqrt(e2 / r2))

        ra = rel_stream(ON.analyze_stream(T, host64(x)), c)
        yref = ON.synthesize_stream(T, lambda s: host64(c[..., s - 1]))
        rs = float(np.linalg.norm(host64(y) - yref) / np.linalg.norm(yref))
        Y = ON.rfft3(host64(y))
        rg = rel_stream(((s, ON.irfft3(Y * M, DIMS)) for s, M in ON.subband_masks(T, analysis=False)), g)
    finally:
        ON.set_fft_workers(1)
    return {"analyze_rel_l2": ra, "synthesize_rel_l2": rs, "adjoint_synthesize_rel_l2": rg,
            "volume": "the first volume of the timed batch, all %d subbands" % S}


def run_decimated(args):
    """The decimated Surfacelet(scales=3, direction_levels=[2,2,3], pyramid_ratio=2) alone:
    analyze + synthesize of a batch of float32 volumes as plain calls on one workspace.  This is
    the workload of its launch list and kernel captures; it prints one JSON line with the step time
    and the per-kernel CUDA-event times of a profiled replay (the headline stays the default
    NSSurfacelet workload)."""
    import ctypes as C

    import torch
    torch.cuda.set_device(0)
    sfl = load_package()
    lib = sfl.lib
    B = args.batch
    N = int(np.prod(DIMS))
    wd = sfl.make_workspace(sfl.Surfacelet(**DEC_KW), "float32", DIMS)
    gen = torch.Generator(device="cuda").manual_seed(1234)
    xs = [sfl.volume_like(DIMS).copy_(torch.randn(DIMS, device="cuda", generator=gen)) for _ in range(B)]
    cds = [torch.empty(wd.ncoeffs, device="cuda") for _ in range(B)]
    yds = [sfl.volume_like(DIMS) for _ in range(B)]

    def step():
        for b in range(B):
            sfl.analyze_(cds[b], wd, xs[b])
            sfl.synthesize_(yds[b], wd, cds[b])

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    rel = float(torch.linalg.vector_norm(yds[0] - xs[0]) / torch.linalg.vector_norm(xs[0]))
    lib.sfl_profile_reset()
    lib.sfl_profile_enable(1)
    step()
    torch.cuda.synchronize()
    lib.sfl_profile_enable(0)
    buf = C.create_string_buffer(8192)
    lib.sfl_profile_tags(buf, 8192)
    kernels = {}
    for tg in [v for v in buf.value.decode().split("\n") if v]:
        tot, cnt = C.c_double(), C.c_int64()
        lib.sfl_profile_read(tg.encode(), C.byref(tot), C.byref(cnt))
        kernels[tg] = {"ms_per_step": tot.value, "launches_per_step": cnt.value}
    lib.sfl_profile_reset()
    r = DEC_KW["pyramid_ratio"]
    print(json.dumps({
        "metric": "Mvoxels/s analyze+synthesize", "value": B * N / (ms / 1e3) / 1e6, "unit": "Mvoxels/s",
        "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"Surfacelet(scales=3, direction_levels=[2,2,3], pyramid_ratio={r}) "
                               + "x".join(str(d) for d in DIMS) + " float32, analyze+synthesize, plain calls",
                   "batch": B},
        "perfect_reconstruction_rel_l2": rel, "kernels": kernels}))


def main():
    global DIMS, NS_KW
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip plain/secondary/cpu legs")
    ap.add_argument("--group", type=int, default=0, help="subbands in flight per launch (0: the plan's default)")
    ap.add_argument("--workspaces", type=int, default=4, help="graph mode: workspaces (concurrent branches, <= 8)")
    ap.add_argument("--dims", type=int, nargs=3, default=list(DIMS),
                    help="volume size (a smaller or larger case for profiling; the extra lines need the default)")
    ap.add_argument("--levels", type=int, nargs="+", default=NS_KW["direction_levels"],
                    help="direction levels per scale (scales = their count)")
    ap.add_argument("--workload", default="ns", choices=["ns", "decimated"],
                    help="decimated: the decimated Surfacelet 128^3 alone, for its profiles (not the headline)")
    ap.add_argument("--mode", default="graph", choices=["graph", "calls"],
                    help="graph: the batch as one CUDA graph over up to 4 workspaces (sfl_batch_*); "
                         "calls: a loop of plain calls on one workspace")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    if tuple(args.dims) != DIMS or list(args.levels) != NS_KW["direction_levels"]:
        DIMS = tuple(args.dims)
        NS_KW = dict(scales=len(args.levels), direction_levels=list(args.levels))
        args.no_extras = True   # the extra lines are defined on the default workload
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "decimated":
        DIMS = tuple(args.dims)
        run_decimated(args)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local))
    sfl = load_package()
    B = args.batch
    N = int(np.prod(DIMS))
    t = sfl.NSSurfacelet(**NS_KW)
    nws = min(args.workspaces, B) if args.mode == "graph" else 1
    wss = [sfl.make_workspace(t, "float32", DIMS) for _ in range(nws)]
    for w in wss:
        if args.group > 0:
            w.set_group(args.group)
    ws = wss[0]
    S = ws.nsubbands
    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    xs = [sfl.volume_like(DIMS).copy_(torch.randn(DIMS, device="cuda", generator=gen)) for _ in range(B)]
    cs = [sfl.volume_like(DIMS + (S,)) for _ in range(B)]
    gs = [sfl.volume_like(DIMS + (S,)) for _ in range(B)]
    ys = [sfl.volume_like(DIMS) for _ in range(B)]

    def step_calls():
        for b in range(B):
            sfl.analyze_(cs[b], ws, xs[b])
            sfl.synthesize_(ys[b], ws, cs[b])
            sfl.adjoint_synthesize_(gs[b], ws, ys[b])

    if args.mode == "graph":
        # volume b on workspace b mod 4: analyze, synthesize, adjoint in order on its branch
        ents = [(wss[b % nws], op, i, o) for b in range(B)
                for op, i, o in (("analyze", xs[b], cs[b]), ("synthesize", cs[b], ys[b]),
                                 ("adjoint_synthesize", ys[b], gs[b]))]
        batch = sfl.Batch([e[0] for e in ents], [e[2] for e in ents], [e[3] for e in ents], [e[1] for e in ents])

        def step():
            batch.run()
    else:
        step = step_calls

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(fn, steps):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1) / steps
        if world > 1:
            v = torch.tensor([ms], device="cuda")
            dist.all_reduce(v, op=dist.ReduceOp.MAX)
            ms = float(v.item())
        return ms

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local) if rank == 0 else None
    if clocks:
        clocks.start()
    ms = timed(step, args.steps)
    clk = clocks.stop() if clocks else None
    value = B * N * world / (ms / 1e3) / 1e6

    # correctness of the timed data: perfect reconstruction and A^T = A (tight)
    rel_pr = max(float(torch.linalg.vector_norm(ys[b] - xs[b]) / torch.linalg.vector_norm(xs[b])) for b in range(B))
    rel_adj = float(torch.linalg.vector_norm(gs[0] - cs[0]) / torch.linalg.vector_norm(cs[0]))
    # and against the float64 oracle: one timed volume's three outputs (rank 0, outside the timed region)
    vs_oracle = oracle_errors(xs[0], cs[0], ys[0], gs[0]) if rank == 0 else None

    # profiled replay: launch counts and per-kernel CUDA-event times
    lib = sfl.lib
    lib.sfl_profile_reset()
    lib.sfl_profile_enable(1)
    prof_steps = 2
    for _ in range(prof_steps):
        step_calls()
    torch.cuda.synchronize()
    lib.sfl_profile_enable(0)
    import ctypes as C
    buf = C.create_string_buffer(4096)
    lib.sfl_profile_tags(buf, 4096)
    tags = [s for s in buf.value.decode().split("\n") if s]
    per_tag, tag_bytes = {}, {}
    for tg in tags:
        tot, cnt, nb = C.c_double(), C.c_int64(), C.c_double()
        lib.sfl_profile_read(tg.encode(), C.byref(tot), C.byref(cnt))
        lib.sfl_profile_bytes(tg.encode(), C.byref(nb))
        per_tag[tg] = (tot.value / prof_steps, cnt.value // prof_steps)
        tag_bytes[tg] = nb.value / prof_steps
    lib.sfl_profile_reset()
    launches_per_step = sum(c for _, c in per_tag.values())
    dom = max(per_tag, key=lambda k: per_tag[k][0])
    dom_ms, dom_launches = per_tag[dom]
    # items processed per step by the dominant kernel (sum of grid.y over its launches)
    # spectra/volumes each kernel tag processes per step (grid.y summed over its launches):
    # analyze = rfft3 + per subband (mask pass, axis-2 pass, C2R); synthesize = per subband
    # (R2C, axis-2 pass, accumulation) + irfft3; the adjoint of synthesize is an analysis.
    nz_total = {
        "ns_r2c_axis1": B * (S + 2), "ns_c2r_axis1": B * (2 * S + 1), "ns_c2c_axis2": B * (3 * S + 3),
        "ns_c2c_axis3": B * 3, "ns_mask_axis3": B * 2 * S, "ns_accum_axis3": B * S,
    }.get(dom, 0)
    hbm, peak_kind = peaks()
    alg = tag_bytes.get(dom) or kernel_bytes(dom, None, dom_launches, nz_total)
    achieved = alg / (dom_ms / 1e3) / 1e9 if alg else None
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile) and DIMS == (128, 128, 128) and S == 49:   # the captured workload
        tj = json.load(open(tfile)).get(dom)
        if tj:
            traffic = tj.get("bytes_per_launch_full_size")
    op_bytes = 12.0 * (1 + S) * N * B * world     # 4(1+S)*3 B a voxel: 600 at S = 49
    line = {
        "metric": METRIC, "value": value, "unit": "Mvoxels/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"NSSurfacelet(scales={NS_KW['scales']}, direction_levels="
                               f"[{','.join(str(v) for v in NS_KW['direction_levels'])}]) "
                               + ("128^3" if DIMS == (128, 128, 128) else "x".join(str(d) for d in DIMS))
                               + " float32, analyze+synthesize+adjoint(synthesize) per volume",
                   "batch_per_gpu": B, "global_batch": B * world, "volume": list(DIMS),
                   "parallelism": f"replicas x{world} (no collective)",
                   "execution": ("one CUDA graph a step (sfl_batch_*): volume b on workspace b mod "
                                 f"{nws}, workspaces on concurrent branches" if args.mode == "graph"
                                 else "a loop of plain calls on one workspace"),
                   "kernel_times": "CUDA events around every launch, from a replay as plain calls",
                   "l2": "inputs larger than L2 (411 MB of coefficients a volume)"},
        "gpu_launches": launches_per_step * args.steps,
        "rel_err": {"perfect_reconstruction_rel_l2": rel_pr, "adjoint_vs_analyze_rel_l2": rel_adj,
                    "vs_fp64_oracle": vs_oracle},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                     "peak_kind": peak_kind,
                     "launches_per_step": dom_launches, "ms_per_step": dom_ms,
                     "share_of_kernel_time": dom_ms / sum(v[0] for v in per_tag.values())},
        "op_roofline": {"algorithmic_bytes_per_voxel": 12 * (1 + S), "achieved_gbs": op_bytes / (ms / 1e3) / 1e9 / world,
                        "frac": op_bytes / (ms / 1e3) / 1e9 / world / hbm, "peak_kind": peak_kind},
        "kernel_ms_per_step": {k: v[0] for k, v in per_tag.items()},
        "kernel_algorithmic_gbs": {k: tag_bytes[k] / (v[0] / 1e3) / 1e9 for k, v in per_tag.items()
                                   if tag_bytes.get(k)},
    }
    # The co-limit: FP32 arithmetic on the CUDA cores.  The FLOPs a voxel are
    # measured (ncu thread-instruction counts FADD + FMUL + 2 FFMA over every
    # launch of one step, profiles/fp32_flops.json) on the default workload;
    # the peak is cuBLAS SGEMM (TF32 off) measured here, with the nominal FMA
    # rate at the sampled SM clock beside it.
    mhz = clk["sm_mhz"] if clk else 1965.0
    ffile = os.path.join(ROOT, "profiles", "fp32_flops.json")
    if os.path.exists(ffile) and DIMS == (128, 128, 128) and S == 49:
        flop_vox, flop_kind = json.load(open(ffile))["flop_per_voxel_step"], "measured (ncu, one step)"
    else:
        flop_vox, flop_kind = 3.0 * (1 + S) * 2.5 * np.log2(N), "estimate: 2.5 N log2 N a real 3-D FFT, unpruned"
    fp32_ach = flop_vox * N * B / (ms / 1e3) / 1e12
    line["fp32_roofline"] = {"bound": "fp32", "flop_per_voxel": flop_vox, "flop_kind": flop_kind,
                             "achieved": fp32_ach, "peak": sgemm_tflops(), "unit": "TFLOP/s",
                             "frac": fp32_ach / sgemm_tflops(), "peak_kind": "measured: cuBLAS SGEMM 8192^3, TF32 off",
                             "nominal_fma_peak": 148 * 128 * 2 * mhz * 1e6 / 1e12}
    if clk:
        line["clocks"] = {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"]}

    # e2e: public API with pinned host buffers, copies inside the timed region
    hx = [torch.empty(DIMS[::-1], dtype=torch.float32).pin_memory() for _ in range(B)]
    hy = [torch.empty(DIMS[::-1], dtype=torch.float32).pin_memory() for _ in range(B)]
    for b in range(B):
        hx[b].copy_(xs[b].permute(2, 1, 0))

    if args.mode == "graph":
        # the host copies inside the graph, on each volume's branch: H2D, the three
        # transforms, D2H of the synthesized volume
        ents = []
        for b in range(B):
            w = wss[b % nws]
            ents += [(w, "copy_volume", hx[b], xs[b]), (w, "analyze", xs[b], cs[b]), (w, "synthesize", cs[b], ys[b]),
                     (w, "adjoint_synthesize", ys[b], gs[b]), (w, "copy_volume", ys[b], hy[b])]
        ebatch = sfl.Batch([e[0] for e in ents], [e[2] for e in ents], [e[3] for e in ents], [e[1] for e in ents])

        def e2e_step():
            ebatch.run()
    else:
        def e2e_step():
            for b in range(B):
                xs[b].permute(2, 1, 0).copy_(hx[b], non_blocking=True)
            step()
            for b in range(B):
                hy[b].copy_(ys[b].permute(2, 1, 0), non_blocking=True)

    e2e_step()
    ms_e2e = timed(e2e_step, max(3, args.steps // 2))
    line["e2e"] = {"value": B * N * world / (ms_e2e / 1e3) / 1e6, "unit": "Mvoxels/s",
                   "h2d_bytes_per_step": 4 * N * B, "d2h_bytes_per_step": 4 * N * B,
                   "scope": "volume in, volume out: each step copies every input volume from pinned host memory "
                            "and every synthesized volume back; the coefficients (analyze's output and the "
                            "adjoint's) stay on the device"}

    if not args.no_extras and rank == 0:
        # plain unfused single-volume GPU form: the reference's device path
        # (materialized masks, one cuFFT call per subband) through torch.fft
        sys.path.insert(0, ROOT)
        from oracle import ns as ON
        T = ON.make_tables(ON.NSParams.make(**NS_KW), DIMS)
        masks = [(s, torch.from_numpy(M.astype(np.float32).transpose().copy()).cuda())
                 for s, M in ON.subband_masks(T, analysis=True)]
        xt = xs[0].permute(2, 1, 0)       # C-order (n3, n2, n1): the rfft axis is last

        def plain_step():
            X = torch.fft.rfftn(xt)
            cpl = [None] * S
            for s, M in masks:
                cpl[s - 1] = torch.fft.irfftn(X * M, s=xt.shape)
            acc = None
            for s, M in masks:
                F = torch.fft.rfftn(cpl[s - 1]) * M
                acc = F if acc is None else acc + F
            y = torch.fft.irfftn(acc, s=xt.shape)
            X2 = torch.fft.rfftn(y)
            for s, M in masks:
                torch.fft.irfftn(X2 * M, s=xt.shape)

        for _ in range(2):
            plain_step()
        ms_plain = timed(plain_step, 3)
        plain = N / (ms_plain / 1e3) / 1e6
        line["plain_gpu"] = {"value": plain, "unit": "Mvoxels/s",
                             "form": "torch.fft (cuFFT) + materialized masks, one volume, unfused",
                             "fused_over_plain_per_volume": (value / world) / plain}
        del masks
        torch.cuda.empty_cache()

        # secondary line: the decimated Surfacelet at 128^3 (pyramid_ratio 2): plain calls on one
        # workspace, and the same batch as one graph over four workspaces
        u = sfl.Surfacelet(**DEC_KW)
        wds = [sfl.make_workspace(u, "float32", DIMS) for _ in range(min(4, B))]
        wd = wds[0]
        cds = [torch.empty(wd.ncoeffs, device="cuda") for _ in range(B)]
        yds = [sfl.volume_like(DIMS) for _ in range(B)]

        def dec_step():
            for b in range(B):
                sfl.analyze_(cds[b], wd, xs[b])
                sfl.synthesize_(yds[b], wd, cds[b])

        dents = []
        for b in range(B):
            w = wds[b % len(wds)]
            dents += [(w, "analyze", xs[b], cds[b]), (w, "synthesize", cds[b], yds[b])]
        dbatch = sfl.Batch([e[0] for e in dents], [e[2] for e in dents], [e[3] for e in dents], [e[1] for e in dents])
        for _ in range(3):
            dec_step()
        ms_dec = timed(dec_step, max(3, args.steps // 2))
        ms_decg = timed(dbatch.run, max(3, args.steps // 2))
        rel_dec = float(torch.linalg.vector_norm(yds[B - 1] - xs[B - 1]) / torch.linalg.vector_norm(xs[B - 1]))
        dbatch.close()
        line["secondary"] = {"workload": "Surfacelet(scales=3, direction_levels=[2,2,3], pyramid_ratio=2) "
                                         "128^3 float32, analyze+synthesize",
                             "value": B * N / (ms_decg / 1e3) / 1e6, "unit": "Mvoxels/s",
                             "execution": "one CUDA graph over 4 workspaces (as the headline)",
                             "plain_calls_value": B * N / (ms_dec / 1e3) / 1e6,
                             "perfect_reconstruction_rel_l2": rel_dec,
                             "algorithmic_bytes_per_voxel": 4 * 2 * (1 + wd.ncoeffs / N)}

        # downstream consumer: the fused soft-threshold denoiser against the three calls
        tau = 0.05
        yn = sfl.volume_like(DIMS)

        def den_step():
            for b in range(B):
                yn.copy_(sfl.denoise(ws, xs[b], tau))

        tt = torch.full((S,), tau, device="cuda")
        tt[0] = 0

        def three_step():
            for b in range(B):
                sfl.analyze_(cs[b], ws, xs[b])
                cs[b].copy_(torch.sign(cs[b]) * torch.clamp(cs[b].abs() - tt, min=0))
                sfl.synthesize_(ys[b], ws, cs[b])

        for _ in range(2):
            den_step()
            three_step()
        ms_den = timed(den_step, max(3, args.steps // 2))
        ms_three = timed(three_step, max(3, args.steps // 2))
        line["denoiser"] = {"workload": "soft threshold 0.05 of every directional subband, same NSSurfacelet "
                                        "128^3, one workspace, plain calls",
                            "fused_value": B * N / (ms_den / 1e3) / 1e6,
                            "three_calls_value": B * N / (ms_three / 1e3) / 1e6, "unit": "Mvoxels/s",
                            "equal_bit_for_bit": bool(torch.equal(yn, ys[B - 1]))}

        # batch workload: 64 volumes, axes from {64, 96, 128, 160}, scales from {2, 3, 4},
        # levels from {1, 2, 3}; analyze + synthesize + adjoint as one graph against a loop
        brng = np.random.default_rng(64)
        bws, bx, bc, by, nvox = [], [], [], [], 0
        t0 = time.perf_counter()
        for _ in range(64):
            d3 = tuple(int(v) for v in brng.choice([64, 96, 128, 160], 3))
            J = int(brng.choice([2, 3, 4]))
            w = sfl.make_workspace(sfl.NSSurfacelet(scales=J, direction_levels=[int(v) for v in brng.choice([1, 2, 3], J)]),
                                   "float32", d3)
            xv = sfl.volume_like(d3).copy_(torch.randn(d3, device="cuda"))
            w.autotune(xv)
            bws.append(w)
            bx.append(xv)
            bc.append(sfl.similar_coefficients(w.transform, xv))
            by.append(sfl.volume_like(d3))
            nvox += int(np.prod(d3))
        t_setup = time.perf_counter() - t0
        bents = []
        for w, xv, cv, yv in zip(bws, bx, bc, by):
            bents += [(w, "analyze", xv, cv), (w, "synthesize", cv, yv), (w, "adjoint_synthesize", yv, cv)]
        bb = sfl.Batch([e[0] for e in bents], [e[2] for e in bents], [e[3] for e in bents], [e[1] for e in bents])

        def loop_step():
            for w, xv, cv, yv in zip(bws, bx, bc, by):
                sfl.analyze_(cv, w, xv)
                sfl.synthesize_(yv, w, cv)
                sfl.adjoint_synthesize_(cv, w, yv)

        loop_step()
        ms_graph = timed(bb.run, 3)
        ms_loop = timed(loop_step, 3)
        line["batch64"] = {"workload": "64 NSSurfacelet volumes, axes from {64,96,128,160}, scales from {2,3,4}, "
                                       "levels from {1,2,3} (seed 64), analyze+synthesize+adjoint, autotuned plans",
                           "graph_value": nvox / (ms_graph / 1e3) / 1e6, "loop_value": nvox / (ms_loop / 1e3) / 1e6,
                           "unit": "Mvoxels/s", "voxels": nvox, "setup_s": t_setup}
        bb.close()
        del bb, bws, bx, bc, by
        torch.cuda.empty_cache()

        # large streaming workload: NSSurfacelet(scales=4, [2,2,3,3]) at 256^3, one subband at a
        # time (analysis -> soft threshold -> synthesis, the adjoint by per-subband recompute),
        # and the bfloat16 coefficient format against float32
        L3 = (256, 256, 256)
        tl = sfl.NSSurfacelet(scales=4, direction_levels=[2, 2, 3, 3])
        wa, wsy = sfl.make_workspace(tl, "float32", L3), sfl.make_workspace(tl, "float32", L3)
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from phantoms import ellipsoid_phantom
        xl_host = ellipsoid_phantom(L3, count=24, seed=5)
        xl = sfl.to_device(xl_host)
        yl = sfl.volume_like(L3)
        # the soft threshold sign(b) max(|b| - 0.05, 0) as one torch kernel (softshrink: the same values)
        shrink = lambda i, b: sfl.as_colmajor(torch.nn.functional.softshrink(b, 0.05))
        sfl.analyze_synthesize_stream(lambda i, b: b, yl, xl, wa, wsy)
        pr32 = float(torch.linalg.vector_norm(yl - xl) / torch.linalg.vector_norm(xl))
        sfl.analyze_synthesize_stream(shrink, yl, xl, wa, wsy)   # warm-up of the thresholding callback
        ms_stream = timed(lambda: sfl.analyze_synthesize_stream(shrink, yl, xl, wa, wsy), 2)
        c32 = sfl.analyze(wa, xl)
        c16, sc16 = sfl.analyze_bf16(wa, xl)
        ce = sfl.as_colmajor(c16.float() * sc16)
        rel16 = float(torch.linalg.vector_norm(ce - c32) / torch.linalg.vector_norm(c32))
        y16 = sfl.synthesize_bf16(wsy, c16, sc16)
        pr16 = float(torch.linalg.vector_norm(y16 - xl) / torch.linalg.vector_norm(xl))
        # both coefficient formats against the float64 oracle, streamed subband by subband
        ON.set_fft_workers(os.cpu_count() or 1)
        Tl = ON.make_tables(ON.NSParams.make(scales=4, direction_levels=[2, 2, 3, 3]), L3)
        e32 = e16 = r2 = 0.0
        for s_, band in ON.analyze_stream(Tl, xl_host.astype(np.float64)):
            e32 += float(np.sum((host64(c32[..., s_ - 1]) - band) ** 2))
            e16 += float(np.sum((host64(ce[..., s_ - 1]) - band) ** 2))
            r2 += float(np.sum(band ** 2))
        ON.set_fft_workers(1)
        line["large_stream"] = {"workload": "NSSurfacelet(scales=4, direction_levels=[2,2,3,3]) 256^3 float32, S = 73, "
                                            "analysis -> soft threshold -> synthesis one subband at a time",
                                "value": float(np.prod(L3)) / (ms_stream / 1e3) / 1e6, "unit": "Mvoxels/s",
                                "input": "ellipsoid phantom: 24 seeded ellipsoids + N(0, 0.05^2)",
                                "fp32_coefficients_rel_l2_vs_fp64_oracle": float(np.sqrt(e32 / r2)),
                                "bf16_coefficients_rel_l2_vs_fp64_oracle": float(np.sqrt(e16 / r2)),
                                "fp32_reconstruction_rel_l2": pr32,
                                "bf16_coefficients_rel_l2_vs_fp32": rel16,
                                "bf16_reconstruction_rel_l2": pr16,
                                "coefficient_bytes": {"fp32": c32.numel() * 4, "bf16": c16.numel() * 2 + 4 * 73}}
        del c32, c16, ce, y16, wa, wsy, xl, yl
        torch.cuda.empty_cache()

        # CPU baseline: the oracle port on the host cores, bounded sample
        from oracle.cpu_baseline import NSBaseline
        cores = os.cpu_count()
        base = NSBaseline(ON.NSParams.make(**NS_KW), DIMS, np.float32, workers=cores)
        xh = xs[0].permute(2, 1, 0).cpu().numpy().transpose()
        reps = 2
        t0 = time.perf_counter()
        for _ in range(reps):
            cb = base.analyze(xh)
            yb = base.synthesize(cb)
            base.analyze(yb, synth_masks=True)
        dt = (time.perf_counter() - t0) / reps
        line["cpu_baseline"] = {"value": N / dt / 1e6, "unit": "Mvoxels/s", "cores": cores, "kind": "port",
                                "sample": f"{reps} x (analyze+synthesize+adjoint) of one 128^3 volume, "
                                          f"scipy.fft workers={cores}, float32"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
