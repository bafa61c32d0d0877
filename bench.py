#!/usr/bin/env python
"""Benchmark of the SIFT matching path on B200.

Default workload (one step): batched all-pairs matching of 200 synthetic images (1000..12000
uint8 SIFT-like features each, 15% shared tracks): all 19,900 pairs in one call, minScore 0.7,
ratio 0.8.  Metric: image pairs per second.  `value` times the steps with descriptors resident
in HBM (the device-output C-ABI call, replayed as a CUDA graph); `e2e` times the same step
through the host C-ABI calls (pinned host descriptors in, host (pair, left, right) triples out,
copies inside the timed region).
Other workloads (--workload): pair (one 4096 x 4096 pair, putative), stereo (one 16384 x 16384
pair, putative + F-guided), voctree (2M descriptors through a BF 10, depth 6 tree), proposal
(learned candidate proposal against exhaustive matching), float (float descriptors, BF16 hi/lo
path), batch-float (the all-pairs workload with float descriptors), batch-guided (the all-pairs
workload as guided calls), ingest (feature files to device descriptors), retrieval (the voctree
app's image-retrieval scoring of a 4096-image sequence) and ransac (batched essential-matrix
RANSAC).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload ...]

Under torchrun each rank runs an independent replica on its own GPU (pairs are independent; the
path shards with no exchange), timed on the device, max over ranks.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for p in (str(ROOT / "eth-v3d-lgpl_b200"), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)

MIN_SCORE, MIN_RATIO, GATE_PX = 0.7, 0.8, 2.0
N_SIDE = 16384
L2_FLUSH_BYTES = 512 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["batch", "batch-float", "pair", "stereo", "voctree", "proposal", "float",
                                           "ingest", "retrieval", "ransac", "batch-guided"],
                    default="batch")
    ap.add_argument("--kernel", choices=["tcgen05", "simt"], default="tcgen05")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--tile-config", type=int, default=-1, help="fused-kernel tile configuration (-1: autotune)")
    ap.add_argument("--images", type=int, default=200, help="batch workload: number of images")
    ap.add_argument("--cache-dir", default="", help="voctree workload: keep the generated tree and queries here")
    ap.add_argument("--float-tree", action="store_true",
                    help="voctree workload: a float k-means tree of unit-L2 descriptors and float queries (the "
                         "apps' trees), quantised in the reference CPU tree's sequential FP32 order")
    ap.add_argument("--cells", type=int, default=128, help="proposal workload: cells of the projection")
    ap.add_argument("--probes", type=int, default=4, help="proposal workload: probed cells per left")
    ap.add_argument("--probes-right", type=int, default=4, help="proposal workload: cells each right is listed under")
    ap.add_argument("--proposal-config", type=int, default=0, help="proposal workload: tile configuration")
    ap.add_argument("--proposal-schedule", type=int, default=2, help="proposal workload: row schedule")
    ap.add_argument("--prop-images", type=int, default=200, help="proposal workload: test images (8000 features)")
    ap.add_argument("--prop-train-images", type=int, default=100, help="proposal workload: held-out training images")
    ap.add_argument("--train-steps", type=int, default=600, help="proposal workload: Adam steps")
    ap.add_argument("--temperature", type=float, default=0.2, help="proposal workload: InfoNCE temperature")
    ap.add_argument("--rt-images", type=int, default=4096, help="retrieval workload: images in the sequence")
    ap.add_argument("--rs-pairs", type=int, default=256, help="ransac workload: image pairs per call")
    ap.add_argument("--refine", action="store_true",
                    help="ransac workload: the loop's iterative refinement (the apps' mode)")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------------
def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if os.environ.get("V3DM_BENCH_BACKEND", "nccl") == "nccl" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, x: float, device=None) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs"), "bf16_tflops": d.get("bf16_tflops"),
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained"), "src": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "src": "fallback"}


def sustained_fields(achieved: float, peaks: dict, scale: float) -> dict:
    """The same kernel against the sustained bf16 figure (a seconds-long GEMM loop under the power
    cap), for kernels timed inside long back-to-back steps; `frac` stays the burst fraction."""
    sus = peaks.get("bf16_tflops_sustained")
    if not sus:
        return {}
    return {"peak_sustained": scale * sus, "frac_sustained": achieved / (scale * sus)}


def traffic_from_profiles(kernel_tag: str):
    """Per-launch DRAM bytes of a kernel from its committed ncu summary, or None."""
    for f in sorted((ROOT / "profiles").glob(f"*{kernel_tag}*.md")):
        for line in f.read_text().splitlines():
            if line.strip().startswith("traffic_bytes_per_launch:"):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(gpu_index), "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
def cpu_stereo(L, R, lpos, rpos, F, threads: int = 0):
    """Oracle putative + F-guided matching of the whole pair from one score computation (the
    reference's guided call masks the putative call's stored matrix); returns seconds."""
    from oracle import oracle
    t0 = time.perf_counter()
    oracle.match_calls(L, R, MIN_SCORE, MIN_RATIO, [[], [("F", F, GATE_PX)]], lpos=lpos, rpos=rpos,
                       threads=threads)
    return time.perf_counter() - t0


def ref_gpu_key(desc, offs, pairs, reps, positions=None, F=None, what=""):
    """The reference's own CUDA matcher (v3d_cudamatching.cu built unmodified for sm_100a: cuBLAS
    SGEMM of the full score matrix, its maxima kernels, blocking copies) in the apps' per-pair
    loop on this GPU, wall time per repetition; None when that build is absent."""
    from oracle import oracle
    if not oracle.ref_cuda_available():
        return None
    try:
        r = oracle.ref_cuda_time_pairs(desc, offs, pairs, MIN_SCORE, MIN_RATIO, reps + 1, positions=positions,
                                       F=F, thr=GATE_PX)
    except Exception as e:  # the reference exits on CUDA errors; report instead of failing the arm
        return {"unavailable": f"reference matcher failed: {str(e)[-200:]}"}
    sec = r["seconds"][1:]  # the first repetition warms cuBLAS and the allocator
    t = statistics.mean(sec)
    n = len(pairs)
    return {"value": n / t, "unit": "pairs/s", "ms_per_step": 1000.0 * t, "reps": len(sec),
            "pairs_per_rep": n, "matches_found": r["matches"],
            "what": "the reference's CUDA SIFT_Matching (cublasSgemm + its maxima kernels, built unmodified for "
                    "sm_100a) on this GPU in the apps' loop: setLeft/RightFeatures from pageable host memory, "
                    "findPutativeMatches" + (", runGuidedMatching" if F is not None else "") +
                    " per pair; counts rounded down to multiples of 32 as the apps do; wall time " + what}


def run_reference_arm(args, ws, rank):
    if args.workload == "retrieval":
        return run_reference_retrieval(args, ws, rank)
    if args.workload == "ransac":
        return run_reference_ransac(args, ws, rank)
    if args.workload == "batch":
        return run_reference_batch(args, ws, rank)
    if args.workload == "pair":
        return run_reference_pair(args, ws, rank)
    if args.workload == "stereo":
        return run_reference_stereo(args, ws, rank)
    print(json.dumps({"impl": "reference", "unavailable": f"no reference arm for workload {args.workload}"}),
          flush=True)


def _reference_line(args, metric, v, ms, config, sample, dtype="u8"):
    from oracle import oracle
    return {
        "impl": "reference", "metric": metric, "value": v, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded generator)",
        "config": config,
        "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": oracle.num_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference_stereo(args, ws, rank):
    """The reference's path on the host cores: the oracle port (the reference has no CPU
    matcher of its own), all host threads, the whole 16384 x 16384 pair per step: one score
    computation, putative then F-guided decisions."""
    from v3dm import synth
    if rank != 0:
        return
    L, R, lpos, rpos, F, _ = synth.stereo(args.seed, N_SIDE, N_SIDE)
    for _ in range(args.warmup):
        cpu_stereo(L, R, lpos, rpos, F)
    times = [cpu_stereo(L, R, lpos, rpos, F) for _ in range(args.steps)]
    ms = 1000.0 * statistics.mean(times)
    line = _reference_line(args, "image pairs/s (16384x16384 putative + F-guided)", 1000.0 / ms, ms,
                           stereo_config(args, "cpu"),
                           "the whole pair per step (one score computation, putative and guided decisions)")
    off = np.array([0, N_SIDE, 2 * N_SIDE], np.int32)
    line["reference_gpu"] = ref_gpu_key(np.concatenate([L, R]), off, np.array([[0, 1]], np.int32), 5,
                                        positions=np.concatenate([lpos, rpos]), F=np.asarray(F).reshape(1, 9),
                                        what="of the pair's putative + guided calls")
    print(json.dumps(line), flush=True)


def stereo_config(args, where):
    return {"workload": "stereo pair 16384x16384 uint8 SIFT-like, putative + F-guided (2 px), "
                        "minScore 0.7, ratio 0.8", "n_left": N_SIDE, "n_right": N_SIDE, "seed": args.seed,
            "kernel": args.kernel if where == "gpu" else "oracle",
            "l2": "flushed between steps (512 MiB write on the matcher stream, outside the step events)",
            "work_per_step": "one full 16384 x 16384 contraction (the putative call's); the guided call reuses its "
                             "chunk records and applies the gates, as the reference's guided call masks the "
                             "putative call's stored score matrix" if where == "gpu" else
                             "putative and guided matching of the sample"}


def run_stereo(args, ws, rank, local):
    import torch

    import v3dm
    from v3dm import synth
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L, R, lpos, rpos, F, _ = synth.stereo(args.seed, N_SIDE, N_SIDE)
    kern = v3dm.KERNEL_TCGEN05 if args.kernel == "tcgen05" else v3dm.KERNEL_SIMT
    m = v3dm.SIFTMatching(local, kern)
    m.allocate(N_SIDE, N_SIDE, True)
    stream = torch.cuda.ExternalStream(m.stream(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    # ---------------- value: inputs resident in HBM ----------------
    m.set_left_features(L)
    m.set_right_features(R)
    d_lpos = torch.from_numpy(lpos).to(dev)
    d_rpos = torch.from_numpy(rpos).to(dev)
    d_pairs = torch.empty((N_SIDE, 2), dtype=torch.int32, device=dev)
    d_pairs2 = torch.empty((N_SIDE, 2), dtype=torch.int32, device=dev)
    d_cnt = torch.zeros(2, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()

    def step_device():
        n = 0
        m.putative_device(MIN_SCORE, MIN_RATIO, d_pairs.data_ptr(), d_cnt.data_ptr())
        n += m.last_launches()
        m.guided_F_device(F, GATE_PX, d_lpos.data_ptr(), d_rpos.data_ptr(), MIN_SCORE, MIN_RATIO,
                          d_pairs2.data_ptr(), d_cnt.data_ptr() + 4)
        n += m.last_launches()
        return n

    if args.tile_config < 0:
        tuned_cfg, tuned_ms = m.autotune(MIN_SCORE, MIN_RATIO, 3)
    else:
        m.set_config(args.tile_config)
    cfg_id, cfg_rows, cfg_cols = m.config()
    for _ in range(args.warmup + 3):
        step_device()
        try:
            m.wait()
        except v3dm.V3DMError as e:  # the candidate list grew: the next call repeats it
            if e.status != v3dm.ERR_CANDIDATES:
                raise
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches = 0
    m.profile(True)
    clocks = Clocks(local) if rank == 0 or True else None
    barrier(ws)
    torch.cuda.synchronize()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        ev[i][0].record(stream)
        launches += step_device()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop() if clocks else None
    m.wait()
    ms_steps = [a.elapsed_time(b) for a, b in ev]
    ms = max_over_ranks(ws, statistics.mean(ms_steps), dev)
    kms, kl = m.profile_read(0)
    kms_b, kl_b = m.profile_read(1)
    m.profile(False)
    k_avg_ms = max_over_ranks(ws, kms / max(kl, 1), dev)
    kb_avg_ms = max_over_ranks(ws, kms_b / max(kl_b, 1), dev)
    n_put = int(d_cnt[0].item())
    n_gui = int(d_cnt[1].item())

    # ---------------- e2e: host buffers through the C ABI ----------------
    Lp = torch.from_numpy(L).pin_memory().numpy()
    Rp = torch.from_numpy(R).pin_memory().numpy()
    lpp = torch.from_numpy(lpos).pin_memory().numpy()
    rpp = torch.from_numpy(rpos).pin_memory().numpy()

    def step_host():
        m.set_left_features(Lp)
        m.set_right_features(Rp)
        a = m.find_putative_matches(MIN_SCORE, MIN_RATIO)
        b = m.run_guided_matching(F, GATE_PX, lpp, rpp, MIN_SCORE, MIN_RATIO)
        return a.shape[0] + b.shape[0]

    for _ in range(args.warmup):
        step_host()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    npairs_out = 0
    barrier(ws)
    torch.cuda.synchronize()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        ev2[i][0].record(stream)
        npairs_out = step_host()
        ev2[i][1].record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    ms_e2e = max_over_ranks(ws, statistics.mean([a.elapsed_time(b) for a, b in ev2]), dev)
    h2d = L.nbytes + R.nbytes + lpos.nbytes + rpos.nbytes
    d2h = npairs_out * 8 + 2 * 16
    m.close()

    if rank != 0:
        return
    peaks = load_peaks()
    int8_peak = 2.0 * peaks["bf16_tflops"]  # kind::i8 runs at twice the kind::f16 rate
    ops_per_launch = 2.0 * N_SIDE * N_SIDE * 128
    achieved = ops_per_launch / (k_avg_ms * 1e-3) / 1e12
    traffic = traffic_from_profiles("k_side_stereo" if args.kernel == "tcgen05" else "k_match_simt")
    line = {
        "metric": "image pairs/s (16384x16384 putative + F-guided)", "value": ws * 1000.0 / ms, "unit": "pairs/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
        "config": stereo_config(args, "gpu"),
        "int8_tops_per_kernel": achieved,
        "tile": {"config": cfg_id, "left_rows": cfg_rows, "right_cols": cfg_cols,
                 "chosen_by": "autotune" if args.tile_config < 0 else "flag"},
        "pairs_found": {"putative": n_put, "guided": n_gui},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOPS(int8)",
                     "frac": achieved / int8_peak, "traffic": traffic,
                     "peak_src": f"2 x {peaks['src']} bf16 dense ({peaks['bf16_tflops']} TFLOP/s burst)",
                     "kernel_ms": k_avg_ms, "ops_per_launch": ops_per_launch,
                     "kernel": "k_side pass A (every left x every right)",
                     "pass_b_ms": kb_avg_ms},
        "e2e": {"value": ws * 1000.0 / ms_e2e, "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and ws == 1:
        from oracle import oracle
        dt = cpu_stereo(L, R, lpos, rpos, F)
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "pairs/s", "cores": oracle.num_threads(), "kind": "port",
                                "sample": "the whole pair once: one score computation, putative and guided "
                                          "decisions"}
    print(json.dumps(line), flush=True)


N_PAIR = 4096


def pair_config(args, where):
    return {"workload": "one pair 4096x4096 uint8 SIFT-like (30% planted noisy copies), putative, minScore 0.7, "
                        "ratio 0.8", "n_left": N_PAIR, "n_right": N_PAIR, "seed": args.seed,
            "kernel": args.kernel if where == "gpu" else "oracle",
            "l2": "flushed between steps (512 MiB write on the matcher stream, outside the step events)"}


def run_pair(args, ws, rank, local):
    """One 4096 x 4096 pair, putative matching: a step is one findPutativeMatches call."""
    import torch

    import v3dm
    from v3dm import synth
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L, R, _ = synth.pair(args.seed, N_PAIR, N_PAIR)
    kern = v3dm.KERNEL_TCGEN05 if args.kernel == "tcgen05" else v3dm.KERNEL_SIMT
    m = v3dm.SIFTMatching(local, kern)
    m.allocate(N_PAIR, N_PAIR)
    stream = torch.cuda.ExternalStream(m.stream(), device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    m.set_left_features(L)
    m.set_right_features(R)
    d_pairs = torch.empty((N_PAIR, 2), dtype=torch.int32, device=dev)
    d_cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    if args.tile_config < 0:
        m.autotune(MIN_SCORE, MIN_RATIO, 3)
    else:
        m.set_config(args.tile_config)
    cfg_id, cfg_rows, cfg_cols = m.config()
    for _ in range(max(args.warmup, 3)):
        m.putative_device(MIN_SCORE, MIN_RATIO, d_pairs.data_ptr(), d_cnt.data_ptr())
        try:
            m.wait()
        except v3dm.V3DMError as e:  # the candidate list grew: the next call repeats it
            if e.status != v3dm.ERR_CANDIDATES:
                raise
    steps = max(args.steps, 200)  # a 4096^2 call is tens of microseconds: enough steps for the clock sampler
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    launches = 0
    m.profile(True)
    clocks = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize()
    for i in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        ev[i][0].record(stream)
        m.putative_device(MIN_SCORE, MIN_RATIO, d_pairs.data_ptr(), d_cnt.data_ptr())
        launches += m.last_launches()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    m.wait()
    ms = max_over_ranks(ws, statistics.mean(a.elapsed_time(b) for a, b in ev), dev)
    kms, kl = m.profile_read(0)
    m.profile(False)
    k_avg_ms = max_over_ranks(ws, kms / max(kl, 1), dev)
    n_found = int(d_cnt[0].item())

    Lp = torch.from_numpy(L).pin_memory().numpy()
    Rp = torch.from_numpy(R).pin_memory().numpy()

    def step_host():
        m.set_left_features(Lp)
        m.set_right_features(Rp)
        return m.find_putative_matches(MIN_SCORE, MIN_RATIO).shape[0]

    for _ in range(max(args.warmup, 3)):
        step_host()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    n_host = 0
    barrier(ws)
    torch.cuda.synchronize()
    for i in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        ev2[i][0].record(stream)
        n_host = step_host()
        ev2[i][1].record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    ms_e2e = max_over_ranks(ws, statistics.mean(a.elapsed_time(b) for a, b in ev2), dev)
    m.close()
    if rank != 0:
        return
    peaks = load_peaks()
    int8_peak = 2.0 * peaks["bf16_tflops"]
    ops = 2.0 * N_PAIR * N_PAIR * 128
    achieved = ops / (k_avg_ms * 1e-3) / 1e12
    line = {
        "metric": "image pairs/s (4096x4096 putative)", "value": ws * 1000.0 / ms, "unit": "pairs/s",
        "n_gpus": ws, "steps": steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
        "config": pair_config(args, "gpu"),
        "tile": {"config": cfg_id, "left_rows": cfg_rows, "right_cols": cfg_cols,
                 "chosen_by": "autotune" if args.tile_config < 0 else "flag"},
        "pairs_found": n_found,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOPS(int8)",
                     "frac": achieved / int8_peak, "traffic": traffic_from_profiles("k_side_pair4096"),
                     "peak_src": f"2 x {peaks['src']} bf16 dense ({peaks['bf16_tflops']} TFLOP/s burst)",
                     "kernel_ms": k_avg_ms, "ops_per_launch": ops,
                     "kernel": "k_side pass A (every left x every right)"},
        "e2e": {"value": ws * 1000.0 / ms_e2e, "unit": "pairs/s", "h2d_bytes_per_step": int(L.nbytes + R.nbytes),
                "d2h_bytes_per_step": int(n_host * 8 + 16)},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and ws == 1:
        from oracle import oracle
        reps = 0
        t0 = time.perf_counter()
        while reps < 3 or time.perf_counter() - t0 < 5.0:
            oracle.match(L, R, MIN_SCORE, MIN_RATIO)
            reps += 1
        dt = (time.perf_counter() - t0) / reps
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": "pairs/s", "cores": oracle.num_threads(), "kind": "port",
                                "sample": f"the whole pair, {reps} times"}
    print(json.dumps(line), flush=True)


def run_reference_pair(args, ws, rank):
    """The reference's path on the host cores for the 4096 x 4096 pair: the oracle port, all host
    threads, the whole pair per step."""
    from oracle import oracle
    from v3dm import synth
    if rank != 0:
        return
    L, R, _ = synth.pair(args.seed, N_PAIR, N_PAIR)
    for _ in range(args.warmup):
        oracle.match(L, R, MIN_SCORE, MIN_RATIO)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.match(L, R, MIN_SCORE, MIN_RATIO)
        times.append(time.perf_counter() - t0)
    ms = 1000.0 * statistics.mean(times)
    line = _reference_line(args, "image pairs/s (4096x4096 putative)", 1000.0 / ms, ms, pair_config(args, "cpu"),
                           "the whole pair per step")
    off = np.array([0, N_PAIR, 2 * N_PAIR], np.int32)
    line["reference_gpu"] = ref_gpu_key(np.concatenate([L, R]), off, np.array([[0, 1]] * 20, np.int32), 5,
                                        what="of 20 putative calls on the pair")
    print(json.dumps(line), flush=True)


def run_batch(args, ws, rank, local):
    """All 19,900 pairs of 200 synthetic images (1000..12000 features, 15% shared tracks),
    minScore 0.7, ratio 0.8: one batched call per step (two persistent side-pass launches,
    replayed as a CUDA graph)."""
    import torch

    import v3dm
    from v3dm import synth
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    desc, counts, offs = synth.images(args.seed + 1, n_images=args.images)
    b = v3dm.BatchMatching(local)
    b.set_images(desc, counts)
    b.set_pairs(None)
    ops, n_pairs = b.work()
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    if args.tile_config < 0:
        cfg, sch, tune_ms = b.autotune(MIN_SCORE, MIN_RATIO, 1)
    else:
        b.set_config(args.tile_config, 0)
    cfg, sch = b.config()
    d_cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    for _ in range(max(args.warmup, 3)):
        b.match_device(MIN_SCORE, MIN_RATIO, d_cnt.data_ptr())
        while b.wait() == v3dm.ERR_CANDIDATES:  # buffers grown: repeat
            b.match_device(MIN_SCORE, MIN_RATIO, d_cnt.data_ptr())
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches = 0
    clocks = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize()
    for i in range(args.steps):
        ev[i][0].record(stream)
        b.match_device(MIN_SCORE, MIN_RATIO, d_cnt.data_ptr())
        ev[i][1].record(stream)
        launches += b.last_launches()
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    assert b.wait() == v3dm.OK
    ms = max_over_ranks(ws, statistics.mean(a.elapsed_time(c) for a, c in ev), dev)
    n_out = int(d_cnt.item())
    # pass timing with events (a separate run without the graph)
    b.profile(True)
    for _ in range(3):
        b.match_device(MIN_SCORE, MIN_RATIO, d_cnt.data_ptr())
        assert b.wait() == v3dm.OK
    ka, na = b.profile_read(0)
    kb, nb = b.profile_read(1)
    b.profile(False)
    # e2e: images from pinned host memory, triples back to the host
    desc_p = torch.from_numpy(desc).pin_memory().numpy()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for _ in range(2):
        b.set_images(desc_p, counts)
        b.match(MIN_SCORE, MIN_RATIO)
    barrier(ws)
    torch.cuda.synchronize()
    n_host = 0
    for i in range(args.steps):
        ev2[i][0].record(stream)
        b.set_images(desc_p, counts)
        n_host = b.match(MIN_SCORE, MIN_RATIO).shape[0]
        ev2[i][1].record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    ms_e2e = max_over_ranks(ws, statistics.mean(a.elapsed_time(c) for a, c in ev2), dev)
    b.close()
    if rank != 0:
        return
    peaks = load_peaks()
    int8_peak = 2.0 * peaks["bf16_tflops"]
    k_ms = ka / max(na, 1)
    achieved = ops / (k_ms * 1e-3) / 1e12
    line = {
        "metric": f"image pairs/s (all {n_pairs} pairs of {args.images} images)", "value": ws * n_pairs * 1000.0 / ms,
        "unit": "pairs/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generator)",
        "config": batch_config(args, n_pairs, int(counts.sum()), desc.nbytes),
        "aggregate_int8_tops": ops / (ms * 1e-3) / 1e12,
        "tile": {"config": cfg, "schedule": sch, "chosen_by": "autotune" if args.tile_config < 0 else "flag"},
        "pairs_found": n_out,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOPS(int8)",
                     "frac": achieved / int8_peak, "traffic": traffic_from_profiles("k_side_batch"),
                     "peak_src": f"2 x {peaks['src']} bf16 dense ({peaks['bf16_tflops']} TFLOP/s burst)",
                     "kernel_ms": k_ms, "ops_per_launch": ops, "kernel": "k_side pass A (every pair)",
                     "pass_b_ms": kb / max(nb, 1), **sustained_fields(achieved, peaks, 2.0)},
        "e2e": {"value": ws * n_pairs * 1000.0 / ms_e2e, "unit": "pairs/s",
                "h2d_bytes_per_step": int(desc.nbytes), "d2h_bytes_per_step": int(n_host * 12 + 48)},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and ws == 1:
        from oracle import oracle
        n_s, dt = cpu_batch_sample(desc, counts, offs, BATCH_CPU_SAMPLE, 0)
        line["cpu_baseline"] = {"value": n_s / dt, "unit": "pairs/s", "cores": oracle.num_threads(), "kind": "port",
                                "sample": f"{n_s} pairs drawn uniformly from the {n_pairs} (seed 0), each matched "
                                          f"in full ({dt:.1f} s); value = pairs / time, not extrapolated"}
    print(json.dumps(line), flush=True)


def run_batch_float(args, ws, rank, local):
    """The all-pairs workload's images with float descriptors that are not u/512 (u / 512 with
    N(0, 0.004^2) noise, renormalised): one batched call per step on the BF16 hi/lo layouts (K =
    384 BF16 products per score), replayed as a CUDA graph; each pair's result is the single-pair
    float matcher's."""
    import torch

    import v3dm
    from v3dm import synth
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    desc8, counts, offs = synth.images(args.seed + 1, n_images=args.images)
    desc = synth.float_from_u8(desc8, args.seed + 1)
    del desc8
    b = v3dm.BatchMatching(local)
    b.set_images(desc, counts)
    assert b.float_mode
    b.set_pairs(None)
    ops, n_pairs = b.work()
    flops = 3 * ops  # three BF16 products per score (2 * 128 * nL * nR each)
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    d_cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    for _ in range(max(args.warmup, 3)):
        b.match_device(MIN_SCORE, MIN_RATIO, d_cnt.data_ptr())
        while b.wait() == v3dm.ERR_CANDIDATES:
            b.match_device(MIN_SCORE, MIN_RATIO, d_cnt.data_ptr())
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches = 0
    clocks = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize()
    for i in range(args.steps):
        ev[i][0].record(stream)
        b.match_device(MIN_SCORE, MIN_RATIO, d_cnt.data_ptr())
        ev[i][1].record(stream)
        launches += b.last_launches()
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    assert b.wait() == v3dm.OK
    ms = max_over_ranks(ws, statistics.mean(a.elapsed_time(c) for a, c in ev), dev)
    n_out = int(d_cnt.item())
    b.profile(True)
    for _ in range(2):
        b.match_device(MIN_SCORE, MIN_RATIO, d_cnt.data_ptr())
        assert b.wait() == v3dm.OK
    ka, na = b.profile_read(0)
    kb, nb = b.profile_read(1)
    b.profile(False)
    # e2e: float images from pinned host memory, triples back to the host
    desc_p = torch.from_numpy(desc).pin_memory().numpy()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    b.set_images(desc_p, counts)
    b.match(MIN_SCORE, MIN_RATIO)
    barrier(ws)
    torch.cuda.synchronize()
    n_host = 0
    for i in range(args.steps):
        ev2[i][0].record(stream)
        b.set_images(desc_p, counts)
        n_host = b.match(MIN_SCORE, MIN_RATIO).shape[0]
        ev2[i][1].record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    ms_e2e = max_over_ranks(ws, statistics.mean(a.elapsed_time(c) for a, c in ev2), dev)
    b.close()
    if rank != 0:
        return
    peaks = load_peaks()
    k_ms = ka / max(na, 1)
    achieved = flops / (k_ms * 1e-3) / 1e12
    line = {
        "metric": f"image pairs/s (all {n_pairs} pairs of {args.images} images, float descriptors)",
        "value": ws * n_pairs * 1000.0 / ms, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16x3/f32", "data": "synthetic (seeded generator)",
        "config": {"workload": f"{args.images} images, 1000..12000 SIFT-like float descriptors each (u/512 + "
                               f"N(0, 0.004^2), renormalised; not u/512), 15% shared tracks, all {n_pairs} pairs, "
                               f"minScore 0.7, ratio 0.8", "pairs": n_pairs, "descriptors": int(counts.sum()),
                   "seed": args.seed + 1,
                   "l2": f"inputs larger than L2 ({2 * desc.nbytes * 3 // 2 / 1e6:.0f} MB of BF16 hi/lo layouts)"},
        "pairs_found": n_out,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s(bf16)",
                     "frac": achieved / peaks["bf16_tflops"], "traffic": traffic_from_profiles("batch_float_side"),
                     "peak_src": f"{peaks['src']} bf16 dense burst", "kernel_ms": k_ms, "flops_per_launch": flops,
                     "kernel": "k_side_f<true> pass A (every pair, K = 384 BF16)", "pass_b_ms": kb / max(nb, 1),
                     **sustained_fields(achieved, peaks, 1.0)},
        "e2e": {"value": ws * n_pairs * 1000.0 / ms_e2e, "unit": "pairs/s", "h2d_bytes_per_step": int(desc.nbytes),
                "d2h_bytes_per_step": int(n_host * 12 + 48)},
        "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_batch_guided(args, ws, rank, local):
    """All pairs of a scene with geometry (args.images cameras along a line, 1000..12000 features
    per image, 15% shared tracks observed at their projections with 1 px noise): one guided call
    per step, i.e. every pair's findPutativeMatches and then its runGuidedMatching with the pair's
    fundamental matrix and a 2 px epipolar gate, minScore 0.7, ratio 0.8 -- the apps' per-pair
    putative -> guided sequence for a batch.  The step is the host call: the gates go up, the
    triples come back."""
    import torch

    import v3dm
    from v3dm import synth
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    desc, counts, offs, pos, cams = synth.scene(args.seed + 6, args.images, 1000, 12000, track_frac=0.15)
    pairs = synth.all_pairs(args.images)
    F = np.stack([synth.fundamental(cams, i, j) for i, j in pairs])
    thr = 2.0
    b = v3dm.BatchMatching(local)
    b.set_images(desc, counts)
    b.set_pairs(None)
    b.set_positions(pos)
    ops, n_pairs = b.work()
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    if args.tile_config < 0:
        b.autotune(MIN_SCORE, MIN_RATIO, 1)
    else:
        b.set_config(args.tile_config, 0)
    cfg, sch = b.config()
    for _ in range(max(args.warmup, 3)):
        b.match_guided(F, thr, MIN_SCORE, MIN_RATIO)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches = 0
    n_out = 0
    clocks = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize()
    for i in range(args.steps):
        ev[i][0].record(stream)
        n_out = b.match_guided(F, thr, MIN_SCORE, MIN_RATIO).shape[0]
        ev[i][1].record(stream)
        launches += b.last_launches()
    torch.cuda.synchronize()
    barrier(ws)
    clk = clocks.stop()
    ms = max_over_ranks(ws, statistics.mean(a.elapsed_time(c) for a, c in ev), dev)
    b.profile(True)
    for _ in range(3):
        b.match_guided(F, thr, MIN_SCORE, MIN_RATIO)
    ka, na = b.profile_read(0)
    kb, nb = b.profile_read(1)
    b.profile(False)
    # e2e: images and positions from pinned host memory, then the guided call
    desc_p = torch.from_numpy(desc).pin_memory().numpy()
    pos_p = torch.from_numpy(pos).pin_memory().numpy()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(ws)
    torch.cuda.synchronize()
    for i in range(args.steps):
        ev2[i][0].record(stream)
        b.set_images(desc_p, counts)
        b.set_positions(pos_p)
        b.match_guided(F, thr, MIN_SCORE, MIN_RATIO)
        ev2[i][1].record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    ms_e2e = max_over_ranks(ws, statistics.mean(a.elapsed_time(c) for a, c in ev2), dev)
    b.close()
    if rank != 0:
        return
    peaks = load_peaks()
    int8_peak = 2.0 * peaks["bf16_tflops"]
    k_ms = ka / max(na, 1)
    achieved = ops / (k_ms * 1e-3) / 1e12
    line = {
        "metric": f"image pairs/s, guided (all {n_pairs} pairs of {args.images} images)",
        "value": ws * n_pairs * 1000.0 / ms, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic (seeded generator with cameras)",
        "config": {"workload": f"{args.images} images with cameras along a line, 1000..12000 uint8 SIFT-like "
                               f"features each, 15% shared tracks at their projections (1 px noise), all {n_pairs} "
                               f"pairs, putative then guided with each pair's F, 2 px gate, minScore 0.7, ratio 0.8",
                   "pairs": n_pairs, "descriptors": int(counts.sum()), "seed": args.seed + 6,
                   "l2": "inputs larger than L2 (descriptors, positions and the per-pair state)"},
        "tile": {"config": cfg, "schedule": sch},
        "pairs_found": n_out,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOPS(int8)",
                     "frac": achieved / int8_peak, "traffic": None,
                     "peak_src": f"2 x {peaks['src']} bf16 dense ({peaks['bf16_tflops']} TFLOP/s burst)",
                     "kernel_ms": k_ms, "ops_per_launch": ops, "kernel": "k_side pass A (every pair)",
                     "pass_b_ms": kb / max(nb, 1)},
        "e2e": {"value": ws * n_pairs * 1000.0 / ms_e2e, "unit": "pairs/s",
                "h2d_bytes_per_step": int(desc.nbytes + pos.nbytes + F.size * 8 + n_pairs * 4),
                "d2h_bytes_per_step": int(n_out * 12 + 48)},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and ws == 1:
        from oracle import oracle
        sample = batch_sample(args.images, BATCH_CPU_SAMPLE, 0)
        index = {(int(i), int(j)): k for k, (i, j) in enumerate(pairs)}
        t0 = time.perf_counter()
        for i, j in sample:
            oracle.match(desc[offs[i]:offs[i + 1]], desc[offs[j]:offs[j + 1]], MIN_SCORE, MIN_RATIO,
                         gates=[("F", F[index[(int(i), int(j))]], thr)], lpos=pos[offs[i]:offs[i + 1]],
                         rpos=pos[offs[j]:offs[j + 1]])
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": len(sample) / dt, "unit": "pairs/s", "cores": oracle.num_threads(),
                                "kind": "port",
                                "sample": f"{len(sample)} pairs drawn uniformly from the {n_pairs} (seed 0), each "
                                          f"scored once and gated ({dt:.1f} s); value = pairs / time"}
    print(json.dumps(line), flush=True)


BATCH_CPU_SAMPLE = 150   # pairs in the cpu_baseline leg (about 10 s of oracle work on 16 threads)
BATCH_REF_STEP = 16      # pairs per step of the reference arm
BATCH_REF_GPU = 400      # pairs per repetition of the reference's CUDA matcher


def batch_config(args, n_pairs, n_desc, l2_bytes):
    return {"workload": f"{args.images} images, 1000..12000 uint8 SIFT-like features each, 15% shared "
                        f"tracks, all {n_pairs} pairs, minScore 0.7, ratio 0.8", "pairs": n_pairs,
            "descriptors": n_desc, "seed": args.seed + 1,
            "l2": f"inputs larger than L2 ({l2_bytes / 1e6:.0f} MB of descriptors and the per-pair state)"}


def batch_sample(n_images, k, seed):
    from v3dm import synth
    pairs = synth.all_pairs(n_images)
    rng = np.random.default_rng(seed)
    return pairs[rng.choice(len(pairs), min(k, len(pairs)), replace=False)]


def cpu_batch_sample(desc, counts, offs, k, seed, threads: int = 0):
    """The oracle on k pairs drawn uniformly from all pairs, each matched in full; returns
    (pairs matched, seconds)."""
    from oracle import oracle
    sample = batch_sample(len(counts), k, seed)
    t0 = time.perf_counter()
    for i, j in sample:
        oracle.match(desc[offs[i]:offs[i + 1]], desc[offs[j]:offs[j + 1]], MIN_SCORE, MIN_RATIO, threads=threads)
    return len(sample), time.perf_counter() - t0


def run_reference_batch(args, ws, rank):
    """The reference's path on the host cores for the all-pairs workload: the oracle port, all
    host threads; each step matches BATCH_REF_STEP pairs drawn uniformly from the 19,900 (a new
    draw per step), each in full.  value = pairs matched / time (a sample, not extrapolated)."""
    from v3dm import synth
    if rank != 0:
        return
    desc, counts, offs = synth.images(args.seed + 1, n_images=args.images)
    n_pairs = args.images * (args.images - 1) // 2
    for w in range(args.warmup):
        cpu_batch_sample(desc, counts, offs, 2, 1000 + w)
    times, done = [], 0
    for k in range(args.steps):
        n, dt = cpu_batch_sample(desc, counts, offs, BATCH_REF_STEP, 1 + k)
        times.append(dt)
        done += n
    ms = 1000.0 * statistics.mean(times)
    line = _reference_line(args, f"image pairs/s (all {n_pairs} pairs of {args.images} images)",
                           done / sum(times), ms, batch_config(args, n_pairs, int(counts.sum()), desc.nbytes),
                           f"{BATCH_REF_STEP} pairs per step drawn uniformly from the {n_pairs} (a new draw per "
                           "step), each matched in full; value = pairs / time, not extrapolated")
    sample = batch_sample(len(counts), BATCH_REF_GPU, 0)
    line["reference_gpu"] = ref_gpu_key(desc, offs, sample, 3,
                                        what=f"of {len(sample)} pairs drawn uniformly from the {n_pairs} (seed 0)")
    print(json.dumps(line), flush=True)


def run_voctree(args, ws, rank, local):
    """Vocabulary-tree quantization: BF 10, depth 6 (1,111,110 nodes without the root, HKM
    centres from 500k descriptors), 2,000,000 query descriptors.  Per-level figures come from
    the same kernel on the depth-d prefix trees (breadth-first order makes the first d levels a
    tree of depth d)."""
    import torch

    import v3dm
    from v3dm import synth
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    bf, depth, n = 10, 6, 2_000_000
    fl = args.float_tree
    tag = "f32_" if fl else ""
    cache = Path(args.cache_dir) / f"voctree_{tag}{args.seed + 2}.npz" if args.cache_dir else None
    if cache is not None and cache.exists():
        d = np.load(cache)
        nodes, keys = d["nodes"], d["keys"]
    else:
        nodes, keys = synth.voctree(args.seed + 2, bf, depth, 500_000, n, floats=fl)
        if cache is not None:
            cache.parent.mkdir(parents=True, exist_ok=True)
            np.savez(cache, nodes=nodes, keys=keys)
    t = v3dm.VocabularyTreeTraversal(bf, depth, local)
    t.allocate(n)
    t.set_nodes(nodes)
    stream = torch.cuda.ExternalStream(t.stream(), device=dev)
    d_keys = torch.from_numpy(keys).to(dev)
    d_ids = torch.empty(n, dtype=torch.int32, device=dev)

    def quantize(tree):
        if fl:
            tree.quantize_f32_device(n, d_keys.data_ptr(), d_ids.data_ptr())
        else:
            tree.quantize_device(n, d_keys.data_ptr(), d_ids.data_ptr())

    def timed(tree, steps):
        s = torch.cuda.ExternalStream(tree.stream(), device=dev)
        for _ in range(max(args.warmup, 3)):
            quantize(tree)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize()
        for a, c in evs:
            a.record(s)
            quantize(tree)
            c.record(s)
        torch.cuda.synchronize()
        return statistics.mean(a.elapsed_time(c) for a, c in evs)

    torch.cuda.synchronize()
    barrier(ws)
    clocks = Clocks(local)
    ms = max_over_ranks(ws, timed(t, args.steps), dev)
    clk = clocks.stop()
    launches_per_call = t.last_launches()
    ids = d_ids.cpu().numpy()
    # per level: the same kernel on the depth-d prefix trees
    level_ms, prev = [], 0.0
    for d in range(1, depth + 1):
        if d == depth:
            td = ms
        else:
            tr = v3dm.VocabularyTreeTraversal(bf, d, local)
            tr.allocate(n)
            tr.set_nodes(nodes[: v3dm.voctree_counts(bf, d)[0]])
            td = timed(tr, args.steps)
            tr.close()
        level_ms.append(td - prev)
        prev = td
    # e2e: keys from pinned host memory, ids back to the host
    kp = torch.from_numpy(keys).pin_memory().numpy()
    for _ in range(2):
        t.traverse_tree(kp)
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for a, c in ev2:
        a.record(stream)
        t.traverse_tree(kp)
        c.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(ws, statistics.mean(a.elapsed_time(c) for a, c in ev2), dev)
    t_replays = t.replays()
    t.close()
    if rank != 0:
        return
    peaks = load_peaks()
    esz = 4 if fl else 1
    replays = t_replays if fl else None
    node_bytes = nodes.shape[0] * 128 * esz
    alg_bytes = n * 128 * esz + n * 4 + node_bytes
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    level_bytes = n * bf * 128 * esz
    line = {
        "metric": "descriptors/s (vocabulary-tree quantization, BF 10, depth 6)", "value": ws * n * 1000.0 / ms,
        "unit": "desc/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32" if fl else "u8",
        "data": "synthetic (seeded generator)",
        "config": {"workload": "voctree BF 10 depth 6 (1,111,110 HKM nodes from 500k descriptors), 2,000,000 "
                               + ("unit-L2 float queries, float k-means centres (the reference CPU tree's sequential "
                                  "FP32 order)" if fl else "uint8 SIFT-like queries"), "seed": args.seed + 2,
                   "l2": "inputs larger than L2 (%d MB of keys, %d MB of nodes)" % (n * 128 * esz // 10**6,
                                                                                  node_bytes // 10**6)},
        "sequential_replays": replays,
        "per_level": [{"level": d + 1, "ms": level_ms[d], "gathered_GBps": level_bytes / (level_ms[d] * 1e-3) / 1e9
                       if level_ms[d] > 0 else None} for d in range(depth)],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"],
                     "traffic": traffic_from_profiles("k_voctree_f32" if fl else "k_vtc"),
                     "peak_src": f"{peaks['src']} copy bandwidth",
                     "bytes_per_launch": alg_bytes,
                     "kernel": "k_voctree_f32 (all levels, one launch)" if fl else
                               "k_vtc x 3 (two levels per phase, tcgen05) + k_vt_scan + k_vt_scatter (one call)"},
        "e2e": {"value": ws * n * 1000.0 / ms_e2e, "unit": "desc/s", "h2d_bytes_per_step": int(keys.nbytes),
                "d2h_bytes_per_step": int(n * 4)},
        "gpu_launches": args.steps * launches_per_call,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and ws == 1:
        from oracle import oracle
        sample = 200_000
        kf = keys[:sample].astype(np.float32) if fl else keys[:sample].astype(np.float32) / 512
        nf = nodes.astype(np.float32) if fl else nodes.astype(np.float32) / 512
        if oracle.ref_voctree_available():
            t0 = time.perf_counter()
            ref = oracle.ref_voctree(bf, depth, nf, kf)
            dt = time.perf_counter() - t0
            kind = "reference"
            line["parity_sample"] = bool(np.array_equal(ref + sum(bf ** k for k in range(1, depth)),
                                                        ids[:sample]))
        else:
            t0 = time.perf_counter()
            oracle.voctree(bf, depth, nodes, keys[:sample], True)
            dt = time.perf_counter() - t0
            kind = "port"
        line["cpu_baseline"] = {"value": sample / dt, "unit": "desc/s", "cores": oracle.num_threads(), "kind": kind,
                                "sample": f"first {sample} of the 2,000,000 queries"}
    print(json.dumps(line), flush=True)


def run_proposal(args, ws, rank, local):
    """Learned candidate proposal against exhaustive matching on the same GPU: 200 test images
    x 8000 features (19,900 pairs), the projection trained on matches that exhaustive matching
    found in 100 held-out images of the same generator."""
    import torch

    import v3dm
    from v3dm import proposal, synth
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n_tr, n_te = args.prop_train_images, args.prop_images
    tr_desc, tr_counts, tr_offs = synth.images(args.seed + 40, n_images=n_tr, n_min=8000, n_max=8000)
    te_desc, te_counts, te_offs, te_track = synth.images(args.seed + 41, n_images=n_te, n_min=8000, n_max=8000,
                                                         tracks=True)
    b = v3dm.BatchMatching(local)
    b.set_images(tr_desc, tr_counts)
    b.set_pairs(None)
    t_tr = time.perf_counter()
    anchors, positives = proposal.mine_pairs(tr_desc, tr_offs, synth.all_pairs(n_tr), b.match(MIN_SCORE, MIN_RATIO))
    net = v3dm.Projection(local, seed=args.seed)
    losses = proposal.train(net, anchors, positives, steps=args.train_steps, batch=2048,
                            temperature=args.temperature, lr=2e-3, device=local)
    net.set_cells(proposal.fit_cells(net.embed(tr_desc), args.cells, seed=args.seed))
    train_s = time.perf_counter() - t_tr
    b.set_images(te_desc, te_counts)
    b.set_pairs(None)
    ops, n_pairs = b.work()
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    d_cnt = torch.zeros(1, dtype=torch.int32, device=dev)

    def timed(call):
        for _ in range(max(args.warmup, 3)):
            call()
            while b.wait() == v3dm.ERR_CANDIDATES:
                call()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        torch.cuda.synchronize()
        n = 0
        for a0, a1 in ev:
            a0.record(stream)
            call()
            a1.record(stream)
            n += b.last_launches()
        torch.cuda.synchronize()
        assert b.wait() == v3dm.OK
        return max_over_ranks(ws, statistics.mean(x.elapsed_time(y) for x, y in ev), dev), n

    if args.tile_config < 0:
        b.autotune(MIN_SCORE, MIN_RATIO, 1)  # exhaustive at its fastest configuration
    else:
        b.set_config(args.tile_config, 0)
    exh_cfg = b.config()
    ms_exh, _ = timed(lambda: b.match_device(MIN_SCORE, MIN_RATIO, d_cnt.data_ptr()))
    exh = b.match(MIN_SCORE, MIN_RATIO)
    b.set_config(args.proposal_config, args.proposal_schedule)
    clocks = Clocks(local)
    torch.cuda.nvtx.range_push("proposal")  # profilers can select the proposal launches by this range
    ms_prop, launches = timed(lambda: b.match_proposal_device(net, args.probes, MIN_SCORE, MIN_RATIO, d_cnt.data_ptr(), args.probes_right))
    torch.cuda.nvtx.range_pop()
    clk = clocks.stop()
    got = b.match_proposal(net, args.probes, MIN_SCORE, MIN_RATIO, probes_right=args.probes_right)
    rec, prec = proposal.recall(exh, got)
    # recall of the exhaustive matches that join two views of one track (the rest are chance
    # matches between unrelated descriptors, which no candidate proposal can find)
    pairs_all = synth.all_pairs(n_te)
    inl = synth.inlier_mask(exh, pairs_all, te_offs, te_track)
    rec_in, _ = proposal.recall(exh[inl], got)
    scored, exhaustive = b.proposal_scored()
    b.profile(True)
    for _ in range(3):
        b.match_proposal_device(net, args.probes, MIN_SCORE, MIN_RATIO, d_cnt.data_ptr(), args.probes_right)
        assert b.wait() == v3dm.OK
    ka, na = b.profile_read(0)
    kv, nv = b.profile_read(1)
    b.profile(False)
    # ablation: the same cells fitted to the untrained network
    net0 = v3dm.Projection(local, seed=args.seed)
    net0.set_cells(proposal.fit_cells(net0.embed(tr_desc), args.cells, seed=args.seed))
    ms0, _ = timed(lambda: b.match_proposal_device(net0, args.probes, MIN_SCORE, MIN_RATIO, d_cnt.data_ptr(), args.probes_right))
    got0 = b.match_proposal(net0, args.probes, MIN_SCORE, MIN_RATIO, probes_right=args.probes_right)
    rec0, prec0 = proposal.recall(exh, got0)
    rec0_in, _ = proposal.recall(exh[inl], got0)
    scored0, _ = b.proposal_scored()
    net0.close()
    # e2e: descriptors from pinned host memory, triples back
    desc_p = torch.from_numpy(te_desc).pin_memory().numpy()
    for _ in range(2):
        b.set_images(desc_p, te_counts)
        b.match_proposal(net, args.probes, MIN_SCORE, MIN_RATIO, probes_right=args.probes_right)
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    n_host = 0
    for a0, a1 in ev2:
        a0.record(stream)
        b.set_images(desc_p, te_counts)
        n_host = b.match_proposal(net, args.probes, MIN_SCORE, MIN_RATIO, probes_right=args.probes_right).shape[0]
        a1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(ws, statistics.mean(x.elapsed_time(y) for x, y in ev2), dev)
    net.close()
    b.close()
    if rank != 0:
        return
    peaks = load_peaks()
    int8_peak = 2.0 * peaks["bf16_tflops"]
    k_ms = ka / max(na, 1)
    ops_prop = 2.0 * 128 * scored
    achieved = ops_prop / (k_ms * 1e-3) / 1e12
    line = {
        "metric": f"image pairs/s (learned proposal, all {n_pairs:,} pairs of {n_te} images x 8000 features)",
        "value": ws * n_pairs * 1000.0 / ms_prop, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_prop, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator)",
        "config": {"workload": f"{n_te} test images x 8000 uint8 SIFT-like features, 15% shared tracks, all {n_pairs:,} pairs, "
                               f"minScore 0.7, ratio 0.8; projection 128-64-32 trained on {n_tr} held-out images",
                   "cells": args.cells, "probes": args.probes, "probes_right": args.probes_right,
                   "tile_config": args.proposal_config, "row_schedule": args.proposal_schedule,
                   "exhaustive_tile_config": list(exh_cfg),
                   "train_steps": args.train_steps,
                   "temperature": args.temperature, "train_pairs": int(anchors.shape[0]),
                   "l2": f"inputs {'larger' if te_desc.nbytes > 126e6 else 'smaller'} than L2 "
                         f"({te_desc.nbytes / 1e6:.0f} MB of descriptors)"},
        "exhaustive": {"value": ws * n_pairs * 1000.0 / ms_exh, "unit": "pairs/s", "ms_per_step": ms_exh},
        "speedup_vs_exhaustive": ms_exh / ms_prop,
        "recall": rec, "precision": prec, "recall_inliers": rec_in,
        "matches_exhaustive": int(len(exh)), "inliers_exhaustive": int(inl.sum()), "matches_proposal": int(len(got)),
        "scored_fraction": scored / exhaustive,
        "verification_ms": kv / max(nv, 1),
        "ablation_untrained": {"recall": rec0, "precision": prec0, "recall_inliers": rec0_in,
                               "scored_fraction": scored0 / exhaustive,
                               "ms_per_step": ms0},
        "training": {"seconds": train_s, "loss_first": losses[0][1], "loss_last": losses[-1][1]},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOPS(int8)",
                     "frac": achieved / int8_peak, "traffic": None,
                     "peak_src": f"2 x {peaks['src']} bf16 dense ({peaks['bf16_tflops']} TFLOP/s burst)",
                     "kernel_ms": k_ms, "ops_per_launch": ops_prop,
                     "kernel": "k_side pass A over the candidate blocks (scored pairs x 256 ops)"},
        "e2e": {"value": ws * n_pairs * 1000.0 / ms_e2e, "unit": "pairs/s", "h2d_bytes_per_step": int(te_desc.nbytes),
                "d2h_bytes_per_step": int(n_host * 12 + 64)},
        "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def float_pair(seed, n):
    """16384 x 16384 unit-length SIFT-like float descriptors (not u/512), 30% noisy planted copies."""
    rng = np.random.default_rng(seed)

    def make(k):
        x = rng.gamma(0.6, 1.0, size=(k, 128))
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        np.minimum(x, 0.2, out=x)
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        return x

    L = make(n)
    n_p = int(0.3 * n)
    cp = np.abs(L[rng.integers(0, n, n_p)] + rng.normal(0, 0.015, (n_p, 128)))
    cp /= np.linalg.norm(cp, axis=1, keepdims=True)
    R = np.concatenate([cp, make(n - n_p)])[rng.permutation(n)]
    return L.astype(np.float32), R.astype(np.float32)


def run_float(args, ws, rank, local):
    """Float descriptors (not u/512) through the BF16 hi/lo path: putative matching of one
    16384 x 16384 pair per step; the score error against float64 on a 1024 x 16384 block."""
    import torch

    import v3dm
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    L, R = float_pair(args.seed, N_SIDE)
    m = v3dm.SIFTMatching(local, v3dm.KERNEL_TCGEN05)
    m.allocate(N_SIDE, N_SIDE)
    m.set_left_features(L)
    m.set_right_features(R)
    stream = torch.cuda.ExternalStream(m.stream(), device=dev)
    d_pairs = torch.empty((N_SIDE, 2), dtype=torch.int32, device=dev)
    d_cnt = torch.zeros(2, dtype=torch.int32, device=dev)
    for _ in range(max(args.warmup, 3) + 4):
        m.putative_device(MIN_SCORE, MIN_RATIO, d_pairs.data_ptr(), d_cnt.data_ptr())
        try:
            m.wait()
        except v3dm.V3DMError as e:  # the candidate list grew: the call is repeated
            if e.status != v3dm.ERR_CANDIDATES:
                raise
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = Clocks(local)
    torch.cuda.synchronize()
    launches = 0
    m.profile(True)
    for a0, a1 in ev:
        a0.record(stream)
        m.putative_device(MIN_SCORE, MIN_RATIO, d_pairs.data_ptr(), d_cnt.data_ptr())
        a1.record(stream)
        launches += m.last_launches()
    torch.cuda.synchronize()
    clk = clocks.stop()
    m.wait()
    kms, kl = m.profile_read(0)
    m.profile(False)
    ms = max_over_ranks(ws, statistics.mean(x.elapsed_time(y) for x, y in ev), dev)
    n_pairs = int(d_cnt[0].item())
    # e2e: float descriptors from pinned host memory
    Lp = torch.from_numpy(L).pin_memory().numpy()
    Rp = torch.from_numpy(R).pin_memory().numpy()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for a0, a1 in ev2:
        a0.record(stream)
        m.set_left_features(Lp)
        m.set_right_features(Rp)
        got = m.find_putative_matches(MIN_SCORE, MIN_RATIO)
        a1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(ws, statistics.mean(x.elapsed_time(y) for x, y in ev2), dev)
    # score error on a block
    m2 = v3dm.SIFTMatching(local, v3dm.KERNEL_TCGEN05)
    m2.allocate(1024, N_SIDE)
    m2.set_left_features(L[:1024])
    m2.set_right_features(R)
    S = m2.scores_f32().astype(np.float64)
    S64 = L[:1024].astype(np.float64) @ R.astype(np.float64).T
    err = np.abs(S - S64)
    m2.close()
    m.close()
    if rank != 0:
        return
    peaks = load_peaks()
    k_ms = kms / max(kl, 1)
    flops = 3 * 2.0 * 128 * N_SIDE * N_SIDE  # three BF16 products per score
    achieved = flops / (k_ms * 1e-3) / 1e12
    line = {
        "metric": "image pairs/s (16384x16384 float descriptors, putative, BF16 hi/lo scores)",
        "value": ws * 1000.0 / ms, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3/f32",
        "data": "synthetic (seeded generator)",
        "config": {"workload": "16384 x 16384 unit-length SIFT-like float descriptors (not u/512), putative, "
                               "minScore 0.7, ratio 0.8", "l2": "flush not needed: inputs are re-read from L2 "
                                                                 "by design (16 MB of operands)"},
        "pairs_found": n_pairs,
        "score_error_vs_fp64": {"max_abs": float(err.max()), "mean_abs": float(err.mean()),
                                "sample": "1024 x 16384 scores"},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s(bf16)",
                     "frac": achieved / peaks["bf16_tflops"], "traffic": traffic_from_profiles("k_side_f"),
                     "peak_src": f"{peaks['src']} bf16 dense burst", "kernel_ms": k_ms,
                     "flops_per_launch": flops, "kernel": "k_side_f row walk, pass A (K = 384 BF16)"},
        "e2e": {"value": ws * 1000.0 / ms_e2e, "unit": "pairs/s", "h2d_bytes_per_step": int(L.nbytes + R.nbytes),
                "d2h_bytes_per_step": int(got.shape[0] * 8 + 16)},
        "gpu_launches": launches,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_ingest(args, ws, rank, local):
    """Feature-file ingestion: 200 binary feature archives (the reference's .features format) of
    8000 SIFT-like features each, read into device-resident u8 descriptors ready for the batched
    matcher (v3dm_loader_load: host threads parse the files into pinned memory, one copy to the
    device, u8 re-quantisation there).  The files are written once (to --cache-dir when given,
    else a temporary directory) and read from the page cache."""
    import tempfile

    import torch

    import v3dm
    from v3dm import synth
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n_img, n_feat = args.images, 8000
    root = Path(args.cache_dir) / f"features_{args.seed}_{n_img}" if args.cache_dir else \
        Path(tempfile.mkdtemp(prefix="v3dm_features_"))
    root.mkdir(parents=True, exist_ok=True)
    desc, counts, offs = synth.images(args.seed + 50, n_images=n_img, n_min=n_feat, n_max=n_feat)
    rng = np.random.default_rng(args.seed)
    paths = []
    for i in range(n_img):
        p = root / f"view{i:04d}.features"
        if not p.exists():
            synth.write_features(p, synth.feature_arrays(rng, int(counts[i]), desc[offs[i]:offs[i + 1]]))
        paths.append(str(p))
    file_bytes = sum(os.path.getsize(p) for p in paths)
    ld = v3dm.Loader(local)
    for p in paths:  # page cache
        with open(p, "rb") as fh:
            while fh.read(1 << 24):
                pass
    for _ in range(max(args.warmup, 3)):
        kept = ld.load(paths)
    total = int(kept.sum())
    assert total == n_img * n_feat
    # the loaded descriptors are the images' u8 descriptors
    d_ptr, nt = ld.descriptors_device()
    check = torch.empty(nt * 128, dtype=torch.uint8, device=dev)
    src = torch.as_tensor(type("V", (), {"__cuda_array_interface__": {
        "shape": (nt * 128,), "typestr": "|u1", "data": (d_ptr, False), "version": 3}})(), device=dev)
    check.copy_(src)
    assert np.array_equal(check.cpu().numpy().reshape(nt, 128), desc)
    # each step: every file from the page cache to device-resident u8 descriptors; the events are
    # recorded on the device around the (blocking) call
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize()
    for a0, a1 in evs:
        a0.record()
        ld.load(paths)
        a1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(ws, statistics.mean(a.elapsed_time(c) for a, c in evs), dev)
    # the device kernel on its own: u8 re-quantisation of the same number of floats
    x = torch.rand(total * 128, device=dev)
    q = torch.empty(total * 128, dtype=torch.uint8, device=dev)
    for _ in range(3):
        v3dm.quantize_u8_device(x.data_ptr(), x.numel(), q.data_ptr(), 0)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(10)]
    for a0, a1 in kev:
        a0.record()
        v3dm.quantize_u8_device(x.data_ptr(), x.numel(), q.data_ptr(), 0)
        a1.record()
    torch.cuda.synchronize()
    k_ms = statistics.mean(a.elapsed_time(c) for a, c in kev)
    ld.close()
    if rank != 0:
        return
    peaks = load_peaks()
    k_bytes = total * 128 * 5  # 4-byte float in, 1-byte code out
    k_gbs = k_bytes / (k_ms * 1e-3) / 1e9
    line = {
        "metric": f"features/s ingested ({n_img} binary feature files x {n_feat} features to device u8)",
        "value": ws * total * 1000.0 / ms, "unit": "features/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32->u8", "data": "synthetic (seeded generator), written in the reference's "
                                                       "binary archive format",
        "config": {"workload": f"{n_img} .features files x {n_feat} SIFT features (540 B each, "
                               f"{file_bytes / 1e6:.0f} MB), page-cached, to device-resident u8",
                   "files": n_img, "features_per_file": n_feat, "file_bytes": file_bytes,
                   "host_threads": os.cpu_count(), "l2": "not applicable: each step streams the files once"},
        "roofline": {"bound": "hbm", "achieved": k_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": k_gbs / peaks["hbm_gbs"], "traffic": None,
                     "peak_src": f"{peaks['src']} copy bandwidth", "kernel_ms": k_ms, "bytes_per_launch": k_bytes,
                     "kernel": "k_quantize_u8 (5 bytes per value)"},
        "e2e": {"value": ws * total * 1000.0 / ms, "unit": "features/s", "h2d_bytes_per_step": total * 128 * 4,
                "d2h_bytes_per_step": 0},
        "gpu_launches": args.steps,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and ws == 1:
        from oracle import oracle
        if oracle.ref_features_available():
            sample = paths[:20]
            t0 = time.perf_counter()
            nref = sum(oracle.ref_features_count(p) for p in sample)
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": nref / dt, "unit": "features/s", "cores": 1, "kind": "reference",
                                    "sample": f"{len(sample)} of the {n_img} files read with the reference's "
                                              "serializeDataFromFile, one thread (as the apps read them)"}
    print(json.dumps(line), flush=True)


RT_LEAVES, RT_BEST, RT_PMATCH = 125_000, 20, 0.1  # VocabularyTree<3, 50, 128>; the app's defaults


def retrieval_config(n_img, n_words):
    return {"workload": f"retrieval scoring of a {n_img}-image sequence ({n_words} visual words, 2000..6000 per "
                        f"image), {RT_LEAVES}-leaf vocabulary (VocabularyTree<3,50,128>), "
                        f"POTENTIAL_VIEWS_COUNT {RT_BEST}, VISUAL_WORD_MATCH_PROPABILITY {RT_PMATCH}",
            "images": n_img, "words": n_words, "leaves": RT_LEAVES, "n_best": RT_BEST, "p_match": RT_PMATCH,
            "l2": "flushed between steps (512 MiB write)"}


def retrieval_words(args, n_img):
    from v3dm import synth
    return synth.sequence_words(args.seed + 3, n_images=n_img, n_leaves=RT_LEAVES)


def ref_retrieval_sample(off, w, stride, phase):
    """One pass of the reference's loop (every image inserted, every stride-th image queried);
    returns (estimated seconds of the whole loop, seconds run, queries)."""
    from oracle import oracle
    n_img = off.shape[0] - 1
    t0 = time.perf_counter()
    tq, ti, nq, _ = oracle.ref_retrieval_sampled(RT_LEAVES, off, w, RT_PMATCH, RT_BEST, stride, phase)
    return ti + tq * n_img / max(nq, 1), time.perf_counter() - t0, nq


def run_reference_retrieval(args, ws, rank):
    """The reference's own LeafDocuments loop (match_using_voctree.cpp:176-222, compiled from the
    reference into oracle/_ref), one thread as the app runs it.  A step is one pass with every
    image inserted and every 512th image queried (phase varied per step); the whole loop's time
    is the insertions plus the sampled queries scaled to all images."""
    from oracle import oracle
    if rank != 0:
        return
    if not oracle.ref_retrieval_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libv3dref_retrieval.so not built"}))
        return
    off, w = retrieval_words(args, args.rt_images)
    stride = 512
    small = off[:min(args.rt_images, 512) + 1]
    for k in range(args.warmup):  # warm-up on the first 512 images
        ref_retrieval_sample(small, w[:small[-1]], stride, 0)
    est = []
    for k in range(args.steps):
        est.append(ref_retrieval_sample(off, w, stride, (k * 37) % stride)[0])
    ms = 1000.0 * statistics.mean(est)
    v = args.rt_images * 1000.0 / ms
    sample = (f"each step one pass of the loop over all {args.rt_images} images (all inserted) with every "
              f"{stride}th image queried; whole-loop time = insertions + sampled queries x {stride}")
    line = {
        "impl": "reference", "metric": "images/s retrieval-scored (voctree binomial scores + nBest selection)",
        "value": v, "unit": "images/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded visual-word sequence)", "config": retrieval_config(args.rt_images, int(off[-1])),
        "cpu_baseline": {"value": v, "unit": "images/s", "cores": 1, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_retrieval(args, ws, rank, local):
    """Retrieval scoring of one image sequence per GPU (independent replicas): the voctree app's
    loop of computeBinomialScores + insertDocument over 4096 images with 2000..6000 visual words
    each, in one call.  value: words, offsets and outputs in device memory
    (v3dm_retrieval_binomial_device); e2e: host words from pinned memory in, host results out
    (v3dm_retrieval_binomial)."""
    import torch

    import v3dm
    from oracle import oracle
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n_img = args.rt_images
    off, w = retrieval_words(args, n_img)
    r = v3dm.Retrieval(local)
    stream = torch.cuda.ExternalStream(r.stream(), device=dev)
    dw = torch.from_numpy(w).to(dev)
    docs = torch.empty((n_img, RT_BEST), dtype=torch.int32, device=dev)
    sc = torch.empty((n_img, RT_BEST), dtype=torch.float32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()

    def step_device():
        r.binomial_device(RT_LEAVES, off, dw.data_ptr(), RT_PMATCH, RT_BEST, docs.data_ptr(), sc.data_ptr())

    for _ in range(max(args.warmup, 3)):
        step_device()
    r.wait()
    # the whole result against the oracle (bit-exact docs and scores)
    exp_docs, exp_sc = oracle.retrieval(RT_LEAVES, off, w, RT_PMATCH, RT_BEST)
    assert np.array_equal(docs.cpu().numpy(), exp_docs)
    assert np.array_equal(sc.cpu().numpy().view(np.uint32), exp_sc.view(np.uint32))
    recall = float(np.mean([np.isin([i - 1, i - 2], exp_docs[i]).mean() for i in range(2, n_img)]))
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize()
    for a0, a1 in evs:
        with torch.cuda.stream(stream):
            flush.fill_(1)
        a0.record(stream)
        step_device()
        a1.record(stream)
    r.wait()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(ws, statistics.mean(a.elapsed_time(b) for a, b in evs), dev)
    # kernel times (a separate pass with per-kernel events)
    r.profile(True)
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        step_device()
    r.wait()
    k_ms, k_n = r.profile_read(1)
    p_ms, p_n = r.profile_read(0)
    r.profile(False)
    k_ms /= max(k_n, 1)
    p_ms /= max(p_n, 1)

    # e2e: pinned host words in, host results out, through the host C-ABI call
    wp = torch.from_numpy(w).pin_memory().numpy()
    for _ in range(max(args.warmup, 3)):
        r.binomial(RT_LEAVES, off, wp, RT_PMATCH, RT_BEST)
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(ws)
    torch.cuda.synchronize()
    for a0, a1 in ev2:
        with torch.cuda.stream(stream):
            flush.fill_(1)
        a0.record(stream)
        hd, hs = r.binomial(RT_LEAVES, off, wp, RT_PMATCH, RT_BEST)
        a1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(ws, statistics.mean(a.elapsed_time(b) for a, b in ev2), dev)
    assert np.array_equal(hd, exp_docs)
    r.close()
    if rank != 0:
        return
    peaks = load_peaks()
    # algorithmic bytes of k_rt_score: per query image i, its words (4 B each), the first
    # ceil(i / 32) 32-bit words of the bitmap row of each of its words, its offsets / logarithms
    # (40 B per earlier image) and its outputs (8 B per kept image)
    cnt = np.diff(off).astype(np.int64)
    nw = (np.arange(n_img, dtype=np.int64) + 31) // 32
    k_bytes = int(4 * cnt.sum() + 4 * (cnt * nw).sum() + 40 * (np.arange(n_img, dtype=np.int64)).sum()
                  + 8 * n_img * RT_BEST)
    achieved = k_bytes / (k_ms * 1e-3) / 1e9
    line = {
        "metric": "images/s retrieval-scored (voctree binomial scores + nBest selection)",
        "value": ws * n_img * 1000.0 / ms, "unit": "images/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded visual-word sequence)", "config": retrieval_config(n_img, int(off[-1])),
        "neighbour_recall": recall,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic_from_profiles("k_rt_score"),
                     "peak_src": f"{peaks['src']} copy bandwidth", "kernel_ms": k_ms, "bytes_per_launch": k_bytes,
                     "kernel": "k_rt_score (bitmap rows of every query word; the bitmap stays in L2)",
                     "bitmap_kernel_ms": p_ms},
        "e2e": {"value": ws * n_img * 1000.0 / ms_e2e, "unit": "images/s",
                "h2d_bytes_per_step": int(w.nbytes + off.nbytes + 32 * n_img),
                "d2h_bytes_per_step": int(n_img * RT_BEST * 8)},
        "gpu_launches": 2 * args.steps,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and ws == 1 and oracle.ref_retrieval_available():
        est, ran, nq = ref_retrieval_sample(off, w, 256, 0)
        line["cpu_baseline"] = {"value": n_img / est, "unit": "images/s", "cores": 1, "kind": "reference",
                                "sample": f"the reference's loop over all {n_img} images (all inserted), {nq} "
                                          f"queried (every 256th); whole-loop time = insertions + sampled "
                                          f"queries x 256 ({ran:.1f} s run)"}
    print(json.dumps(line), flush=True)


RS_THR, RS_SAMPLES = 2.0, 1000  # inlier threshold (pixels), nSamples of the apps (match_sequence.cpp:261)
# double operations of one truncated Sampson evaluation: F p and F^T q (5 x 4), the residual (4),
# its square (1), the denominator (7), the division (1), the truncation and the sum (2)
RS_FLOPS_PER_EVAL = 35
FP64_NOMINAL_TFLOPS = 37.0


def ransac_data(args, n_pairs):
    from v3dm import synth
    return synth.two_view_pairs(args.seed + 7, n_pairs=n_pairs, n_min=500, n_max=3000)


def ransac_config(n_pairs, n_corrs, refine=False):
    return {"workload": f"essential-matrix RANSAC of {n_pairs} image pairs ({n_corrs} putative correspondences, "
                        f"500..3000 per pair, 30..80% inliers), nSamples {RS_SAMPLES}, threshold {RS_THR} px, "
                        + ("iterative refinement of each accepted pose (the apps' mode)" if refine
                           else "no iterative refinement"),
            "pairs": n_pairs, "correspondences": n_corrs, "n_samples": RS_SAMPLES, "threshold_px": RS_THR,
            "iterative_refinement": refine, "l2": "flushed between steps (512 MiB write)"}


def ref_ransac_pairs(off, corrs, K, pairs, refine=False):
    """The reference loop (its five-point solver and pose recovery, the loop restated) on the given
    pairs with the app's own sample sequence; returns seconds."""
    from oracle import oracle
    t = 0.0
    for p in pairs:
        c = corrs[off[p]:off[p + 1]]
        smp = oracle.ref_shuffle_samples(c.shape[0], RS_SAMPLES, 1000 + p)  # the reference's own draws
        t0 = time.perf_counter()
        oracle.ref_ransac(c, K[p, 0], K[p, 1], RS_THR, RS_SAMPLES, smp, refine=refine)
        t += time.perf_counter() - t0
    return t


def run_reference_ransac(args, ws, rank):
    """The reference's relative orientation (computeEssentialsFromFiveCorrs and
    relativePoseFromEssential compiled from the reference into oracle/_ref, in the loop of
    computeRobustOrientationMLE restated, one pair at a time as the apps run it, one thread) on the
    same pairs; each step is a sample of 8 pairs."""
    from oracle import oracle
    if rank != 0:
        return
    if not oracle.ref_ransac_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libv3dref_ransac.so not built"}))
        return
    n_pairs = args.rs_pairs
    off, corrs, K, _, _, _ = ransac_data(args, n_pairs)
    k = min(8, n_pairs)
    for w in range(args.warmup):
        ref_ransac_pairs(off, corrs, K, [(w * 37) % n_pairs], args.refine)
    per_pair = []
    for st in range(args.steps):
        sel = [(st * k + j) * 29 % n_pairs for j in range(k)]
        per_pair.append(ref_ransac_pairs(off, corrs, K, sel, args.refine) / k)
    ms = 1000.0 * statistics.mean(per_pair) * n_pairs
    v = n_pairs * 1000.0 / ms
    line = {
        "impl": "reference", "metric": "image pairs/s robust relative orientation (5-point RANSAC, Sampson costs)",
        "value": v, "unit": "pairs/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded two-view correspondences)", "config": ransac_config(n_pairs, int(off[-1]), args.refine),
        "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": 1, "kind": "reference",
                         "sample": f"{k} of the {n_pairs} pairs per step with the app's own sample sequence; "
                                   "whole-call time = mean per pair x pairs"},
        "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ransac(args, ws, rank, local):
    """Essential-matrix RANSAC of 256 image pairs per GPU in one call (independent replicas):
    every pair's 1001 samples (nSamples + 1, drawn on the device), their five-point solutions,
    the truncated Sampson cost of every solution over the pair's correspondences, and the apps'
    sequential choice with the adaptive sample budget.  value: correspondences, outputs in device
    memory (v3dm_ransac_essential_device); e2e: host correspondences from pinned memory in, models
    and inlier flags out (v3dm_ransac_essential)."""
    import torch

    import v3dm
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n_pairs = args.rs_pairs
    off, corrs, K, R, t, inl = ransac_data(args, n_pairs)
    n_corrs = int(off[-1])
    n_draw = RS_SAMPLES + 1
    r = v3dm.Ransac(local)
    r.set_refinement(args.refine)
    stream = torch.cuda.ExternalStream(r.stream(), device=dev)
    dc = torch.from_numpy(corrs).to(dev)
    dm = torch.empty((n_pairs, 31), dtype=torch.float64, device=dev)
    dn = torch.empty(n_pairs, dtype=torch.int32, device=dev)
    df = torch.empty(n_corrs, dtype=torch.uint8, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()

    def step_device():
        r.essential_device(off, dc.data_ptr(), K, RS_THR, RS_SAMPLES, n_draw, None, args.seed, dm.data_ptr(),
                           dn.data_ptr(), df.data_ptr())

    for _ in range(max(args.warmup, 3)):
        step_device()
    r.wait()
    # quality of the result against the generator's poses
    Rg = dm.cpu().numpy()[:, 18:27].reshape(-1, 3, 3)
    nin = dn.cpu().numpy()
    rot_ok = float(np.mean([np.linalg.norm(Rg[p] - R[p]) < 0.05 for p in range(n_pairs) if nin[p] >= 0]))
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize()
    for a0, a1 in evs:
        with torch.cuda.stream(stream):
            flush.fill_(1)
        a0.record(stream)
        step_device()
        a1.record(stream)
    r.wait()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(ws, statistics.mean(a.elapsed_time(b) for a, b in evs), dev)
    launches = r.last_launches()
    r.profile(True)
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        step_device()
    r.wait()
    hyp_ms, hyp_n = r.profile_read(0)
    score_ms, score_n = r.profile_read(1)
    r.profile(False)
    rounds = hyp_n // max(args.steps, 1)  # launches of each kernel per call (one per round)
    hyp_ms /= args.steps  # per call, all rounds
    score_ms /= args.steps
    n_cand, n_evals = r.candidates()  # candidates scored and their Sampson evaluations, last call
    res = r.essential(off, corrs, K, RS_THR, RS_SAMPLES, seed=args.seed, flags=False)
    np.testing.assert_array_equal(res["models"], dm.cpu().numpy())
    # e2e: pinned host correspondences in, models and flags out
    cp = torch.from_numpy(corrs).pin_memory().numpy()
    for _ in range(max(args.warmup, 3)):
        r.essential(off, cp, K, RS_THR, RS_SAMPLES, seed=args.seed)
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(ws)
    torch.cuda.synchronize()
    for a0, a1 in ev2:
        with torch.cuda.stream(stream):
            flush.fill_(1)
        a0.record(stream)
        r.essential(off, cp, K, RS_THR, RS_SAMPLES, seed=args.seed)
        a1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(ws, statistics.mean(a.elapsed_time(b) for a, b in ev2), dev)
    r.close()
    if rank != 0:
        return
    line = {
        "metric": "image pairs/s robust relative orientation (5-point RANSAC, Sampson costs)",
        "value": ws * n_pairs * 1000.0 / ms, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded two-view correspondences)", "config": ransac_config(n_pairs, n_corrs, args.refine),
        "pose_recovered": rot_ok,
        "candidates": n_cand, "sampson_evaluations": n_evals,
        "kernels_ms_per_call": {"k_rs_hyp (five-point solutions)": hyp_ms, "k_rs_score (costs of the candidates)": score_ms,
                                "rounds": rounds},
        "roofline": {"bound": "fp64", "achieved": RS_FLOPS_PER_EVAL * n_evals / (score_ms * 1e-3) / 1e12,
                     "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                     "frac": RS_FLOPS_PER_EVAL * n_evals / (score_ms * 1e-3) / 1e12 / FP64_NOMINAL_TFLOPS,
                     "traffic": None, "peak_src": "nominal B200 FP64 (no measured FP64 peak on this pool)",
                     "kernel_ms": score_ms, "flops_per_call": RS_FLOPS_PER_EVAL * n_evals,
                     "kernel": f"k_rs_score, all rounds of one call ({RS_FLOPS_PER_EVAL} double operations per "
                               "Sampson evaluation)"},
        "e2e": {"value": ws * n_pairs * 1000.0 / ms_e2e, "unit": "pairs/s",
                "h2d_bytes_per_step": int(corrs.nbytes + off.nbytes + K.nbytes),
                "d2h_bytes_per_step": int(n_pairs * (31 * 8 + 4) + n_corrs)},
        "gpu_launches": launches * args.steps,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and ws == 1:
        from oracle import oracle
        if oracle.ref_ransac_available():
            sel = list(range(0, n_pairs, max(1, n_pairs // 16)))[:16]
            sec = ref_ransac_pairs(off, corrs, K, sel, args.refine)
            line["cpu_baseline"] = {"value": len(sel) / sec, "unit": "pairs/s", "cores": 1, "kind": "reference",
                                    "sample": f"{len(sel)} of the {n_pairs} pairs, the reference's solver and pose "
                                              "recovery in the loop restated, the app's own sample sequence "
                                              f"({sec:.1f} s)"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_init()
    try:
        if args.impl == "reference":
            run_reference_arm(args, ws, rank)
        elif args.workload == "pair":
            run_pair(args, ws, rank, local)
        elif args.workload == "stereo":
            run_stereo(args, ws, rank, local)
        elif args.workload == "batch":
            run_batch(args, ws, rank, local)
        elif args.workload == "batch-guided":
            run_batch_guided(args, ws, rank, local)
        elif args.workload == "batch-float":
            run_batch_float(args, ws, rank, local)
        elif args.workload == "voctree":
            run_voctree(args, ws, rank, local)
        elif args.workload == "proposal":
            run_proposal(args, ws, rank, local)
        elif args.workload == "float":
            run_float(args, ws, rank, local)
        elif args.workload == "ingest":
            run_ingest(args, ws, rank, local)
        elif args.workload == "retrieval":
            run_retrieval(args, ws, rank, local)
        elif args.workload == "ransac":
            run_ransac(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
