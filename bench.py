"""Benchmark: 3-phonon RTA linewidths on the 20x20x20 diamond mesh.

Workload (one "step"): the whole PhScatteringMatrix builder in linewidth mode
-- every (q1, q2) pair of the 8000-point Gamma-centred mesh (64,000,000
pairs, both +/- processes, all 216 branch triplets, 3 temperatures
100/300/600 K, adaptive smearing from group velocities) -- on synthetic
force constants of the diamond cell (seeded generator, phoebe_b200.synth).

metric: triplets/s, where a triplet is one (q1,q2) pair (q3 fixed by
momentum); linewidths/s = Nq*nb*nT / step time is reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision fp64|split_bf16|split_fp16] [--mesh 20]

Under torchrun each rank processes a contiguous slice of q2 and the
per-rank partial A_out vectors are summed with one NCCL all-reduce
(the reference's allReduceSum of the linewidths, ph_scattering.cpp:800).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

TEMPS_K = (100.0, 300.0, 600.0)
# FP32 FFMA throughput of a B200 (packed and scalar FFMA stream, all SMs, CUDA
# events), the denominator of the pair kernel's CUDA-core view
FFMA_PEAK_TFLOPS = 72.0
# nominal FP64 rate of a B200 (no measured FP64 peak exists for this pool)
FP64_PEAK_TFLOPS = 37.0
# ncu DRAM bytes (read + write) of one pair-kernel launch, per (precision,
# mesh, q2 per launch, slots) of the launch plan; None where not captured
PAIR_TRAFFIC_BYTES = {("split_bf16", 20, 448, 7): 87476992 + 5594112,
                      ("split_bf16", 20, 1792, 28): 337188096 + 29478400,
                      ("split_fp16", 20, 1792, 28): 339046144 + 134754304,
                      ("split_bf16", 16, 448, 7): 85.2e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="3ph", choices=["3ph", "elph", "smatrix", "perovskite", "relaxons", "twelve", "screening"],
                    help="3ph: the headline linewidth builder; elph: electron-phonon linewidths "
                         "(8 Wannier functions, 343 x 343 coupling vectors, 40^3 k, 20^3 q); smatrix: "
                         "the scattering matrix of the 3ph workload stored in device memory and its "
                         "matrix-vector products, beside the matrix-free product; perovskite: the batched "
                         "uneven instances (5-atom cell, 15 branches, 24^3 mesh, per-q1 q2 window) on a q2 "
                         "slice of --q2-slice points per step; relaxons: the relaxon solver (a2Omega, full "
                         "eigensolve, relaxon conductivity) on the stored matrix of the 3ph workload at --mesh; "
                         "twelve: the 12-atom cell (36 branches, 4000 FC3 pairs, 16^3 mesh) of the learned-screening "
                         "workload, split and FP64 on q2 slices of --q2-slice points; screening: learned screening "
                         "on the 12-atom cell at 16^3 (exact split run, training pairs from the exact builder, "
                         "screened run, errors)")
    ap.add_argument("--train-q2", type=int, default=512, help="screening: q2 points whose vertices train the network")
    ap.add_argument("--q2-slice", type=int, default=256, help="q2 points per perovskite step")
    ap.add_argument("--elph-k1", type=int, default=64, help="outer k points timed per elph step")
    ap.add_argument("--precision", default=os.environ.get("PHX_BENCH_PRECISION", "split_fp16"),
                    choices=["fp64", "split_bf16", "split_fp16"])
    ap.add_argument("--mesh", type=int, default=20)
    ap.add_argument("--num-relaxons", type=int, default=0,
                    help="relaxons workload: eigenpairs computed (0: all; k: the smallest k)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-fp64", action="store_true",
                    help="skip the plain FP64 GPU step that the split path is compared with")
    ap.add_argument("--kernels-only", action="store_true",
                    help="profiling aid: time the builder only (no e2e leg, no CPU baseline)")
    args = ap.parse_args()
    args.precision_given = any(a.startswith("--precision") for a in sys.argv[1:])
    return args


def workload(mesh):
    from phoebe_b200 import synth
    cr = synth.diamond_crystal()
    fc2 = synth.diamond_fc2(cr)
    fc3 = synth.random_fc3(cr, 400, synth.SEED_BASE)
    return cr, fc2, fc3, (mesh, mesh, mesh)


class Clocks:
    """nvidia-smi sampler for the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, n in enumerate(names):
                if len(s) > 4 + i and s[4 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def flops_per_pair(nb, nr3):
    """FLOPs the fused kernel executes per (q1,q2) pair (complex MAC = 8):
    the '+' vertex R3 transform (nb^3 nr3 MACs) and the e1 / e3 contractions
    (2 nb^4 MACs); the e2 contraction is folded per q2."""
    return 8 * nb ** 3 * nr3 + 8 * 2 * nb ** 4


def flops_per_pair_reference(nb, nr3):
    """F_pair of the reference's formulation (both vertices, three contractions)."""
    return 16 * nb ** 3 * nr3 + 16 * nb ** 4 + 16 * nb ** 4 + 8 * nb ** 4 * 2 + 3 * nb ** 3 * 2


def host_cpu():
    """CPU model, hardware threads and physical cores of this host (/proc/cpuinfo)."""
    model, cores = None, set()
    phys = core = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name" and model is None:
                    model = v
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    core = v
                elif not k and phys is not None:
                    cores.add((phys, core))
                    phys = core = None
        if phys is not None:
            cores.add((phys, core))
    except OSError:
        pass
    return {"cpu_model": model, "hardware_threads": os.cpu_count(),
            "physical_cores": len(cores) or None}


def cpu_baseline(cr, fc2, fc3, mesh, budget_s, q2_hint=None):
    """Oracle (restatement of the reference CPU path) on a q2 sample."""
    import oracle
    from phoebe_b200 import constants as C
    from phoebe_b200 import lattice
    m = lattice.Mesh(cr, mesh)
    q = m.cartesian_coords()
    h0 = oracle.PhononH0(cr, fc2)
    E, U = h0.diagonalize(q)
    vg = h0.velocities(q)
    v3 = oracle.Interaction3Ph(cr, fc3)
    T = np.array([C.kelvin_to_ry(t) for t in TEMPS_K])
    nq = m.num_points
    rng = np.random.default_rng(0)
    order = rng.permutation(nq)
    t0 = time.perf_counter()
    v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0,
                  q2_list=order[:1], finalize=False)
    t1 = time.perf_counter() - t0
    n = max(1, min(nq - 1, int(budget_s / max(t1, 1e-3))))
    if q2_hint:
        n = q2_hint
    t0 = time.perf_counter()
    v3.linewidths(mesh, E, U, vg, q, cr.reciprocal_cell, T, "adaptive", 0.0,
                  q2_list=order[1:1 + n], finalize=False)
    dt = time.perf_counter() - t0
    pairs = n * nq
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return dict({"value": pairs / dt, "unit": "triplets/s", "cores": threads, "kind": "port",
                 "sample": "%d q2 points x all %d q1 of the %s mesh (%d pairs, %.1f s), OpenMP oracle"
                           % (n, nq, "x".join(map(str, mesh)), pairs, dt),
                 "sample_wall_s": t1 + dt}, **host_cpu())


def headline_config(n, nr3, precision, world):
    """The `config` of the headline line (n^3 mesh); the reference arm prints the same."""
    nq = n ** 3
    return {"workload": "diamond %dx%dx%d (%d q, %ge6 pairs), 400 FC3 pairs "
                        "(nr3=%d), adaptive smearing, T=100/300/600 K" % (n, n, n, nq, nq * nq / 1e6, nr3),
            "precision": precision, "l2": "flushed between steps (256 MB write)",
            "parallelism": "q2-sliced x%d" % world}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    cr, fc2, fc3, mesh = workload(args.mesh)
    import oracle
    oracle.lib()
    vals = []
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(cr, fc2, fc3, mesh, max(2.0, args.cpu_seconds / 3), q2_hint=None)
        if i >= args.warmup:
            vals.append(b["value"])
    v = float(np.median(vals))
    nq = int(np.prod(mesh))
    # a step is the whole builder (nq^2 pairs); each step here times a bounded
    # q2 sample, so the step time is projected from the measured rate
    line = {"impl": "reference", "metric": "3ph triplets/s @20^3 mesh", "value": v,
            "unit": "triplets/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * nq * nq / v, "projected_from_sample": True,
            "sample_wall_s_per_step": b["sample_wall_s"], "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            # the workload of the GPU arm's line; what this arm ran of it per step is
            # cpu_baseline.sample (a q2 sample of the same FP64 builder, on the host)
            "config": headline_config(args.mesh, fc3.D3.shape[3], args.precision, world),
            "cpu_baseline": dict(b, value=v),
            "e2e": {"value": v, "unit": "triplets/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from phoebe_b200 import _abi
    from phoebe_b200 import constants as C
    from phoebe_b200.core import (Context, Interaction3Ph, PhononH0, PhScatteringMatrix,
                                  finalize_linewidths, q2_slice)
    import ctypes

    cr, fc2, fc3, mesh = workload(args.mesh)
    nq = int(np.prod(mesh))
    nb = cr.num_bands
    nr3 = fc3.D3.shape[3]
    T = np.array([C.kelvin_to_ry(t) for t in TEMPS_K])
    nT = len(T)
    torch.cuda.set_device(local)
    ctx = Context(local)
    h0 = PhononH0(ctx, cr, fc2)
    bands = h0.populate(mesh, withVelocities=True)
    v3 = Interaction3Ph(ctx, cr, fc3, precision=args.precision)
    sm = PhScatteringMatrix(v3, bands, T, "adaptive")
    q2b, q2e = q2_slice(rank, world, nq)
    A = torch.zeros(nT * nq * nb, dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    L = _abi.load()

    def step():
        p = sm._params(q2b, q2e, finalize=(world == 1))
        st = _abi.LwStats()
        _abi.check(L.phx_ph_linewidths_d(v3.h, bands.h, ctypes.byref(p),
                                         ctypes.c_void_p(A.data_ptr()), ctypes.byref(st)), ctx.h)
        return st

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
        flush.zero_()
    barrier()
    dev_ms = []
    vertex_ms = []
    pair_ms = []
    pair_launches = 0
    launches = 0
    with Clocks(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            st = step()
            dev_ms.append(st.ms_total)
            vertex_ms.append(st.ms_vertex)
            pair_ms.append(st.ms_pair)
            pair_launches += st.pair_launches
            launches += st.kernel_launches
            plan = {"q2_chunk": st.plan_chunk, "slots": st.plan_slots,
                    "cuda_graph": ["eager", "captured", "replayed"][st.graph]}
        barrier()
        wall = time.perf_counter() - t0
    total_ms = float(np.sum(dev_ms))
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_step = total_ms / args.steps
    pairs_step = nq * nq
    value = pairs_step / (ms_step / 1000.0)

    # end to end through the public API with host buffers, every step:
    # FC2/FC3 host->device, band structure, builder, A_out device->host
    h2d = fc2.nbytes + fc3.D3.nbytes + fc3.R2.nbytes + fc3.R3.nbytes + fc3.w2.nbytes + \
        fc3.w3.nbytes + T.nbytes
    d2h = nT * nq * nb * 8

    # the step's inputs in pinned host memory (copied there outside the timed region)
    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()
    from phoebe_b200.synth import FC3
    fc2p = pinned(fc2)
    fc3p = FC3(pinned(fc3.D3), pinned(fc3.R2), pinned(fc3.R3), pinned(fc3.w2), pinned(fc3.w3), fc3.num_pairs)
    Tp = pinned(T)
    e2e_times = []
    for i in range(0 if args.kernels_only else 1 + min(args.steps, 3)):
        barrier()
        t0 = time.perf_counter()
        h0e = PhononH0(ctx, cr, fc2p)
        be = h0e.populate(mesh, withVelocities=True)
        ve = Interaction3Ph(ctx, cr, fc3p, precision=args.precision)
        se = PhScatteringMatrix(ve, be, Tp, "adaptive")
        Ae = se.setup(q2b, q2e, finalize=(world == 1))
        if dist:
            At = torch.from_numpy(Ae).cuda()
            dist.all_reduce(At)
            Ae = finalize_linewidths(At.cpu().numpy(), be.get(velocities=False)[0])
        ve.close()
        be.close()
        h0e.close()
        dt = time.perf_counter() - t0
        if i > 0:
            e2e_times.append(dt)
    e2e_value = pairs_step / float(np.median(e2e_times)) if e2e_times else None

    # roofline of the dominant kernel (fused pair kernel): algorithmic FLOPs of
    # all its launches / their CUDA-event time (events around each launch)
    fl = flops_per_pair(nb, nr3)
    achieved = fl * (q2e - q2b) * nq * args.steps / (float(np.sum(pair_ms)) / 1000.0) / 1e12
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    if args.precision == "fp64":
        roof = {"bound": "fp64", "achieved": achieved, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
                "frac": achieved / FP64_PEAK_TFLOPS, "traffic": None,
                "note": "plain FP64 SIMT path; peak is the nominal B200 FP64 rate (no measured "
                        "FP64 peak available)"}
    else:
        pk = peaks.get("bf16_tflops_sustained", 1394.6)
        # DRAM bytes per launch of the pair kernel, ncu dram__bytes_read.sum +
        # dram__bytes_write.sum of one launch of the plan in use
        roof = {"bound": "tensor", "achieved": achieved, "peak": pk, "unit": "TFLOP/s",
                "frac": achieved / pk,
                "traffic": PAIR_TRAFFIC_BYTES.get((args.precision, args.mesh, plan["q2_chunk"], plan["slots"])),
                "peak_source": "measured (sustained)",
                "simt_view": {"what": "FP32 epilogue (e1, e3 contractions of all 216 triplets) "
                                      "against the measured FFMA rate",
                              "flops_per_pair": 16 * nb ** 4,
                              "achieved": 16 * nb ** 4 * achieved / fl, "peak": FFMA_PEAK_TFLOPS,
                              "frac": 16 * nb ** 4 * achieved / fl / FFMA_PEAK_TFLOPS}}
    roof["flops_per_pair"] = fl
    roof["pair_launches"] = pair_launches
    roof["ms_per_pair_launch"] = float(np.sum(pair_ms)) / max(1, pair_launches)
    roof["flops_per_pair_reference_formulation"] = flops_per_pair_reference(nb, nr3)

    # the plain FP64 GPU path on the same workload, timed like the split path:
    # two untimed calls (eager, then captured into a CUDA graph), then replays
    fp64 = None
    edge_peak = int(st.edge_events_peak)
    if args.precision != "fp64" and not args.kernels_only and not args.no_fp64:
        A_split = A.clone()   # the last timed step's A_out
        v3.setPrecision("fp64")
        for _ in range(2):
            step()
        flush.zero_()
        barrier()
        ms64s, pms64, pl64 = [], [], 0
        for _ in range(3):
            flush.zero_()
            torch.cuda.synchronize()
            st64 = step()
            ms64s.append(st64.ms_total)
            pms64.append(st64.ms_pair)
            pl64 += st64.pair_launches
        barrier()
        ms64 = float(np.mean(ms64s))
        if dist:
            t = torch.tensor([ms64], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms64 = float(t.item())
        v3.setPrecision(args.precision)
        ach64 = fl * (q2e - q2b) * nq * 3 / (float(np.sum(pms64)) / 1000.0) / 1e12
        fp64 = {"ms_per_step": ms64, "value": pairs_step / (ms64 / 1000.0), "unit": "triplets/s",
                "dtype": "f64", "steps": 3, "timing": "CUDA graph replays after an eager and a captured call",
                "split_speedup": ms64 / ms_step,
                "roofline": {"bound": "fp64", "achieved": ach64, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
                             "frac": ach64 / FP64_PEAK_TFLOPS, "flops_per_pair": fl,
                             "ms_per_pair_launch": float(np.sum(pms64)) / max(1, pl64),
                             "peak_source": "fallback: nominal B200 FP64 rate (no measured FP64 peak)"}}
        if world == 1:
            # accuracy of the split path on this workload: relative error of the
            # linewidths (A_out / n(n+1), the same ratio) of non-excluded states
            # with A_out above 1e-8 of the largest, and of the RTA conductivity
            a64 = A.cpu().numpy().reshape(nT, -1)
            a16 = A_split.cpu().numpy().reshape(nT, -1)
            Eb = bands.get(velocities=False)[0].reshape(-1)
            big = (Eb >= C.phExcludeCutoff)[None, :] & (np.abs(a64) > 1e-8 * np.abs(a64).max())
            rel = np.abs(a16 - a64)[big] / np.abs(a64)[big]
            fp64["split_linewidth_rel_err"] = {"max": float(rel.max()), "p99": float(np.quantile(rel, 0.99)),
                                               "median": float(np.median(rel)), "states": int(big.sum())}

            def kappa(a):
                k = np.zeros((nT, 3, 3))
                _abi.check(L.phx_ph_rta_kappa(bands.h, nT, T.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                              np.ascontiguousarray(a).ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                              float(cr.volume), k.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                           ctx.h)
                return k
            k64, k16 = kappa(a64), kappa(a16)
            d64 = np.array([np.diagonal(k) for k in k64])
            d16 = np.array([np.diagonal(k) for k in k16])
            fp64["split_kappa_rel_err"] = {"max": float(np.abs(d16 - d64).max() / np.abs(d64).max()),
                                           "per_temperature": [float(np.abs(d16[t] - d64[t]).max() /
                                                                     np.abs(d64[t]).max()) for t in range(nT)],
                                           "what": "diagonal RTA conductivity, each temperature"}

    out = None
    if rank == 0:
        cpu = None if args.kernels_only else cpu_baseline(cr, fc2, fc3, mesh, args.cpu_seconds)
        out = {"metric": "3ph triplets/s @20^3 mesh", "value": value, "unit": "triplets/s",
               "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
               "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else
               ("bf16x3->f32" if args.precision == "split_bf16" else "fp16x3->f32"),
               "data": "synthetic",
               "config": headline_config(args.mesh, nr3, args.precision, world),
               "linewidths_per_s": nq * nb * nT / (ms_step / 1000.0),
               "branch_triplets_per_s": value * 2 * nb ** 3,
               "wall_s_timed": wall,
               "e2e": {"value": e2e_value, "unit": "triplets/s", "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(d2h)},
               "gpu_launches": launches,
               "launch_plan": plan,
               "near_cutoff_events": {"peak_per_pair_launch": edge_peak,
                                      "capacity": int(st.edge_events_cap)},
               "roofline": roof,
               "cpu_baseline": cpu,
               "fp64_path": fp64,
               "clocks": clk.summary()}
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_elph(args):
    """Electron-phonon linewidths on a bounded sample of outer k points; the FP64 path is timed beside
    the split one."""
    import torch
    from phoebe_b200 import constants as C
    from phoebe_b200 import synth
    from phoebe_b200.core import (Context, ElectronH0Wannier, ElScatteringMatrix, InteractionElPhWan,
                                  PhononH0)
    model = synth.elph_model(nw=8, ncell_h=3, ncell_e=3, ncell_p=3)
    cr = model.crystal
    kmesh, qmesh = (40, 40, 40), (20, 20, 20)
    torch.cuda.set_device(0)
    ctx = Context(0)
    wan = ElectronH0Wannier(ctx, cr, model.Re, model.degE, model.H)
    el = wan.populate(kmesh, withVelocities=True)
    h0 = PhononH0(ctx, cr, synth.diamond_fc2(cr))
    ph = h0.populate(qmesh, withVelocities=False)
    elph = InteractionElPhWan(ctx, model.Re, model.degE, model.Rp, model.degP, model.g)
    Ek = el.get(velocities=False)[0]
    mu = float(np.median(Ek))
    window = 0.3 / C.energyRyToEv
    lo, hi = synth.active_window(Ek, mu, window)
    active = np.nonzero(hi > lo)[0]
    T = np.array([C.kelvin_to_ry(300.0)])
    sm = ElScatteringMatrix(elph, el, ph, T, mu, window, "adaptive")
    prec = "fp64" if args.precision == "fp64" else "split_bf16"

    def timed(precision):
        elph.setPrecision(precision)
        rng = np.random.default_rng(0)
        ms = []
        for i in range(args.warmup + args.steps):
            k1 = np.sort(rng.choice(active, args.elph_k1, replace=False)).astype(np.int32)
            sm.setup(k1)
            if i >= args.warmup:
                ms.append(sm.stats.ms_total)
        return float(np.mean(ms)), k1

    ms_step, k1 = timed(prec)
    ms64 = ms_step if prec == "fp64" else timed("fp64")[0]
    pairs = sm.stats.pairs
    states = int(np.sum(hi[k1] - lo[k1]))
    line = {"metric": "el-ph (k1,q) pairs/s, 8 Wannier bands, 343x343 vectors, 40^3 k x 20^3 q",
            "value": pairs / (ms_step / 1000.0), "unit": "pairs/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "bf16x3/f32 Rp transform, f64 rest",
            "data": "synthetic",
            "config": {"workload": "el-ph linewidths, %d outer k (of %d active of 64000), all 8000 q, "
                                   "window +-0.3 eV, adaptive smearing, 300 K" % (args.elph_k1, len(active)),
                       "coupling_bytes": int(model.g.nbytes)},
            "carrier_linewidths_per_s": states / (ms_step / 1000.0),
            "fp64_path": {"ms_per_step": ms64, "value": pairs / (ms64 / 1000.0), "split_speedup": ms64 / ms_step},
            "pairs_per_step": int(pairs)}
    print(json.dumps(line), flush=True)


def run_smatrix(args):
    """Scattering-matrix modes on the 3ph workload at one temperature: the stored matrix (FP64,
    ns x ns in device memory) is built once, then its matrix-vector product A x (3 components) is
    timed; the matrix-free product (one builder pass) is timed beside it."""
    import ctypes

    import torch
    from phoebe_b200 import _abi
    from phoebe_b200 import constants as C
    from phoebe_b200.core import Context, Interaction3Ph, PhononH0, PhScatteringMatrix
    cr, fc2, fc3, mesh = workload(args.mesh)
    torch.cuda.set_device(0)
    ctx = Context(0)
    h0 = PhononH0(ctx, cr, fc2)
    bands = h0.populate(mesh, withVelocities=True)
    prec = args.precision if args.precision_given else "fp64"
    v3 = Interaction3Ph(ctx, cr, fc3, precision=prec)
    T = [C.kelvin_to_ry(300.0)]
    ns = bands.nq * bands.nb
    sm = PhScatteringMatrix(v3, bands, T, "adaptive", in_memory=True)
    sm.setup()
    ms_build = sm.stats.ms_total
    L = _abi.load()
    x = torch.randn(1, 3, ns, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    ms = ctypes.c_float()
    times = []
    with Clocks(0) as clk:
        for i in range(args.warmup + args.steps):
            _abi.check(L.phx_smatrix_dot_d(sm._m, 1, ctypes.c_void_p(x.data_ptr()), 0,
                                           ctypes.c_void_p(y.data_ptr()), ctypes.byref(ms)), ctx.h)
            if i >= args.warmup:
                times.append(ms.value)
    ms_dot = float(np.mean(times))
    # matrix-free product of the same x, one builder pass
    free = PhScatteringMatrix(v3, bands, T, "adaptive")
    yf = free.dot(x.cpu().numpy())
    ms_free = free.stats.ms_total
    err = float(np.abs(yf - y.cpu().numpy()).max() / np.abs(yf).max())
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    nbytes = 8.0 * ns * ns + 8.0 * 3 * ns * 2
    achieved = nbytes / (ms_dot / 1000.0) / 1e9
    line = {"metric": "stored scattering-matrix products A x per second (3 components), diamond 20^3, 48000 states",
            "value": 1000.0 / ms_dot, "unit": "products/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_dot, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "diamond %dx%dx%d, 400 FC3 pairs, adaptive smearing, 300 K; matrix %d x %d "
                                   "FP64 (%.1f GB) in device memory, larger than L2" % (*mesh, ns, ns,
                                                                                         8e-9 * ns * ns)},
            "matrix_build_ms": ms_build,
            "build_precision": prec,
            "matrix_free_product_ms": ms_free,
            "stored_vs_matrix_free_speedup": ms_free / ms_dot,
            "stored_vs_matrix_free_rel_err": err,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": None, "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    sm.close()


def run_relaxons(args):
    """Relaxon solver on the stored FP64 matrix of the 3ph workload (one temperature, boundary
    scattering of 3e4 Bohr): a2Omega in device memory, the eigensolve of the ns x ns matrix
    (cuSOLVER, in place; all eigenpairs, or the smallest --num-relaxons), then the relaxon
    conductivity.  One pass (the eigensolve destroys the
    matrix); each stage is a synchronous library call, timed by the host clock around it.  The
    process does not load PyTorch: beyond the single-GPU eigensolvers' size the library opens
    cuSOLVER's multi-GPU solver, which needs the toolkit's own cuBLAS."""
    from phoebe_b200 import constants as C
    from phoebe_b200 import lattice, solvers
    from phoebe_b200.core import Context, Interaction3Ph, PhononH0, PhScatteringMatrix
    cr, fc2, fc3, mesh = workload(args.mesh)
    ctx = Context(0)
    h0 = PhononH0(ctx, cr, fc2)
    bands = h0.populate(mesh, withVelocities=True)
    E, _, vg = bands.get()
    v3 = Interaction3Ph(ctx, cr, fc3)
    T = C.kelvin_to_ry(300.0)
    ns = bands.nq * bands.nb
    P = solvers.BteProblem(E, vg, [T], int(np.prod(mesh)), lattice.calc_volume(cr.direct_cell))
    sm = PhScatteringMatrix(v3, bands, [T], "adaptive", boundary_length=3.0e4, in_memory=True)
    with Clocks(0) as clk:
        sm.setup()
        ms_build = sm.stats.ms_total
        t0 = time.perf_counter()
        sm.a2Omega()
        t1 = time.perf_counter()
        lam = sm.diagonalize(args.num_relaxons)
        t2 = time.perf_counter()
        kappa = solvers.relaxons(P, sm.relaxonSolve)[0]
        t3 = time.perf_counter()
    total = t3 - t0
    line = {"metric": "relaxon solver wall time after the matrix build, diamond %d^3, %d states" % (args.mesh, ns),
            "value": total, "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": 1000.0 * total,
            "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "diamond %dx%dx%d, 400 FC3 pairs, adaptive smearing, boundary 3e4 Bohr, 300 K; "
                                   "matrix %d x %d FP64 (%.2f GB) in device memory" % (*mesh, ns, ns,
                                                                                        8e-9 * ns * ns)},
            "matrix_build_ms": ms_build, "a2omega_s": t1 - t0, "eigensolve_s": t2 - t1,
            "relaxon_kappa_s": t3 - t2, "eigenpairs": int(lam.size), "positive_eigenvalues": int((lam > 0).sum()),
            "kappa_diag_au": np.diagonal(kappa).tolist(), "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    sm.close()


def run_perovskite(args):
    """Batched uneven instances (the 15-branch perovskite cell on the 24^3 mesh with per-q1 q2
    windows): the band structure of all 13 824 points in one launch, then the windowed FP64
    builder over a slice of q2 per step (every q1); the full run is projected from the rate."""
    import torch
    from phoebe_b200 import constants as C
    from phoebe_b200 import synth
    from phoebe_b200.core import Context, Interaction3Ph, PhononH0, PhScatteringMatrix
    w = synth.config2()
    torch.cuda.set_device(0)
    ctx = Context(0)
    h0 = PhononH0(ctx, w.crystal, w.fc2)
    t0 = time.perf_counter()
    bands = h0.populate(w.mesh, withVelocities=True)
    bands_s = time.perf_counter() - t0
    E = bands.get(velocities=False)[0]
    energy, cut = synth.q2_window(E, w.mesh)
    v3 = Interaction3Ph(ctx, w.crystal, w.fc3)
    T = np.array([C.kelvin_to_ry(t) for t in w.temperatures_k])
    sm = PhScatteringMatrix(v3, bands, T, "adaptive", window=(energy, cut))
    nq = bands.nq
    keep = energy[None, :] <= cut[:, None]                     # (q1, q2)
    per_q2 = keep.sum(axis=0)                                 # windowed q1 per q2
    rng = np.random.default_rng(0)
    ms, pairs = [], []
    with Clocks(0) as clk:
        for i in range(args.warmup + args.steps):
            q0 = int(rng.integers(0, nq - args.q2_slice))
            sm.setup(q0, q0 + args.q2_slice, finalize=False)
            if i >= args.warmup:
                ms.append(sm.stats.ms_total)
                pairs.append(int(per_q2[q0:q0 + args.q2_slice].sum()))
    ms_step = float(np.mean(ms))
    rate = float(np.sum(pairs) / (np.sum(ms) / 1000.0))
    total = int(keep.sum())
    # the split path (many-branch builder, tcgen05 R3 transform) on the same slices
    prec = args.precision if args.precision != "fp64" else "split_fp16"
    v3.setPrecision(prec)
    rng = np.random.default_rng(0)
    ms16, pairs16 = [], []
    for i in range(args.warmup + args.steps):
        q0 = int(rng.integers(0, nq - args.q2_slice))
        sm.setup(q0, q0 + args.q2_slice, finalize=False)
        if i >= args.warmup:
            ms16.append(sm.stats.ms_total)
            pairs16.append(int(per_q2[q0:q0 + args.q2_slice].sum()))
    rate16 = float(np.sum(pairs16) / (np.sum(ms16) / 1000.0))
    tile = {"register_tile": int(sm.stats.tile_rt), "q1_planes_per_pass": int(sm.stats.tile_qp)}
    line = {"metric": "windowed (q1,q2) pairs/s, 15 branches, 24^3 mesh, per-q1 q2 window",
            "value": rate, "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "perovskite 5-atom cell, 1500 FC3 pairs (nr3=%d), 24x24x24 mesh, q2 window "
                                   "keeping 20-100%% per q1, adaptive smearing, 300 K; %d q2 x all q1 per step "
                                   "(random slice)" % (v3.nr3, args.q2_slice),
                       "windowed_pairs_total": total, "window_fill": total / float(nq * nq)},
            "bands_s_13824_points": bands_s,
            "projected_full_run_s": total / rate,
            "split_path": {"precision": prec, "value": rate16, "unit": "pairs/s", "ms_per_step": float(np.mean(ms16)),
                           "tile_shape": tile,
                           "speedup_over_fp64": rate16 / rate, "projected_full_run_s": total / rate16},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_twelve(args):
    """The 12-atom cell (36 branches, 4000 FC3 pairs, 16^3 mesh, adaptive smearing, 300 K) on the
    many-branch builder: the split path and the FP64 path on the same random q2 slices (every q1),
    their linewidth partial sums compared; the full run is projected from the rates."""
    import torch
    from phoebe_b200 import constants as C
    from phoebe_b200 import synth
    from phoebe_b200.core import Context, Interaction3Ph, PhononH0, PhScatteringMatrix
    t0 = time.perf_counter()
    w = synth.twelve_atom_workload()
    gen_s = time.perf_counter() - t0
    torch.cuda.set_device(0)
    ctx = Context(0)
    h0 = PhononH0(ctx, w.crystal, w.fc2)
    t0 = time.perf_counter()
    bands = h0.populate(w.mesh, withVelocities=True)
    bands_s = time.perf_counter() - t0
    prec = args.precision if args.precision != "fp64" else "split_fp16"
    v3 = Interaction3Ph(ctx, w.crystal, w.fc3, precision=prec)
    T = np.array([C.kelvin_to_ry(t) for t in w.temperatures_k])
    sm = PhScatteringMatrix(v3, bands, T, "adaptive")
    nq, nb, nr3 = bands.nq, bands.nb, v3.nr3
    rng = np.random.default_rng(0)
    starts = [int(rng.integers(0, nq - args.q2_slice)) for _ in range(args.warmup + args.steps)]
    ms, parts, pms, plaunch = [], [], [], 0
    with Clocks(0) as clk:
        for i, q0 in enumerate(starts):
            A = sm.setup(q0, q0 + args.q2_slice, finalize=False)
            if i >= args.warmup:
                ms.append(sm.stats.ms_total)
                pms.append(sm.stats.ms_pair)
                plaunch += sm.stats.pair_launches
                parts.append(A)
    ms_step = float(np.mean(ms))
    pairs_step = nq * args.q2_slice
    rate = pairs_step / (ms_step / 1000.0)
    tile = {"register_tile": int(sm.stats.tile_rt), "q1_planes_per_pass": int(sm.stats.tile_qp),
            "q1_per_item": 8, "ctas": int(sm.stats.plan_slots), "q2_per_chunk": int(sm.stats.plan_chunk)}
    # FP64 on the same slices (the first two timed ones)
    v3.setPrecision("fp64")
    ms64, rel = [], []
    for i, q0 in enumerate(starts[args.warmup:args.warmup + 2]):
        A64 = sm.setup(q0, q0 + args.q2_slice, finalize=False)
        ms64.append(sm.stats.ms_total)
        big = np.abs(A64) > 1e-8 * np.abs(A64).max()
        rel.append(float((np.abs(parts[i] - A64)[big] / np.abs(A64)[big]).max()))
    rate64 = pairs_step / (float(np.mean(ms64)) / 1000.0)
    fl_tc = 8 * nb ** 3 * nr3            # R3 transform per pair (tensor cores)
    fl_simt = 16 * nb ** 4               # e1 and e3 contractions per pair (CUDA cores, FP32)
    ach = fl_tc * pairs_step * len(pms) / (float(np.sum(pms)) / 1000.0) / 1e12
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    pk = peaks.get("bf16_tflops_sustained", 1346.1)
    ach_simt = fl_simt * pairs_step * len(pms) / (float(np.sum(pms)) / 1000.0) / 1e12
    line = {"metric": "3ph (q1,q2) pairs/s, 12-atom cell (36 branches), 16^3 mesh",
            "value": rate, "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "fp16x3->f32" if prec == "split_fp16" else "bf16x3->f32", "data": "synthetic",
            "config": {"workload": "12-atom cell, 36 branches, 4000 FC3 pairs (nr3=%d), 16x16x16 mesh, adaptive "
                                   "smearing, 300 K; %d q2 x all %d q1 per step (random slice)"
                                   % (nr3, args.q2_slice, nq), "fc3_generation_s": gen_s},
            "bands_s_4096_points": bands_s,
            "projected_full_run_s": nq * nq / rate,
            "tile_shape": tile,
            "fp64_path": {"value": rate64, "unit": "pairs/s", "ms_per_step": float(np.mean(ms64)),
                          "split_speedup": rate / rate64, "projected_full_run_s": nq * nq / rate64,
                          "split_partial_linewidth_rel_err_max": max(rel)},
            "roofline": {"bound": "tensor", "achieved": ach, "peak": pk, "unit": "TFLOP/s", "frac": ach / pk,
                         "traffic": None, "flops_per_pair": fl_tc, "peak_source": "measured (sustained)",
                         "ms_per_pair_launch": float(np.sum(pms)) / max(1, plaunch),
                         "simt_view": {"what": "FP32 e1/e3 contractions on CUDA cores", "flops_per_pair": fl_simt,
                                       "achieved": ach_simt, "peak": FFMA_PEAK_TFLOPS,
                                       "frac": ach_simt / FFMA_PEAK_TFLOPS}},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_screening(args):
    """Learned screening on the 12-atom cell (36 branches, 4000 FC3 pairs, 16^3 mesh, adaptive
    smearing, 300 K).  The exact split builder over every (q1, q2) vertex; the network
    (12 -> 256 -> 256 -> 256 -> 1, tensor-core kernels) trained on the exact contributions of the
    vertices of --train-q2 q2 points (every q1), each from a one-q2 call of the builder; the
    threshold calibrated on those; then the screened builder over every vertex.  FP64 is timed on a
    q2 slice for the three-way comparison."""
    import torch
    from phoebe_b200 import constants as C
    from phoebe_b200 import screening, synth
    from phoebe_b200.core import Context, Interaction3Ph, PhononH0, PhScatteringMatrix
    w = synth.twelve_atom_workload()
    torch.cuda.set_device(0)
    ctx = Context(0)
    h0 = PhononH0(ctx, w.crystal, w.fc2)
    bands = h0.populate(w.mesh, withVelocities=True)
    E = bands.get(velocities=False)[0]
    prec = args.precision if args.precision != "fp64" else "split_fp16"
    v3 = Interaction3Ph(ctx, w.crystal, w.fc3, precision=prec)
    T = np.array([C.kelvin_to_ry(t) for t in w.temperatures_k])
    sm = PhScatteringMatrix(v3, bands, T, "adaptive")
    nq, nb = bands.nq, bands.nb
    with Clocks(0) as clk:
        A_exact = sm.setup()
        ms_exact = sm.stats.ms_total
        k_exact = sm.thermalConductivity(w.crystal.volume)
        # training pairs from the exact builder, one q2 at a time
        rng = np.random.default_rng(4)
        q2_train = np.sort(rng.choice(nq, size=min(args.train_q2, nq), replace=False))
        t0 = time.perf_counter()
        u = screening.pair_contributions(sm, q2_train)                  # (nt, nq, nb)
        gen_s = time.perf_counter() - t0
        A0 = A_exact[0].reshape(nq, nb)
        X = screening.pair_features(w.mesh, E, q2_train).reshape(-1, screening.NIN)
        y = screening.pair_targets(u, A0).reshape(-1)
        net = screening.ScreeningMLP(ctx, seed=7)
        t0 = time.perf_counter()
        epochs = 6
        losses = net.train(X, y, epochs=epochs, batch=4096, lr=1e-3)
        train_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        pred = net.infer(X).reshape(len(q2_train), nq)
        infer_s = time.perf_counter() - t0
        # threshold: the largest whose drops, scaled from the training q2 to the whole mesh,
        # move no training linewidth by more than 5e-4
        frac = u / np.where(A0 > 0, A0, np.inf)[None]
        scale = nq / float(len(q2_train))
        thr = None
        for cand in np.arange(-3.0, -12.01, -0.25):
            drop = pred < cand
            err = (np.where(drop[:, :, None], frac, 0.0).sum(axis=0) * scale).max()
            if err <= 5e-4:
                thr = float(cand)
                break
        # perfect screen on the training vertices: the most vertices of each q1 that can go
        # (smallest largest-fraction first) with the scaled drop <= 1e-3 for every mode
        fmax = frac.max(axis=2)                                        # (nt, nq)
        perfect = 0
        for q1 in range(nq):
            order = np.argsort(fmax[:, q1])
            cum = np.cumsum(frac[order, q1, :], axis=0) * scale          # (nt, nb)
            ok = np.nonzero(cum.max(axis=1) <= 1e-3)[0]
            perfect += 0 if ok.size == 0 else ok[-1] + 1
        perfect_frac = perfect / float(fmax.size)
        A_scr = sm.setup_screened(net, thr if thr is not None else -np.inf)
        ms_scr = sm.stats.ms_total
        skipped = int(sm.stats.pairs_screened_out)
        k_scr = sm.thermalConductivity(w.crystal.volume)
    ok = (E.reshape(-1) >= C.phExcludeCutoff)[None, :]
    big = ok & (np.abs(A_exact) > 1e-8 * np.abs(A_exact).max())
    lw_err = float((np.abs(A_scr - A_exact)[big] / np.abs(A_exact)[big]).max())
    d0, d1 = np.diagonal(k_exact[0]), np.diagonal(k_scr[0])
    kappa_err = float(np.abs(d1 - d0).max() / np.abs(d0).max())
    # FP64 on a q2 slice
    v3.setPrecision("fp64")
    sl = min(args.q2_slice, nq)
    sm.setup(0, sl, finalize=False)
    ms64 = sm.stats.ms_total
    rate64 = nq * sl / (ms64 / 1000.0)
    pairs = nq * nq
    line = {"metric": "3ph (q1,q2) pairs/s with learned screening, 12-atom cell (36 branches), 16^3 mesh",
            "value": pairs / (ms_scr / 1000.0), "unit": "pairs/s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "ms_per_step": ms_scr, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "fp16x3->f32" if prec == "split_fp16" else "bf16x3->f32", "data": "synthetic",
            "config": {"workload": "12-atom cell, 36 branches, 4000 FC3 pairs (nr3=%d), 16x16x16 mesh (%d vertices), "
                                   "adaptive smearing, 300 K" % (v3.nr3, pairs),
                       "network": "12-256-256-256-1 GELU, BF16 weights, FP32 accumulation, tcgen05 GEMMs"},
            "exact_split": {"value": pairs / (ms_exact / 1000.0), "ms": ms_exact},
            "exact_fp64": {"value": rate64, "ms_per_%d_q2" % sl: ms64, "projected_full_run_s": pairs / rate64},
            "screened_split": {"value": pairs / (ms_scr / 1000.0), "ms": ms_scr, "vertices_dropped": skipped,
                               "fraction_dropped": skipped / float(pairs),
                               "speedup_over_exact_split": ms_exact / ms_scr,
                               "speedup_over_fp64": (pairs / (ms_scr / 1000.0)) / rate64,
                               "log10_threshold": thr, "linewidth_rel_err_max": lw_err,
                               "kappa_rel_err": kappa_err},
            "training": {"vertices": int(X.shape[0]), "q2_points": int(len(q2_train)), "epochs": epochs,
                         "data_generation_s": gen_s, "train_s": train_s,
                         "train_samples_per_s": X.shape[0] * epochs / train_s,
                         "loss_first_last": [float(losses[0]), float(losses[-1])],
                         "inference_ns_per_vertex": 1e9 * infer_s / X.shape[0]},
            "perfect_screen_bound": {"fraction_of_training_vertices": perfect_frac,
                                     "what": "vertices a perfect screen could drop with every linewidth within 1e-3"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "screening":
        run_screening(args)
        return
    if args.workload == "twelve":
        run_twelve(args)
        return
    if args.workload == "perovskite":
        run_perovskite(args)
        return
    if args.workload == "elph":
        run_elph(args)
        return
    if args.workload == "smatrix":
        run_smatrix(args)
        return
    if args.workload == "relaxons":
        run_relaxons(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
