"""Benchmark of the B200 PyOP2 backend on the airfoil loop chain.

Workload: the airfoil finite-volume chain on a synthetic
1200 x 600 quad mesh (720,000 cells, 1,438,200 interior edges, 3,600 boundary
edges) with randomly permuted cell and node numbering, FP64.  One step = one
outer iteration: save_soln, then twice (adt_calc, res_calc, bres_calc, update
with the rms reduction) -- 9 par_loops, 565.6 MB of algorithmic traffic.

Metric: par_loop achieved HBM GB/s = algorithmic bytes of the step / device
time of the step.

* ``value``: the step replayed as a CUDA graph recorded through the op2 API,
  inputs resident in HBM, L2 flushed (256 MB write) before every step; each
  step timed by its own pair of CUDA events on the op2 stream, summed.
* ``e2e``: the configuration's 100 iterations run end to end through the
  public op2 API from pinned host arrays: declaring the problem uploads maps
  and Dats (H2D inside the timed region), every iteration issues its 9
  par_loops from Python and reads rms back (D2H), and the final solution is
  read back.
* ``roofline``: res_calc, the largest loop: the mean duration of its two
  launches per step, read from CUDA event nodes around them in the recorded
  step, replayed as in the timed region (L2 flushed before each step).
* ``cpu_baseline``: the oracle's restated OpenMP backend (pyop2/openmp.py) on
  all host cores (a bounded sample of the same mesh), beside the sequential
  oracle (pyop2/sequential.py) on one core over the end-to-end run's 100
  iterations and over the P2 1024 x 1024 FP64 assembly.
* ``parity``: the end-to-end run's final q and its 100 rms values against the
  sequential oracle's (max relative error; the bar is 1e-12).
* ``mat_assembly`` / ``batching`` / ``serving``: summaries of the other
  legs (Mat assembly nnz/s and fraction of HBM peak with the P2 errors
  against the sequential oracle; batched and served requests/s against the
  plain per-loop drop-in).  The full figures go to stderr (``bench
  detail:``) and to ``--detail FILE``.

``--impl reference`` times the reference's CPU implementation of the path
(the restated OpenMP backend; the Python 2 reference itself cannot run here)
on the same workload and prints its line.

Multi-GPU: replicas only (each rank runs its own mesh on its own GPU, no data
exchange); torch.distributed supplies the barrier and the max over ranks.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

NX, NY = 1200, 600
SEED = 0


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class _Dist(object):
    """Barrier and max-over-ranks through torch.distributed (N > 1 only)."""

    def __init__(self, ws, rank, local, backend):
        self.ws, self.rank = ws, rank
        self.pg = None
        if ws > 1:
            import datetime
            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(local)
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
            self.dist, self.torch, self.backend = dist, torch, backend

    def barrier(self):
        if self.ws > 1:
            self.dist.barrier()

    def max(self, v):
        if self.ws == 1:
            return v
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor([float(v)], dtype=self.torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.ws > 1:
            self.dist.destroy_process_group()


class ClockSampler(object):
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _set_mesh(nx, ny):
    global NX, NY
    NX, NY = nx, ny


def _bytes():
    from pyop2_b200.workloads.meshes import airfoil_grid
    from pyop2_b200.workloads import airfoil
    g = airfoil_grid(NX, NY, SEED, permute=False)
    return airfoil.bytes_per_iteration(g.ncells, g.nnodes, g.nedges, g.nbedges)


def _traffic_from_profile():
    """DRAM bytes (read + write) per res_calc launch (staged form, the
    default) from the committed ncu summary of that kernel, if one exists."""
    p = os.path.join(HERE, "profiles", "res_calc_staged_airfoil_1200x600.md")
    try:
        with open(p) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return int(line.split(":")[1])
    except (OSError, ValueError):
        pass
    return None


def _peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


# ----------------------------------------------------------------- CPU leg
E2E_ITERS = 100   # the airfoil configuration's iteration count


def workload_config(ws):
    """The workload both arms run (rank-independent description)."""
    return {"workload": "airfoil %dx%d permuted FP64, 9 par_loops/step" % (NX, NY),
            "bytes_per_step": _bytes()["iteration"],
            "parallelism": "replicas" if ws > 1 else "single"}


def cpu_airfoil(seconds=20.0, max_iters=50, threads=None, warmup=1):
    """Restated OpenMP backend on the full mesh: iterations until ~seconds of
    element-loop time; returns (GB/s, iterations, threads, loop seconds)."""
    from oracle import seq
    from pyop2_b200.workloads import airfoil
    from pyop2_b200.workloads.meshes import airfoil_grid
    nthreads = threads or os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(nthreads)
    seq._CONSTS.clear()
    grid = airfoil_grid(NX, NY, SEED)
    A = airfoil.build(seq, NX, NY, SEED, grid=grid)
    loop_time = [0.0]
    orig = seq.par_loop

    def timed(*a, **k):
        return orig(*a, openmp=True, part_size=1024, timer=lambda dt: loop_time.__setitem__(0, loop_time[0] + dt), **k)
    seq.par_loop = timed
    try:
        for _ in range(max(1, warmup)):  # compile + plan, not timed
            airfoil.iteration(seq, A)
        loop_time[0] = 0.0
        iters = 0
        while iters < max_iters and (loop_time[0] < seconds or iters == 0):
            airfoil.iteration(seq, A)
            iters += 1
    finally:
        seq.par_loop = orig
        seq._CONSTS.clear()
    bpi = _bytes()["iteration"]
    return bpi * iters / loop_time[0] / 1e9, iters, nthreads, loop_time[0]


def cpu_sequential_airfoil(iters):
    """The sequential oracle (one host thread) over ``iters`` outer
    iterations of the full mesh from the initial state: element-loop time
    summed (code generation excluded).  Returns (GB/s, loop seconds, final q,
    per-iteration rms sums): the timed run doubles as the checker of the
    GPU's end-to-end run of the same iterations."""
    from oracle import seq
    from pyop2_b200.workloads import airfoil
    from pyop2_b200.workloads.meshes import airfoil_grid
    seq._CONSTS.clear()
    grid = airfoil_grid(NX, NY, SEED)
    A = airfoil.build(seq, NX, NY, SEED, grid=grid)
    loop_time = [0.0]
    orig = seq.par_loop

    def timed(*a, **k):
        return orig(*a, timer=lambda dt: loop_time.__setitem__(0, loop_time[0] + dt), **k)
    seq.par_loop = timed
    rms = []
    try:
        for _ in range(iters):
            rms.append(float(airfoil.iteration(seq, A).data[0]))
    finally:
        seq.par_loop = orig
        seq._CONSTS.clear()
    return (_bytes()["iteration"] * iters / loop_time[0] / 1e9, loop_time[0], A.p_q.data.copy(),
            np.array(rms))


def cpu_sequential_p2(n=1024):
    """The sequential oracle's FP64 P2 stiffness + mass assembly on the
    n x n grid, timed (element loops only).  Returns (nnz per second over
    both Mats, seconds, K values, M values, nnz): the values are the checker
    of the GPU's FP64 and precision-form assemblies."""
    from oracle import seq
    from pyop2_b200.workloads import fem
    O = fem.build_p2(seq, n, seed=0)
    t = [0.0]
    orig = seq.par_loop

    def timed(*a, **k):
        return orig(*a, timer=lambda dt: t.__setitem__(0, t[0] + dt), **k)
    seq.par_loop = timed
    try:
        fem.assemble_p2(seq, O)
    finally:
        seq.par_loop = orig
    nz = O.sparsity.nz
    return 2 * nz / t[0], t[0], O.K.array, O.M.array, nz


def run_reference(args, ws, rank, local):
    """--impl reference: the reference's CPU path (restated OpenMP backend)."""
    if rank != 0:
        return 0
    t0 = time.time()
    steps = max(1, args.steps)
    # bounded: about 60 s of element-loop work in total
    gbs, iters, nthreads, secs = cpu_airfoil(seconds=min(60.0, 2.0 * steps), max_iters=steps,
                                             warmup=args.warmup)
    line = {"metric": "par_loop achieved HBM GB/s (airfoil chain)", "value": round(gbs, 3),
            "unit": "GB/s", "n_gpus": ws, "steps": iters, "warmup": args.warmup,
            "ms_per_step": round(1e3 * secs / iters, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": dict(workload_config(ws),
                           timing="host wall clock around each element loop, rank 0 only"),
            "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": nthreads,
                             "kind": "port",
                             "sample": "%d airfoil iterations of the %dx%d mesh, restated "
                                       "OpenMP backend (oracle), element loops timed"
                                       % (iters, NX, NY)},
            "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_s": round(time.time() - t0, 1)}
    print(json.dumps(line))
    return 0


# ----------------------------------------------------------------- GPU leg
def run_gpu(args, ws, rank, local):
    from pyop2_b200 import op2, b200, base
    from pyop2_b200.workloads import airfoil
    from pyop2_b200.workloads.meshes import airfoil_grid
    d = _Dist(ws, rank, local, "nccl" if ws > 1 else "gloo")
    opts = {}
    if args.part_size:
        opts["partition_size"] = args.part_size
    if args.block_size:
        opts["block_size"] = args.block_size
    if args.l2_fetch >= 0:
        opts["l2_fetch_granularity"] = args.l2_fetch
    if args.min_blocks >= 0:
        opts["min_blocks_per_sm"] = args.min_blocks
    if args.inc_mode:
        opts["inc_mode"] = args.inc_mode
    if args.staged_block_size:
        opts["staged_block_size"] = args.staged_block_size
    if args.region_size:
        opts["region_size"] = args.region_size
    op2.init(backend="b200", device=local, **opts)
    if args.assembly_only:
        # the Mat assembly legs alone (profiling their kernels); not a bench line
        if rank == 0:
            print(json.dumps({"mat_assembly": bench_assembly(op2, b200)}))
        d.close()
        return 0
    if args.batching_only:
        if rank == 0:
            print(json.dumps({"batching": bench_batching(op2, b200, args.batch_meshes or 4096)}))
        d.close()
        return 0
    if args.solve_only:
        if rank == 0:
            print(json.dumps({"solve": bench_solve(op2, b200)}))
        d.close()
        return 0
    if args.serving_only:
        if rank == 0:
            print(json.dumps({"serving": bench_serving(op2, b200, args.serve_requests or 3000,
                                                       args.serve_rate)}))
        d.close()
        return 0
    bytes_ = _bytes()
    bpi = bytes_["iteration"]
    grid = airfoil_grid(NX, NY, SEED, permute=not args.no_permute)

    # ---------------- device-resident throughput (graph replay)
    A = airfoil.build(op2, NX, NY, SEED, grid=grid)
    rms = op2.Global(1, 0.0, np.float64, "rms")

    def step():
        rms.zero()
        airfoil.iteration(op2, A, rms)

    for _ in range(max(1, args.warmup)):
        step()
    b200.synchronize()
    with b200.capture() as graph:
        step()
    for _ in range(args.warmup):
        b200.l2_flush()
        graph.launch()
    b200.synchronize()
    launches = sum(bl.plan.ncolors if bl.indirect else 1 for bl in _step_loops(A))
    ev = [(b200.Event(), b200.Event()) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    sampler.start()
    # keep the GPU busy ~1 s so the 200 ms clock samples see it under load;
    # the timed steps below follow without a pause
    soak_end = time.time() + 1.0
    while time.time() < soak_end:
        for _ in range(20):
            b200.l2_flush()
            graph.launch()
        b200.synchronize()
    d.barrier()
    b200.synchronize()
    for k in range(args.steps):
        b200.l2_flush()
        ev[k][0].record()
        graph.launch()
        ev[k][1].record()
    b200.synchronize()
    d.barrier()
    clocks = sampler.stop()
    step_ms = [a.elapsed_ms(b) for a, b in ev]
    total_ms = d.max(sum(step_ms))
    value = ws * bpi * args.steps / (total_ms * 1e-3) / 1e9
    final_rms = float(np.sqrt(rms.data[0] / grid.ncells))

    # ---------------- roofline: res_calc's launches inside the step.  The
    # step is recorded once more with a CUDA event pair around each of its
    # two res_calc launches (event nodes of the graph, on the op2 stream)
    # and replayed as in the timed region (L2 flush, then the step); each
    # replay's two res_calc durations are read back.  A second recording
    # marks every loop the same way for the per-loop breakdown (each event
    # node adds a little to the loop it follows, so short loops read high).
    def marked_step(names):
        marks = []

        def marked(name, fn):
            if name not in names:
                fn()
                return
            e0, e1 = b200.Event(), b200.Event()
            e0.record(node=True)
            fn()
            e1.record(node=True)
            marks.append((name, e0, e1))

        def run():
            rms.zero()
            marked("save_soln", lambda: airfoil.save_soln(op2, A))
            for k in range(2):
                marked("adt_calc", lambda: airfoil.adt_calc(op2, A))
                marked("res_calc", lambda: airfoil.res_calc(op2, A))
                marked("bres_calc", lambda: airfoil.bres_calc(op2, A))
                marked("update", lambda: airfoil.update(op2, A, rms))

        with b200.capture() as gm:
            run()
        for _ in range(3):
            b200.l2_flush()
            gm.launch()
        out = {}
        for _ in range(max(10, min(args.steps, 50))):
            b200.l2_flush()
            gm.launch()
            b200.synchronize()
            for name, a, b in marks:
                out.setdefault(name, []).append(a.elapsed_ms(b))
        gm.close()
        return out

    res_in_step = marked_step(("res_calc",))["res_calc"]
    res_avg = statistics.mean(res_in_step)
    in_step = marked_step(("save_soln", "adt_calc", "res_calc", "bres_calc", "update"))

    # ---------------- per-loop breakdown: each loop's mean time inside the
    # replayed step (above), and beside it ("alone_ms") the loop replayed
    # from its own CUDA graph right after an L2 flush, where the events also
    # hold the graph launch.
    loop_fns = (("save_soln", lambda: airfoil.save_soln(op2, A)),
                ("adt_calc", lambda: airfoil.adt_calc(op2, A)),
                ("res_calc", lambda: airfoil.res_calc(op2, A)),
                ("bres_calc", lambda: airfoil.bres_calc(op2, A)),
                ("update", lambda: airfoil.update(op2, A, rms)))
    breakdown = {}
    res_alone = None
    for name, fn in loop_fns:
        with b200.capture() as g1:
            fn()
        reps = 20
        for _ in range(3):
            g1.launch()
        ts = []
        for _ in range(reps):
            b200.l2_flush()
            e0 = b200.Event().record()
            g1.launch()
            e1 = b200.Event().record()
            e1.synchronize()
            ts.append(e0.elapsed_ms(e1))
        g1.close()
        ms = statistics.median(ts)
        if name == "res_calc":
            res_alone = statistics.mean(ts)
        step_ms = statistics.mean(in_step[name])
        breakdown[name] = {"ms": round(step_ms, 4),
                           "GB/s": round(bytes_[name] / (step_ms * 1e-3) / 1e9, 1),
                           "alone_ms": round(ms, 4)}
    # the form res_calc ran in (before other legs bind loops of that kernel)
    res_form = _RES_FORM.get(_loop_mode("res_calc"), "all colour launches")
    # one-off cost of the staged form: building res_calc's locality partition
    partition_ms = None
    staged = [bl for bl in b200.ParLoop._bound_cache.values()
              if bl.spec.kernel_name == "res_calc" and bl.spec.mode == "staged"]
    if staged:
        rp = staged[-1].region_plan
        b200.synchronize()
        t0 = time.perf_counter()
        b200.RegionPlan(rp.set_size, rp.part_size, rp.region_size, rp._keep[0], rp._keep[1:],
                        rp.stage_inc)
        b200.synchronize()
        partition_ms = round((time.perf_counter() - t0) * 1e3, 3)
    res_bytes = bytes_["res_calc"]
    peak, peak_kind = _peaks()
    achieved = res_bytes / (res_avg * 1e-3) / 1e9
    # the committed capture covers the default workload in the default INC mode
    default_run = ((NX, NY) == (1200, 600) and op2_cfg_inc_mode() == "staged"
                   and not args.no_permute and not args.block_size and not args.part_size)
    traffic = _traffic_from_profile() if default_run else None

    e2e_val = e2e_ms = h2d = d2h = q_out = None
    e2e_iters = E2E_ITERS
    rms_hist = [0.0]
    if not args.no_e2e:
        # ---------------- end to end through the public API: the
        # configuration's 100 iterations from the initial state, the problem
        # declared from pinned host arrays inside the timed region
        for c in list(base.Const._defs):
            c.remove_from_namespace()
        del graph

        def pin(src):
            dst = b200.pinned_empty(src.shape, src.dtype)
            dst[...] = src
            return dst

        class PinnedGrid(object):
            pass
        pg = PinnedGrid()
        for k, v in vars(grid).items():
            setattr(pg, k, pin(v) if isinstance(v, np.ndarray) else v)
        q0 = airfoil.initial_q(grid.ncells, SEED)
        host = {"q": pin(q0), "qold": pin(q0), "adt": pin(np.zeros(grid.ncells)),
                "res": pin(np.zeros((grid.ncells, 4)))}
        d.barrier()
        b200.synchronize()
        t0 = b200.Event().record()
        E = airfoil.build(op2, NX, NY, SEED, grid=pg, q0=host["q"], qold0=host["qold"],
                          zeros=(host["adt"], host["res"]))
        rms_hist = []
        for _ in range(e2e_iters):
            r = airfoil.iteration(op2, E)
            rms_hist.append(float(r.data[0]))
        q_out = E.p_q.data_ro
        t1 = b200.Event().record()
        t1.synchronize()
        e2e_ms = d.max(t0.elapsed_ms(t1))
        e2e_val = ws * bpi * e2e_iters / (e2e_ms * 1e-3) / 1e9
        h2d = (sum(getattr(pg, k).nbytes for k in ("pedge", "pecell", "pbedge", "pbecell", "pcell",
                                                   "p_bound", "x")) +
               sum(v.nbytes for v in host.values()) + e2e_iters * 2 * 8)
        d2h = e2e_iters * 2 * 8 + q_out.nbytes
        q_out = np.array(q_out)

    # ---------------- CPU baseline (rank 0 at N=1): the restated OpenMP
    # backend on all host cores, the sequential oracle on one core over the
    # same 100 iterations as the end-to-end run (its results are the parity
    # checker of that run), and the sequential FP64 P2 assembly (the checker
    # of the GPU's P2 assemblies)
    cpu = parity = p2_ref = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        gbs, iters, nthreads, secs = cpu_airfoil(seconds=args.cpu_seconds, max_iters=50)
        seq_iters = e2e_iters if q_out is not None else 3
        s_gbs, s_secs, s_q, s_rms = cpu_sequential_airfoil(seq_iters)
        p2_nnz_s, p2_s, p2_k, p2_m, p2_nz = cpu_sequential_p2()
        p2_ref = (p2_k, p2_m)
        cpu = {"value": round(gbs, 3), "unit": "GB/s", "cores": nthreads, "kind": "port",
               "sample": "OpenMP port, %d iters" % iters,
               "sequential": {"value": round(s_gbs, 3), "cores": 1, "iters": seq_iters,
                              "p2_Mnnz_s": round(p2_nnz_s / 1e6, 1)}}
        if q_out is not None:
            rel = np.abs(np.array(rms_hist) - s_rms) / np.maximum(np.abs(s_rms), 1e-300)
            parity = {"iters": seq_iters,
                      "max_rel_q": float(np.abs(q_out - s_q).max() / np.abs(s_q).max()),
                      "max_rel_rms": float(rel.max()), "tol": 1e-12}
        del s_q

    # the other legs are single-GPU figures: rank 0 runs them, the other
    # replicas stop here (no collective follows)
    assembly = batching = serving = solve = None
    if rank == 0:
        if not args.no_assembly:
            assembly = bench_assembly(op2, b200, p2_ref=p2_ref)
        if args.batch_meshes > 0:
            batching = bench_batching(op2, b200, args.batch_meshes)
        if args.serve_requests > 0:
            serving = bench_serving(op2, b200, args.serve_requests, args.serve_rate)
        if args.solve:
            solve = bench_solve(op2, b200)
    del p2_ref

    line = {
        "metric": "par_loop achieved HBM GB/s (airfoil chain)",
        "value": round(value, 2), "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": dict(workload_config(ws), l2="256 MB flush before each step"),
        "gpu_launches": launches * args.steps,
        "roofline": {"kernel": "res_calc", "bound": "hbm",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic},
        "e2e": None if e2e_val is None else {
            "value": round(e2e_val, 2), "unit": "GB/s", "h2d_bytes_per_step": int(h2d // e2e_iters),
            "d2h_bytes_per_step": int(d2h // e2e_iters), "iters": e2e_iters},
        "clocks": {k: clocks.get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons")},
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if parity is not None:
        line["parity"] = {k: (float("%.3g" % v) if isinstance(v, float) else v)
                          for k, v in parity.items()}
    if assembly is not None:
        line["mat_assembly"] = assembly["summary"]
    if batching is not None:
        line["batching"] = batching["summary"]
    if serving is not None:
        line["serving"] = serving["summary"]
    detail = {"peak_kind": peak_kind, "res_calc_form": res_form, "res_calc_avg_ms": round(res_avg, 4),
              "res_calc_alone_ms": round(res_alone, 4),
              "res_calc_algorithmic_bytes": res_bytes, "loops": breakdown,
              "res_calc_partition_build_ms": partition_ms, "inc_mode": op2_cfg_inc_mode(),
              "clocks": clocks, "e2e_ms": e2e_ms, "cpu_baseline": cpu, "parity": parity,
              "rms_graph_final": final_rms,
              "mat_assembly": assembly, "batching": batching, "serving": serving,
              "solve": solve}
    if rank == 0:
        # the full figures go to stderr (and to --detail), the one bench line
        # to stdout
        text = json.dumps(detail, default=str)
        sys.stderr.write("bench detail: " + text + "\n")
        if args.detail:
            with open(args.detail, "w") as f:
                f.write(text + "\n")
        print(json.dumps(line))
    d.close()
    return 0


_RES_FORM = {"staged": "one launch over the locality partition", "atomic": "one atomic launch",
             "gather": "thread per cell over its incidence",
             "lma": "contribution launch + per-target reduction"}


def _loop_mode(kernel_name):
    """The form (staged / atomic / plan ...) the backend chose for the most
    recently bound loop of a kernel."""
    from pyop2_b200 import b200
    mode = None
    for bl in b200.ParLoop._bound_cache.values():
        if bl.spec.kernel_name == kernel_name:
            mode = bl.spec.mode
    return mode


def op2_cfg_inc_mode():
    from pyop2_b200 import configuration as cfg
    return cfg.cfg['inc_mode']


def _timed(fn, reps, b200, flush=True, graph=False, overlap=False):
    """Median device time (ms) of fn() over reps runs, L2 flushed before each.
    ``graph``: fn's launches recorded once as a CUDA graph (after one eager
    run that binds its loops) and the graph replayed, so the events see the
    device work and not the host's issue rate; ``overlap``: recorded as an
    overlapped graph (loops that share no written data run side by side)."""
    g = None
    if graph:
        fn()
        b200.synchronize()
        with b200.capture(overlap=overlap) as g:
            fn()
        run = g.launch
    else:
        run = fn
    ts = []
    for _ in range(reps):
        if flush:
            b200.l2_flush()
        e0 = b200.Event().record()
        run()
        e1 = b200.Event().record()
        e1.synchronize()
        ts.append(e0.elapsed_ms(e1))
    if g is not None:
        g.close()
    return statistics.median(ts)


def bench_batching(op2, b200, nmesh, reps=5, seed=0):
    """Batching form: nmesh uneven P1 meshes (elements log-uniform in
    [2^8, 2^16], random aspect ratio, permuted numbering), each with mass and
    stiffness Mat assembly and an RHS INC loop.

    * batched: the three loops of all meshes as three tuned BatchLoops (one
      persistent launch each) recorded in one CUDA graph, replayed after an
      L2 flush, CUDA events around the replay;
    * plain: the same 3 x nmesh loops issued one by one through
      op2.par_loop (objects already resident, stubs compiled), CUDA events
      around the whole sequence (the device timeline, host gaps included).
    Requests = meshes.  Parity: the batched Mats and RHS of sample meshes
    against the plain path's."""
    from pyop2_b200 import autotune
    from pyop2_b200.workloads import batching
    t0 = time.time()
    shapes = batching.mesh_shapes(nmesh, seed)
    probs = batching.build(op2, shapes, seed)
    mass, stiff, rhs = batching.instances(op2, probs)
    setup_s = time.time() - t0
    elements = sum(P.n_elem for P in probs)
    nbytes = sum(batching.bytes_per_mesh(P) for P in probs)
    nnz = sum(int(P.sparsity.nz) for P in probs)
    t1 = time.time()
    loops, tuned = [], {}
    for name, insts in (("mass", mass), ("stiffness", stiff), ("rhs", rhs)):
        best, times = autotune.tune(insts, reps=3)
        tuned[name] = {"best": best, "candidates_ms": times}
        loops.append(autotune.build(insts, best))
    tune_s = time.time() - t1
    for bl in loops:
        bl.launch()
    b200.synchronize()
    with b200.capture() as g:
        for bl in loops:
            bl.launch(sync_host=False)
    for _ in range(3):
        g.launch()
    ts = []
    for _ in range(reps):
        b200.l2_flush()
        e0 = b200.Event().record()
        g.launch()
        e1 = b200.Event().record()
        e1.synchronize()
        ts.append(e0.elapsed_ms(e1))
    batched_ms = statistics.median(ts)
    # plain per-loop form: warm (stubs, bound loops), then timed
    for P in probs:
        batching.plain(op2, P)
    b200.synchronize()
    pts = []
    for _ in range(2):
        b200.l2_flush()
        e0 = b200.Event().record()
        for P in probs:
            batching.plain(op2, P)
        e1 = b200.Event().record()
        e1.synchronize()
        pts.append(e0.elapsed_ms(e1))
    plain_ms = min(pts)
    # parity on sample meshes: zero, batched graph once, keep; zero, plain
    sample = sorted({0, nmesh // 2, nmesh - 1, int(np.argmax([P.n_elem for P in probs]))})
    for P in probs:
        P.mat.zero(); P.stiff.zero(); P.b.zero()
    g.launch()
    got = {i: (probs[i].mat.array.copy(), probs[i].stiff.array.copy(), probs[i].b.data_ro.copy())
           for i in sample}
    err = 0.0
    for i in sample:
        P = probs[i]
        P.mat.zero(); P.stiff.zero(); P.b.zero()
        batching.plain(op2, P)
        for a, b in zip(got[i], (P.mat.array, P.stiff.array, P.b.data_ro)):
            err = max(err, float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)))
    g.close()
    peak, _ = _peaks()
    summary = {"req_per_s_ratio": round(plain_ms / batched_ms, 1),
               "frac": round(nbytes / (batched_ms * 1e-3) / 1e9 / peak, 3),
               "err_vs_plain": float("%.3g" % err)}
    return {"summary": summary, "meshes": nmesh, "elements": elements, "nnz_per_mat": nnz,
            "loops_per_mesh": 3, "algorithmic_bytes": nbytes,
            "batched_ms": round(batched_ms, 4),
            "batched_req_per_s": round(nmesh / (batched_ms * 1e-3), 1),
            "batched_GBps": round(nbytes / (batched_ms * 1e-3) / 1e9, 1),
            "batched_launches": sum(bl.launches for bl in loops),
            "plain_ms": round(plain_ms, 2),
            "plain_req_per_s": round(nmesh / (plain_ms * 1e-3), 1),
            "plain_launches": 3 * nmesh,
            "speedup_req_per_s": round(plain_ms / batched_ms, 1),
            "max_rel_err_vs_plain": err, "parity_sample_meshes": sample,
            "autotune": tuned, "setup_s": round(setup_s, 1), "tune_s": round(tune_s, 1)}


def bench_serving(op2, b200, nreq, rate, seed=0, n_p1=16, n_quad=16):
    """Serving form: a Poisson trace (``rate`` requests/s, ``nreq`` requests)
    mixing P1 assembly requests (meshes of 10^3..10^6 triangles) and
    10-iteration airfoil-style chains (10^4..10^6 cells) on a pool of
    resident meshes, 120 GB HBM admission budget.  The continuous-batching
    engine and the plain per-request drop-in serve the same trace in real
    time (latency = result on the host - arrival); then both serve it with
    every request released at once (capacity).  Parity: every request's
    results, engine against plain."""
    from pyop2_b200 import autotune, base, serve
    from pyop2_b200.workloads import serving
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    consts = serving.declare_consts(op2)
    pool = serving.mesh_pool(n_p1, n_quad, seed)
    store = serve.MeshStore(budget=120e9)
    serving.register(store, op2, pool, seed)
    t0 = time.time()
    for mid in sorted(pool):
        store.load(mid)
    resident_s = time.time() - t0
    jobs = serving.trace(nreq, rate, pool, seed)
    warm = serving.trace(64, 1e6, pool, seed + 1)
    serve.Engine(store).run(serving.clone_trace(warm, False), realtime=False)
    # the drop-in's first request on a mesh builds the mesh's plans; one
    # untimed request per mesh keeps those builds out of the timed runs
    first = {}
    for j in serving.clone_trace(jobs, False):
        first.setdefault(j.mesh_id, j)
    serve.PlainServer(op2, store).run(list(first.values()), realtime=False)
    t1 = time.time()
    configs = {}
    kinds = {"p1": (("p1_src", "t_src"), ("p1_mass", "t_mass"), ("p1_rhs", "t_rhs")),
             "quad": (("q_init", "t_init"), ("save_soln", "t_save"), ("adt_calc", "t_adt"),
                      ("res_calc", "t_res"), ("bres_calc", "t_bres"), ("update", "t_update"))}
    for mkind, loops in kinds.items():
        meshes = [store.get(m) for m in sorted(pool) if pool[m][0] == mkind]
        for name, attr in loops:
            # patched request instances run the atomic batched form
            configs[name], _ = autotune.tune([getattr(m, attr) for m in meshes], reps=2,
                                             candidates=autotune.DEFAULT_CANDIDATES)
    tune_s = time.time() - t1
    b200.synchronize()
    # results reach the consumer as views of pinned host memory; every 16th
    # request's results are kept for the parity check
    kept = {"engine": {}, "plain": {}}

    def consumer(which):
        def take(job, views):
            if job.rid % 16 == 0:
                kept[which][job.rid] = {k: np.array(v, dtype=np.float64).reshape(-1)
                                        for k, v in views.items()}
        return take

    # one untimed pass over the trace fills the pinned-buffer pool the timed
    # runs reuse (page-locking host memory is a one-off cost)
    serve.Engine(store, configs=configs, consumer=lambda j, v: None).run(
        serving.clone_trace(jobs, False), realtime=False)
    cap_e = serve.Engine(store, configs=configs, consumer=lambda j, v: None, timing=True)
    s_cap_eng = serve.summary(cap_e.run(serving.clone_trace(jobs, False), realtime=False), 0.0)
    s_cap_eng["gpu_busy_fraction"] = round(cap_e.gpu_busy_ms() / (s_cap_eng["span_s"] * 1e3), 3)
    eng = serve.Engine(store, configs=configs, consumer=consumer("engine"))
    done = eng.run(serving.clone_trace(jobs), realtime=True)
    s_eng = serve.summary(done)
    s_eng.update(steps=eng.steps, launches=eng.launches,
                 mean_batch=round(float(np.mean(eng.batch_sizes)), 2),
                 peak_hbm_gb=round(eng.peak_used / 1e9, 3))
    plain = serve.PlainServer(op2, store, consumer=consumer("plain")).run(
        serving.clone_trace(jobs), realtime=True)
    s_plain = serve.summary(plain)
    sub = jobs[:max(1, len(jobs) // 4)]
    s_cap_plain = serve.summary(serve.PlainServer(op2, store, consumer=lambda j, v: None).run(
        serving.clone_trace(sub, False), realtime=False), 0.0)
    err = {"p1": 0.0, "quad": 0.0}
    kinds_by_id = {j.rid: j.kind for j in jobs}
    for rid, pres in kept["plain"].items():
        eres = kept["engine"][rid]
        for k in pres:
            a, b = eres[k], pres[k]
            den = max(float(np.abs(b).max()), 1e-300)
            err[kinds_by_id[rid]] = max(err[kinds_by_id[rid]], float(np.abs(a - b).max()) / den)
    del consts
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    ratio = round(s_eng["req_per_s"] / s_plain["req_per_s"], 2)
    summary = {"req_per_s_ratio": ratio, "req_per_s": s_eng["req_per_s"],
               "p50_ms": s_eng["p50_ms"], "p99_ms": s_eng["p99_ms"],
               "plain_p99_ms": round(s_plain["p99_ms"], 1),
               "err_vs_plain": float("%.3g" % max(err.values()))}
    return {"summary": summary,
            "trace": {"requests": nreq, "rate_per_s": rate, "p1_meshes": n_p1,
                      "quad_meshes": n_quad, "iters_per_chain": 10, "hbm_budget_gb": 120,
                      "p1_triangles": [int(2 * v[1] * v[2]) for v in pool.values() if v[0] == "p1"],
                      "quad_cells": [int(v[1] * v[2]) for v in pool.values() if v[0] == "quad"]},
            "engine": s_eng, "plain": s_plain,
            "req_per_s_ratio": round(s_eng["req_per_s"] / s_plain["req_per_s"], 2),
            "p99_ratio_plain_over_engine": round(s_plain["p99_ms"] / s_eng["p99_ms"], 2),
            "capacity_engine": s_cap_eng, "capacity_plain": s_cap_plain,
            "capacity_ratio": round(s_cap_eng["req_per_s"] / s_cap_plain["req_per_s"], 2),
            "max_rel_err_engine_vs_plain": err, "autotuned": configs,
            "resident_setup_s": round(resident_s, 1), "tune_s": round(tune_s, 1)}


def bench_solve(op2, b200, n=1024, reps=20):
    """Linear solve on an assembled Mat: the P2 mass matrix of the n x n
    grid (48.25 M nonzeros at n = 1024), Jacobi-preconditioned CG from x = 0
    to rtol 1e-8 (op2.solve), and the CSR SpMV alone.  SpMV algorithmic
    bytes: values and column indices (12 B per nonzero), row pointers, x
    read once, y written once.  The residual of the solution is checked with
    scipy's CSR product on the host."""
    import scipy.sparse
    from pyop2_b200._lib import call
    from pyop2_b200.workloads import fem
    P = fem.build_p2(op2, n, seed=0)
    fem.assemble_p2(op2, P)
    b200.synchronize()
    sp = P.sparsity
    rows, nnz = sp._lsize, int(sp.nz)
    rng = np.random.default_rng(11)
    rhs = rng.standard_normal(rows)
    b = op2.Dat(P.dofs, rhs.copy(), np.float64, "b")   # a Dat reshapes the array it keeps
    x = op2.Dat(P.dofs, np.zeros(rows), np.float64, "x")
    solver = b200.Solver(relative_tolerance=1e-8)
    solver.solve(P.M, x, b)                       # warm-up (device copies)
    ts = []
    for _ in range(3):
        b200.l2_flush()
        e0 = b200.Event().record()
        solver.solve(P.M, x, b)
        e1 = b200.Event().record()
        e1.synchronize()
        ts.append(e0.elapsed_ms(e1))
    solve_ms = statistics.median(ts)
    host_m = scipy.sparse.csr_matrix((P.M.array, sp.colidx, sp.rowptr), shape=(rows, rows))
    resid = float(np.abs(host_m @ x.data_ro.ravel() - rhs).max() / np.abs(rhs).max())
    vals = P.M._device_values().ptr
    xd, yd = b._device.ptr, b200.DeviceBuffer(rows * 8)

    by_group = {}
    for group in (0, 1, 2, 4, 8, 16):   # 0: the library's choice from the mean row length
        def spmv(group=group):
            call("op2b_csr_spmv", sp._d_rowptr, sp._d_colidx, vals, rows, nnz, xd, yd.ptr, 1.0,
                 0.0, group, 0)
        by_group[group] = _timed(spmv, reps, b200)
    spmv_ms = by_group[0]
    spmv_bytes = nnz * 12 + (rows + 1) * 4 + rows * 16
    peak, _ = _peaks()
    return {"matrix": "P2 mass %dx%d" % (n, n), "rows": rows, "nnz": nnz,
            "solver": "cg + jacobi, rtol 1e-8, x0 = 0", "iterations": solver.iterations,
            "reason": solver.reason, "solve_ms": round(solve_ms, 3),
            "ms_per_iteration": round(solve_ms / max(1, solver.iterations), 4),
            "max_rel_residual": resid,
            "spmv_ms": round(spmv_ms, 4), "spmv_GBps": round(spmv_bytes / (spmv_ms * 1e-3) / 1e9, 1),
            "spmv_frac_of_measured_peak": round(spmv_bytes / (spmv_ms * 1e-3) / 1e9 / peak, 3),
            "spmv_algorithmic_bytes": spmv_bytes,
            "spmv_ms_by_lanes_per_row": {str(k): round(v, 4) for k, v in by_group.items()}}


def bench_assembly(op2, b200, reps=5, p2_ref=None):
    """Mat assembly legs (each timed as a CUDA graph replay after an L2
    flush).

    * P1 256 x 256 mass + RHS (FP64), the drop-in's default forms.
    * P2 1024 x 1024 stiffness + mass on one Sparsity: FP64 (default atomic
      form), FP64 in the two-phase form (adds in the sequential order), and
      the precision form (FP32 element math and geometry differences from
      FP64 coordinates, FP64 Kahan-compensated two-phase accumulation).

    Bytes: P1 per loop (map, coordinates, values read and written, CSR);
    P2 K+M on one Sparsity (map and coordinates once, CSR once, both Mats'
    values read and written: 1.871 GB).  ``p2_ref`` = the sequential
    oracle's FP64 (K, M) values (from the CPU-baseline leg): each P2 form's
    max relative error per Mat is stated against them."""
    from pyop2_b200 import base
    from pyop2_b200 import configuration as cfg
    from pyop2_b200.workloads import fem
    peak, _ = _peaks()
    out = {}
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    # ---- P1
    P = fem.build_p1(op2, 256)
    t0 = time.time()
    nz = P.sparsity.nz
    sp_s = time.time() - t0
    fem.assemble_p1(op2, P)
    b200.synchronize()

    def mass():
        op2.par_loop(P.k_mass, P.elements(3, 3),
                     P.mat((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC),
                     P.coords(P.elem_vnode, op2.READ))

    def rhs():
        op2.par_loop(P.k_rhs, P.elements(3), P.b(P.elem_node[op2.i[0]], op2.INC),
                     P.coords(P.elem_vnode, op2.READ), P.f(P.elem_node, op2.READ))

    def both():
        mass()
        rhs()
    ms_m = _timed(mass, reps, b200, graph=True)
    ms_r = _timed(rhs, reps, b200, graph=True)
    ms_chain = _timed(both, reps, b200, graph=True)
    # mass and RHS share no written data: the overlapped graph runs them
    # side by side (at 131,072 elements each launch alone leaves most of the
    # GPU idle)
    ms_b = _timed(both, reps, b200, graph=True, overlap=True)
    bm = fem.assembly_bytes(P.n_elem, 3, P.n_nodes, nz)
    br = fem.rhs_bytes(P.n_elem, P.n_nodes)
    out["p1_256"] = {"nnz": nz, "elements": P.n_elem, "sparsity_build_s": round(sp_s, 4),
                     "mass_ms": round(ms_m, 4), "mass_nnz_per_s": round(nz / (ms_m * 1e-3), 1),
                     "mass_GBps": round(bm / (ms_m * 1e-3) / 1e9, 1),
                     "rhs_ms": round(ms_r, 4), "rhs_GBps": round(br / (ms_r * 1e-3) / 1e9, 1),
                     "mass_rhs_ms": round(ms_b, 4), "mass_rhs_chain_ms": round(ms_chain, 4),
                     "mass_rhs_GBps": round((bm + br) / (ms_b * 1e-3) / 1e9, 1),
                     "mass_mode": _loop_mode(P.k_mass.name), "rhs_mode": _loop_mode(P.k_rhs.name)}
    del P
    # ---- P2: the FP64 drop-in, its two-phase form, the precision form
    res = {}
    inc0 = cfg.cfg['inc_mode']
    variants = (("f64", None, False), ("f64", "lma", False), ("f32", "lma", False),
                ("f32", "lma", True))
    for prec, mode, kahan in variants:
        tag = prec + ("_lma" if mode == "lma" else "") + ("_kahan" if kahan else "")
        cfg.configure(kahan=kahan, inc_mode=mode or inc0)
        Q = fem.build_p2(op2, 1024, seed=0, precision=prec)
        t0 = time.time()
        nz = Q.sparsity.nz
        sp_s = time.time() - t0
        fem.assemble_p2(op2, Q)   # compile, slot tables or incidence, values once
        b200.synchronize()
        if p2_ref is not None:
            errs = [float(np.abs(got - ref).max() / np.abs(ref).max())
                    for got, ref in zip((Q.K.array, Q.M.array), p2_ref)]
        else:
            errs = [None, None]
        ms = _timed(lambda: fem.assemble_p2(op2, Q), reps, b200, graph=True)
        nbytes = fem.km_bytes(Q.n_elem, 6, Q.n_dofs, nz)
        res[tag] = {"nnz": nz, "elements": Q.n_elem, "sparsity_build_s": round(sp_s, 3),
                    "K_plus_M_ms": round(ms, 3), "nnz_per_s": round(2 * nz / (ms * 1e-3), 1),
                    "GBps": round(nbytes / (ms * 1e-3) / 1e9, 1), "algorithmic_bytes": nbytes,
                    "frac": round(nbytes / (ms * 1e-3) / 1e9 / peak, 3),
                    "kahan": kahan, "element_math": prec, "mode": _loop_mode(Q.k_km.name),
                    "max_rel_err_K_vs_oracle": errs[0], "max_rel_err_M_vs_oracle": errs[1]}
        del Q
    cfg.configure(kahan=False, inc_mode=inc0)
    out["p2_1024"] = res
    p1, f64, prec = out["p1_256"], res["f64"], res["f32_lma_kahan"]

    def e(v):
        return None if v is None else float("%.3g" % v)
    out["summary"] = {
        "p1_Gnnz_s": round(p1["mass_nnz_per_s"] / 1e9, 2),
        "p1_frac": round(p1["mass_rhs_GBps"] / peak, 3),
        "p2_Gnnz_s": round(f64["nnz_per_s"] / 1e9, 2), "p2_frac": f64["frac"],
        "p2_err": e(max(f64["max_rel_err_K_vs_oracle"] or 0, f64["max_rel_err_M_vs_oracle"] or 0)
                    if p2_ref is not None else None),
        "prec_frac": prec["frac"],
        "prec_err": e(max(prec["max_rel_err_K_vs_oracle"], prec["max_rel_err_M_vs_oracle"])
                      if p2_ref is not None else None)}
    return out


def _step_loops(A):
    """The bound loops of one iteration (for counting launches)."""
    from pyop2_b200 import b200
    out = []
    for bl in b200.ParLoop._bound_cache.values():
        if bl.spec.kernel_name in ("save_soln", "adt_calc", "res_calc", "bres_calc", "update"):
            out.append(bl)
    names = [bl.spec.kernel_name for bl in out]
    mult = {"save_soln": 1, "adt_calc": 2, "res_calc": 2, "bres_calc": 2, "update": 2}
    res = []
    for bl, nm in zip(out, names):
        res += [bl] * mult[nm]
    return res


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--nx", type=int, default=NX, help="cells along x (default 1200)")
    p.add_argument("--ny", type=int, default=NY, help="cells along y (default 600)")
    p.add_argument("--part-size", type=int, default=0, help="plan partition size (0: backend default)")
    p.add_argument("--block-size", type=int, default=0, help="threads per CTA (0: backend default)")
    p.add_argument("--staged-block-size", type=int, default=0,
                   help="threads per CTA of staged loops (0: backend default)")
    p.add_argument("--region-size", type=int, default=0,
                   help="elements per region of the staged form's partition (0: backend default)")
    p.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    p.add_argument("--no-assembly", action="store_true", help="skip the Mat assembly legs")
    p.add_argument("--assembly-only", action="store_true",
                   help="run only the Mat assembly legs and print their figures")
    p.add_argument("--batch-meshes", type=int, default=4096,
                   help="meshes of the batching leg (0 skips it)")
    p.add_argument("--batching-only", action="store_true",
                   help="run only the batching leg and print its figures")
    p.add_argument("--serve-requests", type=int, default=3000,
                   help="requests of the serving leg (0 skips it)")
    p.add_argument("--serve-rate", type=float, default=2000.0,
                   help="mean Poisson arrival rate of the serving leg (requests/s)")
    p.add_argument("--serving-only", action="store_true",
                   help="run only the serving leg and print its figures")
    p.add_argument("--solve", action="store_true", help="add the linear-solve leg")
    p.add_argument("--detail", default="", help="also write the full figures (JSON) to this file")
    p.add_argument("--solve-only", action="store_true",
                   help="run only the linear-solve leg and print its figures")
    p.add_argument("--l2-fetch", type=int, default=-1,
                   help="L2 fetch granularity in bytes (32/64/128; 0 driver default; -1 backend default)")
    p.add_argument("--min-blocks", type=int, default=-1, help="stub __launch_bounds__ min blocks per SM")
    p.add_argument("--no-permute", action="store_true",
                   help="structured (unpermuted) cell/node numbering instead of the random one")
    p.add_argument("--inc-mode", default="", choices=["", "color", "atomic", "lma", "staged", "gather"],
                   help="INC conflict resolution of indirect loops (default: backend default)")
    args = p.parse_args(argv)
    _set_mesh(args.nx, args.ny)
    ws, rank, local = _dist()
    if args.impl == "reference":
        return run_reference(args, ws, rank, local)
    return run_gpu(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
