"""
Benchmark of the sasmodels hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--config cylinder2d|sphere1d|magnetic]

One step = one evaluation of the polydisperse, oriented cylinder 2D
workload (256x256 (qx, qy) grid, 35x35x20x20 = 490000-point dispersity mesh,
3.21e10 weighted q x mesh-point evaluations) through the driver kernels,
inputs resident in HBM.  ``value`` is q x pd-point evaluations per second
(all ranks).  ``e2e`` is the same metric through the public engine API with
host buffers: each step builds a kernel for the q points (upload), evaluates
I(q) from host ``details``/``values`` arrays and reads I(q) back.

Multi-GPU (torchrun, one rank per GPU): every rank evaluates its own copy of
the workload (independent detector images), no collective on the data path;
timing is the max over ranks ("scaling": "weak").

``--impl reference`` times the reference implementation of the same path on
the host cores: the reference DLL kernel built from the reference's own C
(oracle/_ref), q-sharded over all host threads, on a bounded sample of the
same workload per step; rank 0 only.
"""

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = ("q×pd-point evals/s and fit param-sets/s at rel err ≤1e-5 vs FP64, "
          "plain vs batched")
UNIT = "evals/s"
L2_FLUSH_BYTES = 256 << 20     # > 126 MB L2


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def workload(config, grid=256):
    from sasmodels_b200 import workloads
    if config == "cylinder2d":
        return workloads.cylinder_2d(n=grid), "cylinder 2D oriented FP64, %dx%d q, R(35) x L(35) x theta(20) x phi(20) mesh" % (grid, grid)
    if config == "sphere1d":
        return workloads.sphere_1d(), "sphere 1D FP64, 1000 log q, R gaussian pd 0.1 x 35"
    if config == "magnetic":
        return workloads.core_shell_sphere_magnetic(), "core_shell_sphere 2D magnetic FP64, 128x128 q, R(51 lognormal) x t(21)"
    raise ValueError(config)


def sample_workload(config):
    """Bounded CPU sample of the same workload (full mesh, fewer q)."""
    from sasmodels_b200 import workloads
    if config == "cylinder2d":
        return (workloads.cylinder_2d_strided(8),
                "every 8th row and column of the 256x256 grid (32x32 q, the branch mix "
                "of the whole grid), full 490000-point mesh")
    if config == "sphere1d":
        return workloads.sphere_1d(), "full workload"
    if config == "magnetic":
        name, (qx, qy), pars = workloads.core_shell_sphere_magnetic()
        sub = np.arange(0, qx.size, 16)
        return (name, [qx[sub], qy[sub]], pars), "every 16th q point (1024 q), full 1071-point mesh"
    raise ValueError(config)


def marshal(info, pars, q_vectors):
    from sasmodels_b200.details import make_kernel_args
    from sasmodels_b200.direct_model import get_mesh

    class K:
        pass
    k = K()
    k.info = info
    k.dim = '2d' if len(q_vectors) == 2 else '1d'
    k.dtype = np.dtype('d')
    mesh = get_mesh(info, pars, dim=k.dim)
    return make_kernel_args(k, mesh)


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region, on the GPU
    this process runs on (selected by UUID, so a remapped
    CUDA_VISIBLE_DEVICES still samples the right board).  Samples go to a
    temporary file that is removed after the summary is read."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_device, tag=""):
        import tempfile
        self.gpu = gpu_selector(local_device)
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="sasb200_clocks%s_" % tag, suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return None
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fid:
            for line in fid:
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
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "gpu": self.gpu}


def gpu_selector(local_device):
    """nvidia-smi -i argument for torch device `local_device`: its UUID
    ("GPU-..."), which names the same board whatever CUDA_VISIBLE_DEVICES
    remaps; the ordinal only when the UUID is unavailable."""
    try:
        import torch
        uuid = str(torch.cuda.get_device_properties(local_device).uuid)
        if uuid:
            return uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        pass
    return str(local_device)


def dist_setup(n_gpus):
    """(world, rank, device index) from the torchrun environment; one
    process per GPU over NCCL.  SASB200_BENCH_BACKEND=gloo runs the
    collectives on the host instead, with ranks placed round-robin on the
    visible GPUs: a check of the multi-rank logic on a box with fewer GPUs
    than ranks (its timings mean nothing; no kernel waits on another rank)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = os.environ.get("SASB200_BENCH_BACKEND", "nccl")
        if backend == "gloo":
            local = local % max(torch.cuda.device_count(), 1)
            torch.cuda.set_device(local)
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        else:
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
    return world, rank, local


def dist_max(x):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch
    import torch.distributed as dist
    torch.cuda.synchronize()
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
    torch.cuda.synchronize()


def cpu_baseline(config, seconds_hint=None):
    """Reference DLL (oracle/_ref) on a bounded sample with all host threads."""
    from oracle import refdll
    from sasmodels_b200 import load_model_info
    (name, qv, pars), sample = sample_workload(config)
    info = load_model_info(name)
    details, values, magnetic = marshal(info, pars, qv)
    dim = '2d' if len(qv) == 2 else '1d'
    var = "Iq" if dim == '1d' else ("Imagnetic" if magnetic else "Iqxy")
    nout = 2 if info.have_Fq and dim == '1d' else 1
    if dim == '1d':
        q = np.ascontiguousarray(qv[0])
    else:
        q = np.empty(2*len(qv[0]))
        q[0::2], q[1::2] = qv
    threads = host_threads()
    evals = len(qv[0])*details.num_eval
    refdll.run_threads(name, var, q[:2*min(threads, len(qv[0]))] if dim == '2d' else q[:threads],
                       details.buffer, values, nout, threads)
    t0 = time.perf_counter()
    raw = refdll.run_threads(name, var, q, details.buffer, values, nout, threads)
    dt = time.perf_counter() - t0
    cpu_baseline.last[config] = (name, qv, pars, values, nout, raw)
    return evals/dt, threads, sample, evals, dt


cpu_baseline.last = {}


def cpu_model():
    """The host CPU's model name (for the baseline record)."""
    try:
        with open("/proc/cpuinfo") as fid:
            for line in fid:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def normalised_iq(raw, nout, nq, values):
    """scale/V_shell * <F^2> + background from a raw result vector
    (sasmodels/kernel.py:80-188)."""
    total = raw[nout*nq] or 1.0
    shell = raw[nout*nq + 2]/total or 1.0
    return values[0]/shell*raw[0:nout*nq:nout]/total + values[1]


def errors_vs_dll(config, dev):
    """Max relative difference of I(q) from the reference DLL for the FP64
    and FP32c forms on the bounded sample of `config` that cpu_baseline just
    timed (the DLL's output is the checker; nothing here is timed)."""
    from sasmodels_b200 import load_model
    from sasmodels_b200.direct_model import call_kernel
    if config not in cpu_baseline.last:
        cpu_baseline(config)
    name, qv, pars, values, nout, raw = cpu_baseline.last[config]
    ref = normalised_iq(raw, nout, len(qv[0]), values)
    out = {}
    for dtype in ("double", "float32c"):
        kernel = load_model(name, dtype=dtype, device=dev).make_kernel(qv)
        got = call_kernel(kernel, dict(pars))
        kernel.release()
        out["max_rel_err_vs_dll_" + ("f64" if dtype == "double" else "f32c")] = \
            float(np.max(np.abs(got - ref)/np.abs(ref)))
    return out


def cpu_single_thread(config):
    """Reference DLL on one host thread: the first 1/threads of the bounded
    sample's q points (the per-thread share of the threaded run)."""
    from oracle import refdll
    from sasmodels_b200 import load_model_info
    (name, qv, pars), _ = sample_workload(config)
    info = load_model_info(name)
    details, values, magnetic = marshal(info, pars, qv)
    dim = '2d' if len(qv) == 2 else '1d'
    var = "Iq" if dim == '1d' else ("Imagnetic" if magnetic else "Iqxy")
    nout = 2 if info.have_Fq and dim == '1d' else 1
    n1 = max(1, len(qv[0])//host_threads())
    if dim == '1d':
        q = np.ascontiguousarray(qv[0][:n1])
    else:
        q = np.empty(2*n1)
        q[0::2], q[1::2] = qv[0][:n1], qv[1][:n1]
    t0 = time.perf_counter()
    refdll.run_threads(name, var, q, details.buffer, values, nout, 1)
    return n1*details.num_eval/(time.perf_counter() - t0)


def _reference_sets(jobs, threads):
    """Run the reference DLL on (model, variant, q, pars, nout) jobs, one
    set per host thread at a time; returns the wall time."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import refdll
    from sasmodels_b200 import load_model_info
    prepared = []
    for model, variant, q, pars, nout in jobs:
        info = load_model_info(model)
        qv = [q] if variant == "Iq" else [q, np.zeros_like(q)]
        details, values, _ = marshal(info, pars, qv)
        qi = q if variant == "Iq" else np.column_stack([q, np.zeros_like(q)]).ravel()
        prepared.append((refdll.load(model), variant, np.ascontiguousarray(qi),
                         details.buffer, values, nout))

    def one(job):
        dll, variant, q, det, val, nout = job
        return dll.call(variant, q, det, val, nout)

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as pool:
        list(pool.map(one, prepared))
    return time.perf_counter() - t0


def reference_population(stride=255):
    """Reference DLL param-sets/s on every `stride`-th set of the 4096-set
    population, sets spread over the host threads."""
    from sasmodels_b200 import workloads
    pop = workloads.population(n_sets=4096, seed=1)[::stride]
    threads = host_threads()
    jobs = [(name, "Iq", q, pars, 2) for name, q, pars in pop]
    dt = _reference_sets(jobs, threads)
    return len(jobs)/dt, threads, "every %d-th of 4096 seeded sets (%d sets)" % (stride, len(jobs))


def reference_surrogate(n_sets=16, nq=1000, seed=2):
    """Reference DLL samples/s of the plain cylinder on held-out-like sets
    (the surrogate's plain path: 1D orientation average for flag 1, the 2D
    kernel along qx at theta 90, phi 0 for flag 0)."""
    from sasmodels_b200.surrogate import model_pars, sample_q, sample_sets
    rng = np.random.default_rng(seed)
    sets = sample_sets(n_sets, rng)
    qs = [sample_q(nq, rng) for _ in range(n_sets)]
    jobs = []
    for k in range(n_sets):
        flag = int(sets["flag"][k])
        pars = model_pars(sets["radius"][k], sets["length"][k], sets["rpd"][k],
                          sets["lpd"][k], flag)
        jobs.append(("cylinder", "Iq" if flag else "Iqxy", qs[k], pars, 2 if flag else 1))
    threads = host_threads()
    dt = _reference_sets(jobs, threads)
    return n_sets*nq/dt, threads, "%d seeded held-out-like sets x %d q" % (n_sets, nq)


def run_reference(args, world, rank):
    if rank != 0:
        return
    if args.config == "mlp":
        print(json.dumps({"impl": "reference", "unavailable":
                          "sasmodels has no learned surrogate network"}), flush=True)
        return
    if args.config in ("population", "surrogate"):
        fn = reference_population if args.config == "population" else reference_surrogate
        unit = "param-sets/s" if args.config == "population" else "samples/s"
        vals = []
        for step in range(args.warmup + args.steps):
            v, threads, sample = fn()
            if step >= args.warmup:
                vals.append(v)
        value = statistics.median(vals)
        metric = (METRIC if args.config == "population" else
                  "surrogate log I(q) samples/s at <=1% log-I error with fallback")
        line = {
            "impl": "reference", "metric": metric, "value": value, "unit": unit,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": args.config, "sample": sample,
                       "parallelism": "host threads, one set per thread"},
            "cpu_baseline": {"value": value, "unit": unit, "cores": threads,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    values = []
    for step in range(args.warmup + args.steps):
        v, threads, sample, evals, dt = cpu_baseline(args.config)
        if step >= args.warmup:
            values.append(v)
    value = statistics.median(values)
    (_, _, _), desc = workload(args.config, args.grid)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3*evals/value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "sample": sample, "parallelism": "host threads, q-sharded"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                         "kind": "reference", "sample": sample, "cpu": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200(args, world, rank, local):
    import torch
    from sasmodels_b200 import load_model, peaks

    from sasmodels_b200 import multigpu

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    (name, qv, pars), desc = workload(args.config, args.grid)
    model = load_model(name, dtype=args.dtype, device=dev)
    nq_total = len(qv[0])
    split = args.split == "q" and world > 1
    if split:
        # this rank's contiguous block of the image (q partition)
        lo, hi = multigpu.q_blocks(nq_total, world)[rank]
        qv = [np.ascontiguousarray(v[lo:hi]) for v in qv]
    kernel = model.make_kernel(qv)
    details, values, magnetic = marshal(model.info, pars, qv)
    variant = kernel.variant(magnetic)
    nq = kernel.q_input.nq
    n_mesh = details.num_eval
    evals = nq*n_mesh
    evals_all = nq_total*n_mesh if split else world*evals
    dev_d, dev_v = kernel.upload(details, values)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = kernel.stream
    # mesh_prepare, iq_main, finalize (one fused kernel for a small mesh)
    launches_per_step = kernel.lib.launches(variant, nq, n_mesh)
    nout = 2 if model.meta.have_Fq and kernel.dim == '1d' else 1

    def step():
        """One step on the kernel stream: the evaluation of this rank's
        share and, for a split image, the all-gather of every rank's block
        (device tensors, caller's q order) into the whole image."""
        res = kernel.launch(variant, dev_d, dev_v, 0, n_mesh, 0.0, 0)
        if split:
            slots = res[:nout*nq]
            if kernel.q_input.order_dev is not None:
                slots = torch.empty_like(slots).index_copy_(0, kernel.q_input.order_dev,
                                                            slots)
            return multigpu.gather_blocks(slots)
        return res

    tile = 0
    if not args.no_tune:
        from sasmodels_b200 import autotune
        tile = autotune.tune_kernel(kernel, variant, dev_d, dev_v, n_mesh, reps=1,
                                    budget_s=15.0)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    barrier()

    times = []
    with ClockSampler(local) as clocks:
        barrier()
        t_wall = time.perf_counter()
        with torch.cuda.stream(stream):
            for _ in range(args.steps):
                flush.zero_()
                start = torch.cuda.Event(enable_timing=True)
                stop = torch.cuda.Event(enable_timing=True)
                start.record(stream)
                step()
                stop.record(stream)
                times.append((start, stop))
        barrier()
        wall = time.perf_counter() - t_wall
    step_s = [a.elapsed_time(b)*1e-3 for a, b in times]
    t_total = dist_max(sum(step_s))
    value = evals_all*args.steps/t_total
    ms_per_step = 1e3*t_total/args.steps

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        qhost = [np.ascontiguousarray(v) for v in qv]
        h2d = sum(v.nbytes for v in qhost) + details.buffer.nbytes + values.nbytes
        d2h = kernel.result.nbytes

        def e2e_step():
            # the public call on this rank's q points from host arrays, I(q)
            # back on the host; a split image is then all-gathered so every
            # rank holds the whole I(q)
            k2 = model.make_kernel(qhost)
            I = k2(details, values, 0.0, magnetic)
            k2.release()
            if split:
                I = multigpu.gather_blocks(torch.as_tensor(I)).cpu().numpy()
            return I

        # the clock sampler (an nvidia-smi process, costly to start) is
        # started before the untimed warm-up step, and the setup's garbage is
        # collected before the clock starts; the sampler and the collector
        # both stay on while the steps are timed
        with ClockSampler(local, "_e2e") as e2e_clocks:
            e2e_step()
            gc.collect()
            time.sleep(0.5)
            barrier()
            # at least 10 steps: one stall of the host weighs less in the mean
            e2e_steps = max(args.steps, 10)
            t0 = time.perf_counter()
            for _ in range(e2e_steps):
                e2e_step()
            barrier()
            te = dist_max(time.perf_counter() - t0)
        e2e = {"value": evals_all*e2e_steps/te, "unit": UNIT, "steps": e2e_steps,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "breakdown_ms": e2e_breakdown(model, qhost, details, values, magnetic,
                                             variant, n_mesh)}
        s = e2e_clocks.summary()
        if s:
            e2e["clocks"] = s

    line = None
    if rank == 0:
        fp64_peak = peaks.fp64_tflops()
        roofline = {"bound": "fp64", "unit": "TFLOP/s", "peak": fp64_peak,
                    "peak_source": "measured live: csrc/peaks.cu DFMA probe (of measured)",
                    "traffic": TRAFFIC_PER_STEP.get(args.config)}
        sf = SASFLOPS.get(args.config) if args.dtype == "double" else None
        if sf:
            per_eval = sf["eval"]/sf["evals"]
            if sf["evals"] == evals:
                total = sf["eval"] + sf["point"] + sf["q"]
                how = "exact count of this configuration"
            else:
                total = per_eval*evals
                how = "per-evaluation mean of the full configuration x evaluations"
            achieved = total/(ms_per_step*1e-3)/1e12
            roofline.update({
                "achieved": achieved, "frac": achieved/fp64_peak,
                "numerator": "algorithmic SAS-flops: the SAS-flop v1 count of the "
                             "reference's own model C on this configuration's inputs, "
                             "every branch replayed (oracle/sasflops.py); " + how,
                "sasflops_per_step": total, "sasflops_per_eval": per_eval})
        if args.config in ROOFLINE_NOTES and sf:
            roofline["note"] = ROOFLINE_NOTES[args.config]
        issued = ISSUED_FP64_PER_EVAL.get(args.config) if args.dtype == "double" else None
        if issued:
            got = issued*evals/(ms_per_step*1e-3)/1e12
            roofline["fp64_pipe"] = {
                "issued_flops_per_eval": issued, "achieved": got, "frac": got/fp64_peak,
                "source": "ncu DFMA/DMUL/DADD counts of the current iq_main "
                          "(2 x DFMA + DMUL + DADD per evaluation)"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "strong" if split else "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.dtype == "double" else "f32 compensated (f64 phases and sums)",
            "data": "synthetic",
            "config": {"workload": desc, "evals_per_step": evals_all, "nq": nq_total,
                       "tile": "0x%08x (autotuned)" % tile if tile else "library default",
                       "mesh": n_mesh, "l2": "flushed (256 MB write) before each timed step",
                       "parallelism": (
                           "q partition x%d: contiguous q blocks of one image, one per GPU, "
                           "blocks all-gathered as device tensors inside each step" % world
                           if split else "replicas x%d (one workload per GPU)" % world)},
            "e2e": e2e,
            "gpu_launches": launches_per_step*args.steps,
            "wall_s": wall,
            "roofline": roofline,
        }
        if args.dtype != "double":
            mufu = peaks.mufu_tops()
            ops = XU_OPS_PER_EVAL.get(args.config)
            got = ops*evals/(ms_per_step*1e-3)/1e12 if ops else None
            line["roofline"] = {"bound": "xu", "achieved": got, "peak": mufu,
                                "unit": "Tops/s", "frac": (got/mufu) if got else None,
                                "peak_source": "measured live: csrc/peaks.cu MUFU probe",
                                "xu_ops_per_eval": ops,
                                "traffic": TRAFFIC_PER_STEP.get(args.config)}
        s = clocks.summary()
        if s:
            line["clocks"] = s
        if world == 1 and not args.no_cpu:
            v, threads, sample, _, _ = cpu_baseline(args.config)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads,
                                    "kind": "reference", "sample": sample,
                                    "value_1_thread": cpu_single_thread(args.config),
                                    "cpu": cpu_model()}
            line["parity_vs_dll"] = dict(errors_vs_dll(args.config, dev), sample=sample)
        if world == 1 and not args.no_extras and args.config == "cylinder2d":
            line["extra"] = extras(dev, with_dll=not args.no_cpu, tile=tile or None,
                                   surrogate=not args.no_surrogate)
        print(json.dumps(line), flush=True)
    return line


def e2e_breakdown(model, qhost, details, values, magnetic, variant, n_mesh):
    """Where one end-to-end step's time goes (host clock, synchronised
    between phases): make_kernel (q ordering and upload, buffers), the call
    (values upload, kernels, I(q) back and normalised) with the kernels'
    own device time from CUDA events, and release; plus the tile the call
    ran on."""
    import torch
    from sasmodels_b200 import autotune
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    k = model.make_kernel(qhost)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    k(details, values, 0.0, magnetic)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    dd, dv = k.upload(details, values)
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(k.stream):
        start.record(k.stream)
        k.launch(variant, dd, dv, 0, n_mesh, 0.0, 0)
        stop.record(k.stream)
    stop.synchronize()
    tile = autotune.cached_tile(k, variant, n_mesh)
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    k.release()
    torch.cuda.synchronize()
    t4 = time.perf_counter()
    return {"make_kernel": 1e3*(t1 - t0), "call": 1e3*(t2 - t1),
            "kernels_device": start.elapsed_time(stop), "release": 1e3*(t4 - t3),
            "tile": "0x%08x" % tile}


def time_launches(kernel, variant, dd, dv, n_mesh, reps):
    """Seconds per call of `reps` back-to-back launches on the kernel's
    stream, CUDA events around them (host launch overhead included when it
    exceeds the device time of a call)."""
    import torch
    stream = kernel.stream
    with torch.cuda.stream(stream):
        kernel.launch(variant, dd, dv, 0, n_mesh, 0.0, 0)
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(reps):
            kernel.launch(variant, dd, dv, 0, n_mesh, 0.0, 0)
        stop.record(stream)
    stop.synchronize()
    return start.elapsed_time(stop)*1e-3/reps


def time_graph(kernel, variant, dd, dv, n_mesh, reps):
    """Device seconds per call: `reps` launches captured in one CUDA graph and
    replayed, CUDA events around the replay (no host work between calls)."""
    import torch
    stream = kernel.stream
    with torch.cuda.stream(stream):
        kernel.launch(variant, dd, dv, 0, n_mesh, 0.0, 0)      # workspace, tile, module
    stream.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        for _ in range(reps):
            kernel.launch(variant, dd, dv, 0, n_mesh, 0.0, 0)
    with torch.cuda.stream(stream):
        graph.replay()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        graph.replay()
        stop.record(stream)
    stop.synchronize()
    del graph
    return start.elapsed_time(stop)*1e-3/reps


def single_config(name, qv, pars, dtype, reps, dev, form=None, tile=None):
    """evals/s of one plain call shape (inputs resident); `form` "plugin"
    runs the plugin's C as translated where the model has a hoisted
    binding; `tile` fixes the tile code."""
    from sasmodels_b200 import _abi, load_model
    model = load_model(name, dtype=dtype, device=dev)
    if form is not None:
        model.lib = _abi.load_library(name, form=form)
    kernel = model.make_kernel(qv)
    if tile is not None:
        kernel.tile = tile
    details, values, magnetic = marshal(model.info, pars, qv)
    dd, dv = kernel.upload(details, values)
    t = time_launches(kernel, kernel.variant(magnetic), dd, dv, details.num_eval, reps)
    return len(qv[0])*details.num_eval/t, t


def small_config(name, qv, pars, dtype, reps, dev):
    """evals/s of a call shape whose device time is below the host's launch
    overhead: device time per call from a CUDA graph of `reps` launches, and
    the host-launched loop beside it."""
    from sasmodels_b200 import load_model
    model = load_model(name, dtype=dtype, device=dev)
    kernel = model.make_kernel(qv)
    details, values, magnetic = marshal(model.info, pars, qv)
    dd, dv = kernel.upload(details, values)
    variant = kernel.variant(magnetic)
    t_graph = time_graph(kernel, variant, dd, dv, details.num_eval, reps)
    t_loop = time_launches(kernel, variant, dd, dv, details.num_eval, reps)
    evals = len(qv[0])*details.num_eval
    return {"evals_per_s": evals/t_graph, "ms_per_call": 1e3*t_graph,
            "timing": "device time per call, %d calls replayed from one CUDA graph" % reps,
            "launches_per_call": kernel.lib.launches(variant, kernel.q_input.nq,
                                                     details.num_eval),
            "host_loop_evals_per_s": evals/t_loop, "host_loop_ms_per_call": 1e3*t_loop}


def population_compare(n_sets, stride, dev, tune=True):
    """Batched FP32c vs plain FP64 per-set launches on every `stride`-th set
    of the seeded population: param-sets/s of both and the max relative
    error of the batched I(q) against the FP64 plain results."""
    import torch
    from sasmodels_b200 import autotune, load_model, workloads
    from sasmodels_b200.batch import Population
    from sasmodels_b200.pack import columns_from_sets
    pop = workloads.population(n_sets=n_sets, seed=1)[::stride]
    by = {}
    for k, (name, q, pars) in enumerate(pop):
        by.setdefault(name, []).append((k, q, pars))
    t_batch = t_plain = 0.0
    t_gen_batch = t_gen_plain = t_gen_cols = 0.0
    gen_h2d = gen_d2h = 0
    worst = cols_diff = 0.0
    tuned = {}
    for name, members in by.items():
        sets = [(q, p) for _, q, p in members]
        warps, ipw = autotune.tune_population(name, sets, "float32c") if tune else (8, 8)
        tuned[name] = [warps, ipw]
        P = Population(name, sets, form="float32c", device=dev, warps=warps,
                       items_per_warp=ipw)
        P.run()
        P.stream.synchronize()
        # the batch and the per-set loop below are both timed on the host
        # clock from launch to completion (the per-set loop cannot be
        # bracketed by one stream's events: every set has its own kernel)
        t0 = time.perf_counter()
        P.run()
        P.stream.synchronize()
        t_batch += time.perf_counter() - t0
        iq_batch = P.iq()
        model = load_model(name, device=dev)
        calls = []
        for q, pars in sets:
            k = model.make_kernel([q])
            d, v, _ = marshal(model.info, pars, [q])
            dd, dv = k.upload(d, v)
            calls.append((k, dd, dv, d.num_eval, v))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k, dd, dv, n, _ in calls:
            with torch.cuda.stream(k.stream):
                k.launch("Iq", dd, dv, 0, n, 0.0, 0)
            k.stream.synchronize()
        t_plain += time.perf_counter() - t0
        for (k, dd, dv, n, v), iq_b in zip(calls, iq_batch):
            raw = k._result_dev.cpu().numpy()
            nq = k.q_input.nq
            total = raw[2*nq] or 1.0
            shell = raw[2*nq + 2]/total or 1.0
            iq64 = v[0]/shell*raw[0:2*nq:2]/total + v[1]
            worst = max(worst, float(np.max(np.abs(iq_b - iq64)/np.abs(iq64))))
        # one fit generation end to end (new host values in, I(q) of every
        # set out): batched update + graph replay + readback against the
        # plain path's per-set marshal + upload + launch + readback
        new = [dict(p, scale=1.01*p.get("scale", 1.0)) for _, p in sets]
        P.capture()
        P.update(new)
        P.replay()
        P.iq()
        t0 = time.perf_counter()
        P.update(new)
        P.replay()
        P.iq()
        t_gen_batch += time.perf_counter() - t0
        gen_h2d += 8*P.h_val.numel()
        gen_d2h += 8*P.d_iq.numel()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for (k, _, _, _, _), (q, _), pars in zip(calls, sets, new):
            # the public call: marshal, upload, launch, wait, read back
            d, v, _ = marshal(model.info, pars, [q])
            k.Iq(d, v, 0.0, False)
        t_gen_plain += time.perf_counter() - t0
        # the same generation given as parameter columns (a fit population
        # as the optimiser holds it): the table is expanded into the values
        # vectors on the device inside the replayed graph
        cols0 = columns_from_sets(P.info, [p for _, p in sets])
        cols1 = columns_from_sets(P.info, new)
        PC = Population.from_columns(name, [q for q, _ in sets], cols0, form="float32c",
                                     device=dev, warps=warps, items_per_warp=ipw)
        PC.capture()
        PC.update_columns(cols1)
        PC.replay()
        PC.iq()
        t0 = time.perf_counter()
        PC.update_columns(cols1)
        PC.replay()
        iq_cols = PC.iq()
        t_gen_cols += time.perf_counter() - t0
        for a, b in zip(iq_cols, P.iq()):
            cols_diff = max(cols_diff, float(np.max(np.abs(a - b)/np.abs(b))))
    n = len(pop)
    return {"sets": n, "sample": "every %d-th of %d seeded sets" % (stride, n_sets),
            "headline": "generation_e2e.speedup: one fit generation end to end, host "
                        "values in, every I(q) out, both arms on the host clock",
            "batched_f32c_sets_per_s": n/t_batch, "plain_f64_sets_per_s": n/t_plain,
            "speedup": t_plain/t_batch,
            "speedup_clock": "both arms launch to completion on the host clock",
            "max_rel_err_vs_f64": worst,
            "generation_e2e": {"batched_f32c_ms": 1e3*t_gen_batch,
                               "h2d_bytes": int(gen_h2d), "d2h_bytes": int(gen_d2h),
                               "plain_f64_ms": 1e3*t_gen_plain,
                               "speedup": t_gen_plain/t_gen_batch,
                               "columns_ms": 1e3*t_gen_cols,
                               "columns_speedup": t_gen_plain/t_gen_cols,
                               "columns_max_rel_diff": cols_diff},
            "autotuned": tuned}


def smear_compare(dev, reps=50):
    """One smeared sphere 1D curve (1000 q, 5 % pinhole, 35-point
    dispersity) through the model kernel and the GPU smearing with only the
    smeared curve read back, against the same kernel followed by the
    reference's dense-matrix smearing on the host (theory read back)."""
    import torch
    from sasmodels_b200 import load_model, workloads
    from sasmodels_b200.resolution import Pinhole1D
    name, (q,), pars = workloads.sphere_1d()
    res = Pinhole1D(q, 0.05*q, device=dev)
    W = res.weight_matrix
    model = load_model(name, device=dev)
    kernel = model.make_kernel([res.q_calc])
    details, values, _ = marshal(model.info, pars, [res.q_calc])
    dd, dv = kernel.upload(details, values)

    def fused():
        I = kernel.Iq_device(dd, dv, details.num_eval, values[0], values[1])
        out = res.apply(I, stream=kernel.stream)
        kernel.stream.synchronize()
        return out.cpu().numpy()

    def host():
        I = kernel.Iq_device(dd, dv, details.num_eval, values[0], values[1])
        kernel.stream.synchronize()
        return np.dot(I.cpu().numpy()[None, :], W).flatten()

    out = {"n_q": len(q), "n_calc": len(res.q_calc)}
    for key, fn in (("gpu_smear_ms", fused), ("host_matrix_smear_ms", host)):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        out[key] = 1e3*(time.perf_counter() - t0)/reps
    a, b = fused(), host()
    out["max_rel_diff"] = float(np.max(np.abs(a - b)/np.abs(b)))
    return out


def extras(dev, with_dll=True, tile=None, surrogate=True):
    """Secondary measurements of the other headline configurations; with
    `with_dll`, each FP64 and FP32c form's max relative error against the
    reference DLL on that configuration's bounded CPU sample."""
    from sasmodels_b200 import workloads
    out = {}
    name, qv, pars = workloads.sphere_1d()
    for dtype in ("double", "float32c"):
        out["sphere1d_" + dtype] = small_config(name, qv, pars, dtype, 200, dev)
    name, qv, pars = workloads.cylinder_2d()
    v, t = single_config(name, qv, pars, "float32c", 3, dev)
    out["cylinder2d_float32c"] = {"evals_per_s": v, "ms_per_call": 1e3*t}
    v, t = single_config(name, qv, pars, "double", 3, dev, form="plugin", tile=tile)
    out["cylinder2d_plugin_f64"] = {
        "evals_per_s": v, "ms_per_call": 1e3*t, "tile": "0x%08x" % tile if tile else None,
        "what": "the plugin's Iqac as translated, without the hoisted binding, on the "
                "headline's tile"}
    name, qv, pars = workloads.core_shell_sphere_magnetic()
    for dtype in ("double", "float32c"):
        v, t = single_config(name, qv, pars, dtype, 20, dev)
        out["magnetic_" + dtype] = {"evals_per_s": v, "ms_per_call": 1e3*t,
                                    "spin_channels": 6}
    v, t = single_config(name, qv, pars, "double", 20, dev, form="plugin")
    out["magnetic_plugin_f64"] = {
        "evals_per_s": v, "ms_per_call": 1e3*t,
        "what": "the plugin's Fq called once per spin channel, without the fused binding"}
    if with_dll:
        for config, keys in (("sphere1d", ("sphere1d_double", "sphere1d_float32c")),
                             ("cylinder2d", (None, "cylinder2d_float32c")),
                             ("magnetic", ("magnetic_double", "magnetic_float32c"))):
            errs = errors_vs_dll(config, dev)
            for key, tag in zip(keys, ("f64", "f32c")):
                if key is not None:
                    out[key]["max_rel_err_vs_dll"] = errs["max_rel_err_vs_dll_" + tag]
                    out[key]["dll_sample"] = sample_workload(config)[1]
    out["population"] = population_compare(4096, 7, dev)
    if with_dll:
        out["population"]["vs_dll"] = population_vs_dll(dev)
    out["smear_pinhole1d"] = smear_compare(dev)
    if surrogate:
        out["surrogate"] = surrogate_extra(dev)
    return out


def surrogate_extra(dev, n_train_sets=50000, epochs=32, gate_epochs=16, n_holdout_sets=3000):
    """The learned surrogate at its stated budget: 5e7 training samples
    (50,000 sets x 1000 q), 32 epochs, the error gate on 1e7 fresh samples,
    gate thresholds calibrated on 2000 held-out sets judged by the plain FP64
    kernel and the measurement on the other 1000 held-out sets (1e6
    samples): samples/s at 1 % log-I error with automatic fallback, against
    the plain FP64 path on the same points."""
    from sasmodels_b200.surrogate import train_and_evaluate
    t0 = time.perf_counter()
    S, rep = train_and_evaluate(n_train_sets=n_train_sets, nq=1000, epochs=epochs,
                                gate_epochs=gate_epochs, n_holdout_sets=n_holdout_sets,
                                device=dev)
    wall = time.perf_counter() - t0
    op = rep["operating_points"]["0.01"]
    return {"samples_per_s_at_1pct": op["samples_per_s"],
            "mlp_kernels": mlp_kernel_times(S.net),
            "speedup_vs_plain_f64": op["speedup"],
            "speedup_vs_plain_f32c": op["speedup_vs_plain_f32c"],
            "fallback_frac": op["fallback_frac"], "frac_within_1pct": op["frac_within"],
            "max_log_err": op["max_err"], "heldout_samples": rep["holdout_samples"],
            "net_only_median_err": rep["net_median_err"], "net_only_p99_err": rep["net_p99_err"],
            "train_samples": rep["train_samples"], "epochs": rep["epochs"],
            "data_s": rep["data_s"], "train_s": rep["train_s"], "gate_s": rep["gate_s"],
            "wall_s": wall,
            "labels": "batched FP32c engine (within 1e-5 of FP64); judged by plain FP64",
            "report": rep}


#: Multiply-adds of the surrogate network per row, counted as 2 flops each:
#: 16 -> 256, three 256 -> 256 layers and the 256 -> 1 output (0.402 MFLOP).
#: The kernels issue the hidden layers twice (the compensated hi and lo
#: activations), which this algorithmic count leaves out.
MLP_FLOPS_PER_ROW = 2*(16*256 + 3*256*256 + 256)
#: DRAM bytes (read + write) of one mlp_serve launch over 4,000,000 rows, from
#: ncu (profiles/mlp_surrogate.md): the features in and the outputs out
MLP_SERVE_TRAFFIC = 278.5e6


def bf16_peak():
    """Dense BF16 burst peak in TFLOP/s and where it comes from."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fid:
            return float(json.load(fid)["bf16_tflops"]), "of measured (cuBLAS bf16 burst)"
    except (OSError, KeyError, ValueError):
        return 1590.0, "of fallback"


def mlp_kernel_times(net, rows=4_000_000, reps=5):
    """Device time of one inference launch over `rows` rows (features of
    2 x 128 MB, more than L2) for the overlapped serving kernel (mlp_serve)
    and the pipelined training forward without planes (mlp_infer), median of
    `reps` CUDA-event timings on the network's stream after 3 warm-up
    launches; algorithmic TFLOP/s from MLP_FLOPS_PER_ROW."""
    import torch
    from sasmodels_b200.surrogate import pad128
    n_pad = pad128(rows)
    g = torch.Generator(device=net.device).manual_seed(5)
    x = (0.5*torch.randn(n_pad, 16, device=net.device, generator=g)).to(torch.bfloat16)
    x_lo = (1e-3*torch.randn(n_pad, 16, device=net.device, generator=g)).to(torch.bfloat16)
    peak, source = bf16_peak()
    out = {"rows": rows, "mflop_per_row": MLP_FLOPS_PER_ROW/1e6, "peak_tflops": peak,
           "peak_source": source}
    torch.cuda.synchronize()
    for name in ("serve", "infer"):
        fn = getattr(net, name)
        with torch.cuda.stream(net.stream):
            for _ in range(3):
                fn(x, x_lo, rows)
            times = []
            for _ in range(reps):
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                ev[0].record(net.stream)
                fn(x, x_lo, rows)
                ev[1].record(net.stream)
                ev[1].synchronize()
                times.append(ev[0].elapsed_time(ev[1]))
        ms = float(np.median(times))
        got = rows*MLP_FLOPS_PER_ROW/(ms*1e-3)/1e12
        out["mlp_" + name] = {"ms": ms, "rows_per_s": rows/(ms*1e-3),
                              "algorithmic_tflops": got, "frac": got/peak}
    if net.errors():
        raise RuntimeError("surrogate kernel pipeline error %d" % net.errors())
    return out


def population_vs_dll(dev, stride=97, nq_sub=8, max_mesh=60000):
    """Batched FP32c and FP64 I(q) against the reference DLL on every
    `stride`-th set of the seeded population with a dispersity mesh of at
    most `max_mesh` points, each at `nq_sub` of its q points (smallest and
    largest kept), the DLL sharded over host threads by mesh range."""
    from oracle import refdll
    from sasmodels_b200 import load_model_info, workloads
    from sasmodels_b200.batch import Population
    pop = workloads.population(n_sets=4096, seed=1)[::stride]
    by = {}
    for name, q, pars in pop:
        idx = np.unique(np.linspace(0, len(q) - 1, nq_sub).round().astype(int))
        info = load_model_info(name)
        details, values, _ = marshal(info, pars, [q[idx]])
        if details.num_eval > max_mesh:
            continue
        by.setdefault(name, []).append((q[idx], pars, details, values))
    out = {"sets": sum(len(v) for v in by.values()),
           "sample": "every %d-th of 4096 seeded sets with <= %d mesh points, %d q each"
                     % (stride, max_mesh, nq_sub)}
    threads = host_threads()
    for form in ("double", "float32c"):
        worst = 0.0
        for name, members in by.items():
            P = Population(name, [(q, p) for q, p, _, _ in members], form=form, device=dev)
            P.run()
            for (q, _, details, values), iq in zip(members, P.iq()):
                raw = refdll.run_mesh_threads(name, "Iq", q, details.buffer, values, 2,
                                              threads)
                ref = normalised_iq(raw, 2, len(q), values)
                worst = max(worst, float(np.max(np.abs(iq - ref)/np.abs(ref))))
        out["max_rel_err_vs_dll_" + ("f64" if form == "double" else "f32c")] = worst
    return out


#: Algorithmic work of each configuration per step, in SAS-flops (the
#: "SAS-flop v1" convention: +,-,*,compare 1; / and sqrt 4; sin, cos, exp,
#: log 16; sincos 24): the reference's own model C run on the
#: configuration's inputs with a counting arithmetic type, every branch
#: replayed, split into per-evaluation, per-mesh-point and per-q work.
#: Produced by `python oracle/build_oracle.py && python oracle/sasflops.py
#: sphere1d magnetic cylinder2d` (profiles/sasflops_counts.md).
SASFLOPS = {
    "cylinder2d": {"evals": 32112640000, "eval": 3316854138640, "point": 73500000, "q": 0},
    "sphere1d": {"evals": 35000, "eval": 1672720, "point": 350, "q": 0},
    "magnetic": {"evals": 17547264, "eval": 11053000224, "point": 12852, "q": 13074432},
}
#: FP64 flops issued per evaluation by the current iq_main of each
#: configuration, from ncu's instruction counters (2 x DFMA + DMUL + DADD
#: per thread instruction) over the evaluations of the captured launch; the
#: issued count includes the operations CUDA's sin, sqrt and division expand
#: into, so it sits above the algorithmic count (profiles/iq_main_*.md).
ISSUED_FP64_PER_EVAL = {"cylinder2d": 95.1, "magnetic": 157.3}
#: configurations whose kernel skips work the reference repeats, so that the
#: algorithmic count divided by the kernel's time can exceed the peak
ROOFLINE_NOTES = {
    "magnetic": "the count is the reference's work, which evaluates both Bessel terms "
                "once per spin channel; the kernel's channels share them (five times "
                "fewer), so achieved/peak exceeds 1: fp64_pipe is the kernel's own "
                "FP64 rate"}
#: XU-pipe (MUFU sin/cos/rcp/rsqrt and conversions) thread operations per
#: evaluation of the FP32c form of iq_main: ncu's sm__inst_executed_pipe_xu
#: (51.6 % of a 16-lane-per-clock peak over the elapsed cycles) x 32 lanes
#: / evaluations of the captured launch (profiles/iq_main_cylinder2d_f32c.md)
XU_OPS_PER_EVAL = {"cylinder2d": 12.3}
#: dram read+write bytes of the dominant kernel per launch (ncu, on the
#: 64x64-q case of the same mesh): the 490,000 hoisted 48-byte rows of the
#: mesh table are read once from DRAM and then served from L2, so the figure
#: does not grow with the number of q points (profiles/iq_main_cylinder2d.md)
TRAFFIC_PER_STEP = {"cylinder2d": 23.62e6}


def run_population(args, world, rank, local):
    """Fit population: batched FP32c persistent launch vs plain FP64 per-set
    launches on every `--pop-stride`-th set of the 4096-set population."""
    if rank != 0:
        return
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    rep = population_compare(4096, args.pop_stride, dev, tune=not args.no_tune)
    gen = rep["generation_e2e"]
    line = {
        "metric": METRIC, "value": rep["batched_f32c_sets_per_s"], "unit": "param-sets/s",
        "e2e": {"value": rep["sets"]/(1e-3*gen["batched_f32c_ms"]), "unit": "param-sets/s",
                "h2d_bytes_per_step": gen["h2d_bytes"], "d2h_bytes_per_step": gen["d2h_bytes"],
                "speedup_vs_plain_f64": gen["speedup"],
                "what": "one fit generation: new host values in, every I(q) out"},
        "n_gpus": 1, "steps": 1, "warmup": 1, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 compensated (f64 phases and sums)",
        "data": "synthetic", "config": {"workload": "ellipsoid + core_shell_cylinder 1D population",
                                        "sample": rep["sample"]},
        "population": rep,
    }
    print(json.dumps(line), flush=True)


def run_population_split(args, world, rank, local):
    """The fit-population sample (every `--pop-stride`-th of the 4096 seeded
    sets) split over the ranks by estimated cost (multigpu.shard_by_cost,
    per model); each rank evaluates its share as one batched FP32c launch
    per model and the I(q) of all sets are all-gathered as device tensors
    inside each step.  Total work is fixed as N grows ("strong")."""
    import torch
    from sasmodels_b200 import multigpu, workloads
    from sasmodels_b200.batch import Population
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    pop = workloads.population(n_sets=4096, seed=1)[::args.pop_stride]
    pops = []
    for name in workloads.POP_MODELS:
        sets = [(q, p) for n, q, p in pop if n == name]
        parts = multigpu.shard_by_cost(multigpu.population_cost(name, sets), world)
        mine = [sets[i] for i in parts[rank]]
        if mine:
            pops.append(Population(name, mine, form="float32c", device=dev))
    cur = torch.cuda.current_stream()

    def step():
        for P in pops:
            P.stream.wait_stream(cur)
            P.run()
            cur.wait_stream(P.stream)
        flat = (torch.cat([P.d_iq for P in pops]) if pops else
                torch.zeros(0, dtype=torch.float64, device=dev))
        return multigpu.gather_blocks(flat)

    for _ in range(args.warmup):
        step()
    barrier()
    times = []
    with ClockSampler(local) as clocks:
        barrier()
        for _ in range(args.steps):
            start = torch.cuda.Event(enable_timing=True)
            stop = torch.cuda.Event(enable_timing=True)
            start.record(cur)
            step()
            stop.record(cur)
            times.append((start, stop))
        barrier()
    t_total = dist_max(sum(a.elapsed_time(b)*1e-3 for a, b in times))
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": len(pop)*args.steps/t_total, "unit": "param-sets/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3*t_total/args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 compensated (f64 phases and sums)", "data": "synthetic",
        "config": {"workload": "ellipsoid + core_shell_cylinder 1D population",
                   "sample": "every %d-th of 4096 seeded sets (%d sets)"
                             % (args.pop_stride, len(pop)),
                   "parallelism": "population split by cost x%d, I(q) all-gathered as "
                                  "device tensors inside each step" % world},
        "gpu_launches": 3*len(workloads.POP_MODELS)*args.steps,
    }
    summary = clocks.summary()
    if summary:
        line["clocks"] = summary
    print(json.dumps(line), flush=True)


def run_mlp(args, world, rank, local):
    """The surrogate network's kernels alone, random weights: one inference
    launch over 4,000,000 rows through the overlapped serving kernel (the
    line's value) and the pipelined training forward, and one training step
    at batch 8192 replayed from its CUDA graph."""
    if rank != 0:
        return
    import torch
    from sasmodels_b200.surrogate import MLP
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    net = MLP(seed=3, device=dev)
    reps = max(args.steps, 5)
    times = mlp_kernel_times(net, reps=reps)
    serve = times["mlp_serve"]
    # training: one eager step loads the kernels, then the captured step
    B, nrows = 8192, 8192*64
    g = torch.Generator(device=dev).manual_seed(7)
    x = (0.5*torch.randn(nrows, 16, device=dev, generator=g)).to(torch.bfloat16)
    x_lo = torch.zeros_like(x)
    y = torch.randn(nrows, device=dev, generator=g)
    perm = torch.randperm(nrows, device=dev, generator=g)
    net.train_step(x[:B], x_lo[:B], y[:B], B, 1e-4)
    graph = net.capture_training(x, x_lo, y, B, 1e-3, 100000, 1)
    for i in range(args.warmup + 10):
        graph.step(perm[(i % 64)*B:(i % 64 + 1)*B])
    n_steps = 200
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(net.stream)
    for i in range(n_steps):
        graph.step(perm[(i % 64)*B:(i % 64 + 1)*B])
    ev[1].record(net.stream)
    ev[1].synchronize()
    if net.errors():
        raise RuntimeError("surrogate kernel pipeline error %d" % net.errors())
    peak, source = bf16_peak()
    line = {
        "metric": "surrogate network inference rows/s (mlp_serve)",
        "value": serve["rows_per_s"], "unit": "rows/s", "n_gpus": 1, "steps": reps,
        "warmup": 3, "ms_per_step": serve["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 (compensated activations), f32 accumulate",
        "data": "synthetic (random weights and features)",
        "config": {"workload": "16 -> 4 x 256 SiLU -> 1 network, 4,000,000 rows per launch "
                               "(features 2 x 128 MB, above L2)"},
        "roofline": {"bound": "tensor", "unit": "TFLOP/s",
                     "achieved": serve["algorithmic_tflops"], "peak": peak,
                     "peak_source": source, "frac": serve["frac"],
                     "numerator": "MLP_FLOPS_PER_ROW (0.402 MFLOP) x rows; the hi and lo "
                                  "activation halves double the issued MMAs",
                     "traffic": MLP_SERVE_TRAFFIC},
        "mlp_kernels": times,
        "training_step": {"batch": B, "ms": ev[0].elapsed_time(ev[1])/n_steps,
                          "what": "one replay of the captured training step (gather, schedule, "
                                  "forward with planes, backward, gradients, Adam)"},
    }
    print(json.dumps(line), flush=True)


def run_surrogate(args, world, rank, local):
    """Learned surrogate: train on plain-kernel data, judge on held-out sets,
    time the network with automatic fallback against the plain FP64 path."""
    if rank != 0:
        return
    import torch
    from sasmodels_b200.surrogate import train_and_evaluate
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    S, rep = train_and_evaluate(n_train_sets=args.surrogate_sets, nq=1000,
                                epochs=args.surrogate_epochs,
                                gate_epochs=args.surrogate_gate_epochs,
                                n_holdout_sets=args.surrogate_holdout, device=dev)
    op = rep["operating_points"]["0.01"]
    line = {
        "metric": "surrogate log I(q) samples/s at <=1% log-I error with fallback",
        "value": op["samples_per_s"], "unit": "samples/s", "n_gpus": 1,
        "steps": 1, "warmup": 0, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16 (compensated activations), f32 accumulate",
        "data": "synthetic (plain-kernel labels)",
        "config": {"workload": "polydisperse cylinder surrogate, 7 inputs -> 4x256 SiLU -> log I",
                   "train_samples": rep["train_samples"], "epochs": rep["epochs"]},
        "mlp_kernels": mlp_kernel_times(S.net),
        "surrogate": rep,
    }
    print(json.dumps(line), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="cylinder2d",
                    choices=["cylinder2d", "sphere1d", "magnetic", "surrogate", "population",
                             "mlp"])
    ap.add_argument("--pop-stride", type=int, default=7,
                    help="population config: evaluate every n-th of the 4096 sets")
    ap.add_argument("--surrogate-holdout", type=int, default=3000,
                    help="held-out sets x 1000 q: two thirds calibrate the gate, "
                         "one third (1e6 samples) is measured")
    ap.add_argument("--surrogate-sets", type=int, default=50000,
                    help="training parameter sets (x 1000 q each)")
    ap.add_argument("--surrogate-epochs", type=int, default=32)
    ap.add_argument("--surrogate-gate-epochs", type=int, default=16)
    ap.add_argument("--grid", type=int, default=256,
                    help="q grid edge for cylinder2d (smaller for profiling)")
    ap.add_argument("--dtype", default="double", choices=["double", "float32c"],
                    help="arithmetic of the timed kernel (cylinder2d, magnetic, sphere1d)")
    ap.add_argument("--split", default="q", choices=["q", "replicas"],
                    help="N > 1: split one image into contiguous q blocks (default), or "
                         "run one whole workload per GPU; --config population always "
                         "splits the sets by cost")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the secondary configurations")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the surrogate's training and measurement in the extras "
                         "(about four minutes)")
    args = ap.parse_args(argv)
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.config == "mlp":
            run_mlp(args, world, rank, local)
        elif args.config == "surrogate":
            run_surrogate(args, world, rank, local)
        elif args.config == "population":
            if world > 1:
                run_population_split(args, world, rank, local)
            else:
                run_population(args, world, rank, local)
        else:
            run_b200(args, world, rank, local)
    finally:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
