"""Benchmark: SOAP environments/s of the descriptor + force VJP step on B200.

One step is the reference's force path on one structure of the 3-species
configuration (4096 atoms, Z = {1, 6, 8} at 0.4/0.4/0.2, rho = 0.10 /A^3,
d_min = 0.9 A, poly3gauss alpha = {8,8,8}, l_max = 8, rcut 5.0/4.5, trivial
compression, central species C): get_soap with contract, then soap_contract
with an upstream gradient G ~ N(0,1).  Inputs are seeded synthetic structures
of those shapes (no dataset is involved).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --hessian N_VEC [--scale F] [--steps K] [--warmup W]
  python bench.py --neighbors [--steps K] [--warmup W]

N > 1 runs one process per GPU (torchrun): every rank processes its own
structure (sites are independent; no collective on the data path), so the
scaling is weak and the value is all ranks' sites over the slowest rank's time.
``--impl reference`` times the reference algorithm on the host cores instead:
the FP64 CPU restatement of soap_turbo's get_soap + soap_contract (the
reference is Fortran and no Fortran compiler exists on these machines).
``--hessian N_VEC`` times the central-atom Hessian (soapb_central_hessian,
the reference's get_soap_central_hessian) with N_VEC weight vectors per site
on the same structure (``--scale`` shrinks it, for profiler captures), beside
the oracle's restatement on the host cores; it prints its own JSON line.
``--neighbors`` times the device neighbour-list builder (soapb_build_neighbors)
on the benchmark structure beside the numpy builder the tests check it against.
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

METRIC = "SOAP envs/s (desc+force VJP) 1×B200: mixed/adjoint vs FP64 plain at stated err"
WORKLOAD = ("3-species Z={1,6,8} 0.4/0.4/0.2, 4096 atoms, rho=0.10/A^3, d_min=0.9 A, poly3gauss "
            "alpha={8,8,8}, l_max=8, rcut_hard=5.0, rcut_soft=4.5, compress=trivial, central Z=6")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--hessian", type=int, default=0, metavar="N_VEC",
                    help="time the central-atom Hessian with N_VEC weight vectors instead")
    ap.add_argument("--neighbors", action="store_true",
                    help="time the device neighbour-list builder instead")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="(--hessian, --quick, --fp64) scale the structure's atom count, for profiler "
                         "captures")
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 3, 4, 5],
                    help="synthetic configuration of our arm (default 2, the headline workload)")
    ap.add_argument("--quick", action="store_true",
                    help="time the two kernels only (no FP64 path, e2e, CPU baseline or peak "
                         "measurement); for profiling runs")
    ap.add_argument("--tensor-cores", default="default", choices=["default", "on", "off"],
                    help="the site kernels' contractions on the tensor cores (on), on the CUDA cores "
                         "(off), or the library's default")
    ap.add_argument("--fp64", action="store_true",
                    help="time the plain FP64 form alone (materialised soap_cart_der, then "
                         "contracted) on the configuration; for profiling runs")
    return ap.parse_args()


# the other configurations, for throughput at other sizes (--config; not the headline)
CONFIG_NAMES = {
    1: "poly3 alpha=8, l_max=8, 64 atoms in an 8 A cube, d_min=1.2 A (config 1)",
    3: "512 structures of 16-2048 atoms (log-uniform), rho 0.06-0.14, 3-species poly3gauss as "
       "config 2 (config 3)",
    4: "poly3 alpha=8, l_max=8, 32768 atoms, rho=0.11/A^3, d_min=1.2 A (config 4)",
    5: "3-species poly3gauss as config 2, 262144 atoms (config 5)",
}


def workload(rank, seed, idx=2, scale=1.0):
    from soap_turbo_b200 import synthetic as syn
    return syn.config(idx, seed=seed + 7919 * rank, scale=scale)


def cpu_model():
    """The host CPU's model name (from /proc/cpuinfo), for the CPU baseline."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def fp32_clock_peak_tflops(torch):
    """FP32 CUDA-core peak from the clock: SMs x 128 FP32 lanes x 2 (FMA) x
    the maximum SM clock nvidia-smi reports."""
    try:
        out = subprocess.run(["nvidia-smi", "-i", str(torch.cuda.current_device()),
                              "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits"],
                             capture_output=True, text=True, timeout=30).stdout
        mhz = float(out.strip().splitlines()[0])
    except (OSError, ValueError, IndexError, subprocess.SubprocessError):
        return None
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    return sms * 128 * 2 * mhz * 1e6 / 1e12


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------- reference arm
def cpu_reference_step_rate(w, seconds=10.0, max_steps=None, compare=None):
    """The oracle (FP64 C restatement of get_soap + soap_contract, OpenMP over
    all host threads) timed on the workload; returns (envs/s, threads, steps,
    errors of `compare` against it)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    hp, nl = w.hyper, w.nl
    W, S = compare["W"], compare["S"]
    G = compare["G"]
    times = []
    t_end = time.perf_counter() + seconds
    ref = pair = None
    while True:
        t0 = time.perf_counter()
        ref = O.get_soap(hp, nl, W, S, do_derivatives=True)
        pair = ref.contract(G, 1.0)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() > t_end or (max_steps and len(times) >= max_steps):
            break
    errs = {}
    if compare.get("soap") is not None:
        s = compare["soap"]
        errs["soap_max_rel"] = float((np.abs(s - ref.soap).max(1) / np.abs(ref.soap).max(1)).max())
        errs["soap_median_rel"] = float(np.median(np.abs(s - ref.soap).max(1) / np.abs(ref.soap).max(1)))
        p = compare["pair"]
        errs["vjp_max_rel"] = float(np.abs(p - pair).max() / np.abs(pair).max())
    t = statistics.median(times)
    return nl.n_sites / t, O.num_threads(), len(times), t, errs


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    w = workload(0, args.seed)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    W, S = O.basis_matrices(w.hyper)
    G = np.random.default_rng(args.seed).standard_normal((621, w.nl.n_sites))
    rate, cores, n, t, _ = cpu_reference_step_rate(
        w, seconds=1e9, max_steps=max(args.warmup, 0) + max(args.steps, 1),
        compare={"W": W, "S": S, "G": G})
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "envs/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": WORKLOAD, "sites": w.nl.n_sites,
                                         "pairs": w.nl.n_pairs},
        "cpu_baseline": {"value": rate, "unit": "envs/s", "cores": cores, "kind": "port",
                         "cpu_model": cpu_model(),
                         "sample": f"{n} full steps of the workload ({w.nl.n_sites} sites), median"},
        "e2e": {"value": rate, "unit": "envs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while it runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_flops(w):
    """The reference algorithm's operation count for one step (cnk, W
    transforms, power spectrum, H and the per-pair VJP contractions), with
    transcendentals and recursions counted as zero; see the roofline notes."""
    hp, nl = w.hyper, w.nl
    K = (hp.l_max + 1) * (hp.l_max + 2) // 2
    N = hp.n_max
    alpha = np.asarray(hp.alpha_max)
    mask = nl.mask.astype(bool)
    r = nl.rjs
    first = np.zeros(nl.n_pairs, bool)
    first[np.concatenate([[0], np.cumsum(nl.n_neigh)[:-1]])] = True
    cnt = np.zeros(len(alpha))
    for s in range(len(alpha)):
        cnt[s] = np.sum(mask[s] & (r < 5.0) & ~first)
    F_cnk = float(np.sum(cnt * 4 * alpha * K))
    F_W = float(np.sum(cnt * 4 * alpha ** 2))
    F_vjp = float(np.sum(cnt * 16 * alpha * K))
    n_keep = 69
    F_ps = nl.n_sites * 4.0 * K * n_keep
    F_H = nl.n_sites * 4.0 * N * N * K
    return {"pair": F_W, "descriptor": F_cnk + F_ps, "contract": F_H + F_vjp,
            "total": F_cnk + F_W + F_ps + F_H + F_vjp}


def algorithmic_bytes(w):
    """Bytes each kernel must move: per pair r, theta, phi (FP64) and the mask
    byte per species; per site the CSR offset, the soap row (FP64) and, for the
    contract, G (FP64), the kept c_nlm (FP32) and the pair forces out."""
    nl, hp = w.nl, w.hyper
    K = (hp.l_max + 1) * (hp.l_max + 2) // 2
    per_pair_in = 24 + hp.n_species
    n_soap = 621
    desc = nl.n_pairs * per_pair_in + nl.n_sites * (8 + 8 * n_soap + 8 * hp.n_max * K + 8)
    con = (nl.n_pairs * (per_pair_in + 24) +
           nl.n_sites * (8 + 16 * n_soap + 8 * hp.n_max * K + 8))
    return {"pair": float(nl.n_pairs * per_pair_in), "descriptor": float(desc),
            "contract": float(con)}


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)).get("hbm_gbs")
    return 6650.0


def hbm_peak_source():
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        return "measured (MEASURED_PEAKS.json)"
    return "fallback: 6.65 TB/s, an earlier copy measurement on this pool's B200s (no MEASURED_PEAKS.json)"


def gemm_peak_tflops(torch, dtype):
    """CUDA-core peak measured here: cuBLAS SGEMM with TF32 disabled (FP32)
    or DGEMM (FP64), 8192^3, best of 4."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=dtype)
    b = torch.randn(n, n, device="cuda", dtype=dtype)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    return best


def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    from soap_turbo_b200 import _lib, descriptor as D
    from soap_turbo_b200 import shard
    from soap_turbo_b200.context import Context

    dev = torch.device("cuda", torch.cuda.current_device())
    # a reduced structure only for profiler captures (--quick); timed lines use the full size
    w = workload(rank, args.seed, args.config, args.scale if args.quick else 1.0)
    wname = WORKLOAD if args.config == 2 else CONFIG_NAMES[args.config]
    if args.quick and args.scale != 1.0:
        wname += f", atoms scaled by {args.scale}"
    nl = w.nl
    ctx = Context(w.hyper)
    if args.tensor_cores != "default":
        ctx.set_tensor_cores(args.tensor_cores == "on")
    b = ctx.batch(nl)
    rng = np.random.default_rng(args.seed + rank)
    G_host = rng.standard_normal((ctx.n_soap, nl.n_sites))  # Fortran G(n_sites, n_soap)
    G = torch.as_tensor(G_host).to(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
    stream = torch.cuda.current_stream()

    def step():
        s = ctx.descriptor(b, keep=True)
        p = ctx.contract(b, s, G)
        return s, p

    # the project's autotuner picks the form (tensor or CUDA cores), CTA size and
    # persistent grid cap per site kernel; --tensor-cores on forces the tensor cores
    tune = ctx.autotune(b)
    if args.tensor_cores == "on":
        ctx.set_tensor_cores(True)
        tune["forced"] = "tensor cores"
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    # The timed step is the same two calls captured once as a CUDA graph: a
    # replay is one host launch, so the device-timed step does not include the
    # host's time to issue the calls (which, on a busy host, can exceed the
    # flush that precedes each step).  The eager loop is timed too and reported.
    soap_o = torch.empty(nl.n_sites, ctx.n_soap, dtype=torch.float64, device=dev)
    pair_o = torch.empty(nl.n_pairs, 3, dtype=torch.float64, device=dev)
    side = torch.cuda.Stream(device=dev)
    side.wait_stream(stream)
    with torch.cuda.stream(side):
        ctx.set_stream(side)
        ctx.descriptor(b, out=soap_o, keep=True)  # buffers at size: the capture allocates nothing
        ctx.contract(b, soap_o, G, out=pair_o)
    stream.wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    n0 = ctx.launch_count
    with torch.cuda.graph(graph, stream=side):
        ctx.set_stream(torch.cuda.current_stream())
        ctx.descriptor(b, out=soap_o, keep=True)
        ctx.contract(b, soap_o, G, out=pair_o)
    launches_per_step = ctx.launch_count - n0
    ctx.set_stream(stream)
    for _ in range(max(args.warmup, 3)):
        graph.replay()
    torch.cuda.synchronize()

    K = args.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(K)]
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clk:
        for i in range(K):
            flush.fill_(float(i))
            e0, e1 = ev[i]
            e0.record(stream)
            graph.replay()
            e1.record(stream)
        torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    launches = launches_per_step * K
    # the same K steps issued eagerly, call by call
    ev_eager = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                for _ in range(K)]
    for i in range(K):
        flush.fill_(float(i))
        e0, e1 = ev_eager[i]
        e0.record(stream)
        s, p = step()
        e1.record(stream)
    torch.cuda.synchronize()
    ms_eager = sum(e0.elapsed_time(e1) for e0, e1 in ev_eager) / K
    del graph

    # per-kernel device times: the same K steps again with CUDA events around
    # every kernel launch (kept out of the headline loop: each event between two
    # dependent kernels costs the step ~2 us)
    ctx.kernel_timing(4 * K + 8)
    for i in range(K):
        flush.fill_(float(i))
        step()
    ktimes = ctx.kernel_times()
    ctx.kernel_timing(0)
    kernel_ms = {k: (ktimes[k][1] / ktimes[k][0] if ktimes[k][0] else 0.0)
                 for k in ("prep", "pair", "descriptor", "contract")}
    ms_step = sum(e0.elapsed_time(e1) for e0, e1 in ev) / K
    ms_step_max = shard.max_over_ranks(ms_step, device=dev)
    value = ws * nl.n_sites / (ms_step_max * 1e-3)

    if args.quick or args.config != 2:
        if rank == 0:
            line = {"metric": METRIC, "value": value, "unit": "envs/s", "n_gpus": ws,
                    "steps": K, "warmup": args.warmup, "ms_per_step": ms_step_max,
                    "kernel_ms": kernel_ms, "autotune": tune, "gpu_launches": int(launches),
                    "dtype": "f32", "clocks": clk.summary(),
                    "config": {"workload": wname, "sites_per_gpu": nl.n_sites,
                               "pairs_per_gpu": nl.n_pairs,
                               "l2": "flushed between timed steps (256 MB write)"}}
            if args.quick:
                line["quick"] = True
            else:
                line.update(config_accuracy(args, torch, ctx, w, s, p, G_host))
            print(json.dumps(line), flush=True)
        if ws > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return

    # ---- plain FP64 GPU form (materialised soap_cart_der, then contracted)
    for _ in range(2):
        s64, cart = ctx.descriptor_fp64(b, cart=True)
        ctx.contract_cart_der(b, cart, G)
    torch.cuda.synchronize()
    t64 = []
    for _ in range(10):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s64, cart = ctx.descriptor_fp64(b, cart=True)
        p64 = ctx.contract_cart_der(b, cart, G)
        e1.record(stream)
        torch.cuda.synchronize()
        t64.append(e0.elapsed_time(e1))
    del cart
    ms64 = statistics.median(t64)

    # ---- end to end through the drop-in host API (pinned host buffers)
    def pinned(a, dtype, order="F"):
        a = np.asarray(a, dtype=dtype)
        t = torch.empty(a.size, dtype={np.float64: torch.float64, np.int32: torch.int32,
                                       np.uint8: torch.uint8}[np.dtype(dtype).type],
                        pin_memory=True)
        out = t.numpy().reshape(a.shape, order=order)
        out[...] = a
        return out, t
    hp = w.hyper
    _, _, P_i, P_j, P_el = D.get_compress_indices("trivial", hp.alpha_max, hp.l_max)
    keep = []
    h_mask, t = pinned(nl.mask.T, np.uint8); keep.append(t)
    h_rjs, t = pinned(nl.rjs, np.float64); keep.append(t)
    h_th, t = pinned(nl.thetas, np.float64); keep.append(t)
    h_ph, t = pinned(nl.phis, np.float64); keep.append(t)
    h_nn, t = pinned(nl.n_neigh, np.int32); keep.append(t)
    h_sp, t = pinned(nl.species.T, np.int32); keep.append(t)
    h_sm, t = pinned(nl.species_multiplicity, np.int32); keep.append(t)
    h_G, t = pinned(G_host.T, np.float64); keep.append(t)
    h_soap, t = pinned(np.zeros((ctx.n_soap, nl.n_sites)), np.float64); keep.append(t)
    h_pair, t = pinned(np.zeros((3, nl.n_pairs)), np.float64); keep.append(t)

    # The drop-in C ABI as a Fortran host calls it (soap_turbo_desc_b200.f90
    # passes base addresses and extents): the argument lists are built once,
    # then each step is the two calls on the pinned host arrays.
    lib = _lib.load()
    per_sp = [np.ascontiguousarray(hp.arr(n)) for n in (
        "rcut_hard", "rcut_soft", "nf", "global_scaling", "atom_sigma_r", "atom_sigma_r_scaling",
        "atom_sigma_t", "atom_sigma_t_scaling", "amplitude_scaling")]
    cw = np.ascontiguousarray(hp.arr("central_weight"))
    am = np.ascontiguousarray(hp.alpha_max, dtype=np.int32)
    Pi32, Pj32 = np.ascontiguousarray(P_i, np.int32), np.ascontiguousarray(P_j, np.int32)
    Pel64 = np.ascontiguousarray(P_el, np.float64)
    gs_args = (nl.n_sites, h_nn.ctypes.data, hp.n_species, h_sp.ctypes.data, int(h_sp.shape[0]),
               h_sm.ctypes.data, nl.n_pairs, h_mask.ctypes.data, h_rjs.ctypes.data, h_th.ctypes.data,
               h_ph.ctypes.data, am.ctypes.data, hp.l_max, *[v.ctypes.data for v in per_sp],
               hp.radial_enhancement, cw.ctypes.data, hp.basis.encode(), hp.scaling_mode.encode(), 0, 1, 1,
               len(Pi32), Pi32.ctypes.data, Pj32.ctypes.data, Pel64.ctypes.data, h_soap.ctypes.data,
               ctx.n_soap, None, 1)
    sc_args = (h_soap.ctypes.data, h_G.ctypes.data, 1.0, h_pair.ctypes.data, nl.n_sites, ctx.n_soap,
               nl.n_pairs)

    def e2e_step():
        _lib.check(lib.soapb_get_soap(*gs_args))
        _lib.check(lib.soapb_soap_contract(*sc_args))

    # the same two calls on pageable copies of every array, as a Fortran host
    # passes its allocatable arrays (the library stages them through pinned
    # buffers)
    pg = {k: np.array(v, order="F") for k, v in dict(
        nn=h_nn, sp=h_sp, sm=h_sm, mask=h_mask, rjs=h_rjs, th=h_th, ph=h_ph, G=h_G, soap=h_soap,
        pair=h_pair).items()}
    gs_pg = list(gs_args)
    for i, k in ((1, "nn"), (3, "sp"), (5, "sm"), (7, "mask"), (8, "rjs"), (9, "th"), (10, "ph")):
        gs_pg[i] = pg[k].ctypes.data
    gs_pg[len(gs_pg) - 4] = pg["soap"].ctypes.data
    sc_pg = (pg["soap"].ctypes.data, pg["G"].ctypes.data, 1.0, pg["pair"].ctypes.data, nl.n_sites,
             ctx.n_soap, nl.n_pairs)

    def e2e_step_pageable():
        _lib.check(lib.soapb_get_soap(*gs_pg))
        _lib.check(lib.soapb_soap_contract(*sc_pg))

    def e2e_step_python():  # the same two calls through the Python wrapper (descriptor.py)
        D.get_soap(nl.n_sites, h_nn, hp.n_species, h_sp, h_sm, nl.n_pairs, h_mask, h_rjs, h_th, h_ph,
                   hp.alpha_max, hp.l_max, hp.rcut_hard, hp.rcut_soft, hp.nf, hp.global_scaling,
                   hp.atom_sigma_r, hp.atom_sigma_r_scaling, hp.atom_sigma_t,
                   hp.atom_sigma_t_scaling, hp.amplitude_scaling, hp.radial_enhancement,
                   hp.central_weight, hp.basis, hp.scaling_mode, False, True, True, len(P_i), P_i,
                   P_j, P_el, h_soap, None, contract=True)
        D.soap_contract(h_soap, h_G, 1.0, h_pair)

    def wall(f, n, soap_arr):
        # The caller zeroes soap before each get_soap, as the reference's callers
        # do (a compressed soap is added into); that host write is the caller's
        # and stays outside the timed calls.
        for _ in range(3):
            soap_arr.fill(0.0)
            f()
        torch.cuda.synchronize()
        total = 0.0
        for _ in range(n):
            soap_arr.fill(0.0)
            t0 = time.perf_counter()
            f()
            total += time.perf_counter() - t0
        return total / n
    n_e2e = max(20, min(200, K // 5))
    t_e2e = shard.max_over_ranks(wall(e2e_step, n_e2e, h_soap), device=dev)
    t_e2e_py = shard.max_over_ranks(wall(e2e_step_python, n_e2e, h_soap), device=dev)
    t_e2e_pg = shard.max_over_ranks(wall(e2e_step_pageable, n_e2e, pg["soap"]), device=dev)

    # the two calls of the pinned step timed apart (wall clock, medians)
    def split_calls(n):
        tg, tc = [], []
        for _ in range(n):
            h_soap.fill(0.0)
            t0 = time.perf_counter()
            _lib.check(lib.soapb_get_soap(*gs_args))
            t1 = time.perf_counter()
            _lib.check(lib.soapb_soap_contract(*sc_args))
            t2 = time.perf_counter()
            tg.append(t1 - t0)
            tc.append(t2 - t1)
        return 1e3 * statistics.median(tg), 1e3 * statistics.median(tc)
    ms_get_soap, ms_soap_contract = split_calls(n_e2e)
    # soap_contract reads soap beside G; get_soap adds into the caller's soap,
    # whose rows come in only where they are not all zero (here the caller
    # zeroes it, so they are cleared on the device instead)
    h2d = (h_nn.nbytes + h_sp.nbytes + h_sm.nbytes + h_mask.nbytes + h_rjs.nbytes + h_th.nbytes +
           h_ph.nbytes + h_soap.nbytes + h_G.nbytes)
    d2h = h_soap.nbytes + h_pair.nbytes

    # ---- roofline of the dominant kernel: the one with the largest device time
    # per step, timed by events around each of its launches in the timed steps
    flops = algorithmic_flops(w)
    dominant = max(("pair", "descriptor", "contract"), key=lambda k: kernel_ms[k])
    t_dom = kernel_ms[dominant] * 1e-3
    peak32 = gemm_peak_tflops(torch, torch.float32)
    peak64 = gemm_peak_tflops(torch, torch.float64)
    peak32_clock = fp32_clock_peak_tflops(torch)
    # the pair kernel's arithmetic is FP64 (radial integrals, W transform)
    peak = peak64 if dominant == "pair" else peak32
    achieved = flops[dominant] / t_dom / 1e12
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get("k_" + dominant)

    result = None
    if rank == 0:
        soap_np = s.cpu().numpy()
        pair_np = p.cpu().numpy()
        W, S = ctx.basis()
        cpu_rate, cores, n_cpu, t_cpu, errs = (None, None, 0, None, {})
        if ws == 1:
            cpu_rate, cores, n_cpu, t_cpu, errs = cpu_reference_step_rate(
                w, seconds=10.0, compare={"W": W, "S": S, "G": G_host, "soap": soap_np,
                                          "pair": pair_np})
        result = {
            "metric": METRIC, "value": value, "unit": "envs/s", "n_gpus": ws, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms_step_max, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random periodic structures of the configuration's shape)",
            "config": {"workload": wname, "sites_per_gpu": nl.n_sites, "pairs_per_gpu": nl.n_pairs,
                       "step": "get_soap(do_derivatives, contract) + soap_contract(G), G~N(0,1)",
                       "precision": "FP32 pair/contraction arithmetic; R_n and dR_n/dr from "
                                    "piecewise polynomials fitted to the FP64 expansion and "
                                    "evaluated in FP32 (checked to 5e-7 at context creation); "
                                    "FP64 i_l and e^{-im phi}; FP64 accumulation of c_nlm over "
                                    "groups of 4 pairs",
                       "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"site shards, {ws} GPU(s), no data-path collective"},
            "kernel_ms": kernel_ms,
            "kernel_ms_how": "a second pass of the K steps with CUDA events around each kernel launch",
            "autotune": tune,
            "fp64_plain": {"value": nl.n_sites * ws / (ms64 * 1e-3), "unit": "envs/s",
                           "ms_per_step": ms64,
                           "what": "FP64 staged like the reference: radial, angular, c_nlm, power "
                                   "spectrum, materialised soap_cart_der, contraction with G",
                           "speedup_of_value": value / (nl.n_sites * ws / (ms64 * 1e-3))},
            "error_vs_fp64_oracle": errs,
            "e2e": {"value": ws * nl.n_sites / t_e2e, "unit": "envs/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "path": "the drop-in C ABI, soapb_get_soap(contract=1) + soapb_soap_contract, on pinned "
                            "host arrays, argument lists built once (as the Fortran shim passes them); "
                            "get_soap adds into the caller's compressed soap, as in the reference: the "
                            "caller zeroes it before each step outside the timed calls, and a host scan "
                            "inside the timed call finds its rows all zero, so they are not read back; "
                            "the site kernels write the soap rows and the pair forces into the pinned "
                            "arrays themselves (the d2h bytes cross the host link as the kernels' "
                            "stores, no copy follows); soap_contract copies soap in beside G",
                    "calls_ms": {"get_soap": ms_get_soap, "soap_contract": ms_soap_contract,
                                 "how": "median wall time of each call in a separate pass"},
                    "python_wrapper_ms_per_step": t_e2e_py * 1e3,
                    "pageable_ms_per_step": t_e2e_pg * 1e3},
            "gpu_launches": int(launches),
            "launch": "the step's two calls captured once as a CUDA graph and replayed each step "
                      f"({launches_per_step} kernels per step); issued eagerly: {ms_eager:.4f} ms per step",
            "roofline": {"bound": "fp64" if dominant == "pair" else "fp32",
                         "kernel": "k_" + dominant, "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": traffic,
                         "flops_per_launch": flops[dominant],
                         "launch_ms": kernel_ms[dominant],
                         "peak_source": "CUDA-core rate measured in this run (cuBLAS "
                                        + ("DGEMM" if dominant == "pair" else "SGEMM, TF32 off")
                                        + " 8192^3); MEASURED_PEAKS.json has HBM and bf16 "
                                          "tensor peaks only",
                         "peaks_measured_tflops": {"fp32": peak32, "fp64": peak64},
                         "fp32_clock_peak_tflops": peak32_clock,
                         "frac_of_fp32_clock_peak": (achieved / peak32_clock
                                                     if peak32_clock and dominant != "pair" else None),
                         "step": {"algorithmic_flops": flops["total"],
                                  "achieved_tflops": flops["total"] / (ms_step_max * 1e-3) / 1e12,
                                  "frac_of_fp32": flops["total"] / (ms_step_max * 1e-3) / 1e12 / peak32},
                         "hbm": {"algorithmic_bytes_per_launch": algorithmic_bytes(w).get(dominant),
                                 "algorithmic_GBps": (algorithmic_bytes(w).get(dominant) or 0.0) / t_dom / 1e9,
                                 "peak_GBps": hbm_peak(), "peak_source": hbm_peak_source()}},
            "clocks": clk.summary(),
        }
        if ws == 1:
            result["cpu_baseline"] = {"value": cpu_rate, "unit": "envs/s", "cores": cores,
                                      "kind": "port", "cpu_model": cpu_model(),
                                      "sample": f"{n_cpu} full steps ({nl.n_sites} sites) of the "
                                                f"FP64 C restatement, median {t_cpu * 1e3:.1f} ms"}
        print(json.dumps(result), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def config_accuracy(args, torch, ctx, w, soap_t, pair_t, G_host):
    """Errors of the timed step's outputs against the FP64 oracle on every site
    and pair of the configuration (the oracle over contiguous site ranges), and
    the plain FP64 GPU form beside the mixed path: on the whole configuration
    when its soap_cart_der is at most 20 GB, else (config 5) on a 16384-atom
    slice of the same configuration, both timed and both against the oracle."""
    from soap_turbo_b200 import synthetic as syn
    from soap_turbo_b200.context import Context
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    W, S = ctx.basis()
    nl = w.nl
    t0 = time.perf_counter()
    ref_soap, ref_pair = O.soap_and_vjp_chunked(w.hyper, nl, W, S, G_host)
    t_oracle = time.perf_counter() - t0
    soap, pair = soap_t.cpu().numpy(), pair_t.cpu().numpy()
    rel = np.abs(soap - ref_soap).max(1) / np.abs(ref_soap).max(1)
    out = {"error_vs_fp64_oracle": {
        "soap_max_rel": float(rel.max()), "soap_median_rel": float(np.median(rel)),
        "vjp_max_rel": float(np.abs(pair - ref_pair).max() / np.abs(ref_pair).max()),
        "coverage": f"all {nl.n_sites} sites and {nl.n_pairs} pairs",
        "oracle_s": t_oracle, "oracle_threads": O.num_threads()}}
    dev = soap_t.device
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def timed(f, n=10):
        for _ in range(2):
            f()
        torch.cuda.synchronize()
        ts = []
        for _ in range(n):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            f()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    cart_bytes = 8 * 3 * ctx.n_soap * nl.n_pairs
    if cart_bytes <= 20e9:
        sw, sctx, sb, G_s, where = w, ctx, None, G_host, "the whole configuration"
    else:
        sw = syn.config(args.config, seed=args.seed, scale=16384 / 262144)
        sctx = Context(sw.hyper)
        G_s = np.random.default_rng(args.seed).standard_normal((sctx.n_soap, sw.nl.n_sites))
        where = f"a 16384-atom slice of the configuration ({sw.nl.n_sites} sites, {sw.nl.n_pairs} pairs)"
    sb = sctx.batch(sw.nl)
    Gd = torch.as_tensor(G_s).to(dev)
    res = {}

    def mixed():
        s_ = sctx.descriptor(sb, keep=True)
        res["mixed"] = (s_, sctx.contract(sb, s_, Gd))

    def fp64():
        s_, c_ = sctx.descriptor_fp64(sb, cart=True)
        res["fp64"] = (s_, sctx.contract_cart_der(sb, c_, Gd))

    ms_mixed = timed(mixed)
    ms_fp64 = timed(fp64)
    if sw is w:
        rs, rp = ref_soap, ref_pair
    else:
        Ws, Ss = sctx.basis()
        rs, rp = O.soap_and_vjp_chunked(sw.hyper, sw.nl, Ws, Ss, G_s)
    errs = {}
    for k, (s_, p_) in res.items():
        s_, p_ = s_.cpu().numpy(), p_.cpu().numpy()
        errs[k] = {"soap_max_rel": float((np.abs(s_ - rs).max(1) / np.abs(rs).max(1)).max()),
                   "vjp_max_rel": float(np.abs(p_ - rp).max() / np.abs(rp).max())}
    n = sw.nl.n_sites
    out["fp64_plain"] = {"on": where, "ms_per_step": ms_fp64, "value": n / (ms_fp64 * 1e-3),
                         "mixed_ms_per_step": ms_mixed, "mixed_value": n / (ms_mixed * 1e-3),
                         "speedup_of_mixed": ms_fp64 / ms_mixed, "unit": "envs/s",
                         "error_vs_fp64_oracle": errs,
                         "how": "device time per step (descriptor + VJP; FP64: soap_cart_der materialised, "
                                "then contracted), L2 flushed before each step, median of 10"}
    return out


def run_hessian(args):
    """Central-atom Hessian on the benchmark structure: device time per call
    (CUDA events, inputs resident, L2 flushed between calls), the oracle's
    restatement on the host cores, and the relative error between them."""
    import torch
    from soap_turbo_b200 import synthetic as syn
    from soap_turbo_b200.context import Context
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    w = syn.config(2, seed=args.seed, scale=args.scale)
    nl, n_vec = w.nl, args.hessian
    ctx = Context(w.hyper, legacy_filter_seed=False)
    b = ctx.batch(nl)
    vecs_h = np.random.default_rng(args.seed).standard_normal((nl.n_sites, n_vec, ctx.n_soap))
    vecs = torch.as_tensor(vecs_h).to(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    out = ctx.central_hessian(b, vecs)
    for _ in range(max(args.warmup, 0)):
        ctx.central_hessian(b, vecs, out=out)
    ctx.check_inputs()
    times = []
    n0 = ctx.launch_count
    for _ in range(max(args.steps, 1)):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.central_hessian(b, vecs, out=out)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    launches = (ctx.launch_count - n0) / max(args.steps, 1)
    ms = statistics.median(times)
    W, S = ctx.basis()
    t0 = time.perf_counter()
    ref = O.get_soap(w.hyper, nl, W, S, do_derivatives=True, legacy_filter_seed=False, hessian=True)
    href, selftest = ref.central_hessian(vecs_h)
    t_cpu = time.perf_counter() - t0
    got = out.cpu().numpy()
    line = {"metric": "central-atom Hessian (get_soap_central_hessian), sites/s", "unit": "sites/s",
            "value": nl.n_sites / (ms * 1e-3), "ms_per_call": ms, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "n_vec": n_vec, "gpu_launches_per_call": launches,
            "config": {"workload": WORKLOAD + (f", atoms scaled by {args.scale}" if args.scale != 1.0 else ""),
                       "sites": nl.n_sites, "pairs": nl.n_pairs, "l2": "flushed before each call"},
            "error_vs_fp64_oracle": {"max_rel": float(np.abs(got - href).max() / np.abs(href).max()),
                                     "oracle_selftest": selftest},
            "cpu_baseline": {"value": nl.n_sites / t_cpu, "unit": "sites/s", "cores": O.num_threads(),
                             "kind": "port", "sample": f"one call on the whole structure (get_soap with "
                                                       f"second derivatives + the Hessian), {t_cpu:.3f} s"}}
    print(json.dumps(line), flush=True)


def run_neighbors(args):
    """soapb_build_neighbors on the benchmark structure: positions, cell and
    species resident on the device, the CSR batch get_soap takes out.  The
    call waits once for the pair count, so its time is the host's wall clock
    around it; the device time of its launches is reported beside it."""
    import torch
    from soap_turbo_b200 import synthetic as syn
    from soap_turbo_b200.context import Context
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    w = syn.config(2, seed=args.seed, scale=args.scale)
    st, nl = w.structures[0], w.nl
    ctx = Context(w.hyper)
    pos = torch.as_tensor(np.asarray(st.positions, np.float64)).to(dev)
    sp = torch.as_tensor((st.species + 1).astype(np.int32).reshape(-1, 1)).to(dev)
    sites = torch.as_tensor(nl.site_atom.astype(np.int32)).to(dev)
    lat = np.eye(3) * st.box
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(max(args.warmup, 3)):
        built = ctx.build_neighbors(pos, lat, sp, sites)
    torch.cuda.synchronize()
    wall, dev_ms = [], []
    n0 = ctx.launch_count
    for _ in range(max(args.steps, 1)):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record()
        built = ctx.build_neighbors(pos, lat, sp, sites)
        e1.record()
        torch.cuda.synchronize()
        wall.append((time.perf_counter() - t0) * 1e3)
        dev_ms.append(e0.elapsed_time(e1))
    launches = (ctx.launch_count - n0) / max(args.steps, 1)
    a = built.arrays()
    same = bool(np.array_equal(a["n_neigh"], nl.n_neigh))
    t0 = time.perf_counter()
    syn.neighbour_list(st, 5.0, 3, central_species=1)
    t_np = time.perf_counter() - t0
    ms = statistics.median(wall)
    line = {"metric": "neighbour-list build (soapb_build_neighbors), pairs/s", "unit": "pairs/s",
            "value": nl.n_pairs / (ms * 1e-3), "ms_per_build": ms,
            "device_ms_per_build": statistics.median(dev_ms), "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic", "gpu_launches_per_build": launches,
            "config": {"workload": WORKLOAD, "atoms": int(st.positions.shape[0]), "sites": nl.n_sites,
                       "pairs": nl.n_pairs, "l2": "flushed before each build"},
            "counts_match_numpy_builder": same,
            "cpu_baseline": {"value": nl.n_pairs / t_np, "unit": "pairs/s", "cores": 1, "kind": "port",
                             "sample": f"the numpy builder the tests compare against, one build, {t_np:.3f} s"}}
    print(json.dumps(line), flush=True)


def run_fp64(args):
    """The plain FP64 form alone on the configuration: descriptor with
    soap_cart_der materialised, then the contraction with G; device time per
    step (CUDA events, L2 flushed before each step) and per kernel kind."""
    import torch
    from soap_turbo_b200.context import Context
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    w = workload(0, args.seed, args.config, args.scale)
    nl = w.nl
    ctx = Context(w.hyper)
    b = ctx.batch(nl)
    G = torch.as_tensor(np.random.default_rng(args.seed).standard_normal((ctx.n_soap, nl.n_sites))).to(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(max(args.warmup, 3)):
        s64, cart = ctx.descriptor_fp64(b, cart=True)
        ctx.contract_cart_der(b, cart, G)
    torch.cuda.synchronize()
    times = []
    n0 = ctx.launch_count
    for _ in range(max(args.steps, 1)):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        s64, cart = ctx.descriptor_fp64(b, cart=True)
        ctx.contract_cart_der(b, cart, G)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    launches = (ctx.launch_count - n0) / max(args.steps, 1)
    ms = statistics.median(times)
    cart_bytes = 8 * 3 * ctx.n_soap * nl.n_pairs
    print(json.dumps({"metric": "plain FP64 form, envs/s", "unit": "envs/s",
                      "value": nl.n_sites / (ms * 1e-3), "ms_per_step": ms, "steps": args.steps,
                      "warmup": args.warmup, "gpu_launches_per_step": launches,
                      "soap_cart_der_bytes": cart_bytes,
                      "hbm_floor_ms": 2 * cart_bytes / (hbm_peak() * 1e9) * 1e3,
                      "hbm_peak_source": hbm_peak_source(),
                      "config": {"workload": WORKLOAD if args.config == 2 else CONFIG_NAMES[args.config],
                                 "sites": nl.n_sites, "pairs": nl.n_pairs}}), flush=True)


def main():
    args = parse()
    if args.fp64:
        run_fp64(args)
        return
    if args.neighbors:
        run_neighbors(args)
        return
    if args.hessian > 0:
        run_hessian(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
