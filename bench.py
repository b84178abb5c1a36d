"""Benchmark: COLA particle-updates/s on the 512^3-particle / 1024^3-mesh
workload (512 Mpc/h box, 2LPT at a = 0.02, 10 COLA steps to a = 1), on N
GPUs of one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one iteration of the reference's time loop (script/cola.py:37-44):
PM force at a_x (wrap, CIC deposit, R2C, 3 x (k-space gradient + C2R),
3-component CIC gather), COLA kick, COLA drift, for every particle.  Steps
follow the 10-step schedule from the 2LPT initial conditions; after the 10th
step the state is reset to the initial conditions (outside the timed
region) and the schedule starts again.

N > 1 (torchrun): every rank runs its own realization (seed + rank) on its
own GPU -- the path keeps particles and mesh on one GPU, so ranks are
independent replicas with no data-path collective; `value` sums over ranks
(weak scaling), time is the max over ranks.

--impl reference: the reference cannot be built here as it stands (MPI,
FFTW, GSL, HDF5 absent), so this arm times the CPU restatement of its loops
(oracle/, C with the reference's OpenMP pragmas, pocketfft FFTs; pinned bit
for bit to the reference's own loops) with all host threads, on the same
workload -- same ICs, same schedule, every particle -- and prints the same
metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "COLA particle-updates/s (512^3 particles, 1024^3 mesh)"


def metric_name(w):
    """The metric's name for workload w (METRIC for the default one)."""
    return "COLA particle-updates/s (%d^3 particles, %d^3 mesh)" % (w.nc, w.n)
UNIT = "particle-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="config3",
                    choices=["config1", "config3", "config5"])
    ap.add_argument("--deposit", default="atomic",
                    choices=["atomic", "deterministic"])
    ap.add_argument("--nc", type=int, default=0,
                    help="override particles per dimension (profiling runs)")
    ap.add_argument("--n", type=int, default=0,
                    help="override PM mesh cells per dimension")
    ap.add_argument("--fft-tile", type=int, default=0,
                    help="kz columns per tile of the fused FFT passes (4, 8)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--profile-range", action="store_true",
                    help="config5: run one extra graph evaluation between "
                         "cudaProfilerStart/Stop (for ncu "
                         "--profile-from-start off)")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="leave the config-5 ensemble object out of the "
                         "main line")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the API-loop, deposit and 2LPT timings "
                         "(profiling runs)")
    return ap.parse_args()


def workload(name, nc=0, n=0):
    import dataclasses
    from fs2_b200 import workloads
    w = {"config1": workloads.CONFIG1, "config3": workloads.CONFIG3}[name]
    if nc or n:
        nc = nc or w.nc
        n = n or w.n
        w = dataclasses.replace(w, name="%s_%dp_%dm" % (w.name, nc, n), nc=nc,
                                n=n, boxsize=w.boxsize * nc / w.nc)
    return w


def step_bytes(w):
    """Algorithmic bytes of one COLA step: each stage one read of its inputs
    and one write of its outputs (particles: deposit 12 B, gather 24 B, kick
    + drift 84 B; mesh: clear 4R, R2C 4R + 8K, per axis 8K + 4R, gather
    12R), R = n^3, K = n^2 (n/2+1)."""
    N, n = w.np, w.n
    R, K = n ** 3, n * n * (n // 2 + 1)
    return {
        "clear": 4 * R, "deposit": 12 * N, "r2c": 4 * R + 8 * K,
        "poisson": 3 * (8 * K + 4 * R), "gather": 24 * N + 12 * R,
        # the fused pipeline does R2C and the three axes in five passes
        "fft_fused": 4 * R + 8 * K + 3 * (8 * K + 4 * R),
        "kick_drift": 84 * N, "wrap": 0,
        "total": 120 * N + 32 * R + 32 * K,
    }


def lpt_bytes(nc):
    """Algorithmic bytes of the 2LPT initial conditions (py/lpt.cpp):
    psi(k) 3 x 8K, its derivatives 9 x 8K, 12 C2R (8K + 4R each), the
    real-space source 28R, one R2C (4R + 8K), the psi2(k) pass 32K, the
    particle loop 24R of reads and 56 bytes per particle written;
    R = nc^3, K = nc^2 (nc/2+1): 232 K + 160 R."""
    R, K = nc ** 3, nc * nc * (nc // 2 + 1)
    return 232 * K + 160 * R


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        return self.summarise(self.lines)

    @staticmethod
    def summarise(lines):
        """Median SM clock, maximum clock and the throttle reasons seen
        active in nvidia-smi CSV lines of FIELDS (no header, no units)."""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU
def cpu_steps(w, p, threads, steps=2):
    """Times the oracle (the CPU restatement of the reference's loops, all
    threads) on the first `steps` steps of the schedule from the particles'
    current state (every particle; the GPU arm's initial conditions) and
    returns the seconds of the last step and a description."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from fs2_b200 import workloads
    cosmo = oracle.Cosmology(workloads.OMEGA_M)
    a_x, a_v, _ = p.a
    st = oracle.ParticleState(p.x, p.v, p.dx1, p.dx2, p.id, a_x=a_x,
                              a_v=a_v, a_f=0.0, boxsize=w.boxsize)
    pm = oracle.PM(w.n, w.pm_factor, w.boxsize, nthreads=threads)
    t = 0.0
    for a_vel, a_pos in w.schedule()[:steps]:
        t0 = time.perf_counter()
        oracle.pm_force(st, pm)
        oracle.cola_kick(st, cosmo, a_vel, threads)
        oracle.cola_drift(st, cosmo, a_pos, threads)
        t = time.perf_counter() - t0
    desc = ("every particle (%d^3) through the full step (wrap, deposit, R2C, "
            "3 x (k-space force, C2R, gather), kick, drift) on the %d^3 mesh; "
            "step %d of the schedule from the same initial conditions (the "
            "earlier steps untimed)" % (w.nc, w.n, steps))
    return t, desc


# ------------------------------------------------------------------ adjoint
def adjoint_timing(table, reps=3, deposit="atomic"):
    """Adjoint/forward time ratio of the differentiable run on the 128^3 /
    256^3 / 128 Mpc/h / 10-step workload: CUDA-event times of
    fs2g_diff_forward (2LPT from white noise, 10 checkpointed COLA steps,
    final density) and fs2g_diff_backward (the full gradient)."""
    import torch
    from fs2_b200 import workloads
    from fs2_b200.diff import DifferentiableCOLA
    w = workloads.CONFIG4
    sim = DifferentiableCOLA(w.nc, w.n, w.boxsize, table, w.a_init,
                             w.a_final, w.nstep, workloads.OMEGA_M)
    g = torch.Generator(device="cuda").manual_seed(w.seed)
    noise = torch.randn((w.nc,) * 3, device="cuda", generator=g)
    dbar = torch.randn((w.n,) * 3, device="cuda", generator=g)
    sim.forward_raw(noise)
    sim.backward_raw(dbar)
    tf, tb = [], []
    for _ in range(reps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        sim.forward_raw(noise)
        e[1].record()
        sim.backward_raw(dbar)
        e[2].record()
        torch.cuda.synchronize()
        tf.append(e[0].elapsed_time(e[1]))
        tb.append(e[1].elapsed_time(e[2]))
    f, b = statistics.median(tf), statistics.median(tb)

    # the gradient of the config-4 loss, mean((delta - delta[seed 3])^2),
    # against central differences of this library's own float32 forward
    # along 16 random unit directions at eps = 1e-3 (the loss summed in
    # float64).  The deterministic deposit makes the forward a function of
    # its input: with the atomic deposit's summation order the differences
    # would measure that order, not the gradient.
    import fs2_b200.fs as fs

    def white(seed):
        gen = torch.Generator().manual_seed(seed)
        return torch.randn((w.nc,) * 3, generator=gen,
                           dtype=torch.float64).cuda()

    fs.pm.set_deposit_mode("deterministic")
    try:
        target = sim.forward_raw(white(3).float()).double()
        w0 = white(2)

        def loss(w_):
            return float(((sim.forward_raw(w_.float()).double() - target)
                          ** 2).mean())

        delta = sim.forward_raw(w0.float()).double()
        grad = sim.backward_raw(2.0 * (delta - target) /
                                delta.numel()).double()
        gen = torch.Generator().manual_seed(7)
        dirs = []
        for _ in range(16):
            u = torch.randn((w.nc,) * 3, generator=gen,
                            dtype=torch.float64).cuda()
            dirs.append(u / u.norm())
        ad = [float((grad * u).sum()) for u in dirs]
        fd_err = {}
        for eps in (1e-3, 1e-2, 1e-1):
            fd = [(loss(w0 + eps * u) - loss(w0 - eps * u)) / (2 * eps)
                  for u in dirs]
            fd_err["%g" % eps] = round(math.sqrt(
                sum((x - y) ** 2 for x, y in zip(fd, ad)) /
                sum(x * x for x in fd)), 6)
    finally:
        fs.pm.set_deposit_mode(deposit)
        sim.close()
    return {"ratio": round(b / f, 3), "forward_ms": round(f, 3),
            "backward_ms": round(b, 3), "workload": w.name,
            "what": "backward (adjoint of 2LPT + 10 COLA steps + CIC, "
                    "each step's force meshes from the forward's "
                    "checkpoints) / forward",
            "fd_rel_err": fd_err["0.001"], "fd_target": 1e-3,
            "fd_rel_err_by_eps": fd_err,
            "fd_what": "|fd - g.u| / |fd| over 16 random unit directions u "
                       "of the 128^3 noise, fd = central difference of the "
                       "float32 forward's loss (deterministic deposit) at "
                       "eps = 1e-3, and at 1e-2 and 1e-1 beside it.  At "
                       "eps = 1e-3 a unit direction changes the noise by "
                       "7e-7 of its norm and moves a particle by of order "
                       "1e-5 cell, the float32 rounding of a position in the "
                       "128 Mpc/h box (up to 1.5e-5 cell), so at that eps "
                       "the float32 differences are mostly rounding noise; "
                       "the error falls as eps grows.  The differences of "
                       "the float64 "
                       "restatement (tests/test_gpu_adjoint.py) give 3.8e-3 "
                       "for this adjoint and 1.5e-3 for the exact float64 "
                       "adjoint, whose gradient jumps where a particle "
                       "crosses a mesh plane"}


def extra_timings(args, w, p, ps, stream, sched, reset, world, rank, peak):
    """The drop-in API loop, the deposit in both modes at the start and the
    end of the schedule, and the 2LPT initial conditions (device times)."""
    import torch
    import fs2_b200.fs as fs
    N = w.np

    def dev_ms(fn, reps=3):
        """median CUDA-event ms of fn() on the library's stream (after one
        untimed call)"""
        fn()
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    # the drop-in loop of script/cola.py:37-44 (fs.pm.force, fs.cola.kick,
    # fs.cola.drift as separate calls) over one pass of the schedule
    reset()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for a_vel, a_pos in sched:
        fs.pm.force(p)
        fs.cola.kick(p, a_vel)
        fs.cola.drift(p, a_pos)
    e1.record(stream)
    torch.cuda.synchronize()
    api_ms = e0.elapsed_time(e1) / len(sched)
    api_loop = {"ms_per_step": round(api_ms, 4),
                "value": world * N / (api_ms / 1e3), "unit": UNIT,
                "what": "fs.pm.force + fs.cola.kick + fs.cola.drift per step, "
                        "one pass of the schedule (device time)"}

    # the deposit alone in both modes, at the initial conditions and at the
    # end of the schedule (a = 1, the most clustered positions)
    dep = {}
    for label in ("a_init", "a_final"):
        reset()
        if label == "a_final":
            for a_vel, a_pos in sched:
                fs.cola.step(p, a_vel, a_pos)
        fs.pm.send_positions(p)
        for mode in ("atomic", "deterministic"):
            fs.pm.set_deposit_mode(mode)
            dep.setdefault(mode, {})[label] = round(
                dev_ms(lambda: fs.pm.compute_density(p)), 4)
            if mode == "deterministic":
                _, tx, ty, tz = fs.pm.bin_tile()
                dep.setdefault("deterministic_bin_tile", {})[label] = \
                    "%dx%dx%d" % (tx, ty, tz)
    fs.pm.set_deposit_mode(args.deposit)

    # the whole time loop with the other deposit mode: one pass of the
    # schedule to warm up (the deterministic deposit tunes its tile and
    # keeps its counts for the one-pass binning), one timed with the stage
    # timers
    other = "deterministic" if args.deposit == "atomic" else "atomic"
    fs.pm.set_deposit_mode(other)
    try:
        for timed_pass in (False, True):
            reset()
            if timed_pass:
                fs._fs._set_timing(True)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for a_vel, a_pos in sched:
                fs.cola.step(p, a_vel, a_pos)
            e1.record(stream)
            torch.cuda.synchronize()
        st = fs._fs._get_timing()
    finally:
        fs._fs._set_timing(False)
        fs.pm.set_deposit_mode(args.deposit)
    dep["loop_" + other] = {
        "ms_per_step": round(e0.elapsed_time(e1) / len(sched), 4),
        "deposit_ms_per_step": round(st.get("deposit", (0.0, 0))[0] /
                                     len(sched), 4),
        "what": "fs.cola.step over the schedule with the %s deposit "
                "(the main line's stages are the %s deposit's)"
                % (other, args.deposit)}

    # 2LPT initial conditions of the workload (fs.lpt.init, one call)
    def lpt_once():
        q = fs.lpt.init(w.nc, w.boxsize, w.a_init, ps, w.seed + rank, "cola")
        torch.cuda.synchronize()
        del q
    lpt_ms = dev_ms(lpt_once)
    # the same call with the library's stage timers: its kernels alone
    # (the allocation of the scratch meshes and of the particle set, and
    # their release, left out)
    fs._fs._set_timing(True)
    try:
        lpt_once()
        st = fs._fs._get_timing()
    finally:
        fs._fs._set_timing(False)
    kern_ms = sum(st[k][0] for k in ("lpt_k", "lpt_fft", "lpt_real",
                                     "lpt_particles") if k in st)
    lb = lpt_bytes(w.nc)
    lpt = {"ms": round(lpt_ms, 3), "algorithmic_bytes": lb,
           "achieved_gbs": round(lb / (lpt_ms / 1e3) / 1e9, 1),
           "frac": round(lb / (lpt_ms / 1e3) / 1e9 / peak, 4),
           "kernels_ms": round(kern_ms, 3),
           "kernels_frac": round(lb / (kern_ms / 1e3) / 1e9 / peak, 4)
           if kern_ms > 0 else None,
           "what": "fs.lpt.init(%d, %g, a=%g, kind='cola'): draws, psi(k), "
                   "2LPT source, 12 C2R + 1 R2C, particle grid (device "
                   "time, allocation of the particle set included; "
                   "kernels_ms: the stages' kernels alone)"
                   % (w.nc, w.boxsize, w.a_init)}
    return api_loop, dep, lpt


# ------------------------------------------------------------------ ours
def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    import ctypes as C

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    os.environ["FS2_DEVICE"] = str(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(minutes=10))

    import fs2_b200.fs as fs
    from fs2_b200 import capi, workloads
    w = workload(args.config, args.nc, args.n)
    N = w.np
    fs.cosmology.init(workloads.OMEGA_M)
    ps = fs.PowerSpectrum(workloads.eh_table_path())
    # a dedicated stream: the library's kernels and the timing events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    fs._fs._set_stream(stream.cuda_stream)
    fs.pm.set_deposit_mode(args.deposit)
    if args.fft_tile:
        fs.pm.set_fft_tile(args.fft_tile)

    p = fs.lpt.init(w.nc, w.boxsize, w.a_init, ps, w.seed + rank, "cola")
    fs.pm.init(w.n, w.pm_factor, w.boxsize)
    paddr = C.c_void_p(fs._fs._particles_address(p._particles))
    caddr = C.c_void_p(fs._fs._ctx_address())

    # device views of the particle planes, for resets to the ICs
    base, stride = C.c_void_p(), C.c_size_t()
    capi.call("fs2g_particles_device_field", paddr, capi.FIELD_X,
              C.byref(base), C.byref(stride))

    class _Dev:
        def __init__(self, ptr, nbytes):
            self.__cuda_array_interface__ = {
                "shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                "version": 3}

    planes = torch.as_tensor(_Dev(base.value, 15 * stride.value * 4),
                             device="cuda")
    ic = planes.clone()

    def reset():
        torch.cuda.synchronize()
        planes.copy_(ic)
        p.set_a(w.a_init, w.a_init, 0.0)
        torch.cuda.synchronize()

    sched = w.schedule()

    def run_steps(k, timing_events=None):
        """k steps along the schedule; returns device ms (sum of segments)."""
        done, total_ms = 0, 0.0
        while done < k:
            seg = min(k - done, len(sched))
            reset()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for a_vel, a_pos in sched[:seg]:
                fs.cola.step(p, a_vel, a_pos)
            e1.record(stream)
            torch.cuda.synchronize()
            total_ms += e0.elapsed_time(e1)
            done += seg
        return total_ms

    # warm-up
    run_steps(args.warmup)
    # timed
    clocks = ClockSampler(local)
    fs._fs._set_timing(True)
    launches0 = fs._fs._kernel_launches()
    clocks.start()
    t_ms = run_steps(args.steps)
    clk = clocks.stop()
    launches = fs._fs._kernel_launches() - launches0
    stages = fs._fs._get_timing()
    fs._fs._set_timing(False)
    t_max = torch.tensor([t_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    t_ms = float(t_max.item())
    ms_per_step = t_ms / args.steps
    value = world * N * args.steps / (t_ms / 1e3)

    # roofline of the dominant stage group
    import json as _json
    peaks = {}
    try:
        peaks = _json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        peak, peak_src = 6650.0, "fallback"
    B = step_bytes(w)
    groups = {
        "clear": ["clear"], "deposit": ["deposit", "sort"], "r2c": ["r2c"],
        "poisson": ["force_k", "c2r"],
        "fft_fused": ["fz", "fy", "xx", "iy", "iz"],
        "gather": ["gather"],
        "kick_drift": ["kick_drift"], "wrap": ["wrap"],
    }
    per_launch = {"clear": 1, "deposit": 1, "r2c": 1, "poisson": 3,
                  "fft_fused": 1,
                  "gather": 1, "kick_drift": 1, "wrap": 1}
    gtime = {g: sum(stages.get(s, (0.0, 0))[0] for s in ss)
             for g, ss in groups.items()}
    stage_ms = {g: round(v / args.steps, 4) for g, v in gtime.items()}
    dom = max((g for g in gtime if B.get(g, 0) > 0), key=lambda g: gtime[g])
    launches_dom = args.steps * per_launch[dom]
    dur_s = gtime[dom] / 1e3 / launches_dom
    bytes_launch = B[dom] / per_launch[dom]
    achieved = bytes_launch / dur_s / 1e9
    # DRAM traffic of the dominant group's kernels, from the committed ncu
    # launch list of this workload (one capture; per launch)
    traffic = None
    try:
        tj = _json.load(open(os.path.join(
            ROOT, "profiles", "ncu_traffic_cola_step_512p_1024m.json")))
        if tj["workload"] == w.name and dom in tj["group_traffic_bytes"]:
            traffic = int(tj["group_traffic_bytes"][dom]) // per_launch[dom]
    except (OSError, KeyError, ValueError):
        pass
    roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1),
            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic, "peak_source": peak_src + " hbm_gbs",
            "algorithmic_bytes_per_launch": int(bytes_launch),
            "step_achieved_gbs": round(B["total"] / (ms_per_step / 1e3) / 1e9, 1),
            "step_frac": round(B["total"] / (ms_per_step / 1e3) / 1e9 / peak, 4)}

    # end to end through the C ABI with pinned host buffers: H2D of the
    # initial state (x, v, dx1, dx2), the steps, D2H of the final x and v
    e2e = None
    if not args.no_e2e:
        host = {}
        for name, field in (("x", capi.FIELD_X), ("v", capi.FIELD_V),
                            ("dx1", capi.FIELD_DX1), ("dx2", capi.FIELD_DX2)):
            t = torch.empty((N, 3), dtype=torch.float32, pin_memory=True)
            capi.call("fs2g_particles_copy_out", paddr, field,
                      C.c_void_p(t.data_ptr()), 0, N)
            host[name] = t
        reset()
        for name, field in (("x", capi.FIELD_X), ("v", capi.FIELD_V),
                            ("dx1", capi.FIELD_DX1), ("dx2", capi.FIELD_DX2)):
            capi.call("fs2g_particles_copy_out", paddr, field,
                      C.c_void_p(host[name].data_ptr()), 0, N)
        out_x = torch.empty((N, 3), dtype=torch.float32, pin_memory=True)
        out_v = torch.empty((N, 3), dtype=torch.float32, pin_memory=True)
        k = min(args.steps, len(sched))
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for name, field in (("x", capi.FIELD_X), ("v", capi.FIELD_V),
                            ("dx1", capi.FIELD_DX1), ("dx2", capi.FIELD_DX2)):
            capi.call("fs2g_particles_copy_in", paddr, field,
                      C.c_void_p(host[name].data_ptr()), 0, N)
        capi.call("fs2g_particles_set_a", paddr, w.a_init, w.a_init, 0.0)
        for a_vel, a_pos in sched[:k]:
            capi.call("fs2g_cola_step", caddr, paddr, a_vel, a_pos)
        capi.call("fs2g_particles_copy_out", paddr, capi.FIELD_X,
                  C.c_void_p(out_x.data_ptr()), 0, N)
        capi.call("fs2g_particles_copy_out", paddr, capi.FIELD_V,
                  C.c_void_p(out_v.data_ptr()), 0, N)
        torch.cuda.synchronize()
        t_e2e = time.perf_counter() - t0
        te = torch.tensor([t_e2e], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        t_e2e = float(te.item())
        e2e = {"value": world * N * k / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": int(48 * N / k),
               "d2h_bytes_per_step": int(24 * N / k),
               "steps": k, "seconds": round(t_e2e, 4),
               "what": "fs2g_particles_copy_in of x, v, dx1, dx2 from pinned "
                       "host memory, %d fs2g_cola_step calls, "
                       "fs2g_particles_copy_out of x and v" % k}

    api_loop = dep = lpt = None
    if not args.no_extra:
        api_loop, dep, lpt = extra_timings(args, w, p, ps, stream, sched,
                                           reset, world, rank, peak)

    cpu = None
    if rank == 0 and not args.no_cpu and world == 1:
        threads = len(os.sched_getaffinity(0))
        reset()
        t_step, desc = cpu_steps(w, p, threads)
        cpu = {"value": N / t_step, "unit": UNIT, "cores": threads,
               "kind": "port", "sample": desc,
               "seconds_per_step": round(t_step, 3)}

    adj = None
    if rank == 0 and not args.no_adjoint:
        adj = adjoint_timing(workloads.eh_table_path(), deposit=args.deposit)

    ens = None
    if rank == 0 and world == 1 and not args.no_ensemble:
        ens = ensemble_timing(stream, peak)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": metric_name(w), "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": w.name, "particles": "%d^3" % w.nc,
                   "mesh": "%d^3" % w.n, "boxsize_mpc_h": w.boxsize,
                   "a_init": w.a_init, "a_final": w.a_final,
                   "schedule_steps": w.nstep, "deposit": args.deposit,
                   "pk": "Eisenstein-Hu no-wiggle, sigma8=0.81",
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": ("inputs larger than L2" if 60 * N + 4 * w.n ** 3
                          > 126e6 else "inputs within L2 (no flush: a "
                          "parity-size case, not a bench line)")
                         + " (particles %.3f GB, mesh %.3f GB)"
                         % (60 * N / 1e9, 4 * w.n ** 3 / 1e9)},
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clk,
        "stages_ms_per_step": stage_ms,
        "stages_raw_ms_per_step": {k: round(v[0] / args.steps, 4)
                                   for k, v in stages.items()},
        "adjoint_forward_ratio": adj["ratio"] if adj else None,
        "adjoint": adj,
        "api_loop": api_loop,
        "deposit_ms": dep,
        "lpt": lpt,
        "ensemble": ens,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ reference arm
# ------------------------------------------------------------- ensemble
def _ensemble_setup(members, nsteps):
    """The config-5 ensemble over `members`: targets from the forward of
    seed + 1000, white noise from seed (host copies pinned for e2e)."""
    import torch
    from fs2_b200 import workloads
    from fs2_b200.ensemble import Ensemble
    ens = Ensemble(members, workloads.eh_table_path(), 0.1, 1.0, nsteps,
                   workloads.OMEGA_M, autotune=True)
    host_w, host_g = [], []
    for i, m in enumerate(members):
        g = torch.Generator().manual_seed(m.seed + 1000)
        ens.set_noise(i, torch.randn((m.nc,) * 3, generator=g).cuda())
        ens.set_target(i, ens.forward_member(i).clone())
        g = torch.Generator().manual_seed(m.seed)
        host_w.append(torch.randn((m.nc,) * 3, generator=g).pin_memory())
        host_g.append(torch.empty((m.nc,) * 3).pin_memory())
        ens.set_noise(i, host_w[i].cuda())
    torch.cuda.synchronize()
    return ens, host_w, host_g


def ensemble_timing(stream, peak, reps=3):
    """The config-5 ensemble (48 realisations, 5 COLA steps + adjoint) on
    this GPU for the main line: graph replays timed with CUDA events, the
    looped plain path once beside them."""
    import torch
    from fs2_b200.ensemble import (config5_members, eval_bytes,
                                   step_bytes as member_bytes)
    members = config5_members()
    nsteps = 5
    ens, _, _ = _ensemble_setup(members, nsteps)

    def timed(k, graph):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            ens.run(graph=graph)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    try:
        timed(1, True)                  # capture
        t_graph = timed(reps, True)
        timed(1, False)                 # the unbatched runs are made here
        t_loop = timed(1, False)
        kernels = ens.graph_kernels()
        tun = ens.tuning()
    finally:
        ens.close()
    fwd_bytes = sum(nsteps * member_bytes(m) for m in members)
    achieved = fwd_bytes / (t_graph / 1e3) / 1e9
    all_bytes = sum(eval_bytes(m, nsteps) for m in members)
    achieved_all = all_bytes / (t_graph / 1e3) / 1e9
    return {"workload": "ensemble48_5step", "ms_per_eval": round(t_graph, 3),
            "value": round(len(members) / (t_graph / 1e3), 1),
            "unit": "realisation-gradients/s",
            "loop_ms_per_eval": round(t_loop, 3),
            "graph_speedup_vs_loop": round(t_loop / t_graph, 3),
            "graph_kernels": kernels,
            "chunks": sorted({"n=%d: %d members per chunk" % (m.n, t[1])
                              for m, t in zip(members, tun)}),
            "fwd_frac": round(achieved / peak, 4),
            "frac": round(achieved_all / peak, 4),
            "algorithmic_bytes": all_bytes,
            "what": "48 realisations (16 each of 32^3/64^3, 64^3/128^3, "
                    "96^3/192^3): 2LPT from white noise, 5 COLA steps, "
                    "density MSE loss and its adjoint to the noise, per "
                    "evaluation; size classes as batched chunks replayed "
                    "as one CUDA graph; loop = each member alone through "
                    "the unbatched path; frac: forward, adjoint and "
                    "2LPT algorithmic bytes (fs2_b200.ensemble.eval_bytes) "
                    "over the measured HBM peak; fwd_frac: the forward's "
                    "algorithmic bytes only, over the measured HBM peak"}


def run_ensemble(args):
    """Config 5: 48 realisations (16 each of 32^3/64^3, 64^3/128^3 and
    96^3/192^3), 5 COLA steps from a = 0.1 to 1, the density MSE loss and
    its gradient with respect to the white noise, per member.  Each rank
    takes its greedy shard (fs2_b200.ensemble.shard).  A step is one
    evaluation of every member; timed as graph replays (one launch), with
    the looped plain path timed beside it."""
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    os.environ["FS2_DEVICE"] = str(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(minutes=10))
    import fs2_b200.fs as fs
    from fs2_b200 import workloads
    from fs2_b200.ensemble import config5_members, eval_bytes, shard
    fs.cosmology.init(workloads.OMEGA_M)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    fs._fs._set_stream(stream.cuda_stream)
    members = config5_members()
    mine = shard(members, world, rank)
    nsteps = 5
    ens, host_w, host_g = _ensemble_setup(mine, nsteps)

    def timed(k, graph, e2e=False):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            if e2e:
                for i in range(len(mine)):
                    ens.noise(i).copy_(host_w[i], non_blocking=True)
            ens.run(graph=graph)
            if e2e:
                for i in range(len(mine)):
                    host_g[i].copy_(ens.gradient(i), non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64,
                         device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    timed(args.warmup, True)
    if args.profile_range:
        # one more evaluation between cudaProfilerStart/Stop, for
        # ncu --profile-from-start off (not part of any timed figure)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        ens.run(graph=True)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    timed(1, False)
    clocks = ClockSampler(local)
    clocks.start()
    t_graph = timed(args.steps, True)
    clk = clocks.stop()
    launches = ens.graph_kernels() * args.steps
    t_loop = timed(args.steps, False)
    t_e2e = timed(args.steps, True, e2e=True)
    losses = ens.losses()
    tun = ens.tuning()
    ens.close()
    total = len(members)
    value = total * args.steps / (t_graph / 1e3)
    all_bytes = sum(eval_bytes(m, nsteps) for m in members)
    try:
        import json as _json
        peak = float(_json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
        peak_src = "measured hbm_gbs"
    except (OSError, KeyError, ValueError):
        peak, peak_src = 6650.0, "fallback hbm_gbs"
    h2d = sum(4 * m.nc ** 3 for m in mine)
    if rank == 0:
        achieved = all_bytes / (t_graph / args.steps / 1e3) / 1e9
        print(json.dumps({
            "metric": "ensemble gradients/s (48 realisations x 5 COLA steps "
                      "+ adjoint)",
            "value": value, "unit": "realisation-gradients/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_graph / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "ensemble48_5step",
                       "members": "16 x 32^3/64^3 L32, 16 x 64^3/128^3 L64, "
                                  "16 x 96^3/192^3 L96, seeds 100-147",
                       "parallelism": "greedy shards over %d rank(s)" % world,
                       "l2": "members' working sets exceed L2 in total"},
            "loop": {"ms_per_step": t_loop / args.steps,
                     "what": "the same members looped one after another on "
                             "one stream"},
            "graph_speedup_vs_loop": round(t_loop / t_graph, 3),
            "roofline": {"bound": "hbm", "kernel": "ensemble evaluation "
                         "(forward, loss, adjoint)",
                         "achieved": round(achieved, 1),
                         "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None,
                         "peak_source": peak_src,
                         "algorithmic_bytes_per_step": all_bytes,
                         "model": "fs2_b200.ensemble.eval_bytes: per member "
                                  "5 x (forward step 120 N + 32 R + 32 K + "
                                  "backward step 240 N + 68 R + 64 K) + 3 x "
                                  "2LPT (232 K + 160 R at nc) + loss 16 R"},
            "cpu_baseline": None,
            "e2e": {"value": total * args.steps / (t_e2e / 1e3),
                    "unit": "realisation-gradients/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
            "gpu_launches": launches,
            "clocks": clk,
            "autotune": sorted({"n=%d: %s, %d members per chunk"
                                % (m.n, t[0], t[1])
                                for m, t in zip(mine, tun)}),
            "loss_mean": float(np.mean(losses)),
        }), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_reference(args):
    """The CPU arm: the oracle's restatement of the reference's loops (C with
    the reference's OpenMP pragmas -- atomics in the deposit --, pocketfft
    FFTs in float32, all host threads) through the same workload as the GPU
    arm: the same 2LPT initial conditions (the same draws, P(k) and seed),
    the same 10-step schedule restarted from the ICs after its last step,
    every particle in every step.  Each step is the reference's time loop
    (script/cola.py:37-44): wrap, density, force, kick, drift."""
    if args.config == "config5":
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"impl": "reference", "unavailable":
                              "the ensemble's adjoint has no CPU counterpart "
                              "in the reference or the oracle port"}),
                  flush=True)
        return
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from fs2_b200 import workloads
    w = workload(args.config, args.nc, args.n)
    threads = len(os.sched_getaffinity(0))
    table = workloads.eh_table_path()
    t0 = time.perf_counter()
    up, ua = workloads.lpt_draws(w.nc, w.seed)
    cosmo = oracle.Cosmology(workloads.OMEGA_M)
    ic = oracle.lpt(w.nc, w.boxsize, w.a_init, up, ua,
                    oracle.PowerSpectrum(table), cosmo, "cola",
                    workers=threads)
    del up, ua
    t_ic = time.perf_counter() - t0
    pm = oracle.PM(w.n, w.pm_factor, w.boxsize, nthreads=threads)
    sched = w.schedule()
    st = ic.copy()
    times = []
    for s_ in range(args.warmup + args.steps):
        k = s_ % len(sched)
        if k == 0 and s_ > 0:
            st = ic.copy()                       # restart the schedule
        a_vel, a_pos = sched[k]
        t0 = time.perf_counter()
        oracle.pm_force(st, pm)
        oracle.cola_kick(st, cosmo, a_vel, threads)
        oracle.cola_drift(st, cosmo, a_pos, threads)
        dt = time.perf_counter() - t0
        if s_ >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = w.np * len(times) / total
    desc = ("every particle (%d^3) through the full step (wrap, CIC deposit, "
            "R2C, 3 x (k-space force, C2R, gather), kick, drift) along the "
            "%d-step schedule from the same 2LPT ICs; no sampling"
            % (w.nc, len(sched)))
    print(json.dumps({
        "impl": "reference", "metric": metric_name(w), "value": value, "unit": UNIT,
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / len(times), 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": w.name, "particles": "%d^3" % w.nc,
                   "mesh": "%d^3" % w.n, "boxsize_mpc_h": w.boxsize,
                   "a_init": w.a_init, "a_final": w.a_final,
                   "schedule_steps": w.nstep, "deposit": "atomic",
                   "pk": "Eisenstein-Hu no-wiggle, sigma8=0.81",
                   "parallelism": "OpenMP, %d threads" % threads},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                         "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "step_seconds": {"min": round(min(times), 3),
                         "median": round(statistics.median(times), 3),
                         "max": round(max(times), 3)},
        "ic_seconds": round(t_ic, 1),
        "note": "the reference's own build needs MPI, FFTW3, GSL and HDF5, "
                "none of which is installed; this times the oracle's C "
                "restatement of its loops (pinned bit for bit to the "
                "reference's loops compiled from its sources, with the "
                "reference's OpenMP pragmas) with pocketfft FFTs",
    }), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "config5":
        run_ensemble(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
