"""Cloth-step benchmark: vertex-substeps/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config cfg2]

Workload (default): the 256x256 self-colliding drape (65,536 vertices, 1.5 m)
dropped 0.5 m onto a level-5 icosphere mesh collider (10,242 vertices, 20,480
triangles, radius 0.25 m) standing on a ground plane; mesh contacts through the
collider's AABB tree, continuous self-collision, 8 substeps x 20 iterations per
frame (scenes.cfg2). One "step" is one frame, i.e. one scStepCloth(1/60) call =
8 substeps, in both arms. Multi-GPU (torchrun, one process per GPU) runs
independent replicas (a single cloth does not shard): scaling is weak and
`value` is the sum over ranks of the device-timed throughput, using the max time
over ranks. --config cfg3 steps the 512 uneven instances as one batch patch;
under torchrun the instances are partitioned over the ranks (no collective on
the data path, strong scaling) and `value` is all instances' vertex-substeps
over the slowest rank's time.

The line's `learned` object compares the plain solver with the learned warm
start (solidcloth_b200/data/warmstart.npz) on held-out drapes: Gauss-Seidel
iterations a substep to the residual target and vertex-substeps/s.

Timing: W untimed frames, then K frames each bracketed by CUDA events on the
patch's stream; L2 is flushed (a 256 MiB write) before every timed frame,
outside the events. `e2e` replays the same K frames (from the state the timed
frames started from) through the C ABI with host buffers: the state is uploaded
from pinned host memory before each frame and read back after it, wall-clock
timed, so e2e against `value` is the cost of the transfers and the host calls.
SM clocks and throttle reasons are sampled through NVML every 10 ms during the
timed frames.

--impl reference times the SolidCloth reference's own CPU step (compiled from
its sources into oracle/_ref, OpenMP on all host threads) on the same frames:
W untimed frames from the same initial state, then K timed frames, one frame
(8 substeps) per step, with the same `config`.
"""
from __future__ import annotations

import argparse
import contextlib
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
sys.path.insert(0, str(ROOT))

METRIC = "cloth vertex-substeps/s on 1 B200; learned vs plain iters at equal residual"
UNIT = "vertex-substeps/s"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--self", dest="self_mode", default="ccd", choices=["ccd", "proximity", "both"],
                    help="self-collision: the continuous detector (default), the live proximity path, or both")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg2", choices=["cfg0", "cfg1", "cfg2", "cfg3"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--direct", action="store_true",
                    help="launch the kernels one by one instead of replaying the frame graph (for profilers); "
                         "the in-graph section timing is then empty")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the plain-vs-learned warm-start comparison")
    ap.add_argument("--instances", type=int, default=512, help="cfg3: number of instances (the first K of the 512)")
    ap.add_argument("--precision", default="default", choices=["default", "ieee", "fast"],
                    help="solver numerics (scSetSolverPrecision): the library default, IEEE or the fast build")
    return ap.parse_args()


def _scene(name, self_mode="ccd"):
    from solidcloth_b200 import scenes
    return scenes.CONFIGS[name]() if name == "cfg0" else scenes.CONFIGS[name](self_mode=self_mode)


class _Batch:
    """cfg3: the rank's share of the 512 uneven instances, as one batch patch"""

    def __init__(self, insts, rank, ws):
        from solidcloth_b200.shard import shard
        self.all = insts
        self.mine = shard(insts, rank, ws)
        s0 = self.mine[0]
        self.name = f"cfg3_512_uneven_instances_rank{rank}of{ws}"
        self.n = 0
        self.params = s0.params
        self.dt = s0.dt
        self.ccd = s0.ccd
        self.num_vertices = sum(s.num_vertices for s in self.mine)
        self.sdfs, self.meshes, self.walls = s0.sdfs, s0.meshes, None


def _workload(sc):
    if isinstance(sc, _Batch):
        return {"workload": f"cfg3: {len(sc.all)} independent cloths, sides log-uniform in [16, 128] "
                            f"({sum(s.num_vertices for s in sc.all)} vertices in all, {sc.num_vertices} on this rank, "
                            f"{len(sc.mine)} instances), own 32^3 sphere SDF each, 1-4 pinned corners, continuous "
                            f"self-collision, {sc.params.substeps} substeps x {sc.params.iterations} iterations per frame, "
                            f"one batch patch (one graph per frame, one solver launch per substep)",
                "flags": sc.params.flags, "iterations": "fixed",
                "l2": "flushed (256 MiB write) before every timed frame; the batch state (~30 MB/1M vertices) exceeds L2 anyway",
                "step": f"one frame = one scStepCloth(1/60) call on the batch ({sc.params.substeps} substeps)"}
    return {"workload": f"{sc.name}: {sc.n}x{sc.n} grid ({sc.num_vertices} vertices), "
                        f"{sc.params.substeps} substeps x {sc.params.iterations} iterations per frame, dt 1/60",
            "flags": sc.params.flags, "colliders": {"sdf": len(sc.sdfs), "mesh": len(sc.meshes),
                                                      "walls": sc.walls is not None},
            "iterations": "fixed", "l2": "flushed (256 MiB write) before every timed frame",
            "step": f"one frame = one scStepCloth(1/60) call ({sc.params.substeps} substeps)"}


def _peaks():
    """HBM copy bandwidth (GB/s) of this pool's B200s and where it comes from"""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    return 6650.0, "fallback (MEASURED_PEAKS.json absent: an earlier copy measurement on this pool)"


class Clocks:
    """SM clock and throttle-reason sampler running during the timed region:
    NVML read every 10 ms from a thread (nvidia-smi -lms 50 as the fallback)."""

    # NVML clocks-event reason bits
    _REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
                "sw_power_cap": 0x4}

    def __init__(self, index: int):
        self.index = index
        self.rows = []          # (sm MHz, max sm MHz, reason bits)
        self.proc = None
        self.path = None
        self._stop = None
        self._thread = None

    def _nvml_loop(self, nv, h):
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), int(bits)))
            except Exception:
                pass
            self._stop.wait(0.01)

    def __enter__(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = None
            try:
                # the CUDA device's own GPU (NVML numbers GPUs without CUDA_VISIBLE_DEVICES)
                import torch
                pr = torch.cuda.get_device_properties(self.index)
                h = nv.nvmlDeviceGetHandleByPciBusId(
                    f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0".encode())
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self._stop = threading.Event()
            self._thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self._thread.start()
            return self
        except Exception:
            self._thread = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        if self._thread is not None:
            if not self.rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
            reasons = sorted({n for _, _, b in self.rows for n in names if b & self._REASONS[n]})
            return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": max(r[1] for r in self.rows),
                    "reasons": reasons, "samples": len(self.rows), "source": "NVML every 10 ms"}
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        for r in rows:
            for k, n in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows), "source": "nvidia-smi -lms 50"}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


@contextlib.contextmanager
def _reference_output_to_stderr():
    """The reference's C++ prints diagnostics (printf) while it sets a cloth up;
    send file descriptor 1 to stderr meanwhile, so stdout carries only the JSON line."""
    import ctypes as C
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        C.CDLL(None).fflush(None)          # the C library's buffered stdout goes to stderr too
        os.dup2(saved, 1)
        os.close(saved)


def cpu_reference_rate(sc, frames: int = 1, serial: bool = False, substeps: int | None = None):
    """Time the reference's own CPU step (oracle/_ref) on a bounded sample of the
    workload: `frames` whole frames (scStepCloth(1/60), all substeps) from the
    scene's initial state, or, with `substeps`, that many single substeps from
    it. serial=True: the build without OpenMP (one thread, as the reference's
    C-ABI library); else the OpenMP build on all host threads.
    Returns (vertex-substeps/s, seconds, threads)."""
    import ctypes as C
    from oracle.bridge import RefCloth, _load, REF_LIB, REF_SERIAL_LIB
    cores = 1 if serial else _load(REF_LIB, "ref_").ref_max_threads()
    r = RefCloth.from_scene(sc, serial=serial)
    if substeps:
        # one substep per call: a patch with numSteps = 1 and dt = h
        pa = sc.params.as_array().copy()
        pa[9] = 1
        r._fn("set_params")(r.h, pa.ctypes.data_as(C.POINTER(C.c_float)), pa.size)
        h, calls, per_call = sc.dt / sc.params.substeps, substeps, 1
    else:
        h, calls, per_call = sc.dt, frames, sc.params.substeps
    t0 = time.perf_counter()
    for _ in range(calls):
        r.step(h)
    dt = time.perf_counter() - t0
    r.close()
    return sc.num_vertices * calls * per_call / dt, dt, int(cores)


def _cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    from oracle.bridge import available
    if not available("ref"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libscref.so not built (reference sources absent at build time)"}))
        return
    from oracle.bridge import RefCloth, _load, REF_LIB
    lib = _load(REF_LIB, "ref_")
    cores = lib.ref_max_threads()
    if args.config == "cfg3":
        # a bounded sample of the batch: 8 instances spread over the list, one frame each per step
        from solidcloth_b200 import scenes
        insts = scenes.cfg3_instances()[:args.instances]
        sample = insts[::max(1, len(insts) // 8)][:8]
        work = _Batch(insts, 0, 1)
        label = f"{len(sample)} of the {len(insts)} cfg3 instances ({sum(x.num_vertices for x in sample)} vertices)"
    else:
        sample = [_scene(args.config, args.self_mode)]
        work = sample[0]
        label = sample[0].name
    clothes = []
    times = []
    with _reference_output_to_stderr():
        for sc in sample:
            clothes.append(RefCloth.from_scene(sc))
        # the same frames as the GPU arm: W untimed frames from the initial state, then K timed ones
        for _ in range(args.warmup):
            for r, sc in zip(clothes, sample):
                r.step(sc.dt)
        for _ in range(args.steps):
            t0 = time.perf_counter()
            for r, sc in zip(clothes, sample):
                r.step(sc.dt)
            times.append(time.perf_counter() - t0)
    tot = sum(times)
    subs = sample[0].params.substeps
    value = sum(sc.num_vertices for sc in sample) * subs * args.steps / tot
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "strong" if args.config == "cfg3" else "weak", "vs_baseline": None,
            "dtype": "fp32", "data": "synthetic", "config": _workload(work),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "cpu": _cpu_model(),
                             "sample": f"frames {args.warmup + 1}-{args.warmup + args.steps} of {label} (one frame = "
                                       f"{subs} substeps per step) after {args.warmup} untimed frames from the initial "
                                       f"state, the reference's own C++ (oracle/_ref), OpenMP threads = {cores}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _learned_ab(drapes: int = 4, n: int = 256):
    """iterations a substep to the residual target (update residual: the largest
    particle displacement of a Gauss-Seidel iteration, <= 1e-4 m, cap 200) and
    device-timed vertex-substeps/s, plain versus learned warm start, on held-out
    256 x 256 drapes (the first of learned.TEST_SEEDS: seeds neither the training
    nor the output-scale calibration saw)"""
    from solidcloth_b200 import learned
    path = ROOT / "solidcloth_b200" / "data" / "warmstart.npz"
    if not path.exists():
        return {"unavailable": "no trained weights (python -m solidcloth_b200.learned)"}
    z = np.load(path)
    params, norm = z["params"].astype(np.float32), z["norm"].astype(np.float32)
    tol, cap = 1e-4, 200
    seeds = learned.TEST_SEEDS[:drapes]
    rows = [learned.compare([learned.drape_scene(sd, n)], params, norm, frames=3, skip=4, tol=tol, max_iter=cap)
            for sd in seeds]
    per = [{"seed": sd, "plain": r["plain"]["iterations_per_substep"], "learned": r["learned"]["iterations_per_substep"]}
           for sd, r in zip(seeds, rows)]
    s = learned.summary(per)
    plain_it = float(np.mean([x["plain"] for x in per]))
    learn_it = float(np.mean([x["learned"] for x in per]))
    plain_ms = float(np.sum([r["plain"]["ms_per_frame"] for r in rows]))
    learn_ms = float(np.sum([r["learned"]["ms_per_frame"] for r in rows]))
    N = n * n
    subs = 8
    return {"workload": f"{drapes} held-out {n}x{n} drapes (1.5 m) over a sphere SDF, 8 substeps, continuous "
                        f"self-collision, fast solver build; trained on {int(z['drapes'])} drapes at "
                        f"{int(z['n'])}x{int(z['n'])}, correction scaled by "
                        f"{float(z['output_scale']) if 'output_scale' in z else 1.0:g} (calibrated on other drapes)",
            "residual": f"update residual (largest particle displacement of an iteration, metres) <= {tol:g}, cap {cap}",
            "plain_iterations_per_substep": plain_it, "learned_iterations_per_substep": learn_it,
            "iteration_ratio": s["aggregate"], "iteration_ratio_median": s["median"],
            "iteration_ratio_per_drape": s["ratios"],
            "plain_residual_reached": all(r["plain"]["iterations_per_substep"] < cap for r in rows),
            "plain_vertex_substeps_per_s": N * subs * len(rows) / (plain_ms * 1e-3),
            "learned_vertex_substeps_per_s": N * subs * len(rows) / (learn_ms * 1e-3),
            "throughput_ratio": plain_ms / learn_ms if learn_ms else None}


def run_ours(args):
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    from solidcloth_b200 import api, scenes
    if args.config == "cfg3":
        # instances shard over ranks (no collective on the data path): strong scaling
        sc = _Batch(scenes.cfg3_instances()[:args.instances], rank, ws)
        p = api.load_batch(sc.mine)
    else:
        sc = _scene(args.config, args.self_mode)
        w, p = api.load_scene(sc)
    if args.precision != "default":
        p.model.set_fast_math(args.precision == "fast")
    if args.direct:
        p.set_direct_launch(True)
    stream = torch.cuda.ExternalStream(p.cuda_stream(), device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # CUDA events inside the frame graph bracket the solve and the broad phases of
    # every timed substep (fresh events per frame: no host sync in the timed loop)
    p.set_kernel_timing(args.steps)
    for _ in range(args.warmup):
        p.step(sc.dt)
    p.synchronize()
    p.kernel_timing()                      # drop the warm-up frames' records
    st = p.status()
    # the state the timed frames start from: the end-to-end run replays the same frames
    start_state = (p.model.positions(), p.model.prev_positions(), p.model.velocities()) if not args.no_e2e else None
    kernels_per_frame = p.graph_kernel_count()

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with Clocks(local) as clk:
        barrier()
        torch.cuda.nvtx.range_push("timed")     # profilers can select the timed frames (ncu --nvtx-include timed/)
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.fill_(float(k))
                starts[k].record(stream)
                p.step(sc.dt)
                ends[k].record(stream)
        torch.cuda.nvtx.range_pop()
        barrier()
    ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    tot_ms = float(sum(ms))
    sections, timed_frames = p.kernel_timing()
    p.set_kernel_timing(0)
    if ws > 1:
        t = torch.tensor([tot_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        tot_ms = float(t.item())
    vsub = sc.num_vertices * sc.params.substeps
    if isinstance(sc, _Batch):
        # every rank steps its own instances: all ranks' vertex-substeps over the slowest rank's time
        all_vsub = sum(s.num_vertices for s in sc.all) * sc.params.substeps
        value = all_vsub * args.steps / (tot_ms * 1e-3)
    else:
        value = ws * vsub * args.steps / (tot_ms * 1e-3)
    status = st | p.status()

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        pos = torch.empty((sc.num_vertices, 3), dtype=torch.float32).pin_memory().numpy()
        prev = torch.empty_like(torch.from_numpy(pos)).pin_memory().numpy()
        vel = torch.empty_like(torch.from_numpy(pos)).pin_memory().numpy()
        pos[:], prev[:], vel[:] = start_state
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            p.model.set_state(pos, prev, vel)
            p.step(sc.dt)
            pos[:] = p.model.positions()
            prev[:] = p.model.prev_positions()
            vel[:] = p.model.velocities()
        barrier()
        e2e_s = time.perf_counter() - t0
        if ws > 1:
            t = torch.tensor([e2e_s], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e_units = (sum(s.num_vertices for s in sc.all) * sc.params.substeps) if isinstance(sc, _Batch) else ws * vsub
        e2e = {"value": e2e_units * args.steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": 3 * 16 * sc.num_vertices,
               "d2h_bytes_per_step": 3 * 16 * sc.num_vertices,
               "path": "scSetParticleState -> scStepCloth -> scGetParticlePositions/Prev/Velocities"}

    # roofline of the dominant kernel, from the in-graph events of the timed frames
    T, B, E, N = p.model.num_tris(), p.model.num_bends(), p.model.num_edges(), sc.num_vertices
    it = max(1, sc.params.iterations)
    peak, peak_kind = _peaks()
    ee_pairs = len(p.model.ccd_candidates(1)) if sc.ccd else 0
    algo = {
        # iterations x 144 B per FEM projection + bend iterations x 144 B per bend + velocity 48 B per vertex
        "gs_solve": it * 144 * T + ((it + 1) // 2) * 144 * B + 48 * N,
        # per query: 2 endpoints x (pos, prev) 64 B + edge 16 B + count 4 B; 4 B per pair; tree read once
        "ccd_broad_ee": E * 84 + 4 * ee_pairs + 32 * (2 * E - 1),
        # per particle: pos + prev 32 B read, one 64 B contact slot written per collider hit (upper bound: one per particle)
        "colliders": 96 * N,
    }
    ch, _ = p.model.solver_choice()
    solver = {1: "k_gs_cluster (one substep's Gauss-Seidel loop + velocity, one cluster launch)",
              2: f"k_gs_grid variant {ch[1]} ({ch[3]} threads, {ch[2]} CTAs/SM; one substep's Gauss-Seidel loop + velocity, one cooperative launch)",
              3: "k_fem / k_bends per colour (one substep's Gauss-Seidel loop)",
              4: f"k_gs_band ({ch[3]} threads per CTA, one {p.model.band_plan()[0]}-CTA cluster of particle bands; "
                 f"one substep's Gauss-Seidel loop + velocity, one cluster launch)"}.get(ch[0], "solver")
    kernel_names = {"gs_solve": solver,
                    "ccd_broad_ee": "k_bvh_refit + k_ccd_broad_ee + k_ccd_broad_coop (edge-edge swept-box LBVH "
                                    "refit and query: one walk per lane, long lists one warp per query)",
                    "colliders": "k_vertex_colliders (+ k_tri_colliders, k_edge_colliders when continuous collision is "
                                 "off: with it on they run on another branch, untimed)"}
    walk, walk_ms = p.model.broad_phase_mode()
    per = {}
    for k in algo:
        tot, cnt = sections.get(k, (0.0, 0))
        if cnt:
            avg = tot / cnt
            per[k] = {"ms_per_launch": avg, "launches": cnt, "algorithmic_bytes_per_launch": algo[k],
                      "achieved_gbs": algo[k] / (avg * 1e-3) / 1e9, "share_of_frame": tot / tot_ms}
    dom = max(per, key=lambda k: per[k]["ms_per_launch"] * per[k]["launches"]) if per else None
    traffic = None
    tt = ROOT / "profiles" / "traffic.txt"     # DRAM bytes per launch from the ncu captures
    if dom and tt.exists():
        for line in tt.read_text().splitlines():
            f = line.split()
            if len(f) == 3 and not line.startswith("#") and f[0] == args.config and f[1] == dom:
                traffic = int(f[2])
    roofline = None
    if dom:
        d = per[dom]
        roofline = {"bound": "hbm", "achieved": d["achieved_gbs"], "peak": peak, "unit": "GB/s",
                    "frac": d["achieved_gbs"] / peak, "traffic": traffic, "kernel": kernel_names[dom],
                    "algorithmic_bytes_per_launch": d["algorithmic_bytes_per_launch"],
                    "ms_per_launch": d["ms_per_launch"], "launches_timed": d["launches"],
                    "peak_source": peak_kind,
                    "sections": per,
                    "ccd_broad_vt_ms_per_launch": (sections["ccd_broad_vt"][0] / sections["ccd_broad_vt"][1]
                                                   if sections.get("ccd_broad_vt", (0, 0))[1] else None),
                    "broad_phase_walk": {"chosen": p.model.BROAD_WALKS[walk],
                                         "tuned_ms": walk_ms.tolist()}}
        if dom == "gs_solve" and ch[0] == 1:
            # the cluster solve is a chain of colour phases: its latency floor is the
            # phase count times the cost of one phase with no projection arithmetic
            n_fem = len(p.model.constraint_order(0)[1]) - 1
            n_bend = len(p.model.constraint_order(1)[1]) - 1
            phases = it * n_fem + ((it + 1) // 2) * n_bend + (it if sc.sdfs or sc.spheres or sc.walls is not None else 0)
            us0 = float(api.lib().scProbeClusterPhase(0, 20000))
            us1 = float(api.lib().scProbeClusterPhase(1, 20000))
            if us1 > 0:
                floor_ms = phases * us1 * 1e-3
                roofline["latency"] = {"phases_per_launch": phases, "us_per_phase_barrier": us0,
                                       "us_per_phase_barrier_dsmem": us1, "floor_ms": floor_ms,
                                       "frac": floor_ms / d["ms_per_launch"]}

    # plain versus learned warm start at the residual target (trained weights from
    # solidcloth_b200/data/warmstart.npz, held-out 64x64 drapes)
    learned_ab = None
    if rank == 0 and not args.no_learned:
        try:
            learned_ab = _learned_ab()
        except Exception as e:  # reported, not fatal
            learned_ab = {"error": str(e)}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            from oracle.bridge import available
            if available("ref") and isinstance(sc, _Batch):
                # a batch: whole first frames of instances spread over the list,
                # until about 10 s of reference time
                picks = sc.mine[::max(1, len(sc.mine) // 64)]
                units = secs = 0.0
                used = []
                with _reference_output_to_stderr():
                    for inst in picks:
                        v1, s1, cores = cpu_reference_rate(inst, frames=1)
                        units += v1 * s1
                        secs += s1
                        used.append(inst)
                        if secs >= 10.0:
                            break
                ref_sc = used[len(used) // 2]
                cpu = {"value": units / secs, "unit": UNIT, "cores": cores, "kind": "reference", "cpu": _cpu_model(),
                       "sample": f"the first frame ({ref_sc.params.substeps} substeps) of {len(used)} of the "
                                 f"{len(sc.mine)} instances, spread over the list ({int(sum(x.num_vertices for x in used))} "
                                 f"vertices, {secs:.1f} s), the reference's own C++ (oracle/_ref, OpenMP {cores} threads)"}
                if available("ref_serial"):
                    units1 = secs1 = 0.0
                    with _reference_output_to_stderr():
                        for inst in used:
                            v1, s1, _ = cpu_reference_rate(inst, serial=True, substeps=inst.params.substeps)
                            units1 += v1 * s1
                            secs1 += s1
                    cpu["single_thread"] = {
                        "value": units1 / secs1, "unit": UNIT, "cores": 1,
                        "sample": f"the first {ref_sc.params.substeps} substeps of the same {len(used)} instances "
                                  f"({secs1:.1f} s), the reference built without OpenMP (oracle/_ref/libscref_serial.so), "
                                  f"as its C-ABI library ships"}
            elif available("ref"):
                ref_sc = sc
                with _reference_output_to_stderr():
                    v, secs, cores = cpu_reference_rate(ref_sc, frames=1)
                cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "cpu": _cpu_model(),
                       "sample": f"the first frame ({ref_sc.params.substeps} substeps) of {ref_sc.name} from its "
                                 f"initial state ({secs:.1f} s), the reference's own C++ (oracle/_ref, OpenMP "
                                 f"{cores} threads)"}
                if available("ref_serial"):
                    nsub = 2 if ref_sc.num_vertices > 16384 else ref_sc.params.substeps
                    with _reference_output_to_stderr():
                        v1, secs1, _ = cpu_reference_rate(ref_sc, serial=True, substeps=nsub)
                    cpu["single_thread"] = {
                        "value": v1, "unit": UNIT, "cores": 1,
                        "sample": f"the first {nsub} substeps of {ref_sc.name} from its initial state ({secs1:.1f} s), "
                                  f"the reference built without OpenMP (oracle/_ref/libscref_serial.so), as its "
                                  f"C-ABI library ships"}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
                "scaling": "strong" if isinstance(sc, _Batch) else "weak", "vs_baseline": None, "dtype": "fp32",
                "data": "synthetic", "config": _workload(sc), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "learned": learned_ab,
                "gpu_launches": kernels_per_frame * args.steps, "kernels_per_frame": kernels_per_frame,
                "clocks": clk.summary(), "device_status": status,
                "solver_precision": "fast" if p.model.fast_math() else "ieee"}
        print(json.dumps(line))
    p.free()
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
