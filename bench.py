"""Benchmark of the hydro / ideal-MHD step on B200.

Workload (one GPU): 3-D ideal MHD on a 256^3 periodic mesh split into 64 blocks
of 64^3, gamma = 5/3, PLM + HLLD + CT, Heun RK2, Orszag-Tang-type vortex with
seeded 1e-3 velocity noise (synthetic, seeded; no dataset involved).  A "step" is
one Heun step over the whole mesh.  The state (1.6 GB) is larger than L2, so no
flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--modes fp64,mixed]

Prints one JSON line (rank 0).  `value` is whole-job zone-cycles/s of the
headline mode; every measured mode is listed under "modes".
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-cycles/s, 256³ MHD: learned FP32/64 vs plain FP64 HLLD at stated L1 error"
UNIT = "zone-cycles/s"
NB, N = (4, 4, 4), (64, 64, 64)
GAMMA = 5.0 / 3.0
SEED = 2
# algorithmic bytes: 8 FP64 state words (5 conserved + 3 face B) x 5 transfers
BYTES_PER_ZONE_CYCLE = 320
# The flux sweep (the kernel with the largest share of the step): per face it
# reads the 8 primitive words of one cell (neighbouring faces share the rest of
# the stencil through L1) and the face's normal B (FP64), and writes 7 flux
# words -- 68 B in the FP32 modes, 128 B in FP64.  Faces per launch include
# the transverse ghost lines the edge EMF reads: (n+1) ((n+2)^2 - 4) per block.
FLUX_BYTES_PER_FACE = {4: 8 * 4 + 8 + 7 * 4, 8: 8 * 8 + 8 + 7 * 8}
# DRAM bytes per face of one FP32 flux launch, ncu dram__bytes_read.sum +
# dram__bytes_write.sum on this workload (three launches of the first timed
# step, 1319.3 MB on average) divided by its 18.1 M faces
FLUX_DRAM_BYTES_PER_FACE = 72.9
# DRAM bytes per zone-cycle of one whole mixed step, ncu on this workload, one
# kernel kind per capture (profiles/step_dram_mixed_ot256.md)
STEP_DRAM_BYTES_PER_ZONE_CYCLE_MIXED = 1343.2
WORKLOAD = "ot 256^3 periodic MHD, 64 blocks of 64^3, PLM+HLLD+CT, Heun RK2"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--modes", default="fp64,mixed,learned,vl2")
    p.add_argument("--mesh", type=int, default=256, choices=[128, 256],
                   help="global cells per axis (128: profiling-sized sample, 8 blocks of 64^3)")
    p.add_argument("--cpu-baseline", type=int, default=1, help="0: skip the CPU baseline leg")
    p.add_argument("--boxes", type=int, default=1024,
                   help="batched-box leg: boxes of the seeded batch (0: skip)")
    p.add_argument("--smr", type=int, default=1,
                   help="1: also time the statically refined hydro mesh (1 GPU only)")
    p.add_argument("--blast", type=int, default=1,
                   help="also time the magnetized blast on the criterion-refined MHD mesh (0: skip)")
    p.add_argument("--ref-cuda", type=int, default=1,
                   help="1: also time the reference's own CUDA build (baseline/_ref) on this GPU")
    p.add_argument("--turb", type=int, default=512, choices=[0, 128, 256, 512],
                   help="turbulence leg: global cells per axis (64^3 blocks; 0: skip)")
    args = p.parse_args()
    global NB
    NB = (args.mesh // 64,) * 3
    return args


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clock and throttle reasons with NVML while running."""

    def __init__(self, index):
        self.index, self.samples, self.reasons = index, [], set()
        self.max_mhz, self._stop = None, threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.nv = pynvml
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        except Exception:
            self.nv = None
        return self

    def _run(self):
        nv = self.nv
        names = {
            getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8): "hw_slowdown",
            getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40): "hw_thermal_slowdown",
            getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20): "sw_thermal_slowdown",
            getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4): "sw_power_cap",
        }
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in names.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.05)

    def __exit__(self, *a):
        self._stop.set()
        if self.nv is not None:
            self.t.join(timeout=1)

    def summary(self):
        s = sorted(self.samples)
        med = s[len(s) // 2] if s else None
        return {"sm_mhz": med, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(s)}


# --------------------------------------------------------------------------- CPU
def run_reference_cpu(steps, nb=None, n=N, threads=None):
    """Time the original Kratos solver (its CPU path, built from source into
    oracle/_ref/kratos_ref) on an OT mesh; returns (zone-cycles/s, cores) from
    its own `Speed = ... cell/s` line (cycle.cpp:184-190)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "kratos_ref")
    if not os.path.exists(exe):
        return None
    nb = nb or NB
    threads = threads or os.cpu_count()
    with tempfile.TemporaryDirectory() as tmp:
        par = os.path.join(tmp, "b.par")
        ng = [nb[a] * n[a] for a in range(3)]
        with open(par, "w") as f:
            f.write("\n".join([
                "[problem]", "name = ot", "seed = %d" % SEED, "[mesh]", "x_min = 0 0 0", "x_max = 1 1 1",
                "n_cell_global = %d %d %d" % tuple(ng), "n_cell_block = %d %d %d" % tuple(n),
                "[cycle]", "prefix_output = %s/s" % tmp, "n_cycle_lim = %d" % (steps - 1),
                "final_output = 0", "t_output_next = 1e99", "n_display_freq = 1000000",
                "[dynamics]", "gamma = %r" % GAMMA, "thread_limit = 1", "bnd_thread_limit = 1",
                "[boundary]", "kinds = per per per per per per", ""]))
        env = dict(os.environ, KR_REF_THREADS=str(threads))
        out = subprocess.run([exe, par], cwd=tmp, env=env, capture_output=True, text=True, timeout=1800)
    m = re.search(r"Speed = ([0-9.eE+-]+) cell/s", out.stdout)
    if not m:
        return None
    return float(m.group(1)), threads


def run_reference_cuda(steps, precision, nb=None, n=N, timeout=900):
    """Time the original Kratos solver's own CUDA path (baseline/Makefile.cuda:
    its sources built with nvcc for sm_100a) on the benchmark's OT mesh, on
    the current GPU; returns its own `Speed = ... cell/s` (zone-cycles/s over
    its n_cycle_lim + 1 steps, cycle.cpp:184-190), or None if not built."""
    exe = os.path.join(ROOT, "baseline", "_ref", "kratos_cuda_p%d" % precision)
    if not os.path.exists(exe):
        return None
    nb = nb or NB
    with tempfile.TemporaryDirectory() as tmp:
        par = os.path.join(tmp, "b.par")
        ng = [nb[a] * n[a] for a in range(3)]
        with open(par, "w") as f:
            f.write("\n".join([
                "[problem]", "name = ot", "seed = %d" % SEED, "[mesh]", "x_min = 0 0 0", "x_max = 1 1 1",
                "n_cell_global = %d %d %d" % tuple(ng), "n_cell_block = %d %d %d" % tuple(n),
                "[cycle]", "prefix_output = %s/s" % tmp, "n_cycle_lim = %d" % (steps - 1),
                "final_output = 0", "t_output_next = 1e99", "n_display_freq = 1000000",
                "[dynamics]", "gamma = %r" % GAMMA,
                "[boundary]", "kinds = per per per per per per", ""]))
        env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", "0"))
        out = subprocess.run([exe, par], cwd=tmp, env=env, capture_output=True, text=True, timeout=timeout)
    m = re.search(r"Speed = ([0-9.eE+-]+) cell/s", out.stdout)
    if out.returncode != 0 or not m:
        return {"value": None, "error": (out.stderr or out.stdout)[-400:]}
    return {"value": float(m.group(1)), "unit": UNIT, "steps": steps,
            "sample": "the benchmark's %d^3 OT mesh (%d blocks of 64^3), %d steps, the reference's "
                      "default [dynamics] thread_limit / bnd_thread_limit (64), PRECISION=%d"
                      % (ng[0], nb[0] * nb[1] * nb[2], steps, precision)}


def run_oracle_cpu(steps, nb=None, n=N):
    from oracle.kr_oracle import OracleMesh
    nb = nb or NB
    o = OracleMesh(True, nb, n, GAMMA)
    o.init_problem("ot", SEED)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    return nb[0] * nb[1] * nb[2] * n[0] * n[1] * n[2] * steps / dt, os.cpu_count()


REF_SAMPLE_NOTE = ("original Kratos CPU path (its ARCH=HIPCPU code, PRECISION=2) built from source "
                   "with the project's HIP-CPU-compatible header, one thread per CTA "
                   "(thread_limit = bnd_thread_limit = 1), CTAs on all host threads")


def cpu_baseline(steps=2):
    r = run_reference_cpu(steps)
    sample = "%d Heun steps of the same %d^3 OT mesh (%d blocks of 64^3), PRECISION=2" % (
        steps, NB[0] * N[0], NB[0] * NB[1] * NB[2])
    if r is not None:
        return {"value": r[0], "unit": UNIT, "cores": r[1], "kind": "reference",
                "sample": sample + ", " + REF_SAMPLE_NOTE}
    v, cores = run_oracle_cpu(steps)
    return {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": sample + ", CPU restatement (oracle/)"}


# The reference arm runs the benchmark's own mesh (same workload, same
# config) on the host cores; at ~1.4e6 zone-cycles/s on 16 cores one 256^3
# step takes ~12 s, so it times at most this many steps (one run: the
# reference's own `Speed` line over its steps).
REF_ARM_MAX_STEPS = 8


def bench_config(world, mode, n_cells):
    """The `config` object both arms print (same workload, same keys)."""
    workload = WORKLOAD
    if world > 1:
        nb_g, _ = weak_mesh(world)
        workload = WORKLOAD.replace(
            "256^3 periodic MHD, 64 blocks", "%dx%dx%d periodic MHD (256^3 per GPU), %d blocks"
            % (nb_g[0] * N[0], nb_g[1] * N[1], nb_g[2] * N[2], nb_g[0] * nb_g[1] * nb_g[2]))
    elif NB[0] * N[0] != 256:
        workload = WORKLOAD.replace("256^3", "%d^3" % (NB[0] * N[0])).replace(
            "64 blocks", "%d blocks" % (NB[0] * NB[1] * NB[2]))
    return {"workload": workload, "mode": mode, "global_cells": n_cells,
            "parallelism": ("%d GPUs: mesh sharded by blocks (%d blocks of 64^3 per GPU), "
                            "NCCL halo exchange + dt all-reduce in the step graph" % (world, NB[0] * NB[1] * NB[2]))
                           if world > 1 else "1 GPU",
            "l2": "state 1.6 GB > 126 MB L2; no flush needed"}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    steps = max(2, min(args.steps + args.warmup, REF_ARM_MAX_STEPS))
    r = run_reference_cpu(steps)
    if r is not None:
        kind, v, cores, note = "reference", r[0], r[1], REF_SAMPLE_NOTE
    else:
        kind = "port"
        v, cores = run_oracle_cpu(steps)
        note = "CPU restatement (oracle/)"
    n_cells = NB[0] * NB[1] * NB[2] * N[0] * N[1] * N[2] * world
    sample = "%d Heun steps of the benchmark's %d^3 OT mesh (%d blocks of 64^3), %s" % (
        steps, NB[0] * N[0], NB[0] * NB[1] * NB[2], note)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(world, "learned", n_cells),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- GPU
MODES = {"fp64": dict(precision=2, riemann=0), "mixed": dict(precision=1, riemann=0),
         "hlle_mixed": dict(precision=1, riemann=1), "learned": dict(precision=1, riemann=2, sel_period=16),
         "learned_p1": dict(precision=1, riemann=2, sel_period=1),
         "learned_p4": dict(precision=1, riemann=2, sel_period=4),
         "vl2": dict(precision=1, riemann=0, integrator=1),
         "vl2_fp64": dict(precision=2, riemann=0, integrator=1)}


def train_selector(local_rank):
    """Selector for the learned mode, trained on the GPU from faces logged on
    a 128^3 OT run (mixed step) and a 64^3 one: ~1.9 M samples (one face in 32,
    under the collection cap, so the training data do not depend on the order
    in which device threads log them), 20 epochs."""
    from kratos_b200 import Dynamics, selector as S

    def make(nb):
        def f():
            d = Dynamics(True, nb, N, gamma=GAMMA, precision=1, device=local_rank)
            d.init_problem("ot", SEED + 1)
            return d
        return f
    t0 = time.perf_counter()
    w, info = S.build_selector([make((1, 1, 1)), make((2, 2, 2))], steps=4, stride=32,
                               epochs=20, device=local_rank)
    info["train_s"] = time.perf_counter() - t0
    info["threshold"] = S.DEFAULT_THRESHOLD
    return w, info


def weak_mesh(world):
    """Global block grid for `world` ranks: NB blocks (of N cells) per rank,
    the per-rank grid repeated along z, y, x in turn (powers of two) or
    along x; the domain grows with it (cell size fixed)."""
    f = [1, 1, 1]
    w, a = world, 2
    while w > 1 and w % 2 == 0:
        f[a] *= 2
        w //= 2
        a = (a - 1) % 3
    f[0] *= w
    nb = tuple(NB[i] * f[i] for i in range(3))
    return nb, tuple(float(f[i]) for i in range(3))


def time_mode(mode, args, local_rank, world, dist):
    import torch
    from kratos_b200 import Dynamics
    if world > 1:
        # weak scaling: NB blocks per rank, block-sharded mesh, NCCL halo exchange
        from kratos_b200.shard import sharded_dynamics
        nb_g, x_max = weak_mesh(world)
        d = sharded_dynamics(True, nb_g, N, gamma=GAMMA, device=local_rank, x_max=x_max, **MODES[mode])
    else:
        d = Dynamics(True, NB, N, gamma=GAMMA, device=local_rank, **MODES[mode])
    sel_info = None
    if mode.startswith("learned"):
        # one selector for every rank: faces shared by two blocks must get the
        # same solver on both sides
        got = [None]
        if dist is None or dist.get_rank() == 0:
            got = [train_selector(local_rank)]
        if dist is not None:
            dist.broadcast_object_list(got, src=0)
        w, sel_info = got[0]
        d.set_selector(w, sel_info["threshold"])
    stream = torch.cuda.Stream(device=local_rank)
    d.set_stream(stream.cuda_stream)
    d.init_problem("ot", SEED)
    d.step(args.warmup)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        t0.record(stream)
        d.step(args.steps)
        t1.record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = t0.elapsed_time(t1)
    if dist is not None:
        x = torch.tensor([ms], device="cuda:%d" % local_rank)
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
        ms = float(x.item())
    if d.status() != 0:
        raise RuntimeError("device status %d in mode %s" % (d.status(), mode))
    div_b, _ = d.diagnostics()
    if dist is not None:
        x = torch.tensor([div_b], device="cuda:%d" % local_rank)
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
        div_b = float(x.item())
    n_all = d.n_cells
    if dist is not None:
        x = torch.tensor([float(d.n_cells)], device="cuda:%d" % local_rank)
        dist.all_reduce(x)
        n_all = int(x.item())
    zcs = n_all * args.steps / (ms * 1e-3)
    prof = d.profile_step()
    out = {"value": zcs, "ms_per_step": ms / args.steps, "clocks": clk.summary(),
           "kernels_ms_per_step": prof, "launches_per_step": d.launches_per_step()}
    # end-to-end through the C ABI with host buffers: upload the state from pinned
    # host memory, run the steps, read the state back, all inside the timed region
    import numpy as np
    u, bf = d.get_state()
    hu = torch.from_numpy(u).pin_memory().numpy()
    hb = torch.from_numpy(bf).pin_memory().numpy()
    e2e_steps = args.steps
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    d.set_state(hu, hb)
    d.step(e2e_steps)
    d.get_state(hu, hb)
    w1 = time.perf_counter()
    wall = w1 - w0
    if dist is not None:
        x = torch.tensor([wall], device="cuda:%d" % local_rank)
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
        wall = float(x.item())
    # final density (every mode runs warm-up + timed + end-to-end steps from the
    # same initial state) for the error of the FP32 modes against the FP64 one
    out["rho"] = np.array(hu[..., 0])
    out["e2e"] = {"value": n_all * e2e_steps / wall, "unit": UNIT,
                  "h2d_bytes_per_step": d.state_bytes() // e2e_steps,
                  "d2h_bytes_per_step": d.state_bytes() // e2e_steps,
                  "steps_per_transfer": e2e_steps,
                  "basis": "kr_set_state from pinned host memory, kr_step(%d), kr_get_state to pinned host "
                           "memory, all inside the wall-clock region; the state crosses PCIe once each way "
                           "per %d steps" % (e2e_steps, e2e_steps)}
    out["n_cells"] = n_all
    out["div_b_max"] = div_b
    if sel_info is not None:
        faces, cheap = d.selector_stats()
        sel_info = dict(sel_info, hlle_fraction=cheap / max(faces, 1))
        out["selector"] = sel_info
        out["selector_weights"] = w
    del np
    d.close()
    return out


# Statically refined hydro mesh: root 128^3 in 512 blocks of 16^3, the shock
# plane x = 0.5 covered by a level-1 slab (x in [0.4, 0.6]) and a level-2 slab
# (x in [0.45, 0.55]) over the whole y-z extent.
SMR_NB, SMR_N = (8, 8, 8), (16, 16, 16)
SMR_REGIONS = [(1, (0.4, 0.0, 0.0), (0.6, 1.0, 1.0)), (2, (0.45, 0.0, 0.0), (0.55, 1.0, 1.0))]


def time_smr(args, local_rank):
    """Zone-cycles/s of the refined hydro step (every block of every level in
    one captured graph per step), FP64 and mixed."""
    import torch
    from kratos_b200 import Dynamics
    out = {"workload": "shock, root 128^3 (512 blocks of 16^3), level-1 slab x in [0.4, 0.6] and "
                       "level-2 slab x in [0.45, 0.55], periodic, PLM + HLLC, Heun RK2"}
    for mode, prec in (("fp64", 2), ("mixed", 1)):
        d = Dynamics(False, SMR_NB, SMR_N, gamma=1.4, precision=prec, device=local_rank,
                     regions=SMR_REGIONS)
        stream = torch.cuda.Stream(device=local_rank)
        d.set_stream(stream.cuda_stream)
        d.init_problem("shock", SEED)
        d.step(args.warmup)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        d.step(args.steps)
        t1.record(stream)
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1)
        if d.status() != 0:
            raise RuntimeError("device status %d in the refined %s step" % (d.status(), mode))
        out[mode] = {"value": d.n_cells * args.steps / (ms * 1e-3), "unit": UNIT,
                     "ms_per_step": ms / args.steps, "kernels_ms_per_step": d.profile_step(),
                     "launches_per_step": d.launches_per_step()}
        out["blocks_per_level"] = [int((d.level == l).sum()) for l in range(int(d.level.max()) + 1)]
        out["cells"] = d.n_cells
        d.close()
    return out


def time_blast(args, local_rank):
    """Zone-cycles/s of the magnetized blast on a mesh that the gradient
    criterion refines at t = 0 (kratos_b200/amr.py): root 128^3 in 16^3 blocks,
    three refinement levels, PLM + HLLD + CT, every block of every level in one
    captured graph per step; mixed and FP64."""
    import torch
    from kratos_b200.blast import blast_mesh
    out = {"workload": "magnetized blast (p = 100 inside r < 0.1 of the centre, 0.1 outside, rho = 1, "
                       "B = (1, 1, 0) / sqrt 2), root 128^3 in 512 blocks of 16^3, three levels refined at "
                       "t = 0 where max_axes(|d rho| / 2 rho + |d p| / 2 p) > 0.5 (kratos_b200/amr.py), "
                       "periodic, PLM + HLLD + CT, Heun RK2"}
    for mode, prec in (("mixed", 1), ("fp64", 2)):
        d, regions = blast_mesh(prec, local_rank)
        out["refine_regions"] = len(regions)
        stream = torch.cuda.Stream(device=local_rank)
        d.set_stream(stream.cuda_stream)
        d.init_problem("blast", SEED)
        d.step(args.warmup)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        d.step(args.steps)
        t1.record(stream)
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1)
        if d.status() != 0:
            raise RuntimeError("device status %d in the blast %s step" % (d.status(), mode))
        div, _ = d.diagnostics()
        out[mode] = {"value": d.n_cells * args.steps / (ms * 1e-3), "unit": UNIT,
                     "ms_per_step": ms / args.steps, "kernels_ms_per_step": d.profile_step(),
                     "launches_per_step": d.launches_per_step(), "div_b_max": div}
        out["blocks_per_level"] = [int((d.level == l).sum()) for l in range(int(d.level.max()) + 1)]
        out["cells"] = d.n_cells
        d.close()
    return out


def time_boxes(args, local_rank, sel=None):
    """Zone-cycles/s of a batch of independent periodic MHD boxes (seed 5,
    edge lengths 16..64), each on its own CFL dt: one KR_FLAG_BOXES context per
    edge length, each on its own stream; CUDA events from a start event that
    every stream waits on to an end event after all of them."""
    import torch
    from kratos_b200.boxes import BoxBatch
    out = {"workload": "%d independent periodic MHD boxes (seed 5), edge lengths from {16, 24, 32, 48, 64}, "
                       "random rho, p, velocity amplitude, B orientation and beta, PLM + HLLD + CT, "
                       "Heun RK2, per-box dt" % args.boxes,
           "how": "<mode>: one context and one graph per edge length, each on its own stream; "
                  "<mode>_batched: one persistent launch per kernel kind over a work list of every box's "
                  "CTA tiles (kr_batch), one graph per step, CTA counts autotuned first"}
    box_modes = [("fp64", MODES["fp64"]), ("mixed", MODES["mixed"])]
    if sel is not None:
        box_modes.append(("learned", MODES["learned"]))
    runs = [(m, kw, False) for m, kw in box_modes] + [(m + "_batched", kw, True) for m, kw in box_modes]
    for mode, kw, batched in runs:
        bb = BoxBatch(5, args.boxes, device=local_rank, batched=batched, **kw)
        if mode.startswith("learned"):
            bb.set_selector(sel[0], sel[1]["threshold"])
        streams = {}
        for n, (d, _) in bb.groups.items():
            streams[n] = torch.cuda.Stream(device=local_rank)
            d.set_stream(streams[n].cuda_stream)
        tuned = None
        if batched:
            with tempfile.TemporaryDirectory() as tmp:
                tuned, _ = bb.autotune(os.path.join(tmp, "tune.txt"))
        bb.step(args.warmup)
        torch.cuda.synchronize()
        main_s = torch.cuda.Stream(device=local_rank)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(main_s)
        for st in streams.values():
            st.wait_event(t0)
        bb.step(args.steps)
        for st in streams.values():
            e = torch.cuda.Event()
            e.record(st)
            main_s.wait_event(e)
        t1.record(main_s)
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1)
        if bb.status() != 0:
            raise RuntimeError("device status %d in the %s box batch" % (bb.status(), mode))
        t, _ = bb.times()
        out[mode] = {"value": bb.n_cells * args.steps / (ms * 1e-3), "unit": UNIT,
                     "ms_per_step": ms / args.steps, "launches_per_step": bb.launches_per_step(),
                     "box_time_range": [float(t.min()), float(t.max())]}
        if tuned is not None:
            out[mode]["grid"] = tuned
        if mode.startswith("learned"):
            faces, cheap = bb.selector_stats()
            out[mode]["hlle_fraction"] = cheap / max(faces, 1)
        out["cells"] = bb.n_cells
        out["boxes_per_size"] = {str(n): int(len(ids)) for n, (_, ids) in bb.groups.items()}
        bb.close()
    return out


TURB_SEED = 4


def time_turb(args, local_rank, sel):
    """The learned step on decaying supersonic MHD turbulence at the stated
    size (512^3, 512 blocks of 64^3), next to the plain FP64 and the mixed
    step from the same initial state: zone-cycles/s, HLLE share, relative L1
    density error against the FP64 step after the same steps, |div B|."""
    import numpy as np
    import torch
    from kratos_b200 import Dynamics
    ng = args.turb
    nb = (ng // N[0],) * 3
    out = {"workload": "turb %d^3 periodic MHD (%d blocks of 64^3): rho 1, rms Mach 5 random-phase solenoidal "
                       "velocity with a k^-2 spectrum at 1 <= |k| <= 4 (seed %d), uniform B_x at beta 0.1, "
                       "decaying; PLM + HLLD + CT, Heun RK2; the learned mode's network is the one trained "
                       "on the OT mesh's faces" % (ng, nb[0] * nb[1] * nb[2], TURB_SEED)}
    d = Dynamics(True, nb, N, gamma=GAMMA, precision=1, device=local_rank)
    t0 = time.perf_counter()
    d.init_problem("turb", TURB_SEED)
    u0, bf0 = d.get_state()
    out["init_s"] = time.perf_counter() - t0
    out["cells"] = d.n_cells
    d.close()
    rho = {}
    for mode in ("fp64", "mixed", "learned"):
        d = Dynamics(True, nb, N, gamma=GAMMA, device=local_rank, **MODES[mode])
        if mode == "learned":
            d.set_selector(sel[0], sel[1]["threshold"])
        stream = torch.cuda.Stream(device=local_rank)
        d.set_stream(stream.cuda_stream)
        d.set_state(u0, bf0)
        d.step(args.warmup)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if d.status() != 0:
            raise RuntimeError("device status %d in the turbulence %s step" % (d.status(), mode))
        div_b, _ = d.diagnostics()
        r = {"value": d.n_cells * args.steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / args.steps,
             "div_b_max": div_b}
        if mode == "learned":
            faces, cheap = d.selector_stats()
            r["hlle_fraction"] = cheap / max(faces, 1)
        u, _ = d.get_state()
        rho[mode] = np.array(u[..., 0])
        del u
        out[mode] = r
        d.close()
    den = np.abs(rho["fp64"]).sum()
    for mode in ("mixed", "learned"):
        out[mode]["l1_density_vs_fp64"] = float(np.abs(rho[mode] - rho["fp64"]).sum() / den)
    out["learned_over_fp64"] = out["learned"]["value"] / out["fp64"]["value"]
    out["learned_over_mixed"] = out["learned"]["value"] / out["mixed"]["value"]
    out["steps_compared"] = args.warmup + args.steps
    return out


def flux_roofline(h, head, world, peak, peak_kind):
    """Roofline line of the flux sweep: algorithmic bytes per launch over the
    mean launch duration (CUDA events around each launch, kr_profile_step)."""
    rsize = 8 if head == "fp64" else 4
    nblk = NB[0] * NB[1] * NB[2]
    faces = nblk * (N[0] + 1) * ((N[1] + 2) * (N[2] + 2) - 4)
    k = h["kernels_ms_per_step"]
    launch_ms = (k["flux_x"] + k["flux_y"] + k["flux_z"]) / 6.0      # 3 sweeps x 2 stages
    gbs = faces * FLUX_BYTES_PER_FACE[rsize] / (launch_ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": "k_flux (one sweep, %s mode)" % head,
            "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
            "traffic": FLUX_DRAM_BYTES_PER_FACE * faces if rsize == 4 else None,
            "algorithmic_bytes_per_launch": faces * FLUX_BYTES_PER_FACE[rsize],
            "launch_ms": launch_ms,
            "basis": "%d B/face x %d faces per launch (%s peak); the sweep is bound by instruction "
                     "issue and latency (FP32 PLM + HLLD), not by HBM" % (FLUX_BYTES_PER_FACE[rsize], faces, peak_kind)}


def main():
    args = parse()
    rank, world, local_rank = dist_env()
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    torch.cuda.set_device(local_rank)
    results = {}
    sel = None
    for mode in [m for m in args.modes.split(",") if m]:
        results[mode] = time_mode(mode, args, local_rank, world, dist)
        if "selector_weights" in results[mode]:
            sel = (results[mode].pop("selector_weights"), results[mode]["selector"])
    if "fp64" in results:
        import numpy as np
        ref = results["fp64"]["rho"]
        den = np.abs(ref).sum()
        for m, r in results.items():
            if m != "fp64":
                r["l1_density_vs_fp64"] = float(np.abs(r["rho"] - ref).sum() / den)
    head = next((m for m in ("learned", "mixed", "fp64") if m in results), next(iter(results)))
    h = results[head]
    peak, peak_kind = measured_peaks()
    flux_ms = h["kernels_ms_per_step"]["flux_x"] + h["kernels_ms_per_step"]["flux_y"] + h["kernels_ms_per_step"]["flux_z"]
    kernels = h["kernels_ms_per_step"]
    top = max(kernels, key=kernels.get)
    step_gbs = h["value"] / world * BYTES_PER_ZONE_CYCLE / 1e9
    summary = {}
    for m in ("fp64", "mixed", "learned", "hlle_mixed", "vl2"):
        if m in results:
            summary[m + "_value"] = results[m]["value"]
    if "fp64" in results:
        for m in ("mixed", "learned", "hlle_mixed", "vl2"):
            if m in results:
                summary[m + "_over_fp64"] = results[m]["value"] / results["fp64"]["value"]
                summary[m + "_l1_density_vs_fp64"] = results[m]["l1_density_vs_fp64"]
    if "learned" in results and "mixed" in results:
        summary["learned_over_mixed"] = results["learned"]["value"] / results["mixed"]["value"]
    if "learned" in results:
        summary["learned_hlle_fraction"] = results["learned"]["selector"]["hlle_fraction"]
    summary["div_b_max"] = max(r["div_b_max"] for r in results.values())
    line = {
        "metric": METRIC, "value": h["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": h["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32/f64" if head != "fp64" else "f64", "data": "synthetic",
        **summary,
        "config": bench_config(world, head, h["n_cells"]),
        "modes": {m: dict({"value": r["value"], "ms_per_step": r["ms_per_step"],
                           "kernels_ms_per_step": r["kernels_ms_per_step"]},
                          **({"selector": r["selector"]} if "selector" in r else {}),
                  **{"div_b_max": r["div_b_max"]},
                          **({"l1_density_vs_fp64": r["l1_density_vs_fp64"],
                              "steps_compared": args.warmup + 2 * args.steps}
                             if "l1_density_vs_fp64" in r else {}))
                  for m, r in results.items()},
        "roofline": flux_roofline(h, head, world, peak, peak_kind),
        "step_roofline": {"bound": "hbm", "achieved": step_gbs, "peak": peak, "unit": "GB/s",
                          "frac": step_gbs / peak,
                          "dram_bytes_per_zone_cycle": STEP_DRAM_BYTES_PER_ZONE_CYCLE_MIXED if head != "fp64" else None,
                          "basis": "whole step: %d B/zone-cycle algorithmic (%s peak); longest kernel kind %s; "
                                   "DRAM bytes per zone-cycle of the mixed step from ncu captures "
                                   "of each kernel kind on this workload"
                                   % (BYTES_PER_ZONE_CYCLE, peak_kind, top)},
        "clocks": h["clocks"],
        "e2e": h["e2e"],
        "gpu_launches": h["launches_per_step"] * args.steps,
    }
    line["flux_ms_per_step"] = flux_ms
    if rank == 0 and world == 1 and args.smr:
        line["smr"] = time_smr(args, local_rank)
    if rank == 0 and world == 1 and args.blast:
        line["blast"] = time_blast(args, local_rank)
    if rank == 0 and world == 1 and args.boxes:
        line["boxes"] = time_boxes(args, local_rank, sel)
    if rank == 0 and world == 1 and args.turb and sel is not None:
        line["turb"] = time_turb(args, local_rank, sel)
    if rank == 0 and world == 1 and args.ref_cuda:
        # the GPU bar: the reference's own CUDA path on this GPU, same mesh
        rc = {}
        for prec, name in ((2, "fp64"), (1, "mixed")):
            r = run_reference_cuda(args.steps, prec)
            if r is not None:
                rc[name] = r
        if rc.get("fp64", {}).get("value"):
            line["reference_cuda_fp64"] = rc["fp64"]["value"]
            if "fp64" in results:
                line["fp64_over_reference_cuda_fp64"] = results["fp64"]["value"] / rc["fp64"]["value"]
            line["value_over_reference_cuda_fp64"] = h["value"] / rc["fp64"]["value"]
        if rc.get("mixed", {}).get("value"):
            line["reference_cuda_mixed"] = rc["mixed"]["value"]
            if "mixed" in results:
                line["mixed_over_reference_cuda_mixed"] = results["mixed"]["value"] / rc["mixed"]["value"]
            line["value_over_reference_cuda_mixed"] = h["value"] / rc["mixed"]["value"]
        if rc:
            line["reference_cuda"] = rc
    if rank == 0:
        if args.cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline()
            except Exception as e:  # the baseline is reported, never required
                line["cpu_baseline"] = {"value": None, "error": str(e)}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
