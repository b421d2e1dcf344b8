"""Throughput of the B200 force step: atom-steps/s on a 96,000-atom water box.

One step = one velocity-Verlet MD step of the whole system (updateX, device-side list check and
rebuild, ghost update, pair + bonded (+ network) forces, updateV), replayed from CUDA graphs.
Contract: W untimed warm-up steps, then exactly K steps bracketed by a barrier and
torch.cuda.synchronize() on both sides, timed with CUDA events on the library's stream, max over
ranks; rank 0 prints one JSON line. With --gpus N each rank runs its own replica (weak scaling,
no collective on the data path: the force step of one system runs on one GPU).

--impl reference times the reference's own CPU implementation (oracle/_ref, its OpenMP code) on
the same workload, bounded to a few seconds of CPU work per step sample.
"""
from __future__ import annotations

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
sys.path.insert(0, os.path.join(ROOT, "tests"))

WORKLOADS = {
    # name: (n_side, bl, nmol, description)
    "water96k-classical": dict(n_side=32, bl=99.3, nmol=32000, nnp=None,
                               desc="96,000-atom water (32,000 molecules, 99.3 A box), tabulated LJ + DSF Coulomb at "
                                    "10 A, 2 A skin, bonds + angles, dt 0.5 fs NVE, FP64 Verlet state"),
}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], d["bf16_tflops"], d.get("bf16_tflops_sustained", d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampler run during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_system(wl):
    import cases
    from nnpengine_b200 import systems as S
    s = S.water_box(wl["n_side"], wl["bl"], seed=2, nmol=wl["nmol"])
    r, F, U = S.water_lj_table(10.0, 1000)
    return s, (r, F, U)


def make_engine(s, table, device):
    import cases
    from nnpengine_b200 import engine as E
    F, U = cases.table_as_loaded(table[1], table[2])
    e = E.Engine(device)
    e.set_system(s)
    e.setup(10.0, 2.0, 10.0, 1024)
    e.set_pair_table(F, U)
    e.set_bonded(s, [E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)], [E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)])
    return e


def cpu_reference(wl, steps: int):
    """The reference's OpenMP force step (oracle/_ref/ref_dump_fast) on the same workload, timed
    over its MD loop only; returns (atom-steps/s, threads, sample description)."""
    from oracle import orc
    import cases
    s, table = build_system(wl)
    with tempfile.TemporaryDirectory() as d:
        f = cases.write_inputs(s, table, d)
        cfg = {"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2, "gr_cutoff": 10,
               "bond": [f"1.0 {cases.WATER_BOND_K}"], "angle": [f"109.47 0 0 {cases.WATER_ANGLE_KC}"],
               "velocity": f["vel"], "mode": "md", "steps": steps, "dt": 0.5, "log_interval": steps}
        out = orc.run_ref_dump(cfg, os.path.join(d, "o"), fast=True, timeout=1800)
    t = float(out["info"]["t_loop"])
    n = steps + 1   # md_step = 0..steps inclusive
    return s.natom * n / t, int(out["info"]["threads"]), f"{n} MD steps of the {s.natom}-atom workload, MD loop only"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="water96k-classical", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--exact", action="store_true", help="pair forces in the reference's exact float sequence")
    ap.add_argument("--cpu-steps", type=int, default=10)
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        rate, threads, sample = cpu_reference(wl, args.cpu_steps)
        print(json.dumps({
            "impl": "reference", "metric": "atom-steps/s", "value": rate, "unit": "atom-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "description": wl["desc"]},
            "cpu_baseline": {"value": rate, "unit": "atom-steps/s", "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": rate, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist = dist_mod
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    s, table = build_system(wl)
    e = make_engine(s, table, local)
    e.pair_exact(args.exact)
    stream = torch.cuda.ExternalStream(e.lib.nnpe_stream(e.h))
    # untimed equilibration from the lattice start (Andersen, 300 K), then NVE at dt=0.5 fs
    e.verlet(1.0, True)
    e.thermostat("andersen", 300.0, 300.0, interval=1, frac=0.1, seed=11, total_steps=0)
    e.run(300, log_interval=300, graph=True)
    e.thermostat("none")
    e.verlet(0.5, True)
    e.run(args.warmup, log_interval=max(args.warmup, 1), graph=True)

    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t0.record(stream)
        log = e.run(args.steps, log_interval=args.steps, graph=True)
        t1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    if dist:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    info = e.list_info()
    value = s.natom * args.steps * world / (ms / 1e3)

    # dominant kernel: the pair force, timed alone with CUDA events on the library stream
    nlist = info["entries"] / s.natom
    reps = 50
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e.compute_forces(ev=False)
    k0.record(stream)
    for _ in range(reps):
        e.lib.nnpe_profile_enqueue(e.h, 0)
    k1.record(stream)
    torch.cuda.synchronize()
    pair_ms = k0.elapsed_time(k1) / reps
    hbm, bf16, bf16s, src = peaks()
    alg_bytes = s.natom * (4 * nlist + 48)
    achieved = alg_bytes / (pair_ms / 1e3) / 1e9

    # end to end through the public API with host buffers: positions in, forces + energy out
    n3 = s.natom * 3
    x_host = torch.empty(n3, dtype=torch.float32, pin_memory=True)
    f_host = torch.empty(n3, dtype=torch.float32, pin_memory=True)
    x0 = e.positions().astype(np.float32)
    v0 = e.velocities().astype(np.float32)
    import ctypes as C
    erg = C.c_double(0)
    e2e_steps = max(10, args.steps // 4)
    xs = [(x0 + np.float32(k * 0.5) * v0).ravel() for k in range(e2e_steps + 3)]
    for k in range(3):
        x_host.numpy()[:] = xs[k]
        e._ok(e.lib.nnpe_force_step(e.h, x_host.data_ptr(), f_host.data_ptr(), C.byref(erg), None))
    torch.cuda.synchronize()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for k in range(e2e_steps):
        x_host.numpy()[:] = xs[3 + k]
        e._ok(e.lib.nnpe_force_step(e.h, x_host.data_ptr(), f_host.data_ptr(), C.byref(erg), None))
    h1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = h0.elapsed_time(h1) / e2e_steps
    e2e_value = s.natom * world / (e2e_ms / 1e3)

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            try:
                rate, threads, sample = cpu_reference(wl, args.cpu_steps)
                cpu = {"value": rate, "unit": "atom-steps/s", "cores": threads, "kind": "reference", "sample": sample}
            except Exception as ex:  # the reference harness is optional on a box without it
                cpu = {"value": None, "unit": "atom-steps/s", "cores": 0, "kind": "reference",
                       "sample": f"unavailable: {ex}"}
        out = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded water box, lattice start equilibrated 300 steps)",
            "config": {"workload": args.workload, "description": wl["desc"], "natom": s.natom,
                       "list_entries_per_atom": round(nlist, 1), "nbuild": info["nbuild"],
                       "l2": "inputs larger than L2 (neighbour list %.0f MB)" % (info["entries"] * 4 / 1e6),
                       "ns_per_day": value / world / s.natom * 0.5 * 86400 * 1e-6},
            "roofline": {"bound": "hbm", "kernel": "k_pair", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": None, "peak_source": src,
                         "kernel_ms": pair_ms, "alg_bytes_per_launch": alg_bytes},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "atom-steps/s", "h2d_bytes_per_step": n3 * 4,
                    "d2h_bytes_per_step": n3 * 4 + 8, "ms_per_step": e2e_ms},
            "clocks": clk.summary(),
            "gpu_launches": int(e.lib.nnpe_launches_per_step(e.h)) * args.steps,
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    e.close()


if __name__ == "__main__":
    main()
