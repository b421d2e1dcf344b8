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
    "water96k-nnp-bf16": dict(n_side=32, bl=99.3, nmol=32000, nnp="bf16", cpu_steps=2,
                              desc="96,000-atom water (32,000 molecules, 99.3 A box): tabulated LJ + DSF Coulomb at 10 A "
                                   "plus the radial-embedding network at 6 A (1->32->64 per species, 4 special-class "
                                   "slots, fitting 256->128->128->1, tanh) with BF16 tcgen05 GEMMs and FP32 accumulation; "
                                   "2 A skin, bonds + angles, dt 0.5 fs NVE, FP64 Verlet state"),
    "water96k-nnp-tbl": dict(n_side=32, bl=99.3, nmol=32000, nnp="tbl", cpu_steps=2,
                             desc="the reference's own tabulated NNP on the 96,000-atom water box: NNPOTENTIAL_TBL at 6 A "
                                  "(20 Gaussian descriptors per special class, 20->128->128->1 tanh fitting network in "
                                  "FP32, its pair tables) plus LJ/DSF at 10 A and bonds + angles, dt 0.5 fs NVE"),
    "water96k-nnp-fp32": dict(n_side=32, bl=99.3, nmol=32000, nnp="fp32", cpu_steps=2,
                              desc="the same 96,000-atom NNP + tabulated workload with the network in FP32 on CUDA cores "
                                   "(the plain form)"),
    "water96k-classical": dict(n_side=32, bl=99.3, nmol=32000, nnp=None, cpu_steps=20,
                               desc="96,000-atom water (32,000 molecules, 99.3 A box), tabulated LJ + DSF Coulomb at "
                                    "10 A, 2 A skin, bonds + angles, dt 0.5 fs NVE, FP64 Verlet state"),
    "water3k-classical": dict(n_side=10, bl=31.04, nmol=None, nnp=None, cpu_steps=400,
                              desc="3,000-atom water (1,000 molecules, 31.04 A box), tabulated LJ + DSF Coulomb at 10 A, "
                                   "2 A skin, bonds + angles, dt 0.5 fs NVE"),
    "gr-refine-30k": dict(mixture=True, natom=30000, rho=0.035, nnp=None, cpu_steps=20,
                          desc="g(r)/S(q) refinement: 30,000-atom two-species LJ + DSF Coulomb liquid (60/40, sigma "
                               "3.0/3.4 A, eps 0.15/0.25 kcal/mol, charges +-0.5 e) at 0.035 A^-3 (94.99 A box); g(r) "
                               "to 15 A in 0.01 A bins (uint64 counts) every step (cell-based every 10), S(q) on 512 "
                               "points in FP64, RMDF (gamma 1) against the weighted S(q) of the same liquid with eps "
                               "x1.1, Andersen 300 K, dt 1 fs"),
    "sqd96k": dict(sqd=True, n_side=32, bl=99.3, nmol=32000, nnp=None, nq=512, qmax=10.0, cpu_qmax=1.2,
                   desc="direct S(q) (SQD) of the 96,000-atom water box: every reciprocal lattice vector of the "
                        "half space with |G| <= 10 A^-1 (2 pi/L spacing), S_t and C_t per type summed over all atoms, "
                        "512 bins; one step = one evaluation on the current positions"),
    "serve256": dict(serve=True, nnp="bf16",
                     desc="served replica stream: 256 seeded requests, water boxes of log-uniform 300-30,000 atoms at "
                          "0.95-1.05 g/cm^3 and 250-400 K (Andersen every 20 steps), 100-5000 steps each (uniform "
                          "integers), Poisson arrivals at 20 req/s; LJ/DSF at 10 A + the BF16 embedding network at 6 A, "
                          "dt 0.5 fs; all replica state device-resident, HBM-budget admission"),
}


def nnp_flops_per_step(natom, pairs6):
    """Algorithmic network FLOPs of one force evaluation: per pair the embedding's two layers
    forward and their input-gradient backward (2*(32 + 32*64) MAC each way), per atom the fitting
    network forward (256*128 + 128*128 + 128 MAC) and backward (128*128 + 128*256 MAC)."""
    per_pair = 2 * 2 * (32 + 32 * 64)
    per_atom = 2 * (256 * 128 + 128 * 128 + 128) + 2 * (128 * 128 + 128 * 256)
    return pairs6 * per_pair + natom * per_atom


def max_over_ranks(x: float, dist=None, device="cuda") -> float:
    """The largest of the ranks' values (the slowest replica's time): every rank calls it at the
    same point; without a process group it returns x."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(base: int, rank: int) -> int:
    """Velocity seed of rank's replica: independent systems of the same workload on each GPU."""
    return base + 7919 * rank


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
        self.first = 0   # index of the last sample taken before the timed region
        self.bracketed = False

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a few hundred ms to start: wait for its first sample so that sampling
            # is running when the timed region begins (a region of a few tens of ms can otherwise
            # end before the first sample)
            t_end = time.time() + 5
            while not self.lines and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
            self.first = max(len(self.lines) - 1, 0)
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            # one sample after the region: with the last one before it, a region shorter than the
            # 50 ms interval is still bracketed by samples taken next to it under the same load
            n = len(self.lines)
            if n - self.first < 3:
                self.bracketed = True
                t_end = time.time() + 1
                while len(self.lines) <= n and time.time() < t_end and self.proc.poll() is None:
                    time.sleep(0.005)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines[self.first:]:
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
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
               "samples": len(sm)}
        if self.bracketed:
            out["note"] = "timed region shorter than a few 50 ms intervals: the samples include the last one before it and the first one after it"
        return out


MIX_SIGMA, MIX_EPS = (3.0, 3.4), (0.15, 0.25)


def build_system(wl, rank=0):
    import cases
    from nnpengine_b200 import systems as S
    if wl.get("mixture"):
        s = S.lj_mixture(wl["natom"], wl["rho"], 0.6, seed=replica_seed(4, rank))
        return s, S.lj_table(2, MIX_SIGMA, MIX_EPS, 10.0, 1000)
    s = S.water_box(wl["n_side"], wl["bl"], seed=replica_seed(2, rank), nmol=wl.get("nmol"))
    r, F, U = S.water_lj_table(10.0, 1000)
    return s, (r, F, U)


def make_engine(s, table, device, nnp=None):
    import cases
    from nnpengine_b200 import engine as E
    from nnpengine_b200 import nnp_model as NM
    F, U = cases.table_as_loaded(table[1], table[2])
    e = E.Engine(device)
    e.set_system(s)
    mixture = s.moltypes[0].n_atom == 1
    e.setup(10.0, 2.0, 15.0 if mixture else 10.0, 1024)
    e.set_pair_table(F, U)
    if not mixture:
        e.set_bonded(s, [E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)], [E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)])
    if nnp == "tbl":   # the reference's tabulated NNP, from its paramfile and weight file
        with tempfile.TemporaryDirectory() as d:
            paths = cases.write_nnp_inputs(NM.gauss_model(h1=128, h2=128), d)
            e.nnp_load(6.0, 750, paths["param"], paths["wt"])
    elif nnp:
        e.nnp_set(NM.embed_model(), 6.0, 750)
        e.nnp_precision(nnp == "bf16")
    return e


def ref_layouts():
    """The reference harness's two thread layouts: its default 3x3x3 = 27 threads as it runs
    (unbound), and its 2x2x2 = 8-thread layout bound one thread per core (OMP_PROC_BIND=close,
    OMP_PLACES=cores)."""
    return [(27, {}), (8, {"OMP_PROC_BIND": "close", "OMP_PLACES": "cores"})]


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_reference(wl, steps: int):
    """The reference's own OpenMP force step on the same system (oracle/_ref/ref_dump_fast*): its
    LJTableCoulDSF + bonded terms, and for network workloads its tabulated NNP (NNPOTENTIAL_TBL at
    6 A, 20 Gaussians per special class, with a 20->128->128->1 float fitting network behind the TF
    C-API shim, serial as the reference configures TF; the reference cannot run the embedding
    network). The MD loop runs `steps` and 2*`steps` steps; the rate is natom*steps over the
    difference of the two loop times, so that set-up and the first list build cancel. Both thread
    layouts run; the faster gives the value. Returns (atom-steps/s, threads, sample, details)."""
    from oracle import orc
    import cases
    from nnpengine_b200 import nnp_model as NM
    s, table = build_system(wl)
    details = []
    with tempfile.TemporaryDirectory() as d:
        f = cases.write_inputs(s, table, d)
        cfg = {"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2, "gr_cutoff": 10,
               "bond": [f"1.0 {cases.WATER_BOND_K}"], "angle": [f"109.47 0 0 {cases.WATER_ANGLE_KC}"],
               "velocity": f["vel"], "mode": "md", "dt": 0.5}
        what = "LJ/DSF table + bonded"
        if wl.get("mixture"):
            from nnpengine_b200 import systems as S
            q, sqex, wt, ff = S.synthetic_sq_target(512, 20.0, 2)
            tpath = os.path.join(d, "sq_target.txt")
            S.write_sq_target(tpath, q, sqex, wt, ff)
            cfg.update({"gr_cutoff": 15, "nq": 512, "qmax": 20, "gr_interval": "1 10", "rmdf": f"0.02 1.0 {tpath}",
                        "dt": 1.0})
            what = "LJ/DSF table, g(r) every step (cell-based every 10), S(q) and RMDF"
        if wl.get("nnp"):
            paths = cases.write_nnp_inputs(NM.gauss_model(h1=128, h2=128), d)
            cfg["nnp"] = f"6.0 750 {paths['param']} {paths['wt']}"
            what += (" + its tabulated NNP (20 Gaussians per special class, 20->128->128->1 float network via the "
                     "C-API shim, serial as the reference configures TF)")
        for threads, envx in ref_layouts():
            env = dict(os.environ, **envx)
            t = []
            for n in (steps, 2 * steps):
                out = orc.run_ref_dump({**cfg, "steps": n, "log_interval": n}, os.path.join(d, f"o{threads}_{n}"),
                                       fast=True, timeout=1800, threads=threads, env=env)
                t.append(float(out["info"]["t_loop"]))
            dt = max(t[1] - t[0], 1e-9)
            details.append({"threads": threads, "env": envx, "loop_s": t, "steps": [steps, 2 * steps],
                            "atom_steps_per_s": s.natom * steps / dt})
    best = max(details, key=lambda r: r["atom_steps_per_s"])
    ncpu = os.cpu_count()
    sample = (f"{s.natom}-atom system ({what}); MD loop of {steps} and {2 * steps} steps, rate from the difference; "
              f"layouts 27 threads (3x3x3, unbound) and 8 threads (2x2x2, one per core), the faster reported; "
              f"{ncpu}-CPU host ({cpu_model()})")
    return best["atom_steps_per_s"], best["threads"], sample, details


def cpu_sqd_reference(wl):
    """The reference's SQD (grsq.cpp:362-573, its OpenMP code in oracle/_ref) on the same positions, at
    a smaller q_max so that the sample takes seconds; returns (atom-G evaluations/s, threads, sample)."""
    from oracle import orc
    import cases
    s, table = build_system(wl)
    with tempfile.TemporaryDirectory() as d:
        f = cases.write_inputs(s, table, d)
        cfg = {"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2, "gr_cutoff": 10,
               "velocity": f["vel"], "mode": "md", "steps": 0, "dt": 0.5, "log_interval": 1,
               "sqd": f"{wl['nq']} {wl['cpu_qmax']}"}
        out = orc.run_ref_dump(cfg, os.path.join(d, "o"), fast=True, timeout=1800)
    info = out["info"]
    rate = s.natom * int(info["sqd_ngv"]) / float(info["t_sqd"])
    return rate, int(info["threads"]), (f"SQD of the {s.natom}-atom box at q_max {wl['cpu_qmax']} A^-1 "
                                        f"({int(info['sqd_ngv'])} G vectors), {info['threads']} OpenMP threads on a "
                                        f"{os.cpu_count()}-CPU host")


def sqd_bench(args, wl, local):
    """Direct S(q) on the device: atom-G evaluations per second over K evaluations (CUDA events on the
    library stream), the same through nnpe_sqd_compute with its result copied back (e2e)."""
    import torch
    s, table = build_system(wl)
    e = make_engine(s, table, local, None)
    stream = torch.cuda.ExternalStream(e.lib.nnpe_stream(e.h))
    ngv = e.sqd_setup(wl["nq"], wl["qmax"])
    for _ in range(args.warmup):
        e.lib.nnpe_sqd_compute(e.h)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t0.record(stream)
        for _ in range(args.steps):   # each call also copies the per-bin result back and synchronises
            e._ok(e.lib.nnpe_sqd_compute(e.h))
        t1.record(stream)
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / args.steps
    evals = s.natom * ngv
    value = evals / (ms / 1e3)
    # arithmetic per atom-G pair: one complex multiply (4 mul/fma) + two adds = 8 FLOP; nominal FP32
    # CUDA-core peak 148 SMs x 128 lanes x 2 x 1.965 GHz
    peak = 148 * 128 * 2 * 1.965e9 / 1e12
    ach = evals * 8 / (ms / 1e3) / 1e12
    e.close()
    return dict(value=value, ms=ms, ngv=ngv, clocks=clk.summary(),
                roofline={"bound": "fp32", "kernel": "k_sqd_runs + k_sqd_bins", "achieved": ach, "peak": peak,
                          "unit": "TFLOP/s", "frac": ach / peak, "traffic": None,
                          "peak_source": "nominal FP32 CUDA-core rate (no measured FP32 peak on this pool)",
                          "alg_flops_per_launch": evals * 8})


def serve_bench(args, wl):
    """The served replica stream: requests are submitted at their Poisson arrival times by a host
    thread while the server's worker runs the resident replicas; throughput is the stream's work
    over its makespan (first arrival to last completion, host clock, as a client sees it) and
    latency is completion time minus arrival time per request."""
    import torch
    import cases
    from nnpengine_b200 import engine as E
    from nnpengine_b200 import nnp_model as NM
    from nnpengine_b200 import systems as S
    from nnpengine_b200.serve import Server
    nreq = args.serve_requests
    trace = S.serving_trace(nreq, seed=3, rate=args.serve_rate)
    for t in trace:
        t["nsteps"] = max(20, int(round(t["nsteps"] * args.serve_scale)))
    boxes = [S.water_request_box(t["natom"], t["density"], t["seed"], t["temperature"]) for t in trace]
    r, F, U = S.water_lj_table(10.0, 1000)
    F, U = cases.table_as_loaded(F, U)
    free, total = torch.cuda.mem_get_info()
    budget = int(min(0.8 * free, 120e9))
    srv = Server(0, ntype=2, table=(F, U), bcoef=[E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)],
                 acoef=[E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)], nnp=NM.embed_model(), bf16=True,
                 chunk_steps=20, dt=0.5, max_replicas=args.serve_slots, hbm_budget=budget,
                 autotune=not args.no_autotune)
    # warm-up requests (module loading, first graph captures), untimed
    warm = [srv.submit(S.water_request_box(n, 1.0, 90 + k, 300.0), 40, 300.0, k)
            for k, n in enumerate([300, 3000, 30000][:max(1, args.warmup)])]
    for w in warm:
        srv.wait(w, 600)
    ids = [None] * nreq
    t_arr = [0.0] * nreq

    def submitter():
        t0 = time.perf_counter()
        for k, (t, b) in enumerate(zip(trace, boxes)):
            delay = t["t"] - trace[0]["t"] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            t_arr[k] = time.perf_counter()
            ids[k] = srv.submit(b, t["nsteps"], t["temperature"], t["seed"])

    with ClockSampler(0) as clk:
        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        t_wait = time.perf_counter()
        while True:   # progress on stderr while the stream drains
            try:
                srv.drain(10.0)
                break
            except Exception:
                inf = srv.info()
                sys.stderr.write(f"serving: {time.perf_counter() - t_wait:.0f}s after the last arrival: {inf}\n")
                sys.stderr.flush()
                if time.perf_counter() - t_wait > args.serve_timeout:
                    raise RuntimeError(f"served stream not drained after {args.serve_timeout} s: {inf}")
    t_end = time.perf_counter()
    # the server clock (t_submit/t_done) and the host clock differ by a constant offset per request
    stats = [srv.stats(i) for i in ids]
    first_error = None
    for i, st in sorted(zip(ids, stats), key=lambda x: x[1]["t_done"]):
        if st["status"] < 0:
            try:
                srv.wait(i, 0.0)
            except Exception as ex:
                first_error = f"{ex} (request {i}, {st['natom']} atoms, {st['nsteps']} steps)"
            break
    lat = np.array([st["t_done"] - st["t_submit"] for st in stats])
    ok = sum(1 for st in stats if st["status"] == 2)
    first_submit = min(st["t_submit"] for st in stats)
    makespan = max(st["t_done"] for st in stats) - first_submit
    steps = sum(t["nsteps"] for t in trace)
    atom_steps = sum(t["nsteps"] * b.natom for t, b in zip(trace, boxes))
    info = srv.info()
    srv.close()
    return dict(replica_steps_per_s=steps / makespan, atom_steps_per_s=atom_steps / makespan, makespan_s=makespan,
                p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)), mean_s=float(lat.mean()),
                completed=ok, requests=nreq, total_steps=steps, total_atom_steps=atom_steps,
                peak_resident=info["peak_resident"], peak_bytes=info["peak_bytes"], hbm_budget=budget, first_error=first_error,
                clocks=clk.summary(), wall_after_last_submit_s=t_end - t_arr[-1])


def refine_setup(e, s, wl, device, args):
    """RMDF target: the weighted S(q) that the reference itself computed (RMDF's sq, what
    RMDF::dumpSQ writes) for the same 30,000-atom liquid with every eps scaled by 1.1, after 500
    steps at 1 fs under its Andersen thermostat at 300 K (tests/golden/mixture30k.npz, written by
    tests/golden/make_golden.py from oracle/_ref). Then g(r) every step (cell-based every 10) and
    RMDF with gamma 1 on the workload's engine."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "mixture30k.npz"))
    target, wt, ff = g["target_sq"].astype(np.float64), g["target_wt"], g["target_ff"]
    e.gr_setup(1000, 512, 20.0, gr_interval=1, gr_interval_long=10)
    e.rmdf_set(target[None], wt[None], ff[None], args.rmdf_strength, 1.0)
    return target


def nve_drift(e, natom, ps, dt=0.5):
    """Total energy over `ps` picoseconds of NVE (FP64 energies on log steps): linear-fit slope and
    largest excursion from the first value."""
    nsteps = int(round(ps * 1000 / dt))
    every = max(1, nsteps // 40)
    lg = e.run(nsteps + 1, log_interval=every, graph=True)
    t = np.array([r["step"] for r in lg], float)
    t = (t - t[0]) * dt / 1000.0
    etot = np.array([r["erg"] + r["ekin"] for r in lg])
    slope = float(np.polyfit(t, etot, 1)[0]) if len(t) > 1 else 0.0
    return {"ps": ps, "dt_fs": dt, "steps": nsteps, "log_points": len(lg), "etot_first": float(etot[0]),
            "etot_last": float(etot[-1]), "max_abs_dev_kcal_mol": float(np.abs(etot - etot[0]).max()),
            "slope_kcal_mol_per_ps": slope, "slope_kcal_mol_per_atom_per_ns": slope * 1000.0 / natom,
            "ekin_mean_kcal_mol": float(np.mean([r["ekin"] for r in lg])),
            "temperature_mean_k": float(np.mean([r["temperature"] for r in lg]))}


def profile_traffic(kernel_names):
    """DRAM bytes per launch of the named kernels from the committed ncu summary (None if absent)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p)).get("kernels", {})
    if not all(k in d for k in kernel_names):
        return None
    return sum(d[k]["dram_bytes_per_launch"] for k in kernel_names)


def time_enqueue(e, stream, which, reps):
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e._ok(e.lib.nnpe_profile_enqueue(e.h, which))
    a.record(stream)
    for _ in range(reps):
        e._ok(e.lib.nnpe_profile_enqueue(e.h, which))
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def force_errors(s, table, x, device, m=None):
    """Force and energy errors of the GPU forms against the FP64 oracle at positions x (float32,
    atom-id order): the BF16 tensor-core network and the plain FP32 network, each as the network
    term alone (6 A) and as the whole force (LJ/DSF at 10 A + bonded + network). Error = RMS of the
    per-atom force difference over the RMS of the FP64 force; energies relative."""
    import cases
    from nnpengine_b200 import engine as E
    from nnpengine_b200 import nnp_model as NM
    from oracle import orc
    m = m or NM.embed_model()
    F, U = cases.table_as_loaded(table[1], table[2])
    e = make_engine(s, table, device, "bf16")
    e.set_positions(x)
    e.set_velocities(np.zeros_like(x))
    e.list_build()
    got = {}
    for prec in ("bf16", "fp32"):
        e.nnp_precision(prec == "bf16")
        erg, _ = e.compute_forces(True)
        got[prec] = (e.forces().astype(np.float64), erg)
    e.pair_enable(False)
    e.set_bonded(s, [], [], [])
    for prec in ("bf16", "fp32"):
        e.nnp_precision(prec == "bf16")
        erg, _ = e.compute_forces(True)
        got[prec + "_net"] = (e.forces().astype(np.float64), erg)
    errors = e.device_errors()
    e.close()
    sx = dataclass_replace_x(s, x)
    o = orc.Restated(sx, "f64")
    assert o.rebuild(x, 10, 2, 12) == 0
    fp, ep, _ = o.pair_forces(F, U, 10.0)
    fb, eb, _ = o.bonded(E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)[None],
                         E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)[None], np.zeros((1, 4), np.float32))
    o6 = orc.Restated(sx, "f64")
    assert o6.rebuild(x, 6, 2, 8) == 0
    r = o6.nnp_emb(6.0, m.scale, m.e1, m.e2, m.embw, m.h1, m.h2, m.fitw)
    ref_net, ref_tot = r["f"], fp + fb + r["f"]
    e_net, e_tot = r["e_net"], ep + eb + r["e_net"]
    out = {"oracle": "FP64 C restatement (oracle/restate) at the final state of the timed run", "natom": s.natom,
           "device_error_bits": errors, "force_rms_fp64": {"network": float(np.sqrt((ref_net ** 2).sum(1).mean())),
                                                           "total": float(np.sqrt((ref_tot ** 2).sum(1).mean()))}}
    for prec in ("bf16", "fp32"):
        out[prec] = {"force_rel_rmse_network": cases.rel_rms(got[prec + "_net"][0], ref_net),
                     "force_rel_rmse_total": cases.rel_rms(got[prec][0], ref_tot),
                     "energy_rel_err_network": abs(got[prec + "_net"][1] - e_net) / abs(e_net),
                     "energy_rel_err_total": abs(got[prec][1] - e_tot) / abs(e_tot)}
    out["bar"] = "BF16: force RMSE <= 1% of the FP64 force RMS; FP32: 1e-5 force, 1e-6 energy"
    return out


def dataclass_replace_x(s, x):
    import dataclasses
    return dataclasses.replace(s, x=np.asarray(x, np.float32).reshape(-1, 3))


def same_model_gpu(s, table, x, v, device, steps, warmup=10):
    """The reference's own tabulated NNP (the model its CPU path runs: 20 Gaussians per special
    class, 20->128->128->1, read from the reference-format paramfile and weight file) plus LJ/DSF
    and bonded terms on the GPU (FP32 network on CUDA cores), NVE at 0.5 fs from state (x, v);
    atom-steps/s over `steps` graph-replayed steps (CUDA events on the library's stream)."""
    import torch
    e = make_engine(s, table, device, "tbl")
    e.set_positions(x)
    e.set_velocities(v)
    e.verlet(0.5, True)
    e.run(warmup, log_interval=warmup, graph=True)
    stream = torch.cuda.ExternalStream(e.lib.nnpe_stream(e.h))
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    e.run(steps, log_interval=steps, graph=True)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    e.close()
    return s.natom / (ms / 1e3), ms


def reference_workload(name):
    """The workload the reference's CPU path runs for a GPU workload: the same system; for the
    embedding network (which the reference cannot run) its own tabulated NNP; for serving one
    3000-atom replica."""
    wl = WORKLOADS[name]
    if wl.get("serve"):
        return WORKLOADS["water3k-classical"] | {"nnp": "bf16", "cpu_steps": 10}
    return wl


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=0, help="timed steps (0: 2000 for gr-refine-30k, the configured "
                    "refinement length, else 1000)")
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="water96k-nnp-bf16", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip timing the plain FP32 network alongside")
    ap.add_argument("--no-errors", action="store_true", help="skip the FP64 force-error evaluation")
    ap.add_argument("--no-same-model", action="store_true", help="skip the GPU run of the reference's own model")
    ap.add_argument("--exact", action="store_true", help="pair forces in the reference's exact float sequence")
    ap.add_argument("--no-autotune", action="store_true", help="default grids for the tensor-core kernels")
    ap.add_argument("--prune", type=float, default=None,
                    help="dynamic list-pruning margin in A (0: off; default: the library's 0.5 A)")
    ap.add_argument("--cpu-steps", type=int, default=0, help="reference MD-loop sample: N and 2N steps (0: per workload)")
    ap.add_argument("--equil", type=int, default=5000)
    ap.add_argument("--serve-requests", type=int, default=256)
    ap.add_argument("--serve-scale", type=float, default=1.0, help="multiply every request's step count")
    ap.add_argument("--serve-slots", type=int, default=64)
    ap.add_argument("--serve-rate", type=float, default=20.0, help="Poisson arrival rate of the request stream [1/s]")
    ap.add_argument("--serve-timeout", type=float, default=900.0)
    ap.add_argument("--drift-ps", type=float, default=-1.0,
                    help="after the timed steps, NVE for this many ps (-1: 10 ps for the network workloads)")
    ap.add_argument("--rmdf-strength", type=float, default=0.02)
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.steps <= 0:
        args.steps = 2000 if wl.get("mixture") else 1000

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        rwl = reference_workload(args.workload)
        unit = "atom-G evaluations/s" if wl.get("sqd") else "atom-steps/s"
        details = None
        if wl.get("sqd"):
            rate, threads, sample = cpu_sqd_reference(wl)
        else:
            rate, threads, sample, details = cpu_reference(rwl, args.cpu_steps or rwl.get("cpu_steps", 20))
        cfg = {"workload": args.workload, "description": wl["desc"]}
        if wl.get("nnp") == "bf16" or wl.get("serve"):
            cfg["model"] = ("the reference's own tabulated NNP (it cannot run the embedding network of this "
                            "workload); the GPU on this same model is the 'same_model' block of the GPU arm's line")
        print(json.dumps({
            "impl": "reference", "metric": unit, "value": rate, "unit": unit, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "config": cfg,
            "cpu_baseline": {"value": rate, "unit": unit, "cores": threads, "kind": "reference", "sample": sample,
                             "layouts": details},
            "e2e": {"value": rate, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import torch
    torch.cuda.set_device(local)
    if wl.get("sqd"):
        if rank != 0:
            return
        r = sqd_bench(args, wl, local)
        cpu = None
        if not args.no_cpu_baseline:
            rate, threads, sample = cpu_sqd_reference(wl)
            cpu = {"value": rate, "unit": "atom-G evaluations/s", "cores": threads, "kind": "reference", "sample": sample}
        nq = wl["nq"]
        print(json.dumps({
            "metric": "atom-G evaluations/s", "value": r["value"], "unit": "atom-G evaluations/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 phases and bin sums)",
            "data": "synthetic (seeded water box, lattice start)",
            "config": {"workload": args.workload, "description": wl["desc"], "natom": 96000, "g_vectors": r["ngv"],
                       "nq": nq, "qmax": wl["qmax"], "l2": "inputs in L2 (1.5 MB of positions); compute-bound"},
            "roofline": r["roofline"], "cpu_baseline": cpu, "clocks": r["clocks"],
            "e2e": {"value": r["value"], "unit": "atom-G evaluations/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": nq * 3 * 8, "note": "positions are device-resident; each step returns "
                    "the per-bin S(q) to the host inside the timed region"},
            "gpu_launches": 2 * args.steps}))
        return
    if wl.get("serve"):
        if rank != 0:
            return
        res = serve_bench(args, wl)
        cpu = None
        if not args.no_cpu_baseline:
            try:
                rwl = reference_workload(args.workload)
                rate, threads, sample, details = cpu_reference(rwl, args.cpu_steps or rwl["cpu_steps"])
                cpu = {"value": rate, "unit": "atom-steps/s", "cores": threads, "kind": "reference",
                       "sample": sample + "; the reference runs one system per process, so a stream is sequential runs",
                       "layouts": details}
            except Exception as ex:
                cpu = {"value": None, "unit": "atom-steps/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {ex}"}
        print(json.dumps({
            "metric": "replica-steps/s", "value": res["replica_steps_per_s"], "unit": "replica-steps/s", "n_gpus": 1,
            "steps": res["total_steps"], "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16", "data": "synthetic (seeded request stream)",
            "config": {"workload": args.workload,
                       "description": wl["desc"].replace("at 20 req/s", "at %g req/s" % args.serve_rate),
                       "serve_scale": args.serve_scale,
                       "arrival_rate_per_s": args.serve_rate,
                       "slots": args.serve_slots, "autotune": not args.no_autotune, "timing": "host clock: first arrival to last completion"},
            "latency_s": {"p50": res["p50_s"], "p99": res["p99_s"], "mean": res["mean_s"]},
            "serving": res, "cpu_baseline": cpu, "clocks": res["clocks"],
            "e2e": {"value": res["replica_steps_per_s"], "unit": "replica-steps/s",
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "note": "every request's system goes host->device at admission and its final state device->host"}}))
        return
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist = dist_mod
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    s, table = build_system(wl, rank)
    e = make_engine(s, table, local, wl.get("nnp"))
    e.pair_exact(args.exact)
    if args.prune is not None:
        e.set_prune(args.prune)
    stream = torch.cuda.ExternalStream(e.lib.nnpe_stream(e.h))
    refine = wl.get("mixture")
    if refine:
        refine_setup(e, s, wl, local, args)
    # untimed equilibration of the classical model from the lattice start (Andersen at 300 K,
    # dt 1 fs, the 5 ps of the workload's definition), then the network on and NVE at dt=0.5 fs
    e.verlet(1.0, True)
    e.thermostat("andersen", 300.0, 300.0, interval=1, frac=0.1, seed=replica_seed(11, rank), total_steps=0)
    if wl.get("nnp"):
        e.nnp_enable(False)
    if args.equil:
        e.run(args.equil, log_interval=args.equil, graph=True)
    if wl.get("nnp"):
        e.nnp_enable(True)
    if refine:   # the refinement runs under the thermostat at dt 1 fs, as the reference's classical mode
        e.thermostat("andersen", 300.0, 300.0, interval=10, frac=0.1, seed=12, total_steps=0)
    else:
        e.thermostat("none")
        e.verlet(0.5, True)
    grids = None
    if wl.get("nnp") == "bf16":
        grids = e.nnp_autotune(reps=5) if not args.no_autotune else e.nnp_get_grids()
    wlog = e.run(args.warmup, log_interval=max(args.warmup, 1), graph=True)
    nbuild0 = wlog[-1]["nbuild"] if wlog else 0
    nprune0 = e.prune_info()["nprune"]

    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t0.record(stream)
        log = e.run(args.steps, log_interval=max(1, args.steps // 10) if refine else args.steps, graph=True)
        t1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(t0.elapsed_time(t1), dist)
    info = e.list_info()
    nbuild_timed = (log[-1]["nbuild"] if log else info["nbuild"]) - nbuild0
    pinfo = e.prune_info()
    pruning = {"delta_A": round(pinfo["delta"], 3), "active": pinfo["active"],
               "prunes_in_timed_steps": pinfo["nprune"] - nprune0,
               "entries_per_atom": round(pinfo["entries"] / s.natom, 1) if pinfo["active"] else None}
    value = s.natom * args.steps * world / (ms / 1e3)
    launches = int(e.lib.nnpe_launches_per_step(e.h))

    # state of the timed run, the start of the host-buffer (e2e) steps below
    x_e2e0, v_e2e0 = e.positions().astype(np.float32), e.velocities().astype(np.float32)

    drift = None
    drift_ps = args.drift_ps if args.drift_ps >= 0 else (10.0 if wl.get("nnp") else 0.0)
    if drift_ps > 0 and not refine:
        drift = nve_drift(e, s.natom, drift_ps)

    plain = None
    if wl.get("nnp") == "bf16" and not args.no_compare:
        e.nnp_precision(False)
        e.run(5, log_interval=5, graph=True)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        nfp = min(60, max(20, args.steps // 4))
        a.record(stream)
        e.run(nfp, log_interval=nfp, graph=True)
        b.record(stream)
        torch.cuda.synchronize()
        plain = s.natom * world / (max_over_ranks(a.elapsed_time(b), dist) / nfp / 1e3)
        e.nnp_precision(True)

    # per-kernel-class device time (CUDA events on the library stream); these launches change the
    # dynamical state (forces accumulate, velocities advance), so they come after every run that
    # evolves it
    reps = 20
    e.compute_forces(ev=False)
    kms = {"pair": time_enqueue(e, stream, 0, reps), "bonded": time_enqueue(e, stream, 2, reps),
           "verlet": time_enqueue(e, stream, 4, reps), "rebuild": time_enqueue(e, stream, 1, 5),
           "pair_energy_step": time_enqueue(e, stream, 7, reps)}
    if wl.get("nnp"):
        kms["network"] = time_enqueue(e, stream, 3, reps)
    hbm, bf16, bf16s, src = peaks()
    nlist = info["entries"] / s.natom
    if wl.get("nnp") in ("bf16", "fp32"):
        # network pairs inside 6 A from the compact list of the last evaluation
        G, dG, ea = e.nnp_get()
        pairs6 = int(e.lib.nnpe_nnp_pairs(e.h))
        flops = nnp_flops_per_step(s.natom, pairs6)
        ach = flops / (kms["network"] / 1e3) / 1e12
        tc_kernels = ["k_tc_desc2", "k_tc_fit", "k_tc_force2<0>"]
        roof = {"bound": "tensor", "kernel": "network (k_tc_desc2 + k_tc_fit + k_tc_force2)" if wl["nnp"] == "bf16"
                else "network (FP32 CUDA cores)", "achieved": ach, "peak": bf16, "unit": "TFLOP/s", "frac": ach / bf16,
                "traffic": profile_traffic(tc_kernels) if wl["nnp"] == "bf16" else None,
                "traffic_unit": "bytes per launch (DRAM read+write, ncu)", "peak_source": src,
                "kernel_ms": kms["network"], "alg_flops_per_launch": flops, "pairs_in_6A_per_atom": pairs6 / s.natom}
    else:
        # the entries the pair kernel reads: the pruned copy's when pruning is on
        alg_bytes = s.natom * (4 * (pruning["entries_per_atom"] or nlist) + 48)
        ach = alg_bytes / (kms["pair"] / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": "k_pair", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "traffic": profile_traffic([f"k_pair<0,0>:{args.workload}"]), "traffic_unit": "bytes per launch (DRAM read+write, ncu)",
                "peak_source": src, "kernel_ms": kms["pair"], "alg_bytes_per_launch": alg_bytes}
    gr_info = None
    if refine:
        kms["gr_cell"] = time_enqueue(e, stream, 5, 10)
        kms["gr_list"] = time_enqueue(e, stream, 6, 10)
        ordered = float(e.gr_counts(False).sum())
        exp = [r["erg_exp"] for r in log]
        gr_info = {"ordered_pairs_per_cell_tally": ordered,
                   "cell_tally_pair_evaluations_per_s": ordered / (kms["gr_cell"] / 1e3),
                   "rmdf_penalty_first_last": [exp[0], exp[-1]] if exp else None, "rmdf_strength": args.rmdf_strength,
                   "target": "weighted S(q) of the eps x1.1 liquid after 500 steps under the reference's Andersen thermostat, "
                             "computed by the reference (oracle/_ref, RMDF's sq)"}

    # the stated error of the timed state against the FP64 oracle, and the GPU on the reference's
    # own model (rank 0; no collective inside either)
    errs = None
    if wl.get("nnp") == "bf16" and not args.no_errors and rank == 0:
        errs = force_errors(s, table, x_e2e0, local)
    same = None
    if wl.get("nnp") == "bf16" and not args.no_same_model and rank == 0:
        nsm = max(20, min(200, args.steps))
        rate_g, ms_g = same_model_gpu(s, table, x_e2e0, v_e2e0, local, nsm)
        same = {"workload": "water96k-nnp-tbl", "description": WORKLOADS["water96k-nnp-tbl"]["desc"],
                "gpu_value": rate_g, "gpu_ms_per_step": ms_g, "gpu_steps": nsm, "unit": "atom-steps/s",
                "reference_value": None, "gpu_over_reference": None}

    e2e = None
    if not args.no_e2e:
        import ctypes as C
        n3 = s.natom * 3
        f_host = torch.empty(n3, dtype=torch.float32, pin_memory=True)
        x0, v0 = x_e2e0, v_e2e0
        erg = C.c_double(0)
        e2e_steps = min(100, max(10, args.steps // 4))   # each step has its own pinned buffer (1.15 MB at 96k)
        # each step's positions in their own pinned host buffer, as a host run loop holds its state
        xs = [torch.from_numpy((x0 + np.float32(k * 0.5) * v0).ravel().astype(np.float32)).pin_memory()
              for k in range(e2e_steps + 3)]
        for k in range(3):
            e._ok(e.lib.nnpe_force_step(e.h, xs[k].data_ptr(), f_host.data_ptr(), None, None))
        torch.cuda.synchronize()
        nb_e2e0 = e.list_info()["nbuild"]
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        for k in range(e2e_steps):   # forces every step; the energy only on log steps, as run.cpp:309-342
            e._ok(e.lib.nnpe_force_step(e.h, xs[3 + k].data_ptr(), f_host.data_ptr(), None, None))
        h1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(h0.elapsed_time(h1), dist) / e2e_steps
        e2e = {"value": s.natom * world / (e2e_ms / 1e3), "unit": "atom-steps/s", "h2d_bytes_per_step": n3 * 4,
               "d2h_bytes_per_step": n3 * 4, "ms_per_step": e2e_ms, "steps": e2e_steps,
               "list_builds": e.list_info()["nbuild"] - nb_e2e0,
               "call": "nnpe_force_step (positions in, forces out, list check/rebuild on device; energies are "
                       "evaluated on log steps only, as the reference's step)"}

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            try:
                rwl = reference_workload(args.workload)
                rate, threads, sample, details = cpu_reference(rwl, args.cpu_steps or rwl.get("cpu_steps", 20))
                cpu = {"value": rate, "unit": "atom-steps/s", "cores": threads, "kind": "reference", "sample": sample,
                       "layouts": details}
                if same is not None:
                    same["reference_value"] = rate
                    same["gpu_over_reference"] = same["gpu_value"] / rate
            except Exception as ex:  # the reference harness is optional on a box without it
                cpu = {"value": None, "unit": "atom-steps/s", "cores": 0, "kind": "reference",
                       "sample": f"unavailable: {ex}"}
        cfg = {"workload": args.workload, "description": wl["desc"], "natom": s.natom,
               "list_entries_per_atom": round(nlist, 1), "rebuilds_in_timed_steps": nbuild_timed,
               "list_pruning": pruning,
               "l2": "inputs larger than L2 (neighbour list %.0f MB)" % (info["entries"] * 4 / 1e6),
               "ns_per_day": value / world / s.natom * 0.5 * 86400 * 1e-6, "kernel_ms": kms,
               "pair_math": "exact float sequence" if args.exact else "rsqrt+FMA (same cutoff test)"}
        if grids is not None:
            cfg["tc_grids"] = {"desc": grids[0], "force": grids[1], "autotuned": not args.no_autotune}
        if plain is not None:
            cfg["plain_fp32_value"] = plain
            cfg["bf16_over_fp32"] = value / plain
        if gr_info is not None:
            cfg["gr_refinement"] = gr_info
        if drift is not None:
            cfg["nve_drift"] = drift
        if errs is not None:
            cfg["force_error_vs_fp64"] = errs
        if same is not None:
            cfg["same_model"] = same
        out = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16" if wl.get("nnp") == "bf16" else "f32",
            "data": "synthetic (seeded water box, lattice start equilibrated %d steps)" % args.equil,
            "config": cfg, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
            "gpu_launches": launches * args.steps,
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    e.close()


if __name__ == "__main__":
    main()
