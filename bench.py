#!/usr/bin/env python
"""Benchmark: wide-box virtual screen through the batched + adjoint docking path.

Workload (synthetic stand-in for the reference's screening sets): an 8,000
heavy-atom receptor (uniform in a 60 A-radius ball, >= 2.8 A separation),
a 70x70x70 A box at 0.375 A (188^3 points x 8 XS maps, built once and
reported separately), and ligands of 15-45 heavy atoms / 2-12 torsions,
each docked with 6,500 Monte-Carlo chains (RILC-BFGS local search, heuristic
search depth) followed by GPU clustering, refinement and rescoring of its
top 20 poses.  One step = one batch of ligands through vd_dock_batched (one
persistent launch over all (ligand, chain) items).  The plain form
(vd_dock_plain, one ligand per launch) is timed beside it on the ligands of
the first timed batch.

Run: python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Under torchrun each rank docks its own ligand batches (weak scaling, no
data-path collective); time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "vina-cuda_b200"))

METRIC = "ligands/s (batched + adjoint docking, wide-box screen)"
UNIT = "ligands/s"
BOX = 70.0
REC_ATOMS, REC_RADIUS = 8000, 60.0
LIG_ATOMS, LIG_TORS = (15, 45), (2, 12)
CHAINS = 6500
SEED = 20261203


def args_():
    a = argparse.ArgumentParser()
    a.add_argument("--gpus", type=int, default=1)
    a.add_argument("--steps", type=int, default=8)
    a.add_argument("--warmup", type=int, default=3)
    a.add_argument("--impl", default="ours", choices=["ours", "reference"])
    a.add_argument("--batch", type=int, default=64, help="ligands per step")
    a.add_argument("--chains", type=int, default=CHAINS)
    a.add_argument("--e2e-steps", type=int, default=0,
                   help="timed batches re-run end to end (0 = all K, the same batches as the timed region)")
    a.add_argument("--no-cpu-baseline", action="store_true")
    a.add_argument("--cpu-ligands", type=int, default=3, help="whole ligands per CPU sample step")
    a.add_argument("--no-configs", action="store_true", help="skip the plain / adjoint / uneven-batch lines")
    a.add_argument("--launch-shape", type=int, default=0, help="docking kernel shape (0 = autotuned, 1-3 pinned)")
    a.add_argument("--configs", default="plain,adjoint,uneven", help="secondary lines to run (comma list)")
    a.add_argument("--only-configs", action="store_true", help="skip the headline; print the secondary lines")
    return a.parse_args()


def dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_inputs(rank, n_ligs):
    from vdock import synth
    xyz, xs = synth.receptor(REC_ATOMS, REC_RADIUS, SEED)
    ligs = synth.ligand_set(n_ligs, LIG_ATOMS, LIG_TORS, SEED + 7919 * (rank + 1))
    return xyz, xs, ligs


def lig_bytes(lig):
    """Algorithmic bytes of one BFGS evaluation: 8 FP32 grid corners per
    heavy atom and two (e, dE/dr) table entries per intra pair."""
    heavy = int((lig["xs"] >= 0).sum())
    return 32 * heavy + 16 * len(lig["pairs"])


def lig_flops(lig):
    """Algorithmic FP32 operations of one BFGS evaluation (forward + adjoint):
    ~115 per heavy atom (trilinear value and gradient ~70, kinematics ~30,
    adjoint ~15) and ~25 per intra pair."""
    heavy = int((lig["xs"] >= 0).sum())
    return 115 * heavy + 25 * len(lig["pairs"])


def fp32_roof(flops, ms, clk, device):
    """Fraction of the FP32 peak (SMs x 128 lanes x 2 flops per FMA x median
    SM clock) the docking kernel's algorithmic flops reach."""
    import torch
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = clk.get("sm_mhz") or 1965.0
    peak = sms * 128 * 2 * mhz * 1e6
    return {"achieved_tflops": flops / (ms / 1e3) / 1e12, "peak_tflops": peak / 1e12,
            "frac": flops / (ms / 1e3) / peak, "model": "115 x heavy atoms + 25 x intra pairs per evaluation"}


# DRAM bytes and L1 data-pipe (LSU) wavefronts of dock_kernel per
# algorithmic byte (lig_bytes x evaluations), per launch shape, from a
# one-pass ncu capture of one full launch of this workload (the first timed
# batch: 64 ligands x 6,500 chains, 266 M evaluations, 1.91 TB algorithmic;
# dram__bytes_read.sum + dram__bytes_write.sum = 151.5 GB,
# l1tex__data_pipe_lsu_wavefronts.sum = 195.2 G; summarised in
# profiles/dock_kernel_wide_box_screen.txt).  Wavefronts track the
# algorithmic bytes across ligand sizes (0.1009 per byte on a 4-ligand
# launch of small ligands, 0.1020 on the full one) where a per-evaluation
# figure does not (463 vs 733), so the bench scales them by the algorithmic
# bytes of each timed launch.  The kernel's limit is that pipe, one
# wavefront per SM per cycle.  Shapes not captured report neither.
DOCK_DRAM_PER_ABYTE = {4: 0.07919}
DOCK_L1_WAVEFRONTS_PER_ABYTE = {4: 0.10198}
DOCK_SHAPES = 3  # launch shapes the docking autotuner explores (register budgets 64 / 80 / 128)
# L1 data-pipe (LSU) wavefronts of one grid build of this workload (188^3
# points x 8 maps, 8,000-atom receptor), from the ncu capture summarised in
# profiles/grid_build_kernel_70A_8types.txt (l1tex__data_pipe_lsu_wavefronts.sum
# of one grid_build_kernel launch).  The kernel's limit is that pipe: one
# wavefront per SM per cycle; every in-range (point, receptor atom) pair reads
# one 32-byte table row, about one wavefront.
GRID_L1_WAVEFRONTS = 128_461_116


def grid_l1_roof(ms, clk, device):
    """Fraction of the L1 data-pipe wavefront roof the grid build reaches:
    wavefronts per build (ncu) / (build time x SMs x SM clock x 1 wavefront
    per SM per cycle), at the median SM clock sampled during the timed region."""
    if GRID_L1_WAVEFRONTS is None:
        return {"frac_of_l1_wavefront_roof": None}
    import torch
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = clk.get("sm_mhz") or 1965.0
    peak = sms * mhz * 1e6  # wavefronts per second
    return {"l1_wavefronts": GRID_L1_WAVEFRONTS, "l1_wavefronts_per_s": GRID_L1_WAVEFRONTS / (ms / 1e3),
            "frac_of_l1_wavefront_roof": GRID_L1_WAVEFRONTS / (ms / 1e3) / peak}


def dock_l1_roof(shape, abytes, ms, clk, device):
    """Fraction of the L1 data-pipe wavefront roof the docking kernel
    reaches over the timed launches: ncu wavefronts per algorithmic byte x
    the algorithmic bytes timed / (kernel time x SMs x median SM clock x 1
    wavefront per SM per cycle)."""
    if shape not in DOCK_L1_WAVEFRONTS_PER_ABYTE:
        return None
    import torch
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = clk.get("sm_mhz") or 1965.0
    wf = DOCK_L1_WAVEFRONTS_PER_ABYTE[shape] * abytes
    return {"wavefronts_per_algorithmic_byte": DOCK_L1_WAVEFRONTS_PER_ABYTE[shape],
            "wavefronts_per_s": wf / (ms / 1e3), "peak_per_s": sms * mhz * 1e6,
            "frac": wf / (ms / 1e3) / (sms * mhz * 1e6)}


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(xyz, xs, ligs, chains_per_lig, n_sample, orc=None, warm=None):
    """Oracle port (double precision restatement of the reference's search,
    clustering and refinement) timed on the host cores on a bounded sample
    of the same workload: n_sample whole ligands (all chains, top-20
    refinement).  orc: an oracle with this receptor, box and maps already
    set up (its grid build is then not timed again); warm: a ligand docked
    untimed first (thread start-up, first-touch page faults)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle_lib
    from vdock import synth
    threads = os.cpu_count() or 1
    t_grid = None
    if orc is None:
        orc = oracle_lib.Oracle()
        orc.set_receptor(xyz, xs)
        orc.set_box([0, 0, 0], [BOX] * 3)
        t_grid = orc.grid_seconds(synth.TYPES8, threads)
    if warm is not None:
        lw = orc.add_ligand(warm)
        dw = max(1, int((0.24 * warm["n_atoms"] + 0.29 * orc.ntors[lw] - 3.41) * 2))
        orc.mc_chains(lw, SEED, lw, dw, (30 + warm["n_atoms"]) // 3, 0, chains_per_lig, threads=threads)
    total_t, total_evals, desc = 0.0, 0, []
    for lig in ligs[:n_sample]:
        lo = orc.add_ligand(lig)
        n_all, nt = lig["n_atoms"], orc.ntors[lo]
        depth = max(1, int((0.24 * n_all + 0.29 * nt - 3.41) * 2))
        steps = (30 + n_all) // 3
        t0 = time.perf_counter()
        conf, e, evals = orc.mc_chains(lo, SEED, lo, depth, steps, 0, chains_per_lig, threads=threads)
        kept = orc.cluster(lo, conf, e, 1.0, 20)
        for i in kept:
            _, _, ev = orc.refine(lo, conf[i], steps)
            evals += ev
        total_t += time.perf_counter() - t0
        total_evals += evals
        desc.append(f"{n_all}/{nt}")
    return {"value": len(desc) / total_t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(desc)} whole ligands (atoms/torsions {', '.join(desc)}), {chains_per_lig} chains "
                      f"each, heuristic depth, top-20 refinement; {total_evals} BFGS evals in {total_t:.1f} s",
            "grid_build_s": t_grid, "bfgs_evals_per_s": total_evals / total_t}


def secondary_configs(hbm, cpu, which=("plain", "adjoint", "uneven")):
    """The reference's other named workloads, measured once each on one GPU
    (synthetic inputs of the named shapes; seeded):
      plain_single_ligand : 24-atom / 5-torsion ligand, 2,000-atom receptor,
                            20 A box, 1,024 chains x 1,000 MC steps, one
                            vd_dock_plain call (timed after the autotuner's
                            three exploring calls);
      adjoint_poses       : 65,536 random poses of a 40-atom / 10-torsion
                            ligand, energy + gradient (vd_energy_grad_device)
                            and energy only, inputs resident on the device;
      batched_uneven      : 512 ligands of 10-60 atoms / 0-15 torsions, 4,000-
                            atom receptor, 30 A box, 8,192 chains (16 per
                            ligand) x 2,000 MC steps in one batched call.
    Each carries the oracle port timed on a bounded sample on the host cores."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    threads = os.cpu_count() or 1
    out = {}
    if "plain" in which:
        out["plain_single_ligand"] = _plain_line(hbm, cpu, threads)
    if "adjoint" in which:
        out["adjoint_poses"] = _adjoint_line(hbm, cpu)
    if "uneven" in which:
        out["batched_uneven"] = _uneven_line(cpu, threads)
    return out


def _plain_line(hbm, cpu, threads):
    import torch
    import vdock
    from vdock import synth
    import oracle_lib

    def lig_cost_bytes(lig):
        return 32 * int((lig["xs"] >= 0).sum()) + 16 * len(lig["pairs"])
    cfg = synth.CONFIGS["plain"]
    xyz, xs = synth.receptor(cfg["rec_atoms"], cfg["rec_radius"], SEED + 1)
    lig = synth.ligand(cfg["lig_atoms"], cfg["lig_tors"], SEED + 2)
    ctx = vdock.Context()
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0, 0, 0], [cfg["box"]] * 3)
    ctx.build_grids(sorted(set(int(t) for t in lig["xs"] if t >= 0)))
    lid = ctx.add_ligand(lig)
    sp = vdock.search_params(seed=SEED, n_chains=cfg["chains"], search_depth=cfg["steps"], refine=1)
    for _ in range(DOCK_SHAPES + 1):  # the autotuner runs each shape once, then keeps the fastest
        ctx.dock_plain(lid, sp)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = ctx.dock_plain(lid, sp)
    wall = time.perf_counter() - t0
    st = ctx.stats()
    line = {"s_per_ligand": wall, "dock_ms": st["dock_ms"], "post_ms": st["post_ms"],
            "bfgs_evals": int(r["bfgs_evals"]), "bfgs_evals_per_s": r["bfgs_evals"] / (st["dock_ms"] / 1e3),
            "best_energy": float(r["energy"][0]), "launch_shape": st["dock_shape"]}
    line["frac_of_hbm"] = line["bfgs_evals_per_s"] * lig_cost_bytes(lig) / 1e9 / hbm
    ctx.close()
    if cpu:
        orc = oracle_lib.Oracle()
        orc.set_receptor(xyz, xs)
        orc.set_box([0, 0, 0], [cfg["box"]] * 3)
        orc.build_grids(sorted(set(int(t) for t in lig["xs"] if t >= 0)))
        lo = orc.add_ligand(lig)
        n_s = 128
        t0 = time.perf_counter()
        _, _, ev = orc.mc_chains(lo, SEED, lid, cfg["steps"], (30 + lig["n_atoms"]) // 3, 0, n_s, threads=threads)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"s_per_ligand": dt * cfg["chains"] / n_s, "bfgs_evals_per_s": ev / dt,
                                "cores": threads, "kind": "port",
                                "sample": f"{n_s} of {cfg['chains']} chains x {cfg['steps']} steps, "
                                          f"extrapolated to all chains (MC search only)"}
    return line


def _adjoint_line(hbm, cpu):
    import numpy as np
    import torch
    import vdock
    from vdock import synth
    import oracle_lib

    def lig_cost_bytes(lig):
        return 32 * int((lig["xs"] >= 0).sum()) + 16 * len(lig["pairs"])
    cfg = synth.CONFIGS["adjoint"]
    xyz, xs = synth.receptor(cfg["rec_atoms"], cfg["rec_radius"], SEED + 1)
    lig = synth.ligand(cfg["lig_atoms"], cfg["lig_tors"], SEED + 3)
    ctx = vdock.Context()
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0, 0, 0], [cfg["box"]] * 3)
    ctx.build_grids(sorted(set(int(t) for t in lig["xs"] if t >= 0)))
    lid = ctx.add_ligand(lig)
    n = cfg["poses"]
    half = cfg["pos_box"] / 2
    poses = synth.random_poses(n, ctx.ntors[lid], -half, half, SEED + 4)
    dp = torch.from_numpy(poses).cuda()
    de = torch.empty(n, device="cuda")
    dg = torch.empty(n, 6 + ctx.ntors[lid], device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    line = {"poses": n, "pairs": len(lig["pairs"]), "heavy_atoms": int((lig["xs"] >= 0).sum())}
    for name, call in (("energy_grad", lambda: ctx.energy_grad_device(lid, n, dp.data_ptr(), de.data_ptr(),
                                                                      dg.data_ptr(), stream)),
                       ("energy", lambda: ctx.energy_device(lid, n, dp.data_ptr(), de.data_ptr(), stream))):
        for _ in range(3):
            call()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            call()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 10
        line[name] = {"ms": ms, "evals_per_s": n / (ms / 1e3),
                      "gbs": n * lig_cost_bytes(lig) / (ms / 1e3) / 1e9,
                      "frac_of_hbm": n * lig_cost_bytes(lig) / (ms / 1e3) / 1e9 / hbm}
    ctx.close()
    if cpu:
        orc = oracle_lib.Oracle()
        orc.set_receptor(xyz, xs)
        orc.set_box([0, 0, 0], [cfg["box"]] * 3)
        orc.build_grids(sorted(set(int(t) for t in lig["xs"] if t >= 0)))
        lo = orc.add_ligand(lig)
        n_s = 4096
        t0 = time.perf_counter()
        for p in poses[:n_s].astype(np.float64):
            orc.eval_deriv(lo, p)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"evals_per_s": n_s / dt, "cores": 1, "kind": "port",
                                "sample": f"{n_s} of {n} poses, energy + gradient, one thread"}
    return line


def _uneven_line(cpu, threads):
    import torch
    import vdock
    from vdock import synth
    import oracle_lib
    cfg = synth.CONFIGS["batched"]
    xyz, xs = synth.receptor(cfg["rec_atoms"], cfg["rec_radius"], SEED + 5)
    ligs = synth.ligand_set(cfg["ligands"], cfg["atoms"], cfg["tors"], SEED + 6)
    ctx = vdock.Context()
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0, 0, 0], [cfg["box"]] * 3)
    ctx.build_grids(synth.TYPES8)
    ids = [ctx.add_ligand(l) for l in ligs]
    per = cfg["total_chains"] // cfg["ligands"]
    sp = vdock.search_params(seed=SEED, n_chains=per, search_depth=cfg["steps"], refine=1)
    for _ in range(DOCK_SHAPES):  # untimed: the autotuner runs each of its shapes once
        ctx.dock_batched(ids, sp)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = ctx.dock_batched(ids, sp)
    wall = time.perf_counter() - t0
    st = ctx.stats()
    evals = sum(int(r["bfgs_evals"]) for r in res)
    line = {"s": wall, "ligands_per_s": len(ids) / wall, "dock_ms": st["dock_ms"], "post_ms": st["post_ms"],
            "bfgs_evals": evals, "bfgs_evals_per_s": evals / (st["dock_ms"] / 1e3), "chains_per_ligand": per,
            "launch_shape": st["dock_shape"], "graph_launches": st["graph_launches"],
            "untimed_warmup_calls": DOCK_SHAPES}
    ctx.close()
    if cpu:
        orc = oracle_lib.Oracle()
        orc.set_receptor(xyz, xs)
        orc.set_box([0, 0, 0], [cfg["box"]] * 3)
        orc.build_grids(synth.TYPES8)
        t0, cev = time.perf_counter(), 0
        n_s = 2
        for i in range(n_s):
            lo = orc.add_ligand(ligs[i])
            _, _, ev = orc.mc_chains(lo, SEED, ids[i], cfg["steps"], (30 + ligs[i]["n_atoms"]) // 3, 0, per,
                                     threads=threads)
            cev += ev
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"bfgs_evals_per_s": cev / dt, "cores": threads, "kind": "port",
                                "sample": f"{n_s} of {len(ids)} ligands, {per} chains x {cfg['steps']} steps "
                                          f"(MC search only)"}
    return line


def run_reference(a):
    """The reference arm: the oracle port of the reference's CPU path on all
    host cores, W untimed and K timed steps, each step a bounded sample of
    the workload: the first a.cpu_ligands whole ligands of the batch the GPU
    arm docks in that step (same ligand set and order as run_ours)."""
    world, rank, _ = dist()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle_lib
    from vdock import synth
    n, B = a.cpu_ligands, a.batch
    xyz, xs, ligs = make_inputs(0, (a.warmup + a.steps) * B)
    orc = oracle_lib.Oracle()
    orc.set_receptor(xyz, xs)
    orc.set_box([0, 0, 0], [BOX] * 3)
    t_grid = orc.grid_seconds(synth.TYPES8, os.cpu_count() or 1)
    t_wall = time.perf_counter()
    for w in range(a.warmup):
        cpu_baseline(xyz, xs, ligs[w * B:w * B + n], a.chains, n, orc)
    total_t, evals, descs = 0.0, 0, []
    for k in range(a.steps):
        chunk = ligs[(a.warmup + k) * B:(a.warmup + k) * B + n]
        cb = cpu_baseline(xyz, xs, chunk, a.chains, n, orc)
        total_t += n / cb["value"]
        evals += cb["bfgs_evals_per_s"] * n / cb["value"]
        descs.append(cb["sample"].split(" (")[1].split(")")[0])
    value = a.steps * n / total_t
    wall = time.perf_counter() - t_wall
    sample = (f"{a.steps} steps x {n} whole ligands ({'; '.join(descs)}), {a.chains} chains each, heuristic "
              f"depth, top-20 refinement; {evals:.0f} BFGS evals in {total_t:.1f} s (after {a.warmup} warm-up steps)")
    threads = os.cpu_count() or 1
    # ms_per_step: the measured time of one step's sample (a.cpu_ligands whole
    # ligands), not an extrapolation to the GPU arm's batch
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * total_t / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "wide-box screen", "ligands_per_step": a.batch,
                       "ligands_timed_per_step": n, "chains_per_ligand": a.chains,
                       "search_depth": "heuristic (main.cpp:369)", "box_A": BOX, "receptor_atoms": REC_ATOMS,
                       "ligand_atoms": list(LIG_ATOMS), "ligand_torsions": list(LIG_TORS),
                       "parallelism": "host threads (oracle port)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "grid_build_s": t_grid,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


def run_ours(a):
    import numpy as np
    import torch
    import vdock
    from vdock import synth
    world, rank, local = dist()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = td
    B, W, K = a.batch, a.warmup, a.steps
    n_ligs = (W + K) * B
    xyz, xs, ligs = make_inputs(rank, n_ligs)
    ctx = vdock.Context(local)
    ctx.set_receptor(xyz, xs)
    ctx.set_box([0, 0, 0], [BOX] * 3)
    grid_ms = []
    for _ in range(3):
        ctx.build_grids(synth.TYPES8)
        grid_ms.append(ctx.stats()["grid_ms"])
    cells_ms = ctx.stats()["cells_ms"]
    n_pts = int(np.prod(ctx.grid_dims()[0]))
    grid_bytes = 4 * n_pts * 8 + 16 * REC_ATOMS
    ids = [ctx.add_ligand(l) for l in ligs]
    sp = vdock.search_params(seed=SEED, n_chains=a.chains, search_depth=0, refine=1, launch_shape=a.launch_shape)
    batches = [ids[i * B:(i + 1) * B] for i in range(W + K)]
    # untimed: W warm-up steps, repeated until the autotuner has run each of
    # its launch shapes once on this workload (it then keeps the fastest)
    n_warm = W if a.launch_shape else max(W, DOCK_SHAPES)
    for k in range(n_warm):
        ctx.dock_batched(batches[k % W], sp)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = Clocks(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    dock_ms, post_ms, evals, abytes, aflops, launches = 0.0, 0.0, 0, 0, 0, 0
    t_wall = time.perf_counter()
    step_wall = []
    for k in range(W, W + K):
        t_step = time.perf_counter()
        res = ctx.dock_batched(batches[k], sp)
        step_wall.append(time.perf_counter() - t_step)  # the call returns after its GPU work
        st = ctx.stats()
        shapes = {"dock_launch_shape": st["dock_shape"], "grid_shape": st["grid_shape"]}
        dock_ms += st["dock_ms"]
        post_ms += st["post_ms"]
        for lid, r in zip(batches[k], res):
            evals += r["bfgs_evals"]
            abytes += r["bfgs_evals"] * lig_bytes(ligs[lid])
            aflops += r["bfgs_evals"] * lig_flops(ligs[lid])
        launches += 5  # dock, cluster, gather, refine, score
    ev1.record()
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall
    clk = clocks.stop()
    elapsed = ev0.elapsed_time(ev1) / 1e3
    if pg:
        from vdock import multi
        elapsed = multi.max_over_ranks(elapsed, device="cuda")
        pg.barrier()
    value = K * B * world / elapsed
    # plain form, like for like: one ligand per launch (vd_dock_plain) over the
    # same ligands, seed and chains as the first timed batch; per ligand the
    # docking kernel's time, the post-processing kernels' time and the rest
    # (host work, uploads, launch and synchronisation gaps), beside the same
    # split of the batched steps
    for i in range(DOCK_SHAPES):  # warm-up: the autotuner tries each launch shape
        ctx.dock_plain(batches[0][i % len(batches[0])], sp)
    torch.cuda.synchronize()
    p_dock = p_post = 0.0
    p_evals, p_shapes, p_blocks = 0, set(), 0
    t0 = time.perf_counter()
    for lid in batches[W]:
        r = ctx.dock_plain(lid, sp)
        st = ctx.stats()
        p_dock += st["dock_ms"]
        p_post += st["post_ms"]
        p_evals += r["bfgs_evals"]
        p_shapes.add(st["dock_shape"])
        p_blocks = st["dock_blocks"]
    torch.cuda.synchronize()
    p_wall = time.perf_counter() - t0
    plain_value = B / p_wall
    blocks_per_sm = {1: 8, 2: 10, 3: 12, 4: 6, 5: 4}  # four-chain blocks per SM of each register budget
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    plain_split = {
        "ligands": B, "same_ligands_as": "timed step 1", "wall_ms_per_ligand": 1e3 * p_wall / B,
        "dock_kernel_ms_per_ligand": p_dock / B, "post_kernels_ms_per_ligand": p_post / B,
        "host_and_gaps_ms_per_ligand": 1e3 * p_wall / B - (p_dock + p_post) / B,
        "dock_kernel_evals_per_s": p_evals / (p_dock / 1e3), "launch_shapes": sorted(p_shapes),
        "dock_waves": [p_blocks / (n_sm * blocks_per_sm[s]) for s in sorted(p_shapes)]}
    batched_split = {
        "wall_ms_per_ligand": 1e3 * elapsed / (K * B), "dock_kernel_ms_per_ligand": dock_ms / (K * B),
        "post_kernels_ms_per_ligand": post_ms / (K * B),
        "host_and_gaps_ms_per_ligand": 1e3 * elapsed / (K * B) - (dock_ms + post_ms) / (K * B),
        "dock_kernel_evals_per_s": evals / (dock_ms / 1e3)}
    # end to end through the public API with host buffers: ligand topologies
    # copied in (vd_add_ligands, which packs the batch on host threads, + pool
    # upload), results read back
    e2e_times, h2d_steps = [], []
    n_e2e = K if a.e2e_steps <= 0 else min(a.e2e_steps, K)
    for k in range(n_e2e):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.clear_ligands()
        eids = ctx.add_ligands([ligs[lid] for lid in batches[W + k]])
        res = ctx.dock_batched(eids, sp)
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
        h2d_steps.append(ctx.stats()["ligand_bytes"])  # the batch's ligand blobs, uploaded by the call
    h2d = int(sum(h2d_steps) / max(1, len(h2d_steps)))
    import ctypes
    d2h = B * ctypes.sizeof(vdock.DockResult)  # one vd_dock_result per ligand
    e2e_total = sum(e2e_times)
    if pg:
        e2e_total = multi.max_over_ranks(e2e_total, device="cuda")
    e2e_value = B * n_e2e * world / e2e_total if e2e_times else None
    if rank != 0:
        return
    hbm, src = peaks()
    achieved = abytes / (dock_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": 1e3 * elapsed / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic",
        "config": {"workload": "wide-box screen", "ligands_per_step": B, "chains_per_ligand": a.chains,
                   "search_depth": "heuristic (main.cpp:369)", "box_A": BOX, "receptor_atoms": REC_ATOMS,
                   "ligand_atoms": list(LIG_ATOMS), "ligand_torsions": list(LIG_TORS),
                   "parallelism": f"weak x{world} (ligand shards)",
                   "l2": "inputs larger than L2 (8 maps x 188^3 x 4 B = 213 MB)",
                   "untimed_warmup_calls": n_warm, **shapes},
        "bfgs_evals_per_s": evals * world / elapsed,
        "bfgs_evals_per_step": evals / K,
        "plain": {"value": plain_value * world, "unit": UNIT, "batched_over_plain": value / (plain_value * world),
                  "batched_over_plain_same_ligands": (B / step_wall[0]) / plain_value,
                  "batched_same_ligands_value": B / step_wall[0], **plain_split},
        "batched_split": batched_split,
        "grid_build": {"ms": min(grid_ms), "points": n_pts, "types": 8,
                       "gbs": grid_bytes / (min(grid_ms) / 1e3) / 1e9,
                       "frac_of_hbm": grid_bytes / (min(grid_ms) / 1e3) / 1e9 / hbm,
                       "corner_cells_ms": cells_ms,
                       **grid_l1_roof(min(grid_ms), clk, local)},
        "roofline": {"kernel": "dock_kernel", "bound": "hbm", "achieved": achieved, "peak": hbm,
                     "peak_source": src, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": (DOCK_DRAM_PER_ABYTE[shapes["dock_launch_shape"]] * abytes / K
                                 if shapes["dock_launch_shape"] in DOCK_DRAM_PER_ABYTE else None),
                     "l1_wavefront_roof": dock_l1_roof(shapes["dock_launch_shape"], abytes, dock_ms, clk, local),
                     "fp32_roof": fp32_roof(aflops, dock_ms, clk, local),
                     "note": "algorithmic bytes = evals x (32 x heavy atoms + 16 x intra pairs); traffic = "
                             "ncu DRAM bytes per algorithmic byte x algorithmic bytes per launch; the kernel's "
                             "limit is the L1 data pipe (l1_wavefront_roof), HBM is a reference point"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk,
        "wall_s": t_wall,
    }
    if world == 1 and not a.no_cpu_baseline:
        # the first ligand of every timed batch (each also in the reference
        # arm's sample, which docks the first cpu_ligands of every batch), after
        # one untimed warm-up ligand: a sample spread over the timed region
        sample = [ligs[k * B] for k in range(W, W + K)]
        cb = cpu_baseline(xyz, xs, sample, a.chains, len(sample), warm=ligs[0])
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        line["grid_build"]["cpu_s"] = cb["grid_build_s"]
    ctx.close()
    if world == 1 and not a.no_configs:
        line["configs"] = secondary_configs(hbm, not a.no_cpu_baseline, a.configs.split(","))
    print(json.dumps(line), flush=True)


def main():
    a = args_()
    if a.only_configs:
        import torch
        torch.cuda.set_device(0)
        hbm, _ = peaks()
        print(json.dumps({"configs": secondary_configs(hbm, not a.no_cpu_baseline, a.configs.split(","))}), flush=True)
        return
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as td
        if td.is_initialized():
            td.destroy_process_group()


if __name__ == "__main__":
    main()
