#!/usr/bin/env python
"""Grains3D DEM time step on B200: particle-steps/s for 1,000,000 polydisperse
spheres in a triply periodic box (granular-gas cooling), FP32-split vs FP64.

One step = one kick-drift-kick leapfrog step of the whole system: the force
evaluation (narrow phase over the skin pair list, Hooke / HookeMemory contact
force with hashed tangential history, per-particle force/torque reduction)
fused with the closing kick, the next opening kick and the drift; the pair
list (counting sort on the cell key + 27-cell search) is rebuilt when a
particle has moved half the skin.  Inputs: the seeded FCC stand-in of the
1M-sphere configuration (pacific_b200.scenarios.periodic_gas), synthetic.

Other legs on the same line: per-particle and per-contact force error against
the CPU FP64 oracle, the batched sweep against sequential runs, the convex
(cube + tetrahedron) pour, the end-to-end run through the public API with host
buffers, and the CPU baseline (the Grains3D reference sources compiled here,
single thread, on a bounded sample).

Multi-GPU: the workload does not shard without a halo exchange, so each rank
runs an independent replica (weak scaling, no data-path collective); the
timed region is bracketed by barriers and the max over ranks is reported.

`--impl reference` times the Grains3D reference's own CPU step (compiled from
its sources by oracle/build_ref.sh; the CPU FP64 restatement when that build
is absent) on the host, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s, 1M spheres: FP32-split vs FP64 on one B200, at stated error"
UNIT = "particle-steps/s"


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = None

    def __enter__(self):
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        time.sleep(0.2)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.flush()
        rows = []
        for line in Path(self.out.name).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), float(f[3]), f[5:9]))
            except ValueError:
                continue
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        # samples under load: power well above idle
        pmax = max(r[2] for r in rows)
        load = [r for r in rows if r[2] > 0.5 * pmax] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in load for k in range(4) if r[3][k] == "Active"})
        return {"sm_mhz": float(np.median([r[0] for r in load])), "sm_max_mhz": rows[0][1],
                "reasons": reasons, "samples": len(load)}


# --------------------------------------------------------------- roofline --
def algorithmic_bytes(kernel, n, entries, contacts, ncells, fp64):
    """Compulsory DRAM bytes of one launch of each phase of a spheres-only
    step: each input read once, each output written once, neighbour re-reads
    counted as cache hits.  Per particle unless noted.  The particle state is
    x, v, w, w_bf, q in FP64; FP32-split spheres keep no w_bf (w is their
    angular state).  entries: pair-list entries (each pair twice); contacts:
    pairs in contact (the pairs the contact filter keeps are these, up to the
    FP32 margin of the test)."""
    vel = 24
    state = 24 + (3 if fp64 else 2) * vel + 32
    pairs = entries // 2
    touched = min(n, 2 * contacts)    # particles with a contact
    share = 64 if fp64 else 32        # one side of a contact, per row entry
    hist = 8 + (72 if fp64 else 36)   # history key + values
    if kernel == "filter":
        # per particle its FP32 position; per pair its compact-list word
        # pair; per kept pair its index in the kept list and the two
        # candidate marks
        return n * 16 + pairs * 8 + contacts * (4 + 8)
    if kernel in ("pairlaw64", "pairlaw32"):
        # per kept pair: its index, compact-list words and row positions;
        # both partners' id type wrap x v w and row offsets; the history
        # read and written; the two shares and the two flags
        return contacts * (4 + 8 + 4 + 2 * (4 + 4 + 4 + 24 + 2 * vel + 4) + 2 * hist
                           + 2 * share + 2 * 4)
    if kernel == "move":
        # state type inst posf0 wrap flags | state wrap posf flags, and
        # for a particle in contact its row offset and length, the first
        # word of each share of its row and the rest of each share in use
        rowlen = entries / max(n, 1)
        return int(n * (state + 8 + 16 + 4 + 4 + state + 4 + 16 + 4)
                   + touched * (8 + rowlen * 16) + 2 * contacts * (share - 16))
    if kernel == "bin":          # x inst | skey rank; cell-count RMW
        return n * (24 + 4 + 8 + 8)
    if kernel == "scan":         # counts | starts (per cell)
        return ncells * 8
    if kernel == "place":        # skey rank start[skey] | order
        return n * 16
    if kernel == "cellsort":     # starts, count reset (per cell); order, id of shared cells
        return ncells * 8 + n * 8
    if kernel == "permute":      # order skey ids state F T | ids state F T cellc + pos / offset
        return n * (4 + 4 + 12 + 2 * (state + 48) + 16 + (32 if fp64 else 16))
    if kernel == "copyback":     # ids state F T | ids state F T wrap posf posf0
        return n * (12 + 2 * (state + 48) + 12 + 4 + 32)
    if kernel in ("pairs_count64", "pairs_count32"):   # cellc + own position | row length
        return n * (16 + (32 if fp64 else 16) + 4) + 4 * ncells
    if kernel == "row_scan":     # row lengths | row offsets
        return n * 8
    if kernel in ("pairs_fill64", "pairs_fill32"):
        # cellc + own position + row offset and length | rows, compact list
        return n * (16 + (32 if fp64 else 16) + 8) + 4 * ncells + 4 * entries + 12 * pairs
    if kernel == "link":         # compact list, partner's row | row positions
        return pairs * (8 + 4 + 4 + 4)
    return None


def read_ncu_traffic(kernel):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    for p in (ROOT / "profiles").glob("*.md"):
        for line in p.read_text().splitlines():
            if line.startswith(f"traffic_bytes_per_launch[{kernel}]:"):
                try:
                    return float(line.split(":", 1)[1])
                except ValueError:
                    return None
    return None


# ------------------------------------------------------------------ helpers --
def dist_setup(world):
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return dist


def barrier_sync(dist):
    import torch
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(dist, value):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_system(xml, sc, precision, graphs=True, skin_factor=None):
    from pacific_b200 import Grains
    g = Grains(xml, precision)
    g.use_graphs(graphs)
    g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
    if skin_factor is not None:
        g.set_tuning(skin_factor=skin_factor)
    g.do_before_time_stepping()
    return g


def timed_steps(g, dist, steps):
    barrier_sync(dist)
    g.step(steps)
    barrier_sync(dist)
    return max_over_ranks(dist, g.last_step_ms)


def pinned(a):
    import torch
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    t.numpy()[...] = a
    return t


def e2e_run(g, dist, steps, every):
    """Public-API run with host buffers, as a Grains3D run between two
    outputs: the state goes up from pinned host memory (gdem_set_state), the
    leapfrog runs `every` steps per call of Grains.Simulation (which reads
    back the status word, the reference's exceptions), each output time
    reads back max/mean |v| (what Grains::Simulation writes to
    *_VelocityMaxMean.dat at its output times, Grains.cpp:390-408), and the
    final state comes back down into pinned memory."""
    s = g.download_state()
    host = {k: pinned(s[k]) for k in ("x", "v", "w", "q", "F", "T")}
    outs = {k: pinned(np.zeros_like(s[k])) for k in ("x", "v", "w", "q", "F", "T")}
    barrier_sync(dist)
    t0 = time.perf_counter()
    g.set_state(host["x"].numpy(), host["v"].numpy(), host["w"].numpy(), host["q"].numpy(),
                host["F"].numpy(), host["T"].numpy())
    done = 0
    outputs = 0
    while done < steps:
        k = min(every, steps - done)
        g.Simulation(k)
        g.velocity_stats()
        done += k
        outputs += 1
    from pacific_b200.grains import _dp, library
    lib = library()
    rc = lib.gdem_download_state(g._h, _dp(outs["x"].numpy()), _dp(outs["v"].numpy()),
                                 _dp(outs["w"].numpy()), None, _dp(outs["q"].numpy()),
                                 _dp(outs["F"].numpy()), _dp(outs["T"].numpy()))
    assert rc == 0
    barrier_sync(dist)
    dt = max_over_ranks(dist, time.perf_counter() - t0)
    n = g.n
    up = n * 8 * (3 + 3 + 3 + 4 + 3 + 3)
    down = up
    # per output: the status word (4 B) and max/mean |v| (16 B)
    return dt, up / steps, (down + outputs * 20) / steps, outputs


def error_sample(n_fcc, steps_before, precision):
    """Per-particle force error of one GPU step against the FP64 oracle from
    the same state (normaliser: the particle's sum of contact-force magnitudes)."""
    from pacific_b200 import scenarios
    from tests.helpers import (contact_forces, contact_scale, force_errors, gpu_from_oracle,
                               oracle_for, per_contact_errors, radii_of)
    sc = scenarios.periodic_gas(n_fcc=n_fcc, seed=1236)
    with tempfile.TemporaryDirectory() as d:
        xml = str(sc.write_xml(Path(d) / "err.xml"))
        o = oracle_for(sc, xml)
        o.init()
        o.step(steps_before)
        g = gpu_from_oracle(xml, sc, o, precision)
        g.set_diagnostics(True)
        o.step(1)
        g.step(1)
        id0, id1, dl, pt, f = o.contacts()
        scale = contact_scale(sc.n, id0, id1, f)
        fe, te = force_errors(o.state(), g.download_state(), scale, radii_of(sc))
        g0, g1, _, gf = g.download_contacts(forces=True)
        pe = per_contact_errors(contact_forces(id0, id1, f), contact_forces(g0, g1, gf))
        nlaw, nre = g.law_counts()
        m = scale > 0
        g.close()
    out = {"force_max": float(fe[m].max()), "force_p99": float(np.percentile(fe[m], 99)),
           "torque_max": float(te[m].max()), "per_contact_max": float(pe.max(initial=0.0)),
           "particles_in_contact": int(m.sum()), "contacts": int(len(id0))}
    from pacific_b200 import FP32_SPLIT
    if precision == FP32_SPLIT:
        out["fp64_reevaluated"] = int(nre)
        out["law_evaluations"] = int(nlaw)
    return out


def error_full(sc, xml, advance, tmpdir):
    """Parity of one step at the full size against the Grains3D reference
    itself: the GPU FP64 system advanced `advance` steps (a state with
    contacts) writes its Format2024 particle file; the reference (oracle/_ref,
    own process, its reload path) and the GPU in both precisions each read
    that file and take one step.  Cells and contact sets are compared
    exactly, forces per particle (normaliser: the particle's sum of
    contact-force magnitudes)."""
    from pacific_b200 import FP32_SPLIT, FP64
    from tests.helpers import radii_of, step_parity
    g = make_system(xml, sc, FP64)
    g.step(advance)
    pfile = Path(tmpdir) / "state_Particles"
    t0 = time.perf_counter()
    g.write_reload_particles(pfile)
    t_write = time.perf_counter() - t0
    g.close()
    period = np.subtract(sc.maxc, sc.origin) * np.asarray(sc.periodic, float)
    r = step_parity(xml, pfile, sc.n, radii_of(sc), (FP64, FP32_SPLIT), period=period)
    out = {"sample": f"periodic_gas n={sc.n}, one step from the FP64 GPU state after "
                     f"{advance} steps (written as a Format2024 particle file), vs the Grains3D "
                     "reference itself (oracle/_ref) reading the same file",
           "n": sc.n, "reference": r["reference"], "write_s": t_write,
           "fp64": r[FP64], "fp32_split": r[FP32_SPLIT],
           "tolerance": {"fp64": 1e-10, "fp32_split": 1e-5}}
    return out


def _quiet(f, *a):
    """Runs f with the process's stdout silenced (the reference prints its
    construction log)."""
    sys.stdout.flush()
    fd = os.dup(1)
    nul = os.open(os.devnull, os.O_WRONLY)
    os.dup2(nul, 1)
    try:
        return f(*a)
    finally:
        os.dup2(fd, 1)
        os.close(fd)
        os.close(nul)


def cpu_system(sc, xml):
    """The Grains3D reference itself (oracle/_ref, compiled from the reference
    sources) when it was built, else the CPU FP64 restatement.  Returns
    (kind, step function, label)."""
    from oracle import reference
    if reference.available():
        r = _quiet(reference.Reference, xml)
        assert _quiet(r.set_particles, sc.type, sc.x, sc.v, sc.w, sc.q) == 0
        assert _quiet(r.init) == 0
        return "reference", (lambda k: _quiet(r.step, k)), \
            "Grains3D reference sources (serial Type=Standard step), g++ -O3"
    from tests.helpers import oracle_for
    o = oracle_for(sc, xml)
    o.init()
    return "port", o.step, "CPU FP64 restatement oracle/grains_oracle.cpp"


def cpu_baseline(sc, xml, budget_s=15.0):
    """Times the reference CPU path on a bounded sample of the same workload
    (single thread: the reference step has no threading inside an MPI rank)."""
    kind, step, label = cpu_system(sc, xml)
    t0 = time.perf_counter()
    step(1)
    one = time.perf_counter() - t0
    k = max(1, min(50, int(budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    step(k)
    dt = time.perf_counter() - t0
    return {"value": sc.n * k / dt, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{k} steps of the full {sc.n}-sphere system after 1 warm-up step ({label}, "
                      "FP64, 1 thread)"}


def batched_measure(n_inst, steps, warmup=3):
    """The batched sweep: n_inst independent closed-box settling instances
    (500-20,000 spheres each, their own kn/en/muc) stepped together in one
    launch chain, with the launch settings the autotuner picks (and, beside
    it, with the default ones), against the same instances stepped one after
    another with the default settings (device time of each gdem_step,
    creation and tuning excluded on both sides)."""
    from pacific_b200 import FP32_SPLIT, Grains, scenarios
    inst = scenarios.batched_boxes(n_inst=n_inst)
    with tempfile.TemporaryDirectory() as d:
        xmls = [str(s.write_xml(Path(d) / f"i{k}.xml")) for k, s in enumerate(inst)]
        ins, typ, x, v, w, q = scenarios.concat_state(inst)
        times = {}
        for label in ("default", "autotuned"):
            g = Grains(xmls, FP32_SPLIT)
            g.upload_state(typ, x, v, w, q, inst=ins)
            if label == "autotuned":
                tuned = g.autotune(trial_steps=20)
            g.do_before_time_stepping()
            g.step(warmup)
            g.step(steps)
            times[label] = g.last_step_ms
            st = g.status()
            g.close()
        t_batch = times["autotuned"]
        t_seq = 0.0
        for k, s in enumerate(inst):
            gi = Grains(xmls[k], FP32_SPLIT)
            gi.upload_state(s.type, s.x, s.v, s.w, s.q)
            gi.do_before_time_stepping()
            gi.step(warmup)
            gi.step(steps)
            t_seq += gi.last_step_ms
            gi.close()
    ntot = int(len(ins))
    return {"instances": n_inst, "particles": ntot, "steps": steps,
            "batched_value": ntot * steps / (t_batch * 1e-3),
            "autotune": tuned,
            "batched_default_value": ntot * steps / (times["default"] * 1e-3),
            "sequential_value": ntot * steps / (t_seq * 1e-3),
            "speedup": t_seq / t_batch, "unit": UNIT, "precision": "fp32_split",
            "status": st, "workload": "batched_boxes (seeded), FP32-split, device time"}


def convex_measure(n, steps, warmup=3, graphs=True):
    """Cubes (2 mm) and regular tetrahedra (3 mm edge) poured into a
    0.1 x 0.1 x 0.3 m box (GJK narrow phase, 3D rotation).  Two starts: the
    pour as specified (at rest on the lattice: no contact for the first ~9,800
    steps) and the same lattice launched at up to 2 m/s per component so that
    the timed steps are collisional.  Device time per step in FP64 and
    FP32-split, with the FP64 re-evaluation count of FP32-split."""
    from pacific_b200 import FP32_SPLIT, FP64, Grains, scenarios
    out = {"workload": f"convex_pour n={n} (cubes + tetrahedra), dt=2e-6", "steps": steps}
    with tempfile.TemporaryDirectory() as d:
        poly = scenarios.write_tetrahedron(Path(d) / "tet.poly")
        for label, vmax in (("at_rest", 0.0), ("collisional", 2.0)):
            sc = scenarios.convex_pour(n=n, seed=1238, poly_path=poly, vmax=vmax)
            xml = str(sc.write_xml(Path(d) / f"convex_{label}.xml"))
            row = {}
            for name, prec in (("fp64", FP64), ("fp32_split", FP32_SPLIT)):
                g = Grains(xml, prec)
                g.use_graphs(graphs)
                g.upload_state(sc.type, sc.x, sc.v, sc.w, sc.q)
                g.do_before_time_stepping()
                g.step(warmup)
                g.law_counts(reset=True)
                g.gjk_counts(reset=True)
                g.step(steps)
                ms = g.last_step_ms
                entries, contacts = g.pair_counts()
                calls, iters, most = g.gjk_counts()
                r = {"value": n * steps / (ms * 1e-3), "ms_per_step": ms / steps,
                     "status": g.status(), "contacts_last_step": contacts,
                     "gjk": {"calls_per_step": calls / steps,
                             "mean_iterations": iters / calls if calls else 0.0,
                             "max_iterations": most}}
                if prec == FP32_SPLIT:
                    nlaw, nre = g.law_counts()
                    r["law_evaluations"] = nlaw
                    r["fp64_reevaluated"] = nre
                if vmax > 0:
                    # per-kernel device times over a few more steps (plain launches)
                    g.set_profiling(True)
                    g.step(10)
                    r["phases"] = {k: {"total_ms": round(v[0], 4), "launches": v[1]}
                                   for k, v in g.kernel_times().items()}
                    g.set_profiling(False)
                row[name] = r
                g.close()
            row["fp32_split_speedup"] = row["fp32_split"]["value"] / row["fp64"]["value"]
            out[label] = row
    out["unit"] = UNIT
    return out


def adjoint_measure(n, steps, every):
    """Calibration gradients (the adjoint): 4,096 spheres released in a
    0.02 x 0.02 x 0.08 m box, loss = squared error of positions and
    velocities after `steps` steps against the trajectory at kn = 2e4,
    en = 0.6, muc = 0.35, gradients at parameters perturbed by 5 %, with
    checkpoints every `every` steps; checked against dual-number forward
    mode and against central differences of the loss (relative steps 1e-5
    to 1e-9).  Wall-clock time of each call (device work dominates)."""
    from pacific_b200 import scenarios
    from pacific_b200.adjoint import Adjoint
    p_t = np.array([2.0e4, 0.6, 0.35])
    p_s = p_t * np.array([1.05, 0.95, 1.05])
    sc = scenarios.adjoint_box(n=n)
    with tempfile.TemporaryDirectory() as d:
        xml = sc.write_xml(Path(d) / "adj.xml")
        a = Adjoint(xml)
        a.set_particles(sc.type, sc.x, sc.v)
        t0 = time.perf_counter()
        tx, tv, _ = a.run(p_t, steps)
        t_fwd = time.perf_counter() - t0
        t0 = time.perf_counter()
        loss, gp, gv = a.gradients(p_s, tx, tv, steps, every)
        t_adj = time.perf_counter() - t0
        t0 = time.perf_counter()
        loss_f, gp_f = a.forward_mode(p_s, tx, tv, steps)
        t_dual = time.perf_counter() - t0
        # central differences of the loss (steps relative to each parameter)
        # over the full horizon and over shorter ones.  The loss is smooth
        # only between contact events: the normal damping force starts with a
        # jump when a contact opens, so the loss jumps where a perturbation
        # moves a contact's first step.  Over a short horizon no event lies
        # between p - h and p + h and the quotients agree with the adjoint;
        # over the full one such jumps lie inside every interval tried, and
        # the quotient (jump / 2h) grows as h shrinks.
        def differences(p, n_steps, x_t, v_t, g_adj, steps_rel):
            out = {}
            for h_rel in steps_rel:
                g_fd = np.zeros(3)
                for j in range(3):
                    dp = np.zeros(3)
                    dp[j] = h_rel * p[j]
                    lp = a.run(p + dp, n_steps, x_t, v_t)[2]
                    lm = a.run(p - dp, n_steps, x_t, v_t)[2]
                    g_fd[j] = (lp - lm) / (2 * dp[j])
                out[f"{h_rel:g}"] = {
                    "dL_dparams": g_fd.tolist(),
                    "rel_diff_vs_adjoint": (np.abs(g_adj - g_fd) /
                                            np.maximum(np.abs(g_adj), 1e-300)).tolist()}
            return out

        fd = {f"{steps}_steps": differences(p_s, steps, tx, tv, gp, (1e-5, 1e-6, 1e-7, 1e-8, 1e-9))}
        for short in sorted({max(1, min(steps, k)) for k in (20, 100)}):
            sx, sv, _ = a.run(p_t, short)
            _, gp_short, _ = a.gradients(p_s, sx, sv, short, every)
            fd[f"{short}_steps"] = {"dL_dparams_adjoint": gp_short.tolist(),
                                    **differences(p_s, short, sx, sv, gp_short, (1e-6, 1e-8))}
        a.close()
    rel = np.abs(gp - gp_f) / np.abs(gp_f)
    return {"workload": f"adjoint_box n={n}, {steps} steps, checkpoint every {every}",
            "loss": loss, "dL_dparams": gp.tolist(), "dL_dparams_forward_mode": gp_f.tolist(),
            "max_rel_diff_vs_forward_mode": float(rel.max()),
            "central_differences": fd,
            "dL_dv0_norm": float(np.linalg.norm(gv)),
            "forward_s": t_fwd, "gradient_s": t_adj, "forward_mode_s": t_dual}


# --------------------------------------------------------------- reference --
def run_reference(args, rank, world):
    if rank != 0:
        return
    from pacific_b200 import scenarios
    from oracle import oracle as orc
    orc.build()
    sc = scenarios.periodic_gas(n_fcc=args.n_fcc, seed=1236)
    with tempfile.TemporaryDirectory() as d:
        xml = str(sc.write_xml(Path(d) / "gas.xml"))
        kind, step, label = cpu_system(sc, xml)
        # each step is a bounded sample: the whole --steps/--warmup run stays
        # within a few minutes on one core
        t0 = time.perf_counter()
        step(1)
        one = time.perf_counter() - t0
        k = max(1, min(args.steps, int(60.0 / max(one, 1e-6))))
        w = min(args.warmup, 2)
        step(w)
        t0 = time.perf_counter()
        step(k)
        dt = time.perf_counter() - t0
    value = sc.n * k / dt
    sample = (f"{k} of the requested {args.steps} steps of the full {sc.n}-sphere system "
              f"after {1 + w} warm-up steps ({label}, FP64), 1 thread (the reference step "
              "is single-threaded per MPI rank)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": k, "warmup": 1 + w, "ms_per_step": 1e3 * dt / k,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "periodic_gas_1M", "n": sc.n, "steps_config": 2000,
                       "dt": sc.dt, "phi": scenarios.solid_fraction(sc),
                       "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (~0.5 GB of state per replica)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------- main --
def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-fcc", type=int, default=63)
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--output-every", type=int, default=50,
                    help="e2e: steps between two output times (status + max/mean |v| read back)")
    ap.add_argument("--advance", type=int, default=1000,
                    help="untimed steps before the warm-up, so that the timed window starts "
                         "from a state with contacts, in the middle of the configured run")
    ap.add_argument("--no-full-config", action="store_true",
                    help="skip the device-timed run of the whole configured run from its start")
    ap.add_argument("--profile-steps", type=int, default=50)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-error", action="store_true")
    ap.add_argument("--batched-instances", type=int, default=512)
    ap.add_argument("--batched-steps", type=int, default=50)
    ap.add_argument("--convex-n", type=int, default=200_000)
    ap.add_argument("--adjoint-n", type=int, default=4096)
    ap.add_argument("--adjoint-steps", type=int, default=500)
    ap.add_argument("--no-graphs", action="store_true",
                    help="plain kernel launches instead of graph replay (for per-kernel profilers)")
    ap.add_argument("--convex-steps", type=int, default=500)
    ap.add_argument("--only-fp32-split", action="store_true",
                    help="skip the FP64 leg (profiling the FP32-split step alone)")
    ap.add_argument("--skin-factor", type=float, default=None,
                    help="pair-list skin as a multiple of the largest circumscribed radius "
                         "(default: the library's)")
    ap.add_argument("--only-convex", action="store_true",
                    help="run the convex-pour leg alone and print its result (profiling)")
    ap.add_argument("--only-adjoint", action="store_true",
                    help="run the adjoint leg alone and print its result")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    dist = dist_setup(world)
    from pacific_b200 import FP32_SPLIT, FP64, build, scenarios
    if rank == 0:
        build.build()
    if dist is not None:
        dist.barrier()
    if args.only_convex:
        out = convex_measure(args.convex_n, args.convex_steps, graphs=not args.no_graphs)
        if rank == 0:
            print(json.dumps({"convex": out}), flush=True)
        return
    if args.only_adjoint:
        out = adjoint_measure(args.adjoint_n, args.adjoint_steps, 50)
        if rank == 0:
            print(json.dumps({"adjoint": out}), flush=True)
        return
    sc = scenarios.periodic_gas(n_fcc=args.n_fcc, seed=1236 + 1000 * rank)
    tmp = tempfile.TemporaryDirectory()
    xml = str(sc.write_xml(Path(tmp.name) / f"gas{rank}.xml"))
    n = sc.n

    res = {}
    legs = (("fp32_split", FP32_SPLIT),) if args.only_fp32_split else \
        (("fp64", FP64), ("fp32_split", FP32_SPLIT))
    for name, prec in legs:
        g = make_system(xml, sc, prec, graphs=not args.no_graphs, skin_factor=args.skin_factor)
        if args.advance > 0:
            g.step(args.advance)
        g.step(args.warmup)
        e0, r0 = g.step_counts()
        if name == "fp32_split":
            with ClockSampler(local) as clk:
                ms = timed_steps(g, dist, args.steps)
            clocks = clk.summary()
        else:
            ms = timed_steps(g, dist, args.steps)
        e1, r1 = g.step_counts()
        st = g.status()
        entries, contacts = g.pair_counts()
        # per-phase device times with CUDA events (plain launches)
        g.set_profiling(True)
        g.step(args.profile_steps)
        kt = g.kernel_times()
        g.set_profiling(False)
        res[name] = dict(ms=ms, status=st, entries=entries, contacts=contacts, kt=kt, g=g,
                         ncells=int(np.prod(g.grid()[0])), evals=(e0, e1), rebuilds=r1 - r0)
        if name == "fp64":
            g.close()

    g = res["fp32_split"]["g"]
    e2e_dt, h2d, d2h, e2e_outputs = e2e_run(g, dist, args.e2e_steps, args.output_every)
    g.close()

    # the whole configured run (2,000 steps from the start), device-timed
    full = None
    if not args.no_full_config:
        full = {}
        for name, prec in (("fp32_split", FP32_SPLIT), ("fp64", FP64)):
            gf = make_system(xml, sc, prec, graphs=not args.no_graphs, skin_factor=args.skin_factor)
            ms = timed_steps(gf, dist, 2000)
            _, rb = gf.step_counts()
            full[name] = {"value": world * n * 2000 / (ms * 1e-3), "ms_per_step": ms / 2000,
                          "rebuilds": rb, "status": gf.status()}
            gf.close()
        full["fp32_split_speedup"] = full["fp32_split"]["value"] / full["fp64"]["value"]
        full["steps"] = 2000

    if rank == 0:
        fp32 = res["fp32_split"]
        fp64 = res.get("fp64", fp32)
        value = world * n * args.steps / (fp32["ms"] * 1e-3)
        v64 = world * n * args.steps / (fp64["ms"] * 1e-3)
        # roofline of the dominant kernel of the FP32-split step
        kt = fp32["kt"]
        dom = max((k for k in kt if k not in ("decide", "hist_fill")), key=lambda k: kt[k][0])
        avg_ms = kt[dom][0] / kt[dom][1]
        ncells = fp32["ncells"]
        ab = algorithmic_bytes(dom, n, fp32["entries"], fp32["contacts"], ncells, False)
        peaks = {}
        pk = ROOT / "MEASURED_PEAKS.json"
        if pk.exists():
            peaks = json.loads(pk.read_text())
        hbm = peaks.get("hbm_gbs")
        peak_src = "measured" if hbm else "fallback"
        hbm = hbm or 6650.0
        achieved = ab / (avg_ms * 1e-3) / 1e9 if ab else None
        traffic = read_ncu_traffic(dom)
        def phase_table(kts, res_, fp64):
            out = {}
            for k, v in kts.items():
                avg = v[0] / v[1]
                row = {"total_ms": round(v[0], 4), "launches": v[1],
                       "avg_us": round(1e3 * avg, 2)}
                b = algorithmic_bytes(k, n, res_["entries"], res_["contacts"], ncells, fp64)
                if b:
                    row["algorithmic_GBs"] = round(b / (avg * 1e-3) / 1e9, 1)
                out[k] = row
            return out
        phases = phase_table(kt, fp32, False)
        # whole step: the step kernels once per step, the rebuild kernels as
        # often as the timed window rebuilt
        per_step = ("filter", "pairlaw32", "move")
        rebuild_k = ("bin", "scan", "place", "cellsort", "permute", "copyback", "pairs_count32",
                     "row_scan", "pairs_fill32", "link")
        step_bytes = sum(algorithmic_bytes(k, n, fp32["entries"], fp32["contacts"], ncells, False)
                         for k in per_step)
        step_bytes += (fp32["rebuilds"] / max(args.steps, 1)) * sum(
            algorithmic_bytes(k, n, fp32["entries"], fp32["contacts"], ncells, False)
            for k in rebuild_k)
        step_achieved = step_bytes / (fp32["ms"] / args.steps * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": fp32["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-split (f64 leapfrog)",
            "data": "synthetic",
            "config": {"workload": "periodic_gas_1M", "n": n, "steps_config": 2000,
                       "dt": sc.dt, "phi": scenarios.solid_fraction(sc),
                       "parallelism": f"replicas{world}",
                       "window": f"steps {args.advance + args.warmup + 1}-"
                                 f"{args.advance + args.warmup + args.steps} of the run "
                                 f"({args.advance} untimed + {args.warmup} warm-up steps first)",
                       "l2": "inputs larger than L2 (~0.5 GB of state per replica)"},
            "fp64": {"value": v64, "ms_per_step": fp64["ms"] / args.steps,
                     "fp32_split_speedup": value / v64, "status": fp64["status"]},
            "status": fp32["status"],
            "pairs": {"directed_entries": fp32["entries"], "contacts": fp32["contacts"]},
            "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm,
                         "peak_source": peak_src, "unit": "GB/s",
                         "frac": (achieved / hbm) if achieved else None,
                         "algorithmic_bytes_per_launch": ab, "avg_launch_us": 1e3 * avg_ms,
                         "traffic": traffic,
                         "step": {"algorithmic_bytes_per_step": step_bytes,
                                  "achieved": step_achieved, "frac": step_achieved / hbm,
                                  "note": "whole graph-replayed step: filter + pair kernel + "
                                          "leapfrog + the window's rebuilds, over ms_per_step"}},
            "phases_fp32_split": phases,
            "phases_fp64": phase_table(fp64["kt"], fp64, True) if "fp64" in res else None,
            "clocks": clocks,
            "e2e": {"value": world * n * args.e2e_steps / e2e_dt, "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": args.e2e_steps, "output_every": args.output_every,
                    "outputs": e2e_outputs,
                    "how": "Grains.set_state from pinned host memory, Grains.Simulation per "
                           "output interval (status read back), max/mean |v| read back at "
                           "each output time, final state downloaded to pinned memory; "
                           "host wall clock"},
            "gpu_launches": None,
        }
        # kernels launched in the timed region: the opening move, per step
        # k_decide, the contact filter, the pair kernel and the move, per
        # pair-list rebuild its 14 kernels (bin, scan x3, place, cellsort,
        # permute, copyback, row count, row scan x3, row fill, link), and the
        # history-table refills (every 512 evaluations per table)
        e0, e1 = fp32["evals"]
        fills = sum(1 for e in range(e0 + 1, e1 + 1) if e % 512 < 2)
        line["gpu_launches"] = 1 + 4 * args.steps + 14 * fp32["rebuilds"] + fills
        if "fp64" not in res:
            line["fp64"] = None
        line["pair_list"] = {"rebuilds_fp32_split": fp32["rebuilds"],
                             "rebuilds_fp64": fp64["rebuilds"], "steps": args.steps}
        line["window"] = {"contacts_at_end": fp32["contacts"], "rebuilds": fp32["rebuilds"],
                          "first_step": args.advance + args.warmup + 1, "steps": args.steps}
        if full is not None:
            line["full_config"] = full
        if not args.no_error:
            from oracle import reference
            if reference.available():
                line["error"] = error_full(sc, xml, args.advance, tmp.name)
            else:
                line["error"] = {"unavailable": "oracle/_ref was not built"}
            line["error"]["restatement_32k"] = {
                "sample": "periodic_gas n_fcc=20 (32,000 spheres), one step after 100 steps of "
                          "the CPU FP64 restatement, from its state",
                "fp32_split": error_sample(20, 100, FP32_SPLIT),
                "fp64": error_sample(20, 100, FP64)}
        if args.batched_instances > 0:
            line["batched"] = batched_measure(args.batched_instances, args.batched_steps)
        if args.convex_n > 0:
            line["convex"] = convex_measure(args.convex_n, args.convex_steps,
                                            graphs=not args.no_graphs)
        if args.adjoint_n > 0:
            line["adjoint"] = adjoint_measure(args.adjoint_n, args.adjoint_steps, 50)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(sc, xml)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    tmp.cleanup()


if __name__ == "__main__":
    main()
