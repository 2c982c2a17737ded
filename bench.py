#!/usr/bin/env python
"""Benchmark of the AKMC force path on B200: atom-force evaluations per second.

Workload (default, ``--workload ionic``): the rocksalt oxide of the ionic configuration
-- 5x5x5 conventional cells, one Schottky pair removed (998 ions, a0 = 4.21 A, charges
+2/-2), Buckingham Mg-O / O-O (Mg-Mg listed as zero), Ewald eta = 0.3 1/A with a 10 A
real-space cutoff and the reference's k-space rule (501 k-vectors) -- with
``--batch`` (default 16, the configuration's 16 Dimer searches) independently jittered
replicas (sigma 0.03 A, seeds 4321 + 1000*rank + k) per GPU.  One step = one force and
energy evaluation of every system of the batch.

``--workload eam``: the batched-walker metal configuration -- 512 FCC systems with
4^3..10^3 cells (256-4000 sites), 1-3 vacancies, sigma 0.02 A, tabulated FS-type EAM.

Arms:
  default             this repository's CUDA path (libakmc_b200.so)
  --impl reference    the reference's own Field::calculateForces (oracle/_ref, compiled
                      from the reference sources) on the host cores: one process per
                      core, each evaluating one system per step (the reference's MPI
                      task farm of independent searches, without MPI)

Saddle searches (``"saddles"`` in the JSON line, skip with ``--no-saddles``): the
batched-walker configuration -- 512 uneven FCC walkers per GPU, FIRE-relaxed to
max|F| < 1e-3 eV/A, then one Dimer search each from a random local displacement
(sigma 0.1 A on atoms within 4 A of a vacancy site), dimer separation 0.005 A, rotation
tolerance 0.1 eV/A^2, L-BFGS translation, saddle at max|F| < 5e-3 eV/A (the reference's
forceTol 1e-2 halved), at most 200 steps -- timed end to end (seeds
copied in from pinned host memory, results read back); converged saddles per second, with
the barrier error of a sample against the FP64 oracle and the FP64 oracle Dimer on the host
cores as CPU baseline.  ``"learned"`` (skip with ``--no-learned``): the same walkers seeded
by the learned proposal (akmc_b200.proposals, trained on plain searches of four other
512-walker sets), with the random seeds as fallback, timed the same way.

Multi-GPU (torchrun): every rank evaluates its own batch (independent walkers), no
collective in the data path; time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

ATOMS_PER_ION_SYSTEM = 998
RC_IONIC = 10.0
ETA = 0.3


# ------------------------------------------------------------------------------------
# inputs
# ------------------------------------------------------------------------------------
def write_potentials(d):
    from akmc_b200 import configs as cf
    precis = cf.ewald_precision_for_eta(ETA, RC_IONIC)
    # the product reads the 10 A cutoff with `nbrlist 0.0` (no Verlet shell); the reference
    # reads it without, and its setup guard is lifted through the harness (oracle/ref_harness.cpp)
    cf.write_ionic_potentials(os.path.join(d, "ion.pot"), RC_IONIC, precis, shell=0.0)
    cf.write_ionic_potentials(os.path.join(d, "ion_ref.pot"), RC_IONIC, precis)
    cf.write_setfl(os.path.join(d, "fs.setfl"))
    cf.write_eam_potentials(os.path.join(d, "eam.pot"), os.path.join(d, "fs.setfl"))


def make_systems(workload, batch, rank):
    from akmc_b200 import configs as cf
    if workload == "ionic":
        return [cf.rocksalt_schottky_system(5, 4.21, 0.03, 4321 + 1000 * rank + k) for k in range(batch)]
    return cf.uneven_fcc_batch(512, seed=2024 + rank)


# ------------------------------------------------------------------------------------
# CPU side: the reference (or the oracle port) on the host cores
# ------------------------------------------------------------------------------------
def _cpu_worker(args):
    kind, family, pot, pos, charge, labels, lat, warmup, steps, barrier, out_q = args
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    import oracle
    n = len(pos)
    if kind == "reference":
        override = 2 * (RC_IONIC + 1.0) + 1e-6 if family == "pair" else 0.0
        R = oracle.ReferenceField(family, pot, lat, n, override)
        call = lambda: R.forces(pos, charge, labels)
    else:
        if family == "pair":
            S = oracle.ionic_setup(pot, lat)
            call = lambda: oracle.ionic_forces(S, pos, charge, labels, lat)
        else:
            call = lambda: oracle.eam_forces(pot, pos, labels, lat)
    for _ in range(warmup):
        call()
    times = []
    for _ in range(steps):
        barrier.wait()
        t0 = time.perf_counter()
        call()
        times.append(time.perf_counter() - t0)
    out_q.put(times)


def cpu_run(workload, d, procs, warmup, steps):
    """procs processes, each evaluating one system per step; every step starts on a
    barrier and lasts as long as its slowest process.  Returns (atom-forces/s, kind,
    seconds of the timed steps, atoms evaluated)."""
    import oracle
    kind = "reference" if oracle.reference_available("pair" if workload == "ionic" else "eam") else "port"
    if not os.path.exists(oracle.LIB_PATH) and kind == "port":
        oracle.build(reference=False)
    systems = make_systems(workload, procs, 0)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs)
    q = ctx.Queue()
    jobs = []
    for p in range(procs):
        s = systems[p % len(systems)]
        if workload == "ionic":
            fam, pot = "pair", os.path.join(d, "ion_ref.pot" if kind == "reference" else "ion.pot")
        else:
            fam, pot = "eam", os.path.join(d, "eam.pot")
        jobs.append(ctx.Process(target=_cpu_worker, args=((kind, fam, pot, s.pos, s.charge, s.labels,
                                                           s.lat, warmup, steps, barrier, q),)))
    for j in jobs:
        j.start()
    per_proc = [q.get(timeout=7200) for _ in jobs]
    for j in jobs:
        j.join()
    step_s = [max(t[k] for t in per_proc) for k in range(steps)]
    secs = sum(step_s)
    atoms = sum(systems[p % len(systems)].n for p in range(procs)) * steps
    return atoms / secs, kind, secs, atoms


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def probe_reps(workload, d, target_s):
    """Reps per process so one process runs about target_s seconds."""
    import oracle
    s = make_systems(workload, 1, 0)[0]
    kind = "reference" if oracle.reference_available("pair" if workload == "ionic" else "eam") else "port"
    os.environ["OMP_NUM_THREADS"] = "1"
    if workload == "ionic":
        if kind == "reference":
            R = oracle.ReferenceField("pair", os.path.join(d, "ion_ref.pot"), s.lat, s.n, 2 * (RC_IONIC + 1.0) + 1e-6)
            call = lambda: R.forces(s.pos, s.charge, s.labels)
        else:
            S = oracle.ionic_setup(os.path.join(d, "ion.pot"), s.lat)
            call = lambda: oracle.ionic_forces(S, s.pos, s.charge, s.labels, s.lat)
    else:
        if kind == "reference":
            R = oracle.ReferenceField("eam", os.path.join(d, "eam.pot"), s.lat, s.n)
            call = lambda: R.forces(s.pos, s.charge, s.labels)
        else:
            call = lambda: oracle.eam_forces(os.path.join(d, "eam.pot"), s.pos, s.labels, s.lat)
    call()
    t = time.perf_counter()
    call()
    dt = time.perf_counter() - t
    return max(1, int(target_s / max(dt, 1e-6))), dt


# ------------------------------------------------------------------------------------
# saddle searches
# ------------------------------------------------------------------------------------
SADDLE_DELTA = 0.005          # dimer separation of the batched-walker configuration, A
SADDLE_ROT_TOL = 0.1          # rotation tolerance, eV/A^2
SADDLE_MAX_ITER = 200         # the configuration's 200-step horizon of a search
SADDLE_FORCE_TOL = 5e-3       # saddle at max|F| below this, eV/A (reference forceTol 1e-2; half of
                              # it keeps barriers a few tenths of a meV from the converged saddle)


def saddle_workload(rank, n=512):
    """512 uneven walkers and the site of each walker's first vacancy (the seeding centre)."""
    from akmc_b200 import configs as cf
    systems = cf.uneven_fcc_batch(n, seed=2024 + rank)
    centers = [cf.fcc_sites(s.meta["ncell"], s.meta["a0"])[s.meta["vacancies"][0]] for s in systems]
    return systems, centers


def saddle_seeds(xmin, systems, offsets, centers, rank):
    from akmc_b200 import configs as cf
    return np.concatenate([cf.local_displacements(xmin[offsets[k]:offsets[k + 1]], systems[k].box,
                                                  centers[k], 1, seed=7000 + 100003 * rank + k)[0]
                           for k in range(len(systems))])


def _cpu_saddle_worker(args):
    pot, jobs, budget_s, barrier, out_q = args
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    from oracle import walkers as W
    p = W.DimerParams(delta=SADDLE_DELTA, rot_tol=SADDLE_ROT_TOL, force_tol=SADDLE_FORCE_TOL,
                      max_iter=SADDLE_MAX_ITER)
    barrier.wait()
    t0 = time.perf_counter()
    done = conv = 0
    for lat, labels, xmin, seed in jobs:
        eo = W.EamOracle(pot, lat, labels)
        o = W.dimer_search(eo, xmin + seed, seed, p)
        done += 1
        conv += int(o["status"] == 1)
        if time.perf_counter() - t0 > budget_s:
            break
    out_q.put((done, conv, time.perf_counter() - t0))


def cpu_saddles(pot, small_jobs, procs, budget_s):
    """The FP64 oracle Dimer (oracle/walkers.py) on the host cores: procs processes, each
    searching its share of the small walkers until budget_s has passed."""
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs)
    q = ctx.Queue()
    ps = []
    for p in range(procs):
        ps.append(ctx.Process(target=_cpu_saddle_worker,
                              args=((pot, small_jobs[p::procs], budget_s, barrier, q),)))
    for x in ps:
        x.start()
    res = [q.get(timeout=7200) for _ in ps]
    for x in ps:
        x.join()
    done = sum(r[0] for r in res)
    conv = sum(r[1] for r in res)
    secs = max(r[2] for r in res)
    return conv / secs, done, conv, secs


PROPOSAL_TRAIN_BATCHES = 4     # plain-search batches (other seeds) the proposal learns from
LEARNED_MAX_ITER = 200         # a learned start not converged in 200 steps goes to the fallback


def train_proposer(f, rank, dev, p, n=512):
    """Two proposal models (akmc_b200.proposals) trained on the saddles of plain searches
    over PROPOSAL_TRAIN_BATCHES other 512-walker sets of the same configuration (seeds
    9000 + 10 * rank + t): the stand-in for the searches of earlier KMC steps."""
    import torch
    from akmc_b200 import configs as cf
    from akmc_b200 import proposals as P
    from akmc_b200.walkers import Walkers, fire_params, CONVERGED
    t0 = time.perf_counter()
    parts = {"direction": [], "score": []}
    for t in range(PROPOSAL_TRAIN_BATCHES):
        systems = cf.uneven_fcc_batch(n, seed=9000 + 10 * rank + t)
        centers = [cf.fcc_sites(s.meta["ncell"], s.meta["a0"])[s.meta["vacancies"][0]] for s in systems]
        w = Walkers.from_systems(f, systems)
        x = torch.tensor(np.concatenate([s.pos for s in systems]), device=dev)
        rr = w.relax(x, fire_params(force_tol=1e-3))
        xm = x.cpu().numpy()
        sd = saddle_seeds(xm, systems, w.offsets, centers, rank + 1000 * (t + 1))
        xs = torch.tensor(xm + sd, device=dev)
        res = w.dimer(xs, torch.tensor(sd, device=dev), p)
        desc, B = w.descriptors(x, with_basis=True)
        usable = (res["status"] == CONVERGED) & (res["energy"] - rr["energy"] < 2.0)
        r = P.hop_rows(desc.cpu().numpy(), B.cpu().numpy(), xm, xs.cpu().numpy(), w.offsets,
                       [s.box for s in systems], usable)
        for k in parts:
            parts[k].append(r[k])
        w.close()
    rows = {k: tuple(np.concatenate(z) for z in zip(*v)) for k, v in parts.items()}
    data_s = time.perf_counter() - t0
    prop = P.Proposer(seed=rank)
    t1 = time.perf_counter()
    h1, h2 = prop.fit(rows)
    torch.cuda.synchronize(dev)
    info = {"plain_batches": PROPOSAL_TRAIN_BATCHES, "direction_rows": int(len(rows["direction"][0])),
            "score_rows": int(len(rows["score"][0])), "data_s": data_s,
            "train_s": time.perf_counter() - t1,
            "direction_loss": [float(np.mean(h1[:5])), float(np.mean(h1[-5:]))],
            "score_loss": [float(np.mean(h2[:5])), float(np.mean(h2[-5:]))]}
    return prop, info


def run_learned(args, w, prop, xmin, seeds, emin, p, dev, stream, barrier):
    """The learned arm, timed end to end per search batch: minima and fallback seeds copied
    in from pinned host memory, descriptors + both models + akmc_proposal_seeds, the Dimer
    searches from the proposals, a second pass from the random seeds for the walkers whose
    learned search did not converge (akmc_walkers_dimer_subset), positions read back."""
    import torch
    from akmc_b200.walkers import CONVERGED, dimer_params
    xm_h = torch.tensor(xmin).pin_memory()
    fb_h = torch.tensor(seeds).pin_memory()
    xm_d = torch.empty_like(xm_h, device=dev)
    fb_d = torch.empty_like(fb_h, device=dev)
    counts = torch.tensor(np.diff(w.offsets), device=dev)
    pl = dimer_params(delta=p.delta, rot_tol=p.rot_tol, force_tol=p.force_tol,
                      max_iter=min(p.max_iter, LEARNED_MAX_ITER))
    ms, res, n_fb, n_noprop, prop_ms = [], None, 0, 0, []
    x_out = torch.empty(xm_h.shape, dtype=xm_h.dtype).pin_memory()     # positions read back
    for rep in range(1 + args.saddle_reps):
        barrier()
        torch.cuda.synchronize(dev)
        e0, e1, ep, el = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        xm_d.copy_(xm_h, non_blocking=True)
        fb_d.copy_(fb_h, non_blocking=True)
        disp, _, chosen = prop.propose(w, xm_d, seed=4242, counter=0, fallback=fb_d)
        x_d = xm_d + disp
        m_d = disp.clone()
        ep.record(stream)
        torch.cuda.nvtx.range_push("learned_search")       # profiling marker (no effect otherwise)
        res = w.dimer(x_d, m_d, pl, stream=stream.cuda_stream)
        torch.cuda.nvtx.range_pop()
        el.record(stream)
        fail = res["status"] != CONVERGED
        fail_status = np.bincount(res["status"][fail], minlength=6).tolist()
        if fail.any():
            mask = torch.tensor(fail.astype(np.int32), device=dev)
            x2 = xm_d + fb_d
            m2 = fb_d.clone()
            r2 = w.dimer_subset(x2, m2, mask, p, stream=stream.cuda_stream)
            res[fail] = r2[fail]
            rows = mask.bool().repeat_interleave(counts)[:, None]
            x_d = torch.where(rows, x2, x_d)
            m_d = torch.where(rows, m2, m_d)
        x_out.copy_(x_d, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if rep > 0:
            ms.append(e0.elapsed_time(e1))
            prop_ms.append((e0.elapsed_time(ep), ep.elapsed_time(el), el.elapsed_time(e1), fail_status))
        n_fb = int(fail.sum())
        n_noprop = int((chosen < 0).sum())
    return ms, res, x_out, m_d.cpu(), n_fb, n_noprop, prop_ms, proposal_kernels(w, prop, xm_d, dev, stream)


def proposal_kernels(w, prop, x, dev, stream, reps=5):
    """CUDA-event times of the proposal's parts on the walkers' minima (best of reps):
    descriptors (one force call on the walkers' batch + the descriptor kernel), each model's
    forward (tcgen05), the seeding kernel."""
    import torch
    from akmc_b200 import proposals as P
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    best = {}
    for _ in range(reps):
        e = [ev() for _ in range(5)]
        e[0].record(stream)
        desc, basis = w.descriptors(x, with_basis=True)
        e[1].record(stream)
        pred = prop.direction.predict(desc, basis)
        e[2].record(stream)
        score = prop.score.predict(desc)
        e[3].record(stream)
        begin, box = w.device_geometry()
        P.seeds(begin, x, box, pred, score)
        e[4].record(stream)
        torch.cuda.synchronize(dev)
        t = [e[k].elapsed_time(e[k + 1]) for k in range(4)]
        for name, v in zip(("descriptors_ms", "direction_forward_ms", "score_forward_ms", "seeds_ms"), t):
            best[name] = min(best.get(name, 1e30), v)
    rows = int(w.n_total)
    flops = 2.0 * rows * (64 * 128 + 2 * 128 * 128 + 128 * 3)
    best["rows"] = rows
    best["forward_tflops"] = flops / (best["score_forward_ms"] * 1e-3) / 1e12
    return best


def run_saddles(args, world, rank, dev, d, barrier):
    """Batched FIRE + Dimer walkers (akmc_walkers_*) on the batched-walker configuration."""
    import torch
    from akmc_b200 import Field, PREC_FP64, PREC_MIXED
    from akmc_b200.walkers import Walkers, dimer_params, fire_params

    systems, centers = saddle_workload(rank, args.saddle_walkers)
    pot = os.path.join(d, "eam.pot")
    f = Field().readPotential(pot).setup(systems[0].lat, None, max(s.n for s in systems))
    f.setPrecision(PREC_FP64 if args.fp64 else PREC_MIXED)
    w = Walkers.from_systems(f, systems)
    natoms = np.diff(w.offsets)
    stream = torch.cuda.current_stream(dev)
    pos = torch.tensor(np.concatenate([s.pos for s in systems]), device=dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    rr = w.relax(pos, fire_params(force_tol=1e-3))
    relax_s = time.perf_counter() - t0
    xmin = pos.cpu().numpy()
    emin = rr["energy"].copy()
    seeds = saddle_seeds(xmin, systems, w.offsets, centers, rank)
    x_h = torch.tensor(xmin + seeds).pin_memory()
    m_h = torch.tensor(seeds).pin_memory()
    x_d = torch.empty_like(x_h, device=dev)
    m_d = torch.empty_like(m_h, device=dev)
    p = dimer_params(delta=SADDLE_DELTA, rot_tol=SADDLE_ROT_TOL, force_tol=SADDLE_FORCE_TOL,
                     max_iter=SADDLE_MAX_ITER)
    ms, res = [], None
    x_out = torch.empty(x_h.shape, dtype=x_h.dtype).pin_memory()       # positions read back
    for rep in range(1 + args.saddle_reps):          # the first search is the warm-up
        barrier()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        x_d.copy_(x_h, non_blocking=True)
        m_d.copy_(m_h, non_blocking=True)
        torch.cuda.nvtx.range_push("plain_search")         # profiling marker (no effect otherwise)
        res = w.dimer(x_d, m_d, p, stream=stream.cuda_stream)
        torch.cuda.nvtx.range_pop()
        x_out.copy_(x_d, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if rep > 0:
            ms.append(e0.elapsed_time(e1))
    from akmc_b200 import shard
    secs = shard.max_over_ranks(sum(ms) / 1e3, device=dev)
    conv = res["status"] == 1
    n_conv = int(conv.sum())
    if world > 1:
        # the one exchange: fixed-size per-walker records to rank 0 (ids are global)
        ids = rank * len(systems) + np.arange(len(systems))
        allr = shard.gather_records(shard.records(ids, res, emin), world * len(systems), device=dev)
        if rank == 0:
            n_conv_all = int((allr[:, 1] == 1).sum())
    calls = int(res["force_calls"].sum())
    atom_forces = float((res["force_calls"] * natoms).sum())
    barriers = res["energy"][conv] - emin[conv]
    if world == 1:
        n_conv_all = n_conv
    elif rank != 0:
        n_conv_all = 0
    out = {"metric": "converged saddles/s", "value": n_conv_all * len(ms) / secs,
           "unit": "saddles/s", "walkers_per_gpu": len(systems), "converged": n_conv,
           "lost": int((res["status"] == 3).sum()), "max_iter": int((res["status"] == 2).sum()),
           "unique": n_conv, "reps": len(ms), "s_per_search_batch": secs / len(ms),
           "force_calls": calls, "atom_forces_per_s": world * atom_forces * len(ms) / secs,
           "iters_mean": float(res["iters"].mean()), "iters_max": int(res["iters"].max()),
           "barrier_eV_median": float(np.median(barriers)) if n_conv else None,
           "relax_s": relax_s, "dimer": {"delta_A": SADDLE_DELTA, "rot_tol": SADDLE_ROT_TOL,
                                        "force_tol": p.force_tol, "max_iter": p.max_iter},
           "timing": "device events around H2D of seeds, the batched search and D2H of positions "
                     "(pinned host buffers both ways)",
           "config": f"{len(systems)} uneven FCC walkers (4^3..10^3 cells, 1-3 vacancies, sigma 0.02 A), "
                     "one search each; unique = converged (one walker per system)"}
    if not args.no_learned:
        prop, tinfo = train_proposer(f, rank, dev, p, args.saddle_walkers)
        lms, lres, lx, lm, n_fb, n_noprop, prop_ms, pk = run_learned(args, w, prop, xmin, seeds, emin, p, dev,
                                                                 stream, barrier)
        lsecs = shard.max_over_ranks(sum(lms) / 1e3, device=dev)
        lconv = lres["status"] == 1
        l_all = shard.sum_over_ranks(int(lconv.sum()), device=dev)
        p_all = shard.sum_over_ranks(n_conv, device=dev)
        lb = lres["energy"][lconv] - emin[lconv]
        pb = barriers
        out["learned"] = {
            "value": l_all * len(lms) / lsecs, "unit": "saddles/s", "converged": int(lconv.sum()),
            "s_per_search_batch": lsecs / len(lms),
            "propose_ms": float(np.mean([q[0] for q in prop_ms])),
            "learned_pass_ms": float(np.mean([q[1] for q in prop_ms])),
            "fallback_pass_ms": float(np.mean([q[2] for q in prop_ms])),
            "learned_pass_failures_by_status": prop_ms[-1][3],
            "fallback_walkers": n_fb, "walkers_without_proposal": n_noprop,
            "learned_max_iter": LEARNED_MAX_ITER, "force_calls": int(lres["force_calls"].sum()),
            "iters_mean": float(lres["iters"].mean()), "iters_max": int(lres["iters"].max()),
            "barrier_eV_pct_5_50_95": [float(v) for v in np.percentile(lb, [5, 50, 95])] if len(lb) else None,
            "plain_barrier_eV_pct_5_50_95": [float(v) for v in np.percentile(pb, [5, 50, 95])] if len(pb) else None,
            "vs_plain": (l_all * len(lms) / lsecs) / (p_all * len(ms) / secs) if p_all else None,
            "training": tinfo, "proposal_kernels": pk,
            "timing": "device events around H2D of minima and fallback seeds, descriptors, both "
                      "models, seeding kernel, the batched search, the fallback pass and D2H of "
                      "positions (pinned host buffers both ways; fallback_pass_ms includes the "
                      "read-back); training (plain searches of other sets) is outside"}
    # barrier error against the FP64 oracle, on the converged 4^3 walkers (cheap on the host)
    def barrier_errors(xs, ms, r):
        """On up to 8 converged 4^3 walkers: |barrier - FP64 oracle barrier at the same
        positions| (the arithmetic); |barrier - barrier of the FP64 oracle Dimer continued
        from the saddle and mode to max|F| < 1e-5 eV/A| (the convergence); and |barrier -
        barrier of the reference's own ART (optim/ART.cpp on the reference Field) started at
        the saddle nudged 0.05 A along the mode| (the reference's saddle search)."""
        import oracle
        from oracle import walkers as W
        errs, conv, art = [], [], []
        tight = W.DimerParams(delta=SADDLE_DELTA, rot_tol=SADDLE_ROT_TOL, force_tol=1e-5, max_iter=500)
        for k in [k for k in range(len(systems)) if r["status"][k] == 1 and systems[k].meta["ncell"] == 4][:8]:
            sl = slice(w.offsets[k], w.offsets[k + 1])
            eo = W.EamOracle(pot, systems[k].lat, systems[k].labels)
            _, es, _ = eo(xs[sl])
            _, em, _ = eo(xmin[sl])
            errs.append(abs((r["energy"][k] - emin[k]) - (es - em)))
            o = W.dimer_search(eo, xs[sl], ms[sl], tight)
            if o["status"] == 1:
                conv.append(abs((r["energy"][k] - emin[k]) - (o["energy"] - em)))
            if oracle.reference_available("eam"):
                q = systems[k]
                ref = oracle.ReferenceField("eam", pot, q.lat, q.n)
                e_ref = ref.forces(xmin[sl], q.charge, q.labels)[0]["total"]
                st, e_art, _ = ref.art(xs[sl], q.charge, q.labels, 0.05 * ms[sl], init_dt=0.0005, max_dt=0.001,
                                       max_par_iter=3000)
                ref.close()
                if st == 0:
                    art.append(abs((r["energy"][k] - emin[k]) - (e_art - e_ref)))
        if not errs:
            return None
        return {"max": float(max(errs)), "walkers": len(errs), "bar": 1e-3,
                "vs_saddle_at_1e-5_max": float(max(conv)) if conv else None, "tight_walkers": len(conv),
                "vs_reference_art_max": float(max(art)) if art else None, "art_walkers": len(art)}

    if rank == 0:
        out["barrier_error_vs_fp64_oracle_eV"] = barrier_errors(x_out.numpy(), m_d.cpu().numpy(), res)
        if "learned" in out:
            out["learned"]["barrier_error_vs_fp64_oracle_eV"] = barrier_errors(lx.numpy(), lm.numpy(), lres)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        jobs = [(systems[k].lat, systems[k].labels, xmin[w.offsets[k]:w.offsets[k + 1]],
                 seeds[w.offsets[k]:w.offsets[k + 1]]) for k in range(len(systems))
                if systems[k].meta["ncell"] == 4]
        procs = args.cpu_procs or cpu_cores()
        rate, done, cc, cs = cpu_saddles(pot, jobs, procs, args.cpu_seconds)
        out["cpu_baseline"] = {"value": rate, "unit": "saddles/s", "cores": procs, "kind": "port",
                               "sample": f"FP64 oracle Dimer (oracle/walkers.py; the reference's Dimer is "
                                         f"a stub) on the 4^3 walkers of the same set, {procs} processes, "
                                         f"{done} searches, {cc} converged in {cs:.1f} s"}
    w.close()
    return out


# ------------------------------------------------------------------------------------
# the AKMC loop at scale (opt-in: --akmc-steps)
# ------------------------------------------------------------------------------------
def run_akmc(args, rank, dev, d):
    """The full-loop configuration: FCC 20^3 (32 000 sites) with a seeded 6-vacancy cluster
    and 10 isolated vacancies, 1024 Dimer walkers per KMC step seeded around the 16 vacancy
    sites, FP64 event table, rates at 1e13 1/s and 600 K.  Two trajectories of the same
    number of steps: random seeds throughout, and learned proposals (the first step random,
    its saddles train the proposer, later steps learned within each walker's 4 A region).
    Per step: converged saddles, distinct events, Dimer force calls, wall time."""
    import torch
    from akmc_b200 import Field, PREC_MIXED
    from akmc_b200 import configs as cf
    from akmc_b200 import proposals as P
    from akmc_b200.akmc_loop import AkmcLoop
    s = cf.fcc_cluster_system(20, seed=2026 + rank)
    f = Field().readPotential(os.path.join(d, "eam.pot")).setup(s.lat, None, s.n)
    f.setPrecision(PREC_MIXED)
    find = cf.fcc_vacancy_finder(20, 3.615)
    out = {"config": f"FCC 20^3 ({s.n} atoms), 6-vacancy cluster + 10 isolated vacancies, "
                     f"{args.akmc_walkers} walkers per KMC step, nu 1e13 1/s, 600 K",
           "dimer": {"delta_A": 0.01, "rot_tol": 0.1, "force_tol": 1e-3}}
    for arm, proposer in (("plain", None), ("learned", P.Proposer(seed=rank))):
        loop = AkmcLoop(f, s, find, n_walkers=args.akmc_walkers, seed=7 + rank, proposer=proposer,
                        proposal_threshold=0.0)
        steps = []
        for _ in range(args.akmc_steps):
            torch.cuda.synchronize(dev)
            t = time.perf_counter()
            rec = loop.step()
            torch.cuda.synchronize(dev)
            dt = time.perf_counter() - t
            steps.append({"s": dt, "converged": rec.n_saddles, "unique": rec.n_unique,
                          "dimer_force_calls": rec.force_calls, "learned": rec.learned,
                          "fallback": rec.n_fallback, "barrier_eV": rec.barrier, "kmc_dt_s": rec.dt})
        secs = sum(x["s"] for x in steps)
        out[arm] = {"steps": steps, "converged_saddles_per_s": sum(x["converged"] for x in steps) / secs,
                    "unique_events_per_s": sum(x["unique"] for x in steps) / secs,
                    "dimer_atom_forces_per_s": sum(x["dimer_force_calls"] for x in steps) * s.n / secs}
    return out


# ------------------------------------------------------------------------------------
# clocks
# ------------------------------------------------------------------------------------
QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    def __init__(self, path):
        self.path = path
        self.p = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={QUERY}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self, gpu_index=None):
        rows = []
        try:
            for line in open(self.path):
                c = [x.strip() for x in line.split(",")]
                if len(c) < 9:
                    continue
                if gpu_index is not None and c[0] != str(gpu_index):
                    continue
                rows.append(c)
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "samples": len(rows), "reasons": sorted(reasons)}


# ------------------------------------------------------------------------------------
# algorithmic bytes per launch (compulsory DRAM traffic; neighbour re-reads excluded)
# ------------------------------------------------------------------------------------
def algorithmic_bytes(kernel, n_atoms, nsys, nk):
    per_atom = {"ionic_force": 32 + 4 + 24 + 16,          # spos, slabel in; force, energies out
                "structure_factor": 32,                    # spos in
                "eam_force": 32 + 4 + 16 + 24 + 8,         # spos, slabel, {F',rho} in; force, E out
                "eam_density": 32 + 4 + 16 + 8,            # spos, slabel in; {F',rho}, E out
                "cell_sort": 24 + 4 + 8 + 24 + 32 + 4 + 4 + 16,
                "energy_reduce": 16 + 8}
    per_k = {"ionic_force": 16 + 8 + 16, "structure_factor": 16 + 16, "energy_reduce": 16 + 8}
    return n_atoms * per_atom.get(kernel, 0) + nsys * nk * per_k.get(kernel, 0)


def ncu_traffic(kernel, workload):
    """DRAM bytes per launch from the committed ncu summary, when present."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        w = line.split()
        if len(w) >= 3 and not line.startswith("#") and w[0] == kernel and w[1] == workload:
            try:
                return float(w[2])
            except ValueError:
                return None
    return None


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# ------------------------------------------------------------------------------------
# arms
# ------------------------------------------------------------------------------------
def run_reference_arm(args, world, rank):
    if rank != 0:
        return 0
    d = tempfile.mkdtemp(prefix="akmc_bench_")
    write_potentials(d)
    procs = args.cpu_procs or cpu_cores()
    value, kind, t_total, atoms_total = cpu_run(args.workload, d, procs, max(1, args.warmup), args.steps)
    line = {"impl": "reference", "metric": "atom-forces/s", "value": value, "unit": "atom-forces/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, procs_note=procs),
            "cpu_baseline": {"value": value, "unit": "atom-forces/s", "cores": procs, "kind": kind,
                             "sample": f"{procs} processes x 1 Field::calculateForces call per step "
                                       f"({'998-ion rocksalt' if args.workload == 'ionic' else 'FCC walker'} "
                                       f"system each), {args.steps} steps"},
            "e2e": {"value": value, "unit": "atom-forces/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def workload_config(args, procs_note=None, nk=None):
    if args.workload == "ionic":
        c = {"workload": f"rocksalt 5x5x5 Schottky (998 ions), Buckingham + Ewald eta 0.3, rc 10 A; "
                         f"{args.batch} independent systems per GPU",
             "systems_per_gpu": args.batch, "atoms_per_system": ATOMS_PER_ION_SYSTEM,
             "cutoff_A": RC_IONIC, "eta": ETA}
        if nk is not None:
            c["k_vectors"] = nk
    else:
        c = {"workload": "512 uneven FCC walkers (4^3..10^3 cells, 1-3 vacancies), tabulated FS EAM, rc 5 A",
             "systems_per_gpu": 512}
    c["l2"] = "flushed between timed steps (256 MiB write, untimed)"
    if getattr(args, "skin", 0.0) > 0.0 and args.workload == "eam":
        c["neighbour_lists"] = f"reused (skin {args.skin} A; built on the first call)"
    c["precision"] = "FP32 pair terms, FP64 geometry/near pairs/accumulation" if not args.fp64 else "FP64"
    if procs_note:
        c["host_processes"] = procs_note
        c["precision"] = "FP64 (the reference's own code)"
    return c


def run_ours(args, world, rank, local_rank):
    import torch
    import torch.distributed as dist
    from akmc_b200 import Field, PREC_FP64, PREC_MIXED

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    d = tempfile.mkdtemp(prefix=f"akmc_bench_{rank}_")
    write_potentials(d)
    systems = make_systems(args.workload, args.batch, rank)
    pot = os.path.join(d, "ion.pot" if args.workload == "ionic" else "eam.pot")
    f = Field().readPotential(pot).setup(systems[0].lat, None, max(s.n for s in systems))
    f.setPrecision(PREC_FP64 if args.fp64 else PREC_MIXED)
    nat = [s.n for s in systems]
    b = f.batch(nat, np.array([s.box for s in systems]), np.concatenate([s.labels for s in systems]),
                np.concatenate([s.charge for s in systems]), skin=args.skin)
    nk = f.ewald()["nk"] if args.workload == "ionic" else 0
    n_total = b.n_total
    pos = torch.tensor(np.concatenate([s.pos for s in systems]), device=dev)
    force, energy, status = b.alloc(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MiB > L2
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()

    # the library's autotuner picks the work-item size for this batch (part of set-up)
    home_chunk = b.autotune(pos, force, energy, status, stream.cuda_stream)
    for _ in range(args.warmup):
        b.forces_(pos, force, energy, status, stream.cuda_stream)
    torch.cuda.synchronize(dev)
    if int(status.max().item()) != 0:
        raise RuntimeError(f"force call reported status {status.max().item()}")

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks_path = os.path.join(tempfile.mkdtemp(), "clocks.csv")
    barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(clocks_path) as cs:
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            b.forces_(pos, force, energy, status, stream.cuda_stream)
            ends[k].record(stream)
        torch.cuda.synchronize(dev)
        barrier()
    dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    # Per-kernel device times from a second pass of the same steps: the events the library
    # records around each kernel would serialise the overlapped launches of the timed pass.
    b.profile(True)
    for k in range(args.steps):
        flush.zero_()
        b.forces_(pos, force, energy, status, stream.cuda_stream)
    torch.cuda.synchronize(dev)
    ktimes = b.kernel_times()
    b.profile(False)
    if int(status.max().item()) != 0:
        raise RuntimeError(f"force call reported status {status.max().item()}")
    t = torch.tensor([dev_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world * n_total * args.steps / (max_ms / 1e3)

    # end to end through the host-buffer call: pinned inputs in, forces/energies out
    pos_h = torch.tensor(np.concatenate([s.pos for s in systems])).pin_memory()
    force_h = torch.empty((n_total, 3), dtype=torch.float64).pin_memory()
    energy_h = torch.empty((len(nat), 5), dtype=torch.float64).pin_memory()
    status_h = torch.empty((len(nat),), dtype=torch.int32).pin_memory()
    for _ in range(max(1, args.warmup)):
        b.forces_host(pos_h, force_h, energy_h, status_h, stream.cuda_stream)
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize(dev)
    for k in range(args.steps):
        flush.zero_()
        e0[k].record(stream)
        b.forces_host(pos_h, force_h, energy_h, status_h, stream.cuda_stream)
        e1[k].record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    e2e_ms = sum(a.elapsed_time(c) for a, c in zip(e0, e1))
    t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * n_total * args.steps / (float(t.item()) / 1e3)

    # roofline of the dominant kernel
    dom = max(ktimes, key=lambda k: ktimes[k][0])
    dom_ms, dom_n = ktimes[dom]
    avg_s = dom_ms / dom_n / 1e3
    alg = algorithmic_bytes(dom, n_total, len(nat), nk)
    peaks, peak_kind = measured_peaks()
    achieved = alg / avg_s / 1e9
    tr = ncu_traffic(dom, args.workload)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "peak_source": peak_kind,
                "traffic": tr, "alg_bytes_per_launch": alg, "launch_ms": avg_s * 1e3,
                "note": "compulsory bytes only; the kernel is FP64/FP32-pipe bound, see profiles/"}

    line = {"metric": "atom-forces/s", "value": value, "unit": "atom-forces/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.fp64 else "f64+f32", "data": "synthetic",
            "config": dict(workload_config(args, nk=nk), home_chunk=home_chunk),
            "roofline": roofline,
            "kernels": {k: {"ms_per_launch": v[0] / v[1], "launches": v[1]} for k, v in ktimes.items()},
            "gpu_launches": b.launches * args.steps,
            "e2e": {"value": e2e_value, "unit": "atom-forces/s",
                    "h2d_bytes_per_step": n_total * 3 * 8,
                    "d2h_bytes_per_step": n_total * 3 * 8 * 2 + len(nat) * (5 * 8 + 4)},
            "clocks": cs.summary(None if world == 1 else local_rank)}

    if not args.no_saddles:
        line["saddles"] = run_saddles(args, world, rank, dev, d, barrier)
    if args.akmc_steps > 0:
        line["akmc"] = run_akmc(args, rank, dev, d)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        reps, dt = probe_reps(args.workload, d, args.cpu_seconds)
        procs = args.cpu_procs or cpu_cores()
        rate, kind, secs, atoms = cpu_run(args.workload, d, procs, 1, reps)
        line["cpu_baseline"] = {"value": rate, "unit": "atom-forces/s", "cores": procs, "kind": kind,
                                "sample": f"{procs} processes x {reps} Field::calculateForces calls "
                                          f"({'one 998-ion system' if args.workload == 'ionic' else 'one FCC walker'}"
                                          f" each, {secs:.1f} s)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["ionic", "eam"], default="ionic")
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--fp64", action="store_true", help="every pair term in FP64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--cpu-procs", type=int, default=0)
    ap.add_argument("--no-saddles", action="store_true", help="skip the batched Dimer measurement")
    ap.add_argument("--skin", type=float, default=0.0,
                    help="EAM neighbour-list skin (A) of the force-path batch; every timed step then "
                         "reuses the lists of the first call (positions do not move between steps)")
    ap.add_argument("--saddle-reps", type=int, default=2, help="timed batched searches")
    ap.add_argument("--saddle-walkers", type=int, default=512,
                    help="walkers of the saddle measurement (the configuration has 512; fewer for profiling)")
    ap.add_argument("--akmc-steps", type=int, default=0,
                    help="also run the AKMC loop at scale (32 000-site crystal) for this many KMC steps "
                         "per arm (minutes per arm; off by default)")
    ap.add_argument("--akmc-walkers", type=int, default=1024, help="walkers per KMC step of --akmc-steps")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-proposal arm of the saddle measurement")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, world, rank)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        return run_ours(args, world, rank, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
