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
by the learned proposal (akmc_b200.proposals, trained on plain searches of other 512-walker
sets until ``--train-saddles`` converged saddles are in hand), with the random seeds as
fallback, timed the same way.

The ionic configuration's 16 Dimer searches (``"ionic_searches"``, skip with
``--no-ionic-searches``): mixed precision against all-FP64 from the same nearest-neighbour hop
starts, and every mixed saddle's energy, forces and barrier against the FP64 oracle at the
same positions.  The full-loop configuration (``"akmc"``, ``--akmc-steps`` KMC steps per arm,
6 by default, 0 skips it): the AKMC loop on the 32 000-site crystal, walkers over local
regions with the rate-relevant unique saddles polished in the crystal, random and learned
seeds (``--akmc-arms``).

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


def cpu_run(workload, d, procs, warmup, steps, systems=None):
    """procs processes, each evaluating one system per step (the workload's, or from
    ``systems``); every step starts on a barrier and lasts as long as its slowest process.
    Returns (atom-forces/s, kind, seconds of the timed steps, atoms evaluated)."""
    import oracle
    kind = "reference" if oracle.reference_available("pair" if workload == "ionic" else "eam") else "port"
    if not os.path.exists(oracle.LIB_PATH) and kind == "port":
        oracle.build(reference=False)
    systems = systems or make_systems(workload, procs, 0)
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


def saddle_workload(rank, n=512, per_system=4):
    """n uneven walkers: n / per_system systems, each searched by per_system consecutive
    walkers from different random starts (so that duplicate saddles can be found and unique
    ones counted), and the site of each walker's first vacancy (the seeding centre)."""
    from akmc_b200 import configs as cf
    base = cf.uneven_fcc_batch(max(1, n // per_system), seed=2024 + rank)
    systems = [q for q in base for _ in range(per_system)][:n]
    centers = [cf.fcc_sites(q.meta["ncell"], q.meta["a0"])[q.meta["vacancies"][0]] for q in systems]
    return systems, centers


SADDLE_REGION = 4.0           # A: the plain seeds' radius around the centre, the learned candidates' region
UNIQUE_E_TOL = 1e-3           # eV: saddles of one system closer than this in energy ...
UNIQUE_D_TOL = 0.1            # ... and than this for every atom (A) are the same saddle


def unique_saddles(w, x_d, res, per_system, dev, stream):
    """Converged saddles that do not repeat an earlier saddle of the same system
    (akmc_events_dedup on the device).  Returns the host mask."""
    import torch
    from akmc_b200 import kmc
    W_ = len(res["status"])
    begin, box = w.device_geometry()
    group = torch.tensor((np.arange(W_) // per_system).astype(np.int32), device=dev)
    usable = torch.tensor((res["status"] == 1).astype(np.int32), device=dev)
    energy = torch.tensor(np.asarray(res["energy"], dtype=np.float64), device=dev)
    natoms = (begin[1:] - begin[:-1]).to(torch.int32)
    dup = kmc.dedup(group, usable, energy, x_d, begin[:-1].contiguous(), natoms, box,
                    e_tol=UNIQUE_E_TOL, d_tol=UNIQUE_D_TOL, stream=stream.cuda_stream)
    return (res["status"] == 1) & (dup.cpu().numpy() < 0)


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


def _barrier_check_worker(job):
    """One converged GPU saddle against the checkers (a spawned process; oracle code only):
    |barrier - FP64 oracle barrier at the same positions| (the arithmetic); |barrier -
    barrier of the FP64 oracle Dimer continued from the saddle and mode to max|F| < 1e-5
    eV/A| (the convergence); |barrier - barrier of the reference's own ART (optim/ART.cpp on
    the reference Field) started at the saddle nudged 0.05 A along the mode| (the
    reference's saddle search)."""
    pot, lat, labels, charge, xmin, xs, ms, barrier, threads = job
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, ROOT)
    import oracle
    from oracle import walkers as W
    out = {}
    eo = W.EamOracle(pot, lat, labels)
    _, es, _ = eo(xs)
    _, em, _ = eo(xmin)
    out["arith"] = abs(barrier - (es - em))
    tight = W.DimerParams(delta=SADDLE_DELTA, rot_tol=SADDLE_ROT_TOL, force_tol=1e-5, max_iter=500)
    o = W.dimer_search(eo, xs, ms, tight)
    out["tight"] = abs(barrier - (o["energy"] - em)) if o["status"] == 1 else None
    out["art"] = None
    if oracle.reference_available("eam"):
        ref = oracle.ReferenceField("eam", pot, lat, len(xs))
        e_ref = ref.forces(xmin, charge, labels)[0]["total"]
        st, e_art, _ = ref.art(xs, charge, labels, 0.05 * ms, init_dt=0.0005, max_dt=0.001, max_par_iter=3000)
        ref.close()
        if st == 0:
            out["art"] = abs(barrier - (e_art - e_ref))
    return out


def barrier_checks(pot, systems, offsets, xmin, emin, arms, per_class, procs):
    """Barrier errors of converged GPU saddles, per_class walkers from each size class
    (4^3, 6^3, 8^3, 10^3 cells) of every arm, checked in a spawned process pool (after the
    GPU work; nothing here touches the GPU).  Returns {arm: summary}."""
    jobs, keys = [], []
    classes = sorted({s.meta["ncell"] for s in systems})
    for name, xs, ms, r in arms:
        for c in classes:
            ks = [k for k in range(len(systems)) if r["status"][k] == 1 and systems[k].meta["ncell"] == c][:per_class]
            for k in ks:
                sl = slice(offsets[k], offsets[k + 1])
                q = systems[k]
                jobs.append((pot, q.lat, q.labels, q.charge, xmin[sl], xs[sl], ms[sl],
                             float(r["energy"][k] - emin[k]), 1))
                keys.append((name, c, k))
    if not jobs:
        return {name: None for name, *_ in arms}
    nproc = max(1, min(procs, len(jobs)))
    threads = max(1, procs // nproc)
    jobs = [j[:-1] + (threads,) for j in jobs]
    with mp.get_context("spawn").Pool(nproc) as pool:
        results = pool.map(_barrier_check_worker, jobs, chunksize=1)
    out = {}
    for name, *_ in arms:
        rows = [(c, k, res) for (a, c, k), res in zip(keys, results) if a == name]
        per = {}
        for c in classes:
            rc = [res for cc, _, res in rows if cc == c]
            if not rc:
                continue
            t = [x["tight"] for x in rc if x["tight"] is not None]
            a = [x["art"] for x in rc if x["art"] is not None]
            per[f"{c}^3"] = {"walkers": len(rc), "max": max(x["arith"] for x in rc),
                             "vs_saddle_at_1e-5_max": max(t) if t else None,
                             "vs_reference_art_max": max(a) if a else None, "art_walkers": len(a)}
        allr = [res for _, _, res in rows]
        t = [x["tight"] for x in allr if x["tight"] is not None]
        a = [x["art"] for x in allr if x["art"] is not None]
        out[name] = {"max": max(x["arith"] for x in allr), "walkers": len(allr), "bar": 1e-3,
                     "vs_saddle_at_1e-5_max": max(t) if t else None, "tight_walkers": len(t),
                     "vs_reference_art_max": max(a) if a else None, "art_walkers": len(a),
                     "per_size_class": per,
                     "sample": f"{per_class} converged walkers per size class"}
    return out


PROPOSAL_TRAIN_MAX_BATCHES = 40   # plain-search batches (other seeds) at most
LEARNED_MAX_ITER = 200         # a learned start not converged in 200 steps goes to the fallback
LEARNED_PATIENCE = 40          # ... and so does one whose max|F| has not fallen 2 % below its best in 40 steps


def train_proposer(f, rank, dev, p, n=512, min_saddles=10000):
    """Two proposal models (akmc_b200.proposals) trained on the saddles of plain searches
    over other 512-walker sets of the same configuration (seeds 9000 + 10 * rank + t), as
    many as give min_saddles usable converged saddles (their displacement fields): the
    stand-in for the searches of earlier KMC steps."""
    import torch
    from akmc_b200 import configs as cf
    from akmc_b200 import proposals as P
    from akmc_b200.walkers import Walkers, fire_params, CONVERGED
    t0 = time.perf_counter()
    parts = {"direction": [], "score": []}
    n_saddles, batches = 0, 0
    for t in range(PROPOSAL_TRAIN_MAX_BATCHES):
        if n_saddles >= min_saddles:
            break
        batches += 1
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
        n_saddles += int(usable.sum())
        r = P.hop_rows(desc, B, xm, xs.cpu().numpy(), w.offsets, [s.box for s in systems], usable)
        for k in parts:
            parts[k].append(r[k])
        w.close()
    rows = {k: tuple(np.concatenate(z) for z in zip(*v)) for k, v in parts.items()}
    data_s = time.perf_counter() - t0
    prop = P.Proposer(seed=rank)
    t1 = time.perf_counter()
    h1, h2 = prop.fit(rows)
    torch.cuda.synchronize(dev)
    info = {"plain_batches": batches, "saddles": n_saddles, "direction_rows": int(len(rows["direction"][0])),
            "score_rows": int(len(rows["score"][0])), "data_s": data_s,
            "train_s": time.perf_counter() - t1,
            "direction_loss": [float(np.mean(h1[:5])), float(np.mean(h1[-5:]))],
            "score_loss": [float(np.mean(h2[:5])), float(np.mean(h2[-5:]))]}
    return prop, info


def run_learned(args, w, prop, xmin, seeds, emin, p, dev, stream, barrier, centers):
    """The learned arm, timed end to end per search batch: minima and fallback seeds copied
    in from pinned host memory, descriptors + both models + akmc_proposal_seeds, the Dimer
    searches from the proposals, a second pass from the random seeds for the walkers whose
    learned search did not converge (akmc_walkers_dimer_subset), positions read back.  The
    candidates of a walker are the atoms within SADDLE_REGION of its seeding centre, the
    region the plain arm's random displacements cover; only they get descriptors and
    predictions."""
    import torch
    from akmc_b200 import proposals as P
    from akmc_b200.walkers import CONVERGED, dimer_params
    xm_h = torch.tensor(xmin).pin_memory()
    fb_h = torch.tensor(seeds).pin_memory()
    ctr_d = torch.tensor(np.asarray(centers, dtype=np.float64), device=dev)
    xm_d = torch.empty_like(xm_h, device=dev)
    fb_d = torch.empty_like(fb_h, device=dev)
    counts = torch.tensor(np.diff(w.offsets), device=dev)
    pl = dimer_params(delta=p.delta, rot_tol=p.rot_tol, force_tol=p.force_tol,
                      max_iter=min(p.max_iter, LEARNED_MAX_ITER), patience=LEARNED_PATIENCE)
    ms, res, n_fb, n_noprop, prop_ms = [], None, 0, 0, []
    x_out = torch.empty(xm_h.shape, dtype=xm_h.dtype).pin_memory()     # positions read back
    for rep in range(1 + args.saddle_reps):
        barrier()
        torch.cuda.synchronize(dev)
        e0, e1, ep, el = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        xm_d.copy_(xm_h, non_blocking=True)
        fb_d.copy_(fb_h, non_blocking=True)
        disp, _, chosen = prop.propose(w, xm_d, P.proposal_params(group=args.walkers_per_system,
                                                                   region=SADDLE_REGION, scale=args.proposal_scale),
                                       seed=4242, counter=0, fallback=fb_d, center=ctr_d)
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
        uniq = unique_saddles(w, x_d, res, args.walkers_per_system, dev, stream)
        x_out.copy_(x_d, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if rep > 0:
            ms.append(e0.elapsed_time(e1))
            prop_ms.append((e0.elapsed_time(ep), ep.elapsed_time(el), el.elapsed_time(e1), fail_status))
        n_fb = int(fail.sum())
        n_noprop = int((chosen < 0).sum())
    return ms, res, x_out, m_d.cpu(), n_fb, n_noprop, prop_ms, proposal_kernels(w, prop, xm_d, dev, stream,
                                                                                  ctr_d), uniq


def proposal_kernels(w, prop, x, dev, stream, center, reps=5):
    """CUDA-event times of the proposal's parts on the walkers' minima (best of reps): the
    candidate rows (atoms within SADDLE_REGION of the centre) and their descriptors (one force
    call on the walkers' batch + the descriptor kernel on those rows), each model's forward
    (tcgen05) on them, the seeding kernel; and, as a tensor-core measurement, one model's
    forward over every atom of the set."""
    import torch
    from akmc_b200 import proposals as P
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    best = {}
    begin, box = w.device_geometry()
    all_desc = w.descriptors(x)
    for _ in range(reps):
        e = [ev() for _ in range(7)]
        e[0].record(stream)
        rows = P.region_rows(begin, x, box, center, SADDLE_REGION + 0.5)
        desc, basis = w.descriptors(x, with_basis=True, rows=rows)
        e[1].record(stream)
        pred = prop.direction.predict(desc, basis)
        e[2].record(stream)
        score = prop.score.predict(desc)
        e[3].record(stream)
        pf = torch.zeros((x.shape[0], 3), dtype=torch.float32, device=dev)
        sf = torch.zeros_like(pf)
        pf[rows.long()] = pred
        sf[rows.long()] = score
        P.seeds(begin, x, box, pf, sf, P.proposal_params(region=SADDLE_REGION), center=center)
        e[4].record(stream)
        e[5].record(stream)
        prop.score.predict(all_desc)
        e[6].record(stream)
        torch.cuda.synchronize(dev)
        t = [e[k].elapsed_time(e[k + 1]) for k in (0, 1, 2, 3, 5)]
        for name, v in zip(("descriptors_ms", "direction_forward_ms", "score_forward_ms", "seeds_ms",
                            "full_set_forward_ms"), t):
            best[name] = min(best.get(name, 1e30), v)
        best["rows"] = int(rows.numel())
    n_all = int(w.n_total)
    best["full_set_rows"] = n_all
    best["forward_tflops"] = 2.0 * n_all * (64 * 128 + 2 * 128 * 128 + 128 * 3) / (best["full_set_forward_ms"] * 1e-3) / 1e12
    return best


def run_saddles(args, world, rank, dev, d, barrier):
    """Batched FIRE + Dimer walkers (akmc_walkers_*) on the batched-walker configuration."""
    import torch
    from akmc_b200 import Field, PREC_FP64, PREC_MIXED
    from akmc_b200.walkers import Walkers, dimer_params, fire_params

    systems, centers = saddle_workload(rank, args.saddle_walkers, args.walkers_per_system)
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
        uniq = unique_saddles(w, x_d, res, args.walkers_per_system, dev, stream)
        x_out.copy_(x_d, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if rep > 0:
            ms.append(e0.elapsed_time(e1))
    from akmc_b200 import shard
    secs = shard.max_over_ranks(sum(ms) / 1e3, device=dev)
    conv = res["status"] == 1
    n_conv = int(conv.sum())
    n_uniq = int(uniq.sum())
    u_all = shard.sum_over_ranks(n_uniq, device=dev)
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
           "unique": n_uniq, "unique_fraction": n_uniq / max(n_conv, 1),
           "unique_saddles_per_s": u_all * len(ms) / secs, "walkers_per_system": args.walkers_per_system,
           "reps": len(ms), "s_per_search_batch": secs / len(ms),
           "force_calls": calls, "atom_forces_per_s": world * atom_forces * len(ms) / secs,
           "iters_mean": float(res["iters"].mean()), "iters_max": int(res["iters"].max()),
           "barrier_eV_median": float(np.median(barriers)) if n_conv else None,
           "relax_s": relax_s, "work_items_per_size_class": w.tuning(1),
           "dimer": {"delta_A": SADDLE_DELTA, "rot_tol": SADDLE_ROT_TOL,
                                        "force_tol": p.force_tol, "max_iter": p.max_iter},
           "timing": "device events around H2D of seeds, the batched search, the duplicate-saddle "
                     "removal and D2H of positions (pinned host buffers both ways)",
           "config": f"{len(systems)} uneven FCC walkers (4^3..10^3 cells, 1-3 vacancies, sigma 0.02 A): "
                     f"{len(systems) // args.walkers_per_system} systems x {args.walkers_per_system} searches "
                     f"from different random starts; unique = converged and not within {UNIQUE_E_TOL} eV and "
                     f"{UNIQUE_D_TOL} A (every atom) of an earlier saddle of the same system"}
    if not args.no_learned:
        prop, tinfo = train_proposer(f, rank, dev, p, args.saddle_walkers, args.train_saddles)
        lms, lres, lx, lm, n_fb, n_noprop, prop_ms, pk, luniq = run_learned(args, w, prop, xmin, seeds, emin, p,
                                                                        dev, stream, barrier, centers)
        lsecs = shard.max_over_ranks(sum(lms) / 1e3, device=dev)
        lconv = lres["status"] == 1
        l_all = shard.sum_over_ranks(int(lconv.sum()), device=dev)
        lu_all = shard.sum_over_ranks(int(luniq.sum()), device=dev)
        p_all = shard.sum_over_ranks(n_conv, device=dev)
        lb = lres["energy"][lconv] - emin[lconv]
        pb = barriers
        out["learned"] = {
            "value": l_all * len(lms) / lsecs, "unit": "saddles/s", "converged": int(lconv.sum()),
            "unique": int(luniq.sum()), "unique_fraction": int(luniq.sum()) / max(int(lconv.sum()), 1),
            "unique_saddles_per_s": lu_all * len(lms) / lsecs,
            "vs_plain_unique": (lu_all * len(lms) / lsecs) / (u_all * len(ms) / secs) if u_all else None,
            "s_per_search_batch": lsecs / len(lms),
            "propose_ms": float(np.mean([q[0] for q in prop_ms])),
            "learned_pass_ms": float(np.mean([q[1] for q in prop_ms])),
            "fallback_pass_ms": float(np.mean([q[2] for q in prop_ms])),
            "learned_pass_failures_by_status": prop_ms[-1][3],
            "fallback_walkers": n_fb, "walkers_without_proposal": n_noprop,
            "learned_max_iter": LEARNED_MAX_ITER, "learned_patience": LEARNED_PATIENCE,
            "force_calls": int(lres["force_calls"].sum()),
            "iters_mean": float(lres["iters"].mean()), "iters_max": int(lres["iters"].max()),
            "barrier_eV_pct_5_50_95": [float(v) for v in np.percentile(lb, [5, 50, 95])] if len(lb) else None,
            "plain_barrier_eV_pct_5_50_95": [float(v) for v in np.percentile(pb, [5, 50, 95])] if len(pb) else None,
            "vs_plain": (l_all * len(lms) / lsecs) / (p_all * len(ms) / secs) if p_all else None,
            "training": tinfo, "proposal_kernels": pk,
            "timing": "device events around H2D of minima and fallback seeds, descriptors, both "
                      "models, seeding kernel, the batched search, the fallback pass and D2H of "
                      "positions (pinned host buffers both ways; fallback_pass_ms includes the "
                      "read-back); training (plain searches of other sets) is outside"}
    if rank == 0 and not args.no_barrier_check:
        arms = [("plain", x_out.numpy(), m_d.cpu().numpy(), res)]
        if "learned" in out:
            arms.append(("learned", lx.numpy(), lm.numpy(), lres))
        errs = barrier_checks(pot, systems, w.offsets, xmin, emin, arms, args.barrier_walkers_per_class,
                              args.cpu_procs or cpu_cores())
        out["barrier_error_vs_fp64_oracle_eV"] = errs["plain"]
        if "learned" in out:
            out["learned"]["barrier_error_vs_fp64_oracle_eV"] = errs["learned"]
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
# the ionic configuration's 16 Dimer searches: mixed against FP64 and the FP64 oracle
# ------------------------------------------------------------------------------------
def run_ionic_searches(args, dev, d):
    """16 Dimer searches on the ionic configuration (the 998-ion rocksalt, 10 A cutoff,
    eta 0.3), started on the nearest-neighbour hops into its two vacancies, in the mixed
    precision (FP32 pair terms, FP64 accumulation) and all-FP64 from the same starts.  Per
    search pair that reaches the same saddle: the barrier difference; at every mixed saddle:
    energy, force and barrier errors against the FP64 oracle (the C restatement) at the same
    positions."""
    import torch
    import oracle
    from akmc_b200 import Field, PREC_FP64, PREC_MIXED
    from akmc_b200 import configs as cf
    from akmc_b200.walkers import Walkers, dimer_params, fire_params
    s = cf.rocksalt_schottky_system(5, 4.21, 0.03, 4321)
    pot = os.path.join(d, "ion.pot")
    nw = 16
    out, runs = {}, {}
    for prec in (PREC_FP64, PREC_MIXED):
        f = Field().readPotential(pot).setup(s.lat, None, s.n)
        f.setPrecision(prec)
        one = Walkers.from_systems(f, [s])
        x = torch.tensor(s.pos, device=dev)
        r = one.relax(x, fire_params(force_tol=1e-4, norm_tol=1e-6, max_iter=4000))   # the barriers subtract it
        one.close()
        xmin, emin = x.cpu().numpy(), float(r["energy"][0])
        if prec == PREC_FP64:
            seeds = cf.rocksalt_hop_starts(xmin, s.labels, s.box, per_site=nw // 2, seed=31)
            x_ref = xmin
        w = Walkers.from_systems(f, [s] * nw)
        pos = torch.tensor(np.concatenate([x_ref + q for q in seeds]), device=dev)
        mode = torch.tensor(np.concatenate(list(seeds)), device=dev)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        res = w.dimer(pos, mode, dimer_params(max_iter=600, force_tol=1e-3))
        torch.cuda.synchronize(dev)
        runs[prec] = (res, emin, xmin, pos.cpu().numpy(), time.perf_counter() - t0, f)
        w.close()
    (r64, e64, xm64, x64, t64, _), (r32, e32, xm32, x32, t32, f32) = runs[PREC_FP64], runs[PREC_MIXED]
    n = s.n
    same, dbar = 0, []
    for k in range(nw):
        if r64["status"][k] != 1 or r32["status"][k] != 1:
            continue
        dd = x64[k * n:(k + 1) * n] - x32[k * n:(k + 1) * n]
        dd -= s.box * np.rint(dd / s.box)
        if np.abs(dd).max() > 0.05:
            continue
        same += 1
        dbar.append(abs((r64["energy"][k] - e64) - (r32["energy"][k] - e32)))
    # the mixed saddles against the FP64 oracle at the same positions (oracle: the checker)
    S = oracle.ionic_setup(pot, s.lat)
    Eo_min = oracle.ionic_forces(S, xm32, s.charge, s.labels, s.lat)[0]["total"]
    e_rel, f_err, b_err, bars = [], [], [], []
    for k in range(nw):
        if r32["status"][k] != 1:
            continue
        xs = x32[k * n:(k + 1) * n]
        E, F, _ = f32.forces(xs, s.labels, s.charge)
        Eo, Fo, _ = oracle.ionic_forces(S, xs, s.charge, s.labels, s.lat)
        e_rel.append(abs(E["total"] - Eo["total"]) / abs(Eo["total"]))
        f_err.append(float(np.abs(F - Fo).max()))
        b_err.append(abs((r32["energy"][k] - e32) - (Eo["total"] - Eo_min)))
        bars.append(r32["energy"][k] - e32)
    out = {"config": "rocksalt 5x5x5 Schottky (998 ions), 10 A cutoff, eta 0.3; 16 Dimer searches "
                     "from the nearest-neighbour hops into the cation and anion vacancies (1.0 A along "
                     "the hop, N(0, 0.02 A) within 4 A), delta 0.005 A, saddle at max|F| < 1e-3 eV/A",
           "converged_mixed": int((r32["status"] == 1).sum()), "converged_fp64": int((r64["status"] == 1).sum()),
           "same_saddle": same,
           "barrier_mixed_vs_fp64_max_eV": max(dbar) if dbar else None,
           "vs_fp64_oracle_at_mixed_saddles": {
               "energy_rel_max": max(e_rel) if e_rel else None,
               "force_max_eV_per_A": max(f_err) if f_err else None,
               "barrier_max_eV": max(b_err) if b_err else None, "saddles": len(e_rel),
               "bars": {"energy_rel": 1e-6, "force_eV_per_A": 1e-5, "barrier_eV": 1e-3}},
           "barrier_eV_range": [min(bars), max(bars)] if bars else None,
           "search_s": {"mixed": t32, "fp64": t64},
           "saddles_per_s_mixed": int((r32["status"] == 1).sum()) / t32}
    return out


# ------------------------------------------------------------------------------------
# the AKMC loop at scale (--akmc-steps per arm)
# ------------------------------------------------------------------------------------
def run_akmc(args, rank, world, dev, d):
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
    from akmc_b200.walkers import dimer_params
    s = cf.fcc_cluster_system(20, seed=2026 + rank)
    f = Field().readPotential(os.path.join(d, "eam.pot")).setup(s.lat, None, s.n)
    f.setPrecision(PREC_MIXED)
    find = cf.fcc_vacancy_finder(20, 3.615)
    ra = args.akmc_active_radius
    out = {"config": f"FCC 20^3 ({s.n} atoms), 6-vacancy cluster + 10 isolated vacancies, "
                     f"{args.akmc_walkers} walkers per KMC step, nu 1e13 1/s, 600 K; "
                     + (f"walkers over local regions (free radius {ra} A, fixed shell of two cutoffs + 1 A)"
                        if ra > 0 else "every walker a replica of the crystal"),
           "dimer": {"delta_A": 0.01, "rot_tol": 0.1, "force_tol": args.akmc_search_tol},
           "polish": {"force_tol": args.akmc_polish_tol, "window_kT": 30},
           "basin2_region_fire_tol": args.akmc_basin2_tol}
    check_pool = []
    out["learned_explore"] = args.akmc_explore
    out["basin2_unpolished"] = bool(args.akmc_basin2_unpolished)
    arms = [a for a in ("plain", "learned") if a in args.akmc_arms.split(",")]
    for arm in arms:
        proposer = P.Proposer(seed=rank) if arm == "learned" else None
        loop = AkmcLoop(f, s, find, n_walkers=args.akmc_walkers, seed=7 + rank, proposer=proposer,
                        proposal_threshold=0.0, explore=args.akmc_explore, active_radius=ra, keep_saddles=1,
                        dimer=dimer_params(force_tol=args.akmc_search_tol),
                        polish_tol=args.akmc_polish_tol, basin2_tol=args.akmc_basin2_tol,
                        basin2_unpolished=bool(args.akmc_basin2_unpolished))
        steps = []
        for _ in range(args.akmc_steps):
            torch.cuda.synchronize(dev)
            t = time.perf_counter()
            rec = loop.step()
            torch.cuda.synchronize(dev)
            dt = time.perf_counter() - t
            steps.append({"s": dt, "converged": rec.n_saddles, "unique": rec.n_unique,
                          "dimer_force_calls": rec.force_calls, "atoms_per_walker": rec.atoms_per_walker,
                          "atom_forces": rec.atom_forces, "polished": rec.polished,
                          "polish_iters_mean": rec.polish_iters, "recycled": rec.recycled,
                          "recycled_iters_mean": rec.recycled_iters, "recycled_converged": rec.recycled_converged,
                          "unpolished": rec.unpolished, "basin2_rejected": rec.basin2_rejected,
                          "basin2_rejected_unpolished": rec.basin2_rejected_unpolished,
                          "stage_s": {k: round(v, 4) for k, v in rec.stage_s.items()},
                          "learned": rec.learned, "fallback": rec.n_fallback, "barrier_eV": rec.barrier,
                          "kmc_dt_s": rec.dt, "total_rate_per_s": rec.total_rate})
            if len(steps) == 1:                # the first step's saddle against the FP64 oracle
                check_pool += [(arm, q) for q in loop.last_saddles]
        secs = sum(x["s"] for x in steps)
        out[arm] = {"steps": steps, "s_per_kmc_step": secs / max(len(steps), 1),
                    "converged_saddles_per_s": sum(x["converged"] for x in steps) / secs,
                    "unique_events_per_s": sum(x["unique"] for x in steps) / secs,
                    "dimer_atom_forces_per_s": sum(x["atom_forces"] for x in steps) / secs}
    # the reference's CPU force call on the same crystal, on the host cores: the atom-force
    # evaluations of a KMC step at that rate give the reference path's time for the same searches
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        procs = args.cpu_procs or cpu_cores()
        rate, kind, secs, _ = cpu_run("eam", d, procs, 0, 1, systems=[s])   # one call: ~14 s per process
        per_step = {arm: sum(x["atom_forces"] for x in out[arm]["steps"]) / max(len(out[arm]["steps"]), 1)
                    for arm in arms}
        out["cpu_reference"] = {"atom_forces_per_s": rate, "cores": procs, "kind": kind,
                                "sample": f"{procs} processes x 1 Field::calculateForces call on the "
                                          f"{s.n}-atom crystal ({secs:.1f} s)",
                                "s_per_kmc_step_estimate": {arm: v / rate for arm, v in per_step.items()},
                                "note": "the same atom-force evaluations per KMC step as each GPU arm, "
                                        "at the reference's measured rate (an estimate: a whole CPU KMC "
                                        "step at this scale would take hours)"}
    # the loop's barriers against the FP64 oracle on the same (region) positions
    if rank == 0 and check_pool:
        from oracle import walkers as W
        errs = {}
        for arm, (sysq, xm, xs, bar) in check_pool:
            eo = W.EamOracle(os.path.join(d, "eam.pot"), sysq.lat, sysq.labels)
            errs.setdefault(arm, []).append(abs(bar - (eo(xs)[1] - eo(xm)[1])))
        for arm, e in errs.items():
            out[arm]["barrier_error_vs_fp64_oracle_eV"] = {"max": max(e), "saddles": len(e), "bar": 1e-3}
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


# Algorithmic FLOPs of the compute-form roofline, per unit (counts of the arithmetic the
# method needs, a transcendental (erfc, exp, sincos) counted as 20, a division or square root as
# 4): ionic real space 45 per unordered pair inside the cutoff; reciprocal force 36 per (atom,
# k-vector) (the phase and the three force components); structure factor 24 per (atom,
# k-vector); EAM 35 per unordered pair and pass.
FLOPS_PER_PAIR = {"ionic_force": 45.0, "eam_density": 35.0, "eam_force": 35.0}
FLOPS_PER_ATOM_K = {"ionic_force": 36.0, "structure_factor": 24.0}


def algorithmic_flops(kernel, n_atoms, nsys, nk, pairs_per_atom):
    """FLOPs per launch: half the mean neighbour count (unordered pairs) per atom times the
    per-pair count, plus the per-(atom, k-vector) count for every atom and k-vector."""
    per_atom = 0.5 * pairs_per_atom * FLOPS_PER_PAIR.get(kernel, 0.0) + nk * FLOPS_PER_ATOM_K.get(kernel, 0.0)
    return n_atoms * per_atom


def mean_neighbours(systems, rc, sample=2):
    """Mean count of partners inside rc (minimum image) over the first atoms' systems."""
    counts = []
    for s in systems[:sample]:
        L = np.asarray(s.box, dtype=np.float64)
        m = min(len(s.pos), 256)                      # the first atoms against all
        d = s.pos[:m, None, :] - s.pos[None, :, :]
        d -= L * np.rint(d / L)
        r2 = (d * d).sum(-1)
        r2[np.arange(m), np.arange(m)] = np.inf
        counts.append(float((r2 <= rc * rc).sum(1).mean()))
    return float(np.mean(counts))


def vector_peaks(dev):
    """Nominal FP32 and FP64 vector peaks (TFLOP/s): SMs x lanes per SM (128 FP32, 64 FP64)
    x 2 (fused multiply-add) x the maximum SM clock."""
    import torch
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    peaks, _ = measured_peaks()
    mhz = float(peaks.get("sm_max_mhz", 1965.0))
    return sms * 128 * 2 * mhz * 1e6 / 1e12, sms * 64 * 2 * mhz * 1e6 / 1e12, sms, mhz


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
    # sustained soak: the same steps (L2 flushed between them) for at least args.soak_s of
    # device time right before the timed steps, with the clock sampler running through both,
    # so the clock record covers the kernels under sustained load
    probe0, probe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    probe0.record(stream)
    for _ in range(5):
        flush.zero_()
        b.forces_(pos, force, energy, status, stream.cuda_stream)
    probe1.record(stream)
    torch.cuda.synchronize(dev)
    soak_steps = max(1, int(math.ceil(args.soak_s / max(probe0.elapsed_time(probe1) / 5e3, 1e-6))))
    t = torch.tensor([soak_steps], dtype=torch.int64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    soak_steps = int(t.item())
    soak_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * soak_steps)]
    barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(clocks_path) as cs:
        for k in range(soak_steps):
            flush.zero_()
            soak_ev[2 * k].record(stream)
            b.forces_(pos, force, energy, status, stream.cuda_stream)
            soak_ev[2 * k + 1].record(stream)
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            b.forces_(pos, force, energy, status, stream.cuda_stream)
            ends[k].record(stream)
        torch.cuda.synchronize(dev)
        barrier()
    dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    soak_ms = sum(soak_ev[2 * k].elapsed_time(soak_ev[2 * k + 1]) for k in range(soak_steps))
    t = torch.tensor([soak_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    soak_ms = float(t.item())
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
    npair = mean_neighbours(systems, f.cutoff)
    flops = algorithmic_flops(dom, n_total, len(nat), nk, npair)
    p32, p64, sms, mhz = vector_peaks(dev)
    tflops = flops / avg_s / 1e12
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "peak_source": peak_kind,
                "traffic": tr, "alg_bytes_per_launch": alg, "launch_ms": avg_s * 1e3,
                "compute": {"achieved": tflops, "unit": "TFLOP/s", "alg_flops_per_launch": flops,
                            "pairs_per_atom": npair,
                            "fp32_peak": p32, "frac_fp32": tflops / p32,
                            "fp64_peak": p64, "frac_fp64": tflops / p64,
                            "peak_source": f"nominal: {sms} SMs x 128 FP32 (64 FP64) lanes x 2 x {mhz:.0f} MHz",
                            "count": "ionic real space 45 FLOP per unordered pair inside the cutoff, "
                                     "36 per (atom, k-vector) reciprocal force; transcendentals as 20"},
                "note": "HBM fraction on compulsory bytes only (neighbour re-reads from shared memory/L1/L2 "
                        "not counted): the kernel is issue/FP32-pipe bound, not HBM bound; the compute "
                        "form beside it; pipe counters in profiles/"}

    line = {"metric": "atom-forces/s", "value": value, "unit": "atom-forces/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.fp64 else "f64+f32", "data": "synthetic",
            "config": dict(workload_config(args, nk=nk), home_chunk=home_chunk),
            "roofline": roofline,
            "kernels": {k: {"ms_per_launch": v[0] / v[1], "launches": v[1]} for k, v in ktimes.items()},
            "gpu_launches": b.launches * args.steps,
            "sustained": {"value": world * n_total * soak_steps / (soak_ms / 1e3), "unit": "atom-forces/s",
                          "steps": soak_steps, "device_s": soak_ms / 1e3,
                          "note": "the same steps right before the timed ones, L2 flushed between "
                                  "steps; the clock record covers both"},
            "e2e": {"value": e2e_value, "unit": "atom-forces/s",
                    "h2d_bytes_per_step": n_total * 3 * 8,
                    "d2h_bytes_per_step": n_total * 3 * 8 * 2 + len(nat) * (5 * 8 + 4)},
            "clocks": cs.summary(None if world == 1 else local_rank)}

    if not args.no_saddles:
        line["saddles"] = run_saddles(args, world, rank, dev, d, barrier)
    if rank == 0 and not args.no_ionic_searches:
        line["ionic_searches"] = run_ionic_searches(args, dev, d)
    if args.akmc_steps > 0:
        line["akmc"] = run_akmc(args, rank, world, dev, d)
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
    ap.add_argument("--soak-s", type=float, default=1.5,
                    help="device seconds of sustained steps before the timed steps (clock record)")
    ap.add_argument("--cpu-procs", type=int, default=0)
    ap.add_argument("--no-saddles", action="store_true", help="skip the batched Dimer measurement")
    ap.add_argument("--skin", type=float, default=0.0,
                    help="EAM neighbour-list skin (A) of the force-path batch; every timed step then "
                         "reuses the lists of the first call (positions do not move between steps)")
    ap.add_argument("--saddle-reps", type=int, default=2, help="timed batched searches")
    ap.add_argument("--saddle-walkers", type=int, default=512,
                    help="walkers of the saddle measurement (the configuration has 512; fewer for profiling)")
    ap.add_argument("--akmc-steps", type=int, default=6,
                    help="also run the AKMC loop at scale (32 000-site crystal) for this many KMC steps "
                         "per arm (about 3 s a step; 0: off)")
    ap.add_argument("--akmc-walkers", type=int, default=1024, help="walkers per KMC step of --akmc-steps")
    ap.add_argument("--akmc-arms", default="plain,learned", help="AKMC loop arms to run (comma list)")
    ap.add_argument("--akmc-basin2-unpolished", type=int, default=1,
                    help="1: relax the region basin 2 of saddles beyond the polish window too; 0: table them unchecked")
    ap.add_argument("--akmc-explore", type=float, default=0.0,
                    help="learned arm: fraction of each site's walkers started from random seeds")
    ap.add_argument("--akmc-active-radius", type=float, default=6.0,
                    help="free radius (A) of the --akmc-steps walkers' local regions (0: crystal replicas)")
    ap.add_argument("--akmc-search-tol", type=float, default=1e-3,
                    help="max|F| tolerance of the loop's region searches, eV/A")
    ap.add_argument("--akmc-basin2-tol", type=float, default=0.02,
                    help="FIRE tolerance of the region relaxations that tell which basin a saddle leads to, eV/A")
    ap.add_argument("--akmc-polish-tol", type=float, default=2.5e-3,
                    help="max|F| tolerance of the crystal polish of local-region saddles, eV/A")
    ap.add_argument("--no-ionic-searches", action="store_true",
                    help="skip the ionic configuration's 16 Dimer searches (mixed vs FP64)")
    ap.add_argument("--no-barrier-check", action="store_true",
                    help="skip the host-side barrier checks of sampled saddles")
    ap.add_argument("--barrier-walkers-per-class", type=int, default=2,
                    help="converged walkers per size class checked against the FP64 oracle and the reference ART")
    ap.add_argument("--walkers-per-system", type=int, default=4,
                    help="consecutive walkers searching one system from different starts (unique saddles)")
    ap.add_argument("--train-saddles", type=int, default=10000,
                    help="usable plain saddles (other walker sets) the learned proposal is trained on")
    ap.add_argument("--proposal-scale", type=float, default=1.0,
                    help="learned arm: the chosen atom's start as this fraction of its predicted saddle displacement")
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
