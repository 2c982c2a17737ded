"""Adaptive KMC on the GPU: batched saddle searches, the FP64 event table and the KMC step.

One iteration of the reference's loop (kmc/KineticMonteCarlo.cpp:20-275, with
calculateRateConstant :277-611 farming the searches over MPI ranks) becomes:

1. W Dimer walkers from the current minimum (basin 1), each seeded with a random local
   displacement around a defect site (akmc_walkers_dimer, one batched call);
2. for every converged saddle, basin 2: FIRE from the saddle nudged along the mode away
   from basin 1 (akmc_walkers_relax, one batched call);
3. the event table in FP64 on the device: duplicate saddles removed (akmc_events_dedup),
   events whose basin 2 is basin 1 dropped, rates nu exp(-E_a / k_B T) with
   E_a = E_saddle - E_min, the reference's selection and dt = -ln(u2)/R (akmc_kmc_select)
   with seeded Philox uniforms (akmc_kmc_uniforms);
4. basin 1 <- the chosen event's basin 2, time += dt.

The reference keeps events across steps (recycling, superbasins); this loop rebuilds the
table every step.

With a ``proposer`` (akmc_b200.proposals.Proposer) the loop learns where searches should
start: the converged saddles of every step become training rows, the models are refitted,
and from then on walkers start from akmc_proposal_seeds (each walker draws its own candidate
atom, so the walkers of one basin spread over the symmetry-equivalent hops); a walker without
a proposal, or whose learned search does not converge within ``learned_max_iter``, searches
again from its random seed (the reference's rule).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import configs as cf
from . import kmc
from .walkers import CONVERGED, Walkers, dimer_params, fire_params


@dataclass
class KmcRecord:
    step: int
    time: float
    dt: float
    chosen: int
    barrier: float
    n_saddles: int
    n_unique: int
    n_events: int
    total_rate: float
    energy: float
    force_calls: int = 0          # system force evaluations of this step's searches
    learned: bool = False         # walkers started from learned proposals
    n_fallback: int = 0           # learned walkers searched again from their random seeds


@dataclass
class AkmcLoop:
    """A KMC trajectory of one system on one GPU."""
    field: object                 # akmc_b200.Field, set up
    system: cf.System             # start configuration (relaxed on the first step)
    centers: object               # callable: basin-1 positions -> (k, 3) seeding centres
    n_walkers: int = 32
    prefactor: float = 1.0e13
    temperature: float = 600.0
    seed: int = 1
    sigma: float = 0.1            # seeding displacement, A
    radius: float = 4.0           # seeding radius around a defect site, A
    dimer: object = None          # akmc_dimer_params (default: dimer_params(force_tol=1e-3))
    relax_tol: float = 1.0e-3     # FIRE max|F| tolerance of every minimum, eV/A
    e_tol: float = 1.0e-3         # duplicate saddles: energy tolerance, eV
    d_tol: float = 0.1            # ... and per-atom distance, A
    same_basin_tol: float = 0.2   # basin 2 within this of basin 1 for every atom: not an event
    proposer: object = None       # akmc_b200.proposals.Proposer: learn starting displacements
    min_rows: int = 8             # direction rows before the proposer is used
    learned_max_iter: int = 300   # a learned search not converged by then falls back
    proposal_threshold: float = 0.5   # candidate score relative to the region's best (0: every
                                      # eligible atom of the region is a candidate)
    history: list = field(default_factory=list)

    def __post_init__(self):
        import torch
        s = self.system
        self.dev = torch.device("cuda")
        self.W = Walkers.from_systems(self.field, [s] * self.n_walkers)
        self.one = Walkers.from_systems(self.field, [s])
        self.box = np.asarray(s.box, dtype=np.float64)
        self.time = 0.0
        self.iteration = 0            # KMC steps taken (seeds and uniforms are keyed by it)
        self.pos = None
        self.energy = None
        # KMC rates need barriers to well under a meV: saddles at max|F| < 1e-3 eV/A
        self.dimer = self.dimer or dimer_params(force_tol=1e-3)
        self._rows = {"direction": [], "score": []}
        self._fitted = False
        self._fit_rows = 0

    def _relax_basin(self, x):
        import torch
        t = torch.tensor(x, device=self.dev)
        r = self.one.relax(t, fire_params(force_tol=self.relax_tol))
        return t.cpu().numpy(), float(r["energy"][0])

    def _wrapdiff(self, a, b):
        d = a - b
        return d - self.box * np.rint(d / self.box)

    def step(self) -> KmcRecord:
        import torch
        s = self.system
        n = s.n
        if self.pos is None:
            self.pos, self.energy = self._relax_basin(s.pos)
        x1, e1 = self.pos, self.energy
        # 1. seeds around the defect sites of basin 1 (walker k uses site k mod #sites)
        sites = np.atleast_2d(self.centers(x1))
        rng_seed = self.seed * 1_000_003 + self.iteration
        seeds = np.concatenate([
            cf.local_displacements(x1, self.box, sites[k % len(sites)], 1,
                                   self.sigma, self.radius, seed=rng_seed * 997 + k)[0]
            for k in range(self.n_walkers)])
        learned = self.proposer is not None and self._fitted
        if learned:
            centres = np.stack([sites[k % len(sites)] for k in range(self.n_walkers)])
            res, xs, modes = self._learned_searches(x1, seeds, centres)
        else:
            xs = torch.tensor(np.tile(x1, (self.n_walkers, 1)) + seeds, device=self.dev)
            modes = torch.tensor(seeds, device=self.dev)
            res = self.W.dimer(xs, modes, self.dimer)
        conv = res["status"] == CONVERGED
        xs_h = xs.cpu().numpy()
        modes_h = modes.cpu().numpy()
        # 2. basin 2 of every converged saddle: nudge along the mode away from basin 1
        idx = np.where(conv)[0]
        e_s = res["energy"]
        e2 = np.full(self.n_walkers, np.nan)
        x2 = np.zeros_like(xs_h)
        if len(idx):
            # the walker set itself relaxes the converged walkers' nudged saddles
            starts = xs_h.copy()
            for k in idx:
                sl = slice(k * n, (k + 1) * n)
                away = np.sign(np.sum(modes_h[sl] * self._wrapdiff(xs_h[sl], x1))) or 1.0
                starts[sl] = xs_h[sl] + away * 0.1 * modes_h[sl]
            t = torch.tensor(starts, device=self.dev)
            rb = self.W.relax_subset(t, torch.tensor(conv.astype(np.int32), device=self.dev),
                                     fire_params(force_tol=self.relax_tol))
            tb = t.cpu().numpy()
            for k in idx:
                if rb["status"][k] == CONVERGED:
                    x2[k * n:(k + 1) * n] = tb[k * n:(k + 1) * n]
                    e2[k] = rb["energy"][k]
        # 3. the event table on the device
        usable = conv & np.isfinite(e2)
        for k in np.where(usable)[0]:
            if np.all(np.sqrt((self._wrapdiff(x2[k * n:(k + 1) * n], x1) ** 2).sum(1)) < self.same_basin_tol):
                usable[k] = False                        # fell back into basin 1
        t = lambda a, dt=None: torch.tensor(a, device=self.dev, dtype=dt)
        group = t(np.zeros(self.n_walkers, np.int32))
        begin = t(np.arange(self.n_walkers, dtype=np.int64) * n)
        nat = t(np.full(self.n_walkers, n, np.int32))
        boxes = t(np.tile(self.box, (self.n_walkers, 1)))
        es_d = t(e_s.astype(np.float64))
        dup = kmc.dedup(group, t(usable.astype(np.int32)), es_d, t(xs_h), begin, nat, boxes,
                        self.e_tol, self.d_tol).cpu().numpy()
        unique = usable & (dup < 0)
        u = kmc.uniforms(self.seed, self.iteration, 2)    # one Philox block per KMC step
        st, rate, cum = kmc.select(es_d, t(np.full(self.n_walkers, e1)), t(unique.astype(np.int32)),
                                   self.prefactor, self.temperature, u)
        rec = KmcRecord(step=self.iteration, time=self.time, dt=st["dt"], chosen=st["chosen"],
                        barrier=st["barrier"], n_saddles=int(conv.sum()), n_unique=int(unique.sum()),
                        n_events=int(st["n_usable"]), total_rate=st["total_rate"], energy=e1,
                        force_calls=int(res["force_calls"].sum()), learned=learned,
                        n_fallback=self._n_fallback if learned else 0)
        if self.proposer is not None:
            self._learn(x1, xs_h, usable & (e_s - e1 < 5.0))
        # 4. move to the chosen basin 2
        if st["chosen"] >= 0:
            k = st["chosen"]
            self.pos = x2[k * n:(k + 1) * n].copy()
            self.energy = float(e2[k])
            self.time += st["dt"]
            rec.time = self.time
        # the event table of this step, kept for inspection
        self.last_table = dict(e_saddle=e_s.copy(), e_min=e1, unique=unique.copy(), dup=dup,
                               status=res["status"].copy(), e_basin2=e2, u=u.cpu().numpy(),
                               rate=rate.cpu().numpy(), cum=cum.cpu().numpy())
        self.history.append(rec)
        self.iteration += 1
        return rec

    # --- learned proposals
    def _learned_searches(self, x1, seeds, centres):
        """Searches from the proposer's starting displacements, then from the random seeds
        for the walkers that have none or did not converge.  The walkers are replicas of one
        basin: descriptors and predictions are computed once and broadcast; each walker draws
        its own candidate atom among those within ``radius`` of its seeding centre (its local
        region, as its random seed)."""
        import torch
        from . import proposals as P
        W, n = self.n_walkers, self.system.n
        x1_one = torch.tensor(x1, device=self.dev)
        d, B = self.one.descriptors(x1_one, with_basis=True)
        pred, score = self.proposer.predict(d, B)
        x1_t = x1_one.repeat(W, 1)
        fb = torch.tensor(seeds, device=self.dev)
        begin, box = self.W.device_geometry()
        disp, _, chosen = P.seeds(begin, x1_t, box, pred.repeat(W, 1), score.repeat(W, 1),
                                  P.proposal_params(region=self.radius, threshold=self.proposal_threshold),
                                  seed=self.seed, counter=self.iteration,
                                  center=torch.tensor(centres, device=self.dev))
        chosen = chosen.cpu().numpy()
        rows = torch.tensor(np.repeat(chosen < 0, n), device=self.dev)[:, None]
        disp = torch.where(rows, fb, disp)
        xs = x1_t + disp
        modes = disp.clone()
        p = dimer_params(delta=self.dimer.delta, rot_tol=self.dimer.rot_tol, force_tol=self.dimer.force_tol,
                         max_iter=min(self.dimer.max_iter, self.learned_max_iter))
        res = self.W.dimer(xs, modes, p)
        fail = (res["status"] != CONVERGED) | (chosen < 0)
        self._n_fallback = int(fail.sum())
        self.last_learned = dict(chosen=chosen.copy(), status=res["status"].copy(), iters=res["iters"].copy())
        if fail.any():
            x2 = x1_t + fb
            m2 = fb.clone()
            r2 = self.W.dimer_subset(x2, m2, torch.tensor(fail.astype(np.int32), device=self.dev), self.dimer)
            calls = res["force_calls"] + r2["force_calls"] * fail
            res[fail] = r2[fail]
            res["force_calls"] = calls
            rows = torch.tensor(np.repeat(fail, n), device=self.dev)[:, None]
            xs = torch.where(rows, x2, xs)
            modes = torch.where(rows, m2, modes)
        return res, xs, modes

    def _learn(self, x1, xs_h, usable):
        """Training rows from this step's saddles; fit once there are min_rows of them, refit
        when they have grown by half since the last fit."""
        import torch
        from . import proposals as P
        n = self.system.n
        if not usable.any():
            return
        d, B = self.one.descriptors(torch.tensor(x1, device=self.dev), with_basis=True)
        d, B = d.cpu().numpy(), B.cpu().numpy()
        rng = np.random.default_rng(self.seed * 7919 + self.iteration)
        one = np.array([0, n])
        for k in np.where(usable)[0]:           # the walkers are replicas of basin 1
            r = P.hop_rows(d, B, x1, xs_h[k * n:(k + 1) * n], one, [self.box], np.array([True]), rng=rng)
            for key in self._rows:
                self._rows[key].append(r[key])
        rows = {k: tuple(np.concatenate(z) for z in zip(*v)) for k, v in self._rows.items()}
        nr = len(rows["direction"][0])
        if nr >= self.min_rows and nr >= 1.5 * self._fit_rows:
            self.proposer.fit(rows, seed=self.iteration)
            self._fitted = True
            self._fit_rows = nr

    # --- restart: the reference's restart/archive files (Basis::dumpBasis, Basis.cpp:592-649)
    def dump(self, stream, species_names, header=True, title="akmc_b200 basin"):
        """Append the current basin to a restart/archive stream.  The time written is the
        KMC time times the prefactor, as the reference writes it
        (kmc/KineticMonteCarlo.cpp:222-226)."""
        from . import basis
        s = cf.System(pos=self.pos, labels=self.system.labels, charge=self.system.charge,
                      lat=self.system.lat)
        basis.dump(stream, s, species_names, self.time * self.prefactor, self.energy,
                   self.iteration, title=title, header=header)

    def resume(self, path, species_names):
        """Continue from the last basin of a restart/archive file: positions, energy,
        iteration and time (the file's time / prefactor, kmc/KineticMonteCarlo.cpp:90)."""
        from . import basis
        b = basis.read_last(path, species_names)
        if b.n != self.system.n:
            raise ValueError("restart file holds a different number of atoms")
        self.pos = b.pos.copy()
        self.energy = b.meta["energy"]
        self.iteration = int(b.meta["iteration"])
        self.time = float(b.meta["time"]) / self.prefactor
