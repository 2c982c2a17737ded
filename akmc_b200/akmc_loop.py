"""Adaptive KMC on the GPU: batched saddle searches, the FP64 event table and the KMC step.

One iteration of the reference's loop (kmc/KineticMonteCarlo.cpp:20-275, with
calculateRateConstant :277-611 farming the searches over MPI ranks) becomes:

1. W Dimer walkers from the current minimum (basin 1), each seeded with a random local
   displacement around a defect site (akmc_walkers_dimer, one batched call);
2. for every converged saddle, basin 2: FIRE from the saddle nudged along the mode away
   from basin 1 (akmc_walkers_relax, one batched call);
3. the event table in FP64 on the device: duplicate saddles of one site removed
   (akmc_events_dedup), events whose basin 2 is basin 1 dropped, repeats across sites (and
   ranks) removed by the atoms the saddle moves and its energy, rates nu exp(-E_a / k_B T)
   with E_a = E_saddle - E_min, the reference's selection and dt = -ln(u2)/R
   (akmc_kmc_select) with seeded Philox uniforms (akmc_kmc_uniforms);
4. basin 1 <- the chosen event's basin 2, time += dt.

The reference keeps events across steps (recycling, superbasins); this loop rebuilds the
table every step.

With a ``proposer`` (akmc_b200.proposals.Proposer) the loop learns where searches should
start: the converged saddles of every step (on local regions, the distinct ones) become
training rows, the models are refitted, and from then on walkers start from
akmc_proposal_seeds (each walker draws its own candidate atom, so the walkers of one basin
spread over the symmetry-equivalent hops); a walker without a proposal, and the ``explore``
fraction of each site's walkers, start from their random seeds in the same pass; a walker
whose search does not converge within ``learned_max_iter`` searches again from its random
seed (the reference's rule).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import configs as cf
from . import kmc
from . import shard
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
    atoms_per_walker: int = 0     # atoms a walker's force calls evaluate (the region's, or the crystal's)
    atom_forces: float = 0.0      # atom-force evaluations of this step's searches (region and crystal)
    polished: int = 0             # local regions: unique saddles polished in the crystal
    polish_iters: float = 0.0     # ... their mean Dimer iterations
    recycled: int = 0             # ... of them started from the previous step's polished saddle
    unpolished: int = 0           # ... unique saddles left at their region barrier (beyond the polish window)
    recycled_iters: float = 0.0   # ... their mean Dimer iterations
    recycled_converged: int = 0   # ... and how many converged
    basin2_rejected: int = 0      # ... polished saddles whose region basin 2 did not converge or is basin 1
    basin2_rejected_unpolished: int = 0   # ... the same for the saddles beyond the polish window
    stage_s: dict = field(default_factory=dict)   # this rank's wall seconds by stage (device work synchronised)


@dataclass
class AkmcLoop:
    """A KMC trajectory of one system on one GPU per rank.

    With ``active_radius`` > 0 the searches run on local regions
    (akmc_b200.configs.local_region, the reference's active region of
    optim/SaddleSearch.cpp:15-354): each walker holds only the atoms within
    active_radius + 2 cutoffs + 1 A of its seeding site, those beyond active_radius frozen;
    energy differences and free-atom forces equal the crystal's, so barriers do too.  Without
    it every walker is a replica of the whole crystal.

    With ``world`` > 1 (torch.distributed initialised, one rank per GPU) the walkers are split
    into contiguous blocks over the ranks; each rank searches its block, the events' records
    are gathered by every rank (the reference's task farm, kmc/KineticMonteCarlo.cpp:352-464),
    every rank takes the same selection from the same seeded uniforms, and the rank that owns
    the chosen event broadcasts its basin 2 (the reference's MPI_Bcast of the chosen
    positions, kmc/KineticMonteCarlo.cpp:1338-1345)."""
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
    moved_tol: float = 0.4        # atoms displaced farther than this at a saddle identify its event (A)
    proposer: object = None       # akmc_b200.proposals.Proposer: learn starting displacements
    min_rows: int = 8             # direction rows before the proposer is used
    learned_max_iter: int = 300   # a learned search not converged by then falls back
    learned_patience: int = 40    # ... as does one whose max|F| has not fallen 2 % below its best in this many steps
    proposal_threshold: float = 0.5   # candidate score relative to the region's best (0: every
                                      # eligible atom of the region is a candidate)
    explore: float = 0.0          # learned steps: one walker in round(1 / explore) of each site
                                  # starts from its random seed all the same (0: none)
    active_radius: float = 0.0    # > 0: searches on local regions of this free radius (A)
    keep_saddles: int = 0         # converged saddles per step kept for inspection (last_saddles)
    polish_iter: int = 100        # local regions: Dimer steps of the crystal polish of each unique saddle
    polish_tol: float = 0.0       # ... and its max|F| tolerance (0: 2.5e-3 eV/A; the saddle energy
                                  # is then within ~1e-5 eV of the converged one)
    recycle: bool = True          # ... starting from the previous step's polished saddle of the same event
    basin2_tol: float = 0.02      # ... FIRE tolerance of the region relax that tells which basin a saddle leads to
    polish_window: float = 0.0    # ... polish only saddles within this of the lowest region barrier (0: 30 kT)
    basin2_unpolished: bool = True    # ... relax the basin 2 of saddles beyond the window too (False: table
                                      # them unchecked; a chosen one's basin 2 is found as for any other)
    world: int = 1                # ranks sharing the walkers (torch.distributed)
    rank: int = 0
    history: list = field(default_factory=list)

    def __post_init__(self):
        import torch
        s = self.system
        self.dev = torch.device("cuda")
        self.mine = shard.shard_indices(self.n_walkers, self.rank, self.world)
        self.W = None if self.active_radius > 0 else Walkers.from_systems(self.field, [s] * len(self.mine))
        self.one = Walkers.from_systems(self.field, [s])
        self.box = np.asarray(s.box, dtype=np.float64)
        self.time = 0.0
        self.iteration = 0            # KMC steps taken (seeds and uniforms are keyed by it)
        self.pos = None
        self.energy = None
        # KMC rates need barriers to well under a meV: saddles at max|F| < 1e-3 eV/A
        self.dimer = self.dimer or dimer_params(force_tol=1e-3)
        self._rows = {"direction": [], "score": []}
        self._n_dir = 0               # direction rows held (this rank)
        self._polish_cache = {}       # event key -> (row of _polish_prev, its moved atoms)
        self.polish_tol = self.polish_tol or 2.5e-3
        self.polish_window = self.polish_window or 30.0 * kmc.BOLTZMANN_EV * self.temperature
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

    def _region_minima(self, regions, sites):
        """Energies of the sites' regions at basin 1: one batched force call, each region in
        its own cell."""
        import torch
        sites = sorted(set(int(j) for j in sites))
        if not sites:
            return {}
        rs = [regions[j].system for j in sites]
        b = self.field.batch([r.n for r in rs], np.array([r.box for r in rs]), np.concatenate([r.labels for r in rs]),
                             np.concatenate([r.charge for r in rs]))
        force, energy, status = b.alloc()
        b.forces_(torch.tensor(np.concatenate([r.pos for r in rs]), device=self.dev), force, energy, status)
        e = energy[:, 0].cpu().numpy()
        st = status.cpu().numpy()
        b.close()
        if st.any():
            raise RuntimeError(f"region energies: status {st.tolist()}")
        return {j: float(e[k]) for k, j in enumerate(sites)}

    def _polish_walkers(self, k):
        """The crystal-replica walker set of the polish, kept across steps (grown as needed)."""
        Wp = getattr(self, "_wp", None)
        if Wp is None or Wp.W < k:
            if Wp is not None:
                Wp.close()
            Wp = Walkers.from_systems(self.field, [self.system] * (64 * ((k + 63) // 64))).skip_tuning()
            self._wp = Wp
        return Wp

    def _far_from_move(self, x1, idx):
        """The atoms idx are all farther than two cutoffs from every atom the last move displaced."""
        mp = getattr(self, "_moved_pos", None)
        if mp is None or len(mp) == 0:
            return True
        return len(_within(x1[idx], mp, self.box, 2.0 * self.field.cutoff)) == 0

    # --- one KMC step
    def step(self) -> KmcRecord:
        s = self.system
        if self.pos is None:
            self.pos, self.energy = self._relax_basin(s.pos)
        x1, e1 = self.pos, self.energy
        sites = np.atleast_2d(self.centers(x1))
        self._basin2 = {}
        self._saddle_c = {}
        self._stage = {}
        ev = self._search(x1, e1, sites)                 # this rank's walkers
        tab = gather_events(ev, self.world)              # every rank's, in walker order
        return self._select_and_move(tab, ev, x1, e1)

    def _seed(self, k):
        return (self.seed * 1_000_003 + self.iteration) * 997 + int(k)

    def _search(self, x1, e1, sites):
        """Searches of this rank's walkers (ids self.mine; walker k seeds at site k mod
        #sites) and their events: saddle and basin-2 energies of the crystal, basin 2's
        crystal positions (kept here until the selection), the moved-atom fingerprint of each
        saddle, duplicates of one site removed on the device (akmc_events_dedup).

        On local regions the searches run on the regions; the unique converged ones are then
        polished in the whole crystal (a batched Dimer from the region saddle mapped back, at
        most polish_iter steps), because the fixed shell of a region raises a hop's barrier
        (by 0.15 eV for a vacancy hop at a 6 A free radius): the event table holds crystal
        saddles only."""
        import torch
        clock = time.perf_counter
        t0 = clock()
        n_sites = len(sites)
        ids = self.mine
        m = len(ids)
        site_of = (ids % n_sites).astype(np.int32)
        local = self.active_radius > 0
        tt = lambda a, dt=None: torch.tensor(a, device=self.dev, dtype=dt)  # noqa: E731
        if local:
            # regions are crystal-dense spheres in mostly empty cells: size lists for the crystal
            if not getattr(self, "_list_density_set", False):
                self.field.set_list_density(self.system.n / float(np.prod(self.box)))
                self._list_density_set = True
            regions = {int(j): cf.local_region(x1, self.system.labels, self.system.charge, self.box, sites[j],
                                               self.active_radius, self.field.cutoff)
                       for j in np.unique(site_of)}
            subs = [regions[int(j)] for j in site_of]
            W = Walkers.from_systems(self.field, [r.system for r in subs],
                                     frozen=np.concatenate([r.frozen for r in subs])).skip_tuning()
            xmin = np.concatenate([r.system.pos for r in subs])
            self._stage["regions"] = clock() - t0
            centres = np.zeros((m, 3))                             # the site, in region coordinates
        else:
            subs = None
            W = self.W
            xmin = np.tile(x1, (m, 1))
            centres = np.stack([sites[j] for j in site_of])
        offs, boxes = W.offsets, W.boxes
        seeds = np.concatenate([
            cf.local_displacements(xmin[offs[q]:offs[q + 1]], boxes[q], centres[q], 1, self.sigma, self.radius,
                                   seed=self._seed(k))[0]
            for q, k in enumerate(ids)])
        if local:
            seeds[np.concatenate([r.frozen for r in subs]) == 1] = 0.0
        learned = self.proposer is not None and self._fitted
        if learned:
            k = int(round(1.0 / self.explore)) if self.explore > 0 else 0
            explore = ((ids // n_sites) % k == 0) if k else np.zeros(m, bool)
            res, xs, modes = self._learned_searches(W, xmin, seeds, centres, local, explore)
        else:
            xs = torch.tensor(xmin + seeds, device=self.dev)
            modes = torch.tensor(seeds, device=self.dev)
            res = W.dimer(xs, modes, self.dimer)
        xs_h = xs.cpu().numpy()
        modes_h = modes.cpu().numpy()
        self._stage["search"] = clock() - t0
        status = res["status"].astype(np.int32).copy()
        atom_forces = res["force_calls"].astype(np.float64) * np.diff(offs)
        calls = res["force_calls"].astype(np.int64).copy()
        if self.proposer is not None and not local:
            self._learn(W, xmin, xs_h, (status == CONVERGED) & (res["energy"] - e1 < 5.0))
        if local:
            # unique converged region saddles: of each site (positions, on the device), then across
            # sites (the crystal atoms the saddle moves, each with the direction it moves along
            # rounded to the lattice: twice the unit vector, each component to the nearest integer)
            conv_l = status == CONVERGED
            dup = kmc.dedup(tt(site_of), tt(conv_l.astype(np.int32)), tt(res["energy"].astype(np.float64)), tt(xs_h),
                            tt(offs[:-1].astype(np.int64)), tt(np.diff(offs).astype(np.int32)), tt(boxes),
                            self.e_tol, self.d_tol).cpu().numpy()
            keep, keys, seen = [], [], set()
            for q in np.where(conv_l & (dup < 0))[0]:
                sl = slice(offs[q], offs[q + 1])
                d = _wrap(xs_h[sl] - xmin[sl], boxes[q])
                mv = np.where(np.sqrt((d * d).sum(1)) > self.moved_tol)[0]
                dirs = np.rint(2.0 * d[mv] / np.sqrt((d[mv] * d[mv]).sum(1))[:, None]).astype(int)
                key = tuple(sorted((int(subs[q].index[i]),) + tuple(int(v) for v in dirs[u]) for u, i in enumerate(mv)))
                if key not in seen:
                    seen.add(key)
                    keep.append(q)
                    keys.append(key)
            keep = np.asarray(keep, dtype=np.int64)
            if self.proposer is not None:
                # training rows from the distinct saddles only: repeats of one event add no
                # information and would weight the proposals towards the events found most often
                uniq = np.zeros(len(status), bool)
                uniq[keep] = True
                self._learn(W, xmin, xs_h, uniq)
            W.close()
            self._stage["learn_dedup"] = clock() - t0 - self._stage["search"]
            n = self.system.n
            region_atoms = int(np.diff(offs).max())
            out = self._no_events(ids, site_of, status, calls, atom_forces, learned)
            out["atoms"] = region_atoms
            self.last_saddles = []
            # region barriers (saddle less the region at basin 1, both with the same fixed shell);
            # only the saddles within polish_window of the lowest (over every rank) are polished in
            # the crystal: the others' rates are below e^-30 of the fastest event's, and they keep
            # their region barrier, which the fixed shell raises (a mountain pass over fewer paths
            # is no lower)
            e_reg = self._region_minima(regions, site_of[keep])
            bar_r = np.array([res["energy"][q] - e_reg[int(site_of[q])] for q in keep]) if len(keep) else np.zeros(0)
            lo = float(bar_r.min()) if len(keep) else float("inf")
            if self.world > 1:
                import torch.distributed as dist
                parts = [None] * self.world
                dist.all_gather_object(parts, lo)
                lo = min(parts)
            pol = bar_r <= lo + self.polish_window
            keep_u, bar_u = keep[~pol], bar_r[~pol]
            keys = [k for k, f in zip(keys, pol) if f]
            keep = keep[pol]
            out["unpolished"] = len(keep_u)
            if len(keep) == 0 and len(keep_u) == 0:
                return out
            K = len(keep)
            cp = np.zeros(0, dtype=np.int64)
            if K:
                # the crystal polish: a batched Dimer from each region saddle mapped into the
                # crystal, or, for an event polished in the previous step whose atoms lie beyond two
                # cutoffs of the last move, from that polished saddle (its whole displacement field
                # and mode, kept on the device) carried into this basin.  The crystal replicas stay
                # on the device; region rows and moved-atom masks come back.
                cache = self._polish_cache if self.recycle else {}
                rows, pos_v, mode_v, reuse = [], [], [], []
                for t_, q in enumerate(keep):
                    hit = cache.get(keys[t_])
                    if hit is not None and self._far_from_move(x1, hit[1]):
                        reuse.append((t_, hit[0]))
                        continue
                    sl = slice(offs[q], offs[q + 1])
                    rows.append(t_ * n + subs[q].index)
                    pos_v.append(xs_h[sl] - subs[q].shift)
                    mode_v.append(modes_h[sl])
                out["recycled"] = len(reuse)
                t1 = clock()
                Wp = self._polish_walkers(K)
                self._stage["polish_setup"] = clock() - t1
                x1_t = torch.tensor(x1, device=self.dev)
                box_t = torch.tensor(self.box, device=self.dev)
                xs_t = x1_t.repeat(Wp.W, 1)
                m_t = torch.zeros_like(xs_t)
                if rows:
                    r_t = torch.tensor(np.concatenate(rows), device=self.dev)
                    xs_t[r_t] = torch.tensor(np.concatenate(pos_v), device=self.dev)
                    m_t[r_t] = torch.tensor(np.concatenate(mode_v), device=self.dev)
                if reuse:
                    X, M, Dp = xs_t.view(Wp.W, n, 3), m_t.view(Wp.W, n, 3), self._polish_prev
                    dst = torch.tensor([t_ for t_, _ in reuse], device=self.dev)
                    src = torch.tensor([u for _, u in reuse], device=self.dev)
                    X[dst] = x1_t + Dp[0][src]
                    M[dst] = Dp[1][src]
                run = torch.zeros(Wp.W, dtype=torch.int32, device=self.dev)
                run[:K] = 1
                p = dimer_params(delta=self.dimer.delta, rot_tol=self.dimer.rot_tol,
                                 force_tol=self.polish_tol or self.dimer.force_tol, max_iter=self.polish_iter)
                t1 = clock()
                rp = Wp.dimer_subset(xs_t, m_t, run, p)[:K]
                self._stage["polish"] = clock() - t1
                out["polish_iters"] = float(rp["iters"].mean())
                if reuse:
                    ru = np.array([t_ for t_, _ in reuse])
                    out["recycled_iters"] = float(rp["iters"][ru].mean())
                    out["recycled_converged"] = int((rp["status"][ru] == CONVERGED).sum())
                out["status"][keep] = rp["status"]
                out["force_calls"][keep] += rp["force_calls"]
                out["atom_forces"][keep] += rp["force_calls"].astype(np.float64) * n
                # the atoms each saddle moves (crystal), and its region rows (positions, modes)
                D = xs_t[: K * n].view(K, n, 3) - x1_t.view(1, n, 3)
                D -= box_t * torch.round(D / box_t)
                moved = ((D * D).sum(2) > self.moved_tol ** 2).cpu().numpy()
                reg = np.concatenate([t_ * n + subs[q].index for t_, q in enumerate(keep)])
                reg_t = torch.tensor(reg, device=self.dev)
                reg_x, reg_m = xs_t[reg_t].cpu().numpy(), m_t[reg_t].cpu().numpy()
                reg_off = np.concatenate([[0], np.cumsum([len(subs[q].index) for q in keep])])
                # the converged saddles' displacement fields and modes, for the next step
                cp = np.where(rp["status"] == CONVERGED)[0]
                cp_t = torch.tensor(cp, device=self.dev)
                self._polish_prev = (D[cp_t], m_t[: K * n].view(K, n, 3)[cp_t])
                self._polish_cache = {keys[t_]: (u, np.where(moved[t_])[0]) for u, t_ in enumerate(cp)}
                del D
                self.last_saddles = [(self.system, x1.copy(), xs_t[t_ * n:(t_ + 1) * n].cpu().numpy(),
                                      float(rp["energy"][t_] - e1)) for t_ in cp[: self.keep_saddles]]
            out["polished"] = K
            # every event to be tabled -- converged polished saddles and the unpolished ones:
            # (walker, region positions, region mode, saddle energy, moved crystal atoms)
            events = []
            for t_ in cp:
                q = keep[t_]
                sl = slice(reg_off[t_], reg_off[t_ + 1])
                events.append((q, reg_x[sl] + subs[q].shift, reg_m[sl], rp["energy"][t_], np.where(moved[t_])[0]))
            for q, b in zip(keep_u, bar_u):
                sl = slice(offs[q], offs[q + 1])
                d = _wrap(xs_h[sl] - xmin[sl], boxes[q])
                mv = np.where(np.sqrt((d * d).sum(1)) > self.moved_tol)[0]
                events.append((q, xs_h[sl], modes_h[sl], e1 + b, np.sort(subs[q].index[mv])))
            if not events:
                return out
            # basin 2 of each (or of the polished ones only), in its region (which basin it leads
            # to: a loose FIRE tolerance does); the chosen event's basin 2 is relaxed in the crystal
            # after the selection
            n_pol = len(cp)
            n_chk = len(events) if self.basin2_unpolished else n_pol
            rejected = [0, 0]
            self._saddle_c = getattr(self, "_saddle_c", {})

            def table(q, xr, mr, es, mv):
                out["usable"][q] = True
                out["unique_local"][q] = True
                out["e_saddle"][q] = es
                out["fingerprint"][q] = tuple(int(i) for i in mv)
                self._saddle_c[int(ids[q])] = (subs[q].index, xr - subs[q].shift, mr)

            for q, xr, mr, es, mv in events[n_chk:]:
                table(q, xr, mr, es, mv)
            events = events[:n_chk]
            out["basin2_rejected"] = rejected
            if not events:
                return out
            qs = [e[0] for e in events]
            t1 = clock()
            Wr = Walkers.from_systems(self.field, [subs[q].system for q in qs],
                                      frozen=np.concatenate([subs[q].frozen for q in qs])).skip_tuning()
            self._stage["basin2_setup"] = clock() - t1
            ro = Wr.offsets
            start = np.concatenate([e[1] for e in events])
            rmode = np.concatenate([e[2] for e in events])
            rmin = np.concatenate([subs[q].system.pos for q in qs])
            for u in range(len(qs)):
                sl = slice(ro[u], ro[u + 1])
                away = np.sign(np.sum(rmode[sl] * _wrap(start[sl] - rmin[sl], Wr.boxes[u]))) or 1.0
                start[sl] = start[sl] + away * 0.1 * rmode[sl]
            t1 = clock()
            t2 = torch.tensor(start, device=self.dev)
            rb = Wr.relax(t2, fire_params(force_tol=max(self.relax_tol, self.basin2_tol)))
            x2r = t2.cpu().numpy()
            Wr.close()
            self._stage["basin2"] = clock() - t1
            for u, (q, xr, mr, es, mv) in enumerate(events):
                sl = slice(ro[u], ro[u + 1])
                if rb["status"][u] != CONVERGED or \
                        np.all(np.sqrt((_wrap(x2r[sl] - rmin[sl], Wr.boxes[u]) ** 2).sum(1)) < self.same_basin_tol):
                    rejected[int(u >= n_pol)] += 1               # not converged, or fell back into basin 1
                    continue
                table(q, xr, mr, es, mv)
            return out
        ev = self._events(W, xmin, xs_h, modes_h, res, np.full(m, e1), e1, ids, site_of, None)
        ev.update(ids=ids.astype(np.int64), site=site_of, status=status, force_calls=calls,
                  atom_forces=atom_forces, learned=learned, n_fallback=self._n_fallback if learned else 0,
                  atoms=int(np.diff(offs).max()), polished=0)
        return ev

    def _no_events(self, ids, site_of, status, calls, atom_forces, learned):
        m = len(ids)
        return dict(ids=ids.astype(np.int64), site=site_of, status=status, e_saddle=np.full(m, np.nan),
                    e_basin2=np.full(m, np.nan), usable=np.zeros(m, bool), unique_local=np.zeros(m, bool),
                    fingerprint=[None] * m, force_calls=calls, atom_forces=atom_forces, learned=learned,
                    n_fallback=self._n_fallback if learned else 0,
                    atoms=int(self.system.n), polished=0)

    def _events(self, W, xmin, xs_h, modes_h, res, e_min, e1, ids, site_of, _unused):
        """Basin 2 of every converged saddle of a crystal walker set (FIRE from the saddle nudged
        along the mode away from basin 1), the events' energies, fingerprints and basin-2
        positions, and duplicates of one site removed on the device."""
        import torch
        tt = lambda a, dt=None: torch.tensor(a, device=self.dev, dtype=dt)  # noqa: E731
        offs, boxes = W.offsets, W.boxes
        m = W.W
        conv = res["status"] == CONVERGED
        e2 = np.full(m, np.nan)
        x2 = np.zeros_like(xs_h)
        idx = np.where(conv)[0]
        if len(idx):
            starts = xs_h.copy()
            for q in idx:
                sl = slice(offs[q], offs[q + 1])
                away = np.sign(np.sum(modes_h[sl] * _wrap(xs_h[sl] - xmin[sl], boxes[q]))) or 1.0
                starts[sl] = xs_h[sl] + away * 0.1 * modes_h[sl]
            t = torch.tensor(starts, device=self.dev)
            rb = W.relax_subset(t, torch.tensor(conv.astype(np.int32), device=self.dev),
                                fire_params(force_tol=self.relax_tol))
            tb = t.cpu().numpy()
            for q in idx:
                if rb["status"][q] == CONVERGED:
                    x2[offs[q]:offs[q + 1]] = tb[offs[q]:offs[q + 1]]
                    e2[q] = rb["energy"][q]
        usable = conv & np.isfinite(e2)
        fingerprint = [None] * m
        for q in np.where(usable)[0]:
            sl = slice(offs[q], offs[q + 1])
            if np.all(np.sqrt((_wrap(x2[sl] - xmin[sl], boxes[q]) ** 2).sum(1)) < self.same_basin_tol):
                usable[q] = False                        # fell back into basin 1
                continue
            moved = np.where(np.sqrt((_wrap(xs_h[sl] - xmin[sl], boxes[q]) ** 2).sum(1)) > self.moved_tol)[0]
            fingerprint[q] = tuple(int(i) for i in moved)
        dup = kmc.dedup(tt(site_of), tt(usable.astype(np.int32)), tt(res["energy"].astype(np.float64)), tt(xs_h),
                        tt(offs[:-1].astype(np.int64)), tt(np.diff(offs).astype(np.int32)), tt(boxes),
                        self.e_tol, self.d_tol).cpu().numpy()
        barrier = res["energy"] - e_min
        self.last_saddles = []
        for q in np.where(usable)[0][: self.keep_saddles]:
            sl = slice(offs[q], offs[q + 1])
            self.last_saddles.append((self.system, xmin[sl].copy(), xs_h[sl].copy(), float(barrier[q])))
        self._basin2 = getattr(self, "_basin2", {})
        for q in np.where(usable)[0]:
            self._basin2[int(ids[q])] = x2[offs[q]:offs[q + 1]].copy()
        return dict(e_saddle=e1 + barrier, e_basin2=e1 + (e2 - e_min), usable=usable,
                    unique_local=usable & (dup < 0), fingerprint=fingerprint)

    def _select_and_move(self, tab, ev, x1, e1):
        """Unique events across sites and ranks (the moved-atom fingerprint and the saddle
        energy), the FP64 selection on the device, and the move to the chosen basin 2."""
        import torch
        unique = unique_events(tab, self.e_tol)
        t = lambda a, dt=None: torch.tensor(a, device=self.dev, dtype=dt)  # noqa: E731
        n = len(tab["ids"])
        es_d = t(tab["e_saddle"].astype(np.float64))
        u = kmc.uniforms(self.seed, self.iteration, 2)    # one Philox block per KMC step
        st, rate, cum = kmc.select(es_d, t(np.full(n, e1)), t(unique.astype(np.int32)),
                                   self.prefactor, self.temperature, u)
        rec = KmcRecord(step=self.iteration, time=self.time, dt=st["dt"], chosen=st["chosen"],
                        barrier=st["barrier"], n_saddles=int((tab["status"] == CONVERGED).sum()),
                        n_unique=int(unique.sum()), n_events=int(st["n_usable"]), total_rate=st["total_rate"],
                        energy=e1, force_calls=int(tab["force_calls"].sum()), learned=bool(ev["learned"]),
                        n_fallback=int(tab["n_fallback"]), atoms_per_walker=int(tab["atoms"]),
                        atom_forces=float(tab["atom_forces"].sum()), polished=int(tab["polished"]),
                        polish_iters=float(ev.get("polish_iters", 0.0)), recycled=int(ev.get("recycled", 0)),
                        recycled_iters=float(ev.get("recycled_iters", 0.0)),
                        recycled_converged=int(ev.get("recycled_converged", 0)),
                        unpolished=int(ev.get("unpolished", 0)),
                        basin2_rejected=int(ev.get("basin2_rejected", (0, 0))[0]),
                        basin2_rejected_unpolished=int(ev.get("basin2_rejected", (0, 0))[1]))
        t0 = time.perf_counter()
        if st["chosen"] >= 0:
            k = int(tab["ids"][st["chosen"]])
            owner = int(tab["owner"][st["chosen"]])
            mine = None
            if self.active_radius > 0:
                # the chosen event's basin 2 in the crystal, by the rank that holds its saddle
                if k in getattr(self, "_saddle_c", {}):
                    idx, xr, mr = self._saddle_c[k]
                    xs_c, m_c = x1.copy(), np.zeros_like(x1)
                    xs_c[idx], m_c[idx] = xr, mr
                    mine = self._crystal_basin2(x1, xs_c, m_c)
            else:
                mine = (self._basin2[k], float(tab["e_basin2"][st["chosen"]])) if k in self._basin2 else None
            got = broadcast_basin(mine, owner, self.world)
            if got is not None and got[0] is not None:
                self.pos = got[0] - self.box * np.rint(got[0] / self.box)     # the minimum-image cell
                self.energy = float(got[1])
                d = self._wrapdiff(self.pos, x1)
                mv = np.sqrt((d * d).sum(1)) > self.moved_tol
                self._moved_pos = np.concatenate([x1[mv], self.pos[mv]])
            self.time += st["dt"]
            rec.time = self.time
        rec.stage_s = dict(getattr(self, "_stage", {}), move=time.perf_counter() - t0)
        # the event table of this step, kept for inspection
        self.last_table = dict(e_saddle=tab["e_saddle"].copy(), e_min=e1, unique=unique.copy(),
                               status=tab["status"].copy(), e_basin2=tab["e_basin2"].copy(), u=u.cpu().numpy(),
                               rate=rate.cpu().numpy(), cum=cum.cpu().numpy(), ids=tab["ids"].copy())
        self.history.append(rec)
        self.iteration += 1
        return rec

    def _crystal_basin2(self, x1, xs, mode):
        """FIRE in the crystal from a saddle nudged along its mode away from basin 1:
        (positions, energy), or (None, nan) if it does not converge."""
        import torch
        away = np.sign(np.sum(mode * self._wrapdiff(xs, x1))) or 1.0
        t = torch.tensor(xs + away * 0.1 * mode, device=self.dev)
        r = self.one.relax(t, fire_params(force_tol=self.relax_tol))
        if r["status"][0] != CONVERGED:
            return (None, float("nan"))
        return (t.cpu().numpy(), float(r["energy"][0]))

    # --- learned proposals
    def _learned_searches(self, W, xmin, seeds, centres, local, explore):
        """Searches from the proposer's starting displacements (the walkers marked in
        ``explore`` and those without a proposal from their random seeds), then from the
        random seeds again for the walkers that did not converge.  Each walker draws its own
        candidate atom among those within ``radius`` of its seeding centre (its local region,
        as its random seed).  Replicas of the crystal share one set of descriptors and
        predictions; local regions each have their own."""
        import torch
        from . import proposals as P
        m, n = W.W, None
        x_t = torch.tensor(xmin, device=self.dev)
        if local:
            # descriptors and predictions of the candidates only: the atoms within the seeding
            # radius of each walker's centre
            begin, box = W.device_geometry()
            rows = P.region_rows(begin, x_t, box, torch.tensor(centres, device=self.dev), self.radius + 0.5)
            d, B = W.descriptors(x_t, with_basis=True, rows=rows)
            p_r, s_r = self.proposer.predict(d, B)
            pred = torch.zeros((x_t.shape[0], 3), dtype=torch.float32, device=self.dev)
            score = torch.zeros_like(pred)
            pred[rows.long()] = p_r
            score[rows.long()] = s_r
        else:
            n = self.system.n
            d, B = self.one.descriptors(x_t[:n].contiguous(), with_basis=True)
            pred, score = self.proposer.predict(d, B)
            pred, score = pred.repeat(m, 1), score.repeat(m, 1)
        fb = torch.tensor(seeds, device=self.dev)
        begin, box = W.device_geometry()
        disp, _, chosen = P.seeds(begin, x_t, box, pred, score,
                                  P.proposal_params(region=self.radius, threshold=self.proposal_threshold),
                                  seed=self.seed, counter=self.iteration,
                                  center=torch.tensor(centres, device=self.dev))
        chosen = chosen.cpu().numpy()
        counts = np.diff(W.offsets)
        rand = (chosen < 0) | explore
        rows = torch.tensor(np.repeat(rand, counts), device=self.dev)[:, None]
        disp = torch.where(rows, fb, disp)
        xs = x_t + disp
        modes = disp.clone()
        p = dimer_params(delta=self.dimer.delta, rot_tol=self.dimer.rot_tol, force_tol=self.dimer.force_tol,
                         max_iter=min(self.dimer.max_iter, self.learned_max_iter), patience=self.learned_patience)
        res = W.dimer(xs, modes, p)
        fail = res["status"] != CONVERGED
        self._n_fallback = int(fail.sum())
        self.last_learned = dict(chosen=chosen.copy(), explore=explore.copy(), status=res["status"].copy(),
                                 iters=res["iters"].copy())
        if fail.any():
            x2 = x_t + fb
            m2 = fb.clone()
            r2 = W.dimer_subset(x2, m2, torch.tensor(fail.astype(np.int32), device=self.dev), self.dimer)
            calls = res["force_calls"] + r2["force_calls"] * fail
            res[fail] = r2[fail]
            res["force_calls"] = calls
            rows = torch.tensor(np.repeat(fail, counts), device=self.dev)[:, None]
            xs = torch.where(rows, x2, xs)
            modes = torch.where(rows, m2, modes)
        return res, xs, modes

    def _learn(self, W, xmin, xs_h, usable):
        """Training rows from this step's saddles; fit once there are min_rows of them, refit
        when they have grown by half since the last fit.  Rows are kept per step and joined
        only when a fit is due."""
        import torch
        from . import proposals as P
        if not usable.any():
            return
        rng = np.random.default_rng(self.seed * 7919 + self.iteration)
        if self.active_radius > 0:
            # the atoms the rows need are chosen on the host; descriptors of those atoms only
            hops, TD, srows, TS = P.hop_picks(xmin, xs_h, W.offsets, W.boxes, usable, rng=rng)
            if len(hops) == 0:
                return
            nh = len(hops)
            want = torch.tensor(np.concatenate([hops, srows]), dtype=torch.int32, device=self.dev)
            d, B = W.descriptors(torch.tensor(xmin, device=self.dev), with_basis=True, rows=want)
            d, B = d.cpu().numpy(), B.cpu().numpy()
            self._rows["direction"].append((d[:nh], TD, B[:nh]))
            self._rows["score"].append((d[nh:], TS))
            self._n_dir += nh
        else:
            n = self.system.n
            d, B = self.one.descriptors(torch.tensor(xmin[:n], device=self.dev), with_basis=True)
            d, B = d.cpu().numpy(), B.cpu().numpy()
            one = np.array([0, n])
            for q in np.where(usable)[0]:           # the walkers are replicas of basin 1
                r = P.hop_rows(d, B, xmin[:n], xs_h[q * n:(q + 1) * n], one, [self.box], np.array([True]),
                               rng=rng)
                for key in self._rows:
                    self._rows[key].append(r[key])
                self._n_dir += len(r["direction"][0])
        nr = self._n_dir
        if self.world > 1:
            nr = int(shard.sum_over_ranks(nr))      # every rank fits at the same steps
        if nr >= self.min_rows and nr >= 1.5 * self._fit_rows:
            rows = {k: tuple(np.concatenate(z) for z in zip(*v)) for k, v in self._rows.items()}
            self._rows = {k: [v] for k, v in rows.items()}
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


def _wrap(d, box):
    box = np.asarray(box, dtype=np.float64)
    return d - box * np.rint(d / box)


def _within(x, centres, box, radius):
    """Indices of the points x within radius of any of the centres (minimum image)."""
    box = np.asarray(box, dtype=np.float64)
    near = np.zeros(len(x), bool)
    for c in np.atleast_2d(centres):
        d = _wrap(x - c, box)
        near |= (d * d).sum(1) <= radius * radius
    return np.where(near)[0]


EVENT_FIELDS = ("ids", "site", "status", "e_saddle", "e_basin2", "usable", "unique_local", "force_calls",
                "atom_forces")


def gather_events(ev, world):
    """Every rank's events in walker order (every rank gets all of them), with the rank
    that owns each.  One all-gather of small host records; positions never travel here."""
    own = {k: np.asarray(ev[k]) for k in EVENT_FIELDS}
    own["fingerprint"] = list(ev["fingerprint"])
    if world <= 1:
        tab = dict(own)
        tab["owner"] = np.zeros(len(own["ids"]), np.int64)
        tab["n_fallback"] = ev["n_fallback"]
        tab["atoms"] = ev["atoms"]
        tab["polished"] = ev.get("polished", 0)
        return tab
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, (own, int(ev["n_fallback"]), int(ev["atoms"]), int(ev.get("polished", 0))))
    tab = {k: np.concatenate([p[0][k] for p in parts]) for k in EVENT_FIELDS}
    tab["fingerprint"] = [f for p in parts for f in p[0]["fingerprint"]]
    tab["owner"] = np.concatenate([np.full(len(p[0]["ids"]), r, np.int64) for r, p in enumerate(parts)])
    order = np.argsort(tab["ids"], kind="stable")
    for k in list(tab):
        if k == "fingerprint":
            tab[k] = [tab[k][i] for i in order]
        else:
            tab[k] = tab[k][order]
    tab["n_fallback"] = sum(p[1] for p in parts)
    tab["atoms"] = max(p[2] for p in parts)
    tab["polished"] = sum(p[3] for p in parts)
    return tab


def unique_events(tab, e_tol):
    """Usable events that repeat no earlier event in walker order: not a duplicate of its
    own rank's site (positions, on the device) and not the same moved atoms with a saddle
    energy within e_tol of an earlier event of any site or rank."""
    keep = np.asarray(tab["unique_local"], dtype=bool).copy()
    seen = {}
    for i in np.where(keep)[0]:
        fp = tab["fingerprint"][i]
        prev = seen.setdefault(fp, [])
        if any(abs(tab["e_saddle"][i] - e) <= e_tol for e in prev):
            keep[i] = False
        else:
            prev.append(tab["e_saddle"][i])
    return keep


def broadcast_basin(pos, owner, world):
    """The chosen event's basin 2 on every rank (sent by the rank that found it)."""
    if world <= 1:
        return pos
    import torch.distributed as dist
    box = [pos if dist.get_rank() == owner else None]
    dist.broadcast_object_list(box, src=owner)
    return box[0]
