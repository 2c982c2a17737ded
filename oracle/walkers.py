"""FP64 CPU restatements of the walker algorithms (test infrastructure, never the product).

* ``fire_relax``: the reference's FIRE relaxation, Euler variant
  (optim/Relax.cpp:44-315, defaults Common/RelaxCntrl.h:15-38).  It is pinned against the
  reference's own Relax::RelaxStructure compiled from its sources
  (``ReferenceField.relax``), driven by the same forces.
* ``dimer_search``: the minimum-mode saddle search the product runs on the GPU.  The
  reference's optim/Dimer.cpp is an empty stub whose commented design
  (optim/Dimer.cpp:416-618) and controls (Common/DimerCntrl.h:18-88) fix the ingredients:
  a dimer of separation Delta along the unit mode N, forces at both ends, F2 = 2 F0 - F1,
  curvature from the force difference, rotations by a trial angle with a fitted minimum,
  the modified force for the translation, FIRE constants for the translation step.  The
  rotation follows Kaestner and Sherwood, J. Chem. Phys. 128, 014106 (2008), with the
  force interpolation of Heyden, Bell and Keil, J. Chem. Phys. 123, 224101 (2005); the
  modified force follows Henkelman and Jonsson, J. Chem. Phys. 111, 7010 (1999).  This
  restatement is the specification: there is no reference implementation to pin it
  against, so its parity is pinned only through the FIRE translation step it shares with
  ``fire_relax`` and through the saddle properties the tests check (zero force, one
  negative curvature, the energy of a symmetric hop).

Forces come from a callable ``force_fn(pos) -> (F (n,3), E_total, wrapped pos)`` that
wraps positions into the minimum-image cell, as every reference force call does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import eam_forces, ionic_forces, ionic_setup, read_potentials, SetflTables, lib, rcp_of
from . import _d, _i

EVTODL = 9648.530821      # Energy::timeStepUnit (potentials/metal/Energy.h:40)


# --------------------------------------------------------------------------------------
# cached force oracles
# --------------------------------------------------------------------------------------
class EamOracle:
    """The FP64 C restatement of the EAM force path with its tables read once."""

    def __init__(self, potentials_path, lat, labels):
        import ctypes as C
        P = read_potentials(potentials_path)
        self._tab = SetflTables(P["eam"][0][2])
        self._st = self._tab.as_struct()
        self.rc = P["cutoff"]
        self.lat = np.asarray(lat, dtype=np.float64)
        self.box = np.array([self.lat[0], self.lat[4], self.lat[8]])
        self.rcp = rcp_of(self.lat)
        self.labels = np.ascontiguousarray(labels, dtype=np.int32)
        self._mesh = np.zeros(1, dtype=np.int32)
        self._C = C
        self.calls = 0

    def __call__(self, pos):
        C = self._C
        n = len(pos)
        x, y, z = (np.ascontiguousarray(pos[:, k], dtype=np.float64).copy() for k in range(3))
        fx, fy, fz, rho = (np.zeros(n) for _ in range(4))
        e = np.zeros(5)
        st = lib().orc_eam_forces(1, C.byref(self._st), 1, _i(self._mesh), C.c_double(self.rc), n,
                                  _d(x), _d(y), _d(z), _i(self.labels), _d(self.lat), _d(self.rcp),
                                  _d(fx), _d(fy), _d(fz), _d(rho), _d(e))
        if st != 0:
            raise RuntimeError(f"oracle EAM force status {st}")
        self.calls += 1
        return np.stack([fx, fy, fz], 1), float(e[0]), np.stack([x, y, z], 1)


class IonicOracle:
    """The FP64 C restatement of the Buckingham + Ewald force path, set up once."""

    def __init__(self, potentials_path, lat, charge, labels):
        self.setup = ionic_setup(potentials_path, lat)
        self.lat = np.asarray(lat, dtype=np.float64)
        self.box = np.array([self.lat[0], self.lat[4], self.lat[8]])
        self.charge = np.asarray(charge, dtype=np.float64)
        self.labels = np.asarray(labels, dtype=np.int32)
        self.calls = 0

    def __call__(self, pos):
        E, F, w = ionic_forces(self.setup, pos, self.charge, self.labels, self.lat)
        if E["status"] != 0:
            raise RuntimeError(f"oracle ionic force status {E['status']}")
        self.calls += 1
        return F, float(E["total"]), w


# --------------------------------------------------------------------------------------
# FIRE (optim/Relax.cpp:44-315)
# --------------------------------------------------------------------------------------
@dataclass
class FireParams:
    """RelaxCntrl (Common/RelaxCntrl.h:15-38) defaults."""
    max_iter: int = 3000
    norm_tol: float = 1.0e-5
    force_tol: float = 1.0e-4
    n_min: int = 5
    dt0: float = 0.0005
    alpha_dec: float = 0.99
    step_inc: float = 1.1
    step_dec: float = 0.5
    alpha0: float = 0.1
    dt_max: float = 0.00075
    max_move: float = 0.0       # per-atom step cap; 0 = none, as in the reference


def fire_relax(force_fn, pos, frozen=None, p: FireParams = FireParams()):
    """Relax ``pos`` (n,3).  Returns dict(pos, energy, status 1 converged / 2 out of
    iterations, iters, fnorm, fmax, force)."""
    x = np.array(pos, dtype=np.float64, copy=True)
    n = len(x)
    fz = np.zeros(n, bool) if frozen is None else np.asarray(frozen).astype(bool)
    mov = ~fz
    v = np.zeros_like(x)
    F, E, x = force_fn(x)                       # Relax.cpp:95
    F[fz] = 0.0                                 # Relax.cpp:101-109
    nstep, alpha, dt = 1, p.alpha0, p.dt0
    fnorm = fmax = 0.0
    for it in range(1, p.max_iter + 1):
        P = float(np.sum(F * v))                # Relax.cpp:131
        one_less = 1.0 - alpha
        fnorm = math.sqrt(float(np.sum(F * F)))
        vnorm = math.sqrt(float(np.sum(v * v)))
        alpha_force = alpha * vnorm / fnorm if fnorm > 0.0 else 0.0
        if P > 0.0:                             # Relax.cpp:140-162
            v[mov] = one_less * v[mov] + alpha_force * F[mov]
            if nstep > p.n_min:
                dt = min(dt * p.step_inc, p.dt_max)
                alpha *= p.alpha_dec
            nstep += 1
        else:                                   # Relax.cpp:163-174
            nstep = 0
            dt *= p.step_dec
            alpha = p.alpha0
            v[:] = 0.0
        if p.max_move > 0.0:
            vm = math.sqrt(float(np.max(np.sum(v * v, 1)))) if n else 0.0
            if dt * vm > p.max_move:
                v *= p.max_move / (dt * vm)
        fact = dt * EVTODL                      # Relax.cpp:176-191 (Euler)
        x[mov] += dt * v[mov]
        v[mov] += fact * F[mov]
        F, E, x = force_fn(x)                   # Relax.cpp:229-231
        F[fz] = 0.0
        v -= v.mean(0)                          # Relax.cpp:252 centreOfMass
        f2 = np.sum(F * F, 1)
        fnorm = math.sqrt(float(f2.sum()))
        fmax = math.sqrt(float(f2.max())) if n else 0.0
        if fnorm < p.norm_tol or fmax < p.force_tol:      # Relax.cpp:276
            return dict(pos=x, energy=E, status=1, iters=it, fnorm=fnorm, fmax=fmax, force=F)
    return dict(pos=x, energy=E, status=2, iters=p.max_iter, fnorm=fnorm, fmax=fmax, force=F)


# --------------------------------------------------------------------------------------
# Dimer
# --------------------------------------------------------------------------------------
@dataclass
class DimerParams:
    """Controls named as in DimerCntrl (Common/DimerCntrl.h:18-88) where one exists."""
    delta: float = 0.01            # dimerDisplacement
    rot_tol: float = 0.1           # normTol: skip rotation below this |dC/dtheta|/2, eV/A^2
    force_tol: float = 1.0e-2      # forceTol: saddle when max_i |F_i| is below this (barriers
                                   # within 0.3 meV of a saddle converged to 1e-5 eV/A) ...
    max_eigenvalue: float = 0.0    # ... and the curvature is below this (maxEigenvalue)
    max_rotations: int = 1         # rotations per translation step
    max_iter: int = 300
    min_trial: float = 1.0e-3      # smallest trial rotation angle, rad
    max_move: float = 0.02         # per-atom translation cap per step, A
    max_rise: float = 8.0          # lost (status 3) when E rises this far above the start, eV
    translation: str = "lbfgs"     # "lbfgs" (default) or "fire"
    lbfgs_memory: int = 8          # L-BFGS: stored (s, y) pairs
    max_step: float = 0.2          # L-BFGS: per-atom cap of one translation step, A
    convex_step: float = 0.05      # L-BFGS: step along the mode while the curvature is >= 0, A
    n_min: int = 5                 # FIRE constants of the translation (DimerCntrl N_min ...)
    alpha_dec: float = 0.99
    step_inc: float = 1.1
    step_dec: float = 0.5
    alpha0: float = 0.1
    dt0: float = 0.001
    dt_max: float = 0.004


def _rotate(F0, F1, N, C, p, trial_force):
    """One rotation.  Returns (N, F1, C, rotated, torque)."""
    dF = F1 - F0
    dn = float(np.sum(dF * N))
    C = -dn / p.delta
    frot = 2.0 * (dF - dn * N)
    frn = math.sqrt(float(np.sum(frot * frot)))
    torque = frn / (2.0 * p.delta)
    if not (torque > p.rot_tol and frn > 0.0):
        return N, F1, C, False, torque
    th = frot / frn
    t1 = max(0.5 * math.atan(torque / max(abs(C), 1e-12)), p.min_trial)
    c1, s1 = math.cos(t1), math.sin(t1)
    Nt = N * c1 + th * s1
    F1t = trial_force(Nt)
    C1 = float(np.sum((F0 - F1t) * Nt)) / p.delta
    b1 = -torque
    a1 = (C - C1 + b1 * math.sin(2.0 * t1)) / (1.0 - math.cos(2.0 * t1))
    a0 = 2.0 * (C - a1)
    tm = 0.5 * math.atan(b1 / a1)
    Cm = 0.5 * a0 + a1 * math.cos(2.0 * tm) + b1 * math.sin(2.0 * tm)
    if Cm > C:
        tm += 0.5 * math.pi
        Cm = 0.5 * a0 + a1 * math.cos(2.0 * tm) + b1 * math.sin(2.0 * tm)
    cm, sm = math.cos(tm), math.sin(tm)
    Nn = N * cm + th * sm
    Nn /= math.sqrt(float(np.sum(Nn * Nn)))
    st1 = math.sin(t1)
    F1n = (math.sin(t1 - tm) / st1) * F1 + (sm / st1) * F1t + \
          (1.0 - cm - sm * math.tan(0.5 * t1)) * F0
    return Nn, F1n, Cm, True, torque


class _Lbfgs:
    """L-BFGS translation of the dimer on the modified force (Nocedal's two-loop recursion;
    the translation EON-style dimers use), restarted whenever the curvature turns >= 0 or a
    pair has s.y <= 0, and replaced by a fixed step along the mode while C >= 0."""

    def __init__(self, mem, box):
        self.mem = mem
        self.box = None if box is None else np.asarray(box, dtype=np.float64)
        self.S, self.Y, self.rho = [], [], []
        self.xp = self.gp = None

    def reset(self):
        self.S, self.Y, self.rho = [], [], []
        self.xp = self.gp = None

    def step(self, x, F0, N, fn, C, p):
        if C >= 0.0:
            self.reset()
            sgn = 1.0 if fn <= 0.0 else -1.0          # up the energy along the (unit) mode
            return self._cap(sgn * p.convex_step * N, p)
        g = -(F0 - 2.0 * fn * N)
        if self.xp is not None:
            sv = x - self.xp
            if self.box is not None:
                sv -= self.box * np.rint(sv / self.box)
            yv = g - self.gp
            sy = float(np.sum(sv * yv))
            if sy > 1e-12:
                self.S.append(sv)
                self.Y.append(yv)
                self.rho.append(1.0 / sy)
                if len(self.S) > self.mem:
                    self.S.pop(0), self.Y.pop(0), self.rho.pop(0)
            else:
                self.S, self.Y, self.rho = [], [], []
        q = g.copy()
        a = []
        for sv, yv, rho in zip(reversed(self.S), reversed(self.Y), reversed(self.rho)):
            ak = rho * float(np.sum(sv * q))
            a.append(ak)
            q -= ak * yv
        gam = float(np.sum(self.S[-1] * self.Y[-1])) / float(np.sum(self.Y[-1] * self.Y[-1])) if self.S else 0.01
        r = gam * q
        for (sv, yv, rho), ak in zip(zip(self.S, self.Y, self.rho), reversed(a)):
            bk = rho * float(np.sum(yv * r))
            r += sv * (ak - bk)
        st = -r
        if float(np.sum(st * g)) >= 0.0:               # not downhill on the modified force
            self.S, self.Y, self.rho = [], [], []
            st = -0.01 * g
        self.xp, self.gp = x.copy(), g.copy()
        return self._cap(st, p)

    @staticmethod
    def _cap(st, p):
        m = math.sqrt(float(np.max(np.sum(st * st, 1))))
        return st * (p.max_step / m) if m > p.max_step else st


def dimer_search(force_fn, pos, mode, p: DimerParams = DimerParams(), box=None):
    """Climb from ``pos`` along the unit-normalised ``mode`` to a first-order saddle.
    ``box`` (3 lengths) folds the L-BFGS step differences into the minimum image (force
    calls wrap positions in place).  Returns dict(pos, mode, energy, curvature, status
    1 saddle / 2 out of iterations / 3 lost, iters, fmax, force_calls)."""
    x = np.array(pos, dtype=np.float64, copy=True)
    N = np.array(mode, dtype=np.float64, copy=True)
    N /= math.sqrt(float(np.sum(N * N)))
    v = np.zeros_like(x)
    nstep, alpha, dt = 1, p.alpha0, p.dt0
    calls = 0
    C = 0.0
    E = fmax = 0.0
    E_start = None
    if box is None:
        box = getattr(force_fn, "box", None)            # the force oracles carry their box
    lb = _Lbfgs(p.lbfgs_memory, box) if p.translation == "lbfgs" else None
    for it in range(p.max_iter + 1):
        F0, E, x = force_fn(x)
        F1, _, _ = force_fn(x + p.delta * N)
        calls += 2
        if E_start is None:
            E_start = E

        def trial(Nt):
            nonlocal calls
            calls += 1
            return force_fn(x + p.delta * Nt)[0]

        C = float(np.sum((F0 - F1) * N)) / p.delta
        for _ in range(p.max_rotations):
            N, F1, C, rotated, _t = _rotate(F0, F1, N, C, p, trial)
            if not rotated:
                break
        fmax = math.sqrt(float(np.max(np.sum(F0 * F0, 1))))
        if fmax < p.force_tol and C < p.max_eigenvalue:
            return dict(pos=x, mode=N, energy=E, curvature=C, status=1, iters=it, fmax=fmax,
                        force_calls=calls)
        if E - E_start > p.max_rise:
            return dict(pos=x, mode=N, energy=E, curvature=C, status=3, iters=it, fmax=fmax,
                        force_calls=calls)
        if it >= p.max_iter:
            break
        fn = float(np.sum(F0 * N))
        if lb is not None:
            x = x + lb.step(x, F0, N, fn, C, p)
            continue
        Feff = F0 - 2.0 * fn * N if C < 0.0 else -fn * N
        P = float(np.sum(Feff * v))
        one_less = 1.0 - alpha
        fnorm = math.sqrt(float(np.sum(Feff * Feff)))
        vnorm = math.sqrt(float(np.sum(v * v)))
        alpha_force = alpha * vnorm / fnorm if fnorm > 0.0 else 0.0
        if P > 0.0:
            v = one_less * v + alpha_force * Feff
            if nstep > p.n_min:
                dt = min(dt * p.step_inc, p.dt_max)
                alpha *= p.alpha_dec
            nstep += 1
        else:
            nstep = 0
            dt *= p.step_dec
            alpha = p.alpha0
            v[:] = 0.0
        if p.max_move > 0.0:
            vm = math.sqrt(float(np.max(np.sum(v * v, 1))))
            if dt * vm > p.max_move:
                v *= p.max_move / (dt * vm)
        x += dt * v
        v += dt * EVTODL * Feff
    return dict(pos=x, mode=N, energy=E, curvature=C, status=2, iters=p.max_iter, fmax=fmax,
                force_calls=calls)
