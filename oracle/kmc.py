"""FP64 restatement of the reference's KMC selection step (test infrastructure).

* ``rates``: Event::Event, kmc/Event.cpp:66-105 -- rate = prefactor * exp(-E_a * beta),
  beta = 1 / (k_B T), k_B = 8.617333262145e-5 eV/K (potentials/metal/Energy.h:43); here
  E_a = E_saddle - E_min in FP64 (the reference sends E_a as float,
  kmc/KineticMonteCarlo.cpp:1437-1440).
* ``select``: kmc/KineticMonteCarlo.cpp:147-170 (sum the rates in list order, the first
  event whose running sum exceeds u1 * R) and 1151-1160 (dt = (1/R) ln(u2), negated by the
  caller at :172; zero when |R| <= 1e-18).  The reference's runKMC needs MPI and headers
  absent from its tree, so these loops cannot be run as compiled reference code: this
  restatement follows them line by line and the tests check it on hand-worked cases.
* ``uniforms``: numpy.random.Philox (Philox4x64-10) -- the generator the GPU restates.
* ``dedup``: the duplicate-saddle rule of akmc_events_dedup by brute force.
"""
from __future__ import annotations

import math

import numpy as np

K_BOLTZMANN = 8.617333262145e-5


def rates(e_saddle, e_min, usable, prefactor, temperature):
    beta = 1.0 / (K_BOLTZMANN * temperature)
    out = np.zeros(len(e_saddle))
    for i in range(len(e_saddle)):
        if usable[i]:
            out[i] = prefactor * math.exp(-(e_saddle[i] - e_min[i]) * beta)
    return out


def select(rate, u1, u2):
    """(chosen index or -1, total rate, dt)."""
    total = 0.0
    for r in rate:                       # KineticMonteCarlo.cpp:149-157
        total += float(r)
    ran = u1 * total                     # :159
    temp = 0.0
    chosen = -1
    for i, r in enumerate(rate):         # :161-169
        temp += float(r)
        if temp > ran:
            chosen = i
            break
    u2 = u2 if u2 > 0.0 else 2.0 ** -53
    dt = -(1.0 / total) * math.log(u2) if abs(total) > 1.0e-18 else 0.0   # :1151-1160, :172
    return chosen, total, dt


def uniforms(seed, counter, n, key_hi=0):
    bg = np.random.Philox(key=np.array([seed, key_hi], dtype=np.uint64),
                          counter=np.array([counter, 0, 0, 0], dtype=np.uint64))
    return np.random.Generator(bg).random(n)


def dedup(group, usable, energy, pos, begin, natoms, box, e_tol, d_tol):
    n = len(group)
    dup = np.full(n, -1, dtype=np.int64)
    for i in range(n):
        if not usable[i]:
            continue
        for j in range(i):
            if not usable[j] or group[j] != group[i] or natoms[j] != natoms[i]:
                continue
            if not abs(energy[j] - energy[i]) <= e_tol:
                continue
            a = pos[begin[i]:begin[i] + natoms[i]]
            b = pos[begin[j]:begin[j] + natoms[j]]
            d = a - b
            L = np.asarray(box[i])
            d -= L * np.rint(d / L)
            if np.all((d * d).sum(1) <= d_tol * d_tol):
                dup[i] = j
                break
    return dup
