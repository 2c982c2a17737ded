"""KMC step on the GPU (akmc_kmc_*, akmc_events_dedup): FP64 event table, duplicate
saddles, rate selection and time advance.

The reference's selection (kmc/KineticMonteCarlo.cpp:147-199, 1151-1160) on its float event
list (kmc/Event.cpp:66-105) becomes, on device buffers in FP64:

* :func:`uniforms` -- seeded Philox4x64-10 doubles (the reference seeds mt19937_64 from the
  clock, kmc/kmc.cpp:27-28);
* :func:`dedup` -- events that repeat an earlier saddle of the same basin;
* :func:`select` -- E_a = E_saddle - E_min, rates, running sums in list order, the chosen
  event and dt = -ln(u2)/R.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import KmcStep, check

BOLTZMANN_EV = 8.617333262145e-5    # eV/K, the selection kernel's (potentials/metal/Energy.h:43)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is not None:
        return C.c_void_p(int(stream))
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def uniforms(seed: int, counter: int, n: int, key_hi: int = 0, device="cuda", stream=None):
    """n doubles in [0, 1): numpy.random.Philox(key=[seed, key_hi], counter=[counter, 0, 0, 0])
    followed by random() gives the same numbers."""
    import torch
    out = torch.empty(n, dtype=torch.float64, device=device)
    check(_lib.load().akmc_kmc_uniforms(C.c_uint64(seed), C.c_uint64(key_hi), C.c_uint64(counter),
                                        int(n), _ptr(out), _stream(stream)), "kmc_uniforms")
    return out


def dedup(group, usable, energy, pos, begin, natoms, box, e_tol=1e-3, d_tol=0.1, stream=None):
    """Index of the earlier equivalent saddle per event (-1 if unique); all inputs CUDA
    tensors (group/usable/natoms int32, begin int64, energy float64 (n,), pos float64
    (atoms, 3), box float64 (n, 3))."""
    import torch
    n = int(group.numel())
    dup = torch.empty(n, dtype=torch.int32, device=group.device)
    check(_lib.load().akmc_events_dedup(n, _ptr(group), _ptr(usable), _ptr(energy), _ptr(pos),
                                        _ptr(begin), _ptr(natoms), _ptr(box), float(e_tol),
                                        float(d_tol), _ptr(dup), _stream(stream)), "events_dedup")
    return dup


def select(e_saddle, e_min, usable, prefactor, temperature, u, stream=None):
    """One KMC selection.  Returns (akmc_kmc_step as a dict, rates, running sums)."""
    import torch
    n = int(e_saddle.numel())
    dev = e_saddle.device
    rate = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    cum = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    step = torch.empty(C.sizeof(KmcStep), dtype=torch.uint8, device=dev)
    check(_lib.load().akmc_kmc_select(n, _ptr(e_saddle), _ptr(e_min), _ptr(usable),
                                      float(prefactor), float(temperature), _ptr(u), _ptr(rate),
                                      _ptr(cum), _ptr(step), _stream(stream)), "kmc_select")
    raw = step.cpu().numpy().tobytes()
    s = KmcStep.from_buffer_copy(raw)
    out = {k: getattr(s, k) for k, _ in KmcStep._fields_}
    return out, rate[:n], cum[:n]
