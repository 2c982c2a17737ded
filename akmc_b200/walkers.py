"""Batched walkers: FIRE relaxation and Dimer saddle searches on the GPU (akmc_walkers_*).

The reference relaxes one configuration at a time with ``Relax::RelaxStructure``
(optim/Relax.cpp:19-39) and searches saddles one at a time; its Dimer
(optim/Dimer.cpp) is a stub.  :class:`Walkers` runs W independent systems together:

* :meth:`Walkers.relax` -- the reference's FIRE (Euler variant, optim/Relax.cpp:44-315)
  with the controls of ``RelaxCntrl`` (Common/RelaxCntrl.h:15-38);
* :meth:`Walkers.dimer` -- the minimum-mode saddle search of the reference's commented
  Dimer design (optim/Dimer.cpp:416-618, Common/DimerCntrl.h:18-88).

Positions and modes are torch CUDA tensors (device-resident path) or host arrays
(:meth:`relax_host` / :meth:`dimer_host`, which copy in and out).  Results come back as
numpy record arrays with one row per walker.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import DimerParams, FireParams, WalkerResult, check

RUNNING, CONVERGED, MAX_ITER, LOST, FORCE_ERROR, SKIPPED = 0, 1, 2, 3, 4, 5
STATUS_NAMES = {RUNNING: "running", CONVERGED: "converged", MAX_ITER: "max_iter",
                LOST: "lost", FORCE_ERROR: "force_error"}

RESULT_DTYPE = np.dtype([("status", np.int32), ("iters", np.int32), ("force_calls", np.int32),
                         ("reserved", np.int32), ("energy", np.float64),
                         ("curvature", np.float64), ("fmax", np.float64), ("fnorm", np.float64)])


def fire_params(**kw) -> FireParams:
    """akmc_fire_params with the RelaxCntrl defaults, overridden by keyword."""
    p = FireParams()
    _lib.load().akmc_fire_defaults(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def dimer_params(**kw) -> DimerParams:
    """akmc_dimer_params with the defaults of akmc_dimer_defaults, overridden by keyword."""
    p = DimerParams()
    _lib.load().akmc_dimer_defaults(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def _results(buf) -> np.ndarray:
    return np.frombuffer(bytes(buf), dtype=RESULT_DTYPE).copy()


class Walkers:
    """W independent systems of one :class:`~akmc_b200.field.Field` (sizes may differ).

    Atoms of walker w occupy rows ``offsets[w]:offsets[w+1]`` of the (n_total, 3) FP64
    position / mode arrays."""

    def __init__(self, field, natoms, boxes, labels, charges=None, frozen=None):
        self.field = field
        self._lib = field._lib
        self.natoms = np.ascontiguousarray(natoms, dtype=np.int32)
        self.boxes = np.ascontiguousarray(boxes, dtype=np.float64).reshape(-1, 3)
        self.W = len(self.natoms)
        self.n_total = int(self.natoms.sum())
        self.offsets = np.concatenate([[0], np.cumsum(self.natoms)]).astype(np.int64)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        q = None if charges is None else np.ascontiguousarray(charges, dtype=np.float64)
        fz = None if frozen is None else np.ascontiguousarray(frozen, dtype=np.int32)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        self._h = C.c_void_p()
        check(self._lib.akmc_walkers_create(
            field._h, self.W, self.natoms.ctypes.data_as(ip), self.boxes.ctypes.data_as(dp),
            lab.ctypes.data_as(ip), None if q is None else q.ctypes.data_as(dp),
            None if fz is None else fz.ctypes.data_as(ip), C.byref(self._h)), "walkers_create")

    @classmethod
    def from_systems(cls, field, systems, frozen=None):
        return cls(field, [s.n for s in systems], [s.box for s in systems],
                   np.concatenate([s.labels for s in systems]),
                   np.concatenate([s.charge for s in systems]), frozen)

    def device_geometry(self):
        """(atom offsets int64 (W + 1,), boxes float64 (W, 3)) as CUDA tensors (cached)."""
        if getattr(self, "_geom", None) is None:
            import torch
            self._geom = (torch.tensor(self.offsets, dtype=torch.int64, device="cuda"),
                          torch.tensor(self.boxes, dtype=torch.float64, device="cuda"))
        return self._geom

    def skip_tuning(self):
        """akmc_walkers_skip_tuning: keep the default work-item sizes (one-off walker sets)."""
        check(self._lib.akmc_walkers_skip_tuning(self._h), "skip_tuning")
        return self

    def tuning(self, which=1):
        """The per-size-class work-item table of the Dimer's image batch (which=1) or the
        FIRE batch (0): rows {cells, home_chunk, ms_per_call}, empty before the first call."""
        cells = (C.c_int * 16)()
        chunk = (C.c_int * 16)()
        ms = (C.c_float * 16)()
        n = self._lib.akmc_walkers_tuning(self._h, int(which), cells, chunk, ms, 16)
        return [{"cells": cells[k], "home_chunk": chunk[k], "ms_per_call": ms[k]} for k in range(min(n, 16))]

    @property
    def skin(self) -> float:
        return self._lib.akmc_walkers_skin(self._h)

    def set_skin(self, skin: float):
        """akmc_walkers_set_skin: neighbour-list skin of the walkers' force calls (A)."""
        check(self._lib.akmc_walkers_set_skin(self._h, float(skin)), "set_skin")

    @staticmethod
    def _stream(stream):
        if stream is not None:
            return int(stream)
        import torch
        return torch.cuda.current_stream().cuda_stream

    def relax(self, pos, params: FireParams | None = None, stream=None) -> np.ndarray:
        """FIRE-relax in place.  ``pos``: CUDA float64 tensor (n_total, 3)."""
        p = params or fire_params()
        out = (WalkerResult * self.W)()
        check(self._lib.akmc_walkers_relax(self._h, C.c_void_p(pos.data_ptr()), C.byref(p), out,
                                           C.c_void_p(self._stream(stream))), "walkers_relax")
        return _results(out)

    def dimer(self, pos, mode, params: DimerParams | None = None, stream=None) -> np.ndarray:
        """Dimer searches in place.  ``pos``, ``mode``: CUDA float64 tensors (n_total, 3)."""
        p = params or dimer_params()
        out = (WalkerResult * self.W)()
        check(self._lib.akmc_walkers_dimer(self._h, C.c_void_p(pos.data_ptr()),
                                           C.c_void_p(mode.data_ptr()), C.byref(p), out,
                                           C.c_void_p(self._stream(stream))), "walkers_dimer")
        return _results(out)

    def relax_subset(self, pos, run_mask, params: FireParams | None = None, stream=None) -> np.ndarray:
        """FIRE of the walkers whose ``run_mask`` (CUDA int32 tensor (W,)) entry is non-zero;
        the others keep pos and report status SKIPPED."""
        p = params or fire_params()
        out = (WalkerResult * self.W)()
        check(self._lib.akmc_walkers_relax_subset(self._h, C.c_void_p(pos.data_ptr()), C.byref(p),
                                                  C.c_void_p(run_mask.data_ptr()), out,
                                                  C.c_void_p(self._stream(stream))), "walkers_relax_subset")
        return _results(out)

    def dimer_subset(self, pos, mode, run_mask, params: DimerParams | None = None, stream=None) -> np.ndarray:
        """Dimer searches of the walkers whose ``run_mask`` (CUDA int32 tensor (W,)) entry is
        non-zero; the others keep pos and mode and report status SKIPPED."""
        p = params or dimer_params()
        out = (WalkerResult * self.W)()
        check(self._lib.akmc_walkers_dimer_subset(self._h, C.c_void_p(pos.data_ptr()),
                                                  C.c_void_p(mode.data_ptr()), C.byref(p),
                                                  C.c_void_p(run_mask.data_ptr()), out,
                                                  C.c_void_p(self._stream(stream))), "walkers_dimer_subset")
        return _results(out)

    def descriptors(self, pos, with_basis=False, stream=None, rows=None):
        """Descriptors (n_total, 64) float32 of every atom at ``pos`` (CUDA float64 tensor,
        (n_total, 3)), from a force call on the walkers' own batch; with ``with_basis`` also
        the readout vectors (n_total, 3, 3).  With ``rows`` (CUDA int32 tensor of atom
        numbers) only those atoms, in that order: (len(rows), 64) and (len(rows), 3, 3)."""
        import torch
        n = self.n_total if rows is None else int(rows.numel())
        d = torch.empty((n, 64), dtype=torch.float32, device=pos.device)
        B = torch.empty((n, 3, 3), dtype=torch.float32, device=pos.device) if with_basis else None
        Bp = C.c_void_p(B.data_ptr()) if with_basis else None
        if rows is None:
            check(self._lib.akmc_walkers_descriptors(self._h, C.c_void_p(pos.data_ptr()), C.c_void_p(d.data_ptr()),
                                                     Bp, C.c_void_p(self._stream(stream))), "walkers_descriptors")
        else:
            rows = rows.to(torch.int32).contiguous()
            check(self._lib.akmc_walkers_descriptors_rows(self._h, C.c_void_p(pos.data_ptr()),
                                                          C.c_void_p(rows.data_ptr()), n, C.c_void_p(d.data_ptr()),
                                                          Bp, C.c_void_p(self._stream(stream))),
                  "walkers_descriptors_rows")
        return (d, B) if with_basis else d

    def relax_host(self, pos, params: FireParams | None = None):
        """Host arrays in, host arrays out: (relaxed positions, results)."""
        import torch
        d = torch.as_tensor(np.ascontiguousarray(pos, dtype=np.float64)).cuda()
        r = self.relax(d, params)
        return d.cpu().numpy(), r

    def dimer_host(self, pos, mode, params: DimerParams | None = None):
        """Host arrays in, host arrays out: (final positions, final modes, results)."""
        import torch
        d = torch.as_tensor(np.ascontiguousarray(pos, dtype=np.float64)).cuda()
        m = torch.as_tensor(np.ascontiguousarray(mode, dtype=np.float64)).cuda()
        r = self.dimer(d, m, params)
        return d.cpu().numpy(), m.cpu().numpy(), r

    def close(self):
        if self._h:
            self._lib.akmc_walkers_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
