"""The reference's configuration files: ``basis`` input and the restart/archive dump.

Format (Basis::inputBasis, Common/Basis.cpp:356-500; Basis::dumpBasis, :592-649):

    title
    levcfg  imcon  natoms
    [timeStep  iteration  natoms  levcfg  imcon  time  energy]      <- restart files only
    a_x a_y a_z
    b_x b_y b_z
    c_x c_y c_z
    symbol  index                                                  <- per atom
    x  y  z
    [vx vy vz]                                                     <- levcfg >= 1
    [fx fy fz]                                                     <- levcfg >= 2

The reader follows inputBasis: the atom count is the third number of the second line, the
optional ``timeStep`` line carries the restart iteration (second word) and time (sixth
word), velocity and force lines are skipped, species are matched by name (an unknown name
is an error; the reference exits).  ``dump`` writes the reference's dump layout (header
once, then a ``timeStep`` block per call, ten decimals); a file of appended dumps reads back
as its first block, and ``read_last`` returns its last one (the restart point).
"""
from __future__ import annotations

import numpy as np

from .configs import System


class BasisError(ValueError):
    pass


def _parse_block(lines, i, natoms, levcfg, names, charges):
    restart_it, restart_t, energy = 0, 0.0, None
    w = lines[i].split()
    if w and w[0] == "timeStep":
        restart_it = int(w[1])
        restart_t = float(w[5])
        energy = float(w[6]) if len(w) > 6 else None
        i += 1
    lat = np.zeros(9)
    for r in range(3):
        w = lines[i].split()
        lat[3 * r:3 * r + 3] = [float(v) for v in w[:3]]
        i += 1
    pos = np.zeros((natoms, 3))
    lab = np.zeros(natoms, np.int32)
    for j in range(natoms):
        sym = lines[i].split()[0]
        if sym not in names:
            raise BasisError(f"no atom of type {sym} exists")
        lab[j] = names.index(sym)
        i += 1
        pos[j] = [float(v) for v in lines[i].split()[:3]]
        i += 1 + (1 if levcfg >= 1 else 0) + (1 if levcfg >= 2 else 0)
    q = np.asarray(charges, dtype=np.float64)[lab] if charges is not None else np.zeros(natoms)
    return i, System(pos=pos, labels=lab, charge=q, lat=lat,
                     meta=dict(iteration=restart_it, time=restart_t, energy=energy))


def _header(lines):
    if len(lines) < 2:
        raise BasisError("truncated basis file")
    w = lines[1].split()
    return lines[0].rstrip("\n"), int(w[0]), int(w[2])


def read_basis(path, species_names, species_charges=None) -> System:
    """The configuration of a basis (or restart) file: its first block.  meta holds the
    title, and the restart iteration / time / energy when the block has a timeStep line."""
    lines = open(path).read().splitlines()
    title, levcfg, natoms = _header(lines)
    _, s = _parse_block(lines, 2, natoms, levcfg, list(species_names), species_charges)
    s.meta["title"] = title
    return s


def read_last(path, species_names, species_charges=None) -> System:
    """The last block of an archive of appended dumps (the point a run restarts from)."""
    lines = open(path).read().splitlines()
    title, levcfg, natoms = _header(lines)
    i, s = 2, None
    while i < len(lines) and lines[i].strip():
        i, s = _parse_block(lines, i, natoms, levcfg, list(species_names), species_charges)
    if s is None:
        raise BasisError("no configuration in file")
    s.meta["title"] = title
    return s


def dump(stream, system: System, species_names, simulation_time: float, energy: float,
         iteration: int, title: str = "", header: bool = True) -> None:
    """Basis::dumpBasis: header (when ``header``), then one timeStep block."""
    n = system.n
    if header:
        stream.write(f"{title}\n0    3   {n}\n")
    stream.write(f"{'timeStep ':>15s}{iteration}     {n}    0      3   {simulation_time:.10f}     {energy:.10f}\n")
    lat = np.asarray(system.lat, dtype=np.float64)
    for r in range(3):
        stream.write("".join(f"{v:15.10f}" for v in lat[3 * r:3 * r + 3]) + "\n")
    for i in range(n):
        stream.write(f"{species_names[int(system.labels[i])]}      {i + 1}\n")
        x, y, z = system.pos[i]
        stream.write(f"  {x:.10f}  {y:.10f}  {z:.10f}\n")
    stream.flush()
