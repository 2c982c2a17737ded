"""Test oracle for the AKMC force path (test infrastructure, never the product).

Two checkers, both CPU:

* ``restated``: the FP64 C restatement in ``akmc_oracle.c`` (``liboracle.so``).
* ``reference``: the reference's own ``Field`` classes, compiled from the reference
  sources by ``oracle/Makefile`` into ``oracle/_ref/libref_{eam,pair}.so``.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline / reference arm
import this package.  Parsing here is independent of the product's parser: the
setfl reader restates ``MetalPotential::readLEAM`` (potentials/metal/
MetalPotential.cpp:276-361) and the potentials reader restates the keyword loops of
``Field::readPotential`` (potentials/pair/Field.cpp:215-317).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# The reference source tree the reference oracle is compiled from (read in place, never
# copied); AKMC_REFERENCE overrides it.  Where it is absent, only the restatement builds and
# the tests that need the reference skip.
REFERENCE = os.environ.get("AKMC_REFERENCE", "/root/reference")
LIB_PATH = os.path.join(HERE, "liboracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def build(reference: bool = True) -> None:
    """Compile the restatement (always) and the reference oracle (when its tree exists)."""
    targets = ["restatement"]
    if reference and os.path.isdir(REFERENCE):
        targets.append("reference")
        # the reference's relaxation driver on the drop-in Field links the product library
        if os.path.exists(os.path.join(os.path.dirname(HERE), "akmc_b200", "libakmc_b200.so")):
            targets.append("dropin")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE}"] + targets, check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(reference=False)
        L = C.CDLL(LIB_PATH)
        L.orc_eam_forces.restype = C.c_int
        L.orc_ionic_forces.restype = C.c_int
        L.orc_ewald_kvectors.restype = C.c_int
        L.orc_ewald_eta.restype = C.c_double
        L.orc_ewald_eta.argtypes = [C.c_double, C.c_double]
        L.orc_neighbour_counts.restype = C.c_longlong
        L.orc_neighbour_list.restype = C.c_longlong
        _lib = L
    return _lib


class OrcEamPot(C.Structure):
    _fields_ = [("n_embed", C.c_int), ("n_r", C.c_int), ("step_embed", C.c_double),
                ("step_r", C.c_double), ("pot_cutoff", C.c_double),
                ("F", _dp), ("dF", _dp), ("rho", _dp), ("drho", _dp), ("phi", _dp),
                ("dphi", _dp)]


def rcp_of(lat):
    """Reciprocal vectors, Basis::setRcpVec layout (Common/Basis.cpp:987-1010)."""
    L = np.asarray(lat, dtype=np.float64)
    R = np.empty(9)
    R[0] = L[4] * L[8] - L[7] * L[5]
    R[1] = L[6] * L[5] - L[3] * L[8]
    R[2] = L[3] * L[7] - L[6] * L[4]
    R[3] = L[7] * L[2] - L[1] * L[8]
    R[4] = L[0] * L[8] - L[6] * L[2]
    R[7] = L[6] * L[1] - L[0] * L[7]
    R[6] = L[1] * L[5] - L[4] * L[2]
    R[5] = L[2] * L[3] - L[5] * L[0]
    R[8] = L[0] * L[4] - L[3] * L[1]
    det = L[0] * R[0] + L[1] * R[3] + L[2] * R[6]
    return R * (1.0 / det if abs(det) > 0 else 1.0)


# --------------------------------------------------------------------------------------
# independent readers
# --------------------------------------------------------------------------------------
class SetflTables:
    """Tables exactly as MetalPotential::readLEAM leaves them."""

    def __init__(self, path):
        with open(path) as f:
            lines = f.read().split("\n")
        hdr = lines[4].split()
        self.n_embed = int(hdr[0]); self.step_embed = float(hdr[1])
        self.n_r = int(hdr[2]); self.step_r = float(hdr[3]); self.pot_cutoff = float(hdr[4])
        vals = []
        for ln in lines[6:]:
            vals.extend(float(w) for w in ln.split())
        v = np.array(vals, dtype=np.float64)
        ne, nr = self.n_embed, self.n_r
        self.F = v[:ne].copy()
        self.rho = v[ne:ne + nr].copy()
        rphi = v[ne + nr:ne + 2 * nr].copy()
        dist = np.arange(nr) * self.step_r
        with np.errstate(divide="ignore", invalid="ignore"):
            self.phi = rphi / dist                       # MetalPotential.cpp:357 (NaN at 0)
        self.dF = self._deriv(self.F, self.step_embed)
        self.drho = self._deriv(self.rho, self.step_r)
        self.dphi = self._deriv(self.phi, self.step_r)

    @staticmethod
    def _deriv(p, dr):
        # MetalPotential::calculateDerivativeMesh (MetalPotential.cpp:388-392), last = 0
        d = np.zeros_like(p)
        with np.errstate(invalid="ignore"):
            d[:-1] = (p[1:] - p[:-1]) / dr
        return d

    def as_struct(self):
        s = OrcEamPot(self.n_embed, self.n_r, self.step_embed, self.step_r, self.pot_cutoff,
                      _d(self.F), _d(self.dF), _d(self.rho), _d(self.drho), _d(self.phi),
                      _d(self.dphi))
        return s


def read_potentials(path):
    """Minimal restatement of the reference keyword loops for the keys the workloads use.
    The Ewald precision defaults to the reference's madelungAcc = 1e-6 (pair/Field.h:54) when
    the file has no ``ewald precis`` line."""
    out = dict(cutoff=None, species=[], eam=[], buck=[], precis=1.0e-6)
    with open(path) as f:
        lines = f.read().split("\n")
    i = 0
    while i < len(lines):
        w = lines[i].lower().split()
        raw = lines[i].split()
        i += 1
        if not w:
            continue
        k = w[0]
        if k == "cutoff":
            out["cutoff"] = float(w[1])
        elif k == "species":
            for _ in range(int(w[1])):
                s = lines[i].split(); i += 1
                out["species"].append((s[0], float(s[1]), float(s[2])))
        elif k in ("many", "manybody"):
            for _ in range(int(w[1])):
                i += 1                       # "eam"
                s = lines[i].split(); i += 1
                out["eam"].append((s[0], s[1], s[2]))
        elif k == "twobody":
            for _ in range(int(w[1])):
                i += 1                       # "buck"
                s = lines[i].split(); i += 1
                out["buck"].append((s[0], s[1], float(s[2]), float(s[3]), float(s[4])))
        elif k == "ewald":
            if w[1] == "precis":
                out["precis"] = float(w[2])
        elif k == "close":
            break
    return out


# --------------------------------------------------------------------------------------
# restated oracle
# --------------------------------------------------------------------------------------
def eam_forces(potentials_path, pos, labels, lat):
    """FP64 restatement. Returns (energies dict, forces (n,3), rho (n,), wrapped pos)."""
    P = read_potentials(potentials_path)
    # every table of the file, and the species-pair table of ManyBody::calculateEAMEnergyMesh
    # (ManyBody.cpp:937-1000): -1 where no entry names the pair
    tabs = [SetflTables(e[2]) for e in P["eam"]]
    pots = (OrcEamPot * len(tabs))(*[t.as_struct() for t in tabs])
    names = [s_[0] for s_ in P["species"]] or [P["eam"][0][0]]
    ns = len(names)
    mesh = np.full(ns * ns, -1, dtype=np.int32)
    for k, (a, b, _) in enumerate(P["eam"]):
        for i in range(ns):
            for j in range(ns):
                if names[i] == a and names[j] == b:
                    mesh[j * ns + i] = k
                    mesh[i * ns + j] = k
    n = len(pos)
    x = np.ascontiguousarray(pos[:, 0], dtype=np.float64).copy()
    y = np.ascontiguousarray(pos[:, 1], dtype=np.float64).copy()
    z = np.ascontiguousarray(pos[:, 2], dtype=np.float64).copy()
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    lat = np.asarray(lat, dtype=np.float64)
    rcp = rcp_of(lat)
    fx, fy, fz, rho = (np.zeros(n) for _ in range(4))
    e = np.zeros(5)
    rc = P["cutoff"]
    status = lib().orc_eam_forces(len(tabs), pots, ns, _i(mesh), C.c_double(rc), n, _d(x), _d(y),
                                  _d(z), _i(lab), _d(lat), _d(rcp), _d(fx), _d(fy), _d(fz),
                                  _d(rho), _d(e))
    E = dict(total=e[0], rcp=e[1], real=e[2], vdw=e[3], many=e[4], status=status)
    return E, np.stack([fx, fy, fz], 1), rho, np.stack([x, y, z], 1)


def ionic_setup(potentials_path, lat, max_k=200000):
    P = read_potentials(potentials_path)
    names = [s[0] for s in P["species"]]
    ns = len(names)
    buck = np.zeros(3 * ns * ns)
    table = np.zeros(ns * ns, dtype=np.int64)            # TwoBody meshTable default 0
    for k, (a, b, A, rho, Cc) in enumerate(P["buck"]):
        if a in names and b in names:
            ia, ib = names.index(a), names.index(b)
            table[ia * ns + ib] = k
            table[ib * ns + ia] = k
    for ab in range(ns * ns):
        A, rho, Cc = P["buck"][table[ab]][2:]
        buck[3 * ab:3 * ab + 3] = (A, rho, Cc)
    rc = P["cutoff"]
    eta = lib().orc_ewald_eta(P["precis"], rc)
    lat = np.asarray(lat, dtype=np.float64)
    rcp = rcp_of(lat)
    kx, ky, kz, g0 = (np.zeros(max_k) for _ in range(4))
    gc = np.zeros(3, dtype=np.int32)
    nk = lib().orc_ewald_kvectors(C.c_double(eta), C.c_double(rc), C.c_double(P["precis"]),
                                  _d(lat), _d(rcp), max_k, _d(kx), _d(ky), _d(kz), _d(g0), _i(gc))
    assert nk >= 0
    return dict(ns=ns, names=names, buck=buck, cutoff=rc, eta=eta, nk=nk,
                kx=kx[:nk].copy(), ky=ky[:nk].copy(), kz=kz[:nk].copy(), g0=g0[:nk].copy(),
                gcell=gc.copy(), charges=np.array([s[2] for s in P["species"]]))


def ionic_forces(setup, pos, charge, labels, lat):
    n = len(pos)
    x = np.ascontiguousarray(pos[:, 0], dtype=np.float64).copy()
    y = np.ascontiguousarray(pos[:, 1], dtype=np.float64).copy()
    z = np.ascontiguousarray(pos[:, 2], dtype=np.float64).copy()
    q = np.ascontiguousarray(charge, dtype=np.float64)
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    lat = np.asarray(lat, dtype=np.float64)
    rcp = rcp_of(lat)
    fx, fy, fz = (np.zeros(n) for _ in range(3))
    e = np.zeros(5)
    s = setup
    status = lib().orc_ionic_forces(s["ns"], _d(s["buck"]), C.c_double(s["cutoff"]),
                                    C.c_double(s["eta"]), C.c_double(14.3996454784), s["nk"],
                                    _d(s["kx"]), _d(s["ky"]), _d(s["kz"]), _d(s["g0"]), n,
                                    _d(x), _d(y), _d(z), _d(q), _i(lab), _d(lat), _d(rcp),
                                    _d(fx), _d(fy), _d(fz), _d(e))
    E = dict(total=e[0], rcp=e[1], real=e[2], vdw=e[3], many=e[4], status=status)
    return E, np.stack([fx, fy, fz], 1), np.stack([x, y, z], 1)


def neighbour_list(pos, lat, rc):
    """CSR full neighbour list (offsets, neighbours) by brute force."""
    n = len(pos)
    x, y, z = (np.ascontiguousarray(pos[:, k], dtype=np.float64) for k in range(3))
    lat = np.asarray(lat, dtype=np.float64)
    rcp = rcp_of(lat)
    counts = np.zeros(n, dtype=np.int32)
    tot = lib().orc_neighbour_counts(n, _d(x), _d(y), _d(z), _d(lat), _d(rcp), C.c_double(rc),
                                     _i(counts))
    off = np.zeros(n + 1, dtype=np.int64)
    nbr = np.zeros(max(tot, 1), dtype=np.int32)
    m = lib().orc_neighbour_list(n, _d(x), _d(y), _d(z), _d(lat), _d(rcp), C.c_double(rc),
                                 C.c_longlong(tot), off.ctypes.data_as(C.POINTER(C.c_longlong)),
                                 _i(nbr))
    assert m == tot
    return off, nbr[:tot]


# --------------------------------------------------------------------------------------
# reference oracle (the reference's own Field, compiled from its sources)
# --------------------------------------------------------------------------------------
_ref_libs = {}


def reference_available(family: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{family}.so"))


DROPIN_RELAX = os.path.join(REF_DIR, "relax_dropin")


def dropin_available() -> bool:
    """The reference's optim/Relax.cpp built against akmc_b200/cpp/Field.h (oracle/Makefile)."""
    return os.path.exists(DROPIN_RELAX)


DROPIN_ART = os.path.join(REF_DIR, "art_dropin")


def art_dropin_available() -> bool:
    """The reference's optim/ART.cpp built against akmc_b200/cpp/Field.h (oracle/Makefile)."""
    return os.path.exists(DROPIN_ART)


def _ref(family):
    if family not in _ref_libs:
        L = C.CDLL(os.path.join(REF_DIR, f"libref_{family}.so"))
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_char_p, C.c_char_p, _dp, C.c_int, C.c_double]
        L.ref_forces.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp,
                                 _dp, _dp]
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_num_species.argtypes = [C.c_void_p]
        L.ref_species_charge.argtypes = [C.c_void_p, C.c_int]
        L.ref_species_charge.restype = C.c_double
        L.ref_relax.restype = C.c_int
        L.ref_relax.argtypes = [C.c_void_p, C.c_char_p, C.c_int, _dp, _dp, _dp, _dp, _ip, _ip,
                                C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _dp]
        if hasattr(L, "ref_art"):               # the EAM build carries the reference's ART
            L.ref_art.restype = C.c_int
            L.ref_art.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _ip, _dp, C.c_int, C.c_double,
                                  C.c_int, C.c_double, C.c_double, _dp]
        _ref_libs[family] = L
    return _ref_libs[family]


_event_lib = None


def reference_event_rate(e_act, prefactor, temperature):
    """(rate, stored E_a) from the reference's own Event::Event (kmc/Event.cpp:66-105,
    compiled unchanged into oracle/_ref/libref_event.so): the event record carries E_a as a
    float, so the rate is prefactor * exp(-float(E_a) / (k_B T))."""
    global _event_lib
    if _event_lib is None:
        L = C.CDLL(os.path.join(REF_DIR, "libref_event.so"))
        L.ref_event_rate.restype = C.c_double
        L.ref_event_rate.argtypes = [C.c_double, C.c_double, C.c_double, _dp]
        _event_lib = L
    stored = C.c_double()
    r = _event_lib.ref_event_rate(float(e_act), float(prefactor), float(temperature), C.byref(stored))
    return r, stored.value


class ReferenceField:
    """The reference's own Field (metal: family 'eam'; pair: family 'pair')."""

    def __init__(self, family, potentials_path, lat, max_atoms, min_dim_override=0.0):
        """``min_dim_override`` > 0 is passed to Field::setup as the minimum cell
        dimension (see ref_harness.cpp): it lifts the pair Field's Verlet-shell guard
        for cells with cutoff < L/2 < cutoff + shell."""
        self.L = _ref(family)
        self.lat = np.ascontiguousarray(lat, dtype=np.float64)
        self._logdir = tempfile.mkdtemp(prefix="akmc_ref_")
        self.h = self.L.ref_create(potentials_path.encode(),
                                   os.path.join(self._logdir, "field.log").encode(),
                                   _d(self.lat), int(max_atoms), float(min_dim_override))
        if not self.h:
            raise RuntimeError("reference Field could not be created")

    def forces(self, pos, charge, labels):
        n = len(pos)
        x, y, z = (np.ascontiguousarray(pos[:, k], dtype=np.float64).copy() for k in range(3))
        q = np.ascontiguousarray(charge, dtype=np.float64)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        fx, fy, fz = (np.zeros(n) for _ in range(3))
        stress = np.zeros(6)
        e = np.zeros(6)
        self.L.ref_forces(self.h, n, _d(x), _d(y), _d(z), _d(q), _i(lab), _d(fx), _d(fy), _d(fz),
                          _d(stress), _d(e))
        E = dict(total=e[0], rcp=e[1], real=e[2], vdw=e[3], many=e[4], total_get=e[5])
        return E, np.stack([fx, fy, fz], 1), np.stack([x, y, z], 1)

    def relax(self, pos, charge, labels, frozen=None, method="fire", max_iter=3000,
              norm_tol=1.0e-5, force_tol=1.0e-4, init_dt=0.0005, max_dt=0.00075):
        """The reference's own Relax::RelaxStructure (optim/Relax.cpp:19-39).  Returns
        (status: 0 success / 1 failed, energies dict, relaxed wrapped positions)."""
        n = len(pos)
        x, y, z = (np.ascontiguousarray(pos[:, k], dtype=np.float64).copy() for k in range(3))
        q = np.ascontiguousarray(charge, dtype=np.float64)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        fr = np.zeros(n, np.int32) if frozen is None else np.ascontiguousarray(frozen, dtype=np.int32)
        e = np.zeros(6)
        st = self.L.ref_relax(self.h, method.encode(), n, _d(x), _d(y), _d(z), _d(q), _i(lab),
                              _i(fr), int(max_iter), float(norm_tol), float(force_tol),
                              float(init_dt), float(max_dt), _d(e))
        E = dict(total=e[0], rcp=e[1], real=e[2], vdw=e[3], many=e[4], total_get=e[5])
        return st, E, np.stack([x, y, z], 1)

    def art(self, pos, charge, labels, seed, max_par_iter=1000, force_tol=1.0e-3, go_perpendicular=False,
            init_dt=0.001, max_dt=0.002):
        """The reference's own ART saddle search (ART::findSaddlePoint, optim/ART.cpp:17-131;
        ARTCntrl defaults of Common/ArtCntrl.h) from the minimum ``pos`` moved by ``seed``
        (n, 3), every atom active, the initial Lanczos vector along the seed (ref_art.cpp);
        FIRE time steps init_dt -> max_dt (Energy time unit).  The start must already have a
        negative lowest curvature.  Returns (status: 0 success, saddle energy, final
        positions).  EAM build only."""
        if not hasattr(self.L, "ref_art"):
            raise RuntimeError("this reference build has no ART")
        n = len(pos)
        x, y, z = (np.ascontiguousarray(pos[:, k], dtype=np.float64).copy() for k in range(3))
        q = np.ascontiguousarray(charge, dtype=np.float64)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        sd = np.ascontiguousarray(seed, dtype=np.float64).reshape(-1)
        e = np.zeros(1)
        st = self.L.ref_art(self.h, n, _d(x), _d(y), _d(z), _d(q), _i(lab), _d(sd), int(max_par_iter),
                            float(force_tol), int(bool(go_perpendicular)), float(init_dt), float(max_dt), _d(e))
        return st, float(e[0]), np.stack([x, y, z], 1)

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
