"""ctypes mirror of include/cosims_cuda.h (the C ABI of the CCS engine).

The structures here are field-for-field copies of the C declarations; the
helpers build a `cosims_molecule` view over numpy arrays that the caller keeps
alive (the `MoleculeArrays` object holds the references).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

ABI_VERSION = 2

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_IO, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_BUSY = range(8)

PLAIN_F64 = 0
MIXED = 1

WAIT_TEST_STAGING = 0x1
WAIT_TEST_HANDOFF = 0x2

TRAJ_HIT = 0x1
TRAJ_SUCCESS = 0x2
TRAJ_STEPCAP = 0x4
TRAJ_ETRIES_SHIFT = 8
TRAJ_OTRIES_SHIFT = 16

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class Molecule(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32),
        ("x", _dp), ("y", _dp), ("z", _dp),
        ("charge", _dp), ("sig6", _dp), ("eps24m", _dp), ("eps4", _dp),
        ("n_clusters", C.c_int32),
        ("cluster_offset", _ip), ("cluster_atoms", _ip),
        ("cluster_pos", _dp), ("cluster_radius", _dp), ("cluster_charge", _dp),
        ("cluster_dipole", _dp), ("cluster_quad", _dp), ("cluster_replaced", _ip),
    ]


class Params(C.Structure):
    _fields_ = [
        ("force_type", C.c_int32), ("multipole_order", C.c_int32),
        ("projection", C.c_int32), ("charged", C.c_int32),
        ("dt", C.c_double), ("mu", C.c_double), ("dipole_scalar", C.c_double),
        ("r_disp", C.c_double), ("r_mp", C.c_double),
        ("ell_a", C.c_double), ("ell_b", C.c_double), ("ell_c", C.c_double),
        ("b_max", C.c_double), ("start_dist", C.c_double),
        ("g_min", C.c_double), ("g_max", C.c_double),
        ("vdist_a", C.c_double), ("vdist_norm", C.c_double), ("vdist_max", C.c_double),
        ("ccs_const", C.c_double), ("max_steps", C.c_int64),
    ]


class TrajOut(C.Structure):
    _fields_ = [("chi", C.c_double), ("de_pct", C.c_double),
                ("steps", C.c_int32), ("status", C.c_uint32)]


class TrajIn(C.Structure):
    _fields_ = [("b", C.c_double), ("phi", C.c_double), ("theta", C.c_double),
                ("gamma", C.c_double), ("g", C.c_double)]


class CcsSums(C.Structure):
    _fields_ = [("sum", C.c_double), ("sum2", C.c_double), ("max_de_pct", C.c_double),
                ("n", C.c_int64), ("n_hit", C.c_int64), ("n_success", C.c_int64),
                ("n_eff", C.c_int64), ("steps", C.c_int64), ("force_evals", C.c_int64),
                ("pot_evals", C.c_int64), ("pair_lj", C.c_int64), ("pair_es", C.c_int64),
                ("pair_pot", C.c_int64), ("far_terms", C.c_int64),
                ("pair_es_nolj", C.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


TRAJ_OUT_DTYPE = np.dtype([("chi", "<f8"), ("de_pct", "<f8"), ("steps", "<i4"),
                           ("status", "<u4")])
TRAJ_IN_DTYPE = np.dtype([("b", "<f8"), ("phi", "<f8"), ("theta", "<f8"),
                          ("gamma", "<f8"), ("g", "<f8")])
assert TRAJ_OUT_DTYPE.itemsize == C.sizeof(TrajOut)
assert TRAJ_IN_DTYPE.itemsize == C.sizeof(TrajIn)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def vptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


@dataclass
class MoleculeArrays:
    """Owning numpy arrays behind a `Molecule` view (file order, rotated)."""

    xyz: np.ndarray            # (n, 3)
    charge: np.ndarray
    sig6: np.ndarray
    eps24m: np.ndarray
    eps4: np.ndarray
    cluster_offset: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int32))
    cluster_atoms: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    cluster_pos: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    cluster_radius: np.ndarray = field(default_factory=lambda: np.zeros(0))
    cluster_charge: np.ndarray = field(default_factory=lambda: np.zeros(0))
    cluster_dipole: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    cluster_quad: np.ndarray = field(default_factory=lambda: np.zeros((0, 9)))
    cluster_replaced: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))

    def __post_init__(self):
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        self.xyz = f64(self.xyz).reshape(-1, 3)
        self._x = f64(self.xyz[:, 0])
        self._y = f64(self.xyz[:, 1])
        self._z = f64(self.xyz[:, 2])
        for k in ("charge", "sig6", "eps24m", "eps4", "cluster_radius", "cluster_charge"):
            setattr(self, k, f64(getattr(self, k)))
        self.cluster_pos = f64(self.cluster_pos).reshape(-1, 3)
        self.cluster_dipole = f64(self.cluster_dipole).reshape(-1, 3)
        self.cluster_quad = f64(self.cluster_quad).reshape(-1, 9)
        for k in ("cluster_offset", "cluster_atoms", "cluster_replaced"):
            setattr(self, k, i32(getattr(self, k)))

    @property
    def n_atoms(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def n_clusters(self) -> int:
        return int(self.cluster_offset.shape[0] - 1)

    def view(self) -> Molecule:
        m = Molecule()
        m.n_atoms = self.n_atoms
        m.x, m.y, m.z = dptr(self._x), dptr(self._y), dptr(self._z)
        m.charge, m.sig6 = dptr(self.charge), dptr(self.sig6)
        m.eps24m, m.eps4 = dptr(self.eps24m), dptr(self.eps4)
        m.n_clusters = self.n_clusters
        m.cluster_offset = iptr(self.cluster_offset)
        m.cluster_atoms = iptr(self.cluster_atoms)
        m.cluster_pos = dptr(self.cluster_pos)
        m.cluster_radius = dptr(self.cluster_radius)
        m.cluster_charge = dptr(self.cluster_charge)
        m.cluster_dipole = dptr(self.cluster_dipole)
        m.cluster_quad = dptr(self.cluster_quad)
        m.cluster_replaced = iptr(self.cluster_replaced)
        return m

    def to_npz_dict(self, prefix: str = "mol_") -> dict:
        return {prefix + k: v for k, v in (
            ("xyz", self.xyz), ("charge", self.charge), ("sig6", self.sig6),
            ("eps24m", self.eps24m), ("eps4", self.eps4),
            ("cluster_offset", self.cluster_offset), ("cluster_atoms", self.cluster_atoms),
            ("cluster_pos", self.cluster_pos), ("cluster_radius", self.cluster_radius),
            ("cluster_charge", self.cluster_charge), ("cluster_dipole", self.cluster_dipole),
            ("cluster_quad", self.cluster_quad), ("cluster_replaced", self.cluster_replaced))}

    @classmethod
    def from_npz(cls, d, prefix: str = "mol_") -> "MoleculeArrays":
        keys = ("xyz", "charge", "sig6", "eps24m", "eps4", "cluster_offset", "cluster_atoms",
                "cluster_pos", "cluster_radius", "cluster_charge", "cluster_dipole",
                "cluster_quad", "cluster_replaced")
        return cls(**{k: np.array(d[prefix + k]) for k in keys})


PARAM_FIELDS = [k for k, _ in Params._fields_]


def params_to_dict(p: Params) -> dict:
    return {k: getattr(p, k) for k in PARAM_FIELDS}


def params_from_dict(d: dict) -> Params:
    p = Params()
    for k, t in Params._fields_:
        v = d[k]
        setattr(p, k, int(v) if t in (C.c_int32, C.c_int64) else float(v))
    return p


JOB_RUNNING, JOB_DONE = 1, 2


class JobStatus(C.Structure):
    _fields_ = [("job_id", C.c_int64), ("state", C.c_int32), ("rounds", C.c_int32),
                ("omega", C.c_double), ("se", C.c_double), ("rel_se", C.c_double),
                ("device_ms", C.c_double), ("sums", CcsSums)]
