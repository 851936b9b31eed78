"""Python binding of the host-side C ABI (include/cosims_host.h).

`Config` mirrors the reference's input-file parameters (fileParams), `Setup`
its per-molecule setup (molecule2 import and rotation, impactParam boundary
and ellipsoid, PCM clusters, velocity distribution); both run in the C++
library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .engine import check, lib

KEY_NAME, KEY_CHARGE, KEY_PRINT_RATE, KEY_THREADS, KEY_SEED = (1 << i for i in range(5))


class ConfigStruct(C.Structure):
    _fields_ = [
        ("name", C.c_char * 256), ("dir", C.c_char * 1024),
        ("dt", C.c_double), ("temp", C.c_double), ("traj", C.c_int64), ("iter", C.c_int32),
        ("threads", C.c_int32), ("seed", C.c_int64), ("seed_set", C.c_int32),
        ("gmax", C.c_double), ("gmin", C.c_double),
        ("print_mol", C.c_int32), ("proj", C.c_int32), ("print_traj", C.c_int32),
        ("print_traj_fail", C.c_int32), ("print_data", C.c_int32),
        ("print_data_fail", C.c_int32),
        ("dispersion_cutoff", C.c_int32), ("dispersion_radius", C.c_double),
        ("multipole", C.c_int32), ("multipole_radius", C.c_double),
        ("multipole_order", C.c_int32), ("print_rate", C.c_int32),
        ("display_progress", C.c_int32), ("max_cluster_size", C.c_int32),
        ("charge", C.c_double), ("charged", C.c_int32), ("debugging", C.c_int32),
        ("changed", C.c_uint32),
    ]


class SetupInfo(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32), ("n_clusters", C.c_int32), ("n_boundary", C.c_int32),
        ("force_type", C.c_int32),
        ("total_mass", C.c_double), ("mu", C.c_double), ("total_charge", C.c_double),
        ("center", C.c_double * 3), ("radius_gyration", C.c_double),
        ("inertia", C.c_double * 9), ("rotation", C.c_double * 9),
        ("dipole", C.c_double * 3), ("quadrupole", C.c_double * 9),
        ("ell_a", C.c_double), ("ell_b", C.c_double), ("ell_c", C.c_double),
        ("ell_unc", C.c_double * 3),
        ("rmsd", C.c_double), ("avg_axes", C.c_double), ("avg_axes_unc", C.c_double),
        ("surf_area", C.c_double), ("surf_area_unc", C.c_double), ("enlarge", C.c_double),
        ("cov", C.c_double * 9),
        ("b_max", C.c_double), ("g_min", C.c_double), ("g_max", C.c_double),
        ("g_mean", C.c_double), ("g_mode", C.c_double), ("pct_used", C.c_double),
        ("beta", C.c_double), ("ccs_const", C.c_double), ("r_disp", C.c_double),
        ("r_mp", C.c_double),
        ("centers_replaced", C.c_int32),
        ("avg_cluster_size", C.c_double), ("avg_cluster_radius", C.c_double),
        ("setup_ms", C.c_double * 6),
    ]

    def as_dict(self) -> dict:
        out = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            out[k] = list(v) if isinstance(v, C.Array) else v
        return out


_BOUND = False


def _bind():
    global _BOUND
    if _BOUND:
        return lib()
    L = lib()
    P, V = C.POINTER, C.c_void_p
    sig = {
        "cosims_config_defaults": (C.c_int, [P(ConfigStruct), C.c_char_p]),
        "cosims_config_read": (C.c_int, [P(ConfigStruct), C.c_char_p, C.c_char_p, C.c_char_p,
                                         C.c_int64]),
        "cosims_setup_create": (C.c_int, [P(ConfigStruct), C.c_char_p, C.c_char_p, C.c_char_p,
                                          C.c_int64, P(V)]),
        "cosims_setup_create_device": (C.c_int, [P(ConfigStruct), C.c_char_p, C.c_char_p,
                                                 C.c_int32, C.c_char_p, C.c_int64, P(V)]),
        "cosims_setup_create_structure": (C.c_int, [P(ConfigStruct), C.c_char_p, C.c_char_p,
                                                    C.c_int32, C.c_int32, C.c_char_p,
                                                    C.c_int64, P(V)]),
        "cosims_molecule_file_structures": (C.c_int, [C.c_char_p, P(C.c_int32)]),
        "cosims_setup_molecule": (C.c_int, [V, P(abi.Molecule), P(abi.Params)]),
        "cosims_setup_get_info": (C.c_int, [V, P(SetupInfo)]),
        "cosims_setup_boundary": (C.c_int64, [V, V, C.c_int64]),
        "cosims_setup_atom_symbol": (C.c_char_p, [V, C.c_int32]),
        "cosims_setup_destroy": (None, [V]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _BOUND = True
    return L


class Config:
    """Input-file parameters (fileParams.cpp:203-510)."""

    def __init__(self, mol_path: str, input_path: str | None = None, seed: int | None = None,
                 threads: int | None = None):
        L = _bind()
        self.s = ConfigStruct()
        if seed is not None:
            self.s.seed = int(seed)
            self.s.changed |= KEY_SEED
        if threads is not None:
            self.s.threads = int(threads)
            self.s.changed |= KEY_THREADS
        self.log = ""
        if input_path:
            buf = C.create_string_buffer(1 << 16)
            check(L.cosims_config_read(C.byref(self.s), input_path.encode(), mol_path.encode(),
                                       buf, len(buf)))
            self.log = buf.value.decode(errors="replace")
        else:
            check(L.cosims_config_defaults(C.byref(self.s), mol_path.encode()))

    def __getattr__(self, k):
        v = getattr(object.__getattribute__(self, "s"), k)
        return v.decode() if isinstance(v, bytes) else v

    def set(self, **kw):
        for k, v in kw.items():
            setattr(self.s, k, v)
        return self


class Setup:
    """Per-molecule setup: the molecule and path scalars the kernels consume."""

    def __init__(self, cfg: Config, mol_path: str, atom_path: str | None = None,
                 device: int | None = None, structure: int | None = None):
        """device: run the boundary ray march on this GPU (same result).
        structure: coordinate set of a multi-structure file (0-based)."""
        L = _bind()
        h = C.c_void_p()
        buf = C.create_string_buffer(1 << 16)
        if structure is not None:
            check(L.cosims_setup_create_structure(
                C.byref(cfg.s), mol_path.encode(), (atom_path or "").encode(), int(structure),
                -1 if device is None else int(device), buf, len(buf), C.byref(h)))
        elif device is None:
            check(L.cosims_setup_create(C.byref(cfg.s), mol_path.encode(),
                                        (atom_path or "").encode(), buf, len(buf), C.byref(h)))
        else:
            check(L.cosims_setup_create_device(C.byref(cfg.s), mol_path.encode(),
                                               (atom_path or "").encode(), int(device), buf,
                                               len(buf), C.byref(h)))
        self._h = h
        self.log = buf.value.decode(errors="replace")
        m, p = abi.Molecule(), abi.Params()
        check(L.cosims_setup_molecule(h, C.byref(m), C.byref(p)))
        self.params = p
        n, nc = m.n_atoms, m.n_clusters
        arr = lambda ptr, k: np.ctypeslib.as_array(ptr, shape=(k,)).copy()
        xyz = np.stack([arr(m.x, n), arr(m.y, n), arr(m.z, n)], axis=1)
        kw = dict(xyz=xyz, charge=arr(m.charge, n), sig6=arr(m.sig6, n),
                  eps24m=arr(m.eps24m, n), eps4=arr(m.eps4, n))
        if nc:
            kw.update(cluster_offset=arr(m.cluster_offset, nc + 1),
                      cluster_atoms=arr(m.cluster_atoms, n),
                      cluster_pos=arr(m.cluster_pos, 3 * nc), cluster_radius=arr(m.cluster_radius, nc),
                      cluster_charge=arr(m.cluster_charge, nc),
                      cluster_dipole=arr(m.cluster_dipole, 3 * nc),
                      cluster_quad=arr(m.cluster_quad, 9 * nc),
                      cluster_replaced=arr(m.cluster_replaced, nc))
        self.mol = abi.MoleculeArrays(**kw)
        info = SetupInfo()
        check(L.cosims_setup_get_info(h, C.byref(info)))
        self.info = info
        nb = L.cosims_setup_boundary(h, None, 0)
        self.boundary = np.zeros((nb, 3))
        L.cosims_setup_boundary(h, abi.vptr(self.boundary), nb)
        self.symbols = [L.cosims_setup_atom_symbol(h, i).decode() for i in range(n)]

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().cosims_setup_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def setup_from_files(mol_path: str, input_path: str | None = None, atom_path: str | None = None,
                     seed: int | None = None, threads: int | None = None,
                     device: int | None = None, structure: int | None = None) -> Setup:
    return Setup(Config(mol_path, input_path, seed=seed, threads=threads), mol_path, atom_path,
                 device=device, structure=structure)


def count_structures(mol_path: str) -> int:
    """Coordinate sets in an MFJ or PDB file (1 for a single-structure file)."""
    L = _bind()
    k = C.c_int32()
    check(L.cosims_molecule_file_structures(mol_path.encode(), C.byref(k)))
    return k.value


def setup_structures(mol_path: str, input_path: str | None = None,
                     atom_path: str | None = None, seed: int | None = None,
                     threads: int | None = None, device: int | None = None) -> list:
    """One Setup per coordinate set of a multi-structure file, each set up as
    a single-structure file of that set would be; feed them to engine.Batch."""
    cfg = Config(mol_path, input_path, seed=seed, threads=threads)
    return [Setup(cfg, mol_path, atom_path, device=device, structure=s)
            for s in range(count_structures(mol_path))]
