"""Python bindings of oracle/_ref/libcosims_ref.so: the unmodified reference
sources driven through oracle/ref_harness.cpp.  TEST INFRASTRUCTURE ONLY.

Available only where the reference checkout exists (the library is built from
it by oracle/Makefile); `available()` says whether it can be used.  Used to
generate tests/golden fixtures and to pin the oracle restatement.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

from cosims_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcosims_ref.so")
BIN_PATH = os.path.join(HERE, "_ref", "cosims")
# the CoSIMS checkout: $COSIMS_REF, else the directory `reference` beside this
# repository
REF_ROOT = os.environ.get("COSIMS_REF") or os.path.normpath(
    os.path.join(HERE, "..", "..", "reference"))

# order of ref_get_scalars (ref_harness.cpp)
SCALARS = ("mu totalMass beta g_min g_max vdist_max vdist_norm ell_a ell_b ell_c b_max "
           "start_dist const1 const2 dipole_scalar force_type r_disp r_mp multipole_order dt "
           "temp traj_num iterations print_rate projection charged total_charge enlarge "
           "maxX maxY maxZ centerX centerY centerZ max_cluster_size multipole "
           "dispersion_cutoff").split()

_LIB = None


def build() -> bool:
    if not os.path.isdir(os.path.join(REF_ROOT, "src")):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_ROOT}"], check=True)
    return os.path.exists(LIB_PATH)


def available() -> bool:
    return os.path.exists(LIB_PATH) or build()


def lib():
    global _LIB
    if _LIB is None:
        if not available():
            raise RuntimeError("reference harness not built (no reference checkout)")
        L = C.CDLL(LIB_PATH)
        L.ref_setup.argtypes = [C.c_char_p] * 4 + [C.c_longlong]
        L.ref_get_atoms.argtypes = [C.c_void_p] * 6
        L.ref_get_scalars.argtypes = [C.c_void_p, C.c_int]
        L.ref_get_cluster.argtypes = [C.c_int] + [C.c_void_p] * 7
        L.ref_get_boundary.argtypes = [C.c_void_p]
        L.ref_force.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        L.ref_potential.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        L.ref_run_list.argtypes = [C.c_int] + [C.c_void_p] * 6
        L.ref_sample.argtypes = [C.c_int, C.c_ulonglong, C.c_uint] + [C.c_void_p] * 4
        _LIB = L
    return _LIB


class RefSetup:
    """The reference's setup of one molecule, read back through the harness.

    The harness keeps one molecule live at a time (the reference's globals);
    a new `RefSetup` replaces the previous one.
    """

    def __init__(self, mol_path: str, input_path: str = "", atom_path: str = "",
                 seed: int = 123456789, workdir: str | None = None):
        L = lib()
        self.workdir = workdir or tempfile.mkdtemp(prefix="cosims_ref_")
        # the reference prints its whole setup log to stdout; keep it out of the way
        fd = os.dup(1)
        try:
            with open(os.path.join(self.workdir, "stdout.txt"), "w") as f:
                os.dup2(f.fileno(), 1)
                rc = L.ref_setup(mol_path.encode(), input_path.encode(), atom_path.encode(),
                                 self.workdir.encode(), int(seed))
        finally:
            os.dup2(fd, 1)
            os.close(fd)
        if rc != 0:
            raise RuntimeError(f"ref_setup failed with {rc}")
        s = np.zeros(64)
        n = L.ref_get_scalars(abi.vptr(s), 64)
        self.scalars = dict(zip(SCALARS, s[:n].tolist()))
        na = L.ref_num_atoms()
        xyz = np.zeros((na, 3))
        q, sig6, e24, e4, mass = (np.zeros(na) for _ in range(5))
        L.ref_get_atoms(abi.vptr(xyz), abi.vptr(q), abi.vptr(sig6), abi.vptr(e24),
                        abi.vptr(e4), abi.vptr(mass))
        self.mass = mass
        nc = L.ref_num_clusters()
        off = [0]
        members, pos, rad, cq, dip, quad, rep = [], [], [], [], [], [], []
        for k in range(nc):
            sz = L.ref_cluster_size(k)
            mem = np.zeros(sz, np.int32)
            p3, d3, q9 = np.zeros(3), np.zeros(3), np.zeros(9)
            r, qq, rp = C.c_double(), C.c_double(), C.c_int()
            L.ref_get_cluster(k, abi.vptr(mem), abi.vptr(p3), C.byref(r), C.byref(qq),
                              abi.vptr(d3), abi.vptr(q9), C.byref(rp))
            members.append(mem)
            off.append(off[-1] + sz)
            pos.append(p3); rad.append(r.value); cq.append(qq.value)
            dip.append(d3); quad.append(q9); rep.append(rp.value)
        self.mol = abi.MoleculeArrays(
            xyz=xyz, charge=q, sig6=sig6, eps24m=e24, eps4=e4,
            cluster_offset=np.array(off, np.int32),
            cluster_atoms=np.concatenate(members).astype(np.int32) if members else np.zeros(0, np.int32),
            cluster_pos=np.array(pos).reshape(-1, 3), cluster_radius=np.array(rad),
            cluster_charge=np.array(cq), cluster_dipole=np.array(dip).reshape(-1, 3),
            cluster_quad=np.array(quad).reshape(-1, 9), cluster_replaced=np.array(rep, np.int32))
        nb = L.ref_num_boundary()
        self.boundary = np.zeros((nb, 3))
        if nb:
            L.ref_get_boundary(abi.vptr(self.boundary))
        sc = self.scalars
        self.params = abi.params_from_dict(dict(
            force_type=sc["force_type"], multipole_order=sc["multipole_order"],
            projection=sc["projection"], charged=sc["charged"], dt=sc["dt"], mu=sc["mu"],
            dipole_scalar=sc["dipole_scalar"], r_disp=sc["r_disp"], r_mp=sc["r_mp"],
            ell_a=sc["ell_a"], ell_b=sc["ell_b"], ell_c=sc["ell_c"], b_max=sc["b_max"],
            start_dist=sc["start_dist"], g_min=sc["g_min"], g_max=sc["g_max"],
            vdist_a=sc["beta"] / 2.0, vdist_norm=sc["vdist_norm"],
            vdist_max=sc["vdist_max"], ccs_const=sc["const1"] * sc["const2"], max_steps=0))

    def force(self, pos: np.ndarray) -> np.ndarray:
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        out = np.zeros_like(pos)
        lib().ref_force(pos.shape[0], abi.vptr(pos), abi.vptr(out))
        return out

    def potential(self, pos: np.ndarray) -> np.ndarray:
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        out = np.zeros(pos.shape[0])
        lib().ref_potential(pos.shape[0], abi.vptr(pos), abi.vptr(out))
        return out

    def run_list(self, pos0: np.ndarray, vel0: np.ndarray):
        pos0 = np.ascontiguousarray(pos0, dtype=np.float64).reshape(-1, 3)
        vel0 = np.ascontiguousarray(vel0, dtype=np.float64).reshape(-1, 3)
        n = pos0.shape[0]
        chi, de = np.zeros(n), np.zeros(n)
        succ, steps = np.zeros(n, np.int32), np.zeros(n, np.int32)
        lib().ref_run_list(n, abi.vptr(pos0), abi.vptr(vel0), abi.vptr(chi), abi.vptr(succ),
                           abi.vptr(steps), abi.vptr(de))
        return chi, succ, steps, de

    def sample(self, n: int, seed: int, rand_seed: int = 1):
        """monteTraj::setUpTraj driven by mt19937_64(seed): inputs, start states, hits."""
        vals = np.zeros((n, 5))
        pos0, vel0 = np.zeros((n, 3)), np.zeros((n, 3))
        hit = np.zeros(n, np.int32)
        lib().ref_sample(n, seed, rand_seed, abi.vptr(vals), abi.vptr(pos0), abi.vptr(vel0), abi.vptr(hit))
        inputs = np.zeros(n, abi.TRAJ_IN_DTYPE)
        for i, k in enumerate(("b", "phi", "theta", "gamma", "g")):
            inputs[k] = vals[:, i]
        return inputs, pos0, vel0, hit
