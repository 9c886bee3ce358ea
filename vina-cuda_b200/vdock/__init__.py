"""Python binding of libvdock.so (the C ABI in include/vdock.h).

The CUDA kernels and host logic live in the shared library; this module
only marshals numpy arrays through ctypes.  Importing it does not touch the
GPU; creating a Context does, and fails loudly when the library or a CUDA
device is missing (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("VDOCK_LIB") or os.path.join(PKG_DIR, "libvdock.so")  # VDOCK_LIB: another build

MAX_MODES = 20
MAX_TORS = 48
DEFAULT_WEIGHTS = (-0.035579, -0.005156, 0.840245, -0.035069, -0.587439, 5 * 0.05846 / 0.1 - 1)

_lib = None
_dp, _ip, _fp, _vp = C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_float), C.c_void_p


class VdockError(RuntimeError):
    pass


class LigandDesc(C.Structure):
    _fields_ = [("n_atoms", C.c_int32), ("n_nodes", C.c_int32), ("n_pairs", C.c_int32),
                ("xyz", _dp), ("xs", _ip), ("el", _ip), ("atom_node", _ip), ("node_parent", _ip),
                ("node_origin_atom", _ip), ("node_axis_atom", _ip), ("pairs", _ip),
                ("num_tors", C.c_double)]


class EvalParams(C.Structure):
    _fields_ = [("v_intra", C.c_double), ("v_inter", C.c_double), ("slope", C.c_double)]


class SearchParams(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("n_chains", C.c_int32), ("search_depth", C.c_int32),
                ("max_bfgs_steps", C.c_int32), ("num_modes", C.c_int32), ("energy_range", C.c_double),
                ("hunt_cap", C.c_double * 3), ("temperature", C.c_double), ("amplitude", C.c_double),
                ("min_rmsd", C.c_double), ("refine", C.c_int32), ("launch_shape", C.c_int32),
                ("dense_bfgs", C.c_int32), ("visited_history", C.c_int32)]


class DockResult(C.Structure):
    _fields_ = [("n_modes", C.c_int32), ("ntors", C.c_int32), ("energy", C.c_float * MAX_MODES),
                ("rmsd_lb", C.c_float * MAX_MODES), ("rmsd_ub", C.c_float * MAX_MODES),
                ("pose", (C.c_float * (7 + MAX_TORS)) * MAX_MODES), ("bfgs_evals", C.c_int64)]


class Stats(C.Structure):
    _fields_ = [("bfgs_evals", C.c_int64), ("grid_ms", C.c_double), ("dock_ms", C.c_double),
                ("post_ms", C.c_double), ("dock_warps_per_block", C.c_int32), ("dock_blocks", C.c_int32),
                ("dock_shape", C.c_int32), ("grid_shape", C.c_int32), ("graph_launches", C.c_int64),
                ("graph_instantiations", C.c_int64), ("scoring_ms", C.c_double), ("device_bytes", C.c_int64),
                ("pair_force_scale", C.c_double), ("cells_ms", C.c_double), ("ligand_bytes", C.c_int64)]


EXPORTS = [
    "vd_create", "vd_destroy", "vd_last_error", "vd_get_stats", "vd_set_memory_cap", "vd_set_scoring",
    "vd_set_scoring_device", "vd_set_receptor",
    "vd_set_box", "vd_grid_dims", "vd_build_grids", "vd_set_grid_shape", "vd_get_grid", "vd_add_ligand",
    "vd_add_ligands", "vd_ligand_info",
    "vd_clear_ligands", "vd_energy", "vd_energy_grad", "vd_energy_grad_device", "vd_energy_device",
    "vd_pose_coords",
    "vd_local_opt", "vd_mc_chains", "vd_mc_chains_noalloc", "vd_dock_plain", "vd_dock_batched", "vd_refine", "vd_score",
    "vd_rmsd_bounds", "vd_get_tables", "vd_pdbqt_ligand", "vd_pdbqt_receptor", "vd_pdbqt_write_model", "vd_pdbqt_free",
    "vd_conf_to_coords",
]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise VdockError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}`")
        L = C.CDLL(LIB_PATH)
        L.vd_last_error.restype = C.c_char_p
        L.vd_create.argtypes = [C.POINTER(_vp), C.c_int]
        L.vd_destroy.argtypes = [_vp]
        L.vd_get_stats.argtypes = [_vp, C.POINTER(Stats)]
        L.vd_set_scoring.argtypes = [_vp, _dp]
        L.vd_set_scoring_device.argtypes = [_vp, _dp]
        L.vd_set_memory_cap.argtypes = [_vp, C.c_int64]
        L.vd_set_receptor.argtypes = [_vp, C.c_int32, _dp, _ip]
        L.vd_set_box.argtypes = [_vp, _dp, _dp]
        L.vd_grid_dims.argtypes = [_vp, _ip, _dp, _dp]
        L.vd_build_grids.argtypes = [_vp, _ip, C.c_int32]
        L.vd_get_grid.argtypes = [_vp, C.c_int32, _fp]
        L.vd_set_grid_shape.argtypes = [_vp, C.c_int32]
        L.vd_add_ligand.argtypes = [_vp, C.POINTER(LigandDesc), _ip]
        L.vd_add_ligands.argtypes = [_vp, C.POINTER(LigandDesc), C.c_int32, C.POINTER(C.c_int32)]
        L.vd_ligand_info.argtypes = [_vp, C.c_int32, _ip, _ip, _ip]
        L.vd_clear_ligands.argtypes = [_vp]
        L.vd_energy.argtypes = [_vp, C.c_int32, C.c_int32, _fp, C.POINTER(EvalParams), _fp]
        L.vd_energy_grad.argtypes = [_vp, C.c_int32, C.c_int32, _fp, C.POINTER(EvalParams), _fp, _fp]
        L.vd_energy_grad_device.argtypes = [_vp, C.c_int32, C.c_int32, _vp, C.POINTER(EvalParams), _vp, _vp, _vp]
        L.vd_energy_device.argtypes = [_vp, C.c_int32, C.c_int32, _vp, C.POINTER(EvalParams), _vp, _vp]
        L.vd_pose_coords.argtypes = [_vp, C.c_int32, C.c_int32, _fp, _fp]
        L.vd_local_opt.argtypes = [_vp, C.c_int32, C.c_int32, _fp, C.POINTER(EvalParams), C.c_int32, _fp,
                                   C.POINTER(C.c_int64)]
        L.vd_mc_chains.argtypes = [_vp, C.c_int32, C.POINTER(SearchParams), _fp, _fp, C.POINTER(C.c_int64)]
        L.vd_mc_chains_noalloc.argtypes = [_vp, C.c_int32, C.POINTER(SearchParams), _fp, _fp, C.POINTER(C.c_int64)]
        L.vd_dock_plain.argtypes = [_vp, C.c_int32, C.POINTER(SearchParams), C.POINTER(DockResult)]
        L.vd_dock_batched.argtypes = [_vp, _ip, C.c_int32, C.POINTER(SearchParams), C.POINTER(DockResult)]
        L.vd_refine.argtypes = [_vp, C.c_int32, C.c_int32, _fp, C.c_int32, _fp]
        L.vd_score.argtypes = [_vp, C.c_int32, C.c_int32, _fp, _fp, _fp]
        L.vd_rmsd_bounds.argtypes = [_vp, C.c_int32, C.c_int32, _fp, _fp, _fp]
        L.vd_get_tables.argtypes = [_vp, _dp, _dp, _dp]
        for name in ("vd_create", "vd_destroy", "vd_get_stats", "vd_set_memory_cap", "vd_set_scoring", "vd_set_scoring_device",
                     "vd_set_receptor",
                     "vd_set_box", "vd_grid_dims", "vd_build_grids", "vd_set_grid_shape", "vd_get_grid", "vd_add_ligand",
                     "vd_ligand_info", "vd_clear_ligands", "vd_energy", "vd_energy_grad",
                     "vd_energy_grad_device", "vd_energy_device", "vd_pose_coords", "vd_local_opt",
                     "vd_mc_chains", "vd_mc_chains_noalloc", "vd_dock_plain", "vd_dock_batched", "vd_refine", "vd_score", "vd_rmsd_bounds", "vd_get_tables"):
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise VdockError(f"vdock error {status}: {lib().vd_last_error().decode()}")


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_fp)


def search_params(seed=0, n_chains=8192, search_depth=0, max_bfgs_steps=0, num_modes=9,
                  energy_range=3.0, hunt_cap=(10, 10, 10), temperature=1.2, amplitude=2.0,
                  min_rmsd=1.0, refine=1, launch_shape=0, dense_bfgs=0, visited_history=0):
    s = SearchParams()
    s.seed, s.n_chains, s.search_depth, s.max_bfgs_steps = seed, n_chains, search_depth, max_bfgs_steps
    s.num_modes, s.energy_range = num_modes, energy_range
    for i in range(3):
        s.hunt_cap[i] = hunt_cap[i]
    s.temperature, s.amplitude, s.min_rmsd, s.refine = temperature, amplitude, min_rmsd, refine
    s.launch_shape = launch_shape
    s.dense_bfgs = int(dense_bfgs)
    s.visited_history = int(visited_history)
    return s


def eval_params(v_intra=10.0, v_inter=10.0, slope=1e6):
    e = EvalParams()
    e.v_intra, e.v_inter, e.slope = v_intra, v_inter, slope
    return e


class Context:
    """One vd_ctx: a CUDA device with its receptor, box, maps and ligands."""

    def __init__(self, device=0, weights=None):
        self.L = lib()
        h = _vp()
        _check(self.L.vd_create(C.byref(h), device))
        self.h = h
        self._keep = []
        self.ntors = []
        self.n_heavy = []
        if weights is not None:
            w, wp = _d(weights)
            _check(self.L.vd_set_scoring(self.h, wp))

    def close(self):
        if getattr(self, "h", None):
            self.L.vd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stats(self):
        s = Stats()
        _check(self.L.vd_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def set_memory_cap(self, nbytes):
        """Cap on the context's device memory (0 = none); past it calls raise with status 6."""
        _check(self.L.vd_set_memory_cap(self.h, int(nbytes)))

    def set_scoring(self, weights, device=False):
        """New scoring weights (gauss1, gauss2, repulsion, hydrophobic, hydrogen,
        rotor); device=True builds the tables on the GPU."""
        w, wp = _d(np.asarray(weights, dtype=np.float64))
        fn = self.L.vd_set_scoring_device if device else self.L.vd_set_scoring
        _check(fn(self.h, wp))

    def tables(self):
        n = 153 * 2051
        f, fp = _d(np.zeros(n))
        e, ep = _d(np.zeros(n))
        d, dp = _d(np.zeros(n))
        _check(self.L.vd_get_tables(self.h, fp, ep, dp))
        return f.reshape(153, 2051), e.reshape(153, 2051), d.reshape(153, 2051)

    def set_receptor(self, xyz, xs):
        x, xp = _d(np.asarray(xyz).reshape(-1, 3))
        t, tp = _i(xs)
        _check(self.L.vd_set_receptor(self.h, len(t), xp, tp))

    def set_box(self, center, size):
        c, cp = _d(center)
        s, sp = _d(size)
        _check(self.L.vd_set_box(self.h, cp, sp))

    def grid_dims(self):
        n, npp = _i(np.zeros(3))
        b, bp = _d(np.zeros(3))
        e, ep = _d(np.zeros(3))
        _check(self.L.vd_grid_dims(self.h, npp, bp, ep))
        return n.copy(), b.copy(), e.copy()

    def build_grids(self, types):
        t, tp = _i(types)
        _check(self.L.vd_build_grids(self.h, tp, len(t)))

    def set_grid_shape(self, shape):
        _check(self.L.vd_set_grid_shape(self.h, shape))

    def grid(self, t):
        n, _, _ = self.grid_dims()
        out, op = _f(np.zeros(int(np.prod(n)), dtype=np.float32))
        _check(self.L.vd_get_grid(self.h, t, op))
        return out.reshape(n[2], n[1], n[0])

    @staticmethod
    def _desc(desc, s, keep):
        s.n_atoms = int(desc["n_atoms"])
        s.n_nodes = int(len(desc["node_parent"]))
        s.n_pairs = int(len(desc["pairs"]))
        keep["xyz"], s.xyz = _d(desc["xyz"])
        for k in ("xs", "el", "atom_node", "node_parent", "node_origin_atom", "node_axis_atom", "pairs"):
            keep[k], p = _i(desc[k])
            setattr(s, k, p)
        s.num_tors = float(desc["num_tors"])

    def _registered(self, lid, keep):
        nh, nt, npair = C.c_int32(), C.c_int32(), C.c_int32()
        _check(self.L.vd_ligand_info(self.h, lid, C.byref(nh), C.byref(nt), C.byref(npair)))
        self._keep.append(keep)
        self.ntors.append(nt.value)
        self.n_heavy.append(nh.value)

    def add_ligand(self, desc):
        keep = {}
        s = LigandDesc()
        self._desc(desc, s, keep)
        lid = C.c_int32(-1)
        _check(self.L.vd_add_ligand(self.h, C.byref(s), C.byref(lid)))
        self._registered(lid.value, keep)
        return lid.value

    def add_ligands(self, descs):
        """vd_add_ligands: the list built on host threads, ids in list order."""
        n = len(descs)
        arr = (LigandDesc * max(n, 1))()
        keeps = [{} for _ in range(n)]
        for i, d in enumerate(descs):
            self._desc(d, arr[i], keeps[i])
        ids = (C.c_int32 * max(n, 1))()
        _check(self.L.vd_add_ligands(self.h, arr, n, ids))
        for i in range(n):
            self._registered(ids[i], keeps[i])
        return [ids[i] for i in range(n)]

    def clear_ligands(self):
        _check(self.L.vd_clear_ligands(self.h))
        self._keep, self.ntors, self.n_heavy = [], [], []

    def energy(self, lig, poses, ep=None):
        p, pp = _f(poses)
        n = p.shape[0]
        e, epp = _f(np.zeros(n, dtype=np.float32))
        _check(self.L.vd_energy(self.h, lig, n, pp, C.byref(ep or eval_params()), epp))
        return e

    def energy_grad(self, lig, poses, ep=None):
        p, pp = _f(poses)
        n = p.shape[0]
        e, epp = _f(np.zeros(n, dtype=np.float32))
        g, gp = _f(np.zeros((n, 6 + self.ntors[lig]), dtype=np.float32))
        _check(self.L.vd_energy_grad(self.h, lig, n, pp, C.byref(ep or eval_params()), epp, gp))
        return e, g

    def energy_grad_device(self, lig, n, poses_ptr, e_ptr, g_ptr, stream_ptr=0, ep=None):
        _check(self.L.vd_energy_grad_device(self.h, lig, n, _vp(poses_ptr), C.byref(ep or eval_params()),
                                            _vp(e_ptr), _vp(g_ptr), _vp(stream_ptr or None)))

    def energy_device(self, lig, n, poses_ptr, e_ptr, stream_ptr=0, ep=None):
        _check(self.L.vd_energy_device(self.h, lig, n, _vp(poses_ptr), C.byref(ep or eval_params()), _vp(e_ptr),
                                       _vp(stream_ptr or None)))

    def pose_coords(self, lig, poses):
        p, pp = _f(poses)
        n = p.shape[0]
        x, xp = _f(np.zeros((n, self.n_heavy[lig], 3), dtype=np.float32))
        _check(self.L.vd_pose_coords(self.h, lig, n, pp, xp))
        return x

    def local_opt(self, lig, poses, max_steps, ep=None):
        p, pp = _f(np.array(poses, dtype=np.float32))
        n = p.shape[0]
        e, epp = _f(np.zeros(n, dtype=np.float32))
        ev = C.c_int64()
        _check(self.L.vd_local_opt(self.h, lig, n, pp, C.byref(ep or eval_params()), max_steps, epp, C.byref(ev)))
        return e, p, ev.value

    def mc_chains(self, lig, sp):
        n = sp.n_chains
        p, pp = _f(np.zeros((n, 7 + self.ntors[lig]), dtype=np.float32))
        e, epp = _f(np.zeros(n, dtype=np.float32))
        ev = C.c_int64()
        _check(self.L.vd_mc_chains(self.h, lig, C.byref(sp), pp, epp, C.byref(ev)))
        return p, e, ev.value

    def mc_chains_noalloc(self, lig, sp):
        """vd_mc_chains through the entry point that allocates no device memory."""
        n = sp.n_chains
        p, pp = _f(np.zeros((n, 7 + self.ntors[lig]), dtype=np.float32))
        e, epp = _f(np.zeros(n, dtype=np.float32))
        ev = C.c_int64()
        _check(self.L.vd_mc_chains_noalloc(self.h, lig, C.byref(sp), pp, epp, C.byref(ev)))
        return p, e, ev.value

    @staticmethod
    def _results(res, n):
        out = []
        for r in res[:n]:
            k = r.n_modes
            nc = 7 + r.ntors
            out.append(dict(energy=np.array(r.energy[:k]), rmsd_lb=np.array(r.rmsd_lb[:k]),
                            rmsd_ub=np.array(r.rmsd_ub[:k]),
                            pose=np.array([list(r.pose[i])[:nc] for i in range(k)], dtype=np.float32),
                            bfgs_evals=r.bfgs_evals))
        return out

    def dock_plain(self, lig, sp):
        r = (DockResult * 1)()
        _check(self.L.vd_dock_plain(self.h, lig, C.byref(sp), r))
        return self._results(r, 1)[0]

    def dock_batched(self, ligs, sp):
        l, lp = _i(ligs)
        r = (DockResult * len(l))()
        _check(self.L.vd_dock_batched(self.h, lp, len(l), C.byref(sp), r))
        return self._results(r, len(l))

    def refine(self, lig, poses, max_steps=0):
        p, pp = _f(np.array(poses, dtype=np.float32))
        n = p.shape[0]
        e, epp = _f(np.zeros(n, dtype=np.float32))
        _check(self.L.vd_refine(self.h, lig, n, pp, max_steps, epp))
        return e, p

    def score(self, lig, poses):
        p, pp = _f(poses)
        n = p.shape[0]
        a, ap = _f(np.zeros(n, dtype=np.float32))
        i, ipp = _f(np.zeros(n, dtype=np.float32))
        _check(self.L.vd_score(self.h, lig, n, pp, ap, ipp))
        return a, i

    def rmsd_bounds(self, lig, poses):
        """RMSD lower and upper bounds of each pose to pose 0 (heavy atoms)."""
        p, pp = _f(poses)
        n = p.shape[0]
        lb, lbp = _f(np.zeros(n, dtype=np.float32))
        ub, ubp = _f(np.zeros(n, dtype=np.float32))
        _check(self.L.vd_rmsd_bounds(self.h, lig, n, pp, lbp, ubp))
        return lb, ub
