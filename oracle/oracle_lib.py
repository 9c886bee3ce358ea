"""ORACLE -- test infrastructure only: ctypes binding of liboracle.so.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It builds liboracle.so from vina_oracle.cpp on first use when
the library is missing (make -C oracle).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

DEFAULT_WEIGHTS = (-0.035579, -0.005156, 0.840245, -0.035069, -0.587439,
                   5 * 0.05846 / 0.1 - 1)  # main.cpp:649-654, 856-862

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "vina_oracle.cpp")
        if (not os.path.exists(LIB_PATH) or
                os.path.getmtime(LIB_PATH) < os.path.getmtime(src)):
            build()
        L = C.CDLL(LIB_PATH)
        dp, ip, vp = C.POINTER(C.c_double), C.POINTER(C.c_int32), C.c_void_p
        L.or_create.restype = vp
        L.or_create.argtypes = [dp]
        L.or_destroy.argtypes = [vp]
        L.or_tables.argtypes = [vp, dp, dp, dp]
        L.or_set_receptor.argtypes = [vp, C.c_int, dp, ip]
        L.or_set_box.argtypes = [vp, dp, dp]
        L.or_grid_info.argtypes = [vp, ip, dp, dp]
        L.or_build_grids.argtypes = [vp, ip, C.c_int]
        L.or_get_grid.argtypes = [vp, C.c_int, dp]
        L.or_add_ligand.argtypes = [vp, vp]
        L.or_ligand_ntors.argtypes = [vp, C.c_int]
        L.or_term_values_coords.restype = None
        L.or_term_values_coords.argtypes = [vp, C.c_int, dp, dp]
        L.or_conf_independent.restype = C.c_double
        L.or_conf_independent.argtypes = [vp, C.c_int, C.c_double]
        L.or_maps_ready.restype = C.c_int
        L.or_maps_ready.argtypes = [vp, C.c_int]
        L.or_eval_deriv.restype = C.c_double
        L.or_eval_deriv.argtypes = [vp, C.c_int, dp, dp, C.c_double, dp]
        L.or_nc_eval_deriv.restype = C.c_double
        L.or_nc_eval_deriv.argtypes = [vp, C.c_int, dp, dp, C.c_double, dp]
        L.or_coords.argtypes = [vp, C.c_int, dp, dp]
        L.or_eval_intramolecular.restype = C.c_double
        L.or_eval_intramolecular.argtypes = [vp, C.c_int, dp, C.c_double]
        L.or_eval_adjusted.restype = C.c_double
        L.or_eval_adjusted.argtypes = [vp, C.c_int, dp, C.c_double]
        L.or_eval_adjusted_coords.restype = C.c_double
        L.or_eval_adjusted_coords.argtypes = [vp, C.c_int, dp, C.c_double]
        L.or_intramolecular_coords.restype = C.c_double
        L.or_intramolecular_coords.argtypes = [vp, C.c_int, dp]
        L.or_rmsd_upper.restype = C.c_double
        L.or_rmsd_upper.argtypes = [vp, C.c_int, dp, dp]
        L.or_rmsd_lower.restype = C.c_double
        L.or_rmsd_lower.argtypes = [vp, C.c_int, dp, dp]
        L.or_rilc_bfgs.restype = C.c_double
        L.or_rilc_bfgs.argtypes = [vp, C.c_int, dp, dp, C.c_double, C.c_int, C.POINTER(C.c_int64)]
        L.or_bfgs.restype = C.c_double
        L.or_bfgs.argtypes = [vp, C.c_int, dp, dp, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int64)]
        L.or_mc_chains.restype = C.c_int64
        L.or_mc_chains.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, dp, dp, C.c_int]
        L.or_init_conf.argtypes = [vp, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, dp]
        L.or_refine.restype = C.c_double
        L.or_refine.argtypes = [vp, C.c_int, dp, C.c_int, C.POINTER(C.c_int64)]
        L.or_cluster.restype = C.c_int
        L.or_cluster.argtypes = [vp, C.c_int, C.c_int, dp, dp, C.c_double, C.c_int, ip]
        L.or_grid_seconds.restype = C.c_double
        L.or_grid_seconds.argtypes = [vp, ip, C.c_int, C.c_int]
        L.or_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        _lib = L
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(C.POINTER(C.c_int32))


class OrLigand(C.Structure):
    _fields_ = [("n_atoms", C.c_int32), ("n_nodes", C.c_int32), ("n_pairs", C.c_int32),
                ("xyz", C.POINTER(C.c_double)), ("xs", C.POINTER(C.c_int32)),
                ("el", C.POINTER(C.c_int32)), ("atom_node", C.POINTER(C.c_int32)),
                ("node_parent", C.POINTER(C.c_int32)), ("node_origin_atom", C.POINTER(C.c_int32)),
                ("node_axis_atom", C.POINTER(C.c_int32)), ("pairs", C.POINTER(C.c_int32)),
                ("num_tors", C.c_double)]


class OrSearch(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("lig_uid", C.c_uint32), ("search_depth", C.c_int32),
                ("max_bfgs_steps", C.c_int32), ("hunt_cap", C.c_double * 3),
                ("slope", C.c_double), ("temperature", C.c_double), ("amplitude", C.c_double),
                ("dense", C.c_int32), ("visited", C.c_int32)]


class Oracle:
    """Double-precision restatement of the reference scoring/search code."""

    def __init__(self, weights=DEFAULT_WEIGHTS):
        self.L = lib()
        w, wp = _d(np.array(weights))
        self.h = self.L.or_create(wp)
        self._keep = []
        self.ntors = []

    def __del__(self):
        try:
            self.L.or_destroy(self.h)
        except Exception:
            pass

    def tables(self):
        n = 153 * 2051
        f, fp = _d(np.zeros(n))
        e, ep = _d(np.zeros(n))
        d, dp = _d(np.zeros(n))
        self.L.or_tables(self.h, fp, ep, dp)
        return f.reshape(153, 2051), e.reshape(153, 2051), d.reshape(153, 2051)

    def set_receptor(self, xyz, xs):
        x, xp = _d(np.asarray(xyz).reshape(-1, 3))
        t, tp = _i(xs)
        self.L.or_set_receptor(self.h, len(t), xp, tp)

    def set_box(self, center, size):
        c, cp = _d(center)
        s, sp = _d(size)
        self.L.or_set_box(self.h, cp, sp)

    def grid_info(self):
        n, npp = _i(np.zeros(3))
        b, bp = _d(np.zeros(3))
        e, ep = _d(np.zeros(3))
        self.L.or_grid_info(self.h, npp, bp, ep)
        return n.copy(), b.copy(), e.copy()

    def build_grids(self, types):
        t, tp = _i(types)
        assert self.L.or_build_grids(self.h, tp, len(t)) == 0

    def grid_seconds(self, types, threads):
        t, tp = _i(types)
        return self.L.or_grid_seconds(self.h, tp, len(t), threads)

    def grid(self, t):
        n, _, _ = self.grid_info()
        out, op = _d(np.zeros(int(np.prod(n))))
        assert self.L.or_get_grid(self.h, t, op) == 0
        return out.reshape(n[2], n[1], n[0])  # [z][y][x]

    def add_ligand(self, desc):
        keep = {}
        s = OrLigand()
        s.n_atoms = int(desc["n_atoms"])
        s.n_nodes = int(len(desc["node_parent"]))
        s.n_pairs = int(len(desc["pairs"]))
        for k in ("xyz",):
            keep[k], p = _d(desc[k])
            setattr(s, k, p)
        for k in ("xs", "el", "atom_node", "node_parent", "node_origin_atom", "node_axis_atom", "pairs"):
            keep[k], p = _i(desc[k])
            setattr(s, k, p)
        s.num_tors = float(desc["num_tors"])
        lig = self.L.or_add_ligand(self.h, C.byref(s))
        self._keep.append(keep)
        self.ntors.append(self.L.or_ligand_ntors(self.h, lig))
        return lig

    def _need_maps(self, lig):
        if not self.L.or_maps_ready(self.h, lig):
            raise RuntimeError("oracle: grid maps for the ligand's XS types are not built (build_grids)")

    def eval_deriv(self, lig, conf, v=(10, 10, 10), slope=1e6, noncache=False):
        if not noncache:
            self._need_maps(lig)
        c, cp = _d(conf)
        vv, vp = _d(v)
        g, gp = _d(np.zeros(6 + self.ntors[lig]))
        fn = self.L.or_nc_eval_deriv if noncache else self.L.or_eval_deriv
        e = fn(self.h, lig, cp, vp, slope, gp)
        return e, g

    def coords(self, lig, conf, n_atoms):
        c, cp = _d(conf)
        o, op = _d(np.zeros(3 * n_atoms))
        self.L.or_coords(self.h, lig, cp, op)
        return o.reshape(-1, 3)

    def intramolecular(self, lig, conf, v=1000.0):
        c, cp = _d(conf)
        return self.L.or_eval_intramolecular(self.h, lig, cp, v)

    def intramolecular_coords(self, lig, xyz):
        x, xp = _d(xyz)
        return self.L.or_intramolecular_coords(self.h, lig, xp)

    def eval_adjusted(self, lig, conf, intra_best):
        c, cp = _d(conf)
        return self.L.or_eval_adjusted(self.h, lig, cp, intra_best)

    def eval_adjusted_coords(self, lig, xyz, intra_best):
        x, xp = _d(xyz)
        return self.L.or_eval_adjusted_coords(self.h, lig, xp, intra_best)

    def term_values(self, lig, xyz):
        """Unweighted intermolecular terms of heavy-atom coordinates (--score_only breakdown)."""
        x, xp = _d(np.asarray(xyz, dtype=np.float64).ravel())
        out, op = _d(np.zeros(5))
        self.L.or_term_values_coords(self.h, lig, xp, op)
        return out.copy()

    def conf_independent(self, lig, x):
        return self.L.or_conf_independent(self.h, lig, float(x))

    def rmsd(self, lig, a, b):
        a, ap = _d(a)
        b, bp = _d(b)
        return self.L.or_rmsd_lower(self.h, lig, ap, bp), self.L.or_rmsd_upper(self.h, lig, ap, bp)

    def rilc_bfgs(self, lig, conf, max_steps, v=(10, 10, 10), slope=1e6):
        self._need_maps(lig)
        c, cp = _d(np.array(conf, dtype=np.float64))
        vv, vp = _d(v)
        ev = C.c_int64(0)
        e = self.L.or_rilc_bfgs(self.h, lig, cp, vp, slope, max_steps, C.byref(ev))
        return e, c.copy(), ev.value

    def bfgs(self, lig, conf, max_steps, v=(1000, 1000, 1000), slope=1e6, noncache=True):
        if not noncache:
            self._need_maps(lig)
        c, cp = _d(np.array(conf, dtype=np.float64))
        vv, vp = _d(v)
        ev = C.c_int64(0)
        e = self.L.or_bfgs(self.h, lig, cp, vp, slope, max_steps, int(noncache), C.byref(ev))
        return e, c.copy(), ev.value

    def init_conf(self, lig, seed, lig_uid, chain):
        c, cp = _d(np.zeros(7 + self.ntors[lig]))
        self.L.or_init_conf(self.h, lig, seed, lig_uid, chain, cp)
        return c.copy()

    def mc_chains(self, lig, seed, lig_uid, depth, bfgs_steps, chain_begin, chain_end,
                  threads=1, hunt_cap=(10, 10, 10), slope=1e6, temperature=1.2, amplitude=2.0, dense=False,
                  visited=False):
        self._need_maps(lig)
        s = OrSearch()
        s.seed, s.lig_uid, s.search_depth, s.max_bfgs_steps = seed, lig_uid, depth, bfgs_steps
        for i in range(3):
            s.hunt_cap[i] = hunt_cap[i]
        s.slope, s.temperature, s.amplitude = slope, temperature, amplitude
        s.dense = int(bool(dense))
        s.visited = int(bool(visited))
        n = chain_end - chain_begin
        nc = 7 + self.ntors[lig]
        conf, cp = _d(np.zeros(n * nc))
        e, ep = _d(np.zeros(n))
        evals = self.L.or_mc_chains(self.h, lig, C.byref(s), chain_begin, chain_end, cp, ep, threads)
        return conf.reshape(n, nc).copy(), e.copy(), evals

    def refine(self, lig, conf, max_steps):
        c, cp = _d(np.array(conf, dtype=np.float64))
        ev = C.c_int64(0)
        e = self.L.or_refine(self.h, lig, cp, max_steps, C.byref(ev))
        return e, c.copy(), ev.value

    def cluster(self, lig, confs, e, min_rmsd=1.0, max_keep=20):
        c, cp = _d(confs)
        ee, ep = _d(e)
        k, kp = _i(np.zeros(max_keep))
        nk = self.L.or_cluster(self.h, lig, len(ee), cp, ep, min_rmsd, max_keep, kp)
        return k[:nk].copy()


def philox(ctr, key):
    L = lib()
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    L.or_philox(c, k, o)
    return list(o)
