"""Host-side checks that need no GPU: the C-ABI library loads and exports
every entry point include/vdock.h declares, and its PDBQT ingestion,
typing, pair selection and host kinematics agree with the oracle."""
import ctypes as C
import gzip
import os
import re

import numpy as np
import pytest

import oracle_lib as O
import pdbqt_oracle as P

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    import vdock
    return vdock.lib()


def header_functions():
    text = open(os.path.join(REPO, "include", "vdock.h")).read()
    return sorted(set(re.findall(r"\b(vd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point(lib):
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    import vdock
    assert set(vdock.EXPORTS) <= set(names)


def test_checked_build_exports_the_same_entry_points():
    """libvdock_checked.so (make checked: device bounds checks) is a drop-in
    for libvdock.so: it loads without a GPU and exports every declared call."""
    path = os.path.join(REPO, "vina-cuda_b200", "libvdock_checked.so")
    if not os.path.exists(path):
        pytest.skip("checked build not made (make -C vina-cuda_b200 checked)")
    checked = C.CDLL(path)
    for n in header_functions():
        assert hasattr(checked, n), n


def fixture_text(golden_dir, name):
    return gzip.open(os.path.join(golden_dir, "pdbqt", name + ".gz"), "rt").read()


def parse_with_lib(lib, text):
    import vdock
    h = C.c_void_p()
    d = vdock.LigandDesc()
    lib.vd_pdbqt_ligand.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(vdock.LigandDesc)]
    lib.vd_pdbqt_ligand.restype = C.c_int
    st = lib.vd_pdbqt_ligand(text.encode(), C.byref(h), C.byref(d))
    assert st == 0, lib.vd_last_error()
    na, nn, npair = d.n_atoms, d.n_nodes, d.n_pairs
    arr = lambda p, n: np.ctypeslib.as_array(p, shape=(n,)).copy()
    out = dict(n_atoms=na, xyz=arr(d.xyz, 3 * na).reshape(-1, 3), xs=arr(d.xs, na), el=arr(d.el, na),
               atom_node=arr(d.atom_node, na), node_parent=arr(d.node_parent, nn),
               node_origin_atom=arr(d.node_origin_atom, nn), node_axis_atom=arr(d.node_axis_atom, nn),
               pairs=arr(d.pairs, 2 * npair).reshape(-1, 2), num_tors=d.num_tors)
    return h, d, out


@pytest.mark.parametrize("name", ["1u1b_ligand.pdbqt", "2bm2_ligand.pdbqt", "2er7_ligand.pdbqt"])
def test_ligand_parse_matches_oracle(lib, golden_dir, name):
    text = fixture_text(golden_dir, name)
    h, d, got = parse_with_lib(lib, text)
    ref = P.parse_ligand(text).descriptor()
    for k in ("xs", "el", "atom_node", "node_parent", "node_origin_atom", "node_axis_atom", "pairs"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    np.testing.assert_array_equal(got["xyz"], ref["xyz"])
    assert got["num_tors"] == ref["num_tors"]
    lib.vd_pdbqt_free(h)


def test_receptor_parse_matches_oracle(lib, golden_dir):
    text = fixture_text(golden_dir, "1u1b_protein.pdbqt")
    h = C.c_void_p()
    n = C.c_int32()
    xyz = C.POINTER(C.c_double)()
    xs = C.POINTER(C.c_int32)()
    lib.vd_pdbqt_receptor.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int32),
                                      C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.POINTER(C.c_int32))]
    assert lib.vd_pdbqt_receptor(text.encode(), C.byref(h), C.byref(n), C.byref(xyz), C.byref(xs)) == 0
    z = np.load(os.path.join(golden_dir, "kat_vina.npz"))
    np.testing.assert_array_equal(np.ctypeslib.as_array(xs, shape=(n.value,)), z["rec_xs"])
    np.testing.assert_array_equal(np.ctypeslib.as_array(xyz, shape=(3 * n.value,)).reshape(-1, 3), z["rec_xyz"])
    lib.vd_pdbqt_free(h)


def test_parse_errors_are_reported(lib):
    import vdock
    h = C.c_void_p()
    d = vdock.LigandDesc()
    bad = "ROOT\nATOM      1  C   UNL     1       0.000   0.000   0.000  0.00  0.00    +0.000 Xx\nENDROOT\nTORSDOF 0\n"
    assert lib.vd_pdbqt_ligand(bad.encode(), C.byref(h), C.byref(d)) == 5  # VD_ERR_PARSE
    assert b"not a valid AutoDock type" in lib.vd_last_error()
    missing = "ROOT\nATOM      1  C   UNL     1       0.000   0.000   0.000  0.00  0.00    +0.000 C \nENDROOT\n"
    assert lib.vd_pdbqt_ligand(missing.encode(), C.byref(h), C.byref(d)) == 5
    assert b"TORSDOF" in lib.vd_last_error()


def test_conf_to_coords_matches_oracle_and_writer_round_trips(lib, golden_dir):
    import vdock
    text = fixture_text(golden_dir, "1u1b_ligand.pdbqt")
    h, d, got = parse_with_lib(lib, text)
    orc = O.Oracle()
    orc.set_receptor(np.zeros((1, 3)), np.array([0], np.int32))
    orc.set_box([0, 0, 0], [10, 10, 10])
    lid = orc.add_ligand(got)
    nt = orc.ntors[lid]
    rng = np.random.default_rng(0)
    lib.vd_conf_to_coords.argtypes = [C.POINTER(vdock.LigandDesc), C.POINTER(C.c_float), C.POINTER(C.c_double)]
    for _ in range(5):
        pose = np.concatenate([rng.uniform(-5, 5, 3), rng.normal(size=4), rng.uniform(-3, 3, nt)]).astype(np.float32)
        pose[3:7] /= np.linalg.norm(pose[3:7])
        out = np.zeros(3 * got["n_atoms"])
        assert lib.vd_conf_to_coords(C.byref(d), pose.ctypes.data_as(C.POINTER(C.c_float)),
                                     out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        ref = orc.coords(lid, pose.astype(np.float64), got["n_atoms"])
        # the oracle uses the FP32 quaternion unnormalised (|q|^2 - 1 ~ 1e-7)
        np.testing.assert_allclose(out.reshape(-1, 3), ref, atol=1e-5)
    # writing the input coordinates reproduces the input atom lines
    n = C.c_int64()
    lib.vd_pdbqt_write_model.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_char_p, C.c_int64, C.POINTER(C.c_int64)]
    xyz = np.ascontiguousarray(got["xyz"].ravel())
    assert lib.vd_pdbqt_write_model(h, xyz.ctypes.data_as(C.POINTER(C.c_double)), None, 0, C.byref(n)) == 0
    buf = C.create_string_buffer(n.value + 1)
    assert lib.vd_pdbqt_write_model(h, xyz.ctypes.data_as(C.POINTER(C.c_double)), buf, n.value + 1, C.byref(n)) == 0
    assert buf.value.decode().splitlines() == [s.rstrip("\r") for s in text.splitlines()]
    lib.vd_pdbqt_free(h)


def test_synthetic_ligand_topology_follows_reference_rules():
    """Written as PDBQT and re-parsed by the oracle's restatement of the
    reference parser (bonds perceived from distances), a synthetic ligand
    yields the same rigid bodies, intra pairs and N_tors as the generator."""
    from vdock import synth
    for seed in range(6):
        lig = synth.ligand(30, 6, seed)
        ref_lig = P.parse_ligand(to_pdbqt(lig))
        ref = ref_lig.descriptor()
        assert len(ref["node_parent"]) == len(lig["node_parent"])
        num = np.array([a.number - 1 for a in ref_lig.atoms])
        got_pairs = {tuple(sorted((int(num[a]), int(num[b])))) for a, b in ref["pairs"]}
        want = {tuple(sorted((int(a), int(b)))) for a, b in lig["pairs"]}
        assert got_pairs == want
        assert ref["num_tors"] == lig["num_tors"]


def to_pdbqt(lig):
    """ROOT/BRANCH writer for a generated ligand (test helper); a branch
    block starts with its origin atom, as the reference expects."""
    el_name = {1: "C", 2: "N", 3: "O", 4: "S"}
    ad = {0: "C", 1: "C", 2: "N", 3: "N", 4: "NA", 8: "OA", 9: "OA", 10: "S"}
    xyz, node, parent = lig["xyz"], lig["atom_node"], lig["node_parent"]
    origin, axis = lig["node_origin_atom"], lig["node_axis_atom"]
    child_origins = set(int(origin[c]) for c in range(1, len(parent)))
    lines = []

    def atom(i):
        x, y, z = xyz[i]
        t = ad[int(lig["xs"][i])]
        return (f"ATOM  {i + 1:5d}  {el_name[int(lig['el'][i])]:<3s} LIG     1    "
                f"{x:8.3f}{y:8.3f}{z:8.3f}  0.00  0.00    +0.000 {t:<2s}")

    def body_atoms(k):
        return [i for i in np.where(node == k)[0] if int(i) not in child_origins]

    def branches(k):
        for c in np.where(parent == k)[0]:
            lines.append(f"BRANCH {axis[c] + 1:3d} {origin[c] + 1:3d}")
            lines.append(atom(origin[c]))
            for i in body_atoms(c):
                lines.append(atom(i))
            branches(c)
            lines.append(f"ENDBRANCH {axis[c] + 1:3d} {origin[c] + 1:3d}")
    lines.append("ROOT")
    for i in body_atoms(0):
        lines.append(atom(i))
    lines.append("ENDROOT")
    branches(0)
    lines.append(f"TORSDOF {len(parent) - 1}")
    return "\n".join(lines) + "\n"


def test_autotuner_logic(tmp_path):
    """The launch-shape autotuner (csrc/tune.h) compiled into a host check."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "tune_check"
    src = os.path.join(REPO, "tests", "host", "tune_check.cpp")
    inc = os.path.join(REPO, "vina-cuda_b200", "csrc")
    subprocess.run([gxx, "-std=c++17", "-O1", "-Wall", "-I", inc, src, "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_pair_force_scale_host_check(tmp_path):
    """The fixed-point scale of the kernels' pair-force sums (tables.cpp
    pair_force_scale) for weights from 1/100 to 1000 times the defaults:
    a power of two, the largest whose per-atom sums cannot overflow; 2^19
    for the default weights (a compiled host check)."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "fixed_scale_check"
    inc = os.path.join(REPO, "vina-cuda_b200", "csrc")
    srcs = [os.path.join(REPO, "tests", "host", "fixed_scale_check.cpp"), os.path.join(inc, "tables.cpp")]
    subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-ffp-contract=off", "-I", inc, "-I", "/usr/local/cuda/include",
                    *srcs, "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_pair_schedule_host_check(tmp_path):
    """The docking search's pair schedule (csrc/schedule.cpp) on 200 random
    pair sets of 10-128 atoms: every pair scheduled once with its type pair,
    32-lane rounds, deterministic, and a layout search that never raises a
    round's conflict cost (a compiled host check)."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "schedule_check"
    inc = os.path.join(REPO, "vina-cuda_b200", "csrc")
    srcs = [os.path.join(REPO, "tests", "host", "schedule_check.cpp"), os.path.join(inc, "schedule.cpp")]
    subprocess.run([gxx, "-std=c++17", "-O2", "-Wall", "-I", inc, "-I", "/usr/local/cuda/include", *srcs, "-o",
                    str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr


def _mutate(lines, rng):
    keys = ["ROOT", "ENDROOT", "BRANCH   1   2", "ENDBRANCH   1   2", "TORSDOF 3", "MODEL 1", "ENDMDL", "BRANCH",
            "BRANCH 9999 1", "ENDBRANCH 5 5", ""]
    lines = list(lines)
    for _ in range(rng.randint(1, 6)):
        if not lines:
            lines = [""]
        op, i = rng.randint(0, 7), rng.randrange(len(lines))
        if op == 0:
            del lines[i]
        elif op == 1:
            lines.insert(i, lines[rng.randrange(len(lines))])
        elif op == 2:
            j = rng.randrange(len(lines))
            lines[i], lines[j] = lines[j], lines[i]
        elif op == 3:
            lines[i] = lines[i][:rng.randint(0, len(lines[i]))]
        elif op == 4:
            chars = list(lines[i])
            for _ in range(rng.randint(1, 5)):
                if chars:
                    chars[rng.randrange(len(chars))] = rng.choice("0123456789.-+ eEXx\t#ABZ")
            lines[i] = "".join(chars)
        elif op == 5:
            lines.insert(i, rng.choice(keys))
        elif op == 6:
            lines[i] += " " * rng.randint(0, 40) + rng.choice(["1e308", "nan", "inf", "-0", "99999999"])
        else:
            lines[i] = "".join(chr(rng.randint(1, 126)) for _ in range(rng.randint(0, 90)))
    return lines


def test_parser_survives_mutated_inputs(lib, golden_dir):
    """PDBQT input is untrusted: 2,000 randomly mutated ligand and receptor
    files (deleted, duplicated, swapped, truncated and garbled lines, stray
    ROOT/BRANCH/TORSDOF/MODEL records, huge or non-finite numbers) must each
    parse or fail with VD_ERR_PARSE, never crash; every ligand that parses
    goes through the host kinematics and the PDBQT writer."""
    import random
    import vdock
    lib.vd_pdbqt_ligand.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(vdock.LigandDesc)]
    lib.vd_pdbqt_ligand.restype = C.c_int
    lib.vd_pdbqt_receptor.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int32),
                                      C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.POINTER(C.c_int32))]
    lib.vd_pdbqt_receptor.restype = C.c_int
    lib.vd_conf_to_coords.argtypes = [C.POINTER(vdock.LigandDesc), C.POINTER(C.c_float), C.POINTER(C.c_double)]
    lib.vd_conf_to_coords.restype = C.c_int
    lib.vd_pdbqt_write_model.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_char_p, C.c_int64,
                                         C.POINTER(C.c_int64)]
    lib.vd_pdbqt_write_model.restype = C.c_int
    lib.vd_pdbqt_free.argtypes = [C.c_void_p]
    ligs = [fixture_text(golden_dir, n).splitlines() for n in ("1u1b_ligand.pdbqt", "2bm2_ligand.pdbqt",
                                                             "2er7_ligand.pdbqt")]
    rec = fixture_text(golden_dir, "1u1b_protein.pdbqt").splitlines()[:400]
    rng = random.Random(20261203)
    seen = {0: 0, 5: 0}
    for _ in range(2000):
        if rng.random() < 0.8:
            text = "\n".join(_mutate(rng.choice(ligs), rng))
            h, d = C.c_void_p(), vdock.LigandDesc()
            st = lib.vd_pdbqt_ligand(text.encode(), C.byref(h), C.byref(d))
            if st == 0:
                assert d.n_atoms > 0 and d.n_nodes > 0
                pose = (C.c_float * (7 + vdock.MAX_TORS))(*([0.0] * (7 + vdock.MAX_TORS)))
                pose[3] = 1.0
                xyz = (C.c_double * (3 * d.n_atoms))()
                assert lib.vd_conf_to_coords(C.byref(d), pose, xyz) == 0
                n = C.c_int64()
                assert lib.vd_pdbqt_write_model(h, xyz, None, 0, C.byref(n)) == 0
                buf = C.create_string_buffer(n.value + 1)
                assert lib.vd_pdbqt_write_model(h, xyz, buf, n.value + 1, C.byref(n)) == 0
                lib.vd_pdbqt_free(h)
        else:
            text = "\n".join(_mutate(rec, rng))
            h, n = C.c_void_p(), C.c_int32()
            x, s = C.POINTER(C.c_double)(), C.POINTER(C.c_int32)()
            st = lib.vd_pdbqt_receptor(text.encode(), C.byref(h), C.byref(n), C.byref(x), C.byref(s))
            if st == 0:
                lib.vd_pdbqt_free(h)
        assert st in (0, 5), st
        seen[st] += 1
    assert seen[0] > 100 and seen[5] > 100


def test_ctypes_structs_match_the_c_header(tmp_path):
    """The Python mirror's structs (vdock.SearchParams, Stats, DockResult,
    LigandDesc, EvalParams) have the sizes and field offsets of the C
    declarations in include/vdock.h, compiled here with the host C compiler."""
    import ctypes as C
    import subprocess
    import vdock
    structs = {"vd_search_params": vdock.SearchParams, "vd_stats": vdock.Stats, "vd_dock_result": vdock.DockResult,
               "vd_ligand_desc": vdock.LigandDesc, "vd_eval_params": vdock.EvalParams}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "vdock.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])
