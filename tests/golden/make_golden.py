"""Generates the golden fixtures under tests/golden/ from the reference tree.

Runs only where a checkout of the reference exists; its root (the directory
holding Vina-CUDA_v1.1/ and QuickVina-W-CUDA/) is the one argument:

    python tests/golden/make_golden.py <reference root>

The fixtures it writes are committed so the tests need no reference files at
run time.

Outputs
* kat_vina.npz -- known-answer vectors: for each docked ligand the reference
  ships (Vina-CUDA_v1.1/docking_result/1u1b_docking_result.pdbqt and the
  QuickVina-W-CUDA test_out/ results, all docked into the 1u1b box), the
  per-model atom coordinates, the ligand topology the oracle parser derives,
  and the REMARK VINA RESULT triple (energy, rmsd l.b., rmsd u.b.).  The
  receptor is stored as typed atoms (xyz, XS type) with its box.
* pdbqt/*.pdbqt.gz -- a few example inputs (receptor, ligands, config) for
  the product parser and CLI tests.
"""
import glob
import gzip
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import pdbqt_oracle as P  # noqa: E402



def main(ref):
    V11 = os.path.join(ref, "Vina-CUDA_v1.1")
    QW = os.path.join(ref, "QuickVina-W-CUDA", "input_file_example")
    cfg = P.read_config(open(os.path.join(V11, "input_file_example/1u1b_config.txt")).read())
    center = [float(cfg[k]) for k in ("center_x", "center_y", "center_z")]
    size = [float(cfg[k]) for k in ("size_x", "size_y", "size_z")]
    rec_text = open(os.path.join(V11, "input_file_example/1u1b_protein.pdbqt")).read()
    rxyz, rxs = P.parse_receptor(rec_text)
    files = [os.path.join(V11, "docking_result/1u1b_docking_result.pdbqt")]
    files += sorted(glob.glob(os.path.join(QW, "test_out", "*.pdbqt")))
    out = {"rec_xyz": rxyz, "rec_xs": rxs, "center": np.array(center), "size": np.array(size)}
    names = []
    for f in files:
        models = P.split_models(open(f).read())
        ligs = [P.parse_ligand(t) for _, t in models]
        d = ligs[0].descriptor()
        key = f"L{len(names)}"
        names.append(os.path.relpath(f, ref))
        for k in ("xs", "el", "atom_node", "node_parent", "node_origin_atom", "node_axis_atom", "pairs"):
            out[f"{key}_{k}"] = d[k]
        out[f"{key}_num_tors"] = np.array(d["num_tors"])
        out[f"{key}_models"] = np.stack([L.descriptor()["xyz"] for L in ligs])
        out[f"{key}_remarks"] = np.array([m[0] for m in models], dtype=np.float64)
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "kat_vina.npz"), **out)

    os.makedirs(os.path.join(HERE, "pdbqt"), exist_ok=True)
    copies = {
        "1u1b_protein.pdbqt": os.path.join(V11, "input_file_example/1u1b_protein.pdbqt"),
        "1u1b_ligand.pdbqt": os.path.join(V11, "input_file_example/1u1b_ligand.pdbqt"),
        "2bm2_ligand.pdbqt": os.path.join(V11, "input_file_example/2bm2_ligand.pdbqt"),
        "2er7_ligand.pdbqt": os.path.join(V11, "input_file_example/2er7_ligand.pdbqt"),
        "1u1b_config.txt": os.path.join(V11, "input_file_example/1u1b_config.txt"),
        "1u1b_docking_result.pdbqt": os.path.join(V11, "docking_result/1u1b_docking_result.pdbqt"),
    }
    for dst, src in copies.items():
        with open(src, "rb") as fi, gzip.GzipFile(os.path.join(HERE, "pdbqt", dst + ".gz"), "wb", mtime=0) as fo:
            fo.write(fi.read())
    print(f"wrote {len(names)} known-answer ligands")


if __name__ == "__main__":
    if len(sys.argv) != 2 or not os.path.isdir(os.path.join(sys.argv[1], "Vina-CUDA_v1.1")):
        sys.exit("usage: make_golden.py <reference root containing Vina-CUDA_v1.1/>")
    main(sys.argv[1])
