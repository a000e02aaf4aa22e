"""Generate the golden fixtures used by the parity tests.

Reads the reference's own regression data (needs the reference checkout, so it
runs in the build container only; its outputs are committed):

  * test/molecules/HF-HF-MOLPRO/FCIDUMP   -> hf_ccpvdz_fcidump.npz
    (the MOLPRO integral dump of HF/cc-pVDZ, stored as the raw list of
    (value, p, q, r, s) records plus the &FCI namelist)
  * test/python-interface.s.ref           -> hf_ccpvdz_ref.json
    (numbers the reference printed for that run: string counts per graph,
    ME-list lengths, the dgemm shape statistics of one formula evaluation and
    the converged MP2 energy)

usage: python tests/golden/make_golden.py [/path/to/reference]
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_fcidump(path):
    with open(path) as f:
        text = f.read()
    head, body = text.split("/", 1)
    head = head.replace("\n", " ")
    norb = int(re.search(r"NORB\s*=\s*(\d+)", head).group(1))
    nelec = int(re.search(r"NELEC\s*=\s*(\d+)", head).group(1))
    ms2 = int(re.search(r"MS2\s*=\s*(-?\d+)", head).group(1))
    isym = int(re.search(r"ISYM\s*=\s*(\d+)", head).group(1))
    orbsym = [int(x) for x in re.search(r"ORBSYM\s*=\s*([\d,\s]+?),\s*ISYM", head)
              .group(1).replace(",", " ").split()]
    vals, idx = [], []
    for line in body.splitlines():
        p = line.split()
        if len(p) != 5:
            continue
        vals.append(float(p[0].replace("D", "E")))
        idx.append([int(x) for x in p[1:]])
    return dict(norb=norb, nelec=nelec, ms2=ms2, isym=isym, orbsym=np.array(orbsym),
                vals=np.array(vals), idx=np.array(idx, dtype=np.int32))


def read_ref(path):
    lines = open(path).read().splitlines()
    out = {"source": "test/python-interface.s.ref"}
    # string counts: "Graph space electr. MS length" tables
    graphs = []
    i = 0
    while i < len(lines):
        if lines[i].strip() == "Number of strings":
            rows = []
            j = i + 3
            while j < len(lines) and re.match(r"^\s+(\d+\s+)+-?\d+\s+\d+\s*$", lines[j]):
                nums = [int(x) for x in lines[j].split()]
                rows.append(nums)
                j += 1
            g = {"graph": rows[0][0], "space": rows[0][1], "nel": rows[0][2],
                 "ms_len": [[r[-2], r[-1]] for r in rows]}
            graphs.append(g)
            i = j
        else:
            i += 1
    out["graphs"] = graphs
    # ME-list lengths
    lists = {}
    for k, l in enumerate(lines):
        if "idx           list  sym spn      length" in l:
            j = k + 2
            while not lines[j].startswith(" ---"):
                p = lines[j].split()
                lists[p[1]] = {"sym": int(p[2]), "spn": int(p[3]), "length": int(p[4]),
                               "op": p[5]}
                j += 1
            break
    out["lists"] = lists
    # dgemm statistics of the second formula evaluation
    stats = []
    for k, l in enumerate(lines):
        if "calls to dgemm:" in l:
            n = int(l.split()[-1])
            ent = {"calls": n}
            if n:
                for key, lab in (("dim1", "avg dim1"), ("dim2", "avg dim2"), ("cnt", "avg cnt")):
                    m = [x for x in lines[k + 1:k + 4] if lab in x][0]
                    a, s = m.split(":")[1].split()
                    ent[key] = [float(a), float(s)]
            stats.append(ent)
    out["dgemm_stats"] = stats
    m = [l for l in lines if ">>> final energy:" in l][0]
    out["final_energy_12digits"] = float(m.split()[3])
    m = [l for l in lines if "total norm =" in l][-1]
    out["lmp2_norm"] = float(m.split()[-1])
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    fd = read_fcidump(os.path.join(ref, "test/molecules/HF-HF-MOLPRO/FCIDUMP"))
    np.savez_compressed(os.path.join(HERE, "hf_ccpvdz_fcidump.npz"), **fd)
    info = read_ref(os.path.join(ref, "test/python-interface.s.ref"))
    info["orbitals"] = {"occ": [3, 1, 1, 0], "frozen": [1, 0, 0, 0], "nsym": 4}
    with open(os.path.join(HERE, "hf_ccpvdz_ref.json"), "w") as f:
        json.dump(info, f, indent=1)
    print("wrote", len(fd["vals"]), "integral records;", json.dumps(info)[:400])


if __name__ == "__main__":
    main()
