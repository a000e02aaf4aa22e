"""Generate the CH2/DZ fixtures of the reference's CCSDT regression test.

Reads the reference's own regression data (needs the reference checkout, so it
runs in the build container only; its outputs are committed):

  * test/molecules/CH2-DZ-DALTON/SIRIFC, MOTWOINT -> ch2_dz_dalton.npz
    DALTON's interface files as the reference imports them
    (input/read_fock_from_sirifc.f, input/import_h2_dalton.f): the SCF
    energy, the orbital irreps, the inactive Fock matrix (symmetry-blocked
    packed upper triangles, after the 'SIR IPH ' record and five more) and
    the MO two-electron integrals (pq|rs) of the 'MOLTWOEL' records, each a
    buffer of values, a buffer of packed indices (rs in the upper, pq in the
    lower 16 bits, one byte per orbital) and a count (negative at the end);
    stored as the raw (value, p, q, r, s) records.
  * test/CC-energy-I.e.ref -> ch2_dz_ccsdt_ref.json
    the energies the reference printed for CCSDT (CC maxexc=3) with the
    orbital space of test/CC-energy-I.inp: frozen (1,0,0,0), deleted
    (2,1,0,0), occupied (3,1,0,0) as the output lists its shells.
  * test/CC-excite-I.e.ref -> ch2_dz_ccsd_ref.json
    the CCSD ground-state iterations of that run (the block before its first
    'final energy'): frozen (1,0,0,0), nothing deleted.

usage: python tests/golden/make_ch2_dalton.py [/path/to/reference]
"""
import json
import os
import re
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def records(path):
    """the records of a Fortran sequential unformatted file (4-byte markers)"""
    buf = open(path, "rb").read()
    out, pos = [], 0
    while pos < len(buf):
        n = struct.unpack("<i", buf[pos:pos + 4])[0]
        out.append(buf[pos + 4:pos + 4 + n])
        pos += 8 + n
    return out


def after_label(recs, label):
    for i, r in enumerate(recs):
        if r[:8] == b"********" and r[24:32] == label:
            return i + 1
    raise KeyError(label)


def read_sirifc(path):
    recs = records(path)
    i = after_label(recs, b"SIR IPH ")
    potnuc, emy, eactiv, emcscf = struct.unpack("<4d", recs[i][:32])
    nactel = struct.unpack("<i", recs[i][40:44])[0]
    # the inactive Fock matrix: nskip_in_sirifc = 6 records after the label's
    # first one, or the next when that one does not start negative
    fock = np.frombuffer(recs[i + 6], "<f8").copy()
    if fock[0] >= 0:
        fock = np.frombuffer(recs[i + 7], "<f8").copy()
    j = after_label(recs, b"TRCCINT ")
    nsym, norbt = struct.unpack("<2i", recs[j][:8])
    orb_en = np.frombuffer(recs[j + 1][:8 * norbt], "<f8").copy()
    orbsym = np.frombuffer(recs[j + 1][8 * norbt:12 * norbt], "<i4").astype(np.int64)
    eref = emcscf if nactel == 0 else emy + potnuc
    return dict(eref=eref, potnuc=potnuc, fock_packed=fock, orb_en=orb_en, orbsym=orbsym)


def read_motwoint(path):
    recs = records(path)
    lbuf = struct.unpack("<i", recs[1][:4])[0]
    i = after_label(recs, b"MOLTWOEL")
    vals, idx = [], []
    for r in recs[i:]:
        n = struct.unpack("<i", r[12 * lbuf:12 * lbuf + 4])[0]
        if n < 0:
            break
        x = np.frombuffer(r[:8 * n], "<f8")
        ib = np.frombuffer(r[8 * lbuf:8 * lbuf + 4 * n], "<u4")
        rs, pq = ib >> 16, ib & 0xFFFF
        vals.append(x)
        idx.append(np.stack([pq >> 8, pq & 0xFF, rs >> 8, rs & 0xFF], 1).astype(np.int64))
    return np.concatenate(vals), np.concatenate(idx)


def read_history(path):
    """the '>>> iteration energy residual' lines up to the first final energy"""
    hist = []
    for line in open(path).read().splitlines():
        if re.match(r">>>\s+\d+\s", line):
            hist.append((int(line.split()[1]), float(line.split()[2]), float(line.split()[3])))
        elif "final energy" in line:
            return {"history": hist, "final_energy": float(line.split()[3])}
    raise ValueError(path)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    mol = os.path.join(ref, "test/molecules/CH2-DZ-DALTON")
    sir = read_sirifc(os.path.join(mol, "SIRIFC"))
    vals, idx = read_motwoint(os.path.join(mol, "MOTWOINT"))
    np.savez_compressed(os.path.join(HERE, "ch2_dz_dalton.npz"), vals=vals, idx=idx, **sir)
    info = read_history(os.path.join(ref, "test/CC-energy-I.e.ref"))
    info["orbitals"] = {"occ": [3, 1, 0, 0], "frozen": [1, 0, 0, 0], "deleted": [2, 1, 0, 0]}
    info["method"] = "CC maxexc=3 (CCSDT), DIIS maxsub 8, conv 1e-10"
    with open(os.path.join(HERE, "ch2_dz_ccsdt_ref.json"), "w") as f:
        json.dump(info, f, indent=1)
    ccsd = read_history(os.path.join(ref, "test/CC-excite-I.e.ref"))
    ccsd["orbitals"] = {"occ": [3, 1, 0, 0], "frozen": [1, 0, 0, 0], "deleted": [0, 0, 0, 0]}
    ccsd["method"] = "CC maxexc=2 (CCSD) ground state, DIIS maxsub 8"
    with open(os.path.join(HERE, "ch2_dz_ccsd_ref.json"), "w") as f:
        json.dump(ccsd, f, indent=1)
    print("wrote", len(vals), "integral records; E_ref", sir["eref"], "final", info["final_energy"],
          "CCSD final", ccsd["final_energy"], len(ccsd["history"]))


if __name__ == "__main__":
    main()
