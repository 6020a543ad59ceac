"""Extract the reference's legacy end-to-end SCF energy pins into legacy_pins.json.

Source: the reference's oldTests.tgz (an uncompressed tar), member tests/chronus-ref.val,
lines "testNNNN/<energy>/..." written by the reference's 2016 test generator, and the
matching inputs tests/testNNNN_serial_direct.inp (geometry, charge, multiplicity,
reference type and basis).  Only the Hartree-Fock rows the two-electron path drives
(water RHF, Li and O2 UHF) are kept.

    python tests/golden/make_pins.py <reference>/oldTests.tgz
"""
import json
import os
import sys
import tarfile

KEEP = ["test0001", "test0002", "test0003", "test0007", "test0008", "test0009",
        "test0010", "test0011", "test0012"]
# the same molecules in a static electric field (Real RHF 0043-0045 and Real UHF 0049-0054,
# the field jobs with recorded values): energy and dipole moment (Debye), written to
# legacy_field_pins.json
FIELD_KEEP = ["test0043", "test0044", "test0045"] + ["test%04d" % i for i in range(49, 55)]


def parse_inp(text):
    out = {"geom": []}
    sec, in_geom = None, False
    for raw in text.splitlines():
        line = raw.split("#")[0].rstrip()
        if not line.strip():
            continue
        s = line.strip()
        if s.startswith("["):
            sec = s.strip("[]").lower()
            in_geom = False
            continue
        if sec == "molecule":
            if s.lower().startswith("geom"):
                in_geom = True
                continue
            if in_geom and len(s.split()) == 4 and "=" not in s:
                sym, x, y, z = s.split()
                out["geom"].append([sym, float(x), float(y), float(z)])
                continue
            if "=" in s:
                k, v = [t.strip() for t in s.split("=", 1)]
                out[k.lower()] = v
        elif sec == "qm" and "=" in s:
            k, v = [t.strip() for t in s.split("=", 1)]
            out[k.lower()] = v
        elif sec == "scf" and "=" in s:
            k, v = [t.strip() for t in s.split("=", 1)]
            if k.lower() == "field":
                out["field"] = [float(x) for x in v.split()]
    return out


def _pin(tf, rows, t):
    inp = parse_inp(tf.extractfile("tests/%s_serial_direct.inp" % t).read().decode())
    basis = {"sto3g.gbs": "sto-3g", "6-31G.gbs": "6-31g", "6-31g.gbs": "6-31g",
             "cc-pVDZ.gbs": "cc-pvdz", "cc-pvdz.gbs": "cc-pvdz"}.get(inp["basis"], inp["basis"])
    pin = {"test": t, "energy": float(rows[t][1]), "reference": inp["reference"],
           "charge": int(inp.get("charge", 0)), "mult": int(inp.get("mult", 1)),
           "basis": basis, "geom_angstrom": inp["geom"]}
    if "field" in inp:
        pin["field"] = inp["field"]
        pin["dipole_debye"] = [float(x) for x in rows[t][2:5]]
    return pin


def main(tgz):
    tf = tarfile.open(tgz)
    vals = tf.extractfile("tests/chronus-ref.val").read().decode().splitlines()
    rows = {line.split("/")[0]: line.split("/") for line in vals}
    here = os.path.dirname(os.path.abspath(__file__))
    for name, keep in (("legacy_pins.json", KEEP), ("legacy_field_pins.json", FIELD_KEEP)):
        pins = [_pin(tf, rows, t) for t in keep]
        with open(os.path.join(here, name), "w") as f:
            json.dump(pins, f, indent=1)
        print(name, len(pins))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/oldTests.tgz")
