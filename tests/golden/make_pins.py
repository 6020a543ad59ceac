"""Extract the reference's legacy end-to-end SCF energy pins into legacy_pins.json.

Source: the reference's oldTests.tgz (an uncompressed tar), member tests/chronus-ref.val,
lines "testNNNN/<energy>/..." written by the reference's 2016 test generator, and the
matching inputs tests/testNNNN_serial_direct.inp (geometry, charge, multiplicity,
reference type and basis).  Only the Hartree-Fock rows the two-electron path drives
(water RHF, Li and O2 UHF) are kept.

    python tests/golden/make_pins.py /root/reference/oldTests.tgz
"""
import json
import os
import sys
import tarfile

KEEP = ["test0001", "test0002", "test0003", "test0007", "test0008", "test0009",
        "test0010", "test0011", "test0012"]


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
    return out


def main(tgz):
    tf = tarfile.open(tgz)
    vals = tf.extractfile("tests/chronus-ref.val").read().decode().splitlines()
    energies = {}
    for line in vals:
        f = line.split("/")
        if f[0] in KEEP:
            energies[f[0]] = float(f[1])
    pins = []
    for t in KEEP:
        inp = parse_inp(tf.extractfile("tests/%s_serial_direct.inp" % t).read().decode())
        basis = {"sto3g.gbs": "sto-3g", "6-31G.gbs": "6-31g", "6-31g.gbs": "6-31g",
                 "cc-pVDZ.gbs": "cc-pvdz", "cc-pvdz.gbs": "cc-pvdz"}.get(inp["basis"], inp["basis"])
        pins.append({"test": t, "energy": energies[t], "reference": inp["reference"],
                     "charge": int(inp.get("charge", 0)), "mult": int(inp.get("mult", 1)),
                     "basis": basis, "geom_angstrom": inp["geom"]})
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "legacy_pins.json"), "w") as f:
        json.dump(pins, f, indent=1)
    print(json.dumps(pins, indent=1))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/oldTests.tgz")
