"""ChronusQ INI input files for the SCF jobs this engine runs.

Reads the reference's input format (src/python/src/parse/parseInput.py, section and
keyword tables in src/python/src/parse/meta/knownKeywords.py) with the standard
``configparser`` the reference uses, and runs the job on the GPU engine:

* ``[Molecule]``  CHARGE, MULT, GEOM (``<symbol> x y z`` or ``<symbol> <isotope> x y z``
  per line, Angstrom; parseMolecule.py readGeom), PRINT ignored.
* ``[QM]``        REFERENCE = ``[Real] RHF | UHF`` (parseQM.py handleReference; complex,
  two-component and Kohn-Sham references are not handled by this engine and are
  rejected), JOB = SCF.
* ``[BASIS]``     BASIS (a .gbs name such as STO-3G, 6-31G*, cc-pVDZ), FORCECART (only
  false is handled: the engine evaluates pure shells for l > 1).
* ``[SCF]``       DENTOL, ENETOL, MAXITER, GUESS (SAD, CORE, LEARNED), DIIS (parseQM.py
  parseSCF), FIELD (a static field, a.u.: SingleSlater.setField); ITP and DT are
  rejected.  A one-atom molecule uses the CORE guess, as parseSCF does.
* ``[MISC]``, ``[INTS]``  accepted and ignored (thread counts and the integral algorithm
  have no meaning here).

Unknown sections or keywords raise ``InputError``, like the reference's CErrMsg.

    python -m chronusq_public_b200.inp job.inp
"""
from __future__ import annotations

import configparser
import sys
from dataclasses import dataclass, field
from typing import Dict, List, Optional

from .molecule import Molecule

KNOWN = {
    "MOLECULE": {"CHARGE": "I", "MULT": "I", "GEOM": "S", "PRINT": "I"},
    "QM": {"REFERENCE": "S", "JOB": "S", "EXCHANGE": "S", "CORR": "S", "DFT_NRAD": "I", "DFT_NANG": "I",
           "DFT_SCREEN": "B", "DFT_SCRTOL": "D", "PRINT": "I"},
    "BASIS": {"BASIS": "S", "FORCECART": "B"},
    "SCF": {"DENTOL": "D", "ENETOL": "D", "MAXITER": "I", "FIELD": "D3", "GUESS": "S", "DIIS": "B", "ITP": "B",
            "DT": "D", "PRINT": "I"},
    "MISC": {"NSMP": "I", "PRINT": "I"},
    "INTS": {"ALG": "S"},
    "RT": None,
}
REQUIRED = {"MOLECULE": ("CHARGE", "MULT", "GEOM"), "QM": ("REFERENCE", "JOB"), "BASIS": ("BASIS",)}


class InputError(ValueError):
    pass


@dataclass
class Job:
    molecule: Molecule
    reference: str                 # "RHF" or "UHF"
    basis: str
    scf: Dict[str, object] = field(default_factory=dict)


def parse_sections(text: str) -> Dict[str, Dict[str, object]]:
    """Sections and typed keyword values (upper-case names), checked against the
    reference's keyword table."""
    cp = configparser.ConfigParser(interpolation=None)
    cp.optionxform = str
    try:
        cp.read_string(text)
    except configparser.Error as e:
        raise InputError("input is not a valid ChronusQ INI file: %s" % e) from None
    out: Dict[str, Dict[str, object]] = {}
    for sec in cp.sections():
        S = sec.upper()
        if S not in KNOWN:
            raise InputError("Section %s not recognized" % sec)
        if KNOWN[S] is None:
            raise InputError("Section %s (real-time propagation) is not handled by this engine" % sec)
        vals: Dict[str, object] = {}
        for opt in cp.options(sec):
            K = opt.upper()
            typ = KNOWN[S].get(K)
            if typ is None:
                raise InputError("Keyword %s.%s not recognized" % (sec, opt))
            raw = cp.get(sec, opt)
            try:
                if typ == "I":
                    vals[K] = int(raw)
                elif typ == "D":
                    vals[K] = float(raw)
                elif typ == "B":
                    vals[K] = cp.getboolean(sec, opt)
                elif typ == "D3":
                    vals[K] = [float(x) for x in raw.split()]
                else:
                    vals[K] = raw
            except ValueError:
                raise InputError("Keyword %s.%s: cannot read %r" % (sec, opt, raw)) from None
        out[S] = vals
    for S, keys in REQUIRED.items():
        for K in keys:
            if K not in out.get(S, {}):
                raise InputError("Required keyword %s.%s not found" % (S.title(), K))
    return out


def _geometry(text: str):
    symbols, coords = [], []
    for line in text.splitlines():
        tok = line.split()
        if not tok:
            continue
        if len(tok) == 4:
            sym, xyz = tok[0], tok[1:]
        elif len(tok) == 5:
            sym, xyz = tok[0], tok[2:]
        else:
            raise InputError("geometry line %r is not '<symbol> [isotope] x y z'" % line.strip())
        try:
            coords.append([float(x) for x in xyz])
        except ValueError:
            raise InputError("geometry line %r has a non-numeric coordinate" % line.strip()) from None
        symbols.append(sym)
    if not symbols:
        raise InputError("Molecule.geom is empty")
    return symbols, coords


def parse_job(text: str) -> Job:
    sec = parse_sections(text)
    mol_s, qm, bas = sec["MOLECULE"], sec["QM"], sec["BASIS"]
    if str(qm["JOB"]).strip().upper() != "SCF":
        raise InputError("QM.Job %s is not handled by this engine (SCF only)" % qm["JOB"])
    ref = str(qm["REFERENCE"]).split()
    words = [w.upper() for w in ref]
    if "COMPLEX" in words or any(w.startswith("X2C") or w.startswith("G") for w in words):
        raise InputError("QM.Reference %s: complex and two-component references are not handled"
                         % qm["REFERENCE"])
    name = words[-1]
    if name not in ("RHF", "UHF"):
        raise InputError("QM.Reference %s: only Hartree-Fock (RHF, UHF) is handled" % qm["REFERENCE"])
    if bas.get("FORCECART", False):
        raise InputError("Basis.forceCart = true is not handled (pure shells for l > 1 only)")
    scf = sec.get("SCF", {})
    if "FIELD" in scf and len(scf["FIELD"]) != 3:
        raise InputError("SCF.Field needs three components, got %d" % len(scf["FIELD"]))
    for k in ("ITP", "DT"):
        if k in scf and (k != "ITP" or scf[k]):
            raise InputError("SCF.%s is not handled by this engine" % k)
    symbols, coords = _geometry(str(mol_s["GEOM"]))
    try:
        mol = Molecule.from_angstrom(symbols, coords, charge=int(mol_s["CHARGE"]), mult=int(mol_s["MULT"]))
    except (KeyError, ValueError) as e:
        raise InputError("Molecule: %s" % e) from None
    return Job(mol, name, str(bas["BASIS"]).strip(), dict(scf))


def run_job(job: Job, device: int = 0, thresholdSchwartz: float = 1e-14, guess_model=None):
    """Converge the job's SCF on the GPU; returns the SingleSlater (energy in
    ``totalEnergy``)."""
    from .basis import BasisSet
    from .scf import SingleSlater
    bs = BasisSet(job.basis, job.molecule.atoms, job.molecule.coords)
    hf = SingleSlater(job.molecule, bs, ref=job.reference, device=device, thresholdSchwartz=thresholdSchwartz)
    s = job.scf
    if "DENTOL" in s:
        hf.denTol = float(s["DENTOL"])
    if "ENETOL" in s:
        hf.eneTol = float(s["ENETOL"])
    if "MAXITER" in s:
        hf.maxSCFIter = int(s["MAXITER"])
    if "DIIS" in s:
        hf.doDIIS = bool(s["DIIS"])
    if "GUESS" in s:
        g = str(s["GUESS"]).strip().upper()
        if g not in ("SAD", "CORE", "LEARNED"):
            raise InputError("SCF.Guess %s is not handled (SAD, CORE, LEARNED)" % s["GUESS"])
        hf.guess = g
    if job.molecule.natoms == 1:
        hf.guess = "CORE"
    if "FIELD" in s:
        hf.setField(s["FIELD"])
    if hf.guess == "LEARNED":
        from .guess_model import PairMLP, default_weights
        if guess_model is None:
            path = default_weights(job.basis)
            if path is None:
                raise InputError("SCF.Guess LEARNED: no trained weights for basis %s" % job.basis)
            guess_model = PairMLP.load(path, device=device)
        hf.guess_model = guess_model
    hf.SCF3()
    return hf


def main(argv: Optional[List[str]] = None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 1:
        print("usage: python -m chronusq_public_b200.inp <input.inp>", file=sys.stderr)
        return 2
    with open(argv[0]) as f:
        job = parse_job(f.read())
    hf = run_job(job)
    print("Total Energy = %.10f Eh  (%d SCF iterations, %s, %s)" % (hf.totalEnergy, hf.nSCFIter, job.reference,
                                                                  job.basis))
    hf.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
