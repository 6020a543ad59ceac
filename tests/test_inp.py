"""ChronusQ INI input files: parsing rules on the CPU, and (GPU) SCF runs of inputs built
from the recorded reference energies' geometries and settings."""
import json
import os

import numpy as np
import pytest

from chronusq_public_b200 import inp

HERE = os.path.dirname(os.path.abspath(__file__))
PINS = json.load(open(os.path.join(HERE, "golden", "legacy_pins.json")))


def make_input(pin, extra_scf=""):
    """An input in the reference's INI format for one recorded job."""
    geom = "\n".join(" %-3s %16.10f %16.10f %16.10f" % tuple(g) for g in pin["geom_angstrom"])
    return ("# generated job\n[Molecule]\ncharge = %d\nmult = %d\ngeom:\n%s\n\n[QM]\nreference = %s\njob = SCF\n\n"
            "[BASIS]\nbasis = %s\n\n[SCF]\n%s\n[MISC]\nnsmp = 1\n"
            % (pin["charge"], pin["mult"], geom, pin["reference"], pin["basis"].upper(), extra_scf))


def test_parse_water_job():
    job = inp.parse_job(make_input(PINS[0], "enetol = 1e-9\ndentol = 1e-7\nmaxiter = 64\ndiis = true\n"))
    assert job.reference == "RHF" and job.basis.lower() == "sto-3g"
    assert job.molecule.atoms == [8, 1, 1] and job.molecule.charge == 0 and job.molecule.mult == 1
    ang = np.array([g[1:] for g in PINS[0]["geom_angstrom"]])
    assert np.allclose(np.asarray(job.molecule.coords) * 0.52917721092, ang, atol=1e-6)
    assert job.scf == {"ENETOL": 1e-9, "DENTOL": 1e-7, "MAXITER": 64, "DIIS": True}


def test_field_is_read():
    job = inp.parse_job(make_input(PINS[0], "field = 0.01 0.0 -0.002\n"))
    assert job.scf["FIELD"] == [0.01, 0.0, -0.002]


def test_isotope_column_and_case_insensitive_keys():
    text = make_input(PINS[0]).replace(" O  ", " O 16").replace("charge", "CHARGE")
    job = inp.parse_job(text)
    assert job.molecule.atoms == [8, 1, 1]


@pytest.mark.parametrize("edit,msg", [
    (("job = SCF", "job = RT"), "SCF only"),
    (("reference = Real RHF", "reference = Real B3LYP"), "Hartree-Fock"),
    (("reference = Real RHF", "reference = Complex RHF"), "complex"),
    (("[SCF]\n", "[SCF]\nfield = 0 0.01\n"), "three components"),
    (("[SCF]\n", "[SCF]\nbogus = 1\n"), "not recognized"),
    (("basis = STO-3G", "basis = STO-3G\nforceCart = true"), "forceCart"),
    (("mult = 1\n", ""), "MULT"),
    (("[MISC]", "[STAB]"), "not recognized"),
])
def test_rejections(edit, msg):
    text = make_input(PINS[0]).replace(*edit)
    with pytest.raises(inp.InputError, match=msg):
        inp.parse_job(text)


@pytest.mark.gpu
@pytest.mark.parametrize("pin", PINS, ids=lambda p: p["test"])
def test_input_jobs_reproduce_recorded_energies(pin):
    job = inp.parse_job(make_input(pin))
    hf = inp.run_job(job)
    assert hf.converged
    assert abs(hf.totalEnergy - pin["energy"]) < 1e-8, (hf.totalEnergy, pin["energy"])
    hf.close()


FIELD_PINS = json.load(open(os.path.join(HERE, "golden", "legacy_field_pins.json")))
DEBYE = 0.393430307      # e bohr per Debye (the reference's phys.debye)


@pytest.mark.gpu
@pytest.mark.parametrize("pin", FIELD_PINS, ids=lambda p: p["test"])
def test_field_jobs_reproduce_recorded_energies_and_dipoles(pin):
    """Field jobs (SCF.FIELD) through the input runner: the reference's recorded energies
    within 1e-8 Eh and dipole moments within 5e-5 relative (Debye)."""
    job = inp.parse_job(make_input(pin, "field = %r %r %r\n" % tuple(pin["field"])))
    hf = inp.run_job(job)
    assert hf.converged
    assert abs(hf.totalEnergy - pin["energy"]) < 1e-8, (hf.totalEnergy, pin["energy"])
    mu = hf.dipoleMoment() / DEBYE
    ref = np.asarray(pin["dipole_debye"])
    assert np.abs(mu - ref).max() < 5e-5 * max(1.0, np.abs(ref).max()), (mu, ref)
    hf.close()
