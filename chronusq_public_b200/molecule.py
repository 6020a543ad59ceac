"""Molecules and seeded water-cluster geometries.

Restates the parts of the reference's ``Molecule`` the two-electron path needs:
coordinates are read in Angstrom and divided by ``phys.bohr = 0.5291772083000001``
(include/global.h:224, include/molecule.h:97), and the nuclear repulsion energy is the
pairwise Z_i Z_j / r_ij sum (src/molecule/molecule.cpp:159-170).

The geometry generators produce the seeded synthetic inputs the workloads are defined
on: a rigid water (O at the origin, O-H lengths uniform in 0.96 +- 0.02 A, H-O-H angle
uniform in 104.5 +- 2 degrees), and clusters of such waters with uniformly random
orientations whose oxygen centres are placed by Poisson-disk (dart-throwing) sampling in
a cube sized for liquid density 1.0 g/cm^3 (0.033428 molecules per A^3), with a minimum
O-O distance of 2.6 A.  Besides the O-O rule, a trial molecule is also rejected when any
of its atoms comes within 1.4 A of an atom of another molecule, which keeps hydrogens of
neighbouring waters from overlapping.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from .basis import ELEMENTS, SYMBOL_TO_Z

BOHR_PER_ANGSTROM_INV = 0.5291772083000001   # phys.bohr: Angstrom per bohr
WATER_NUMBER_DENSITY = 0.033428              # molecules / A^3 at 1.0 g/cm^3


@dataclass
class Molecule:
    atoms: List[int]            # atomic numbers
    coords: np.ndarray          # (natom, 3) in bohr
    charge: int = 0
    mult: int = 1

    @classmethod
    def from_angstrom(cls, symbols_or_z: Sequence, coords_ang, charge: int = 0, mult: int = 1):
        atoms = [s if isinstance(s, (int, np.integer)) else SYMBOL_TO_Z[str(s).upper()]
                 for s in symbols_or_z]
        xyz = np.asarray(coords_ang, dtype=np.float64).reshape(-1, 3) / BOHR_PER_ANGSTROM_INV
        return cls([int(a) for a in atoms], xyz, charge, mult)

    @property
    def natoms(self) -> int:
        return len(self.atoms)

    @property
    def nelectrons(self) -> int:
        return int(sum(self.atoms)) - self.charge

    def nuclear_repulsion(self) -> float:
        e = 0.0
        for i in range(self.natoms):
            for j in range(i + 1, self.natoms):
                d = self.coords[i] - self.coords[j]
                e += self.atoms[i] * self.atoms[j] / math.sqrt(float(d @ d))
        return e

    def symbols(self) -> List[str]:
        return [ELEMENTS[z] for z in self.atoms]


def water_monomer(rng: np.random.Generator) -> np.ndarray:
    """Rigid water in its own frame (Angstrom): rows O, H1, H2."""
    r1 = rng.uniform(0.94, 0.98)
    r2 = rng.uniform(0.94, 0.98)
    th = math.radians(rng.uniform(102.5, 106.5))
    return np.array([[0.0, 0.0, 0.0],
                     [r1, 0.0, 0.0],
                     [r2 * math.cos(th), r2 * math.sin(th), 0.0]])


def single_water(seed: int) -> Molecule:
    rng = np.random.Generator(np.random.PCG64(seed))
    xyz = water_monomer(rng)
    return Molecule.from_angstrom([8, 1, 1], xyz)


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def water_cluster(n: int, seed: int, min_oo: float = 2.6, min_atom: float = 1.4,
                  max_tries: int = 200000) -> Molecule:
    """(H2O)_n at liquid density: seeded orientations and Poisson-disk O centres."""
    rng = np.random.Generator(np.random.PCG64(seed))
    side = (n / WATER_NUMBER_DENSITY) ** (1.0 / 3.0)
    placed: List[np.ndarray] = []
    tries = 0
    while len(placed) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("Poisson-disk sampling failed to place %d waters" % n)
        mono = water_monomer(rng)
        rot = _random_rotation(rng)
        centre = rng.uniform(0.0, side, size=3)
        xyz = mono @ rot.T + centre
        ok = True
        for other in placed:
            if np.linalg.norm(other[0] - xyz[0]) < min_oo:
                ok = False
                break
            d = np.linalg.norm(other[:, None, :] - xyz[None, :, :], axis=-1)
            if d.min() < min_atom:
                ok = False
                break
        if ok:
            placed.append(xyz)
    coords = np.concatenate(placed, axis=0)
    coords -= coords.mean(axis=0)
    return Molecule.from_angstrom([8, 1, 1] * n, coords)


REFERENCE_WATER_ANGSTROM = (
    # tests/test0001.inp:9-12 of the reference
    [8, 1, 1],
    [[0.0, -0.07579184359, 0.0],
     [0.866811829, 0.6014357793, 0.0],
     [-0.866811829, 0.6014357793, 0.0]],
)


def reference_water() -> Molecule:
    z, xyz = REFERENCE_WATER_ANGSTROM
    return Molecule.from_angstrom(z, xyz)
