"""Seeded synthetic molecules of the benchmark workloads, plus fixed test geometries.

Water clusters: oxygens on a jittered cubic lattice (2.9 Angstrom spacing, uniform
+-0.2 Angstrom jitter), each hydrogen at O-H 0.957 Angstrom, H-O-H 104.5 degrees, the
molecule given a seeded random rotation.  Alkanes: all-trans chain, C-C 1.54 Angstrom,
C-H 1.09 Angstrom, tetrahedral angles, every atom jittered +-0.02 Angstrom.

Angstrom is converted to bohr with the reference's factor 1.889725989
(src/molecule.cpp:467).
"""
import numpy as np

ANG2BOHR = 1.889725989
Z_OF = {"H": 1, "C": 6, "N": 7, "O": 8}


class Molecule:
    def __init__(self, symbols, coords_ang, name=""):
        self.symbols = list(symbols)
        self.coords_ang = np.asarray(coords_ang, dtype=np.float64).reshape(-1, 3)
        self.name = name

    @property
    def coords_bohr(self):
        return self.coords_ang * ANG2BOHR

    @property
    def charges(self):
        return np.array([Z_OF[s] for s in self.symbols], dtype=np.float64)

    @property
    def nelec(self):
        return int(self.charges.sum())

    def nuclear_repulsion(self):
        R = self.coords_bohr
        Z = self.charges
        e = 0.0
        for i in range(len(Z)):
            for j in range(i):
                e += Z[i] * Z[j] / np.linalg.norm(R[i] - R[j])
        return e


def _rng(seed):
    return np.random.Generator(np.random.MT19937(seed))


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d],
    ])


def water_cluster(grid, seed=0, spacing=2.9, jitter=0.2, roh=0.957, angle_deg=104.5):
    """(H2O)_N with oxygens on a jittered grid of shape `grid` (e.g. (2, 3), (4, 2, 2))."""
    grid = tuple(grid) + (1,) * (3 - len(grid))
    rng = _rng(seed)
    th = np.deg2rad(angle_deg) / 2.0
    h_local = np.array([[roh * np.sin(th), 0.0, roh * np.cos(th)], [-roh * np.sin(th), 0.0, roh * np.cos(th)]])
    sym, xyz = [], []
    for i in range(grid[0]):
        for j in range(grid[1]):
            for k in range(grid[2]):
                o = np.array([i, j, k], dtype=np.float64) * spacing + rng.uniform(-jitter, jitter, 3)
                R = _random_rotation(rng)
                sym.append("O")
                xyz.append(o)
                for h in h_local:
                    sym.append("H")
                    xyz.append(o + R @ h)
    n = grid[0] * grid[1] * grid[2]
    return Molecule(sym, np.array(xyz), name="(H2O)%d" % n)


def alkane(ncarbon, seed=0, jitter=0.02):
    """All-trans C_n H_{2n+2}: zig-zag carbon chain in the xy plane, staggered hydrogens."""
    rng = _rng(seed)
    cc, ch = 1.54, 1.09
    tet = np.arccos(-1.0 / 3.0)
    half = (np.pi - tet) / 2.0
    dx, dy = cc * np.cos(half), cc * np.sin(half)
    carbons = [np.array([i * dx, (dy / 2.0) * (1.0 if i % 2 else -1.0), 0.0]) for i in range(ncarbon)]
    ez = np.array([0.0, 0.0, 1.0])
    hyd = []
    for i, c in enumerate(carbons):
        nbrs = [carbons[j] for j in (i - 1, i + 1) if 0 <= j < ncarbon]
        bonds = [(n - c) / np.linalg.norm(n - c) for n in nbrs]
        if len(bonds) == 2:
            u = -(bonds[0] + bonds[1])
            u /= np.linalg.norm(u)
            for s in (1.0, -1.0):
                hyd.append(c + ch * (np.cos(tet / 2.0) * u + s * np.sin(tet / 2.0) * ez))
        else:
            b = bonds[0]
            e1 = np.cross(ez, b)
            e1 /= np.linalg.norm(e1)
            # one in-plane H on the outer side of the zig-zag, the other two at +-120 degrees
            ref = e1 if np.dot(e1, np.array([0.0, c[1], 0.0])) > 0 else -e1
            for phi in (0.0, 2.0 * np.pi / 3.0, -2.0 * np.pi / 3.0):
                perp = np.cos(phi) * ref + np.sin(phi) * ez
                hyd.append(c + ch * (np.cos(tet) * b + np.sin(tet) * perp))
    sym = ["C"] * ncarbon + ["H"] * len(hyd)
    xyz = np.array(carbons + hyd)
    xyz = xyz + rng.uniform(-jitter, jitter, xyz.shape)
    return Molecule(sym, xyz, name="C%dH%d" % (ncarbon, 2 * ncarbon + 2))


WORKLOADS = {
    # name: (molecule factory, orbital basis, auxiliary basis)
    "h2o6_dz": (lambda seed=0: water_cluster((2, 3), seed), "cc-pvdz", "cc-pvdz-jkfit"),
    "h2o16_dz": (lambda seed=0: water_cluster((4, 2, 2), seed), "cc-pvdz", "cc-pvdz-jkfit"),
    "c40h82_dz": (lambda seed=0: alkane(40, seed), "cc-pvdz", "cc-pvdz-jkfit"),
    "h2o32_tz": (lambda seed=0: water_cluster((4, 4, 2), seed), "cc-pvtz", "cc-pvtz-jkfit"),
}
