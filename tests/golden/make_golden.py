"""Generates the golden fixtures that pin the engine to taillefu/cudacode.

The reference ships no tests or golden vectors and cannot be built (its glue
files and MKL/GSL/popt are missing), so the pins are taken from its own data
and its one CPU routine:

* ``links16.json``: the 16 x 6 nearest-neighbour table ``links16``
  (Pyrochlore.cu:152-167), parsed from the source text.
* ``reference_energy.json``: energies of seeded spin configurations computed
  by a line-by-line numpy evaluation of the reference's host ``TotalEnergy``
  (Pyrochlore.cu:468-523) with its ``couplings_const`` matrices
  (Pyrochlore.cu:169-184), evaluated at J1 = J2 = J (isotropic Heisenberg),
  J3 = J4 = 0, no field; S^2 = 1/4 (spin one-half normalisation). The
  engine's energy (unit spins, H = J sum S_i.S_j) times 1/4 must equal these.
* ``reference_anisotropic.json``: the anisotropic model. ``couplings_const``
  evaluated at the unit vectors of (J1, J2, J3, J4) (the table is linear in
  them); the site fields of ``InitializeMagneticField`` (Pyrochlore.cu:414-450,
  transcribed line by line, including its tesla -> meV factor) for a few
  (gxy, gz, B); and ``TotalEnergy`` of seeded configurations with the
  reference's default couplings (Pyrochlore.cu:138-141), a J4 case and a field
  (FieldOnSite = the fields above).

Run from the repository root, in a checkout that has the reference at
/root/reference:  python tests/golden/make_golden.py
"""
import json
import os
import re

import numpy as np

REF = "/root/reference/Pyrochlore.cu"
OUT = os.path.dirname(os.path.abspath(__file__))


def parse_links16(text):
    m = re.search(r"#define links16(.*?)\n\n", text, re.S)
    body = m.group(1).replace("\\\n", " ")
    nums = [int(x) for x in re.findall(r"-?\d+", body)]
    assert len(nums) == 16 * 6 * 4, len(nums)
    return np.array(nums).reshape(16, 6, 4)


def parse_couplings(text):
    """couplings_const (Pyrochlore.cu:169-184) as a function of J1..J4."""
    m = re.search(r"#define couplings_const(.*?)\n\n", text, re.S)
    body = m.group(1).replace("\\\n", " ").replace("{", "[").replace("}", "]")

    def C(J1, J2, J3, J4):
        return np.array(eval(body, {"J1": J1, "J2": J2, "J3": J3, "J4": J4}), dtype=np.float64)

    return C


def magnetization_gtensors(gxy, gz):
    """The g1..g4 matrices of MagnetizationGPU (Pyrochlore.cu:283-286), with
    _g1, _g2 set as in InitializeCouplings3D (Pyrochlore.cu:697-701)."""
    g1 = (2.0 * gxy + gz) / 3.0
    g2 = (gz - gxy) / 3.0
    return [[[g1, g2, g2], [g2, g1, g2], [g2, g2, g1]],
            [[g1, g2, -g2], [g2, g1, -g2], [-g2, -g2, g1]],
            [[g1, -g2, -g2], [-g2, g1, g2], [-g2, g2, g1]],
            [[g1, -g2, g2], [-g2, g1, -g2], [g2, -g2, g1]]]


def initialize_magnetic_field(B, gxy, gz):
    """Pyrochlore.cu:414-450 (without its printf)."""
    g1 = (2.0 * gxy + gz) / 3.0
    g2 = (gz - gxy) / 3.0
    g11 = [[g1, g2, g2], [g2, g1, g2], [g2, g2, g1]]
    g21 = [[g1, g2, -g2], [g2, g1, -g2], [-g2, -g2, g1]]
    g3 = [[g1, -g2, -g2], [-g2, g1, g2], [-g2, g2, g1]]
    g4 = [[g1, -g2, g2], [-g2, g1, -g2], [g2, -g2, g1]]
    BSite = [0.0] * 12
    for s in range(3):
        for s1 in range(3):
            BSite[s] += g11[s][s1] * B[s1]
    for s in range(3):
        for s1 in range(3):
            BSite[s + 3] += g21[s][s1] * B[s1]
    for s in range(3):
        for s1 in range(3):
            BSite[s + 6] += g3[s][s1] * B[s1]
    for s in range(3):
        for s1 in range(3):
            BSite[s + 9] += g4[s][s1] * B[s1]
    return [b * 0.0578838261305 for b in BSite]


def total_energy(Sx, Sy, Sz, n, links, C, field=None):
    """Pyrochlore.cu:468-523, TYPE = double, S2 = 1/4; FieldOnSite = field (or 0)."""
    F = field if field is not None else [0.0] * 12
    tmp = 0.0
    for z in range(n):
        for y in range(n):
            for x in range(n):
                for site in range(16):
                    ex = 2.0 * F[3 * (site % 4)]
                    ey = 2.0 * F[3 * (site % 4) + 1]
                    ez = 2.0 * F[3 * (site % 4) + 2]
                    Id = ((y + z * n) * n + x) + site * n ** 3
                    for se in range(6):
                        x1 = (x + links[site][se][0] + n) % n
                        y1 = (y + links[site][se][1] + n) % n
                        z1 = (z + links[site][se][2] + n) % n
                        ne = links[site][se][3]
                        Idd = ((z1 * n + y1) * n + x1) + ne * n ** 3
                        cp = C[site % 4][ne % 4]
                        ex += 0.5 * (cp[0] * Sx[Idd] + cp[1] * Sy[Idd] + cp[2] * Sz[Idd])
                        ey += 0.5 * (cp[3] * Sx[Idd] + cp[4] * Sy[Idd] + cp[5] * Sz[Idd])
                        ez += 0.5 * (cp[6] * Sx[Idd] + cp[7] * Sy[Idd] + cp[8] * Sz[Idd])
                    tmp -= ex * Sx[Id] + ey * Sy[Id] + ez * Sz[Id]
    return tmp * 0.25


def main():
    text = open(REF).read()
    links = parse_links16(text)
    couplings = parse_couplings(text)
    with open(os.path.join(OUT, "links16.json"), "w") as f:
        json.dump({"source": "Pyrochlore.cu:152-167", "links16": links.tolist()}, f)
    cases = []
    rng = np.random.default_rng(20240611)
    for n in (2, 3):
        for J in (1.0, -0.5):
            N = 16 * n ** 3
            v = rng.normal(size=(N, 3))
            v /= np.linalg.norm(v, axis=1, keepdims=True)
            v = v.astype(np.float32).astype(np.float64)
            e = total_energy(v[:, 0], v[:, 1], v[:, 2], n, links, couplings(J, J, 0.0, 0.0))
            cases.append({"L": n, "J": J, "spins": v.tolist(), "energy_reference_units": e})
    with open(os.path.join(OUT, "reference_energy.json"), "w") as f:
        json.dump({"source": "Pyrochlore.cu:468-523 TotalEnergy, couplings_const 169-184",
                   "spin_layout": "plane-major: index = site * L^3 + (z L + y) L + x",
                   "cases": cases}, f)
    # anisotropic model
    basis = [couplings(*np.eye(4)[k]).reshape(4, 4, 9).tolist() for k in range(4)]
    fields = []
    for gxy, gz, B in ((1.0, 1.0, (0.0, 0.0, 1.0)), (2.4, 0.3, (0.7, -0.2, 1.5)),
                       (0.5, 3.0, (-1.0, 2.0, 0.25))):
        fields.append({"gxy": gxy, "gz": gz, "B": list(B),
                       "field_on_site": initialize_magnetic_field(B, gxy, gz),
                       "magnetization_g": magnetization_gtensors(gxy, gz)})
    acases = []
    rng = np.random.default_rng(20240612)
    defaults = (-0.09 / 0.29, -0.22 / 0.29, -1.00, 0.0)  # Pyrochlore.cu:138-141
    for n, Js, fi in ((2, defaults, None), (2, (0.4, -0.3, 0.2, 0.35), 1), (3, defaults, 2)):
        N = 16 * n ** 3
        v = rng.normal(size=(N, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        v = v.astype(np.float32).astype(np.float64)
        F = fields[fi]["field_on_site"] if fi is not None else None
        e = total_energy(v[:, 0], v[:, 1], v[:, 2], n, links, couplings(*Js), F)
        acases.append({"L": n, "J": list(Js), "field_case": fi, "spins": v.tolist(),
                       "energy_reference_units": e})
    with open(os.path.join(OUT, "reference_anisotropic.json"), "w") as f:
        json.dump({"source": "couplings_const Pyrochlore.cu:169-184; InitializeMagneticField "
                             "414-450; TotalEnergy 468-523; defaults 138-141",
                   "couplings_basis": basis, "fields": fields,
                   "spin_layout": "plane-major: index = site * L^3 + (z L + y) L + x",
                   "cases": acases}, f)


if __name__ == "__main__":
    main()
