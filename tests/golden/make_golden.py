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
* ``reference_order.json``: order parameters of seeded configurations, summed
  over cells as the reference's reductions do: the irrep components of
  ``Measurement`` (Pyrochlore.cu:526-641, its expressions evaluated from the
  source text), the quadrupole of ``_CudaQuadrupolarOrder`` (Math.cu:335-372),
  the monopole density of ``CudaCalculateMonopoleSquare`` (Math.cu:386-476),
  ``CudaCalculateAbsSz`` (Math.cu:478-510) and the per-cell masks of
  ``CudaCalculateIsingConf`` (Math.cu:513-541).

Run from the repository root with the path of the reference's Pyrochlore.cu
(or set PYRO_REFERENCE_SOURCE):

    python tests/golden/make_golden.py <path>/Pyrochlore.cu
"""
import json
import os
import re
import sys

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))


def reference_source() -> str:
    path = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYRO_REFERENCE_SOURCE")
    if not path:
        sys.exit("usage: make_golden.py <path to the reference's Pyrochlore.cu> "
                 "(or set PYRO_REFERENCE_SOURCE)")
    return path


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


def parse_measurement(text):
    """The per-cell irrep expressions of Measurement (Pyrochlore.cu:526-641),
    taken from the source text; returns f(s0, s1, s2, s3) -> 12 values in the
    order the kernel stores them."""
    from types import SimpleNamespace as NS
    body = text[text.index("GLOBAL void Measurement"):]
    body = body[body.index("mm1="):body.index("TYPE *Order =")]
    stmts = [" ".join(st.split()) for st in body.split(";") if st.strip()]

    def f(s0, s1, s2, s3):
        env = {"s0": s0, "s1": s1, "s2": s2, "s3": s3, "mm1": 0.0,
               "mm2": NS(x=0.0, y=0.0), "mm3": NS(x=0.0, y=0.0, z=0.0),
               "mm4": NS(x=0.0, y=0.0, z=0.0), "mm5": NS(x=0.0, y=0.0, z=0.0)}
        for st in stmts:
            exec(st, {}, env)
        m2, m3, m4, m5 = env["mm2"], env["mm3"], env["mm4"], env["mm5"]
        return [env["mm1"], m2.x, m2.y, m3.x, m3.y, m3.z, m4.x, m4.y, m4.z, m5.x, m5.y, m5.z]

    return f


def order_parameters(v, n, measurement):
    """Sums over cells of Measurement, the quadrupole, monopole and |Sz|
    kernels (Math.cu:335-510), and the Ising masks (Math.cu:513-541), of one
    configuration v (plane-major, 16 n^3 x 3)."""
    from types import SimpleNamespace as NS
    sz = [[1, 1, 1], [-1, -1, 1], [1, -1, -1], [-1, 1, -1]]
    nc = n ** 3
    tot = np.zeros(20)
    ising = []
    for cell in range(nc):
        sub = []
        for b in range(4):
            s = v[[cell + (4 * k + b) * nc for k in range(4)]].sum(axis=0)
            sub.append(NS(x=s[0], y=s[1], z=s[2]))
        tot[:12] += measurement(*sub)
        q = [0.0] * 6
        for s in range(16):
            x, y, z = v[cell + s * nc]
            q[0] += x * x - 0.333333333333333333333
            q[1] += x * y
            q[2] += x * z
            q[3] += y * y - 0.333333333333333333333
            q[4] += y * z
            q[5] += z * z - 0.333333333333333333333
        tot[12:18] += q
        charge = [0.0] * 4
        A = 0.0
        cs = 0
        for te in range(4):
            for si in range(4):
                scal = float(np.dot(v[cell + (4 * te + si) * nc], sz[si]))
                charge[te] += scal
                A += abs(scal)
                cs |= (1 if scal < 0 else 0) << (4 * te + si)
            charge[te] = abs(np.sqrt(charge[te] * charge[te]))
        tot[18] += sum(charge) / 4.0
        tot[19] += A / np.sqrt(3.0)
        ising.append(cs)
    return tot.tolist(), ising


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
    text = open(reference_source()).read()
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
    measurement = parse_measurement(text)
    ocases = []
    rng = np.random.default_rng(20240613)
    axes = np.array([[1, 1, 1], [-1, -1, 1], [1, -1, -1], [-1, 1, -1]], dtype=np.float64) / np.sqrt(3)
    for n, kind in ((2, "random"), (3, "random"), (2, "tilted all-in-all-out")):
        N = 16 * n ** 3
        if kind == "random":
            v = rng.normal(size=(N, 3))
        else:  # sites along +-a_b with a random tilt, so every irrep is non-zero
            b = np.arange(N) // n ** 3 % 4
            v = axes[b] * np.where(rng.random(N) < 0.8, 1.0, -1.0)[:, None] + 0.3 * rng.normal(size=(N, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        v = v.astype(np.float32).astype(np.float64)
        tot, ising = order_parameters(v, n, measurement)
        ocases.append({"L": n, "kind": kind, "spins": v.tolist(), "order": tot, "ising": ising})
    with open(os.path.join(OUT, "reference_order.json"), "w") as f:
        json.dump({"source": "Measurement Pyrochlore.cu:526-641; Math.cu:335-541",
                   "spin_layout": "plane-major: index = site * L^3 + (z L + y) L + x",
                   "order_layout": "12 irrep components (Order[] order), quadrupole xx xy xz "
                                   "yy yz zz, monopole, |Sz|; sums over cells",
                   "cases": ocases}, f)
    with open(os.path.join(OUT, "reference_anisotropic.json"), "w") as f:
        json.dump({"source": "couplings_const Pyrochlore.cu:169-184; InitializeMagneticField "
                             "414-450; TotalEnergy 468-523; defaults 138-141",
                   "couplings_basis": basis, "fields": fields,
                   "spin_layout": "plane-major: index = site * L^3 + (z L + y) L + x",
                   "cases": acases}, f)


if __name__ == "__main__":
    main()
