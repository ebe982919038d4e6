"""Lattice geometry and colourings: the engine's neighbour table against the
oracle's independent derivation and against the reference's links16."""
import json
import os

import numpy as np
import pytest

import cudacode_b200 as cb
from oracle import binding as orc

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SHELLS = [(0, 6), (6, 18), (18, 24), (24, 30)]


def pos4(s):
    F = np.array([(0, 0, 0), (2, 2, 0), (0, 2, 2), (2, 0, 2)])
    return F[s // 4] + F[s % 4] // 2


@pytest.mark.parametrize("s", range(16))
def test_engine_table_equals_oracle(s):
    assert np.array_equal(cb.neighbour_table(s), orc.neighbours(s))


@pytest.mark.parametrize("s", range(16))
def test_shell_distances(s):
    tab = orc.neighbours(s)
    want = [2, 6, 8, 8]
    for (a, b), r2 in zip(SHELLS, want):
        for dx, dy, dz, t in tab[a:b]:
            v = 4 * np.array([dx, dy, dz]) + pos4(t) - pos4(s)
            assert int(v @ v) == r2
    # J3a: through a site (twice a J1 vector); J3b: not
    nn = [4 * np.array(e[:3]) + pos4(e[3]) - pos4(s) for e in tab[0:6]]
    for dx, dy, dz, t in tab[18:24]:
        v = 4 * np.array([dx, dy, dz]) + pos4(t) - pos4(s)
        assert any(np.array_equal(v, 2 * w) for w in nn)
    for dx, dy, dz, t in tab[24:30]:
        v = 4 * np.array([dx, dy, dz]) + pos4(t) - pos4(s)
        assert not any(np.array_equal(v, 2 * w) for w in nn)


def test_nearest_neighbours_match_reference_links16():
    ref = np.array(json.load(open(os.path.join(GOLDEN, "links16.json")))["links16"])
    for s in range(16):
        mine = sorted(tuple(e) for e in orc.neighbours(s)[:6])
        theirs = sorted(tuple(e) for e in ref[s])
        assert mine == theirs, s


def bonds(L, shells):
    """All bonds (i, j) of an L^3 lattice for the given shells."""
    out = set()
    L3 = L ** 3
    for s in range(16):
        tab = orc.neighbours(s)
        for sh in shells:
            a, b = SHELLS[sh]
            for x in range(L):
                for y in range(L):
                    for z in range(L):
                        i = s * L3 + (z * L + y) * L + x
                        for dx, dy, dz, t in tab[a:b]:
                            j = t * L3 + (((z + dz) % L) * L + (y + dy) % L) * L + (x + dx) % L
                            out.add((min(i, j), max(i, j)))
    return out


@pytest.mark.parametrize("L", [2, 3, 4])
def test_bonds_symmetric_and_counted(L):
    b = bonds(L, [0])
    assert len(b) == 3 * 16 * L ** 3  # 6 neighbours per site, each bond twice
    b2 = bonds(L, [1]) if L >= 3 else None
    if b2 is not None:
        assert len(b2) == 6 * 16 * L ** 3


@pytest.mark.parametrize("L", [2, 3])
def test_four_colour_classes_bond_free_for_J1(L):
    L3 = L ** 3
    colour = lambda i: (i // L3) % 4  # sublattice b of site s = 4f + b
    for i, j in bonds(L, [0]):
        assert colour(i) != colour(j)


@pytest.mark.parametrize("L", [3, 4])
def test_sixteen_colour_classes_bond_free_for_J1_J2_J3(L):
    L3 = L ** 3
    for i, j in bonds(L, [0, 1, 2, 3]):
        assert i // L3 != j // L3


def test_up_tetrahedra_are_consecutive_sites():
    for f in range(4):
        for a in range(4):
            tab = orc.neighbours(4 * f + a)
            intra = {tuple(e) for e in tab[:6] if tuple(e[:3]) == (0, 0, 0)}
            assert {4 * f + b for b in range(4) if b != a} <= {e[3] for e in intra}
