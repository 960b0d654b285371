"""Mechanism layer: parsing, flattening, thermodynamic consistency."""
import numpy as np
import pytest

from pelelmex_b200 import mechanism as M

NAMES = ["synth_h2_9", "synth_ch4_21", "synth_c12_53"]
SIZES = {"synth_h2_9": (9, 21), "synth_ch4_21": (21, 84), "synth_c12_53": (53, 268)}


@pytest.mark.parametrize("name", NAMES)
def test_sizes_and_labels(name):
    m = M.builtin(name)
    assert (m.n_species, m.n_reactions) == SIZES[name]
    import yaml
    doc = yaml.safe_load(open(m.source))
    assert "SYNTHETIC" in doc["description"]


def test_species_order_matches_reference_tables():
    # drm19 ordering from Exec/RegTests/FlameSheet/drm19_pmf.dat:1
    m = M.builtin("synth_ch4_21")
    assert m.names[:5] == ["H2", "H", "O", "O2", "OH"] and m.names[-2:] == ["N2", "AR"]
    m = M.builtin("synth_c12_53")
    assert m.names[0] == "NC12H26" and m.names[-1] == "N2"


@pytest.mark.parametrize("name", NAMES)
def test_element_balance(name):
    m = M.builtin(name)
    E = m.element_matrix()
    idx = {s: i for i, s in enumerate(m.names)}
    for r in m.reactions:
        d = np.zeros(m.n_species)
        for s, c in r.reactants.items():
            d[idx[s]] -= c
        for s, c in r.products.items():
            d[idx[s]] += c
        assert np.allclose(E @ d, 0), r.equation


@pytest.mark.parametrize("name", NAMES)
def test_nasa_continuity(name):
    m = M.builtin(name)
    for s in m.species:
        lo, hi, t = np.array(s.nasa_lo), np.array(s.nasa_hi), s.tmid
        cp = lambda a: a[0] + t * (a[1] + t * (a[2] + t * (a[3] + t * a[4])))
        h = lambda a: cp(a) * 0 + a[0] + t * (a[1] / 2 + t * (a[2] / 3 + t * (a[3] / 4 + t * a[4] / 5))) + a[5] / t
        assert abs(cp(lo) - cp(hi)) < 1e-6 * abs(cp(lo))
        assert abs(h(lo) - h(hi)) < 1e-8 * max(1.0, abs(h(lo)))


def test_flatten_layout():
    m = M.builtin("synth_ch4_21")
    f = M.flatten(m)
    a = f.arrays
    assert a["sp"].shape == (84, 8) and a["nasa"].shape == (21, 15)
    assert a["eff_ptr"][-1] == f.n_eff
    # reactant slots come first, -1 marks an empty slot
    for j, r in enumerate(m.reactions):
        assert sum(1 for s in a["sp"][j, :4] if s >= 0) == len(r.reactants)
        assert sum(1 for s in a["sp"][j, 4:] if s >= 0) == len(r.products)


def test_parse_units_and_errors(tmp_path):
    doc = """
units: {length: m, quantity: kmol, activation-energy: J/kmol}
species:
- name: A
  composition: {H: 2}
  thermo: {model: NASA7, temperature-ranges: [200, 1000, 3500], data: [[3,0,0,0,0,0,0],[3,0,0,0,0,0,0]]}
- name: B
  composition: {H: 1}
  thermo: {model: NASA7, temperature-ranges: [200, 1000, 3500], data: [[2.5,0,0,0,0,1000,0],[2.5,0,0,0,0,1000,0]]}
reactions:
- equation: 2 B <=> A
  rate-constant: {A: 1.0e+10, b: 0.0, Ea: 8314.46261815324}
"""
    p = tmp_path / "m.yaml"
    p.write_text(doc)
    m = M.load(p)
    A, b, EaR = m.reactions[0].arr
    assert A == pytest.approx(1e10 * 1e3)  # m^3/kmol -> cm^3/mol for a 2nd-order rate
    assert EaR == pytest.approx(1.0)
    p.write_text(doc.replace("2 B <=> A", "2 B <=> C"))
    with pytest.raises(M.MechanismError):
        M.load(p)


def test_philox_known_answer():
    # Random123 Philox-4x32-10 known-answer test: counter 0, key 0
    from pelelmex_b200.workloads import philox4x32
    w = philox4x32(np.array([0], dtype=np.uint64), 0, 0, 0)[:, 0]
    assert [hex(int(x)) for x in w] == ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
