"""The constant generator (peregrine_b200/mixgen.py), on the CPU.

Every table set shipped under peregrine_b200/data was written by running the
reference's own mixture code (peregrine_b200/data/export_mixture.py).  The
generator, given the same mechanism files and species library (committed
under tests/golden/mixtures by tests/golden/make_mixture_inputs.py) and no
reference checkout, works out every table again: each key must equal the
shipped one to the bit (thermally perfect fits in ln T, kinetic-theory fits,
Wilke pairs, Lewis numbers, binary-diffusion pair fits, the cubic's constants,
reaction columns, third-body sets, Troe fits, the product-form choice and the
concentration floor).
"""

import os

import numpy as np
import pytest

from peregrine_b200 import mixgen

HERE = os.path.dirname(os.path.abspath(__file__))
G = os.path.join(HERE, "golden", "mixtures")
DATA = os.path.join(os.path.dirname(HERE), "peregrine_b200", "data")
LIB = os.path.join(G, "library.yaml")

SETS = {
    "h2o2_gri30": dict(mechanism="gri30_h2o2.yaml", trans="kinetic-theory", chemistry="finite-rate"),
    "h2o2_gri30_binary": dict(mechanism="gri30_h2o2.yaml", trans="kinetic-theory", chemistry="finite-rate",
                              diffusion="binary"),
    "h2o2_gri30_oneway": dict(mechanism="gri30_h2o2.yaml", trans="kinetic-theory", chemistry="finite-rate",
                              oneway=True),
    "ch4_o2_ffcmy": dict(mechanism="ch4_o2_ffcmy.yaml", trans="kinetic-theory", chemistry="finite-rate"),
    "o2_h2_srk": dict(species=["O2", "H2"], eos="real-gas", trans="kinetic-theory", trange=(100.0, 1000.0)),
    "o2_h2_pr": dict(species=["O2", "H2"], eos="real-gas", trans="kinetic-theory", trange=(100.0, 1000.0),
                     cubic="pr"),
    "ch4_o2_srk": dict(species=["CH4", "O2"], eos="real-gas", trans="kinetic-theory", trange=(100.0, 1500.0)),
}


def generate(tmp_path, mechanism=None, oneway=False, **kw):
    if mechanism is not None:
        path = os.path.join(G, mechanism)
        if oneway:
            # every reaction irreversible: the reference parser's one-way arrow
            with open(path) as f:
                text = f.read().replace("<=>", "=>")
            path = str(tmp_path / mechanism)
            with open(path, "w") as f:
                f.write(text)
        kw["mechanism"] = path
    return mixgen.make_tables(library=LIB, **kw)


def same(a, b):
    if a.dtype.kind in "US":
        return [str(x) for x in np.atleast_1d(a)] == [str(x) for x in np.atleast_1d(b)]
    return a.shape == np.shape(b) and np.array_equal(a, b)


@pytest.mark.parametrize("name", sorted(SETS))
def test_every_shipped_table_is_regenerated_to_the_bit(name, tmp_path):
    with np.load(os.path.join(DATA, f"{name}.npz")) as z:
        ref = {k: z[k] for k in z.files}
    got = generate(tmp_path, **SETS[name])
    assert set(ref) <= set(got), sorted(set(ref) - set(got))
    bad = [k for k in ref if not same(ref[k], got[k])]
    assert not bad, bad


def test_a_config_names_a_mechanism_file():
    from peregrine_b200.config import Config
    from peregrine_b200.mixture import Mixture

    cfg = Config()
    m = cfg["mixture"]
    m["species"], m["eos"], m["trans"], m["chemistry"] = os.path.join(G, "gri30_h2o2.yaml"), "tpg", \
        "kinetic-theory", "finite-rate"
    m["T-range"] = (300.0, 3500.0)
    mix = Mixture(m)
    assert mix.spnames == ["H2", "H", "O", "O2", "OH", "H2O", "HO2", "H2O2", "N2"]
    with np.load(os.path.join(DATA, "h2o2_gri30.npz")) as z:
        for k in ("cppoly", "mupoly", "kappapoly", "rxn_logA", "rxn_lfcpoly", "tb_effsp"):
            assert np.array_equal(mix.constants()[k], z[k]), k
    # a thermally perfect gas's fits need the case's temperatures
    m["T-range"] = None
    with pytest.raises(ValueError, match="T-range"):
        Mixture(m)


def test_units_and_third_bodies_are_read_as_the_reference_reads_them(tmp_path):
    mech = tmp_path / "m.yaml"
    mech.write_text("""
units: {length: cm, quantity: mol, activation-energy: kcal/mol}
phases: [{name: gas, species: [A, B, C]}]
species:
- {name: A, composition: {H: 2}, thermo: {model: NASA7, temperature-ranges: [200, 1000, 3500],
   data: [[3.3, 0.0, 0.0, 0.0, 0.0, -1000.0, -3.0], [3.3, 0.0, 0.0, 0.0, 0.0, -1000.0, -3.0]]}}
- {name: B, composition: {O: 2}, thermo: {model: NASA7, temperature-ranges: [200, 3500],
   data: [[3.5, 0.0, 0.0, 0.0, 0.0, -1000.0, 4.0]]}}
- {name: C, composition: {H: 2, O: 2}, thermo: {model: NASA7, temperature-ranges: [200, 3500],
   data: [[4.0, 0.0, 0.0, 0.0, 0.0, -5000.0, 2.0]]}}
reactions:
- {equation: A + B <=> C, rate-constant: {A: 2.0e12, b: 0.5, Ea: 1.0}}
- {equation: A + B + M <=> C + M, type: three-body, rate-constant: {A: 3.0e15, b: 0.0, Ea: 0.0},
   efficiencies: {A: 2.5}}
- {equation: A + B + C <=> C + C, rate-constant: {A: 1.0e15, b: 0.0, Ea: 0.0}, type: three-body,
   efficiencies: {C: 1.0}}
- {equation: A + B (+C) <=> C (+C), type: falloff, high-P-rate-constant: {A: 1.0e13, b: 0.0, Ea: 0.0},
   low-P-rate-constant: {A: 1.0e16, b: 0.0, Ea: 0.0}}
""")
    sp, rx = mixgen.read_mechanism(str(mech))
    assert sp["A"]["MW"] == 2 * 1.008 and sp["C"]["MW"] == 2 * 1.008 + 2 * 15.999
    # a single NASA-7 range serves both halves
    assert sp["B"]["NASA7"]["low"] == sp["B"]["NASA7"]["high"]
    # A in (cm^3/mol)^(order-1) /s to (m^3/kmol)^(order-1) /s; Ea in kcal/mol over Ru
    A, b, EaR = rx[0]["rate"]
    assert A == pytest.approx(2.0e12 * 1e-3) and b == 0.5 and EaR == pytest.approx(4.184e6 / mixgen.RU)
    assert rx[1]["rate"][0] == pytest.approx(3.0e15 * 1e-6) and rx[1]["defeff"] == 1.0
    # an explicit third body: one C off each side, its efficiency the only one
    assert rx[2]["reactants"] == {"A": 1.0, "B": 1.0} and rx[2]["products"] == {"C": 1.0}
    assert rx[2]["defeff"] == 0.0 and rx[2]["efficiencies"] == {"C": 1.0}
    # an explicit falloff collider: zero default, unit efficiency of the collider
    assert rx[3]["type"] == "lindemann" and rx[3]["defeff"] == 0.0 and rx[3]["efficiencies"] == {"C": 1.0}
    t = mixgen.make_tables(mechanism=str(mech), chemistry="finite-rate")
    assert list(t["rxn_kind"]) == [0, 1, 1, 2]
    # two third-body sets: A's 2.5 over the default 1, and C alone over a zero
    # default, which the explicit third body and the explicit collider share
    assert t["tb_neff"].tolist() == [1, 1] and t["rxn_tb"].tolist() == [-1, 0, 1, 1]


def test_bad_mechanisms_are_refused(tmp_path):
    mech = tmp_path / "m.yaml"
    base = """
phases: [{name: gas, species: [A, B]}]
species:
- {name: A, composition: {H: 2}, thermo: {model: NASA7, temperature-ranges: [200, 3500], data: [[3.3, 0, 0, 0, 0, 0, 0]]}}
- {name: B, composition: {O: 2}, thermo: {model: NASA7, temperature-ranges: [200, 3500], data: [[3.5, 0, 0, 0, 0, 0, 0]]}}
reactions:
"""
    for rxn, why in (("- {equation: A <=> B, rate-constant: {A: 1.0, b: 0, Ea: 0}, efficiencies: {A: 2.0}}", "efficiencies"),
                     ("- {equation: A + M <=> B, rate-constant: {A: 1.0, b: 0, Ea: 0}}", "third body"),
                     ("- {equation: A <=> X, rate-constant: {A: 1.0, b: 0, Ea: 0}}", "outside the phase"),
                     ("- {equation: A (+M) <=> B (+M), type: falloff, high-P-rate-constant: {A: 1, b: 0, Ea: 0}, "
                      "low-P-rate-constant: {A: 1, b: 0, Ea: 0}, efficiencies: {A: 2.0, B: 1.0}, "
                      "default-efficiency: 0.5}", None)):
        mech.write_text(base + rxn + "\n")
        if why is None:
            mixgen.read_mechanism(str(mech))
            continue
        with pytest.raises((ValueError, KeyError), match=why):
            mixgen.read_mechanism(str(mech))
    mech.write_text(base + "- {equation: A => B, rate-constant: {A: -1.0, b: 0, Ea: 0}}\n")
    with pytest.raises(ValueError, match="positive"):
        mixgen.make_tables(mechanism=str(mech), chemistry="finite-rate")
