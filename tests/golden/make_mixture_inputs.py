"""Writes the inputs of the constant generator's test (tests/test_mixgen_cpu.py)
from a checkout of the reference.

    python tests/golden/make_mixture_inputs.py REFERENCE

Run here, where the reference's files are; the files it writes under
tests/golden/mixtures are committed, and nothing at test time reads the
reference.  What it writes:

  gri30_h2o2.yaml   the 9-species H2/O2/N2 subset of the reference's GRI-Mech
                    3.0 mechanism file (Cantera format): its reactions among
                    those species, third-body efficiencies of absent species
                    dropped, by peregrine_b200/data/export_mixture.py's subset;
  ch4_o2_ffcmy.yaml the reference's CH4_O2_FFCMY mechanism file, every species;
  library.yaml      the reference's species library entries (JANAF thermo,
                    critical point, collision parameters) of the species above
                    and of the cubic gases' O2, H2 and CH4, as the reference's
                    mixture supplements a species' missing data from them.

The shipped table sets these regenerate (peregrine_b200/data/*.npz) were
written by export_mixture.py from the same files.
"""

import os
import sys
import tempfile

import yaml

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

H2O2 = ["H2", "H", "O", "O2", "OH", "H2O", "HO2", "H2O2", "N2"]


def main(reference):
    from peregrine_b200.data.export_mixture import subset

    db = os.path.join(reference, "peregrine", "simulator", "mixture", "database")
    out = os.path.join(HERE, "mixtures")
    os.makedirs(out, exist_ok=True)
    names = set(H2O2) | {"CH4"}
    with tempfile.TemporaryDirectory() as tmp:
        for src, keep, dst in (("GRI30.yaml", H2O2, "gri30_h2o2.yaml"), ("CH4_O2_FFCMY.yaml", None, "ch4_o2_ffcmy.yaml")):
            path = subset(os.path.join(db, "mechanisms", src), keep, tmp)
            with open(path) as f:
                text = f.read()
            with open(os.path.join(out, dst), "w") as f:
                f.write(text)
            names |= {s["name"] for s in yaml.safe_load(text)["species"]}
    with open(os.path.join(db, "species.yaml")) as f:
        library = yaml.safe_load(f)
    picked = {n: library[n] for n in sorted(names) if n in library}
    with open(os.path.join(out, "library.yaml"), "w") as f:
        yaml.safe_dump(picked, f, sort_keys=False)
    print(out, sorted(picked))


if __name__ == "__main__":
    main(sys.argv[1])
