"""Extract the reference's golden vectors for the hot path into small fixtures.

Run in a checkout that has the reference workspace available (read-only):

    python tests/golden/make_golden.py /path/to/sonium

It reads the reference's own fixture files (it runs none of the reference's code) and writes:
  - mie_rigid_golden.json     rigid-sphere Mie coefficients a_n at ka = 1 and 5, 100-digit
                              values from crates/sonium-wave/fixtures/scattering-golden-v1.json
  - spherical_bessel_golden.json  j_n, y_n, j_n', y_n' at six arguments, 50-digit Wolfram values
                              from crates/sonium-wave/fixtures/special-golden-wolfram-v1.json
  - sincos_golden.json        correctly rounded sin/cos from
                              crates/sonium-fastmath/fixtures/wolfram-golden-v1.json
Decimal strings are kept as strings so no precision is lost in the fixture itself.
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    wave = os.path.join(ref_root, "crates", "sonium-wave", "fixtures")
    fm = os.path.join(ref_root, "crates", "sonium-fastmath", "fixtures")

    src = json.load(open(os.path.join(wave, "scattering-golden-v1.json")))
    mie = {
        "source": "crates/sonium-wave/fixtures/scattering-golden-v1.json",
        "convention": src["conventions"]["sphere"],
        "radius": src["radius"],
        "cases": [{"ka": c["ka"], "num_terms": c["num_terms"], "coefficients": c["coefficients"]}
                  for c in src["sphere"]],
    }
    json.dump(mie, open(os.path.join(HERE, "mie_rigid_golden.json"), "w"), indent=1)

    src = json.load(open(os.path.join(wave, "special-golden-wolfram-v1.json")))
    bes = {
        "source": "crates/sonium-wave/fixtures/special-golden-wolfram-v1.json",
        "conventions": src["conventions"],
        "cases": [{k: c[k] for k in ("name", "x", "j", "y", "j_derivative", "y_derivative")}
                  for c in src["spherical"]],
    }
    json.dump(bes, open(os.path.join(HERE, "spherical_bessel_golden.json"), "w"), indent=1)

    src = json.load(open(os.path.join(fm, "wolfram-golden-v1.json")))
    sc = {
        "source": "crates/sonium-fastmath/fixtures/wolfram-golden-v1.json",
        "conventions": src["conventions"],
        "cases": src["cases"],
    }
    json.dump(sc, open(os.path.join(HERE, "sincos_golden.json"), "w"), indent=1)
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".json")))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
