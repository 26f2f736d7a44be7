"""Regenerate the golden fixtures in this folder from a reference checkout.

The reference's own high-precision tables (mpmath, 30-90 digits), its Lean-model golden
tables and the known answers written into its test sources are copied value for value;
nothing is recomputed. Only rows that pin the hot path are kept:

- ``spherical_hankel.txt``  <- crates/treams-core/references/spherical_hankel.txt
- ``degrees.txt``           <- formal/golden/degrees.txt (coupling selection rules)
- ``harmonics.txt``         <- formal/golden/harmonics.txt (harmonic table index)
- ``lattice_sums_2d.txt``   <- references/lattice_sums.txt, 2D spherical rows only
- ``kambe.txt``, ``incgamma.txt``, ``incgamma_zero.txt`` <- references/ (Ewald integrals)
- ``known_answers.txt``     <- the literal values of three reference tests, read as text:
  the Mie blocks of a metallic sphere (crates/treams-core/src/coeffs/mie.rs,
  ``metallic_sphere_matches_independent_mie_ratios``), the 30-digit Wigner 3j value of
  tests/special/test_wigner.py (``test_wigner3j_in_every_argument_order``) and the SiC
  chain absorption of tests/tmatrix/test_particle_cluster.py
  (``test_small_wavenumber_high_order_chain_absorption_is_stable``).

Run from the repository root: ``python tests/golden/make_fixtures.py <reference_root>``.
"""
import pathlib
import re
import sys

HERE = pathlib.Path(__file__).resolve().parent

NUM = r"-?[0-9][0-9_]*\.?[0-9_]*(?:e-?[0-9]+)?"


def _f(s: str) -> str:
    """A Rust or Python float literal as plain text (digit separators removed)."""
    return s.replace("_", "")


def _function_body(text: str, name: str) -> str:
    start = text.index(name)
    return text[start:start + 4000]


def known_answers(ref: pathlib.Path) -> list[str]:
    rows = ["# Known answers of reference tests (values copied as written there).",
            "# mie l x eps_re eps_im: diagonal_re diagonal_im off_re off_im  (helicity 2x2 block, vacuum outside)",
            "# wigner3j j1 j2 j3 m1 m2 m3: value",
            "# sic_chain_absorption_1e12: value rtol"]
    mie = (ref / "crates" / "treams-core" / "src" / "coeffs" / "mie.rs").read_text()
    body = _function_body(mie, "fn metallic_sphere_matches_independent_mie_ratios")
    eps = re.search(r"epsilon: Complex::new\((" + NUM + r"), (" + NUM + r")\)", body)
    x = re.search(r"mie\(l, &\[(" + NUM + r")\]", body)
    for m in re.finditer(r"\(\s*(\d+),\s*\((" + NUM + r"), (" + NUM + r")\),\s*\((" + NUM + r"), (" + NUM + r")\),?\s*\)",
                         body):
        l, d0, d1, o0, o1 = m.groups()
        rows.append(f"mie {l} {_f(x.group(1))} {_f(eps.group(1))} {_f(eps.group(2))}: "
                    f"{_f(d0)} {_f(d1)} {_f(o0)} {_f(o1)}")
    wig = (ref / "tests" / "special" / "test_wigner.py").read_text()
    body = _function_body(wig, "def test_wigner3j_in_every_argument_order")
    # the first argument tuple of the parametrize list just above the test
    head = wig[wig.index("def test_wigner3j_in_every_argument_order") - 300:]
    args = re.search(r"\[\((\d+), (\d+), (\d+), (-?\d+), (-?\d+), (-?\d+)\)", head)
    value = re.search(r"assert_allclose\(special\.wigner3j\(\*arguments\), (" + NUM + r")", body)
    rows.append("wigner3j " + " ".join(args.groups()) + ": " + _f(value.group(1)))
    sic = (ref / "tests" / "tmatrix" / "test_particle_cluster.py").read_text()
    body = _function_body(sic, "def test_small_wavenumber_high_order_chain_absorption_is_stable")
    val = re.search(r"assert_allclose\(absorption \* 1e12, (" + NUM + r"), rtol=(" + NUM + r")", body)
    rows.append(f"sic_chain_absorption_1e12: {_f(val.group(1))} {_f(val.group(2))}")
    return rows


def main(root: str) -> None:
    ref = pathlib.Path(root)
    refs = ref / "crates" / "treams-core" / "references"
    copies = {
        "spherical_hankel.txt": refs / "spherical_hankel.txt",
        "degrees.txt": ref / "formal" / "golden" / "degrees.txt",
        "harmonics.txt": ref / "formal" / "golden" / "harmonics.txt",
        "kambe.txt": refs / "kambe.txt",
        "incgamma.txt": refs / "incgamma.txt",
        "incgamma_zero.txt": refs / "incgamma_zero.txt",
    }
    for name, src in copies.items():
        (HERE / name).write_text(src.read_text())
    rows = []
    for line in (refs / "lattice_sums.txt").read_text().splitlines():
        if line.startswith("#"):
            rows.append(line)
            continue
        fields = line.split()
        # `s l m dim ...`: keep the 2D spherical sums
        if len(fields) > 3 and fields[0] == "s" and fields[3] == "2":
            rows.append(line)
    (HERE / "lattice_sums_2d.txt").write_text("\n".join(rows) + "\n")
    (HERE / "known_answers.txt").write_text("\n".join(known_answers(ref)) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <reference_root>")
    main(sys.argv[1])
