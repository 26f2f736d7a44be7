"""Regenerate the golden fixtures in this folder from the reference checkout.

The reference's own high-precision tables (mpmath, 30-90 digits) and its Lean-model
golden tables are copied row for row; nothing is recomputed. Only rows that pin the
hot path are kept:

- ``spherical_hankel.txt``  <- crates/treams-core/references/spherical_hankel.txt
- ``degrees.txt``           <- formal/golden/degrees.txt (coupling selection rules)
- ``harmonics.txt``         <- formal/golden/harmonics.txt (harmonic table index)
- ``lattice_sums_2d.txt``   <- references/lattice_sums.txt, 2D spherical rows only
- ``kambe.txt``, ``incgamma.txt``, ``incgamma_zero.txt`` <- references/ (Ewald integrals)

Run from the repository root: ``python tests/golden/make_fixtures.py [reference_root]``.
"""
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent


def main(root: str = "/root/reference") -> None:
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


if __name__ == "__main__":
    main(*sys.argv[1:])
