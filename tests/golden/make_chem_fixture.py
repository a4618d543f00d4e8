"""Builds the chemistry fixture under tests/golden/chem/ from the reference's input files.

The reacting cases use the reference's 9-species H2/air mechanism (input/chemistry/H2_mech.inp) with
its NASA-7 and transport databases.  This script copies the mechanism and extracts from therm.dat
and tran.dat only the entries of the mechanism's species (plus the section keywords), so the
fixture stays small and the tests do not need the reference tree at run time.

    python tests/golden/make_chem_fixture.py <reference input dir>
"""
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent / "chem"


def species_of(mech: str):
    toks = []
    for line in mech.split("\n"):
        toks += line.split("!")[0].split()
    i = [t.upper() for t in toks].index("SPECIES")
    out = []
    for t in toks[i + 1:]:
        if t.upper() in ("END", "REACTIONS", "REAC", "THERMO"):
            break
        out.append(t.upper())
    return out


def main(src: Path):
    HERE.mkdir(parents=True, exist_ok=True)
    mech = (src / "chemistry" / "H2_mech.inp").read_text()
    names = set(species_of(mech))
    (HERE / "H2_mech.inp").write_text(mech)
    th = (src / "chemistry" / "therm.dat").read_text().split("\n")
    out = th[:2]  # THERMO keyword and the default temperature line
    p = 2
    while p < len(th):
        line = th[p]
        key = line[:18].split()
        if key and key[0].upper() == "END":
            break
        if key and len(line) >= 80 and line[79] == "1":
            if key[0].upper() in names:
                out += th[p:p + 4]
            p += 4
            continue
        p += 1
    out.append("END")
    (HERE / "therm.dat").write_text("\n".join(out) + "\n")
    tr = [l for l in (src / "chemistry" / "tran.dat").read_text().split("\n") if l.split() and l.split()[0].upper() in names]
    (HERE / "tran.dat").write_text("\n".join(tr) + "\n")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_chem_fixture.py <the reference's input directory>")
    main(Path(sys.argv[1]))
