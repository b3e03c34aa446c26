"""Writes the golden fixtures of the reference's own regression tests for
the PMG path: the input decks of the [born], [ionize] and [solv] sections
of tests/test_cases.cfg in the APBS tree, their PQR molecules and the
expected energies listed there, as JSON beside this script.

    APBS_REF_DIR=<APBS tree> python tests/golden/make_fixtures.py

Only the keywords these decks use are read (read/mol pqr, elec blocks of
mg-auto or mg-manual with their grid, physics and surface keywords, print
elecEnergy); the expected values are the "Total electrostatic energy" of
every calculation in order followed by each print statement's "Global net
ELEC energy" (tests/apbs_tester.py:127-135), in kJ/mol.  The unit constants
come from src/generic/vunit.h."""
import json
import os
import re
import sys

REF = os.environ.get("APBS_REF_DIR", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
SECTIONS = {"born": ["apbs-smol-auto", "apbs-mol-auto"],
            "ionize": ["apbs-mol", "apbs-smol"],
            "solv": ["apbs-mol", "apbs-smol"]}


def tokens(path):
    out = []
    for line in open(path):
        line = line.split("#", 1)[0]
        out.extend(line.split())
    return out


def read_pqr(path):
    atoms = []
    for line in open(path):
        if line.startswith(("ATOM", "HETATM")):
            f = line.split()
            # ... x y z charge radius are the last five fields
            x, y, z, q, r = (float(v) for v in f[-5:])
            atoms.append([x, y, z, q, r])
    return atoms


def parse_deck(path):
    t = tokens(path)
    i = 0
    mols, elecs, prints = [], [], []
    while i < len(t):
        w = t[i].lower()
        if w == "read":
            i += 1
            while t[i].lower() != "end":
                assert t[i].lower() == "mol" and t[i + 1].lower() == "pqr", t[i:i + 3]
                mols.append(t[i + 2])
                i += 3
            i += 1
        elif w == "elec":
            i += 1
            blk = {"ions": []}
            while t[i].lower() != "end":
                k = t[i].lower()
                if k == "name":
                    blk["name"] = t[i + 1]; i += 2
                elif k in ("mg-auto", "mg-manual"):
                    blk["type"] = k; i += 1
                elif k in ("lpbe", "npbe"):
                    blk["eq"] = k; i += 1
                elif k in ("dime", "cglen", "fglen", "glen", "grid"):
                    blk[k] = [float(v) for v in t[i + 1:i + 4]]; i += 4
                elif k in ("gcent", "cgcent", "fgcent"):
                    if t[i + 1].lower() == "mol":
                        blk[k] = {"mol": int(t[i + 2])}; i += 3
                    else:
                        blk[k] = [float(v) for v in t[i + 1:i + 4]]; i += 4
                elif k == "mol":
                    blk["mol"] = int(t[i + 1]); i += 2
                elif k == "ion":
                    a = {t[i + 1 + 2 * m].lower(): float(t[i + 2 + 2 * m]) for m in range(3)}
                    blk["ions"].append([a["charge"], a["conc"], a["radius"]]); i += 7
                elif k in ("bcfl", "chgm", "srfm", "calcenergy", "calcforce"):
                    blk[k] = t[i + 1].lower(); i += 2
                elif k in ("pdie", "sdie", "srad", "swin", "sdens", "temp"):
                    blk[k] = float(t[i + 1]); i += 2
                elif k == "write":
                    i += 4
                else:
                    raise SystemExit("%s: keyword %r not handled" % (path, t[i]))
            elecs.append(blk)
            i += 1
        elif w == "print":
            assert t[i + 1].lower() == "elecenergy", t[i:i + 3]
            j = i + 2
            terms = []
            sign = 1.0
            while t[j].lower() != "end":
                if t[j] in ("+", "-"):
                    sign = 1.0 if t[j] == "+" else -1.0
                else:
                    terms.append([sign, t[j]])
                j += 1
            prints.append(terms)
            i = j + 1
        elif w == "quit":
            break
        else:
            raise SystemExit("%s: top-level keyword %r not handled" % (path, t[i]))
    return mols, elecs, prints


def expected(section, deck):
    txt = open(os.path.join(REF, "tests", "test_cases.cfg")).read()
    sec = re.search(r"^\[%s\]\n(.*?)(?=^\[|\Z)" % re.escape(section), txt, re.S | re.M).group(1)
    m = re.search(r"^%s\s*:\s*(.*)$" % re.escape(deck), sec, re.M)
    return [float(v) for v in m.group(1).split()]


def units():
    txt = open(os.path.join(REF, "src", "generic", "vunit.h")).read()
    get = lambda name: float(re.search(r"#define\s+%s\s+([-+0-9.eE]+)" % name, txt).group(1))
    return {"Vunit_kb": get("Vunit_kb"), "Vunit_Na": get("Vunit_Na")}


def main():
    for section, decks in SECTIONS.items():
        d = os.path.join(REF, "examples", section)
        for deck in decks:
            mols, elecs, prints = parse_deck(os.path.join(d, deck + ".in"))
            fx = {"section": section, "deck": deck,
                  "source": "examples/%s/%s.in, tests/test_cases.cfg [%s]" % (section, deck,
                                                                             section),
                  "molecules": [{"file": m, "atoms": read_pqr(os.path.join(d, m))} for m in mols],
                  "elec": elecs, "print": prints, "expected_kJ_per_mol": expected(section, deck),
                  "units": units(),
                  "check": "round both to 6 significant figures; pass if equal or the relative "
                           "error is below 1e-4 (tests/apbs_check_results.py:27-54)"}
            out = os.path.join(HERE, "%s_%s.json" % (section, deck))
            with open(out, "w") as f:
                json.dump(fx, f, indent=1)
            print("wrote", out, len(fx["expected_kJ_per_mol"]), "values")


if __name__ == "__main__":
    sys.exit(main())
