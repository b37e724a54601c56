"""Writes tests/golden/scoring_ref.json from the reference's own sources: the
smina atom-type table (src/lib/atom_constants.h, default_data), vinardo's
table (src/lib/builtinscoring.cpp, vinardo_data), smina's AD4-name
equivalences and non-AD metal names (atom_constants.h), and the builtin
scoring functions' term strings and weights (builtinscoring.cpp,
builtin_scoring::builtin_scoring).  The tests restate the terms and the
tables from this data (tests/scoring_restated.py), so the engine's host
tables are checked against the reference's constants, not against the
engine's own copy of them.

    python tests/golden/make_scoring_ref.py [REFERENCE_TREE]

REFERENCE_TREE defaults to $SMINA_REF (the checked-out reference project).
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

ROW = re.compile(r'\{\s*(\w+),\s*EL_TYPE_(\w+),\s*AD_TYPE_\w+,\s*XS_TYPE_\w+,\s*"(\w+)",\s*"(\w+)",\s*'
                 + r',\s*'.join([r'([-\d.]+)'] * 6) + r',\s*'
                 + r',\s*'.join([r'(true|false)'] * 4) + r'\s*\}')
FIELDS = ("ad_radius", "ad_depth", "ad_solvation", "ad_volume", "covalent_radius", "xs_radius")
FLAGS = ("xs_hydrophobe", "xs_donor", "xs_acceptor", "ad_heteroatom")


def table(text, name):
    start = text.index(f"const info {name}[NumTypes] = {{")
    end = text.index("};", start)
    rows = []
    for m in ROW.finditer(text[start:end]):
        g = m.groups()
        row = {"sm": g[0], "element": g[1], "smina_name": g[2], "adname": g[3]}
        row.update({k: float(v) for k, v in zip(FIELDS, g[4:10])})
        row.update({k: v == "true" for k, v in zip(FLAGS, g[10:14])})
        rows.append(row)
    assert len(rows) == 27, (name, len(rows))
    return rows


def builtins(text):
    start = text.index("builtin_scoring::builtin_scoring()")
    end = text.index("\n}", start)
    funcs = {}
    for line in text[start:end].splitlines():
        m = re.match(r'\s*add\("(\w+)",\s*"([^"]+)",\s*(.+?)\);\s*$', line)
        if m:
            expr = m.group(3)
            assert re.fullmatch(r"[-+*/. 0-9]+", expr), expr
            funcs.setdefault(m.group(1), []).append([m.group(2), eval(expr)])  # plain arithmetic, left to right
        m = re.match(r'\s*functions\["(\w+)"\]\s*=\s*functions\["(\w+)"\];', line)
        if m:
            funcs[m.group(1)] = list(funcs[m.group(2)])
    return funcs


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SMINA_REF", "")
    if not ref:
        sys.exit("give the reference tree as an argument or in SMINA_REF")
    ac = open(os.path.join(ref, "src/lib/atom_constants.h")).read()
    bs = open(os.path.join(ref, "src/lib/builtinscoring.cpp")).read()
    eq = re.search(r"atom_equivalence_data\[\]\s*=\s*\{(.*?)\};", ac, re.S).group(1)
    metals = re.search(r"non_ad_metal_names\[\]\s*=\s*\{(.*?)\};", ac, re.S).group(1)
    out = {
        "source": "src/lib/atom_constants.h (default_data, atom_equivalence_data, non_ad_metal_names); "
                  "src/lib/builtinscoring.cpp (vinardo_data, builtin_scoring::builtin_scoring)",
        "types": table(ac, "default_data"),
        "vinardo_types": table(bs, "vinardo_data"),
        "equivalences": re.findall(r'\{\s*"(\w+)",\s*"(\w+)"\s*\}', eq),
        "non_ad_metals": re.findall(r'"(\w+)"', metals),
        "functions": builtins(bs),
    }
    path = os.path.join(HERE, "scoring_ref.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path, "functions:", sorted(out["functions"]))


if __name__ == "__main__":
    main()
