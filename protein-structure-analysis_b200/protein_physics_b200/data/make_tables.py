"""Regenerates residue_tables.json and ff_params.json from the reference.

Run in a checkout that has the reference tree (the ALMA sources):

    python make_tables.py /path/to/reference

The bonded graph of a residue has to be the reference's exactly — 1-2/1-3
exclusions, j-side sets and the dihedral-record atoms (first neighbour in
adjacency order, physics_engine.cpp:1542-1552) all depend on it, including
the order in which bonds are inserted.  So the per-residue bond lists
(bond_templates(), physics_engine.cpp:577-1007) and rotatable-bond specs
(rot_specs(), :1019-1108) are read out of the reference source text here and
stored as data, in their original order, rather than re-typed.  Likewise the
ff14SB charges / R* / epsilon are looked up through the reference's own
python/amber_params.get_atom_params (amber_params.py:928) for every atom name
the templates and terminal patches can produce.
"""
import json
import os
import re
import sys


def _strip_comments(src):
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _body(src, marker):
    start = src.index(marker)
    start = src.index("= {", start) + 2
    depth, i = 0, start
    while True:
        c = src[i]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return src[start:i + 1]
        i += 1


def _tokens(text):
    return re.findall(r'"[^"]*"|[{}]|K::[A-Z_]+', text)


def _parse_map(body):
    """Parses `{ {"RES", { {..}, {..} }}, ... }` into an ordered dict."""
    toks = _tokens(body)
    out, i = {}, 1  # skip the outer '{'
    while i < len(toks) and toks[i] != "}" or (i < len(toks) and toks[i] == "{"):
        if toks[i] != "{":
            i += 1
            continue
        name = toks[i + 1].strip('"')
        i += 3  # '{' NAME '{'
        entries = []
        while toks[i] == "{":
            j = toks.index("}", i)
            entries.append([t.strip('"').replace("K::", "") for t in toks[i + 1:j]])
            i = j + 1
        assert toks[i] == "}" and toks[i + 1] == "}", (name, toks[i:i + 3])
        out[name] = entries
        i += 2
    return out


def extract_templates(ref_root):
    src = open(os.path.join(ref_root, "src", "physics_engine.cpp"), encoding="utf-8").read()
    src = _strip_comments(src)
    macros = dict(re.findall(r"#define\s+(_BB\w*)\s+([^\n]+)", src))
    b = _body(src, "bond_templates() {")
    for name in sorted(macros, key=len, reverse=True):
        b = re.sub(r"\b%s\b" % name, macros[name], b)
    bonds = _parse_map(b)
    rots = _parse_map(_body(src, "rot_specs() {"))
    return bonds, rots


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ALMA_REFERENCE", "")
    if not ref or not os.path.isdir(ref):
        sys.exit("usage: %s REFERENCE_TREE (or set ALMA_REFERENCE): the reference checkout" % sys.argv[0])
    here = os.path.dirname(os.path.abspath(__file__))
    bonds, rots = extract_templates(ref)
    for k, v in bonds.items():
        assert all(len(e) == 2 for e in v), k
    for k, v in rots.items():
        assert all(len(e) == 3 for e in v), k
    with open(os.path.join(here, "residue_tables.json"), "w") as f:
        json.dump({"bond_templates": bonds, "rot_specs": rots}, f, indent=0, sort_keys=False)

    sys.path.insert(0, os.path.join(ref, "python"))
    import amber_params as ap  # noqa: E402

    params = {}
    terminal = ["H1", "H2", "H3", "OXT", "HE2"]
    for res, pairs in bonds.items():
        names = []
        for a, b_ in pairs:
            for nm in (a, b_):
                if nm not in names:
                    names.append(nm)
        for nm in names + terminal:
            params["%s:%s" % (res, nm)] = list(ap.get_atom_params(res, nm))
    with open(os.path.join(here, "ff_params.json"), "w") as f:
        json.dump(params, f, indent=0)
    print("residues:", len(bonds), "rot-spec residues:", len(rots), "param entries:", len(params))


if __name__ == "__main__":
    main()
