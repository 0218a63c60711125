"""Extracts the ff19SB protein data the synthetic peptide builder needs into
dynamics_b200/data/ff19sb.json:

* residue templates from amino19.lib (atom names, types, charges, template
  coordinates, intra-residue bonds, head/tail atoms);
* masses, LJ (R*, eps), bond, angle, proper and improper dihedral
  parameters from parm19.dat with frcmod.ff19SB applied on top.

The reference ships these files under param_data/ and reads them through
its bio_files dependency; this script is run once where the reference tree
is present and its output is committed:

    python dynamics_b200/data/make_ff19sb.py /path/to/reference/param_data
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_lib(path):
    lines = open(path).read().splitlines()
    res = {}
    cur = None
    i = 0
    while i < len(lines):
        ln = lines[i]
        m = re.match(r"!entry\.(\w+)\.unit\.(\w+)", ln)
        if m:
            name, sec = m.group(1), m.group(2)
            cur = res.setdefault(name, {"atoms": [], "bonds": [], "pos": [], "connect": []})
            i += 1
            while i < len(lines) and not lines[i].startswith("!"):
                t = lines[i].split()
                if sec == "atoms":
                    cur["atoms"].append({"name": t[0].strip('"'), "type": t[1].strip('"'),
                                         "charge": float(t[7])})
                elif sec == "connectivity":
                    cur["bonds"].append([int(t[0]) - 1, int(t[1]) - 1])
                elif sec == "positions":
                    cur["pos"].append([float(x) for x in t[:3]])
                elif sec == "connect":
                    cur["connect"].append(int(t[0]) - 1)
                i += 1
            continue
        i += 1
    return res


def _types(field, n):
    return [t.strip() for t in field.split("-")][:n]


def parse_parm(path, frcmod=False):
    """Sections of a parm .dat or frcmod file as lists of parsed entries."""
    lines = open(path).read().splitlines()
    out = {"mass": {}, "bond": [], "angle": [], "dihe": [], "impr": [], "nonb": {}, "equiv": []}
    if frcmod:
        sec = None
        for ln in lines[1:]:
            s = ln.strip()
            head = s[:4].upper()
            if head in ("MASS", "BOND", "ANGL", "DIHE", "IMPR", "NONB", "CMAP", "HBON"):
                sec = head
                continue
            if not s or sec is None:
                continue
            _entry(out, sec, ln)
        return out
    # parm.dat: fixed section order separated by blank lines
    i = 1
    order = ["MASS", "HYDROPHILIC", "BOND", "ANGL", "DIHE", "IMPR", "HBON", "EQUIV"]
    k = 0
    while k < len(order) and i < len(lines):
        sec = order[k]
        if sec == "HYDROPHILIC":
            i += 1
            k += 1
            continue
        while i < len(lines) and lines[i].strip():
            if sec == "EQUIV":
                out["equiv"].append(lines[i].split())
            elif sec != "HBON":
                _entry(out, sec, lines[i])
            i += 1
        i += 1
        k += 1
    # NONB after "MOD4 RE"
    while i < len(lines) and not lines[i].startswith("MOD4"):
        i += 1
    i += 1
    while i < len(lines) and lines[i].strip() and not lines[i].startswith("END"):
        _entry(out, "NONB", lines[i])
        i += 1
    return out


def _entry(out, sec, ln):
    if sec == "MASS":
        t = ln.split()
        out["mass"][t[0]] = float(t[1])
    elif sec == "BOND":
        ty = _types(ln[:5], 2)
        t = ln[5:].split()
        out["bond"].append([ty, float(t[0]), float(t[1])])
    elif sec == "ANGL":
        ty = _types(ln[:8], 3)
        t = ln[8:].split()
        out["angle"].append([ty, float(t[0]), float(t[1])])
    elif sec == "DIHE":
        ty = _types(ln[:11], 4)
        t = ln[11:].split()
        out["dihe"].append([ty, float(t[0]), float(t[1]), float(t[2]), float(t[3])])
    elif sec == "IMPR":
        ty = _types(ln[:11], 4)
        t = ln[11:].split()
        out["impr"].append([ty, float(t[0]), float(t[1]), float(t[2])])
    elif sec == "NONB":
        t = ln.split()
        if len(t) >= 3:
            out["nonb"][t[0]] = [float(t[1]), float(t[2])]


def merge(parm, frc):
    """frcmod on top of parm: entries for the same types replace the parm
    ones (a dihedral's whole multi-term set is replaced)."""
    m = {"mass": dict(parm["mass"]), "nonb": dict(parm["nonb"])}
    m["mass"].update(frc["mass"])
    m["nonb"].update(frc["nonb"])
    for eq in parm["equiv"]:
        base = eq[0]
        for t in eq[1:]:
            if t not in m["nonb"] and base in m["nonb"]:
                m["nonb"][t] = m["nonb"][base]

    def key(ty):
        return "-".join(ty) if ty <= ty[::-1] else "-".join(ty[::-1])

    for sec in ("bond", "angle"):
        d = {key(e[0]): e for e in parm[sec]}
        for e in frc[sec]:
            d[key(e[0])] = e
        m[sec] = list(d.values())

    def group(entries):
        g = {}
        order = []
        for e in entries:
            k = key(e[0])
            if k not in g:
                g[k] = []
                order.append(k)
            g[k].append(e)
        return g, order

    gp, op = group(parm["dihe"])
    gf, of = group(frc["dihe"])
    for k in of:
        gp[k] = gf[k]
        if k not in op:
            op.append(k)
    m["dihe"] = [e for k in op for e in gp[k]]
    d = {}
    for e in parm["impr"] + frc["impr"]:
        d["-".join(e[0])] = e
    m["impr"] = list(d.values())
    return m


def main(src):
    lib = parse_lib(os.path.join(src, "amino19.lib"))
    parm = parse_parm(os.path.join(src, "parm19.dat"))
    frc = parse_parm(os.path.join(src, "frcmod.ff19SB"), frcmod=True)
    ff = merge(parm, frc)
    out = {"residues": lib, "params": ff,
           "source": "amino19.lib, parm19.dat, frcmod.ff19SB (reference param_data)"}
    with open(os.path.join(HERE, "ff19sb.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("residues", len(lib), "types", len(ff["mass"]), "bonds", len(ff["bond"]), "angles",
          len(ff["angle"]), "dihedrals", len(ff["dihe"]), "impropers", len(ff["impr"]))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_ff19sb.py <reference param_data directory>")
    main(sys.argv[1])
