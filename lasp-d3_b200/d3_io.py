"""Structure files for the CLI and the MD harness: the reference's `.arc` format and
extended XYZ.

.arc (as read by the reference's d3_cpp): a block starts with a header line
``Energy <n> <force> <energy> [symmetry]``, a cell line ``PBC a b c alpha beta gamma``
(Angstrom, degrees) and atom lines of ten tokens ``symbol x y z ...`` (Angstrom).
The cell matrix from lengths and angles follows the crystallographic convention: a along
x, b in the xy plane, c completing the right-handed set.

extxyz: atom count, a comment line with ``Lattice="ax ay az bx by bz cx cy cz"`` (and any
other key=value pairs), then ``symbol x y z ...`` lines.
"""
import math
import re

import numpy as np

SYMBOLS = (
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
    "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb "
    "Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No Lr"
).split()
Z_OF_SYMBOL = {s: i + 1 for i, s in enumerate(SYMBOLS)}


def atomic_number(symbol):
    s = symbol.strip()
    if s in Z_OF_SYMBOL:
        return Z_OF_SYMBOL[s]
    s2 = s[:1].upper() + s[1:].lower()
    if s2 in Z_OF_SYMBOL:
        return Z_OF_SYMBOL[s2]
    raise ValueError("unknown element symbol %r" % symbol)


def cell_from_parameters(a, b, c, alpha, beta, gamma):
    """3x3 cell (rows = lattice vectors) from lengths (A) and angles (degrees)."""
    al, be, ga = (math.radians(x) for x in (alpha, beta, gamma))
    cx = c * math.cos(be)
    cy = c * (math.cos(al) - math.cos(be) * math.cos(ga)) / math.sin(ga)
    cz = math.sqrt(max(c * c - cx * cx - cy * cy, 0.0))
    return np.array([[a, 0.0, 0.0], [b * math.cos(ga), b * math.sin(ga), 0.0], [cx, cy, cz]])


def read_arc(path):
    """All structures of an .arc file: list of dicts with pos [n,3], Z [n], cell [3,3],
    energy (the header's value)."""
    out, cur = [], None
    with open(path) as f:
        for line in f:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "Energy" and len(tok) in (4, 5):
                if cur is not None:
                    out.append(cur)
                cur = {"pos": [], "Z": [], "cell": None, "energy": float(tok[3])}
            elif tok[0] == "PBC" and len(tok) == 7 and cur is not None:
                cur["cell"] = cell_from_parameters(*(float(x) for x in tok[1:7]))
            elif len(tok) == 10 and cur is not None:
                cur["Z"].append(atomic_number(tok[0]))
                cur["pos"].append([float(x) for x in tok[1:4]])
    if cur is not None:
        out.append(cur)
    for s in out:
        if s["cell"] is None:
            raise ValueError("%s: structure without a PBC line" % path)
        s["pos"] = np.array(s["pos"], float).reshape(-1, 3)
        s["Z"] = np.array(s["Z"], np.int64)
    return out


def read_extxyz(path):
    """All frames of an extended-XYZ file (periodic, Lattice key required)."""
    out = []
    with open(path) as f:
        lines = f.read().splitlines()
    k = 0
    while k < len(lines):
        if not lines[k].strip():
            k += 1
            continue
        n = int(lines[k].split()[0])
        comment = lines[k + 1]
        m = re.search(r'Lattice\s*=\s*"([^"]+)"', comment)
        if not m:
            raise ValueError("%s: frame without Lattice" % path)
        cell = np.array([float(x) for x in m.group(1).split()], float).reshape(3, 3)
        Z, pos = [], []
        for line in lines[k + 2:k + 2 + n]:
            tok = line.split()
            Z.append(atomic_number(tok[0]))
            pos.append([float(x) for x in tok[1:4]])
        e = re.search(r"(?:^|\s)energy\s*=\s*([-+0-9.eE]+)", comment)
        out.append({"pos": np.array(pos, float), "Z": np.array(Z, np.int64), "cell": cell,
                    "energy": float(e.group(1)) if e else None})
        k += 2 + n
    return out


def read_structures(path):
    """Frames of an .arc or extxyz file (chosen by the extension)."""
    p = path.lower()
    if p.endswith(".arc"):
        return read_arc(path)
    if p.endswith(".xyz") or p.endswith(".extxyz"):
        return read_extxyz(path)
    raise ValueError("unknown structure format: %s (.arc, .xyz, .extxyz)" % path)


def write_arc(path, structures):
    """Write structures in the .arc layout (header, PBC line, ten-token atom lines)."""
    with open(path, "w") as f:
        for s in structures:
            h = np.asarray(s["cell"], float)
            a, b, c = (np.linalg.norm(h[i]) for i in range(3))
            alpha = math.degrees(math.acos(np.dot(h[1], h[2]) / (b * c)))
            beta = math.degrees(math.acos(np.dot(h[0], h[2]) / (a * c)))
            gamma = math.degrees(math.acos(np.dot(h[0], h[1]) / (a * b)))
            f.write("Energy %d 0.0 %.6f C1\n" % (1, s.get("energy") or 0.0))
            f.write("PBC %.9f %.9f %.9f %.9f %.9f %.9f\n" % (a, b, c, alpha, beta, gamma))
            # positions in the frame of cell_from_parameters (a along x, b in the xy plane)
            target = cell_from_parameters(a, b, c, alpha, beta, gamma)
            frac = np.asarray(s["pos"], float) @ np.linalg.inv(h)
            pos = frac @ target
            for z, r in zip(s["Z"], pos):
                f.write("%-2s %16.9f %16.9f %16.9f CORE %d %s %s 0.0000 %d\n" % (SYMBOLS[int(z) - 1], r[0], r[1], r[2],
                                                                               1, SYMBOLS[int(z) - 1],
                                                                               SYMBOLS[int(z) - 1], 1))
            f.write("end\nend\n")
