"""qdyn's coordinate trajectory (.dcd) and its atom mask.

The file is what Q's trj module writes (src/q6/trj.f90:184-259) as gfortran
sequential unformatted records: a header record of 'CORD' and 20 int32
(frames, steps before the first frame, interval, steps, 0, 0, 0, free degrees
of freedom, 0 fixed atoms, 0, 0, 0 x 8, CHARMM version 0); a title record
(int32 count = 2 + mask rows, then 80-character rows: the title, the
topology file name, each mask row); a record with the number of atoms
written; then per frame three records of float32 x, y and z of the masked
atoms in atom order.

The mask follows mask_add / update (src/q6/mask.f90:118-372): every
[trajectory_atoms] row adds the atoms it selects; a row is a list of words,
ALL, NOT (or -) negating the next property, SOLUTE, EXCLUDED (EXCL),
RESTRAINED (in the restrained shell or excluded), HEAVY, and an atom range
"first [last]" (1-based).  A property not named accepts both values.
Residue numbering and SYBYL types are not part of this path and are refused.
"""
from __future__ import annotations

import struct

import numpy as np

from .inputs import inp_sections  # noqa: F401  (re-exported for the qdyn driver)

TITLE = "Q DCD trajectory version 6.0.1"


def _record(payload: bytes) -> bytes:
    n = struct.pack("<i", len(payload))
    return n + payload + n


def _row(text: str) -> bytes:
    return text.encode("ascii", "replace")[:80].ljust(80, b" ")


def atom_mask(view, rows) -> np.ndarray:
    """Boolean mask over the system's atoms for the given mask rows (no
    rows: every atom, as qdyn does without a [trajectory_atoms] section)."""
    n, ns = view.natom, view.nat_solute
    solute = np.arange(n) < ns
    excl = np.array(view.excl[:n], dtype=bool)
    heavy = np.array(view.heavy[:n], dtype=bool)
    shell = np.array(view.shell[:n], dtype=bool)
    restrained = shell | excl
    mask = np.zeros(n, dtype=bool)
    for line in (rows or ["all"]):
        words = line.replace("\t", " ").split()
        sel = {"solute": None, "excl": None, "restr": None, "heavy": None}
        first, last, empty, neg = 1, n, True, False
        k = 0
        while k < len(words):
            w = words[k].upper()
            if w == "ALL":
                neg, empty = False, False
            elif w in ("NOT", "-"):
                neg = True
            elif w in ("SOLUTE", "EXCLUDED", "EXCL", "RESTRAINED", "HEAVY"):
                key = {"SOLUTE": "solute", "EXCLUDED": "excl", "EXCL": "excl", "RESTRAINED": "restr",
                       "HEAVY": "heavy"}[w]
                sel[key] = not neg
                neg, empty = False, False
            elif w in ("RESIDUE", "RES", "RESI", "SYBYL"):
                raise ValueError("trajectory mask '%s': residue numbering and SYBYL types are not supported" % w)
            else:
                try:
                    first = int(w)
                except ValueError:
                    raise ValueError("trajectory mask: unrecognized property %s" % words[k]) from None
                if first < 1 or first > n:
                    raise ValueError("trajectory mask: invalid first atom %d" % first)
                empty = False
                if k + 1 < len(words):
                    last = int(words[k + 1])
                    if last < first or last > n:
                        raise ValueError("trajectory mask: invalid last atom %s" % words[k + 1])
                else:
                    last = first
                break
            k += 1
        if empty:
            continue
        ok = np.zeros(n, dtype=bool)
        ok[first - 1:last] = True
        for key, prop in (("solute", solute), ("excl", excl), ("restr", restrained), ("heavy", heavy)):
            if sel[key] is not None:
                ok &= prop == sel[key]
        mask |= ok
    return mask


class DcdWriter:
    """Writes qdyn's trajectory: header at creation, one frame per write()."""

    def __init__(self, path: str, mask: np.ndarray, *, frames: int, interval: int, steps: int, degf: int,
                 topology: str, mask_rows):
        self.mask = np.asarray(mask, dtype=bool)
        rows = list(mask_rows) or ["all"]
        hdr = struct.pack("<4s20i", b"CORD", frames, interval, interval, steps, 0, 0, 0, degf,
                          0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0)
        title = struct.pack("<i", 2 + len(rows)) + _row(TITLE) + _row(topology) + b"".join(_row(r) for r in rows)
        self.f = open(path, "wb")
        self.f.write(_record(hdr) + _record(title) + _record(struct.pack("<i", int(self.mask.sum()))))

    def write(self, x) -> None:
        xm = np.asarray(x, dtype=np.float64).reshape(-1, 3)[self.mask].astype("<f4")
        for c in range(3):
            self.f.write(_record(np.ascontiguousarray(xm[:, c]).tobytes()))
        self.f.flush()

    def close(self) -> None:
        self.f.close()


def read_dcd(path: str):
    """(header dict, frames[n, atoms, 3] float32) of a qdyn trajectory."""
    raw = open(path, "rb").read()
    recs, pos = [], 0
    while pos + 4 <= len(raw):
        (n,) = struct.unpack_from("<i", raw, pos)
        recs.append(raw[pos + 4:pos + 4 + n])
        pos += 8 + n
    h = struct.unpack("<4s20i", recs[0])
    nrows = struct.unpack_from("<i", recs[1])[0]
    rows = [recs[1][4 + 80 * k:4 + 80 * (k + 1)].decode().rstrip() for k in range(nrows)]
    natoms = struct.unpack("<i", recs[2])[0]
    fr = recs[3:]
    frames = np.array([np.stack([np.frombuffer(fr[3 * k + c], dtype="<f4") for c in range(3)], axis=1)
                       for k in range(len(fr) // 3)], dtype=np.float32).reshape(-1, natoms, 3)
    header = {"type": h[0].decode(), "frames": h[1], "steps_before": h[2], "interval": h[3], "steps": h[4],
              "degf": h[8], "title": rows[0], "topology": rows[1], "mask_rows": rows[2:], "atoms": natoms}
    return header, frames


def frame_steps(nsteps: int, interval: int) -> list[int]:
    """Completed-step counts at which qdyn writes a frame: after the step of
    every iteration istep > 0 that is a multiple of the interval
    (md.f90:4151), and after the loop when nsteps is one (md.f90:4202)."""
    if interval <= 0:
        return []
    out = [k * interval + 1 for k in range(1, (nsteps - 1) // interval + 1)]
    if nsteps % interval == 0:
        out.append(nsteps)
    return out
