"""Reading and deriving qdyn .inp files (the [section] format of
src/q6/md.f90:2528-3262).

`derive_inp` writes a copy of an input with some keys and sections replaced,
so that a protocol (heating stages, restarts, windows) can be run from the
user's own input without rewriting it by hand, the way QligFEP fills its
templates (qligfep.py:723 write_MD_1, INPUTS/eq1-5.inp).  File names in the
copy stay relative to the original's directory: the copy is written beside it.
"""
from __future__ import annotations

import os

# sections whose lines are lists (kept as rows) rather than "key value" pairs
ROW_SECTIONS = {"lambdas", "sequence_restraints", "distance_restraints", "angle_restraints", "wall_restraints",
                "atom_restraints", "trajectory_atoms", "excluded_groups"}


def inp_sections(path: str) -> dict:
    """{section: [lines]} of a qdyn .inp, in file order (text after '!' or
    '#' dropped, blank lines skipped, section names lower case)."""
    out, cur = {}, None
    for line in open(path):
        line = line.split("!")[0].split("#")[0].rstrip()
        s = line.strip()
        if not s:
            continue
        if s.startswith("[") and "]" in s:
            cur = s[1:s.index("]")].strip().lower()
            out.setdefault(cur, [])
        elif cur is not None:
            out[cur].append(s)
    return out


def derive_inp(src: str, dst_name: str, *, set_keys: dict | None = None, drop_keys: dict | None = None,
               set_rows: dict | None = None) -> str:
    """Write `dst_name` (a file name, placed beside `src`) as a copy of src
    with keys replaced: set_keys = {section: {key: value}} (added when
    missing, a section created when missing), drop_keys = {section: [keys]},
    set_rows = {section: [rows] or None} replaces (or, with None, removes) a
    list section.  Returns the new path."""
    sec = inp_sections(src)
    set_keys = {k.lower(): v for k, v in (set_keys or {}).items()}
    drop_keys = {k.lower(): {x.lower() for x in v} for k, v in (drop_keys or {}).items()}
    set_rows = {k.lower(): v for k, v in (set_rows or {}).items()}
    order = list(sec)
    for name in list(set_keys) + list(set_rows):
        if name not in sec and (name not in set_rows or set_rows[name] is not None):
            order.append(name)
            sec[name] = []
    L = []
    for name in order:
        if name in set_rows:
            if set_rows[name] is None:
                continue
            rows = list(set_rows[name])
        elif name in ROW_SECTIONS:
            rows = sec[name]
        else:
            pairs = []
            for line in sec[name]:
                t = line.split(None, 1)
                key = t[0].lower()
                if key in drop_keys.get(name, ()) or key in {k.lower() for k in set_keys.get(name, {})}:
                    continue
                pairs.append(line)
            pairs += ["%s %s" % (k, v) for k, v in set_keys.get(name, {}).items()]
            rows = pairs
        L += ["[%s]" % name] + rows + [""]
    path = os.path.join(os.path.dirname(os.path.abspath(src)), dst_name)
    with open(path, "w") as f:
        f.write("\n".join(L))
    return path
