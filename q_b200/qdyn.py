"""Drop-in replacement of the `qdyn` executable for one input file.

    python -m q_b200.qdyn md.inp > md.log

Reads the same .inp/.top/.fep/.re as qdyn (src/q6/qdyn.f90:18-134), runs the
MD steps on the GPU, and writes what the reference's scripts consume: the
energy file (.en, put_ene records, nrgy.f90:94-119), the final restart (.re,
write_xfin, md.f90:15452-15470), the coordinate trajectory (.dcd of the
[trajectory_atoms] mask every `trajectory` steps, trj.f90:184-259, written at
md.f90:4151 and 4202; q_b200/trajectory.py) and an energy-summary log laid out
as write_out (md.f90:15292-15440), ending with "terminated normally".
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np


def _fmt_label(label: str, values) -> str:
    # format (A, T17, 6F10.2)
    return "%-16s%s" % (label, "".join("%10.2f" % v for v in values))


def write_out(E, EQ, step: int | None, nstates: int, nwat: int, use_lrf: bool, nqat: int, nat_solute: int,
              offd=None) -> str:
    """One energy summary in write_out's layout; offd = [(i, j, Hij, k, l,
    r_kl)] of the EVB off-diagonal functions (states and Q atoms 1-based)."""
    e = dict(zip(__import__("q_b200").E_NAMES, E))
    L = []
    if step is None:
        L.append("=========================== FINAL %15s =============================" % "Energy summary")
    else:
        L.append("======================= %15s at step %6d ========================" % ("Energy summary", step))
    L.append(" " * 16 + "".join("%10s" % h for h in ("el", "vdW", "bond", "angle", "torsion", "improper")))
    L.append(_fmt_label("solute", [e["pp_el"], e["pp_vdw"], e["p_bond"], e["p_angle"], e["p_torsion"], e["p_improper"]]))
    if nwat > 0:
        L.append(_fmt_label("solvent", [e["ww_el"], e["ww_vdw"], e["w_bond"], e["w_angle"], e["w_torsion"], e["w_improper"]]))
    L.append(_fmt_label("solute-solvent", [e["pw_el"], e["pw_vdw"]]))
    if use_lrf:
        L.append(_fmt_label("LRF", [e["LRF"]]))
    if nqat > 0:
        L.append(_fmt_label("Q-atom", [e["qx_el"], e["qx_vdw"], e["q_bond"], e["q_angle"], e["q_torsion"], e["q_improper"]]))
    L.append("")
    L.append(" " * 16 + "".join("%10s" % h for h in ("total", "fix", "slvnt_rad", "slvnt_pol", "shell", "solute")))
    L.append(_fmt_label("restraints", [e["rst_total"], e["rst_fix"], e["rst_solvent_radial"], e["rst_water_pol"],
                                       e["rst_shell"], e["rst_protein"]]))
    L.append("")
    L.append(" " * 16 + "".join("%10s" % h for h in ("total", "potential", "kinetic")))
    L.append(_fmt_label("SUM", [e["potential"] + e["kinetic"], e["potential"], e["kinetic"]]))
    if nstates > 0:
        if step is None:
            L.append("=========================== FINAL %15s =============================" % "Q-atom energies")
        else:
            L.append("======================= %15s at step %6d ========================" % ("Q-atom energies", step))
        L.append("type   st lambda" + "".join("%10s" % h for h in ("el", "vdW", "bond", "angle", "torsion", "improper")))

        def row(name, st, a, b):
            return "%-7s%2d%7.4f%10.2f%10.2f" % (name, st + 1, EQ[st][0], a, b)

        for st in range(nstates):
            L.append(row("Q-Q", st, EQ[st][8], EQ[st][9]))
        L.append("")
        if nat_solute > nqat:
            for st in range(nstates):
                L.append(row("Q-prot", st, EQ[st][10], EQ[st][11]))
            L.append("")
        if nwat > 0:
            for st in range(nstates):
                L.append(row("Q-wat", st, EQ[st][12], EQ[st][13]))
            L.append("")
        for st in range(nstates):
            L.append(row("Q-surr.", st, EQ[st][10] + EQ[st][12], EQ[st][11] + EQ[st][13]))
        L.append("")
        for st in range(nstates):
            L.append("%-7s%2d%7.4f" % ("Q-any", st + 1, EQ[st][0]) + "".join("%10.2f" % EQ[st][k] for k in (6, 7, 2, 3, 4, 5)))
        L.append("")
        L.append("type   st lambda" + "%10s%10s" % ("total", "restraint"))
        for st in range(nstates):
            L.append(row("Q-SUM", st, EQ[st][1], EQ[st][14]))
        for i, j, h, k, l, r in offd or ():
            L.append("H(%2d,%2d) =%8.2f dist. between Q-atoms%4d%4d =%8.2f" % (i, j, h, k, l, r))
    L.append("=" * 79)
    return "\n".join(L)


def run(inp: str, out=sys.stdout, chunk: int = 1000) -> int:
    from q_b200 import Batch, System, append_energy, write_restart
    from q_b200._lib import QBError

    t0 = time.time()
    try:
        sys_ = System.open(inp)
        v = sys_.view
        batch = Batch([sys_])
    except QBError as e:
        print("!" * 79, file=out)
        print("ABNORMAL TERMINATION of qdyn: %s" % e, file=out)
        return 255
    ns = v.nstates
    d = os.path.dirname(os.path.abspath(inp))
    ene = None
    for line in open(inp):
        t = line.split()
        if len(t) >= 2 and t[0].lower() == "energy" and v.iene_cycle > 0:
            ene = os.path.join(d, t[1])
        if len(t) >= 2 and t[0].lower() == "final":
            final = os.path.join(d, t[1])
    if ene and os.path.exists(ene):
        os.remove(ene)
    trj, frames = None, []
    if v.itrj_cycle > 0:
        from q_b200.trajectory import DcdWriter, atom_mask, frame_steps, inp_sections
        sec = inp_sections(inp)
        files = dict((l.split()[0].lower(), l.split()[1]) for l in sec.get("files", []) if len(l.split()) >= 2)
        rows = sec.get("trajectory_atoms", [])
        try:
            mask = atom_mask(v, rows)
        except ValueError as e:
            print("!" * 79, file=out)
            print("ABNORMAL TERMINATION of qdyn: %s" % e, file=out)
            return 255
        print("Coordinates for%6d atoms will be written to the trajectory." % int(mask.sum()), file=out)
        trj = DcdWriter(os.path.join(d, files["trajectory"]), mask, frames=v.nsteps // v.itrj_cycle,
                        interval=v.itrj_cycle, steps=v.nsteps, degf=v.Ndegfree, topology=files.get("topology", ""),
                        mask_rows=rows)
        frames = frame_steps(v.nsteps, v.itrj_cycle)
    nod = v.noffd
    ij = np.array([[v.offd_i[k], v.offd_j[k]] for k in range(nod)], dtype=np.int32).reshape(-1, 2)

    def offd_rows(rec):
        return [(v.offd_i[k], v.offd_j[k], rec[k][0], v.offd_k[k] + 1, v.offd_l[k] + 1, rec[k][1]) for k in range(nod)]

    T = batch.temperature(0)
    print("Initial temperatures are : Ttot =%10.2f Tfree =%10.2f" % (T[0], T[1]), file=out)
    done = 0
    try:
        while done < v.nsteps:
            n = min(chunk, v.nsteps - done)
            nxt = [f for f in frames if f > done]
            if nxt:
                n = min(n, nxt[0] - done)
            batch.run(n)
            if trj and done + n in frames:
                trj.write(batch.coords(0))
            steps, E, EQ = batch.history(0, 0)
            od = batch.offdiag(0, 0) if nod else None
            for k in range(len(steps)):
                print(write_out(E[k], EQ[k], int(steps[k]), ns, v.nwat, bool(v.use_LRF), v.nqat, v.nat_solute,
                                offd_rows(od[k]) if nod else None), file=out)
            if ene:
                _, _, EQe = batch.history(0, 1)
                ode = batch.offdiag(0, 1) if nod else None
                for k in range(EQe.shape[0]):
                    append_energy(ene, EQe[k], (ij, ode[k]) if nod else None)
            batch.clear_history()
            done += n
        od_last = offd_rows(batch.offdiag(0, 2)[0]) if nod and v.nsteps > 0 else None
        batch.final_energy()
    except QBError as e:
        print("!" * 79, file=out)
        print("ABNORMAL TERMINATION of qdyn", file=out)
        print("Terminating due to %s" % e, file=out)
        return 255
    E, EQ = batch.energy_vectors(0)
    print("", file=out)
    print(write_out(E, EQ, None, ns, v.nwat, bool(v.use_LRF), v.nqat, v.nat_solute, od_last), file=out)
    if v.use_pbc and v.constant_pressure:
        # write_out's summary of the volume moves (md.f90:15425-15436)
        bx = batch.box(0)
        tries, acc = batch.volume_moves(0)
        print("", file=out)
        print("=========================== VOLUME CHANGE SUMMARY ===========================", file=out)
        print("Final volume: %10.3f" % (bx[0] * bx[1] * bx[2]), file=out)
        print("", file=out)
        print("%16s%10s%10s%10s" % ("", "total", "accepted", "ratio"), file=out)
        print("%-16s%10d%10d%10.3f" % ("Attempts", tries, acc, acc / tries if tries else 0.0), file=out)
        print("=" * 79, file=out)
    tc = batch.theta_corr(0, v.nwpolr_shell) if v.nwpolr_shell > 0 else None
    write_restart(final, batch.coords(0), batch.velocities(0), tc, batch.box(0) if v.use_pbc else None)
    if trj:
        trj.close()
    print("Total time of main loop: %24.1f(s)" % (time.time() - t0), file=out)
    print(" qdyn version 6.0.1 terminated normally.", file=out)
    return 0


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print("usage: python -m q_b200.qdyn file.inp", file=sys.stderr)
        return 2
    return run(argv[-1])


if __name__ == "__main__":
    sys.exit(main())
