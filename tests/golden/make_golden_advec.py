"""Generates tests/golden/advec_13x9.npz and advec_dh_9x8.npz from the compiled OP-PIC reference.

Runs oracle/_ref/advec_ref_seq (the reference seq backend and the generated NESO-advection seq
loops, built by oracle/Makefile from the reference sources) for 7 steps of update_pos + move on
a seeded 13 x 9 periodic mesh with fast particles (multi-hop moves), and stores the inputs with
the final positions, move directions and cells.  The second fixture turns the global move on
(opp_init_direct_hop_cg with grid spacing 0.7 on a 9 x 8 mesh of unit cells, so that grid boxes
straddle cell edges) with a quarter of the particles resting on a cell's lower x edge and a
quarter on its lower y edge, where the seed decides the cell; it also stores the reference's
grid (box counts, bounds) and structured map.  Requires the reference sources:

    python tests/golden/make_golden_advec.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "op-pic_b200"))
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

from helpers import advec_edge_particles  # noqa: E402
from oppb.advec import AdvecMesh, particles  # noqa: E402
from oracle import advec as OA  # noqa: E402

NX, NY, CW, DT, PPC, STEPS, V_SD, SEED = 13, 9, 0.7, 0.35, 30, 7, 2.0, 1


def main() -> None:
    m = AdvecMesh(NX, NY, CW)
    pos, vel, mdir, p2c = particles(m, PPC, V_SD, SEED)
    ref = OA.run_reference("seq", NX, NY, CW, DT, pos, vel, mdir, p2c, m.c2c, m.c_pos_ll, STEPS)
    out = HERE / "advec_13x9.npz"
    np.savez_compressed(out, nx=NX, ny=NY, cell_width=CW, dt=DT, steps=STEPS, pos=pos, vel=vel, mdir=mdir, p2c=p2c,
                        ref_pos=ref["pos"], ref_mdir=ref["mdir"], ref_p2c=ref["p2c"])
    print("wrote", out)
    main_dh()


DH = dict(nx=9, ny=8, cell_width=1.0, dt=0.5, ppc=15, steps=7, v_sd=0.5, seed=79, grid_spacing=0.7)


def main_dh() -> None:
    c = DH
    m = AdvecMesh(c["nx"], c["ny"], c["cell_width"])
    pos, vel, mdir, p2c = advec_edge_particles(m, c["ppc"], c["v_sd"], c["seed"])
    ref = OA.run_reference("seq", c["nx"], c["ny"], c["cell_width"], c["dt"], pos, vel, mdir, p2c, m.c2c,
                           m.c_pos_ll, c["steps"], dh_spacing=c["grid_spacing"])
    out = HERE / "advec_dh_9x8.npz"
    np.savez_compressed(out, **c, pos=pos, vel=vel, mdir=mdir, p2c=p2c, ref_pos=ref["pos"], ref_mdir=ref["mdir"],
                        ref_p2c=ref["p2c"], ref_dims=ref["dims"], ref_box=ref["box"], ref_map=ref["map"])
    print("wrote", out)


if __name__ == "__main__":
    main()
