"""Generates tests/golden/advec_13x9.npz from the compiled OP-PIC reference.

Runs oracle/_ref/advec_ref_seq (the reference seq backend and the generated NESO-advection seq
loops, built by oracle/Makefile from the reference sources) for 7 steps of update_pos + move on
a seeded 13 x 9 periodic mesh with fast particles (multi-hop moves), and stores the inputs with
the final positions, move directions and cells.  Requires the reference sources:

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


if __name__ == "__main__":
    main()
