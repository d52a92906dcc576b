"""Generates tests/golden/cabana_4x5x6.npz from the compiled OP-PIC reference.

Runs oracle/_ref/cabana_ref_seq (the reference seq backend and the generated CabanaPIC seq
loops, built by oracle/Makefile from the reference sources): three successive
opp_reset_dat(c_acc) + opp_particle_move__move_deposit_kernel calls on a seeded case with
multi-hop streaks, and stores the inputs with the final particle dats and the last c_acc.
Requires the reference sources (oracle/_ref built):

    python tests/golden/make_golden_cabana.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "op-pic_b200"))
sys.path.insert(0, str(ROOT))

from oppb.cabana import HexMesh, synthetic_interp  # noqa: E402
from oracle import cabana as OC  # noqa: E402

DIMS = (4, 5, 6)
N = 2000
CALLS = 3
CONSTS = dict(qdt_2mc=-0.3, cdt_d=(1.7, 0.9, 2.3), qsp=-1.0)


def case(seed: int = 7):
    mesh = HexMesh(*DIMS)
    rng = np.random.default_rng(seed)
    interp = synthetic_interp(mesh, seed + 1, e_scale=0.2, b_scale=0.3)
    p2c = np.sort(rng.choice(mesh.interior, N)).astype(np.int32)
    pos = rng.uniform(-1.0, 1.0, (N, 3))
    vel = rng.normal(0.0, 1.5, (N, 3))
    weight = rng.uniform(0.5, 1.5, N)
    return mesh, interp, pos, vel, np.zeros((N, 3)), weight, p2c


def main() -> None:
    mesh, interp, pos, vel, streak, weight, p2c = case()
    ref = OC.run_reference("seq", mesh.c2ngc, interp, pos, vel, streak, weight, p2c, CONSTS["qdt_2mc"],
                           CONSTS["cdt_d"], CONSTS["qsp"], calls=CALLS)
    out = HERE / "cabana_4x5x6.npz"
    np.savez_compressed(out, dims=np.array(DIMS), calls=CALLS, qdt_2mc=CONSTS["qdt_2mc"],
                        cdt_d=np.array(CONSTS["cdt_d"]), qsp=CONSTS["qsp"], interp=interp, pos=pos, vel=vel,
                        streak=streak, weight=weight, p2c=p2c, ref_pos=ref["pos"], ref_vel=ref["vel"],
                        ref_streak=ref["streak"], ref_p2c=ref["p2c"], ref_acc=ref["acc"])
    print("wrote", out)


if __name__ == "__main__":
    main()
