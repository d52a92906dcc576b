"""Generates tests/golden/field_loops_4x4x8.npz from the compiled OP-PIC reference: the
generated seq loops compute_node_charge_density_kernel and compute_electric_field_kernel
(oracle/_ref/field_ref_seq, built by oracle/Makefile from the reference sources) on a
4x4x8-hex mesh, with the shape derivatives of FESolver's set-up and seeded charge and
potential.  Requires oracle/_ref:

    python tests/golden/make_golden_field.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "op-pic_b200"))
sys.path.insert(0, str(ROOT))

from oppb.fempic import HostMesh  # noqa: E402
from oracle import field as F  # noqa: E402


def make() -> Path:
    hm = HostMesh(4, 4, 8, 1.0, 1.0, 2.0, solve_field=False)
    fs = F.FieldSystem(hm.n_pos, hm.n_type, F.boundary_potential(hm.n_type, 1.0, 0.0), hm.c2n)
    rng = np.random.default_rng(17)
    den = rng.random(hm.n_nodes) * 50.0
    pot = rng.normal(0.0, 1.0, hm.n_nodes)
    spwt = 0.37
    den_out, ef = F.run_reference(den, hm.n_vol, spwt, hm.c2n, fs.c_sd, pot)
    out = HERE / "field_loops_4x4x8.npz"
    np.savez_compressed(out, dims=np.array([4, 4, 8, 1.0, 1.0, 2.0]), den=den, n_vol=hm.n_vol, spwt=spwt,
                        c2n=hm.c2n, c_sd=fs.c_sd, potential=pot, den_out=den_out, c_ef=ef)
    return out


if __name__ == "__main__":
    print("wrote", make())
