"""Generates the golden fixtures of tests/golden/ from the compiled OP-PIC reference.

Runs oracle/_ref/fempic_ref_seq_stable (the reference seq backend and the generated
FemPIC seq loops, built by oracle/Makefile from the reference sources) on small seeded
cases and stores inputs (mesh arrays, injection tables) with the reference's per-step
records and final particle state.  Requires the reference sources (oracle/_ref built):

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "op-pic_b200"))
sys.path.insert(0, str(ROOT))

from oppb.fempic import HostMesh, injection_randoms  # noqa: E402
from oracle import ref_runner as R  # noqa: E402

CASES = {
    # name: (mesh dims, inject per step, steps, fill, period, seed)
    "fempic_4x4x8_holefill": ((4, 4, 8, 1.0, 1.0, 2.0), 100, 30, "HoleFill_All", 10, 1),
    "fempic_4x4x8_sort": ((4, 4, 8, 1.0, 1.0, 2.0), 100, 30, "Sort_Periodic", 4, 2),
}
# Global-move (direct-hop) case: the reference builds its structured map with grid spacing
# 0.1 and the app's expansion of 4 spacings (fempic_opp.cpp:69-76), and seeds every walk
# from it; dt 0.3 makes particles cross cells each step.
DH_CASES = {
    # name: (mesh dims, inject, steps, fill, period, seed, dt, spacing)
    "fempic_4x4x8_dh": ((4, 4, 8, 1.0, 1.0, 2.0), 100, 30, "Sort_Periodic", 5, 3, 0.3, 0.1),
}


def make(name: str) -> Path:
    dh_spec = DH_CASES.get(name)
    if dh_spec:
        dims, inject, steps, fill, period, seed, dt, spacing = dh_spec
    else:
        dims, inject, steps, fill, period, seed = CASES[name]
        dt, spacing = 0.01, None
    hm = HostMesh(*dims)
    dist = hm.inject_distribution(inject)
    tables = [injection_randoms(seed, s, inject, 0.1) for s in range(steps)]
    extra = {}
    if spacing is None:
        ref = R.run("seq_stable", hm, dist, steps, tables, fill=fill, period=period)
    else:
        ref = R.run("seq_stable", hm, dist, steps, tables, fill=fill, period=period, dt=dt,
                    dh=(spacing, (4 * spacing,) * 3))
        extra = dict(dt=dt, spacing=spacing, n_pos=hm.n_pos, dh_dims=ref["dh_dims"], dh_box=ref["dh_box"],
                     dh_map=ref["dh_map"])
    out = HERE / f"{name}.npz"
    np.savez_compressed(
        out, **extra, dims=np.array(dims), inject=inject, steps=steps, fill=fill, period=period, seed=seed,
        c2n=hm.c2n, c2c=hm.c2c, c_det=hm.c_det, c_vol=hm.c_vol, c_ef=hm.c_ef, if2c=hm.if2c, if_u=hm.if_u,
        if_v=hm.if_v, if_norm=hm.if_norm, if_n_pos=hm.if_n_pos, dist=dist, tables=np.stack(tables),
        records=ref["records"], p2c=ref["p2c"], pos=ref["pos"], vel=ref["vel"], lc=ref["lc"],
        node_charge=ref["node_charge"], n_nodes=hm.n_nodes, n_cells=hm.n_cells, n_ifaces=hm.n_ifaces)
    return out


if __name__ == "__main__":
    if not R.available("seq_stable"):
        sys.exit("oracle/_ref/fempic_ref_seq_stable missing: build it with `make -C oracle`")
    for n in list(CASES) + list(DH_CASES):
        print("wrote", make(n))
