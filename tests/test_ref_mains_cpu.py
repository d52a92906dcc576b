"""The reference's generated NESO-advection and CabanaPIC mains on the reference's own seq
backend (oracle/_ref/advec_opp_seq, oracle/_ref/cabana_opp_seq, built by oracle/Makefile with
oracle/dump_at_exit.cpp): the side the GPU drop-in tests compare against.  Here, without a GPU,
they run a few steps and leave the log and the dat files those tests read."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"


@pytest.mark.skipif(not (REF / "advec_opp_seq").exists(), reason="compiled reference not built (needs its sources)")
@pytest.mark.parametrize("global_move", [False, True])
def test_reference_advection_main_on_seq(tmp_path, global_move):
    (tmp_path / "files").mkdir()
    (tmp_path / "params.txt").write_text(
        "INT num_steps = 12\nINT nx = 20\nINT ny = 16\nREAL dt = 0.5\nREAL cell_width = 0.5\n"
        "INT npart_per_cell = 10\nBOOL verify_particles = true\nREAL opp_allocation_multiple = 1.1\n"
        f"BOOL opp_profile_all = false\nBOOL opp_global_move = {'true' if global_move else 'false'}\n"
        "REAL grid_spacing = 0.5\nBOOL opp_dh_data_generate = true\nSTRING opp_fill = HoleFill_All\n")
    r = subprocess.run([str(REF / "advec_opp_seq"), "params.txt"], capture_output=True, text=True, timeout=120,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stdout[-2000:]
    log = [ln for ln in r.stdout.splitlines() if " - ts: " in ln]
    assert len(log) == 12 and all("errors: 0 |" in ln and "Gbl parts: 3200 " in ln for ln in log)
    names = sorted(p.name for p in (tmp_path / "files").iterdir())
    assert "final_seq_p_pos" in names and "final_seq_p_mesh_rel" in names
    head = (tmp_path / "files" / "final_seq_p_pos").read_text().splitlines()[0]
    assert head == "3200 2 -- 0 0"


@pytest.mark.skipif(not (REF / "cabana_opp_seq").exists(), reason="compiled reference not built (needs its sources)")
def test_reference_cabana_main_on_seq(tmp_path):
    (tmp_path / "files").mkdir()
    (tmp_path / "params.txt").write_text(
        "INT num_steps = 6\nREAL init_vel = 0.0866025403784439\nINT num_part_per_cell = 8\nINT nx = 4\nINT ny = 4\n"
        "INT nz = 12\nREAL c = 1.0\nREAL qsp = -1.0\nREAL me = 1.0\nREAL default_grid_len = 1.0\nREAL eps = 1.0\n"
        "STRING part_enrich = two_stream\nBOOL print_energy = true\nSTRING cluster = block\n"
        "REAL opp_allocation_multiple = 1.1\nBOOL opp_profile_all = false\nBOOL print_final = true\n"
        "STRING opp_fill = HoleFill_All\nINT domain_expansion = 1\nREAL velX_mult_const = 1\n"
        "REAL velY_mult_const = 0.00\nREAL velZ_mult_const = 0.00\n")
    r = subprocess.run([str(REF / "cabana_opp_seq"), "params.txt"], capture_output=True, text=True, timeout=120,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stdout[-2000:]
    log = [ln for ln in r.stdout.splitlines() if re.search(r" - ts: \d+ ", ln)]
    assert len(log) == 6 and all("e_energy:" in ln and "max_bx:" in ln for ln in log)
    energy = np.loadtxt(tmp_path / "energy.csv", delimiter=",", skiprows=1)
    assert energy.shape == (6, 3) and (energy[:, 1] > 0).all()
    names = sorted(p.name for p in (tmp_path / "files").iterdir())
    assert {"final_seq_p_pos", "final_seq_c_e", "final_seq_c_acc"} <= set(names)
