"""The opp_* text I/O against the reference: oracle/io_check.cpp, one source built on the
reference's seq backend (oracle/_ref/io_check_seq) and on include/ + libopp_b200.so
(oracle/_ref/io_check_dropin), reads its cell dats and a map with opp_decl_dat_txt /
opp_decl_map_txt, writes them back with opp_print_dat_to_txtfile / opp_print_map_to_txtfile and
dumps a dat with opp_dump_dat.  The CPU tests pin the reference's output to the format of
opp_lib/src/core/opp_lib_file_core.cpp:35-178 restated here; the GPU tests require the drop-in's
files and stdout to equal the reference's byte for byte (file names aside: the reference's seq
backend writes <prefix>_seq_*, the CUDA backend the drop-in stands in for <prefix>_cuda_* and
<prefix>_cuda0__* for maps, opp_lib/src/cuda/opp_cuda.cu:458-481), and its error exits to match."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"
SEQ, DROPIN = REF / "io_check_seq", REF / "io_check_dropin"
PARAMS = ("STRING opp_fill = HoleFill_All\nINT opp_fill_period = 10\nREAL opp_allocation_multiple = 1.1\n"
          "BOOL opp_profile_all = false\n")
CELLS = 7
DATS = ["c_v1", "c_v3", "c_v16", "c_i2", "p_v"]
MAPS = ["c2n", "c2n1", "p2c"]
P2C = [3, 0, 6, 6, 1]
P_V = [1.5, -0.0, 0.0, -2.25e-300, 1e300, 3.0, -7.0, 0.1, 1.0 / 3.0, -1.0 / 3.0]
need_seq = pytest.mark.skipif(not SEQ.exists(), reason="compiled reference not built (needs its sources)")


def inputs(seed: int = 0) -> dict:
    rng = np.random.default_rng(seed)
    return {"c_v1": rng.normal(size=(CELLS, 1)), "c_v3": rng.normal(size=(CELLS + 1, 3)) * 1e5,
            "c_v16": rng.normal(size=(CELLS, 16)), "c_i2": rng.integers(-100, 100, size=(CELLS, 2)),
            "c2n": rng.integers(0, 9, size=(CELLS, 4))}


def with_one_based(a: dict) -> dict:
    """c2n1: c2n's entries plus 1, declared with OPP_maps_base_index = 1."""
    return {**a, "c2n1": a["c2n"] + 1}


def write_inputs(d: Path, arrays: dict, params: str = PARAMS) -> None:
    """The decl_*_txt files: a "rows dim" header, then one row of values a line (c_v3 holds one
    row more than the set, which the loader allows)."""
    (d / "in").mkdir(parents=True, exist_ok=True)
    (d / "files").mkdir(exist_ok=True)
    (d / "params.txt").write_text(params)
    for name, a in with_one_based(arrays).items():
        fmt = (lambda v: f"{float(v):.17g}") if a.dtype.kind == "f" else str
        rows = "".join(" ".join(fmt(v) for v in r) + "\n" for r in a)
        (d / "in" / f"{name}.txt").write_text(f"{a.shape[0]} {a.shape[1]}\n" + rows)


def run(exe: Path, d: Path, *extra: str) -> subprocess.CompletedProcess:
    return subprocess.run([str(exe), "params.txt", "in", *extra], cwd=d, capture_output=True, text=True, timeout=300)


def dump_block(out: str) -> str:
    return out[out.index("dump begin\n") + len("dump begin\n"):out.index("dump end\n")]


def expected_file(values: np.ndarray, size: int, is_double: bool) -> str:
    """opp_print_dat_to_txtfile_core on one rank: header, `size` rows, both marker lines."""
    dim = values.shape[1]
    lines = [f"{size} {dim} -- 0 0"]
    for r in values[:size]:
        lines.append("".join(" " + (format(0.0 if float(v) == 0.0 else float(v), ".25E") if is_double else str(int(v)))
                             for v in r))
    lines += ["import_exec_below " + "*" * 40, "import_non_exec_below " + "*" * 40]
    return "\n".join(lines) + "\n"


def expected_dump(values: np.ndarray) -> str:
    return "".join("".join("\t " + format(float(v), "+.25E") for v in r) + "\t\n" for r in values)


def names(backend: str) -> dict:
    pre = "io_seq_" if backend == "seq" else "io_cuda_"
    mpre = "io_seq_" if backend == "seq" else "io_cuda0__"
    return {**{n: f"{pre}{n}.dat" for n in DATS}, **{n: f"{mpre}{n}.dat" for n in MAPS}}


@need_seq
def test_reference_output_has_the_restated_format(tmp_path):
    a = inputs()
    write_inputs(tmp_path, a)
    r = run(SEQ, tmp_path)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    f = {k: (tmp_path / "files" / v).read_text() for k, v in names("seq").items()}
    for n in ("c_v1", "c_v3", "c_v16"):
        assert f[n] == expected_file(a[n], CELLS, True), n
    assert f["c_i2"] == expected_file(a["c_i2"], CELLS, False)
    assert f["c2n"] == expected_file(a["c2n"], CELLS, False)
    assert f["c2n1"] == f["c2n"]  # declared 1-based, held 0-based
    assert f["p2c"] == expected_file(np.array(P2C)[:, None], 5, False)
    pv = np.array(P_V).reshape(5, 2)
    assert f["p_v"] == expected_file(pv, 5, True)
    # The print left -0 as +0 in the host copy, so the dump that follows shows +0.
    assert dump_block(r.stdout) == expected_dump(np.where(pv == 0.0, 0.0, pv))


@need_seq
@pytest.mark.parametrize("case", ["missing", "dim", "rows", "value", "dim5"])
def test_reference_loader_errors(tmp_path, case):
    a = inputs()
    if case == "dim5":  # a dim the loader has no format for
        a["c_v1"] = np.zeros((CELLS, 5))
    write_inputs(tmp_path, a)
    p = tmp_path / "in" / "c_v1.txt"
    if case == "missing":
        p.unlink()
    elif case == "dim":
        p.write_text(p.read_text().replace(f"{CELLS} 1\n", f"{CELLS} 2\n", 1))
    elif case == "rows":
        p.write_text(p.read_text().replace(f"{CELLS} 1\n", f"{CELLS - 1} 1\n", 1))
    elif case == "value":
        p.write_text(p.read_text().rsplit("\n", 2)[0] + "\nnot-a-number\n")
    r = run(SEQ, tmp_path)
    assert r.returncode == 255
    assert not any((tmp_path / "files").iterdir())


@pytest.mark.gpu
@need_seq
@pytest.mark.parametrize("seed", [0, 1])
def test_dropin_text_io_equals_reference(tmp_path, seed):
    a = inputs(seed)
    outs = {}
    for backend, exe in (("seq", SEQ), ("dropin", DROPIN)):
        d = tmp_path / backend
        write_inputs(d, a)
        r = run(exe, d)
        assert r.returncode == 0, backend + ": " + r.stdout[-2000:] + r.stderr[-2000:]
        files = {k: (d / "files" / v).read_bytes() for k, v in names("seq" if backend == "seq" else "cuda").items()}
        assert sorted(p.name for p in (d / "files").iterdir()) == sorted(
            names("seq" if backend == "seq" else "cuda").values())
        outs[backend] = (files, dump_block(r.stdout), r.stdout)
    for k in outs["seq"][0]:
        assert outs["dropin"][0][k] == outs["seq"][0][k], k
    assert outs["dropin"][1] == outs["seq"][1]
    halo = [[ln for ln in outs[b][2].splitlines() if ln.startswith("halo ")] for b in ("seq", "dropin")]
    assert halo[0] == halo[1] == ["halo 7 5"]  # one rank: the loop runs over the set's own elements
    fetch = [ln for ln in outs["dropin"][2].splitlines() if ln.startswith("fetch ")]
    assert fetch == [f"fetch 1 {CELLS} {format(float(a['c_v3'][1, 1]), '.17g')}"]


GLOBAL_CASES = {
    "defaults": (PARAMS, ()),
    "periodic_no_period": (PARAMS.replace("HoleFill_All", "Sort_Periodic").replace("INT opp_fill_period = 10\n", ""),
                           ()),
    "periodic": (PARAMS.replace("HoleFill_All", "Shuffle_Periodic"), ()),
    "args": (PARAMS, ("OPP_ALLOC_MULT=2.5", "OPP_MPI_ALLOC_MULT=3", "OPP_DH_DATA_DUMP=1")),
}
GLOBALS_EXPECTED = {"defaults": "globals 2 -1 1.1000000000000001 1 0",
                    "periodic_no_period": "globals 2147483647 -1 1.1000000000000001 1 0",
                    "periodic": "globals 10 -1 1.1000000000000001 1 0",
                    # opp_set_args_core keeps 17 characters of "OPP_ALLOC_MULT=2.5": "2." reads as 2
                    "args": "globals 2 -1 2 3 1"}


def globals_line(out: str) -> str:
    return next(ln for ln in out.splitlines() if ln.startswith("globals "))


@need_seq
@pytest.mark.parametrize("case", sorted(GLOBAL_CASES))
def test_reference_globals(tmp_path, case):
    params, args = GLOBAL_CASES[case]
    write_inputs(tmp_path, inputs(), params)
    r = run(SEQ, tmp_path, "-", *args)
    assert r.returncode == 0, r.stdout[-2000:]
    assert globals_line(r.stdout) == GLOBALS_EXPECTED[case]


@pytest.mark.gpu
@need_seq
@pytest.mark.parametrize("case", sorted(GLOBAL_CASES))
def test_dropin_globals_equal_reference(tmp_path, case):
    """The fill period (a missing opp_fill_period of a periodic fill is INT_MAX, as there), the
    allocation multiples, the direct-hop dump flag and moreX_hops (-1, never counted)."""
    params, args = GLOBAL_CASES[case]
    write_inputs(tmp_path, inputs(), params)
    r = run(DROPIN, tmp_path, "-", *args)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert globals_line(r.stdout) == GLOBALS_EXPECTED[case]


@pytest.mark.gpu
@need_seq
@pytest.mark.parametrize("case", ["missing", "dim", "rows", "value", "dim5", "no_files_dir", "dump_int"])
def test_dropin_error_exits_equal_reference(tmp_path, case):
    """Loader errors end with status -1, an unwritable dump file with 2, and opp_dump_dat of an
    int dat ends the program with status 0 after the reference's message, on both libraries."""
    res = {}
    for backend, exe in (("seq", SEQ), ("dropin", DROPIN)):
        d = tmp_path / backend
        a = inputs()
        if case == "dim5":
            a["c_v1"] = np.zeros((CELLS, 5))
        write_inputs(d, a)
        p = d / "in" / "c_v1.txt"
        extra = ()
        if case == "missing":
            p.unlink()
        elif case == "dim":
            p.write_text(p.read_text().replace(f"{CELLS} 1\n", f"{CELLS} 2\n", 1))
        elif case == "rows":
            p.write_text(p.read_text().replace(f"{CELLS} 1\n", f"{CELLS - 1} 1\n", 1))
        elif case == "value":
            p.write_text(p.read_text().rsplit("\n", 2)[0] + "\nnot-a-number\n")
        elif case == "no_files_dir":
            (d / "files").rmdir()
        elif case == "dump_int":
            extra = ("dump_int",)
        r = run(exe, d, *extra)
        res[backend] = r
    assert res["dropin"].returncode == res["seq"].returncode, (res["seq"].returncode, res["dropin"].stderr[-1000:])
    assert res["seq"].returncode == {"no_files_dir": 2, "dump_int": 0}.get(case, 255)
    if case == "dump_int":
        for r in res.values():
            assert "Unsupported type for dumping int" in r.stdout and "dump end" not in r.stdout
