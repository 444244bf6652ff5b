"""The C++ host layer (edge_matching_puzzle_b200/csrc/host) through its command line,
checked the way the reference's own tests check its binary: the arguments of
tests/*/test.info and the stdout lines they expect.

CPU tests cover argument handling and error behaviour (ERROR line, exit code -1, as
src/main.cpp:137-146); GPU tests run the two CUDA features on the reference examples."""
from __future__ import annotations

import os
import subprocess

import pytest

from edge_matching_puzzle_b200 import build as native_build

CLI = native_build.CLI


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        native_build.build()
    assert os.path.exists(CLI), "the host command line was not built"
    return CLI


@pytest.fixture()
def example(tmp_path, reference_vectors):
    def write(name):
        path = tmp_path / f"{name}.txt"
        path.write_text(reference_vectors["puzzles"][name])
        return str(path)
    return write


def run(cli, *args, timeout=300):
    r = subprocess.run([cli, *args], capture_output=True, text=True, timeout=timeout)
    return r.returncode, r.stdout.splitlines()


def test_unsupported_feature(cli, example):
    rc, out = run(cli, example("3_3"), "ressources", "no_such_feature", "--enable_gui=false")
    assert rc == 255
    assert out[0] == "9 pieces loaded"
    assert out[-1].startswith('ERROR : Unsupported feature "no_such_feature" at ')


def test_missing_definition_file(cli, tmp_path):
    rc, out = run(cli, str(tmp_path / "missing.txt"), "ressources", "CUDA_backtracker")
    assert rc == 255 and out[-1].startswith("ERROR : Unable to open file")


def test_piece_count_mismatch(cli, tmp_path, reference_vectors):
    lines = reference_vectors["puzzles"]["3_3"].strip().splitlines()
    path = tmp_path / "short.txt"
    path.write_text("\n".join(lines[:-1]) + "\n")
    rc, out = run(cli, str(path), "ressources", "CUDA_glutton_max")
    assert rc == 255 and "Inconsistency between puzzle dimensions (3*3) and piece number (8)" in out[-1]


@pytest.mark.parametrize("args,msg", [
    (["--strategy=zigzag"], 'Unable to open file "zigzag"'),
    (["--colour=3"], 'Unknown parameter "colour"'),
    (["--stop_at_first=maybe"], 'Bad boolean value "maybe"'),
])
def test_bad_options(cli, example, args, msg):
    rc, out = run(cli, example("3_3"), "ressources", "CUDA_backtracker", *args)
    assert rc == 255 and msg in out[-1]


def test_usage(cli):
    rc, out = run(cli)
    assert rc == 255 and "usage" in out[-1]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_glutton_max_reference_lines(cli, example, reference_vectors, name):
    """tests/CUDA_glutton_max_<name>/test.info: Launch kernels, the header line, the board."""
    rc, out = run(cli, example(name), "ressources", "CUDA_glutton_max", "--enable_gui=false")
    assert rc == 0, out
    expected = reference_vectors["glutton_max"][name]
    pos = 0
    for line in out:
        if pos < len(expected) and line == expected[pos]:
            pos += 1
    assert pos == len(expected), (expected, out)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_backtracker_first_solution_and_totals(cli, example, reference_vectors, name):
    """tests_CUDA/backtracker_<name>: the first solution board (row-major order); with the
    spiral order, the totals of tests/new_strategy_<name>."""
    rc, out = run(cli, example(name), "ressources", "CUDA_backtracker", "--enable_gui=false")
    assert rc == 0, out
    assert reference_vectors["backtracker_first_solution"][name] in out
    rc, out = run(cli, example(name), "ressources", "CUDA_backtracker", "--strategy=spiral")
    assert rc == 0, out
    expected = [l for l in reference_vectors["new_strategy"][name]["expected_stdout"]
                if l.startswith(("Total situations explored", "Nb solutions"))]
    assert all(l in out for l in expected), (expected, out)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_new_strategy_results_bin_matches_reference(cli, example, reference_vectors, tmp_path, name):
    """tests/new_strategy_<name>: the GPU search writes the reference's own results.bin
    byte for byte (spiral order, every solution with its node index) and the totals."""
    import base64
    dump = tmp_path / "results.bin"
    rc, out = run(cli, example(name), "ressources", "new_strategy", "--enable_gui=false", f"--dump_file={dump}")
    assert rc == 0, out
    golden = reference_vectors["new_strategy"][name]
    assert dump.read_bytes() == base64.b64decode(golden["results_bin_b64"])
    expected = [l for l in golden["expected_stdout"] if l.startswith(("Total situations explored", "Nb solutions"))]
    assert all(l in out for l in expected), (expected, out)


def test_new_strategy_reports_errors_like_the_other_features(cli, tmp_path, reference_vectors):
    """A bad order for new_strategy is refused before any search, with the ERROR line."""
    path = tmp_path / "3_3.txt"
    path.write_text(reference_vectors["puzzles"]["3_3"])
    rc, out = run(cli, str(path), "ressources", "new_strategy", "--strategy=zigzag", f"--dump_file={tmp_path / 'r.bin'}")
    assert rc == 255 and 'Unable to open file "zigzag"' in out[-1]
    assert not (tmp_path / "r.bin").exists()


def _write_strategy(path, positions, comment=True):
    lines = (["# x,y of each position in visiting order"] if comment else []) + [f"{x},{y}" for x, y in positions]
    path.write_text("\n".join(lines) + "\n")


@pytest.mark.parametrize("content,msg", [
    ("0,0\n1\n", "Missing ',' character in line 2"),
    ("0,0\n1,\n", "Missing information after ',' character in line 2"),
    ("0,0\n1,0\n", "Incomplete strategy file"),
    ("0,0\n0,0\n0,1\n0,2\n1,1\n1,2\n2,0\n2,1\n2,2\n", "does not list every position once"),
])
def test_text_strategy_errors(cli, example, tmp_path, content, msg):
    """include/emp_text_strategy_generator.h:66-107: the text strategy's error lines."""
    strat = tmp_path / "strat.txt"
    strat.write_text(content)
    rc, out = run(cli, example("3_3"), "ressources", "CUDA_backtracker", f"--strategy={strat}")
    assert rc == 255 and msg in out[-1], out


def test_bad_initial_situation(cli, example):
    rc, out = run(cli, example("3_3"), "ressources", "CUDA_backtracker", "--initial_situation=1N2N")
    assert rc == 255 and "Situation string of 4 characters, expected 18" in out[-1]


@pytest.mark.gpu
def test_new_text_strategy_reads_strategy_txt(cli, reference_vectors, tmp_path):
    """new_text_strategy takes its order from ./strategy.txt: the spiral written as text
    gives the reference's own new_strategy results.bin."""
    import base64
    from edge_matching_puzzle_b200.puzzle import spiral_order
    (tmp_path / "4_4.txt").write_text(reference_vectors["puzzles"]["4_4"])
    _write_strategy(tmp_path / "strategy.txt", [(p % 4, p // 4) for p in spiral_order(4, 4)])
    r = subprocess.run([cli, "4_4.txt", "ressources", "new_text_strategy", "--dump_file=r.bin"], capture_output=True,
                       text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stdout
    golden = reference_vectors["new_strategy"]["4_4"]
    assert (tmp_path / "r.bin").read_bytes() == base64.b64decode(golden["results_bin_b64"])


@pytest.mark.gpu
def test_new_strategy_initial_situation_matches_reference_build(cli, tmp_path):
    """--initial_situation: totals and results.bin of the reference's own build resumed
    from the same situation (tests/golden/ref_counts.json)."""
    import hashlib
    import json
    recs = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_counts.json")))["records"]
    for rec in [r for r in recs if r["group"] == "resume"][:6]:
        (tmp_path / "p.txt").write_text(rec["csv"])
        dump = tmp_path / "r.bin"
        rc, out = run(cli, str(tmp_path / "p.txt"), "ressources", "new_strategy", f"--strategy={rec['order']}",
                      f"--initial_situation={rec['initial_situation']}", f"--dump_file={dump}")
        assert rc == 0, out
        assert f"Total situations explored : {rec['nodes']}" in out and f"Nb solutions : {rec['solutions']}" in out
        assert hashlib.sha256(dump.read_bytes()).hexdigest() == rec["results_sha256"], rec["name"]


@pytest.mark.gpu
def test_backtracker_trace_mode_lines(cli, example, reference_vectors):
    """--trace=true: the lines of tests_CUDA/backtracker_3_3/test.info, in order."""
    rc, out = run(cli, example("3_3"), "ressources", "CUDA_backtracker", "--enable_gui=false", "--trace=true")
    assert rc == 0, out
    expected = reference_vectors["backtracker_trace"]["3_3"] + [reference_vectors["backtracker_first_solution"]["3_3"]]
    got = [l for l in out if l.startswith("Thread ") or l == expected[-1]]
    assert got == expected, out


def test_trace_mode_refuses_other_orders(cli, example):
    rc, out = run(cli, example("3_3"), "ressources", "CUDA_backtracker", "--trace=true", "--strategy=spiral")
    assert rc == 255 and "row-major" in out[-1], out


def _reference_info_lines(words):
    """CUDA_piece_position_info2's printer (include/CUDA_piece_position_info2.h:315-352),
    restated here to check the host layer's C++ one."""
    lines = []
    for w, word in enumerate(words):
        if not word:
            continue
        lines.append("/" + "-" * 8 + f" Word[{w:2d}] : 0x{word:08x} " + "-" * 8 + "\\")
        lines.append("".join(f"|{8 * w + k:4d}" for k in range(8)) + "|")
        cells = []
        for k in range(8):
            nib = (word >> (4 * k)) & 0xF
            cells.append("|" + "".join("NESW"[o] if (nib >> o) & 1 else " " for o in range(4)))
        lines.append("".join(cells) + "|")
    return lines


@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_glutton_wide_prints_the_first_situation(cli, example, reference_vectors, name):
    """CUDA_glutton_wide: the reference's launcher prints the glutton's first situation
    (src/CUDA_glutton_wide.cu:27-37, CUDA_glutton_situation::print); its infos equal
    the oracle's first glutton level, which the glutton trajectory tests pin."""
    from edge_matching_puzzle_b200 import native
    from edge_matching_puzzle_b200.puzzle import Puzzle
    from oracle.oracle import OraclePuzzle
    pz = Puzzle.from_csv(reference_vectors["puzzles"][name])
    n = pz.width * pz.height
    want = OraclePuzzle(pz.width, pz.height, pz.colors).glutton_initial()
    assert native.glutton_wide_situation(native.NativePuzzle(pz.width, pz.height, pz.colors), n) == want
    rc, out = run(cli, example(name), "ressources", "CUDA_glutton_wide", "--enable_gui=false")
    assert rc == 0
    expect = ["Situation Level 0: ", "Situation Index 0: ", "===== Position index <-> Info index ====="]
    expect += [f"Position[{j}] -> Index {j}" for j in range(n)] + [f"Index[{j}] -> Position {j}" for j in range(n)]
    for title in ("Info", "Theoric info"):
        for j in range(n):
            expect += [f"{title}[{j}]:"] + _reference_info_lines(want[j]) + [""]
    expect += [""]
    assert out[1:] == expect
