"""Extracts the reference's own golden vectors into tests/golden/reference_vectors.json.

    python tests/golden/make_reference_golden.py /path/to/reference

Reads, from the reference project (read-only):
  doc/example/{3_3,4_4,5_5,5_5_bis}.txt           example puzzles (CSV)
  tests/new_strategy_*/test.info                    expected stdout lines (spiral order)
  tests/new_strategy_*/references/results.bin       solution dumps
  tests/CUDA_glutton_max_*/test.info                glutton max final boards
  tests_CUDA/backtracker_*/test.info                row-major first solutions and, for 3_3, the
                                                    variable-space kernel's selection lines
  tests/dump_solutions_*/test.info                  FSM-engine totals (cross-check only)
The JSON is committed; the tests never read the reference at run time.
"""
from __future__ import annotations

import base64
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def expected_lines(path):
    out = []
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            if line.startswith("expected_stdout_string:"):
                out.append(line[len("expected_stdout_string:"):])
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_reference_golden.py /path/to/reference")
    ref = sys.argv[1]
    data = {"source": "reference project tests and doc/example", "puzzles": {}, "new_strategy": {},
            "glutton_max": {}, "backtracker_first_solution": {}, "backtracker_trace": {}, "dump_solutions": {}}
    for name in ("3_3", "4_4", "5_5", "5_5_bis"):
        with open(os.path.join(ref, "doc", "example", name + ".txt")) as f:
            data["puzzles"][name] = f.read()
    for name in ("3_3", "4_4", "5_5"):
        t = os.path.join(ref, "tests", "new_strategy_" + name)
        with open(os.path.join(t, "references", "results.bin"), "rb") as f:
            rb = f.read()
        data["new_strategy"][name] = {"strategy": "spiral", "expected_stdout": expected_lines(os.path.join(t, "test.info")),
                                      "results_bin_b64": base64.b64encode(rb).decode()}
        data["glutton_max"][name] = expected_lines(os.path.join(ref, "tests", "CUDA_glutton_max_" + name, "test.info"))
        bt_lines = expected_lines(os.path.join(ref, "tests_CUDA", "backtracker_" + name, "test.info"))
        data["backtracker_first_solution"][name] = bt_lines[-1]
        data["backtracker_trace"][name] = bt_lines[:-1]
        data["dump_solutions"][name] = expected_lines(os.path.join(ref, "tests", "dump_solutions_" + name, "test.info"))
    with open(os.path.join(HERE, "reference_vectors.json"), "w") as f:
        json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
