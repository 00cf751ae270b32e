"""The autotuner's table selection and header writer, on a synthetic
measurement log (no GPU): the fastest single-system shape per mesh,
cluster size included, and the lane-width rule; the written header compiles
and the no-allocation entry's compile-time bound sees cluster launches."""
import importlib
import os
import subprocess

import pytest


def at():
    return importlib.import_module("hornofusion-full3d_b200.autotune")


LOG = [
    {"mesh": [12, 24, 16], "solver": "single", "block": 256, "grid": 8, "us_per_iter": 6.9},
    {"mesh": [12, 24, 16], "solver": "single", "block": 288, "grid": 16, "cluster": 16,
     "us_per_iter": 3.6},
    {"mesh": [60, 120, 84], "solver": "single", "block": 512, "grid": 148, "us_per_iter": 13.9},
    {"mesh": [60, 120, 84], "solver": "single", "block": 512, "grid": 144, "cluster": 8,
     "us_per_iter": 16.9},
    {"mesh": [60, 120, 84], "solver": "single", "block": 512, "grid": 148, "stream": 1,
     "us_per_iter": 12.5},
    {"mesh": [12, 24, 16], "solver": "lane", "width": 1, "us_per_iter": 7.0},
    {"mesh": [12, 24, 16], "solver": "lane", "width": 2, "us_per_iter": 6.0},
    {"mesh": [12, 24, 16], "solver": "lane", "width": 8, "us_per_iter": 2.0},
]


def test_select_keeps_fastest_shape_with_its_cluster_size():
    single, lanes = at().select(LOG)
    assert single == [((12, 24, 16), 288, 16, 16, 0, 3.6),
                      ((60, 120, 84), 512, 148, 1, 1, 12.5)]
    # least t(w) * w among t(w) <= 2.5 x the fastest: 8 x 2.0 = 16 < 7.0 and 12.0 excluded
    assert lanes == [((12, 24, 16), 8, 2.0)]


def test_written_header_compiles(tmp_path):
    single, lanes = at().select(LOG)
    path = tmp_path / "tune_table.h"
    at().write_header(single, lanes, str(path))
    text = path.read_text()
    assert "{12, 24, 16, 288, 16, 16, 0}," in text and "{60, 120, 84, 512, 148, 1, 1}," in text
    src = tmp_path / "use.cc"
    src.write_text('#include "tune_table.h"\n'
                   "static_assert(eaf::max_tuned_grid_up_to(32768) == 16, \"bound\");\n"
                   "int main() { int b, g, c, t; return eaf::tuned_single_launch(12, 24, 16, &b, &g, &c, &t)"
                   " && c == 16 && t == 0 ? 0 : 1; }\n")
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", str(tmp_path), str(src)],
                   check=True)
