"""The reference scripts' output files (no GPU): Julia's number printing, the column layout
the Matlab readers parse, and the MAT dumps."""
import json
import os

import numpy as np

from conftest import ROOT


def test_numbers_print_as_julia_prints_them():
    """Every number of the reference's own output files (tests/golden/reference_output_lines.json,
    made by tests/golden/make_output_lines.py) is reproduced character for character."""
    from ptstokes.output import jl
    lines = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_output_lines.json")))
    n = 0
    for f, rows in lines.items():
        for row in rows:
            for tok in row.split():
                v = int(tok) if tok.lstrip("-").isdigit() else float(tok)
                assert jl(v) == tok, (f, tok, jl(v))
                n += 1
    assert n > 200


def test_result_lines_have_the_columns_of_each_script():
    from ptstokes.output import result_line
    assert result_line("2d_v", 127, 127, None, 2200, 1, 0.5) == [127, 127, 2200]
    assert result_line("2d_ve", 63, 63, None, 4000, 5, 0.5) == [63, 63, 4000, 5]
    assert len(result_line("2d_ve_perf", 63, 63, None, 101, 1, 0.5)) == 7
    assert result_line("3d_ve", 31, 31, 31, 3400, 5, 1.0) == [31, 31, 31, 3400, 5]
    line = result_line("3d_ve_perf", 31, 31, 31, 201, 1, 0.0314)
    # Stokes3D_ve_perf.jl:229-231: A_eff = 29*n^3*8/1e9, t_it = wtime/(ittot-10), T_eff = A_eff/t_it
    assert line[:5] == [1, 31, 31, 31, 201]
    assert abs(line[6] - 29 * 31 ** 3 * 8 / 1e9) < 1e-15
    assert abs(line[7] - 0.0314 / 191) < 1e-18 and abs(line[8] - line[6] / line[7]) < 1e-9


def test_damped_scripts_lines_and_files():
    """Stokes2D0.jl:168-169 "nx ny iter", Stokes2D_ve0.jl:195-196 "nx ny ittot nt" (the
    columns of the reference's out_Stokes2D_ve0.txt), Stokes3D0_multixpu.jl:242-243
    "nx ny nz iter"; only Stokes2D_ve0.jl writes a MAT file (:199-200)."""
    from ptstokes.output import A_EFF_ARRAYS, LINE_FILES, MAT_FILES, result_line
    assert result_line("2d_v_damp", 511, 511, None, 9000, 1, 0.5) == [511, 511, 9000]
    assert result_line("2d_ve_damp", 31, 31, None, 4000, 5, 0.5) == [31, 31, 4000, 5]
    assert result_line("3d_v_damp", 63, 63, 63, 1500, 1, 0.5) == [63, 63, 63, 1500]
    lines = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_output_lines.json")))
    assert all(len(r.split()) == 4 for r in lines["out_Stokes2D_ve0.txt"])
    assert LINE_FILES["2d_ve_damp"] == "out_Stokes2D_ve0.txt" and LINE_FILES["3d_v_damp"] == "out_Stokes3D0.txt"
    assert set(MAT_FILES) & {"2d_v_damp", "2d_ve_damp", "3d_v_damp"} == {"2d_ve_damp"}
    # A_eff of the scripts: (3*2), (6*2 + 1), (4*2) arrays (Stokes2D0.jl:153, Stokes2D_ve0.jl:178,
    # Stokes3D0_multixpu.jl:222)
    assert (A_EFF_ARRAYS["2d_v_damp"], A_EFF_ARRAYS["2d_ve_damp"], A_EFF_ARRAYS["3d_v_damp"]) == (6, 13, 8)


class _FakeSolver:
    variant, ndim, nx, ny, nz = "3d_ve_perf", 3, 5, 4, 3
    dx, dy, dz = 2.0, 2.5, 10 / 3

    def get(self, name):
        shape = {"Vz": (5, 4, 4), "txz": (4, 2, 2)}.get(name, (5, 4, 3))
        return np.asfortranarray(np.arange(np.prod(shape), dtype=np.float64).reshape(shape, order="F") + len(name))


def test_visu_dump_round_trips(tmp_path):
    from scipy.io import loadmat

    from ptstokes.output import save_line, save_visu
    s = _FakeSolver()
    path = save_visu(s, str(tmp_path))
    m = loadmat(path)
    assert set(k for k in m if not k.startswith("__")) == {"Pt_3D", "Mus_3D", "Txz_3D", "Vz_3D", "dx_3D", "dy_3D",
                                                             "dz_3D"}
    assert np.array_equal(m["Vz_3D"], s.get("Vz")) and float(m["dz_3D"].item()) == s.dz
    p = save_line(s, {"ittot": 201, "iters": [201]}, 0.5, str(tmp_path))
    save_line(s, {"ittot": 201, "iters": [201]}, 0.25, str(tmp_path))
    rows = [r.split() for r in open(p).read().splitlines()]
    assert len(rows) == 2 and all(len(r) == 9 for r in rows) and rows[0][:5] == ["1", "5", "4", "3", "201"]
