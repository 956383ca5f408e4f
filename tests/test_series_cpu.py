"""Time-series output of a run (the paper scripts' HDF5 datasets, written as .npz): file names
of paper/divcleaning_confined_domain.m:162-177, the datasets of :183-190 and the summary line of
:192-199."""
from __future__ import annotations

import re

import numpy as np

from inductioneq_b200.induction_eq import Maps, read_series, series_filename, summary_row, write_series


def _maps(clean=False, form="USE_LAPLACE_WIDE_STENCIL_DIRICHLET"):
    m = Maps()
    m.I_Mesh.update({"NODES_X": 40, "NODES_Y": 40, "NODES_Z": 40})
    m.I_RunOps.update({"order": 6, "testcase": "confined_domain"})
    m.I_IEq.update({"form_uibj": "USE_UIBJ_SPLIT", "form_source": "USE_SOURCE_ZERO", "form_ujbi": "USE_UJBI_PRODUCT"})
    m.I_DC.update({"divergence_cleaning": clean, "divergence_cleaning_form": form})
    return m


def test_file_names_follow_the_paper_scripts():
    assert series_filename(_maps()) == "confined_domain_N_40_order_6_split_zero_product__DC_0.npz"
    for form, label in (("USE_LAPLACE_WIDE_STENCIL_LNS", "WS_LN"), ("USE_LAPLACE_WIDE_STENCIL_DIRICHLET", "WS_D0"),
                        ("USE_LAPLACE_NARROW_STENCIL_DIRICHLET", "NS_D0")):
        assert series_filename(_maps(True, form)) == f"confined_domain_N_40_order_6_split_zero_product__DC_1_{label}.npz"


def test_series_round_trip(tmp_path):
    n = 7
    res = {"time": np.linspace(0.0, 0.3, n + 1), "energy_over_time": np.arange(n + 1) * 1.5,
           "L2error_B_over_time": np.full(n + 1, 1e-7), "L2error_divB_over_time": np.geomspace(1.0, 1e-9, n + 1)}
    path = tmp_path / "run.npz"
    write_series(str(path), res)
    write_series(str(path), res)   # replaces an existing file
    got = read_series(str(path))
    assert sorted(got) == ["L2error_B", "L2error_divB", "energy", "time"]
    np.testing.assert_array_equal(got["time"], res["time"])
    np.testing.assert_array_equal(got["energy"], res["energy_over_time"])
    np.testing.assert_array_equal(got["L2error_B"], res["L2error_B_over_time"])
    np.testing.assert_array_equal(got["L2error_divB"], res["L2error_divB_over_time"])
    assert all(v.dtype == np.float64 for v in got.values())


def test_summary_line_has_the_paper_scripts_format():
    res = {"runtime": 1.25, "energy": 3.0, "abs_err": 1e-6, "divergence_norm": 2.5e-11}
    line = summary_row(_maps(True), res)
    assert line == ("40, 6, USE_UIBJ_SPLIT, USE_SOURCE_ZERO, USE_UJBI_PRODUCT, 1.250000000000000e+00, "
                    "3.000000000000000e+00, 1.000000000000000e-06, 2.500000000000000e-11, 1, "
                    "USE_LAPLACE_WIDE_STENCIL_DIRICHLET \n")
    off = summary_row(_maps(False), res)
    assert re.fullmatch(r"40, 6, \S+, \S+, \S+(, [-+0-9.e]+){4}, 0,   \n", off)
