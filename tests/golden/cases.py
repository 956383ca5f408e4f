"""Small parity cases shared by the golden-vector generator and the tests.

Each case names the reference's discrete switches (operator, testcase, BC, Hall,
dissipation, flux forms, integrator, REAL) plus a small mesh.  Grids are ragged
(NX != NY != NZ) so that index-order mistakes cannot cancel, and wide enough for the
widest boundary closure (2*NUM_BOUNDS nodes per direction).
"""
from __future__ import annotations

import math

TWO_PI = 2.0 * math.pi
HP = 4.0 * math.pi / 3.0      # period of include/hall_periodic.h (k = 1.5)

# name -> settings.  dt: explicit time step.  steps: RK steps run for the fixture.
STEP_CASES = {
    "rot_gauss_4c_ssprk33": dict(order=4, testcase="rotation_gaussian", nodes=(12, 13, 14),
                                 lo=-1.0, hi=1.0, integrator="SSPRK33", dt=0.02, steps=2),
    "rot3d_2c_ck2n54": dict(order=2, testcase="rotation_3D", nodes=(9, 10, 11), lo=-1.0, hi=1.0,
                            integrator="CarpenterKennedy2N54", dt=0.03, steps=2),
    "wave_6c_hall_hod_ck2n54": dict(order=6, testcase="hall_circular_wave", nodes=(12, 12, 14),
                                    lo=0.0, hi=TWO_PI, periodic=True, hall=True,
                                    dissipation="HIGH_ORDER", integrator="CarpenterKennedy2N54",
                                    dt=0.02, steps=2),
    "rot3d_4e_split_kcl": dict(order=4, extended=True, testcase="rotation_3D", nodes=(13, 14, 15),
                               lo=-1.0, hi=1.0, uibj="SPLIT", source="SPLIT", ujbi="SPLIT",
                               integrator="KennedyCarpenterLewis2R54C", dt=0.02, steps=2),
    "confined_6e_hall_fo_cfr": dict(order=6, extended=True, testcase="confined_domain",
                                    nodes=(17, 18, 19), lo=0.0, hi=1.0, hall=True,
                                    dissipation="FIRST_ORDER", integrator="CalvoFrancoRandez2R64",
                                    dt=2e-4, steps=1),
    "alfven_2e_adaptive_td": dict(order=2, extended=True, testcase="alfven_periodic_2D",
                                  nodes=(10, 11, 9), lo=0.0, hi=1.0, periodic=True,
                                  dissipation="ADAPTIVE", uibj="CENTRAL", source="ZERO",
                                  ujbi="PRODUCT", integrator="ToulorgeDesmet2N84F", dt=0.01,
                                  steps=2, variable_u=True),
    "hallper_4c_ssprk104_varu": dict(order=4, testcase="hall_periodic", nodes=(10, 12, 11), lo=0.0,
                                     hi=HP, periodic=True, hall=True, integrator="SSPRK104",
                                     dt=0.01, steps=1, variable_u=True),
    "travel_6c_hall_sat_ssprk33": dict(order=6, testcase="hall_travelling_wave", nodes=(13, 12, 16),
                                       lo=0.0, hi=TWO_PI, hall=True, integrator="SSPRK33",
                                       dt=1e-3, steps=2, variable_u=True),
    "rot_gauss_4c_ssprk33_f32": dict(order=4, testcase="rotation_gaussian", nodes=(12, 13, 14),
                                     lo=-1.0, hi=1.0, integrator="SSPRK33", dt=0.02, steps=2,
                                     real="float"),
}

# divergence cleaning (clean_div.m): confined_domain field + seeded noise, per Laplacian
CG_CASES = {
    "cg_4c_wsd0": dict(order=4, testcase="confined_domain", nodes=(14, 15, 16), lo=0.0, hi=1.0,
                       laplace="WIDE_STENCIL_DIRICHLET", bnodes=1, max_iterations=40, thr=1e-9),
    "cg_4c_nsd0": dict(order=4, testcase="confined_domain", nodes=(14, 15, 16), lo=0.0, hi=1.0,
                       laplace="NARROW_STENCIL_DIRICHLET", bnodes=1, max_iterations=40, thr=1e-9),
    "cg_2c_wsln": dict(order=2, testcase="confined_domain", nodes=(11, 12, 13), lo=0.0, hi=1.0,
                       laplace="WIDE_STENCIL_LNS", bnodes=0, max_iterations=25, thr=1e-9),
    "cg_6c_wsd0": dict(order=6, testcase="confined_domain", nodes=(20, 21, 22), lo=0.0, hi=1.0,
                       laplace="WIDE_STENCIL_DIRICHLET", bnodes=1, max_iterations=30, thr=1e-9),
}

NOISE_SEED = 12345
NOISE_AMPLITUDE = 1e-3


def mesh_args(c: dict) -> dict:
    lo, hi = c["lo"], c["hi"]
    return dict(nodes=tuple(c["nodes"]), xmin=(lo, lo, lo), xmax=(hi, hi, hi),
                periodic=c.get("periodic", False))


def variant_kwargs(c: dict) -> dict:
    keys = ("order", "extended", "testcase", "periodic", "hall", "dissipation", "uibj", "source",
            "ujbi", "laplace", "real")
    return {k: c[k] for k in keys if k in c}
