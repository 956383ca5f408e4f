"""TEST INFRASTRUCTURE ONLY -- restatement of the reference host's stage sequencing.

``rk_step(integrator, hall, variable_u)`` returns the list of kernel names that one time
step enqueues, as built in matlab/+induction_eq/compute_numerical_solution_setup.m:140-371
(SSPRK33 142-174, SSPRK104 176-271, KennedyCarpenterLewis2R54C 273-294,
CalvoFrancoRandez2R64 296-317, CarpenterKennedy2N54 319-340, ToulorgeDesmet2N84F 342-365).
The ``tmp(:)'`` interleave of the 2R/2N schemes is column-major: for every stage the
curl-B kernel, then the velocity kernel, then the "a" kernel, then the "b" kernel.
"""
from __future__ import annotations

INTEGRATORS = ("SSPRK33", "SSPRK104", "KennedyCarpenterLewis2R54C", "CalvoFrancoRandez2R64",
               "CarpenterKennedy2N54", "ToulorgeDesmet2N84F")

NUM_FIELDS = {"SSPRK33": 3, "SSPRK104": 3, "KennedyCarpenterLewis2R54C": 3,
              "CalvoFrancoRandez2R64": 3, "CarpenterKennedy2N54": 2, "ToulorgeDesmet2N84F": 2}


def _ssp(hall: bool, variable_u: bool, stages) -> list[str]:
    # stages: list of (pre-kernel or None, curl index, stage kernel)
    out: list[str] = []
    for pre, curl_k, kern in stages:
        if pre:
            out.append(pre)
        if hall and curl_k:
            out.append(f"calc_curlB_rho_{curl_k}_3args")
        if variable_u and curl_k:
            out.append("calc_u_3_args")
        out.append(kern)
    out.append("calc_time_3_args")
    return out


def rk_step(integrator: str, hall: bool, variable_u: bool) -> list[str]:
    if integrator == "SSPRK33":
        return _ssp(hall, variable_u, [(None, 1, "SSPRK33_1"), ("SSPRK33_2a", 2, "SSPRK33_2b"),
                                      ("SSPRK33_3a", 3, "SSPRK33_3b")])
    if integrator == "SSPRK104":
        st = [(None, 1, "SSPRK104_01"), ("SSPRK104_02a", 2, "SSPRK104_02b"),
              ("SSPRK104_03a", 3, "SSPRK104_03b"), ("SSPRK104_04a", 2, "SSPRK104_04b"),
              ("SSPRK104_05a", 3, "SSPRK104_05b"), ("SSPRK104_06", 2, "SSPRK104_07"),
              ("SSPRK104_08a", 1, "SSPRK104_08b"), ("SSPRK104_09a", 2, "SSPRK104_09b"),
              ("SSPRK104_10a", 1, "SSPRK104_10b"), ("SSPRK104_11a", 2, "SSPRK104_11b")]
        return _ssp(hall, variable_u, st)
    if integrator == "KennedyCarpenterLewis2R54C":
        p = "KennedyCarpenterLewis2R54C_"
        a = [p + "1a", p + "2a", p + "3a", p + "4a", p + "5"]
        b = [p + "1b", p + "2b", p + "3b", p + "4b", "calc_time_3_args"]
        curl = [1, 1, 2, 1, 2]
        return _interleave(a, b, curl, hall, variable_u, 3)
    if integrator == "CalvoFrancoRandez2R64":
        p = "CalvoFrancoRandez2R64_"
        a = [p + "1a", p + "2a", p + "3a", p + "4a", p + "5a", p + "6"]
        b = [p + "1b", p + "2b", p + "3b", p + "4b", p + "5b", "calc_time_3_args"]
        curl = [1, 2, 2, 2, 2, 2]
        return _interleave(a, b, curl, hall, variable_u, 3)
    if integrator in ("CarpenterKennedy2N54", "ToulorgeDesmet2N84F"):
        ns = 5 if integrator == "CarpenterKennedy2N54" else 8
        a = [f"{integrator}_{i}a" for i in range(1, ns + 1)]
        b = [f"{integrator}_{i}b" for i in range(1, ns + 1)]
        return _interleave(a, b, [1] * ns, hall, variable_u, 2) + ["calc_time_2_args"]
    raise ValueError(f"Unkown time integrator {integrator}!")


def _interleave(a, b, curl, hall, variable_u, nf) -> list[str]:
    out: list[str] = []
    for i in range(len(a)):
        if hall:
            out.append(f"calc_curlB_rho_{curl[i]}_{nf}args")
        if variable_u:
            out.append(f"calc_u_{nf}_args")
        out.append(a[i])
        out.append(b[i])
    return out


def stages_per_step(integrator: str) -> int:
    return {"SSPRK33": 3, "SSPRK104": 10, "KennedyCarpenterLewis2R54C": 5,
            "CalvoFrancoRandez2R64": 6, "CarpenterKennedy2N54": 5, "ToulorgeDesmet2N84F": 8}[integrator]
