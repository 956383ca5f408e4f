"""Build step: generate the typed per-kernel C ABI from the reference's kernel list.

Writes ../../include/inductioneq_kernels.h (declarations, each citing the reference
kernel it replaces) and kernel_abi.inc (definitions that forward to the name-dispatched
launcher).  The names and argument orders are the reference's (kernel/*.cl); every entry
point is prefixed with ``ieq_`` so that names such as ``norm2`` or ``init_b`` cannot clash
with a caller's symbols.

    python gen_kernel_abi.py
"""
from __future__ import annotations

import os

TI3 = ["b1", "b2", "b3", "curlB_rho", "u", "rho", "time"]
TI2 = ["b1", "b2", "curlB_rho", "u", "rho", "time"]
KCL3 = ["b1", "b2", "db", "curlB_rho", "u", "rho", "time"]

# (name, args, reference file:line, g_range kind: "grid" | "pad" | "interior")
KERNELS = [
    ("init_b", ["b"], "kernel/kernel_init.cl:3", "grid"),
    ("init_u", ["u"], "kernel/kernel_init.cl:15", "grid"),
    ("init_rho", ["rho"], "kernel/kernel_init.cl:27", "grid"),
    ("analytical_b", ["b", "time"], "kernel/kernel_init.cl:39", "grid"),
    ("norm2", ["field", "output"], "kernel/kernel_operator.cl:11", "pad"),
    ("norm2_diff", ["field_1", "field_2", "output"], "kernel/kernel_operator.cl:55", "pad"),
    ("norm2_S", ["field", "output"], "kernel/kernel_operator.cl:99", "pad"),
    ("calc_div", ["field", "field_div"], "kernel/kernel_operator.cl:145", "grid"),
    ("calc_curl", ["field", "field_curl"], "kernel/kernel_operator.cl:158", "grid"),
    ("calc_grad", ["field", "field_grad"], "kernel/kernel_operator.cl:170", "grid"),
    ("calc_div_divcleaning", ["field", "field_div"], "kernel/kernel_div_cleaning.cl:60", "interior"),
    ("calc_laplace_divcleaning", ["field", "field_laplace"], "kernel/kernel_div_cleaning.cl:75",
     "interior"),
    ("projector_divcleaning", ["field_b", "field_phi"], "kernel/kernel_div_cleaning.cl:96", "grid"),
    ("calc_axpy", ["x", "y", "a"], "kernel/kernel_CG.cl:8", "interior"),
    ("calc_xpay", ["x", "y", "a"], "kernel/kernel_CG.cl:21", "interior"),
    ("dot_product", ["a_vec", "b_vec", "output"], "kernel/kernel_dot_product.cl:47", "pad"),
    ("calc_time_2_args", TI2, "kernel/kernel_time_integrator.cl:42", "grid"),
    ("calc_time_3_args", TI3, "kernel/kernel_time_integrator.cl:65", "grid"),
    ("calc_u_2_args", TI2, "kernel/kernel_time_integrator.cl:93", "grid"),
    ("calc_u_3_args", TI3, "kernel/kernel_time_integrator.cl:112", "grid"),
    ("calc_curlB_rho_1_2args", TI2, "kernel/kernel_time_integrator.cl:136", "grid"),
    ("calc_curlB_rho_2_2args", TI2, "kernel/kernel_time_integrator.cl:150", "grid"),
    ("calc_curlB_rho_1_3args", TI3, "kernel/kernel_time_integrator.cl:168", "grid"),
    ("calc_curlB_rho_2_3args", TI3, "kernel/kernel_time_integrator.cl:182", "grid"),
    ("calc_curlB_rho_3_3args", TI3, "kernel/kernel_time_integrator.cl:196", "grid"),
    ("SSPRK33_1", TI3, "kernel/kernel_time_integrator.cl:224", "grid"),
    ("SSPRK33_2a", TI3, "kernel/kernel_time_integrator.cl:239", "grid"),
    ("SSPRK33_2b", TI3, "kernel/kernel_time_integrator.cl:256", "grid"),
    ("SSPRK33_3a", TI3, "kernel/kernel_time_integrator.cl:272", "grid"),
    ("SSPRK33_3b", TI3, "kernel/kernel_time_integrator.cl:289", "grid"),
]
LINES = {
    "SSPRK104_01": 315, "SSPRK104_02a": 330, "SSPRK104_02b": 347,
    "SSPRK104_03a": 362, "SSPRK104_03b": 379, "SSPRK104_04a": 394,
    "SSPRK104_04b": 411, "SSPRK104_05a": 426, "SSPRK104_05b": 443,
    "SSPRK104_06": 458, "SSPRK104_07": 479, "SSPRK104_08a": 494,
    "SSPRK104_08b": 511, "SSPRK104_09a": 526, "SSPRK104_09b": 543,
    "SSPRK104_10a": 558, "SSPRK104_10b": 575, "SSPRK104_11a": 590,
    "SSPRK104_11b": 607, "KennedyCarpenterLewis2R54C_1a": 630, "KennedyCarpenterLewis2R54C_1b": 643,
    "KennedyCarpenterLewis2R54C_2a": 668, "KennedyCarpenterLewis2R54C_2b": 681, "KennedyCarpenterLewis2R54C_3a": 706,
    "KennedyCarpenterLewis2R54C_3b": 719, "KennedyCarpenterLewis2R54C_4a": 738, "KennedyCarpenterLewis2R54C_4b": 751,
    "KennedyCarpenterLewis2R54C_5": 776, "CalvoFrancoRandez2R64_1a": 801, "CalvoFrancoRandez2R64_1b": 814,
    "CalvoFrancoRandez2R64_2a": 839, "CalvoFrancoRandez2R64_2b": 852, "CalvoFrancoRandez2R64_3a": 877,
    "CalvoFrancoRandez2R64_3b": 890, "CalvoFrancoRandez2R64_4a": 915, "CalvoFrancoRandez2R64_4b": 928,
    "CalvoFrancoRandez2R64_5a": 953, "CalvoFrancoRandez2R64_5b": 966, "CalvoFrancoRandez2R64_6": 991,
    "CarpenterKennedy2N54_1a": 1023, "CarpenterKennedy2N54_1b": 1036, "CarpenterKennedy2N54_2a": 1059,
    "CarpenterKennedy2N54_2b": 1075, "CarpenterKennedy2N54_3a": 1098, "CarpenterKennedy2N54_3b": 1114,
    "CarpenterKennedy2N54_4a": 1137, "CarpenterKennedy2N54_4b": 1153, "CarpenterKennedy2N54_5a": 1176,
    "CarpenterKennedy2N54_5b": 1192, "ToulorgeDesmet2N84F_1a": 1216, "ToulorgeDesmet2N84F_1b": 1229,
    "ToulorgeDesmet2N84F_2a": 1252, "ToulorgeDesmet2N84F_2b": 1268, "ToulorgeDesmet2N84F_3a": 1291,
    "ToulorgeDesmet2N84F_3b": 1307, "ToulorgeDesmet2N84F_4a": 1330, "ToulorgeDesmet2N84F_4b": 1346,
    "ToulorgeDesmet2N84F_5a": 1369, "ToulorgeDesmet2N84F_5b": 1385, "ToulorgeDesmet2N84F_6a": 1408,
    "ToulorgeDesmet2N84F_6b": 1424, "ToulorgeDesmet2N84F_7a": 1447, "ToulorgeDesmet2N84F_7b": 1463,
    "ToulorgeDesmet2N84F_8a": 1486, "ToulorgeDesmet2N84F_8b": 1502,
}
KERNELS += [(n, KCL3 if n.startswith(("Kennedy", "Calvo")) else
             (TI2 if n.startswith(("Carpenter", "Toulorge")) else TI3),
             f"kernel/kernel_time_integrator.cl:{ln}", "grid") for n, ln in LINES.items()]


def main() -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    hdr = os.path.join(here, "..", "..", "include", "inductioneq_kernels.h")
    inc = os.path.join(here, "kernel_abi.inc")
    h = ["/* inductioneq_kernels.h -- one entry point per reference kernel (generated by",
         " * inductioneq_b200/csrc/gen_kernel_abi.py; do not edit).",
         " *",
         " * Each function runs the reference kernel of the same name (without the ieq_ prefix)",
         " * over its reference NDRange on the context's stream: the node grid, {num_nodes_pad,1,1}",
         " * for reductions, or the CG interior NODES-2*BNODES offset by BNODES.  Arguments are",
         " * device pointers in the reference's order and layout (see inductioneq.h).",
         " * Reductions leave the total in output[0] and zeros in output[1..num_groups-1], so a",
         " * host that sums the per-work-group partials (clean_div.m:41) gets the total.",
         " */",
         "#ifndef INDUCTIONEQ_KERNELS_H", "#define INDUCTIONEQ_KERNELS_H", "",
         "#ifdef __cplusplus", 'extern "C" {', "#endif", ""]

    c = ["// Generated by gen_kernel_abi.py -- do not edit.", ""]
    for name, args, cite, kind in KERNELS:
        params = ", ".join(f"void *{a}" for a in args)
        h.append(f"/* replaces {cite} `{name}` (range: {kind}) */")
        h.append(f"ieq_status ieq_{name}(ieq_ctx *ctx, {params});")
        c.append(f'extern "C" ieq_status ieq_{name}(ieq_ctx *ctx, {params}) {{')
        c.append(f"  void *argv_[{len(args)}] = {{{', '.join(args)}}};")
        c.append(f'  return ieq_run_one_default(ctx, "{name}", argv_, {len(args)});')
        c.append("}")
    h += ["", "#ifdef __cplusplus", "}", "#endif", "#endif /* INDUCTIONEQ_KERNELS_H */", ""]
    with open(hdr, "w") as f:
        f.write("\n".join(h))
    with open(inc, "w") as f:
        f.write("\n".join(c) + "\n")
    print(len(KERNELS), "kernels")


if __name__ == "__main__":
    main()
