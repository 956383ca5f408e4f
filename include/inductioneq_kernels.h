/* inductioneq_kernels.h -- one entry point per reference kernel (generated by
 * inductioneq_b200/csrc/gen_kernel_abi.py; do not edit).
 *
 * Each function runs the reference kernel of the same name (without the ieq_ prefix)
 * over its reference NDRange on the context's stream: the node grid, {num_nodes_pad,1,1}
 * for reductions, or the CG interior NODES-2*BNODES offset by BNODES.  Arguments are
 * device pointers in the reference's order and layout (see inductioneq.h).
 * Reductions leave the total in output[0] and zeros in output[1..num_groups-1], so a
 * host that sums the per-work-group partials (clean_div.m:41) gets the total.
 */
#ifndef INDUCTIONEQ_KERNELS_H
#define INDUCTIONEQ_KERNELS_H

#ifdef __cplusplus
extern "C" {
#endif

/* replaces kernel/kernel_init.cl:3 `init_b` (range: grid) */
ieq_status ieq_init_b(ieq_ctx *ctx, void *b);
/* replaces kernel/kernel_init.cl:15 `init_u` (range: grid) */
ieq_status ieq_init_u(ieq_ctx *ctx, void *u);
/* replaces kernel/kernel_init.cl:27 `init_rho` (range: grid) */
ieq_status ieq_init_rho(ieq_ctx *ctx, void *rho);
/* replaces kernel/kernel_init.cl:39 `analytical_b` (range: grid) */
ieq_status ieq_analytical_b(ieq_ctx *ctx, void *b, void *time);
/* replaces kernel/kernel_operator.cl:11 `norm2` (range: pad) */
ieq_status ieq_norm2(ieq_ctx *ctx, void *field, void *output);
/* replaces kernel/kernel_operator.cl:55 `norm2_diff` (range: pad) */
ieq_status ieq_norm2_diff(ieq_ctx *ctx, void *field_1, void *field_2, void *output);
/* replaces kernel/kernel_operator.cl:99 `norm2_S` (range: pad) */
ieq_status ieq_norm2_S(ieq_ctx *ctx, void *field, void *output);
/* replaces kernel/kernel_operator.cl:145 `calc_div` (range: grid) */
ieq_status ieq_calc_div(ieq_ctx *ctx, void *field, void *field_div);
/* replaces kernel/kernel_operator.cl:158 `calc_curl` (range: grid) */
ieq_status ieq_calc_curl(ieq_ctx *ctx, void *field, void *field_curl);
/* replaces kernel/kernel_operator.cl:170 `calc_grad` (range: grid) */
ieq_status ieq_calc_grad(ieq_ctx *ctx, void *field, void *field_grad);
/* replaces kernel/kernel_div_cleaning.cl:60 `calc_div_divcleaning` (range: interior) */
ieq_status ieq_calc_div_divcleaning(ieq_ctx *ctx, void *field, void *field_div);
/* replaces kernel/kernel_div_cleaning.cl:75 `calc_laplace_divcleaning` (range: interior) */
ieq_status ieq_calc_laplace_divcleaning(ieq_ctx *ctx, void *field, void *field_laplace);
/* replaces kernel/kernel_div_cleaning.cl:96 `projector_divcleaning` (range: grid) */
ieq_status ieq_projector_divcleaning(ieq_ctx *ctx, void *field_b, void *field_phi);
/* replaces kernel/kernel_CG.cl:8 `calc_axpy` (range: interior) */
ieq_status ieq_calc_axpy(ieq_ctx *ctx, void *x, void *y, void *a);
/* replaces kernel/kernel_CG.cl:21 `calc_xpay` (range: interior) */
ieq_status ieq_calc_xpay(ieq_ctx *ctx, void *x, void *y, void *a);
/* replaces kernel/kernel_dot_product.cl:47 `dot_product` (range: pad) */
ieq_status ieq_dot_product(ieq_ctx *ctx, void *a_vec, void *b_vec, void *output);
/* replaces kernel/kernel_time_integrator.cl:42 `calc_time_2_args` (range: grid) */
ieq_status ieq_calc_time_2_args(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:65 `calc_time_3_args` (range: grid) */
ieq_status ieq_calc_time_3_args(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:93 `calc_u_2_args` (range: grid) */
ieq_status ieq_calc_u_2_args(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:112 `calc_u_3_args` (range: grid) */
ieq_status ieq_calc_u_3_args(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:136 `calc_curlB_rho_1_2args` (range: grid) */
ieq_status ieq_calc_curlB_rho_1_2args(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:150 `calc_curlB_rho_2_2args` (range: grid) */
ieq_status ieq_calc_curlB_rho_2_2args(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:168 `calc_curlB_rho_1_3args` (range: grid) */
ieq_status ieq_calc_curlB_rho_1_3args(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:182 `calc_curlB_rho_2_3args` (range: grid) */
ieq_status ieq_calc_curlB_rho_2_3args(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:196 `calc_curlB_rho_3_3args` (range: grid) */
ieq_status ieq_calc_curlB_rho_3_3args(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:224 `SSPRK33_1` (range: grid) */
ieq_status ieq_SSPRK33_1(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:239 `SSPRK33_2a` (range: grid) */
ieq_status ieq_SSPRK33_2a(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:256 `SSPRK33_2b` (range: grid) */
ieq_status ieq_SSPRK33_2b(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:272 `SSPRK33_3a` (range: grid) */
ieq_status ieq_SSPRK33_3a(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:289 `SSPRK33_3b` (range: grid) */
ieq_status ieq_SSPRK33_3b(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:315 `SSPRK104_01` (range: grid) */
ieq_status ieq_SSPRK104_01(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:330 `SSPRK104_02a` (range: grid) */
ieq_status ieq_SSPRK104_02a(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:347 `SSPRK104_02b` (range: grid) */
ieq_status ieq_SSPRK104_02b(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:362 `SSPRK104_03a` (range: grid) */
ieq_status ieq_SSPRK104_03a(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:379 `SSPRK104_03b` (range: grid) */
ieq_status ieq_SSPRK104_03b(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:394 `SSPRK104_04a` (range: grid) */
ieq_status ieq_SSPRK104_04a(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:411 `SSPRK104_04b` (range: grid) */
ieq_status ieq_SSPRK104_04b(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:426 `SSPRK104_05a` (range: grid) */
ieq_status ieq_SSPRK104_05a(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:443 `SSPRK104_05b` (range: grid) */
ieq_status ieq_SSPRK104_05b(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:458 `SSPRK104_06` (range: grid) */
ieq_status ieq_SSPRK104_06(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:479 `SSPRK104_07` (range: grid) */
ieq_status ieq_SSPRK104_07(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:494 `SSPRK104_08a` (range: grid) */
ieq_status ieq_SSPRK104_08a(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:511 `SSPRK104_08b` (range: grid) */
ieq_status ieq_SSPRK104_08b(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:526 `SSPRK104_09a` (range: grid) */
ieq_status ieq_SSPRK104_09a(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:543 `SSPRK104_09b` (range: grid) */
ieq_status ieq_SSPRK104_09b(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:558 `SSPRK104_10a` (range: grid) */
ieq_status ieq_SSPRK104_10a(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:575 `SSPRK104_10b` (range: grid) */
ieq_status ieq_SSPRK104_10b(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:590 `SSPRK104_11a` (range: grid) */
ieq_status ieq_SSPRK104_11a(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:607 `SSPRK104_11b` (range: grid) */
ieq_status ieq_SSPRK104_11b(ieq_ctx *ctx, void *b1, void *b2, void *b3, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:630 `KennedyCarpenterLewis2R54C_1a` (range: grid) */
ieq_status ieq_KennedyCarpenterLewis2R54C_1a(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:643 `KennedyCarpenterLewis2R54C_1b` (range: grid) */
ieq_status ieq_KennedyCarpenterLewis2R54C_1b(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:668 `KennedyCarpenterLewis2R54C_2a` (range: grid) */
ieq_status ieq_KennedyCarpenterLewis2R54C_2a(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:681 `KennedyCarpenterLewis2R54C_2b` (range: grid) */
ieq_status ieq_KennedyCarpenterLewis2R54C_2b(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:706 `KennedyCarpenterLewis2R54C_3a` (range: grid) */
ieq_status ieq_KennedyCarpenterLewis2R54C_3a(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:719 `KennedyCarpenterLewis2R54C_3b` (range: grid) */
ieq_status ieq_KennedyCarpenterLewis2R54C_3b(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:738 `KennedyCarpenterLewis2R54C_4a` (range: grid) */
ieq_status ieq_KennedyCarpenterLewis2R54C_4a(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:751 `KennedyCarpenterLewis2R54C_4b` (range: grid) */
ieq_status ieq_KennedyCarpenterLewis2R54C_4b(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:776 `KennedyCarpenterLewis2R54C_5` (range: grid) */
ieq_status ieq_KennedyCarpenterLewis2R54C_5(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:801 `CalvoFrancoRandez2R64_1a` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_1a(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:814 `CalvoFrancoRandez2R64_1b` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_1b(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:839 `CalvoFrancoRandez2R64_2a` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_2a(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:852 `CalvoFrancoRandez2R64_2b` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_2b(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:877 `CalvoFrancoRandez2R64_3a` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_3a(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:890 `CalvoFrancoRandez2R64_3b` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_3b(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:915 `CalvoFrancoRandez2R64_4a` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_4a(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:928 `CalvoFrancoRandez2R64_4b` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_4b(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:953 `CalvoFrancoRandez2R64_5a` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_5a(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:966 `CalvoFrancoRandez2R64_5b` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_5b(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:991 `CalvoFrancoRandez2R64_6` (range: grid) */
ieq_status ieq_CalvoFrancoRandez2R64_6(ieq_ctx *ctx, void *b1, void *b2, void *db, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1023 `CarpenterKennedy2N54_1a` (range: grid) */
ieq_status ieq_CarpenterKennedy2N54_1a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1036 `CarpenterKennedy2N54_1b` (range: grid) */
ieq_status ieq_CarpenterKennedy2N54_1b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1059 `CarpenterKennedy2N54_2a` (range: grid) */
ieq_status ieq_CarpenterKennedy2N54_2a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1075 `CarpenterKennedy2N54_2b` (range: grid) */
ieq_status ieq_CarpenterKennedy2N54_2b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1098 `CarpenterKennedy2N54_3a` (range: grid) */
ieq_status ieq_CarpenterKennedy2N54_3a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1114 `CarpenterKennedy2N54_3b` (range: grid) */
ieq_status ieq_CarpenterKennedy2N54_3b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1137 `CarpenterKennedy2N54_4a` (range: grid) */
ieq_status ieq_CarpenterKennedy2N54_4a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1153 `CarpenterKennedy2N54_4b` (range: grid) */
ieq_status ieq_CarpenterKennedy2N54_4b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1176 `CarpenterKennedy2N54_5a` (range: grid) */
ieq_status ieq_CarpenterKennedy2N54_5a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1192 `CarpenterKennedy2N54_5b` (range: grid) */
ieq_status ieq_CarpenterKennedy2N54_5b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1216 `ToulorgeDesmet2N84F_1a` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_1a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1229 `ToulorgeDesmet2N84F_1b` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_1b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1252 `ToulorgeDesmet2N84F_2a` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_2a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1268 `ToulorgeDesmet2N84F_2b` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_2b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1291 `ToulorgeDesmet2N84F_3a` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_3a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1307 `ToulorgeDesmet2N84F_3b` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_3b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1330 `ToulorgeDesmet2N84F_4a` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_4a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1346 `ToulorgeDesmet2N84F_4b` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_4b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1369 `ToulorgeDesmet2N84F_5a` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_5a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1385 `ToulorgeDesmet2N84F_5b` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_5b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1408 `ToulorgeDesmet2N84F_6a` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_6a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1424 `ToulorgeDesmet2N84F_6b` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_6b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1447 `ToulorgeDesmet2N84F_7a` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_7a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1463 `ToulorgeDesmet2N84F_7b` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_7b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1486 `ToulorgeDesmet2N84F_8a` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_8a(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);
/* replaces kernel/kernel_time_integrator.cl:1502 `ToulorgeDesmet2N84F_8b` (range: grid) */
ieq_status ieq_ToulorgeDesmet2N84F_8b(ieq_ctx *ctx, void *b1, void *b2, void *curlB_rho, void *u, void *rho, void *time);

#ifdef __cplusplus
}
#endif
#endif /* INDUCTIONEQ_KERNELS_H */
