/*
 * dirac.h -- Wilson hopping matrix entry points (plqcd-b200).
 *
 * The reference's include/dirac.h:19-33 entry points on host arrays in the
 * API layout of su3.h, all computed by the sm_100a CUDA kernels:
 *
 *   eo: qout[0, V/2)   = H_eo qin[V/2, V)   (odd input -> even output)
 *   oe: qout[V/2, V)   = H_oe qin[0, V/2)   (even input -> odd output)
 *
 *   (H psi)(x) = sum_mu U_mu(x) (1 - g_mu) psi(x+mu)
 *              + U_mu(x-mu)^dag (1 + g_mu) psi(x-mu)
 *
 * with periodic boundaries, no kappa, the reference's gamma basis and even/odd
 * site order, links u[4*i+mu] = U_mu(x_i) (lib/dirac.c:35-791). Only the
 * output half of qout is written. The return value is the call's wall-clock
 * time in seconds (lib/dirac.c:405-407), host<->device copies included, or a
 * negative value on failure (message in plqcd_last_error()).
 *
 * Results follow the correct operator. The reference as shipped differs in
 * spin components s2/s3 (include/su3.h:135-138 used at lib/dirac.c:373-374,
 * 756-757) and in the oe forward links (lib/dirac.c:643); setting the
 * environment variable PLQCD_REF_COMPAT=1 before init_plqcd reproduces that
 * behaviour exactly.
 *
 * The SSE3-intrinsic names (lib/dirac.c:801, 1272, 1748, 2124) take the same
 * arguments and map to the same correct kernel. Like the reference, every
 * call reads the link array `u`: it is uploaded to the GPU on each call.
 * A caller whose links stay fixed over many calls registers the array once
 * with plqcd_gauge_update(u) (plqcd_b200.h); it is then uploaded once and
 * kept on the device until the next plqcd_gauge_update or finalize_plqcd.
 * After changing registered links in place, call plqcd_gauge_update(u)
 * again.
 */
#ifndef _DIRAC_H
#define _DIRAC_H

#include "plqcd_global_params.h"
#include "start.h"
#include "su3_256.h"
#include "su3_512.h"
#include "utils.h"

#ifdef __cplusplus
extern "C" {
#endif

struct plqcd_timer {
    double total;
    double computation;
};

double plqcd_hopping_matrix_eo_sse3_assymbly(spinor *qin, spinor *qout, su3 *u);
double plqcd_hopping_matrix_oe_sse3_assymbly(spinor *qin, spinor *qout, su3 *u);

double plqcd_hopping_matrix_eo_sse3_intrin(spinor *qin, spinor *qout, su3 *u);
double plqcd_hopping_matrix_oe_sse3_intrin(spinor *qin, spinor *qout, su3 *u);
double plqcd_hopping_matrix_eo_sse3_intrin_blocking(spinor *qin, spinor *qout, su3 *u);
double plqcd_hopping_matrix_oe_sse3_intrin_blocking(spinor *qin, spinor *qout, su3 *u);

/*
 * Split real/imaginary layout (reference include/dirac.h:31-32, 39-40,
 * 55-62; note the argument order, output first). The reference packs 2/4/8
 * x-sites per SIMD lane with its own site tables and gamma convention; here
 * the split layout is the API arrays with real and imaginary parts in
 * separate planes, in even/odd site order, whatever the SIMD width:
 *   qin_re[12*i + 3*spin + colour], u_re[9*(4*i + mu) + 3*row + col]
 * and every name computes the same operator as the AoS entry points above.
 * The *_short names read link rows 0,1 only and rebuild row 2 as
 * conj(row0 x row1), which is exact for SU(3) links.
 */
double plqcd_hopping_matrix_eo_sse3_intrin_nohalfspinor(double *qout_re, double *qout_im, double *u_re,
                                                        double *u_im, double *qin_re, double *qin_im);
double plqcd_hopping_matrix_oe_sse3_intrin_nohalfspinor(double *qout_re, double *qout_im, double *u_re,
                                                        double *u_im, double *qin_re, double *qin_im);
double plqcd_hopping_matrix_eo_avx_nohalfspinor(double *qout_re, double *qout_im, double *u_re, double *u_im,
                                                double *qin_re, double *qin_im);
double plqcd_hopping_matrix_oe_avx_nohalfspinor(double *qout_re, double *qout_im, double *u_re, double *u_im,
                                                double *qin_re, double *qin_im);
double plqcd_hopping_matrix_eo_single_mic_split(double *qout_re, double *qout_im, double *u_re, double *u_im,
                                                double *qin_re, double *qin_im);
double plqcd_hopping_matrix_oe_single_mic_split(double *qout_re, double *qout_im, double *u_re, double *u_im,
                                                double *qin_re, double *qin_im);
double plqcd_hopping_matrix_eo_single_mic_split_nohalfspinor(double *qout_re, double *qout_im, double *u_re,
                                                             double *u_im, double *qin_re, double *qin_im);
double plqcd_hopping_matrix_oe_single_mic_split_nohalfspinor(double *qout_re, double *qout_im, double *u_re,
                                                             double *u_im, double *qin_re, double *qin_im);
double plqcd_hopping_matrix_eo_single_mic_split_nohalfspinor_short(double *qout_re, double *qout_im, double *u_re,
                                                                   double *u_im, double *qin_re, double *qin_im);
double plqcd_hopping_matrix_oe_single_mic_split_nohalfspinor_short(double *qout_re, double *qout_im, double *u_re,
                                                                   double *u_im, double *qin_re, double *qin_im);

/*
 * Lane-packed names (reference include/dirac.h:37-38, 46-51): arrays of
 * spinor_256 / su3_256 (two consecutive even/odd sites per object) or
 * spinor_512 / su3_512 (four), as built by the copy_*_to_*_256/512
 * converters (include/su3_256.h, su3_512.h); eo writes the packed objects
 * of the even half of qout from the odd half of qin, oe the reverse, and
 * every name computes the same operator as the AoS entry points. The
 * *_short name reads link rows 0,1 only and rebuilds row 2 as
 * conj(row0 x row1). Links are cached like the AoS ones.
 */
double plqcd_hopping_matrix_eo_intrin_256(spinor_256 *qin, spinor_256 *qout, su3_256 *u);
double plqcd_hopping_matrix_oe_intrin_256(spinor_256 *qin, spinor_256 *qout, su3_256 *u);
double plqcd_hopping_matrix_eo_intrin_512(spinor_512 *qin, spinor_512 *qout, su3_512 *u);
double plqcd_hopping_matrix_oe_intrin_512(spinor_512 *qin, spinor_512 *qout, su3_512 *u);
double plqcd_hopping_matrix_eo_single_mic(spinor_512 *qin, spinor_512 *qout, su3_512 *u);
double plqcd_hopping_matrix_oe_single_mic(spinor_512 *qin, spinor_512 *qout, su3_512 *u);
double plqcd_hopping_matrix_eo_single_mic_short(spinor_512 *qin, spinor_512 *qout, su3_512 *u);
double plqcd_hopping_matrix_oe_single_mic_short(spinor_512 *qin, spinor_512 *qout, su3_512 *u);

#ifdef __cplusplus
}
#endif
#endif
