/* Oracle: the FP64 variant of the polarized transport and adjoint
 * restatement (test infrastructure; see kp_oracle.h).
 *
 * This is kp_oracle.c compiled with every float quantity computed in double:
 * Stokes vectors and frames, weights, optical depths, phase matrices,
 * peel-off attenuations and adjoint scores, with 1/(4 pi) and 3/(16 pi) as
 * double constants.  The random draws are the same (om_u01 values are
 * exact in either type) and the geometry was double already, so a packet
 * takes the float restatement's path except where a decision falls within
 * float rounding of its threshold.  Its adjoint is the FP64 CPU adjoint the
 * GPU's gradients are checked against (tests/test_adjoint_fp64.py).
 *
 * The exported functions carry a _f64 suffix and live in their own library
 * (_ref/libkporacle64.so); their per-cell and per-pixel float arrays
 * (sigma2, adj_img) become double arrays.  The structs of kp_oracle.h keep
 * their layout: the header is read before float is redefined.
 */
#include "kp_oracle.h"

#define float double
#define sqrtf sqrt
#define floorf floor
#define fabsf fabs
#define OM_INV4PI 0.079577471545947673     /* 1 / (4 pi)  */
#define OM_3_16PI 0.059683103659460755     /* 3 / (16 pi) */

#define kpo_trace          kpo_trace_f64
#define kpo_trace_ex       kpo_trace_ex_f64
#define kpo_transport      kpo_transport_f64
#define kpo_philox         kpo_philox_f64
#define kpo_log_exp        kpo_log_exp_f64
#define kpo_scatter_sample kpo_scatter_sample_f64
#define kpo_set_abs_sink   kpo_set_abs_sink_f64
#define kpo_set_pixel_sink kpo_set_pixel_sink_f64
#define kpo_adjoint        kpo_adjoint_f64

/* kpo_trace calls kpo_trace_ex before defining it */
int kpo_trace_ex( const kpo_mesh_t * m, int precision, long n, double * x,
                  const double * dir, int * cell, int * ib, const double * proper,
                  int * step, int * todo, int fx_shift, double * flux_f,
                  long long * flux_fx, int * fix_shifts );

#include "kp_oracle.c"
