/*
 * lbfgsb_oracle.c -- TEST INFRASTRUCTURE: the CPU oracle.
 *
 * A plain-C restatement of the reference's CPU L-BFGS-B path (culbfgsb/lbfgsbcpu.cpp,
 * which the reference selects with LCM_NO_ACCELERATION), used only to check the CUDA
 * library of this repository.  Nothing in the product includes, links or calls it.
 *
 * Parity pin: tests/test_oracle_pin.py runs this restatement and the reference's own
 * lbfgsbcpu.cpp (built from the reference sources into oracle/_ref/ by the Makefile next
 * to this file) on the same seeded problems and requires the same sequence of callback
 * points, bit for bit; tests/golden/ holds fixtures recorded from the reference build.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_api.h"

/* Test switch for the L-BFGS-B 3.0 subspace step (see subsm); off = the reference's 2.1. */
static int g_subsm_projection = 0;
void orc_set_subsm_projection(int on) { g_subsm_projection = on ? 1 : 0; }

/* lbfgsbdefaultoption, culbfgsb/lbfgsb.cpp:43-66 */
void orc_default_option_f64(orc_option_f64* o) {
  o->eps_f = o->eps_g = o->eps_x = 1e-15;
  o->hessian_approximate_dimension = 8;
  o->machine_epsilon = 1e-15;
  o->machine_maximum = DBL_MAX;
  o->max_iteration = 1000;
  o->step_scaling = 1.0;
}

void orc_default_option_f32(orc_option_f32* o) {
  o->eps_f = o->eps_g = o->eps_x = 1e-15f;
  o->hessian_approximate_dimension = 8;
  o->machine_epsilon = 1e-8f;
  o->machine_maximum = FLT_MAX;
  o->max_iteration = 1000;
  o->step_scaling = 1.0f;
}

#define REAL double
#define SFX f64
#define SQRT sqrt
#define FABS fabs
#define OPT_T orc_option_f64
#define SUM_T orc_summary_f64
#define CB_T orc_cb_f64
#include "lbfgsb_oracle_body.h"
#undef REAL
#undef SFX
#undef SQRT
#undef FABS
#undef OPT_T
#undef SUM_T
#undef CB_T

#define REAL float
#define SFX f32
#define SQRT sqrtf
#define FABS fabsf
#define OPT_T orc_option_f32
#define SUM_T orc_summary_f32
#define CB_T orc_cb_f32
#include "lbfgsb_oracle_body.h"
#undef REAL
#undef SFX
#undef SQRT
#undef FABS
#undef OPT_T
#undef SUM_T
#undef CB_T
