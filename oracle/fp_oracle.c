/* ORACLE TEST INFRASTRUCTURE — never part of the product path.
 * Instantiates the C restatement (fp_oracle_impl.h) in single and double precision. */
#include "fp_oracle.h"

#include <float.h>
#include <math.h>
#include <stddef.h>
#include <string.h>

#define R float
#define SFX _f32
#define R_FLOOR floorf
#define R_ROUND roundf
#define R_SIN sinf
#define R_COS cosf
#define R_FABS fabsf
#define R_SQRT sqrtf
#define R_EPS FLT_EPSILON
#define R_MAT33_STRIDE 12
#include "fp_oracle_impl.h"
#undef R
#undef SFX
#undef R_FLOOR
#undef R_ROUND
#undef R_SIN
#undef R_COS
#undef R_FABS
#undef R_SQRT
#undef R_EPS
#undef R_MAT33_STRIDE

#define R double
#define SFX _f64
#define R_FLOOR floor
#define R_ROUND round
#define R_SIN sin
#define R_COS cos
#define R_FABS fabs
#define R_SQRT sqrt
#define R_EPS DBL_EPSILON
#define R_MAT33_STRIDE 10
#include "fp_oracle_impl.h"
