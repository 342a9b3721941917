/* ffe_oracle.c -- instantiates the oracle restatement (ffe_oracle_impl.h) in
 * float and double.  Test infrastructure only; see ffe_oracle.h. */
#define _GNU_SOURCE
#include "ffe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* TINY of the reference (src/data/typedefs.h:6-12) */
#define REAL float
#define SFX _f32
#define TINYR ((float)(1e-7))
#define TANHR tanhf
#include "ffe_oracle_impl.h"
#undef REAL
#undef SFX
#undef TINYR
#undef TANHR

#define REAL double
#define SFX _f64
#define TINYR 1e-11
#define TANHR tanh
#include "ffe_oracle_impl.h"
#undef REAL
#undef SFX
#undef TINYR
#undef TANHR
