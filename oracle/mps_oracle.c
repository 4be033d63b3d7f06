/* mps_oracle.c -- TEST INFRASTRUCTURE ONLY (see mps_oracle.h).
 * CPU restatement of the reference MPS step; instantiated in float and double.
 * Built by oracle/Makefile into oracle/liboracle.so, loaded by tests/ and by
 * bench.py's CPU-baseline leg, never by the product library. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mps_oracle.h"

#define R float
#define SFX f32
#include "mps_oracle_impl.inc"
#undef R
#undef SFX

#define R double
#define SFX f64
#include "mps_oracle_impl.inc"
#undef R
#undef SFX
