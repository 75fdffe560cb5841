/*
 * FP64 re-solve build of oracle_contact.c -- TEST INFRASTRUCTURE ONLY (see that file's header).
 *
 * The same source compiled once more with every float32 quantity, literal and builtin in
 * float64: this header is force-included (-include) before the source, and the Makefile
 * strips the `f` suffix of the numeric literals on the way in.  The system headers are
 * included here first, so the type and function renames below reach only the oracle's code.
 * The result is the oracle's algorithm -- the same steps, orders and branches -- in double
 * precision: the reference against which the float32 kernels' tolerances are stated.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define float double
#define fmaf fma
#define sqrtf sqrt
#define fabsf fabs
#define fmaxf fmax
#define floorf floor
