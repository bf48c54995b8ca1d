/*
 * qsv_oracle.c -- CPU oracle of the QCLAB++ state-vector apply path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this library, and only as the checker.
 * The product (qclab_b200/libqclab_b200.so) never links or calls it.
 *
 * A plain-C restatement of src/qgates/apply.hpp (lambdas :9-223, index
 * loops :227-371) and of each gate class's apply override
 * (src/qgates/*.cpp), driven by the same qsv_gate records as the library.
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off).
 *
 * Pinned against the reference itself: oracle/_ref/libqclab_ref.so is the
 * reference compiled from its own sources (oracle/Makefile), and
 * tests/golden/ holds fixtures generated by running it
 * (tests/golden/make_golden.py); tests/test_oracle.py checks this oracle
 * against both, bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "qclab_b200.h"

#define ORACLE_EINVAL 1
#define ORACLE_EQUBIT 2
#define ORACLE_EDTYPE 6

#define R double
#define SFX _z
#define IS_CPLX 1
#define SQRT sqrt
#include "oracle_impl.h"
#undef R
#undef SFX
#undef IS_CPLX
#undef SQRT

#define R float
#define SFX _c
#define IS_CPLX 1
#define SQRT sqrtf
#include "oracle_impl.h"
#undef R
#undef SFX
#undef IS_CPLX
#undef SQRT

#define R double
#define SFX _d
#define IS_CPLX 0
#define SQRT sqrt
#include "oracle_impl.h"
#undef R
#undef SFX
#undef IS_CPLX
#undef SQRT

#define R float
#define SFX _s
#define IS_CPLX 0
#define SQRT sqrtf
#include "oracle_impl.h"
#undef R
#undef SFX
#undef IS_CPLX
#undef SQRT

/* Applies `count` gate records with `op` and qubit `offset` to an n-qubit
 * state of element type `dtype` (a qsv_dtype) in host memory, in place.
 * Returns 0, or 1 (invalid record/op), 2 (qubit range), 6 (dtype). */
int oracle_apply(int n, int dtype, void* state, const qsv_gate* gates, size_t count,
                 char op, int offset) {
  if (n < 1 || n > 34 || !state) return ORACLE_EINVAL;
  switch (dtype) {
    case QSV_C128: return apply_list_z(n, (elem_t_z*)state, gates, count, op, offset);
    case QSV_C64:  return apply_list_c(n, (elem_t_c*)state, gates, count, op, offset);
    case QSV_F64:  return apply_list_d(n, (elem_t_d*)state, gates, count, op, offset);
    case QSV_F32:  return apply_list_s(n, (elem_t_s*)state, gates, count, op, offset);
  }
  return ORACLE_EINVAL;
}

/* libm single-precision cos/sin, as std::cos(float) in QAngle<float>. */
float oracle_cosf(float x) { return cosf(x); }
float oracle_sinf(float x) { return sinf(x); }
