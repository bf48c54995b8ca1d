/*
 * Body of the CPU oracle, included once per element type by qsv_oracle.c
 * with R (real type), SFX (name suffix) and IS_CPLX defined.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of QCLAB++'s
 * state-vector apply path, used by tests/, __graft_entry__.smoke() and the
 * CPU baseline of bench.py as the checker.  It is never linked into the
 * product library.
 *
 * Every gate follows the reference's per-class apply override: the same
 * coefficient construction (lambda_*), the same index loop (apply2 ...
 * apply4bc) and the same operation order, with no FMA contraction
 * (compiled with -ffp-contract=off).
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define CT CAT(cplx_, SFX)
#define FN(name) CAT(name, SFX)

typedef struct { R re, im; } CT;

static inline CT FN(mk)(R re, R im) { CT z; z.re = re; z.im = im; return z; }
/* std::complex operator*: (ac - bd, ad + bc) */
static inline CT FN(cmul)(CT a, CT b) {
  return FN(mk)(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
static inline CT FN(cadd)(CT a, CT b) { return FN(mk)(a.re + b.re, a.im + b.im); }
static inline CT FN(csub)(CT a, CT b) { return FN(mk)(a.re - b.re, a.im - b.im); }
/* real * complex (libstdc++ operator*(const T&, const complex<T>&)) */
static inline CT FN(rmul)(R r, CT x) { return FN(mk)(r * x.re, r * x.im); }
static inline CT FN(conj)(CT z) { return FN(mk)(z.re, -z.im); }

#if IS_CPLX
typedef CT FN(elem_t);
#define EL FN(elem_t)
static inline EL FN(e_mul)(EL m, EL x) { return FN(cmul)(m, x); }
static inline EL FN(e_add)(EL a, EL b) { return FN(cadd)(a, b); }
static inline EL FN(e_sub)(EL a, EL b) { return FN(csub)(a, b); }
static inline EL FN(e_rmul)(R r, EL x) { return FN(rmul)(r, x); }
static inline EL FN(e_neg)(EL x) { return FN(mk)(-x.re, -x.im); }
static inline EL FN(e_from)(R re, R im) { return FN(mk)(re, im); }
#else
typedef R FN(elem_t);
#define EL FN(elem_t)
static inline EL FN(e_mul)(EL m, EL x) { return m * x; }
static inline EL FN(e_add)(EL a, EL b) { return a + b; }
static inline EL FN(e_sub)(EL a, EL b) { return a - b; }
static inline EL FN(e_rmul)(R r, EL x) { return r * x; }
static inline EL FN(e_neg)(EL x) { return -x; }
static inline EL FN(e_from)(R re, R im) { (void)im; return re; }
#endif

/* ---- index masks: src/qgates/apply.hpp:227-256 --------------------------- */
static void FN(masks1)(int n, int q, uint64_t* mL, uint64_t* mR) {
  const int nL = q, nR = n - q - 1;
  *mL = ((1ULL << nL) - 1) << nR;
  *mR = (1ULL << nR) - 1;
}
static void FN(masks2)(int n, int q0, int q1, uint64_t* mL, uint64_t* mC, uint64_t* mR) {
  const int nL = q0, nC = q1 - q0 - 1, nR = n - q1 - 1;
  *mL = ((1ULL << nL) - 1) << (nR + nC);
  *mC = ((1ULL << nC) - 1) << nR;
  *mR = (1ULL << nR) - 1;
}

/* A 2x2 "pair" operation: which lambda of apply.hpp it restates. */
#ifndef ORACLE_PAIR_KINDS
#define ORACLE_PAIR_KINDS
enum { P_GENERIC, P_HADAMARD, P_SWAPX, P_PAULIY, P_RX, P_RY, P_RZ };
#endif
typedef struct {
  int kind;
  EL m11, m12, m21, m22;  /* P_GENERIC (lambda_QGate1)                 */
  R c, s1, s2;            /* P_HADAMARD (c = sqrt2), P_RY (c, s1, s2)  */
  CT s;                   /* P_RX                                       */
  CT l1, l2;              /* P_PAULIY, P_RZ                             */
} FN(pairop);

static void FN(do_pair)(const FN(pairop)* P, EL* v, uint64_t a, uint64_t b) {
  const EL x1 = v[a], x2 = v[b];
  switch (P->kind) {
    case P_GENERIC:  /* lambda_QGate1: apply.hpp:19-24 */
      v[a] = FN(e_add)(FN(e_mul)(P->m11, x1), FN(e_mul)(P->m12, x2));
      v[b] = FN(e_add)(FN(e_mul)(P->m21, x1), FN(e_mul)(P->m22, x2));
      break;
    case P_HADAMARD:  /* lambda_Hadamard: apply.hpp:35-40 */
      v[a] = FN(e_add)(FN(e_rmul)(P->c, x1), FN(e_rmul)(P->c, x2));
      v[b] = FN(e_sub)(FN(e_rmul)(P->c, x1), FN(e_rmul)(P->c, x2));
      break;
    case P_SWAPX:  /* lambda_PauliX: apply.hpp:48-50 */
      v[a] = x2;
      v[b] = x1;
      break;
#if IS_CPLX
    case P_PAULIY:  /* lambda_PauliY: swap, then vector[a] *= l1, vector[b] *= l2 */
      v[a] = FN(cmul)(x2, P->l1);
      v[b] = FN(cmul)(x1, P->l2);
      break;
    case P_RX:  /* lambda_RotationX: c*x1 + s*x2, s*x1 + c*x2 */
      v[a] = FN(cadd)(FN(rmul)(P->c, x1), FN(cmul)(P->s, x2));
      v[b] = FN(cadd)(FN(cmul)(P->s, x1), FN(rmul)(P->c, x2));
      break;
    case P_RZ:  /* lambda_RotationZ: vector[a] *= l1, vector[b] *= l2 */
      v[a] = FN(cmul)(x1, P->l1);
      v[b] = FN(cmul)(x2, P->l2);
      break;
#endif
    case P_RY:  /* lambda_RotationY: c*x1 + s1*x2, s2*x1 + c*x2 */
      v[a] = FN(e_add)(FN(e_rmul)(P->c, x1), FN(e_rmul)(P->s1, x2));
      v[b] = FN(e_add)(FN(e_rmul)(P->s2, x1), FN(e_rmul)(P->c, x2));
      break;
    default:
      break;
  }
}

/* apply2: apply.hpp:259-272 */
static void FN(apply2)(int n, int q, const FN(pairop)* P, EL* v) {
  uint64_t mL, mR;
  FN(masks1)(n, q, &mL, &mR);
  const uint64_t cnt = 1ULL << (n - 1), b1 = 1ULL << (n - q - 1);
  for (uint64_t k = 0; k < cnt; k++) {
    const uint64_t a = ((k & mL) << 1) | (k & mR);
    FN(do_pair)(P, v, a, a | b1);
  }
}

/* apply4 (controlled): apply.hpp:311-332 */
static void FN(apply4c)(int n, int q0, int q1, int control, int target, int cs,
                        const FN(pairop)* P, EL* v) {
  uint64_t mL, mC, mR;
  FN(masks2)(n, q0, q1, &mL, &mC, &mR);
  const uint64_t cnt = 1ULL << (n - 2);
  uint64_t a1 = 0, b1 = 1ULL << (n - target - 1);
  if (cs == 1) {
    a1 += 1ULL << (n - control - 1);
    b1 += 1ULL << (n - control - 1);
  }
  for (uint64_t k = 0; k < cnt; k++) {
    const uint64_t i = ((k & mL) << 2) | ((k & mC) << 1) | (k & mR);
    FN(do_pair)(P, v, i | a1, i | b1);
  }
}

/* lambda_Phase/PauliZ on one index: negate (PauliZ) or multiply */
typedef struct { int neg; EL lam; } FN(scaleop);
static inline void FN(do_scale)(const FN(scaleop)* S, EL* v, uint64_t b) {
#if IS_CPLX
  v[b] = S->neg ? FN(e_neg)(v[b]) : FN(cmul)(v[b], S->lam);
#else
  v[b] = S->neg ? FN(e_neg)(v[b]) : v[b] * S->lam;
#endif
}

/* apply2b: apply.hpp:275-287 */
static void FN(apply2b)(int n, int q, const FN(scaleop)* S, EL* v) {
  uint64_t mL, mR;
  FN(masks1)(n, q, &mL, &mR);
  const uint64_t cnt = 1ULL << (n - 1), b1 = 1ULL << (n - q - 1);
  for (uint64_t k = 0; k < cnt; k++) FN(do_scale)(S, v, ((k & mL) << 1) | b1 | (k & mR));
}

/* apply4b: apply.hpp:335-352 */
static void FN(apply4b)(int n, int q0, int q1, int control, int target, int cs,
                        const FN(scaleop)* S, EL* v) {
  uint64_t mL, mC, mR;
  FN(masks2)(n, q0, q1, &mL, &mC, &mR);
  const uint64_t cnt = 1ULL << (n - 2);
  uint64_t b1 = 1ULL << (n - target - 1);
  if (cs == 1) b1 += 1ULL << (n - control - 1);
  for (uint64_t k = 0; k < cnt; k++)
    FN(do_scale)(S, v, ((k & mL) << 2) | ((k & mC) << 1) | (k & mR) | b1);
}

/* apply4 (dense) with lambda_QGate2: apply.hpp:172-198, 290-308 */
static void FN(apply4)(int n, int q0, int q1, const EL* M /* row-major 4x4 */, EL* v) {
  uint64_t mL, mC, mR;
  FN(masks2)(n, q0, q1, &mL, &mC, &mR);
  const uint64_t cnt = 1ULL << (n - 2);
  const uint64_t b1 = 1ULL << (n - q0 - 1), c1 = 1ULL << (n - q1 - 1), d1 = b1 | c1;
  for (uint64_t k = 0; k < cnt; k++) {
    const uint64_t a = (k & mR) + ((k & mC) << 1) + ((k & mL) << 2);
    const uint64_t idx[4] = {a, a | b1, a | c1, a | d1};
    const EL x[4] = {v[idx[0]], v[idx[1]], v[idx[2]], v[idx[3]]};
    for (int r = 0; r < 4; r++) {
      EL acc = FN(e_add)(FN(e_mul)(M[4 * r + 0], x[0]), FN(e_mul)(M[4 * r + 1], x[1]));
      acc = FN(e_add)(acc, FN(e_mul)(M[4 * r + 2], x[2]));
      acc = FN(e_add)(acc, FN(e_mul)(M[4 * r + 3], x[3]));
      v[idx[r]] = acc;
    }
  }
}

/* apply4bc with lambda_SWAP / lambda_iSWAP: apply.hpp:202-223, 355-371 */
static void FN(apply4bc)(int n, int q0, int q1, int mul, CT lam, EL* v) {
  uint64_t mL, mC, mR;
  FN(masks2)(n, q0, q1, &mL, &mC, &mR);
  const uint64_t cnt = 1ULL << (n - 2);
  const uint64_t b1 = 1ULL << (n - q0 - 1), c1 = 1ULL << (n - q1 - 1);
  for (uint64_t k = 0; k < cnt; k++) {
    const uint64_t a = ((k & mL) << 2) | ((k & mC) << 1) | (k & mR);
    const uint64_t b = a | b1, c = a | c1;
    const EL t = v[b];
    v[b] = v[c];
    v[c] = t;
#if IS_CPLX
    if (mul) {
      v[b] = FN(cmul)(v[b], lam);
      v[c] = FN(cmul)(v[c], lam);
    }
#else
    (void)mul; (void)lam;
#endif
  }
}

/* operateInPlace for a row-major dim x dim matrix (transpose.hpp:13-35) */
static void FN(operate)(char op, EL* A, int dim) {
  if (op == 'N') return;
#if IS_CPLX
  if (op == 'C')
    for (int i = 0; i < dim * dim; i++) A[i].im = -A[i].im;
#endif
  for (int i = 0; i < dim; i++)
    for (int j = i + 1; j < dim; j++) {
      const EL t = A[i * dim + j];
      A[i * dim + j] = A[j * dim + i];
      A[j * dim + i] = t;
    }
}

/* column-major (re,im) record matrix -> row-major EL, entries rounded to R;
 * a real state rejects entries with non-zero imaginary part */
static int FN(load_matrix)(const double* src, EL* A, int dim) {
  for (int r = 0; r < dim; r++)
    for (int c = 0; c < dim; c++) {
      const double re = src[2 * (r + c * dim)], im = src[2 * (r + c * dim) + 1];
#if !IS_CPLX
      if (im != 0.0) return ORACLE_EDTYPE;
#endif
      A[r * dim + c] = FN(e_from)((R)re, (R)im);
    }
  return 0;
}

static int FN(apply_gate)(int n, EL* v, const qsv_gate* g, char op, int offset) {
  const int k = g->kind;
  const R cs = (R)g->cos, sn = (R)g->sin;
  (void)cs; (void)sn;
  if (k < 0 || k >= QSV_NUM_GATE_KINDS) return ORACLE_EINVAL;
  if (k <= QSV_MATRIX1) {
    const int q = g->qubit0 + offset;
    if (q < 0 || q >= n) return ORACLE_EQUBIT;
    FN(pairop) P;
    memset(&P, 0, sizeof(P));
    FN(scaleop) S;
    memset(&S, 0, sizeof(S));
    switch (k) {
      case QSV_IDENTITY:  /* Identity.cpp:7-11: no-op */
        return 0;
      case QSV_HADAMARD:  /* Hadamard.cpp:8-14 */
        P.kind = P_HADAMARD;
        P.c = (R)1 / SQRT((R)2);
        FN(apply2)(n, q, &P, v);
        return 0;
      case QSV_PAULI_X:  /* PauliX.cpp:8-13 */
        P.kind = P_SWAPX;
        FN(apply2)(n, q, &P, v);
        return 0;
      case QSV_PAULI_Y:  /* PauliY.cpp:8-13, lambda_PauliY */
#if IS_CPLX
        P.kind = P_PAULIY;
        P.l1 = FN(mk)(0, -1);
        P.l2 = FN(mk)(0, 1);
        if (op == 'T') { CT t = P.l1; P.l1 = P.l2; P.l2 = t; }
        FN(apply2)(n, q, &P, v);
        return 0;
#else
        return ORACLE_EDTYPE;
#endif
      case QSV_PAULI_Z:  /* PauliZ.cpp:8-13 */
        S.neg = 1;
        FN(apply2b)(n, q, &S, v);
        return 0;
      case QSV_ROTATION_X:  /* RotationX.cpp:8-14 */
#if IS_CPLX
        P.kind = P_RX;
        P.c = cs;
        P.s = FN(mk)(0, -sn);
        if (op == 'C') P.s = FN(conj)(P.s);
        FN(apply2)(n, q, &P, v);
        return 0;
#else
        return ORACLE_EDTYPE;
#endif
      case QSV_ROTATION_Y:  /* RotationY.cpp:8-14 */
        P.kind = P_RY;
        P.c = cs;
        P.s1 = -sn;
        P.s2 = sn;
        if (op != 'N') { R t = P.s1; P.s1 = P.s2; P.s2 = t; }
        FN(apply2)(n, q, &P, v);
        return 0;
      case QSV_ROTATION_Z:  /* RotationZ.cpp:8-14 (apply2, full pass) */
#if IS_CPLX
        P.kind = P_RZ;
        P.l1 = FN(mk)(cs, -sn);
        P.l2 = FN(mk)(cs, sn);
        if (op == 'C') { CT t = P.l1; P.l1 = P.l2; P.l2 = t; }
        FN(apply2)(n, q, &P, v);
        return 0;
#else
        return ORACLE_EDTYPE;
#endif
      case QSV_PHASE:    /* Phase.cpp:8-14 */
      case QSV_PHASE45:  /* Phase45.cpp:8-14 */
      case QSV_PHASE90: {  /* Phase90.cpp:8-14 */
#if IS_CPLX
        CT l;
        if (k == QSV_PHASE) l = FN(mk)(cs, sn);
        else if (k == QSV_PHASE45) { const R s2 = (R)1 / SQRT((R)2); l = FN(mk)(s2, s2); }
        else l = FN(mk)(0, 1);
        if (op == 'C') l = FN(conj)(l);
        S.lam = l;
        FN(apply2b)(n, q, &S, v);
        return 0;
#else
        return ORACLE_EDTYPE;
#endif
      }
      case QSV_MATRIX1: {  /* QGate1.cpp:8-13 with lambda_QGate1 */
        EL A[4];
        if (FN(load_matrix)(g->matrix, A, 2)) return ORACLE_EDTYPE;
        FN(operate)(op, A, 2);
        P.kind = P_GENERIC;
        P.m11 = A[0]; P.m12 = A[1]; P.m21 = A[2]; P.m22 = A[3];
        FN(apply2)(n, q, &P, v);
        return 0;
      }
    }
    return ORACLE_EINVAL;
  }

  if (n < 2) return ORACLE_EQUBIT;
  const int qa = g->qubit0 + offset, qb = g->qubit1 + offset;
  if (qa < 0 || qa >= n || qb < 0 || qb >= n || qa == qb) return ORACLE_EQUBIT;
  const int q0 = qa < qb ? qa : qb, q1 = qa < qb ? qb : qa;

  if (k >= QSV_CX && k <= QSV_CONTROLLED1) {
    const int control = qa, target = qb, cst = g->control_state;
    if (cst != 0 && cst != 1) return ORACLE_EINVAL;
    FN(pairop) P;
    memset(&P, 0, sizeof(P));
    FN(scaleop) S;
    memset(&S, 0, sizeof(S));
    switch (k) {
      case QSV_CX:  /* CX.cpp:8-18 */
        P.kind = P_SWAPX;
        FN(apply4c)(n, q0, q1, control, target, cst, &P, v);
        return 0;
      case QSV_CY:  /* CY.cpp:8-18 */
#if IS_CPLX
        P.kind = P_PAULIY;
        P.l1 = FN(mk)(0, -1);
        P.l2 = FN(mk)(0, 1);
        if (op == 'T') { CT t = P.l1; P.l1 = P.l2; P.l2 = t; }
        FN(apply4c)(n, q0, q1, control, target, cst, &P, v);
        return 0;
#else
        return ORACLE_EDTYPE;
#endif
      case QSV_CZ:  /* CZ.cpp:8-18 */
        S.neg = 1;
        FN(apply4b)(n, q0, q1, control, target, cst, &S, v);
        return 0;
      case QSV_CPHASE: {  /* CPhase.cpp:8-19 */
#if IS_CPLX
        CT l = FN(mk)(cs, sn);
        if (op == 'C') l = FN(conj)(l);
        S.lam = l;
        FN(apply4b)(n, q0, q1, control, target, cst, &S, v);
        return 0;
#else
        return ORACLE_EDTYPE;
#endif
      }
      case QSV_CROTATION_Z:  /* CRotationZ.cpp:8-19 */
#if IS_CPLX
        P.kind = P_RZ;
        P.l1 = FN(mk)(cs, -sn);
        P.l2 = FN(mk)(cs, sn);
        if (op == 'C') { CT t = P.l1; P.l1 = P.l2; P.l2 = t; }
        FN(apply4c)(n, q0, q1, control, target, cst, &P, v);
        return 0;
#else
        return ORACLE_EDTYPE;
#endif
      case QSV_CROTATION_X:  /* QControlledGate2.cpp:8-20 + RotationX::matrix */
      case QSV_CROTATION_Y:  /* QControlledGate2.cpp:8-20 + RotationY::matrix */
      case QSV_CONTROLLED1: {
        EL A[4];
        if (k == QSV_CROTATION_X) {
#if IS_CPLX
          A[0] = FN(mk)(cs, 0); A[1] = FN(mk)(0, -sn);
          A[2] = FN(mk)(0, -sn); A[3] = FN(mk)(cs, 0);
#else
          return ORACLE_EDTYPE;
#endif
        } else if (k == QSV_CROTATION_Y) {
          A[0] = FN(e_from)(cs, 0); A[1] = FN(e_from)(-sn, 0);
          A[2] = FN(e_from)(sn, 0); A[3] = FN(e_from)(cs, 0);
        } else if (FN(load_matrix)(g->matrix, A, 2)) {
          return ORACLE_EDTYPE;
        }
        FN(operate)(op, A, 2);
        P.kind = P_GENERIC;
        P.m11 = A[0]; P.m12 = A[1]; P.m21 = A[2]; P.m22 = A[3];
        FN(apply4c)(n, q0, q1, control, target, cst, &P, v);
        return 0;
      }
    }
    return ORACLE_EINVAL;
  }

  switch (k) {
    case QSV_SWAP:  /* SWAP.cpp:9-16 */
      FN(apply4bc)(n, q0, q1, 0, FN(mk)(1, 0), v);
      return 0;
    case QSV_ISWAP:  /* iSWAP.cpp:11-18 */
#if IS_CPLX
      FN(apply4bc)(n, q0, q1, 1, op == 'C' ? FN(mk)(0, -1) : FN(mk)(0, 1), v);
      return 0;
#else
      return ORACLE_EDTYPE;
#endif
    case QSV_ROTATION_XX:
    case QSV_ROTATION_YY:
    case QSV_ROTATION_ZZ: {  /* QGate2.cpp:8-15 with RotationXX/YY/ZZ::matrix */
#if IS_CPLX
      EL M[16];
      memset(M, 0, sizeof(M));
      if (k == QSV_ROTATION_XX) {  /* RotationXX.hpp:136-143 */
        const CT d = FN(mk)(cs, 0), o = FN(mk)(0, -sn);
        M[0] = d; M[3] = o; M[5] = d; M[6] = o; M[9] = o; M[10] = d; M[12] = o; M[15] = d;
      } else if (k == QSV_ROTATION_YY) {  /* RotationYY.hpp:136-143 */
        const CT d = FN(mk)(cs, 0), o = FN(mk)(0, sn), mo = FN(mk)(-(R)0, -sn);
        M[0] = d; M[3] = o; M[5] = d; M[6] = mo; M[9] = mo; M[10] = d; M[12] = o; M[15] = d;
      } else {  /* RotationZZ.hpp:136-143 */
        const CT a = FN(mk)(cs, -sn), b = FN(mk)(cs, sn);
        M[0] = a; M[5] = b; M[10] = b; M[15] = a;
      }
      FN(operate)(op, M, 4);
      FN(apply4)(n, q0, q1, M, v);
      return 0;
#else
      return ORACLE_EDTYPE;
#endif
    }
    case QSV_MATRIX2: {
      /* New gate (no reference class): the 4x4 acts in the kron basis
       * |qubit0 qubit1>.  Applied as a QCLAB++ user would with a QGate2
       * subclass: the matrix is reordered to apply4's amplitude order
       * (x1..x4 = |00>,|10>,|01>,|11> of the sorted qubits q0 < q1,
       * apply.hpp:296-306) and applied by apply4 + lambda_QGate2. */
      EL K[16], M[16];
      int slot_of[4];
      if (FN(load_matrix)(g->matrix, K, 4)) return ORACLE_EDTYPE;
      for (int s = 0; s < 4; s++) {
        const int bq0 = s & 1, bq1 = s >> 1;            /* bits of q0, q1 */
        const int bfirst = (qa == q0) ? bq0 : bq1;      /* bit of qubit0 */
        const int bsecond = (qa == q0) ? bq1 : bq0;     /* bit of qubit1 */
        slot_of[s] = 2 * bfirst + bsecond;
      }
      for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) M[4 * r + c] = K[4 * slot_of[r] + slot_of[c]];
      FN(operate)(op, M, 4);
      FN(apply4)(n, q0, q1, M, v);
      return 0;
    }
  }
  return ORACLE_EINVAL;
}

/* QCircuit::apply order: forward for 'N', reverse for 'T'/'C'
 * (include/qclab/QCircuit.hpp:130-143). */
static int FN(apply_list)(int n, EL* v, const qsv_gate* gates, size_t count, char op,
                          int offset) {
  if (op != 'N' && op != 'T' && op != 'C') return ORACLE_EINVAL;
  for (size_t i = 0; i < count; i++) {
    const size_t src = (op == 'N') ? i : count - 1 - i;
    const int st = FN(apply_gate)(n, v, &gates[src], op, offset);
    if (st) return st;
  }
  return 0;
}

#undef EL
#undef CT
#undef FN
#undef CAT
#undef CAT2
