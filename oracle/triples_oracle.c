/*
 * ORACLE: CPU restatement of libcc's CCSD(T) non-iterative triples correction.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference legs load this file, and only as the checker or as
 * the timed CPU stand-in for the reference's triples.x.  The product path
 * (libcc_b200) never links, imports or calls it.
 *
 * Parity status: PARTIALLY PINNED.
 *   - The reference is Fortran and cannot be compiled here (no Fortran compiler,
 *     DDI ships only as a closed Cray binary), so there is no oracle/_ref build.
 *   - Pinned: the TRANT3 known-answer program (tools/trant3/trant3.f) is
 *     replayed against this file's permutations; the restart-file size formula
 *     reproduces the three published triples.restart sizes.
 *   - Unpinned: the published energies (water aug-cc-pV{D,T,Q}Z, Ar6) need the
 *     GAMESS-written triples.restart inputs, which are not in the reference tree.
 *     Energy parity rests on this literal restatement, cross-checked against an
 *     independent closed-form restatement (oracle/oracle.py) and a long-double
 *     spot check.
 *
 * Conventions: every array is Fortran column-major as in the reference; this
 * file indexes from 0 internally while the reference's occupied indices are
 * 1-based (i_ref = i + 1).  Integers are int64 (the reference builds with
 * -sdefault64, src/triples-ijk/Makefile:10).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t i64;

#define V3(v, a, b, c) (v)[(a) + nu * ((b) + nu * (i64)(c))]

/* ---------------------------------------------------------------------------
 * In-place nu^3 permutations.  TRANT3_SMP ids 1..5:
 *   src/triples-abc/trant3.f:1-81, tools/trant3/trant3.f:36-116,
 *   src/common/common_cc.f90:62-156 (trant3_1/3/4/5).
 *   1: new(a,b,c)=old(a,c,b)   2: new(a,b,c)=old(b,a,c)   3: new(a,b,c)=old(c,b,a)
 *   4: new(a,b,c)=old(b,c,a)   5: new(x,y,z)=old(z,x,y)
 * The loops below walk the same index sets and swap cycles as the reference.
 * ------------------------------------------------------------------------- */
void orc_trant3(double *v, i64 nu, int id)
{
    i64 a, b, c, d;
    double x;
    switch (id) {
    case 1: /* trant3.f:13-24 */
#pragma omp parallel for private(a, c, x) schedule(dynamic, 4)
        for (b = 0; b < nu; b++)
            for (c = 0; c <= b; c++)
                for (a = 0; a < nu; a++) {
                    x = V3(v, a, b, c);
                    V3(v, a, b, c) = V3(v, a, c, b);
                    V3(v, a, c, b) = x;
                }
        break;
    case 2: /* trant3.f:25-36 */
#pragma omp parallel for private(a, b, x) schedule(dynamic, 4)
        for (c = 0; c < nu; c++)
            for (a = 0; a < nu; a++)
                for (b = 0; b <= a; b++) {
                    x = V3(v, a, b, c);
                    V3(v, a, b, c) = V3(v, b, a, c);
                    V3(v, b, a, c) = x;
                }
        break;
    case 3: /* trant3.f:37-48 */
#pragma omp parallel for private(a, c, x) schedule(dynamic, 4)
        for (b = 0; b < nu; b++)
            for (a = 0; a < nu; a++)
                for (c = 0; c <= a; c++) {
                    x = V3(v, a, b, c);
                    V3(v, a, b, c) = V3(v, c, b, a);
                    V3(v, c, b, a) = x;
                }
        break;
    case 4: /* trant3.f:49-66 (the reference splits b over SMP ranks) */
#pragma omp parallel for private(a, c, x) schedule(dynamic, 4)
        for (b = 0; b < nu; b++)
            for (c = 0; c <= b; c++)
                for (a = 0; a <= c; a++) {
                    x = V3(v, a, b, c);
                    V3(v, a, b, c) = V3(v, b, c, a);
                    V3(v, b, c, a) = V3(v, c, a, b);
                    V3(v, c, a, b) = x;
                    if (b == c || c == a) continue;
                    x = V3(v, b, a, c);
                    V3(v, b, a, c) = V3(v, a, c, b);
                    V3(v, a, c, b) = V3(v, c, b, a);
                    V3(v, c, b, a) = x;
                }
        break;
    case 5: /* trant3.f:67-80 (the reference splits a over SMP ranks) */
#pragma omp parallel for private(c, d, x) schedule(dynamic, 4)
        for (a = 0; a < nu; a++)
            for (c = 0; c <= a; c++)
                for (d = 0; d <= c; d++) {
                    x = V3(v, c, d, a);
                    V3(v, c, d, a) = V3(v, a, c, d);
                    V3(v, a, c, d) = V3(v, d, a, c);
                    V3(v, d, a, c) = x;
                    if (a == c || c == d) continue;
                    x = V3(v, a, d, c);
                    V3(v, a, d, c) = V3(v, c, a, d);
                    V3(v, c, a, d) = V3(v, d, c, a);
                    V3(v, d, c, a) = x;
                }
        break;
    default:
        break;
    }
}

/* CPYTSQ: packed lower triangle -> square symmetric (common_functions.f:43-60). */
void orc_cpytsq(const double *a, double *b, i64 na)
{
    i64 ij = 0;
    for (i64 i = 0; i < na; i++)
        for (i64 j = 0; j <= i; j++) {
            b[i + na * j] = a[ij];
            b[j + na * i] = a[ij];
            ij++;
        }
}

/* DDCC_T_GETVE (common_functions.f:106-126): expand the nu packed columns
 * x*nu .. x*nu+nu-1 of VVVO into VE(a,b,c) = (ab|c x).  x is 0-based. */
void orc_getve(const double *vvvo, i64 nu, i64 x, double *ve)
{
    i64 nutr = nu * (nu + 1) / 2;
#pragma omp parallel for schedule(static)
    for (i64 c = 0; c < nu; c++)
        orc_cpytsq(vvvo + (x * nu + c) * nutr, ve + c * nu * nu, nu);
}

/* ---------------------------------------------------------------------------
 * Column-major DGEMM, C = alpha op(A) op(B) + beta C, the BLAS contract the
 * reference calls (src/triples-ijk/dgemm_async.cpp:55-75 forwards the same
 * arguments to cublasDgemm).  Plain loops, OpenMP over columns of C, unless a
 * BLAS DGEMM (Fortran calling convention, 32-bit integers, as the reference's
 * vendor BLAS) has been installed with orc_set_blas: then every call goes to
 * it and its wall time is summed (orc_dgemm_seconds), so the timed CPU
 * baseline can state its DGEMM share.
 * ------------------------------------------------------------------------- */
typedef void (*orc_blas_dgemm_fn)(char *, char *, int *, int *, int *, double *, double *, int *, double *,
                                  int *, double *, double *, int *);
static orc_blas_dgemm_fn g_blas_dgemm = 0;
static double g_dgemm_seconds = 0.0;

void orc_set_blas(void *fn) { g_blas_dgemm = (orc_blas_dgemm_fn)fn; }

/* Seconds spent in the installed BLAS DGEMM since the last reset. */
double orc_dgemm_seconds(int reset)
{
    double s = g_dgemm_seconds;
    if (reset) g_dgemm_seconds = 0.0;
    return s;
}

static void orc_dgemm(char ta, char tb, i64 m, i64 n, i64 k, double alpha,
                      const double *A, i64 lda, const double *B, i64 ldb,
                      double beta, double *C, i64 ldc)
{
    if (g_blas_dgemm) {
        int im = (int)m, in = (int)n, ik = (int)k, ila = (int)lda, ilb = (int)ldb, ilc = (int)ldc;
        double t0 = omp_get_wtime();
        g_blas_dgemm(&ta, &tb, &im, &in, &ik, &alpha, (double *)A, &ila, (double *)B, &ilb, &beta, C, &ilc);
        g_dgemm_seconds += omp_get_wtime() - t0;
        return;
    }
#pragma omp parallel for schedule(static)
    for (i64 j = 0; j < n; j++) {
        double *cj = C + j * ldc;
        if (beta == 0.0)
            for (i64 i = 0; i < m; i++) cj[i] = 0.0;
        else if (beta != 1.0)
            for (i64 i = 0; i < m; i++) cj[i] *= beta;
        if (ta == 'n') {
            for (i64 l = 0; l < k; l++) {
                double blj = (tb == 'n') ? B[l + j * ldb] : B[j + l * ldb];
                if (blj == 0.0) continue;
                double s = alpha * blj;
                const double *al = A + l * lda;
                for (i64 i = 0; i < m; i++) cj[i] += s * al[i];
            }
        } else {
            for (i64 i = 0; i < m; i++) {
                const double *ai = A + i * lda;
                double s = 0.0;
                if (tb == 'n')
                    for (i64 l = 0; l < k; l++) s += ai[l] * B[l + j * ldb];
                else
                    for (i64 l = 0; l < k; l++) s += ai[l] * B[j + l * ldb];
                cj[i] += alpha * s;
            }
        }
    }
}

/* Views used by the reference's tuple kernels (ddcc_t_ijk_big.f:13-19):
 *   t2_x      = T2(1,1,1,x)  as (nu2, no):  t2_x(ab,l) = T2(a,b,l,x)
 *   t2_x(1,y) = T2(1,1,y,x)  as (nu, nu)
 *   vm_xy     = VM(1,1,x,y)  as (no, nu)                                  */
#define T2X(x) (t2 + (i64)(x) * nu2 * no)
#define T2XY(x, y) (t2 + (i64)(x) * nu2 * no + (i64)(y) * nu2)
#define VMXY(x, y) (vm + ((i64)(y) * no + (x)) * nou)

/* ijk_tuple_formv3 (src/triples-abc/ijk_tuple.f90:1-53), smp_np = 1. */
void orc_ijk_formv3(i64 no, i64 nu, i64 i, i64 j, i64 k, const double *t2, const double *vm,
                    const double *ve_i, const double *ve_j, const double *ve_k, double *v3)
{
    const i64 nu2 = nu * nu, nou = no * nu;
    const double om = -1.0, one = 1.0, zero = 0.0;
    orc_dgemm('n', 'n', nu2, nu, no, om, T2X(i), nu2, VMXY(k, j), no, zero, v3, nu2);      /* #0  */
    orc_dgemm('t', 't', nu2, nu, nu, one, ve_i, nu, T2XY(k, j), nu, one, v3, nu2);          /* #11 */
    orc_dgemm('n', 'n', nu, nu2, nu, one, T2XY(i, k), nu, ve_j, nu, one, v3, nu);           /* #8  */
    orc_dgemm('t', 't', nu, nu2, no, om, VMXY(i, k), no, T2X(j), nu2, one, v3, nu);         /* #3  */
    orc_trant3(v3, nu, 1);
    orc_dgemm('n', 'n', nu2, nu, no, om, T2X(i), nu2, VMXY(j, k), no, one, v3, nu2);        /* #1  */
    orc_dgemm('t', 't', nu2, nu, nu, one, ve_i, nu, T2XY(j, k), nu, one, v3, nu2);          /* #10 */
    orc_dgemm('n', 'n', nu, nu2, nu, one, T2XY(i, j), nu, ve_k, nu, one, v3, nu);           /* #6  */
    orc_dgemm('t', 't', nu, nu2, no, om, VMXY(i, j), no, T2X(k), nu2, one, v3, nu);         /* #5  */
    orc_trant3(v3, nu, 4);
    orc_dgemm('n', 'n', nu2, nu, no, om, T2X(j), nu2, VMXY(k, i), no, one, v3, nu2);        /* #2  */
    orc_dgemm('t', 't', nu2, nu, nu, one, ve_j, nu, T2XY(k, i), nu, one, v3, nu2);          /* #9  */
    orc_trant3(v3, nu, 1);
    orc_dgemm('t', 't', nu, nu2, no, om, VMXY(j, i), no, T2X(k), nu2, one, v3, nu);         /* #4  */
    orc_dgemm('n', 'n', nu, nu2, nu, one, T2XY(j, i), nu, ve_k, nu, one, v3, nu);           /* #7  */
    orc_trant3(v3, nu, 4);
    for (i64 a = 0; a < nu; a++) V3(v3, a, a, a) = 0.0; /* ZEROT3, triples-abc/ddcc_aux.f:84-94 */
}

/* ijj_tuple_formv3 (src/triples-abc/ijj_tuple.f90), tuple (i,j,j), i>j. */
void orc_ijj_formv3(i64 no, i64 nu, i64 i, i64 j, const double *t2, const double *vm,
                    const double *ve_i, const double *ve_j, double *v3)
{
    const i64 nu2 = nu * nu, nou = no * nu;
    const double om = -1.0, one = 1.0, zero = 0.0;
    orc_dgemm('n', 'n', nu2, nu, no, om, T2X(i), nu2, VMXY(j, j), no, zero, v3, nu2);
    orc_trant3(v3, nu, 2);
    orc_dgemm('n', 'n', nu2, nu, no, om, T2X(j), nu2, VMXY(j, i), no, one, v3, nu2);
    orc_trant3(v3, nu, 1);
    orc_dgemm('n', 'n', nu2, nu, no, om, T2X(j), nu2, VMXY(i, j), no, one, v3, nu2);
    orc_trant3(v3, nu, 4);
    orc_dgemm('n', 'n', nu, nu2, nu, one, T2XY(i, j), nu, ve_j, nu, one, v3, nu);
    orc_trant3(v3, nu, 3);
    orc_dgemm('n', 'n', nu, nu2, nu, one, T2XY(j, i), nu, ve_j, nu, one, v3, nu);
    orc_trant3(v3, nu, 1);
    orc_dgemm('n', 'n', nu, nu2, nu, one, T2XY(j, j), nu, ve_i, nu, one, v3, nu);
    orc_trant3(v3, nu, 2);
}

/* iij_tuple_formv3 (src/triples-abc/iij_tuple.f90), tuple (i,i,j), i>j. */
void orc_iij_formv3(i64 no, i64 nu, i64 i, i64 j, const double *t2, const double *vm,
                    const double *ve_i, const double *ve_j, double *v3)
{
    const i64 nu2 = nu * nu, nou = no * nu;
    const double om = -1.0, one = 1.0, zero = 0.0;
    orc_dgemm('n', 'n', nu2, nu, no, om, T2X(i), nu2, VMXY(j, i), no, zero, v3, nu2);
    orc_trant3(v3, nu, 1);
    orc_dgemm('n', 'n', nu2, nu, no, om, T2X(i), nu2, VMXY(i, j), no, one, v3, nu2);
    orc_trant3(v3, nu, 2);
    orc_dgemm('n', 'n', nu2, nu, no, om, T2X(j), nu2, VMXY(i, i), no, one, v3, nu2);
    orc_trant3(v3, nu, 2);
    orc_dgemm('n', 'n', nu, nu2, nu, one, T2XY(i, i), nu, ve_j, nu, one, v3, nu);
    orc_trant3(v3, nu, 1);
    orc_dgemm('n', 'n', nu, nu2, nu, one, T2XY(i, j), nu, ve_i, nu, one, v3, nu);  /* t2_i(1,j) */
    orc_trant3(v3, nu, 3);
    orc_dgemm('n', 'n', nu, nu2, nu, one, T2XY(j, i), nu, ve_i, nu, one, v3, nu);  /* t2_j(1,i) */
    orc_trant3(v3, nu, 3);
}

/* SYMT311 (triples-abc/ddcc_aux.f:217-253): id 23 -> V(a,b,c)=V(a,c,b)=V(a,b,c)+V(a,c,b);
 * id 12 -> a<->b; id 13 -> a<->c. */
void orc_symt311(double *v, i64 nu, int id)
{
    i64 a, b, c;
    double x;
    if (id == 23) {
        for (b = 0; b < nu; b++)
            for (c = 0; c <= b; c++)
                for (a = 0; a < nu; a++) {
                    x = V3(v, a, b, c) + V3(v, a, c, b);
                    V3(v, a, b, c) = x;
                    V3(v, a, c, b) = x;
                }
    } else if (id == 12) {
        for (a = 0; a < nu; a++)
            for (b = 0; b <= a; b++)
                for (c = 0; c < nu; c++) {
                    x = V3(v, a, b, c) + V3(v, b, a, c);
                    V3(v, a, b, c) = x;
                    V3(v, b, a, c) = x;
                }
    } else if (id == 13) {
        for (a = 0; a < nu; a++)
            for (b = 0; b < nu; b++)
                for (c = 0; c <= a; c++) {
                    x = V3(v, a, b, c) + V3(v, c, b, a);
                    V3(v, a, b, c) = x;
                    V3(v, c, b, a) = x;
                }
    }
}

/* T3SQUA_SMP (triples-abc/t3squa.f:1-113): x3 over (a,b,c) != (a,a,a);
 * returns CF*x3 with CF = 1/2 when i==j or j==k. */
double orc_t3squa(i64 no, i64 nu, i64 i, i64 j, i64 k, const double *t3, const double *eh, const double *ep)
{
    (void)no;
    double dijk = eh[i] + eh[j] + eh[k];
    double x3 = 0.0;
    /* 16-wide cache blocks of (c, b, a), the c blocks shared out over the
     * threads, as the reference's loops 150/160 */
    const i64 BS = 16, nb = (nu + BS - 1) / BS;
#pragma omp parallel for reduction(+ : x3) schedule(static)
    for (i64 cb = 0; cb < nb; cb++)
        for (i64 bb = 0; bb < nb; bb++)
            for (i64 ab = 0; ab < nb; ab++)
                for (i64 c = cb * BS; c < cb * BS + BS && c < nu; c++)
                    for (i64 b = bb * BS; b < bb * BS + BS && b < nu; b++)
                        for (i64 a = ab * BS; a < ab * BS + BS && a < nu; a++) {
                            if (a == b && b == c) continue;
                            double denom = 1.0 / (dijk - (ep[a] + ep[b] + ep[c]));
                            double d1 = V3(t3, a, b, c);
                            double d2 = V3(t3, a, c, b) + V3(t3, c, b, a) + V3(t3, b, a, c);
                            double d3 = V3(t3, b, c, a) + V3(t3, c, a, b);
                            double f = d1 * 8.0 - 4.0 * d2 + d3 * 2.0;
                            x3 += f * d1 * denom;
                        }
    double cf = (i == j || j == k) ? 0.5 : 1.0;
    return cf * x3;
}

/* ADT3DEN_SMP (triples-abc/ddcc_aux.f:97-115): V3(c,b,a) /= DEH - e_a - e_b - e_c. */
void orc_adt3den(i64 nu, double deh, double *t3, const double *ep)
{
#pragma omp parallel for schedule(static)
    for (i64 a = 0; a < nu; a++)
        for (i64 b = 0; b < nu; b++)
            for (i64 c = 0; c < nu; c++) V3(t3, c, b, a) /= (deh - ep[a] - ep[b] - ep[c]);
}

/* SMT3FOUR_SMP (triples-abc/ddcc_aux.f:189-214). */
static void orc_smt3four(i64 nu, double *t3, const double *v3)
{
#pragma omp parallel for schedule(static)
    for (i64 c = 0; c < nu; c++) {
        for (i64 b = 0; b < nu; b++) V3(t3, b, b, c) = 0.0;
        for (i64 b = 1; b < nu; b++)
            for (i64 a = 0; a < b; a++) {
                V3(t3, a, b, c) = (V3(v3, a, b, c) - V3(v3, b, a, c)) * 2.0 - V3(v3, a, c, b) + V3(v3, b, c, a);
                V3(t3, b, a, c) = -V3(t3, a, b, c);
            }
    }
}

/* T1WT3IJK_SMP (triples-abc/ddcc_aux.f:171-187): v1(:,I) += Z(a,bc) VOE(bc,J,K). */
static void orc_t1wt3ijk(i64 i, i64 j, i64 k, i64 no, i64 nu, double *v1, const double *voe,
                         const double *ti, double *t3)
{
    const i64 nu2 = nu * nu;
    orc_smt3four(nu, t3, ti);
    /* DGEMM('N','N',NU,1,NU2,...): v1(a,I) += sum_bc T3(a,bc) VOE(bc,J,K) */
    const double *x = voe + k * nu2 * no + j * nu2;
    double *y = v1 + i * nu;
    orc_dgemm('n', 'n', nu, 1, nu2, 1.0, t3, nu, x, nu2, 1.0, y, nu);
}

/* DRT1WT3IJK_SMP (triples-abc/ddcc_aux.f:146-169). */
void orc_drt1wt3ijk(i64 i, i64 j, i64 k, i64 no, i64 nu, double *v1, const double *voe, double *ti, double *t3)
{
    orc_t1wt3ijk(i, j, k, no, nu, v1, voe, ti, t3);
    orc_trant3(ti, nu, 1);
    orc_t1wt3ijk(i, k, j, no, nu, v1, voe, ti, t3);
    orc_trant3(ti, nu, 4);
    orc_t1wt3ijk(j, i, k, no, nu, v1, voe, ti, t3);
    orc_trant3(ti, nu, 1);
    orc_t1wt3ijk(j, k, i, no, nu, v1, voe, ti, t3);
    orc_trant3(ti, nu, 5);
    orc_t1wt3ijk(k, i, j, no, nu, v1, voe, ti, t3);
    orc_trant3(ti, nu, 1);
    orc_t1wt3ijk(k, j, i, no, nu, v1, voe, ti, t3);
}

/* DRT1WT3IJ_SMP (triples-abc/ddcc_aux.f:216-226), tuple (i,j,j). */
void orc_drt1wt3ij(i64 i, i64 j, i64 no, i64 nu, double *v1, const double *voe, double *ti, double *t3)
{
    orc_t1wt3ijk(i, j, j, no, nu, v1, voe, ti, t3);
    orc_trant3(ti, nu, 2);
    orc_t1wt3ijk(j, i, j, no, nu, v1, voe, ti, t3);
    orc_trant3(ti, nu, 1);
    orc_t1wt3ijk(j, j, i, no, nu, v1, voe, ti, t3);
}

/* DRT1WT3JK_SMP (triples-abc/ddcc_aux.f:228-238), tuple (j,j,k). */
void orc_drt1wt3jk(i64 j, i64 k, i64 no, i64 nu, double *v1, const double *voe, double *ti, double *t3)
{
    orc_t1wt3ijk(j, j, k, no, nu, v1, voe, ti, t3);
    orc_trant3(ti, nu, 1);
    orc_t1wt3ijk(j, k, j, no, nu, v1, voe, ti, t3);
    orc_trant3(ti, nu, 2);
    orc_t1wt3ijk(k, j, j, no, nu, v1, voe, ti, t3);
}

/* t1wt3_ijk (src/triples-ijk/t1wt3.f90:18-109): the fused a<=b form of the
 * E[4] sum and the v1 update used by the triples-ijk driver.  Returns x3
 * (without the 1/2 degeneracy weight, which the caller applies). */
double orc_t1wt3_fused(i64 i, i64 j, i64 k, i64 no, i64 nu, const double *v3, const double *voe,
                       double *v1, const double *eh, const double *ep)
{
    const i64 nu2 = nu * nu;
#define VOE2(x, y) (voe + ((i64)(y) * no + (x)) * nu2)
    const double *voe_ij = VOE2(i, j), *voe_ji = VOE2(j, i), *voe_ik = VOE2(i, k);
    const double *voe_ki = VOE2(k, i), *voe_jk = VOE2(j, k), *voe_kj = VOE2(k, j);
#undef VOE2
    double dijk = eh[i] + eh[j] + eh[k];
    double x3 = 0.0;
#define W(a, b, c) V3(v3, a, b, c)
    for (i64 c = 0; c < nu; c++)
        for (i64 b = 0; b < nu; b++)
            for (i64 a = 0; a < nu; a++) {
                if (a > b) continue;
                if (a == b && b == c) continue;
                double denom = 1.0 / (dijk - (ep[a] + ep[b] + ep[c]));
                double d1 = W(a, b, c);
                double d2 = W(a, c, b) + W(c, b, a) + W(b, a, c);
                double d3 = W(b, c, a) + W(c, a, b);
                x3 += (d1 * 8.0 - d2 * 4.0 + d3 * 2.0) * d1 * denom;
                if (a == b) continue;
                d1 = W(b, a, c);
                d2 = W(b, c, a) + W(c, a, b) + W(a, b, c);
                d3 = W(a, c, b) + W(c, b, a);
                x3 += (d1 * 8.0 - d2 * 4.0 + d3 * 2.0) * d1 * denom;
                double z1 = (W(a, b, c) - W(b, a, c)) * 2.0 - W(a, c, b) + W(b, c, a);
                double z2 = (W(a, c, b) - W(b, c, a)) * 2.0 - W(a, b, c) + W(b, a, c);
                double z3 = (W(b, a, c) - W(a, b, c)) * 2.0 - W(c, a, b) + W(c, b, a);
                double z4 = (W(b, c, a) - W(a, c, b)) * 2.0 - W(c, b, a) + W(c, a, b);
                double z5 = (W(c, a, b) - W(c, b, a)) * 2.0 - W(b, a, c) + W(a, b, c);
                double z6 = (W(c, b, a) - W(c, a, b)) * 2.0 - W(b, c, a) + W(a, c, b);
                const i64 bc = b + nu * c, ac = a + nu * c;
                v1[a + nu * i] += (z1 * voe_jk[bc] + z2 * voe_kj[bc]) * denom;
                v1[b + nu * i] -= (z1 * voe_jk[ac] + z2 * voe_kj[ac]) * denom;
                v1[a + nu * j] += (z3 * voe_ik[bc] + z5 * voe_ki[bc]) * denom;
                v1[b + nu * j] -= (z3 * voe_ik[ac] + z5 * voe_ki[ac]) * denom;
                v1[a + nu * k] += (z4 * voe_ij[bc] + z6 * voe_ji[bc]) * denom;
                v1[b + nu * k] -= (z4 * voe_ij[ac] + z6 * voe_ji[ac]) * denom;
            }
#undef W
    return x3;
}

/* DDCC_T_TASK (triples-abc/ddcc_aux.f:1-25): task id -> (i,j,k), i>j>k, i outermost.
 * Returns 0-based indices. */
void orc_task(i64 mytask, i64 no, i64 *pi, i64 *pj, i64 *pk)
{
    i64 icntr = 0;
    for (i64 ii = 0; ii < no; ii++)
        for (i64 jj = 0; jj < ii; jj++)
            for (i64 kk = 0; kk < jj; kk++) {
                if (icntr == mytask) {
                    *pi = ii; *pj = jj; *pk = kk;
                    return;
                }
                icntr++;
            }
}

/* DIV_EVEN (triples-abc/ddcc_aux.f:27-42): contiguous block partition; sr 1-based. */
void orc_div_even(i64 n, i64 np, i64 me, i64 *nr, i64 *sr)
{
    i64 ne;
    *nr = n / np;
    ne = n % np;
    if (me < ne) {
        *nr = *nr + 1;
        *sr = (*nr) * me + 1;
    } else {
        *sr = (*nr + 1) * ne + (*nr) * (me - ne) + 1;
    }
}

/* One (T) tuple through the triples-abc CPU pipeline.  kind 0: i>j>k
 * (DDCC_T_IJK_BIG, triples-abc/ddcc_t_ijk_big.f:1-33); kind 1: (i,j,j)
 * (DDCC_T_IJJ_BIG); kind 2: (i,i,k) (DDCC_T_IIJ_BIG,
 * triples-abc/ddcc_t_ijj_iij_big.f:1-203).  (i,j,k) is always the tuple itself.
 * Accumulates into v1 and *etd.  ve_x is the expanded slice of occupied index
 * x after the b<->c swap (tranmd_23); only the slices of distinct indices are read. */
void orc_tuple(int kind, i64 no, i64 nu, i64 i, i64 j, i64 k, const double *t2, const double *vm,
               const double *voe, const double *eh, const double *ep, const double *ve_i,
               const double *ve_j, const double *ve_k, double *v3, double *t3, double *v1, double *etd)
{
    if (kind == 0) {
        orc_ijk_formv3(no, nu, i, j, k, t2, vm, ve_i, ve_j, ve_k, v3);
        *etd += orc_t3squa(no, nu, i, j, k, v3, eh, ep);
        orc_adt3den(nu, eh[i] + eh[j] + eh[k], v3, ep);
        orc_drt1wt3ijk(i, j, k, no, nu, v1, voe, v3, t3);
    } else if (kind == 1) { /* (i,j,j) */
        orc_ijj_formv3(no, nu, i, j, t2, vm, ve_i, ve_j, v3);
        orc_symt311(v3, nu, 23);
        for (i64 a = 0; a < nu; a++) V3(v3, a, a, a) = 0.0;
        *etd += orc_t3squa(no, nu, i, j, j, v3, eh, ep);
        orc_adt3den(nu, eh[i] + eh[j] + eh[j], v3, ep);
        orc_drt1wt3ij(i, j, no, nu, v1, voe, v3, t3);
    } else { /* (i,i,k): DDCC_T_IIJ_BIG(i, j=k) */
        orc_iij_formv3(no, nu, i, k, t2, vm, ve_i, ve_k, v3);
        orc_symt311(v3, nu, 12);
        for (i64 a = 0; a < nu; a++) V3(v3, a, a, a) = 0.0;
        *etd += orc_t3squa(no, nu, i, i, k, v3, eh, ep);
        orc_adt3den(nu, eh[i] + eh[i] + eh[k], v3, ep);
        orc_drt1wt3jk(i, k, no, nu, v1, voe, v3, t3);
    }
}

static void orc_getve_swapped(const double *vvvo, i64 nu, i64 x, double *ve)
{
    orc_getve(vvvo, nu, x, ve);
    orc_trant3(ve, nu, 1); /* tranmd_smp(ve,nu,nu,nu,1,23), triples-abc/triples.f90:238 */
}

/* Whole (T) driver, triples-abc semantics (src/triples-abc/triples.f90:193-342)
 * on one process: ijk tuples in DDCC_T_TASK order, then for i, j<i the ijj
 * and iij tuples, then ets = 2 ddot(trpose(t1), v1).  v1 (nu,no) is written.
 * Returns 0, or -1 when out of memory. */
int orc_cc_triples(i64 no, i64 nu, const double *eh, const double *ep, const double *t1,
                   const double *t2, const double *vm, const double *voe, const double *vvvo,
                   double *v1, double *ets, double *etd)
{
    const i64 nu3 = nu * nu * nu;
    double *v3 = malloc(sizeof(double) * nu3), *t3 = malloc(sizeof(double) * nu3);
    double *ve_i = malloc(sizeof(double) * nu3), *ve_j = malloc(sizeof(double) * nu3);
    double *ve_k = malloc(sizeof(double) * nu3);
    if (!v3 || !t3 || !ve_i || !ve_j || !ve_k) {
        free(v3); free(t3); free(ve_i); free(ve_j); free(ve_k);
        return -1;
    }
    memset(v1, 0, sizeof(double) * nu * no);
    double e = 0.0;
    i64 iold = -1, jold = -1, kold = -1;
    i64 ntuples = no * (no - 1) * (no - 2) / 6;
    for (i64 t = 0; t < ntuples; t++) {
        i64 i, j, k;
        orc_task(t, no, &i, &j, &k);
        if (i != iold) { orc_getve_swapped(vvvo, nu, i, ve_i); iold = i; }
        if (j != jold) { orc_getve_swapped(vvvo, nu, j, ve_j); jold = j; }
        if (k != kold) { orc_getve_swapped(vvvo, nu, k, ve_k); kold = k; }
        orc_tuple(0, no, nu, i, j, k, t2, vm, voe, eh, ep, ve_i, ve_j, ve_k, v3, t3, v1, &e);
    }
    for (i64 i = 0; i < no; i++)
        for (i64 j = 0; j < i; j++) {
            orc_getve_swapped(vvvo, nu, i, ve_i);
            orc_getve_swapped(vvvo, nu, j, ve_j);
            orc_tuple(1, no, nu, i, j, j, t2, vm, voe, eh, ep, ve_i, ve_j, ve_j, v3, t3, v1, &e);
            orc_tuple(2, no, nu, i, i, j, t2, vm, voe, eh, ep, ve_i, ve_i, ve_j, v3, t3, v1, &e);
        }
    /* ets = 2 ddot(trpose(t1), v1): t1 is (no,nu), v1 is (nu,no) (triples.F90:311-312) */
    double s = 0.0;
    for (i64 i = 0; i < no; i++)
        for (i64 a = 0; a < nu; a++) s += t1[i + no * a] * v1[a + nu * i];
    *ets = 2.0 * s;
    *etd = e;
    free(v3); free(t3); free(ve_i); free(ve_j); free(ve_k);
    return 0;
}

/* The reduction half of one tuple (T3SQUA, ADT3DEN, DRT1WT3IJK/IJ/JK) on a W
 * already formed (and, for degenerate tuples, symmetrised) by the caller.
 * kind/(i,j,k) as in orc_tuple.  v3 is divided in place; t3 is scratch. */
void orc_reduce_tuple(int kind, i64 no, i64 nu, i64 i, i64 j, i64 k, double *v3, double *t3,
                      const double *voe, const double *eh, const double *ep, double *v1, double *etd)
{
    *etd += orc_t3squa(no, nu, i, j, k, v3, eh, ep);
    orc_adt3den(nu, eh[i] + eh[j] + eh[k], v3, ep);
    if (kind == 0)
        orc_drt1wt3ijk(i, j, k, no, nu, v1, voe, v3, t3);
    else if (kind == 1)
        orc_drt1wt3ij(i, j, no, nu, v1, voe, v3, t3);
    else
        orc_drt1wt3jk(i, k, no, nu, v1, voe, v3, t3);
}

/* A list of tuples through the same literal pipeline as orc_cc_triples
 * (orc_tuple per tuple, VE slices fetched and b<->c-swapped when a tuple needs
 * an index not already held, as triples-abc/triples.f90:232-313 refetches on a
 * new i/j/k).  list holds 4 integers per tuple: kind (0 i>j>k, 1 (i,j,j),
 * 2 (i,i,k)), i, j, k, 0-based.  Accumulates into v1 (nu,no) and *etd.
 * Returns 0, or -1 when out of memory. */
int orc_cc_triples_list(i64 no, i64 nu, const double *eh, const double *ep, const double *t2, const double *vm,
                        const double *voe, const double *vvvo, const i64 *list, i64 n, double *v1, double *etd)
{
    const i64 nu3 = nu * nu * nu;
    double *v3 = malloc(sizeof(double) * nu3), *t3 = malloc(sizeof(double) * nu3);
    double *slot[3] = {malloc(sizeof(double) * nu3), malloc(sizeof(double) * nu3), malloc(sizeof(double) * nu3)};
    i64 key[3] = {-1, -1, -1};
    if (!v3 || !t3 || !slot[0] || !slot[1] || !slot[2]) {
        free(v3); free(t3); free(slot[0]); free(slot[1]); free(slot[2]);
        return -1;
    }
    for (i64 q = 0; q < n; q++) {
        const int kind = (int)list[4 * q];
        const i64 x[3] = {list[4 * q + 1], list[4 * q + 2], list[4 * q + 3]};
        const double *ve[3];
        for (int r = 0; r < 3; r++) {
            int hit = -1;
            for (int s2 = 0; s2 < 3; s2++)
                if (key[s2] == x[r]) hit = s2;
            if (hit < 0) { /* evict a slot no index of this tuple uses */
                for (int s2 = 0; s2 < 3 && hit < 0; s2++)
                    if (key[s2] != x[0] && key[s2] != x[1] && key[s2] != x[2]) hit = s2;
                orc_getve_swapped(vvvo, nu, x[r], slot[hit]);
                key[hit] = x[r];
            }
            ve[r] = slot[hit];
        }
        orc_tuple(kind, no, nu, x[0], x[1], x[2], t2, vm, voe, eh, ep, ve[0], ve[1], ve[2], v3, t3, v1, etd);
    }
    free(v3); free(t3); free(slot[0]); free(slot[1]); free(slot[2]);
    return 0;
}
