/*
 * CPU restatement of SPR's numeric phase -- the oracle.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/, by the smoke check and by the
 * CPU-baseline leg of bench.py; never linked into the product.
 *
 * Restates, in plain C of its own, the algorithm of
 *   SPRSOL  src/SPR/sprsol.f:5-52      (IOP dispatch)
 *   SPRFC1  src/SPR/sprfc1.f:5-283     (checks, error mapping, MSPAR(1/26/27))
 *   SPRF11  src/SPR/sprfc1.f:286-713   (multifrontal loop, TOL(2)/TOL(3))
 *   SPRF12/13/14 sprfc1.f:716-982      (relative indices, extend-add)
 *   SPRF15/17 sprfc1.f:985-1299        (LDL' of the S fully-summed columns)
 *   SPRFC3/SPRF31/SPRF37 src/SPR/sprfc3.f:5-277, 372-806, 1011-1104
 *                                      (the variant that replaces singular
 *                                       pivots and records them in DCOR)
 *   SPRFC2/SPRF21/SPRF27, CMVY18, CMMY18 src/SPR/sprfc2.f, cmvy18.f,
 *                                      cmmy18.f (Cholesky C C')
 *   SPRFS2/SPRFS7/SPRFS9, SPRBS2/SPRBS7/SPRBS9 src/SPR/sprfs2.f, sprbs2.f
 *                                      (its forward and back solves)
 *   SPRFC4/SPRF41/SPRF47 src/SPR/sprfc4.f (the Cholesky form of SPRFC3)
 *   LMVY18  src/SPR/lmvy18.f:5-173     (column update inside SPRF17)
 *   LMMY18  src/SPR/lmmy18.f:5-192     (Schur update of the update matrix)
 *   SPRFS1/3/5/6, SPRFB1/2 src/SPR/sprfs1.f  (forward + diagonal solve)
 *   SPRBS1/4/6 src/SPR/sprbs1.f        (back solve)
 * for the configurations the GPU path handles: MSPAR(58)=0, no panels
 * (numerically identical, panels only re-block), and MSPAR(57) <= 0 or the
 * partial factorisation of MSPAR(57) > 0: the retained supernodes
 * (SUPSUP > 0) are assembled but not eliminated (sprfc1.f:463-470,
 * 587-608) and skipped by the solves (sprfs1.f:371, sprbs1.f:347), which
 * treat the equations beyond LDB < NEQ as absent (sprfs1.f:201,
 * sprbs1.f:189).
 *
 * Every floating-point update is accumulated in the same order as the
 * reference (the 8-way unrolled groups of LMMY18/LMVY18/SPRFS6 add their
 * terms left to right, i.e. sequentially in k), and the scaling uses the
 * reciprocal of the pivot as SPRF17 does, so with -ffp-contract=off the
 * results are bitwise equal to the reference's.  Fronts are held as dense
 * column-major F x F arrays instead of SPR's packed stack: storage differs,
 * arithmetic does not.
 *
 * Integers are int64_t (the SPR_I8 build).  All arrays are 1-based in the
 * Fortran sense; this file indexes them 0-based.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t I;

typedef struct {
    I neq, nsuper, nofsub, nzerol, mfront;
    const I *xsuper, *xsibl, *sibl, *xlindx, *lindx, *xlnz;
    const I *supsup;     /* SUPSUP(NSUPER), MTREES(XLINDX+NSUPER+1) (sprfc1.f:183) */
    I lpar57;            /* MSPAR(57) */
} sym_t;

/* A retained supernode of a partial factorisation (sprfc1.f:587). */
static int retained(const sym_t *s, I js)
{
    return s->lpar57 > 0 && s->supsup[js] > 0;
}

/* Pointers into MTREES/MSIFA exactly as SPRFC1 derives them (sprfc1.f:165-196). */
static void sym_from_mspar(sym_t *s, const I *mspar, const I *mtrees, const I *msifa)
{
    s->neq = mspar[7];
    s->nsuper = mspar[10];
    s->mfront = mspar[13];
    s->nofsub = mspar[14];
    s->nzerol = mspar[15];
    const I *xs = mtrees + (mspar[44] - 1);
    s->xsuper = xs;
    s->xsibl = xs + (s->nsuper + 1);
    s->sibl = xs + 2 * (s->nsuper + 1);
    s->xlindx = mtrees + (mspar[45] - 1);
    s->lindx = msifa + (mspar[46] - 1);
    s->xlnz = msifa + (mspar[47] - 1);
    s->supsup = s->xlindx + (s->nsuper + 1);
    s->lpar57 = mspar[56];
}

/* ---------------------------------------------------------------------- */
/* Factorisation: SPRFC1 / SPRF11                                          */
/* ---------------------------------------------------------------------- */

typedef struct {
    double *upd;     /* dense (F-S) x (F-S) update matrix, column-major    */
    I n;             /* its order                                          */
} update_t;

/* Returns the SPRF11 ERROR code (0, -30 or -35) and fills numneg/supeqt.
 * With dcor != NULL it follows SPRF31 instead (sprfc3.f:372-806): zero
 * diagonals become 1, pivots at or below TOL(1)|a_jj| are replaced
 * (SPRF37, sprfc3.f:1083-1099), and the code is -31 with supeqt = the number
 * replaced, or 0. */
static I oracle_factor_mode(const sym_t *s, double *diag, double *lnz, double *tol,
                            I *numneg_out, I *supeqt_out, double *dcor, int chol)
{
    const I ns = s->nsuper;
    I numneg = 0, supeqt = 0, error = 0, nsing = 0;
    tol[1] = 0.0;
    tol[2] = 0.0;
    if (s->lpar57 > 0) {                 /* sprfc1.f:463, sprfc3.f:551-554 */
        for (I i = 0; i < s->neq; i++) diag[i] = 0.0;
        if (dcor)
            for (I i = 0; i < 2 * s->neq; i++) dcor[i] = 0.0;
    }
    /* pre-pass: original diagonal, zero check, trace (sprfc1.f:465-488) */
    for (I js = 0; js < ns; js++) {
        if (retained(s, js)) continue;   /* sprfc1.f:467 */
        I len = s->xlindx[js + 1] - s->xlindx[js];
        I p = s->xlnz[js] - 1;
        for (I j = s->xsuper[js]; j < s->xsuper[js + 1]; j++) {
            diag[j - 1] = lnz[p];
            if (dcor) {                  /* sprfc3.f:561-573 */
                dcor[2 * (j - 1)] = 0.0;
                dcor[2 * (j - 1) + 1] = 0.0;
                if (diag[j - 1] == 0.0) {
                    diag[j - 1] = 1.0;
                    dcor[2 * (j - 1) + 1] = 1.0;
                    lnz[p] = 1.0;
                }
            } else if (diag[j - 1] == 0.0) {
                numneg++;
                if (numneg == 1) {
                    supeqt = j;
                    error = -35;
                }
            }
            tol[2] = tol[2] + diag[j - 1];
            p += len;
            len -= 1;
        }
    }
    if (error < 0) {
        *numneg_out = numneg;
        *supeqt_out = supeqt;
        return error;
    }
    update_t *pend = (update_t *)calloc((size_t)ns, sizeof(update_t));
    I *rel = (I *)malloc(sizeof(I) * (size_t)(s->mfront + 1));
    for (I js = 0; js < ns && error == 0; js++) {
        const I fst = s->xsuper[js];
        const I S = s->xsuper[js + 1] - fst;
        const I F = s->xlindx[js + 1] - s->xlindx[js];
        const I *rows = s->lindx + (s->xlindx[js] - 1);
        double *X = (double *)calloc((size_t)(F * F), sizeof(double));
        /* fully-summed columns from LNZ; packed column j has F-j entries */
        I p = s->xlnz[js] - 1;
        for (I j = 0; j < S; j++)
            for (I i = j; i < F; i++)
                X[i + j * F] = lnz[p++];
        /* extend-add of the children, last sibling first (sprfc1.f:534) */
        for (I k = s->xsibl[js + 1] - 1; k >= s->xsibl[js]; k--) {
            const I c = s->sibl[k - 1] - 1;
            const I cS = s->xsuper[c + 1] - s->xsuper[c];
            const I *crow = s->lindx + (s->xlindx[c] - 1) + cS;
            const I n = pend[c].n;
            double *U = pend[c].upd;
            /* SPRF12: monotone merge of the child's rows into the parent's */
            I sup = 0;
            for (I t = 0; t < n; t++) {
                while (rows[sup] < crow[t]) sup++;
                rel[t] = sup;
                sup++;
            }
            for (I b = 0; b < n; b++)
                for (I a = b; a < n; a++)
                    X[rel[a] + rel[b] * F] += U[a + b * n];
            free(U);
            pend[c].upd = NULL;
        }
        /* SPRF17: left-looking LDL' of columns 0..S-1 over all F rows; a
         * retained supernode is only assembled (sprfc1.f:587) */
        const I Se = retained(s, js) ? 0 : S;
        for (I j = 0; j < Se && error == 0; j++) {
            for (I k = 0; k < j; k++) {     /* LMVY18, or CMVY18 without D */
                const double a = chol ? -X[j + k * F] : -(X[j + k * F] * diag[fst - 1 + k]);
                for (I i = j; i < F; i++)
                    X[i + j * F] = X[i + j * F] + a * X[i + k * F];
            }
            const double adiag = diag[fst - 1 + j];
            double d = X[j + j * F];
            if (chol && dcor) {          /* SPRF47, sprfc4.f:978-996 */
                double *dc = dcor + 2 * (fst - 1 + j);
                if (d < -tol[0] * fabs(adiag)) {
                    error = -(j + 1);
                    tol[1] = d;
                    tol[2] = adiag;
                    dc[0] = d;
                    dc[1] = d;
                    break;
                } else if (d <= tol[0] * fabs(adiag)) {
                    nsing++;
                    dc[0] = d;
                    const double m = fabs(tol[3] * adiag);
                    d = tol[0] * (m > 1.0 ? m : 1.0);
                    X[j + j * F] = d;
                    dc[1] = d;
                }
            } else if (chol) {           /* SPRF27, sprfc2.f:1001-1032 */
                if (d <= tol[0] * fabs(adiag)) {
                    error = -(j + 1);
                    tol[1] = d;
                    tol[2] = adiag;
                    break;
                }
            }
            if (chol) {
                const double r0 = adiag / d;
                tol[1] = (tol[1] > r0) ? tol[1] : r0;
                d = sqrt(d);
                diag[fst - 1 + j] = d;
                X[j + j * F] = d;
                d = 1.0 / d;
                for (I i = j + 1; i < F; i++) X[i + j * F] = X[i + j * F] * d;
                continue;
            }
            if (dcor) {                  /* SPRF37, sprfc3.f:1083-1099 */
                double *dc = dcor + 2 * (fst - 1 + j);
                if (fabs(d) <= tol[0] * fabs(adiag)) {
                    nsing++;
                    dc[0] = d;
                    const double m = fabs(tol[3] * adiag);
                    d = copysign(fabs(tol[0] * (m > 1.0 ? m : 1.0)), d);
                    X[j + j * F] = d;
                    dc[1] = d;
                }
                if (d < 0.0 && dc[0] == 0.0) dc[0] = d;
            } else if (fabs(d) <= tol[0] * fabs(adiag)) {
                error = -(j + 1);
                tol[1] = d;
                tol[2] = adiag;
                break;
            }
            if (d < 0.0) numneg++;
            diag[fst - 1 + j] = d;
            const double r = adiag / d;
            tol[1] = (tol[1] > r) ? tol[1] : r;
            d = 1.0 / d;
            for (I i = j + 1; i < F; i++) X[i + j * F] = X[i + j * F] * d;
        }
        if (error != 0) {
            supeqt = fst - error - 1;
            error = (chol && dcor) ? -32 : -30;   /* sprfc4.f:612-616 */
            free(X);
            break;
        }
        /* LMMY18: Y <- Y - X D X' on the lower part of the update matrix */
        const I q = F - S;
        if (q > 0) {
            double *U = (double *)malloc(sizeof(double) * (size_t)(q * q));
            for (I b = 0; b < q; b++) {
                for (I a = b; a < q; a++) U[a + b * q] = X[(S + a) + (S + b) * F];
                for (I k = 0; k < Se; k++) {   /* LMMY18, or CMMY18 without D */
                    const double a1 = chol ? -X[(S + b) + k * F] : -(X[(S + b) + k * F] * diag[fst - 1 + k]);
                    for (I a = b; a < q; a++)
                        U[a + b * q] = U[a + b * q] + a1 * X[(S + a) + k * F];
                }
            }
            pend[js].upd = U;
            pend[js].n = q;
        }
        /* store the S-column trapezoid back into LNZ (sprfc1.f:630-637) */
        p = s->xlnz[js] - 1;
        for (I j = 0; j < S; j++)
            for (I i = j; i < F; i++)
                lnz[p++] = X[i + j * F];
        free(X);
    }
    for (I js = 0; js < ns; js++) free(pend[js].upd);
    free(pend);
    free(rel);
    if (error == 0) {
        double mdiag = 0.0;
        for (I i = 0; i < s->neq; i++)
            if (diag[i] > 0.0 && (mdiag == 0.0 || mdiag > diag[i])) mdiag = diag[i];
        tol[1] = (tol[1] != 0.0) ? 1.0 / tol[1] : 0.0;
        if (chol)                        /* sprfc2.f:712-716 */
            tol[2] = (mdiag != 0.0) ? tol[2] / (mdiag * mdiag) : 0.0;
        else
            tol[2] = (mdiag != 0.0) ? tol[2] / mdiag : 0.0;
    }
    if (dcor && nsing > 0) {             /* sprfc3.f:796-799, sprfc4.f:719-722 */
        supeqt = nsing;
        error = chol ? -33 : -31;
    }
    *numneg_out = numneg;
    *supeqt_out = supeqt;
    return error;
}

static I oracle_factor(const sym_t *s, double *diag, double *lnz, double *tol,
                       I *numneg_out, I *supeqt_out, double *dcor)
{
    return oracle_factor_mode(s, diag, lnz, tol, numneg_out, supeqt_out, dcor, 0);
}

/* ---------------------------------------------------------------------- */
/* Solves: SPRFS3/SPRFS5/SPRFS6 and SPRBS4/SPRBS6                          */
/* ---------------------------------------------------------------------- */

/* chol: the Cholesky forward solve C y = b of SPRFS9 (sprfs2.f:575-610):
 * each column is divided by its diagonal before it updates the others. */
static void oracle_forward(const sym_t *s, const double *lnz, double *b, double *loc, int chol)
{
    I p0 = 0;
    for (I js = 0; js < s->nsuper; js++) {
        const I S = s->xsuper[js + 1] - s->xsuper[js];
        const I F = s->xlindx[js + 1] - s->xlindx[js];
        const I *rows = s->lindx + (s->xlindx[js] - 1);
        const double *L = lnz + p0;
        if (retained(s, js)) {           /* sprfs1.f:371 */
            p0 += F * S - (S * (S - 1)) / 2;
            continue;
        }
        for (I i = 0; i < F; i++) loc[i] = rows[i] <= s->neq ? b[rows[i] - 1] : 0.0;
        /* column j of the packed trapezoid starts at j*F - j(j-1)/2 */
        for (I j = 0; j < S; j++) {
            const I cj = j * F - (j * (j - 1)) / 2;
            if (chol) loc[j] = loc[j] / L[cj];
            const double x = loc[j];
            for (I i = j + 1; i < S; i++) loc[i] = loc[i] - x * L[cj + (i - j)];
        }
        /* SPRFS6 (sprfs1.f:929-1141): the S mod 8 leading columns in
         * ascending order, then groups of 8 taken from the group's last
         * column down to its first. */
        const I lft = S % 8;
        for (I i = S; i < F; i++) {
            double y = loc[i];
            for (I j = 0; j < lft; j++) {
                const I cj = j * F - (j * (j - 1)) / 2;
                y = y - loc[j] * L[cj + (i - j)];
            }
            for (I jg = lft + 7; jg < S; jg += 8) {
                for (I j = jg; j > jg - 8; j--) {
                    const I cj = j * F - (j * (j - 1)) / 2;
                    y = y - loc[j] * L[cj + (i - j)];
                }
            }
            loc[i] = y;
        }
        if (!chol)
            for (I j = 0; j < S; j++) loc[j] = loc[j] / L[j * F - (j * (j - 1)) / 2];
        for (I i = 0; i < F; i++)
            if (rows[i] <= s->neq) b[rows[i] - 1] = loc[i];
        p0 += F * S - (S * (S - 1)) / 2;
    }
}

/* chol: the Cholesky back solve C' x = y of SPRBS9 (sprbs2.f:500-540). */
static void oracle_backward(const sym_t *s, const double *lnz, double *b, double *loc, int chol)
{
    I p0 = s->nzerol;
    for (I js = s->nsuper - 1; js >= 0; js--) {
        const I S = s->xsuper[js + 1] - s->xsuper[js];
        const I F = s->xlindx[js + 1] - s->xlindx[js];
        const I *rows = s->lindx + (s->xlindx[js] - 1);
        p0 -= F * S - (S * (S - 1)) / 2;
        const double *L = lnz + p0;
        if (retained(s, js)) continue;   /* sprbs1.f:347 */
        for (I i = 0; i < F; i++) loc[i] = rows[i] <= s->neq ? b[rows[i] - 1] : 0.0;
        for (I j = S - 1; j >= 0; j--) {
            const I cj = j * F - (j * (j - 1)) / 2;
            double r = 0.0;
            for (I i = j + 1; i < F; i++) r = r + loc[i] * L[cj + (i - j)];
            loc[j] = chol ? (loc[j] - r) / L[cj] : loc[j] - r;
        }
        for (I i = 0; i < F; i++)
            if (rows[i] <= s->neq) b[rows[i] - 1] = loc[i];
    }
}

/* ---------------------------------------------------------------------- */
/* Fortran-ABI entry points (same arguments as the reference routines)     */
/* ---------------------------------------------------------------------- */

void orc_sprfc1_(I *mspar, I *mtrees, I *msifa, double *sm, double *tol,
                 I *iwork, double *rwork, const I *lpu, I *ierr)
{
    (void)iwork;
    (void)rwork;
    (void)lpu;
    if (mspar[0] < 0) {                  /* sprfc1.f:140-148 */
        mspar[0] = -5;
        *ierr = -1;
        return;
    }
    mspar[0] = 5;
    *ierr = 0;
    sym_t s;
    sym_from_mspar(&s, mspar, mtrees, msifa);
    I numneg = 0, supeqt = 0;
    I lierr = oracle_factor(&s, sm, sm + s.neq, tol, &numneg, &supeqt, NULL);
    if (lierr != 0) {                    /* sprfc1.f:251-265 */
        *ierr = (lierr / 10 == -3) ? -3 : -4;
        mspar[26] = supeqt;
    } else if (numneg > 0) {
        *ierr = 3;
    }
    mspar[25] = numneg;
}

/* SPRFC3 (sprfc3.f:5-277): TOL(4), DCOR(2,NEQ); IERR -3 with MSPAR(27) =
 * -(number of replaced pivots) leaves a complete factor. */
void orc_sprfc3_(I *mspar, I *mtrees, I *msifa, double *sm, double *tol,
                 I *iwork, double *rwork, double *dcor, const I *lpu, I *ierr)
{
    (void)iwork;
    (void)rwork;
    (void)lpu;
    if (mspar[0] < 0) {                  /* sprfc3.f:139-143 */
        mspar[0] = -5;
        *ierr = -1;
        return;
    }
    mspar[0] = 5;
    *ierr = 0;
    sym_t s;
    sym_from_mspar(&s, mspar, mtrees, msifa);
    I numneg = 0, supeqt = 0;
    I lierr = oracle_factor(&s, sm, sm + s.neq, tol, &numneg, &supeqt, dcor);
    if (lierr != 0) {                    /* sprfc3.f:249-258 */
        *ierr = (lierr / 10 == -3) ? -3 : -4;
        mspar[26] = (lierr == -31) ? -supeqt : supeqt;
    } else if (numneg > 0) {
        *ierr = 3;
    }
    mspar[25] = numneg;
}

void orc_sprfs1_(I *mspar, I *mtrees, I *msifa, double *sm, double *b,
                 const I *ldb, const I *nrhs, I *iwork, double *rwork,
                 const I *lpu, I *ierr)
{
    (void)iwork;
    (void)rwork;
    (void)lpu;
    if (mspar[0] < 0) {
        mspar[0] = -7;
        *ierr = -1;
        return;
    }
    mspar[0] = 7;
    *ierr = 0;
    sym_t s;
    sym_from_mspar(&s, mspar, mtrees, msifa);
    const double *lnz = sm + s.neq;      /* LNZ = DIAG + NEQ before the reset */
    if (mspar[56] == 1 && *ldb < s.neq) s.neq = *ldb;   /* sprfs1.f:201 */
    if (*ldb < s.neq) {
        mspar[0] = -2;
        *ierr = -2;
        return;
    }
    double *loc = (double *)malloc(sizeof(double) * (size_t)(s.mfront + 1));
    for (I r = 0; r < *nrhs; r++) oracle_forward(&s, lnz, b + r * (*ldb), loc, 0);
    free(loc);
}

void orc_sprbs1_(I *mspar, I *mtrees, I *msifa, double *sm, double *b,
                 const I *ldb, const I *nrhs, double *rwork, const I *lpu, I *ierr)
{
    (void)rwork;
    (void)lpu;
    if (mspar[0] < 0) {                  /* sprbs1.f:131-139 */
        mspar[0] = -7;
        *ierr = -1;
        return;
    }
    mspar[0] = 7;
    *ierr = 0;
    sym_t s;
    sym_from_mspar(&s, mspar, mtrees, msifa);
    const double *lnz = sm + s.neq;
    if (mspar[56] == 1 && *ldb < s.neq) s.neq = *ldb;   /* sprbs1.f:189 */
    if (*ldb < s.neq) {
        mspar[0] = -2;
        *ierr = -2;
        return;
    }
    double *loc = (double *)malloc(sizeof(double) * (size_t)(s.mfront + 1));
    for (I r = 0; r < *nrhs; r++) oracle_backward(&s, lnz, b + r * (*ldb), loc, 0);
    free(loc);
}

void orc_sprsol_(const I *iop, I *mspar, I *mtrees, I *msifa, double *sm, double *b,
                 const I *ldb, const I *nrhs, double *tol, I *iwork, double *rwork,
                 const I *lpu, I *ierr)
{
    *ierr = 0;                           /* sprsol.f:32-49 */
    if (*iop <= 3) orc_sprfc1_(mspar, mtrees, msifa, sm, tol, iwork, rwork, lpu, ierr);
    if (*iop >= 2 && *iop <= 5 && *ierr >= 0)
        orc_sprfs1_(mspar, mtrees, msifa, sm, b, ldb, nrhs, iwork, rwork, lpu, ierr);
    if (*iop >= 3 && *iop != 5 && *ierr >= 0)
        orc_sprbs1_(mspar, mtrees, msifa, sm, b, ldb, nrhs, rwork, lpu, ierr);
}

/* ---------------------------------------------------------------------- */
/* Cholesky C C': SPRFC2, SPRFS2, SPRBS2                                    */
/* ---------------------------------------------------------------------- */

/* SPRFC2 (sprfc2.f:5-270): MSPAR(1) = 6; on an error MSPAR(27) = SUPEQT. */
void orc_sprfc2_(I *mspar, I *mtrees, I *msifa, double *sm, double *tol,
                 I *iwork, double *rwork, const I *lpu, I *ierr)
{
    (void)iwork;
    (void)rwork;
    (void)lpu;
    if (mspar[0] < 0) {                  /* sprfc2.f:123-127 */
        mspar[0] = -6;
        *ierr = -1;
        return;
    }
    mspar[0] = 6;
    *ierr = 0;
    sym_t s;
    sym_from_mspar(&s, mspar, mtrees, msifa);
    I numneg = 0, supeqt = 0;
    I lierr = oracle_factor_mode(&s, sm, sm + s.neq, tol, &numneg, &supeqt, NULL, 1);
    if (lierr != 0) {                    /* sprfc2.f:244-255 */
        *ierr = (lierr / 10 == -3) ? -3 : -4;
        mspar[26] = supeqt;
    }
    mspar[25] = numneg;
}

/* SPRFS2 / SPRBS2 (sprfs2.f:5-265, sprbs2.f:5-250): MSPAR(1) = 8. */
static void orc_chol_solve(int back, I *mspar, I *mtrees, I *msifa, double *sm, double *b,
                           const I *ldb, const I *nrhs, I *ierr)
{
    if (mspar[0] < 0) {
        mspar[0] = -8;
        *ierr = -1;
        return;
    }
    mspar[0] = 8;
    *ierr = 0;
    sym_t s;
    sym_from_mspar(&s, mspar, mtrees, msifa);
    const double *lnz = sm + s.neq;
    if (mspar[56] == 1 && *ldb < s.neq) s.neq = *ldb;
    if (*ldb < s.neq) {
        mspar[0] = -2;
        *ierr = -2;
        return;
    }
    double *loc = (double *)malloc(sizeof(double) * (size_t)(s.mfront + 1));
    for (I r = 0; r < *nrhs; r++) {
        if (back)
            oracle_backward(&s, lnz, b + r * (*ldb), loc, 1);
        else
            oracle_forward(&s, lnz, b + r * (*ldb), loc, 1);
    }
    free(loc);
}

void orc_sprfs2_(I *mspar, I *mtrees, I *msifa, double *sm, double *b,
                 const I *ldb, const I *nrhs, I *iwork, double *rwork,
                 const I *lpu, I *ierr)
{
    (void)iwork;
    (void)rwork;
    (void)lpu;
    orc_chol_solve(0, mspar, mtrees, msifa, sm, b, ldb, nrhs, ierr);
}

void orc_sprbs2_(I *mspar, I *mtrees, I *msifa, double *sm, double *b,
                 const I *ldb, const I *nrhs, double *rwork, const I *lpu, I *ierr)
{
    (void)rwork;
    (void)lpu;
    orc_chol_solve(1, mspar, mtrees, msifa, sm, b, ldb, nrhs, ierr);
}

/* SPRFC4 (sprfc4.f:5-262): the Cholesky form of SPRFC3.  IERR -3 with
 * MSPAR(27) = -(number replaced) leaves a complete factor; a pivot below
 * -TOL(1)|a_jj| stops it with MSPAR(27) = the equation. */
void orc_sprfc4_(I *mspar, I *mtrees, I *msifa, double *sm, double *tol,
                 I *iwork, double *rwork, double *dcor, const I *lpu, I *ierr)
{
    (void)iwork;
    (void)rwork;
    (void)lpu;
    if (mspar[0] < 0) {                  /* sprfc4.f:133-137 */
        mspar[0] = -6;
        *ierr = -1;
        return;
    }
    mspar[0] = 6;
    *ierr = 0;
    sym_t s;
    sym_from_mspar(&s, mspar, mtrees, msifa);
    I numneg = 0, supeqt = 0;
    I lierr = oracle_factor_mode(&s, sm, sm + s.neq, tol, &numneg, &supeqt, dcor, 1);
    if (lierr != 0) {                    /* sprfc4.f:244-256 */
        *ierr = (lierr / 10 == -3) ? -3 : -4;
        mspar[26] = (lierr == -33) ? -supeqt : supeqt;
    }
    mspar[25] = numneg;
}
