/*
 * necg_oracle.c -- CPU restatement of the reference NECG energy+gradient path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it as a checker.
 * Nothing in the product path links or calls it.
 *
 * It restates, step by step and in the same order, the reference Python
 * package (MauricioCafiero/NBO_CorrelatedGaussians, directory python/):
 *   f0 / df0        python/utils.py:78-106   (Pade constants python/shared.py:76-86)
 *   vech            python/utils.py:42-55
 *   matel           python/matel.py:28-210
 *   gradel          python/gradel.py:27-392
 *   outprod         python/outprod.py:20-76
 *   make_grad       python/make_grad.py:18-90
 *   _build_matrices python/necg.py:36-58
 *   rrms            python/rrms.py:21-120
 *   dipole loop     python/necg.py:200-244
 * The only liberty taken is that every Kronecker product kron(X, I3) acting on a
 * 3n-vector is written as X acting on the n x 3 matrix view of that vector
 * (row = particle, column = x/y/z); kron(X, I3) has no other entries, so the
 * sums are the same.  Inverses and determinants use LU with partial pivoting,
 * the factorisation numpy.linalg.inv/det use (python/matel.py:93-99).
 *
 * Parity is pinned against golden vectors produced by executing the reference
 * Python (tests/golden/make_golden.py).
 *
 * Layouts (all row-major, FP64):
 *   mass[n][n], ncv[n+1], scvv[nst] (already divided by nst, as
 *   python/read_input.py:141 does), sml[nst][n][n] (= shared.sml[:,:,stf]),
 *   sms[nst][3n][3n], iv[K*blk] with blk = n(n+1)/2 + 3n, x = [iv, C].
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define NX 8 /* largest particle count the oracle handles */

typedef struct {
    int n, nst, K;
    double efs;
    const double *mass, *ncv, *scvv, *sml, *sms;
} OracleProblem;

typedef double Mat[NX][NX];
typedef double Vec3[NX][3]; /* n x 3 view of a 3n vector: v[3i+c] <-> V[i][c] */

static const double C1 = 0.564691197e-04, C2 = 0.758433197e-03, C3 = 0.769838037e-02,
                    C4 = 0.629344460e-01, C5 = 0.213271302e+00, C6 = 0.720266520e-04,
                    C7 = 0.955528842e-03, C8 = 0.101431553e-01, C9 = 0.738522953e-01,
                    C10 = 0.338450368e+00, C11 = 0.879937801e+00;
/* python/shared.py:71 uses math.pi */
static const double PI_ = 3.141592653589793;

/* ---- python/utils.py:78-90 ------------------------------------------------ */
double oracle_f0(double z) {
    if (z <= 16.3578) {
        double num = (((((C1 * z + C2) * z + C3) * z + C4) * z + C5) * z + 1.0);
        double den = ((((((C6 * z + C7) * z + C8) * z + C9) * z + C10) * z + C11) * z + 1.0);
        return sqrt(num / den);
    }
    double r = 2.0 * z;
    return sqrt(PI_ / (2.0 * r));
}

/* ---- python/utils.py:93-106 ----------------------------------------------- */
double oracle_df0(double z) {
    if (z <= 16.3578) {
        double num = (((((C1 * z + C2) * z + C3) * z + C4) * z + C5) * z + 1.0);
        double den = ((((((C6 * z + C7) * z + C8) * z + C9) * z + C10) * z + C11) * z + 1.0);
        double f0v = sqrt(num / den);
        double z2 = z * z, z3 = z2 * z, z4 = z3 * z, z5 = z4 * z, z6 = z5 * z;
        double anum = C1 * z5 + C2 * z4 + C3 * z3 + C4 * z2 + C5 * z + 1.0;
        double aden = C6 * z6 + C7 * z5 + C8 * z4 + C9 * z3 + C10 * z2 + C11 * z + 1.0;
        double danum = 5.0 * C1 * z4 + 4.0 * C2 * z3 + 3.0 * C3 * z2 + 2.0 * C4 * z + C5;
        double daden = 6.0 * C6 * z5 + 5.0 * C7 * z4 + 4.0 * C8 * z3 + 3.0 * C9 * z2 +
                       2.0 * C10 * z + C11;
        return (1.0 / (2.0 * f0v)) * ((aden * danum - anum * daden) / (aden * aden));
    }
    return -sqrt(PI_ / (4.0 * z)) / (2.0 * z);
}

/* ---- small dense helpers -------------------------------------------------- */
static void mm(int n, const Mat a, const Mat b, Mat c) { /* c = a b */
    Mat t;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += a[i][k] * b[k][j];
            t[i][j] = s;
        }
    memcpy(c, t, sizeof(Mat));
}
static void mtr(int n, const Mat a, Mat c) { /* c = a^T */
    Mat t;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) t[i][j] = a[j][i];
    memcpy(c, t, sizeof(Mat));
}
static void mv3(int n, const Mat a, const Vec3 x, Vec3 y) { /* y = kron(a,I3) x */
    Vec3 t;
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += a[i][k] * x[k][c];
            t[i][c] = s;
        }
    memcpy(y, t, sizeof(Vec3));
}
static double dot3(int n, const Vec3 a, const Vec3 b) {
    double s = 0.0;
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) s += a[i][c] * b[i][c];
    return s;
}
/* outer(a, b)[i][j] = sum_c a[i][c] b[j][c]   (dot2 @ dot1 in python/gradel.py) */
static void outer3(int n, const Vec3 a, const Vec3 b, Mat c) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += a[i][k] * b[j][k];
            c[i][j] = s;
        }
}
/* python/utils.py:42-55: column-major lower triangle */
static void vech_add(int n, const Mat a, double coef, double *v) {
    int k = 0;
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) v[k++] += coef * a[i][j];
}

/* LU with partial pivoting (getrf), then inverse by solving A X = I (getrs) and
 * the determinant as sign * prod(U_ii): what numpy.linalg.inv / det compute. */
static int lu_inv_det(int n, const Mat a, Mat inv, double *det) {
    double lu[NX][NX];
    int piv[NX];
    memcpy(lu, a, sizeof(lu));
    double sign = 1.0;
    for (int k = 0; k < n; ++k) {
        int p = k;
        double amax = fabs(lu[k][k]);
        for (int i = k + 1; i < n; ++i)
            if (fabs(lu[i][k]) > amax) { amax = fabs(lu[i][k]); p = i; }
        piv[k] = p;
        if (lu[p][k] == 0.0) return -1;
        if (p != k) {
            for (int j = 0; j < n; ++j) { double t = lu[k][j]; lu[k][j] = lu[p][j]; lu[p][j] = t; }
            sign = -sign;
        }
        for (int i = k + 1; i < n; ++i) {
            lu[i][k] /= lu[k][k];
            for (int j = k + 1; j < n; ++j) lu[i][j] -= lu[i][k] * lu[k][j];
        }
    }
    double d = sign;
    for (int k = 0; k < n; ++k) d *= lu[k][k];
    *det = d;
    for (int col = 0; col < n; ++col) {
        double x[NX];
        for (int i = 0; i < n; ++i) x[i] = (i == col) ? 1.0 : 0.0;
        for (int k = 0; k < n; ++k) { /* apply row interchanges */
            int p = piv[k];
            if (p != k) { double t = x[k]; x[k] = x[p]; x[p] = t; }
        }
        for (int i = 0; i < n; ++i) /* L y = x (unit lower) */
            for (int k = 0; k < i; ++k) x[i] -= lu[i][k] * x[k];
        for (int i = n - 1; i >= 0; --i) { /* U z = y */
            for (int k = i + 1; k < n; ++k) x[i] -= lu[i][k] * x[k];
            x[i] /= lu[i][i];
        }
        for (int i = 0; i < n; ++i) inv[i][col] = x[i];
    }
    return 0;
}

/* Shared preamble of matel/gradel: python/matel.py:56-136, python/gradel.py:46-102 */
typedef struct {
    int n;
    Mat lk, ell, ak, al, akli, aki, mass;
    Vec3 st1, st2, iv1, iv2, ee, st;
    double i1, i2, i3, ov, dett, detak, detal;
    int bad;
} Pair;

static void pair_setup(const OracleProblem *P, const double *iv, int stf, int ii, int jj,
                       int need_aki, Pair *p) {
    const int n = P->n, svh = n * (n + 1) / 2, skp = 3 * n, blk = svh + skp;
    const int s0 = stf - 1, i0 = ii - 1, j0 = jj - 1;
    memset(p, 0, sizeof(*p));
    p->n = n;
    int kk = i0 * blk, ll = j0 * blk; /* python/matel.py:59-66 */
    for (int i = 0; i < n; ++i)
        for (int j = i; j < n; ++j) {
            p->lk[j][i] = iv[kk++];
            p->ell[j][i] = iv[ll++];
        }
    Mat t;
    mtr(n, p->lk, t); mm(n, p->lk, t, p->ak); /* python/matel.py:69-70 */
    mtr(n, p->ell, t); mm(n, p->ell, t, p->al);
    Mat sm, smT, alt; /* python/matel.py:76-77: al = sml^T (al sml) */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) sm[i][j] = P->sml[(size_t)s0 * n * n + i * n + j];
    mm(n, p->al, sm, alt);
    mtr(n, sm, smT);
    mm(n, smT, alt, p->al);
    double s1[3 * NX], s2[3 * NX], s2t[3 * NX]; /* python/matel.py:83-87 */
    for (int k = 0; k < skp; ++k) {
        s1[k] = iv[i0 * blk + svh + k];
        s2[k] = iv[j0 * blk + svh + k];
    }
    const double *S = P->sms + (size_t)s0 * skp * skp;
    for (int r = 0; r < skp; ++r) {
        double s = 0.0;
        for (int c = 0; c < skp; ++c) s += S[r * skp + c] * s2[c];
        s2t[r] = s;
    }
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            p->st1[i][c] = s1[3 * i + c];
            p->st2[i][c] = s2t[3 * i + c];
        }
    Mat akl; /* python/matel.py:92-104 */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) akl[i][j] = p->ak[i][j] + p->al[i][j];
    double det;
    if (lu_inv_det(n, akl, p->akli, &det) != 0) { p->bad = 1; return; }
    p->dett = fabs(det);
    if (need_aki) {
        double dk;
        if (lu_inv_det(n, p->ak, p->aki, &dk) != 0) { p->bad = 1; return; }
    }
    double pk = 1.0, pl = 1.0;
    for (int i = 0; i < n; ++i) { pk *= p->lk[i][i]; pl *= p->ell[i][i]; }
    p->detak = sqrt(fabs(pk * pk));
    p->detal = sqrt(fabs(pl * pl));
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) p->mass[i][j] = P->mass[i * n + j];
    /* overlap, python/matel.py:125-136 */
    mv3(n, p->ak, p->st1, p->iv1);
    p->i1 = dot3(n, p->st1, p->iv1);
    mv3(n, p->al, p->st2, p->iv2);
    p->i2 = dot3(n, p->st2, p->iv2);
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) p->ee[i][c] = p->iv1[i][c] + p->iv2[i][c];
    mv3(n, p->akli, p->ee, p->st);
    p->i3 = dot3(n, p->ee, p->st);
    double r = p->detak * p->detal / p->dett;
    double prefac = sqrt(pow(8.0, n)) * sqrt(r * r * r);
    p->ov = exp(-(p->i1 + p->i2) + p->i3) * prefac;
}

/* Coulomb pair matrix J for (pp, qq), python/matel.py:167-175 */
static void jij_mat(int n, int pp, int qq, Mat j) {
    memset(j, 0, sizeof(Mat));
    if (pp == 0) {
        j[qq - 1][qq - 1] = 1.0;
    } else {
        j[pp - 1][pp - 1] = 1.0;
        j[qq - 1][qq - 1] = 1.0;
        j[pp - 1][qq - 1] = -1.0;
        j[qq - 1][pp - 1] = -1.0;
    }
    (void)n;
}

static double trace(int n, const Mat a) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += a[i][i];
    return s;
}

/* ---- python/matel.py:28-210 ----------------------------------------------- */
int oracle_matel(const OracleProblem *P, const double *iv, int stf, int ii, int jj,
                 double out[4]) {
    Pair p;
    pair_setup(P, iv, stf, ii, jj, 0, &p);
    if (p.bad) return -1;
    const int n = P->n;
    /* kinetic, python/matel.py:144-155 */
    Mat im1, im2;
    Vec3 dif1, dif2, tv;
    mm(n, p.mass, p.al, im1);
    mm(n, p.ak, im1, im2);
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            dif1[i][c] = p.st[i][c] - p.st1[i][c];
            dif2[i][c] = p.st[i][c] - p.st2[i][c];
        }
    mv3(n, im2, dif2, tv);
    double ke_i3 = dot3(n, dif1, tv);
    mm(n, p.akli, p.al, im1);
    mm(n, p.ak, im1, im2);
    mm(n, p.mass, im2, im1);
    double ke_i2 = 3.0 * trace(n, im1); /* trace of kron(X, I3) */
    double tk = 2.0 * p.ov * (2.0 * ke_i3 + ke_i2);
    /* Coulomb, python/matel.py:162-197 */
    double ert = 0.0;
    for (int pp = 0; pp <= n; ++pp)
        for (int qq = pp + 1; qq <= n; ++qq) {
            Mat jij, ism1, jn;
            jij_mat(n, pp, qq, jij);
            mm(n, jij, p.akli, ism1);
            mm(n, p.akli, ism1, jn);
            Vec3 iv3;
            mv3(n, jn, p.ee, iv3);
            double i3e = dot3(n, p.ee, iv3);
            double i2e = trace(n, ism1);
            if (i2e == 0.0) continue;
            double i1e = i3e / i2e;
            ert += P->ncv[pp] * P->ncv[qq] * 2.0 * p.ov * oracle_f0(i1e) / sqrt(i2e * PI_);
        }
    /* Stark, python/matel.py:205-208 */
    double zs = 0.0;
    for (int i = 1; i <= n; ++i) zs += P->ncv[i] * p.st[i - 1][2];
    out[0] = p.ov;
    out[1] = tk;
    out[2] = ert;
    out[3] = p.ov * zs * P->efs;
    return 0;
}

/* ---- python/gradel.py:27-392 ---------------------------------------------- */
int oracle_gradel(const OracleProblem *P, const double *iv, int stf, int ii, int jj,
                  double *tgvl, double *tgvls) {
    Pair p;
    pair_setup(P, iv, stf, ii, jj, 1, &p);
    if (p.bad) return -1;
    const int n = P->n, svh = n * (n + 1) / 2, skp = 3 * n;
    const double ov = p.ov, efs = P->efs;
    Mat m1, m2, m3, t;
    Vec3 dif1, dif2, v1;
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            dif1[i][c] = p.st[i][c] - p.st1[i][c];
            dif2[i][c] = p.st[i][c] - p.st2[i][c];
        }
    /* ogs, python/gradel.py:108 */
    Vec3 ogs;
    mv3(n, p.ak, dif1, ogs);
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) ogs[i][c] *= 2.0 * ov;
    /* ogl, python/gradel.py:114-148 */
    double ogl[NX * (NX + 1) / 2];
    memset(ogl, 0, sizeof(ogl));
    mm(n, p.aki, p.lk, m1);
    vech_add(n, m1, 1.5, ogl);
    mm(n, p.akli, p.lk, m1);
    vech_add(n, m1, -3.0, ogl);
    outer3(n, p.st1, p.st1, m1);
    mm(n, m1, p.lk, m2);
    vech_add(n, m2, -2.0, ogl);
    outer3(n, p.ee, p.ee, m1);
    mm(n, m1, p.akli, m2);
    mm(n, p.akli, m2, m1);
    mm(n, m1, p.lk, m2);
    vech_add(n, m2, -2.0, ogl);
    outer3(n, p.ee, p.st1, m1);
    mm(n, p.akli, m1, m2);
    mm(n, m2, p.lk, m3);
    vech_add(n, m3, 2.0, ogl);
    mtr(n, m2, t);
    mm(n, t, p.lk, m1);
    vech_add(n, m1, 2.0, ogl);
    for (int k = 0; k < svh; ++k) ogl[k] *= ov;
    /* kinetic, python/gradel.py:153-164 */
    mm(n, p.mass, p.al, m1);
    mm(n, p.ak, m1, m2);
    mv3(n, m2, dif2, v1);
    double ke_i3 = dot3(n, dif1, v1);
    mm(n, p.akli, p.al, m1);
    mm(n, p.ak, m1, m2);
    mm(n, p.mass, m2, m1);
    double ke_i2 = 3.0 * trace(n, m1);
    double kfac = 2.0 * ke_i3 + ke_i2;
    /* kgs, python/gradel.py:167-184 */
    Mat al_mass, aklp, aklpt, im1t, im2t, im3t;
    mm(n, p.mass, p.al, al_mass);
    mm(n, p.mass, p.al, m1);
    mm(n, p.ak, m1, aklp);
    mtr(n, aklp, aklpt);
    mm(n, p.akli, p.ak, im1t);
    mm(n, aklp, im1t, im2t);
    mtr(n, im2t, t);
    Vec3 iv2k, iv1k;
    mv3(n, t, dif1, iv2k);
    mm(n, aklpt, im1t, im2t);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) im3t[i][j] = im2t[i][j] - aklpt[i][j];
    mtr(n, im3t, t);
    mv3(n, t, dif2, iv1k);
    Vec3 kgs;
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c)
            kgs[i][c] = 2.0 * kfac * ogs[i][c] + 4.0 * ov * iv2k[i][c] + 4.0 * ov * iv1k[i][c];
    /* kgl, python/gradel.py:187-261 */
    double kgl[NX * (NX + 1) / 2];
    for (int k = 0; k < svh; ++k) kgl[k] = kfac * ogl[k];
    mm(n, p.akli, p.lk, m1);
    mm(n, al_mass, m1, m2);
    mm(n, p.ak, m2, m3);
    mm(n, p.akli, m3, m1);
    vech_add(n, m1, -ov * 6.0, kgl);
    mm(n, p.akli, p.lk, m1);
    mm(n, al_mass, m1, m2);
    vech_add(n, m2, ov * 6.0, kgl);
    Mat sds, sdsk, skdsk, sldsk, slds, aklp_ne, aklpt_ne, kcm, sum;
    outer3(n, p.st, p.st, sds);
    outer3(n, p.st, p.st1, sdsk);
    outer3(n, p.st1, p.st1, skdsk);
    outer3(n, p.st2, p.st1, sldsk);
    outer3(n, p.st2, p.st, slds);
    mm(n, p.ak, al_mass, aklp_ne);
    mtr(n, aklp_ne, aklpt_ne);
    memset(kcm, 0, sizeof(kcm));
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) sum[i][j] = aklp_ne[i][j] + aklpt_ne[i][j];
    Mat ab;
    mm(n, p.akli, sum, ab); /* akli (aklp + aklpt) */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) t[i][j] = al_mass[i][j] - ab[i][j];
    mm(n, t, sds, m1); /* term 1 */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) kcm[i][j] += m1[i][j];
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) t[i][j] = ab[i][j] - al_mass[i][j];
    mm(n, t, sdsk, m1); /* term 2 */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) kcm[i][j] += m1[i][j];
    Mat akl_aklpt, akl_aklp, sdskT;
    mm(n, p.akli, aklpt_ne, akl_aklpt);
    mtr(n, sdsk, sdskT);
    mm(n, akl_aklpt, sdskT, m1); /* term 3 */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) kcm[i][j] += m1[i][j];
    mm(n, p.akli, aklp_ne, akl_aklp);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) t[i][j] = akl_aklp[i][j] - al_mass[i][j];
    mm(n, t, slds, m1); /* term 4 */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) kcm[i][j] += m1[i][j];
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) t[i][j] = al_mass[i][j] - akl_aklp[i][j];
    mm(n, t, sldsk, m1); /* term 5 */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) kcm[i][j] += m1[i][j];
    mm(n, akl_aklpt, skdsk, m1); /* term 6 */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) kcm[i][j] -= m1[i][j];
    mm(n, kcm, p.lk, m1);
    vech_add(n, m1, 2.0 * ov, kgl);
    mtr(n, kcm, t);
    mm(n, t, p.lk, m1);
    vech_add(n, m1, 2.0 * ov, kgl);
    for (int k = 0; k < svh; ++k) kgl[k] *= 2.0;
    /* Coulomb gradients, python/gradel.py:266-337 */
    Vec3 ergst;
    double erglt[NX * (NX + 1) / 2];
    memset(ergst, 0, sizeof(ergst));
    memset(erglt, 0, sizeof(erglt));
    for (int pp = 0; pp <= n; ++pp)
        for (int qq = pp + 1; qq <= n; ++qq) {
            Mat jij, ism1, jn, jb;
            jij_mat(n, pp, qq, jij);
            mm(n, jij, p.akli, ism1);
            mm(n, p.akli, ism1, jn);
            Vec3 iv3;
            mv3(n, jn, p.ee, iv3);
            double i3e = dot3(n, p.ee, iv3);
            double i2e = trace(n, ism1);
            if (i2e == 0.0) continue;
            double i1e = i3e / i2e;
            const double qq2 = P->ncv[pp] * P->ncv[qq];
            const double f0v = oracle_f0(i1e), df0v = oracle_df0(i1e);
            mm(n, p.ak, jn, jb); /* akb @ jijb */
            Vec3 iv3t;
            mv3(n, jb, p.ee, iv3t);
            for (int i = 0; i < n; ++i)
                for (int c = 0; c < 3; ++c)
                    ergst[i][c] += (qq2 * 2.0 * f0v / sqrt(i2e * PI_)) * ogs[i][c] +
                                   qq2 * 4.0 * ov * df0v * iv3t[i][c] /
                                       sqrt(PI_ * i2e * i2e * i2e);
            double ergl[NX * (NX + 1) / 2];
            memset(ergl, 0, sizeof(ergl));
            Mat ijl;
            mm(n, jn, p.lk, ijl);
            const double a1 = 2.0 * f0v / sqrt(i2e * PI_);
            const double a2 = 2.0 * ov * f0v / sqrt(PI_ * i2e * i2e * i2e);
            for (int k = 0; k < svh; ++k) ergl[k] = a1 * ogl[k];
            vech_add(n, ijl, a2, ergl);
            vech_add(n, ijl, 4.0 * ov * df0v * i3e / sqrt(PI_ * pow(i2e, 5)), ergl);
            const double c3 = 4.0 * ov * df0v / sqrt(PI_ * i2e * i2e * i2e);
            /* m2 term */
            Mat e2, a, b;
            outer3(n, p.ee, p.ee, e2);
            mm(n, p.akli, e2, a);
            mm(n, a, jn, b);
            mm(n, b, p.lk, a);
            vech_add(n, a, -c3, ergl);
            mtr(n, b, t);
            mm(n, t, p.lk, a);
            vech_add(n, a, -c3, ergl);
            /* m1 term */
            outer3(n, p.st1, p.ee, e2);
            mm(n, e2, jn, b);
            mm(n, b, p.lk, a);
            vech_add(n, a, c3, ergl);
            mtr(n, b, t);
            mm(n, t, p.lk, a);
            vech_add(n, a, c3, ergl);
            for (int k = 0; k < svh; ++k) erglt[k] += qq2 * ergl[k];
        }
    /* Stark gradients, python/gradel.py:342-370 */
    Vec3 zgs;
    memset(zgs, 0, sizeof(zgs));
    Mat imz;
    mm(n, p.ak, p.akli, imz);
    for (int i = 1; i <= n; ++i)
        for (int a = 0; a < n; ++a)
            for (int c = 0; c < 3; ++c) {
                double col = (c == 2) ? imz[a][i - 1] : 0.0; /* column 3i-1 of kron */
                zgs[a][c] += P->ncv[i] * (ogs[a][c] * p.st[i - 1][2] + ov * col) * efs;
            }
    double zgl[NX * (NX + 1) / 2];
    memset(zgl, 0, sizeof(zgl));
    for (int kk = 1; kk <= n; ++kk) {
        Mat z1, z2, zt;
        memset(z1, 0, sizeof(z1));
        for (int a = 0; a < n; ++a) z1[a][kk - 1] = p.st1[a][2] - p.st[a][2];
        mm(n, z1, p.akli, z2);
        mm(n, z2, p.lk, z2);
        double v1z[NX * (NX + 1) / 2], v2z[NX * (NX + 1) / 2];
        memset(v1z, 0, sizeof(v1z));
        memset(v2z, 0, sizeof(v2z));
        vech_add(n, z2, 1.0, v1z);
        mtr(n, z1, zt);
        mm(n, p.akli, zt, z2);
        mm(n, z2, p.lk, z2);
        vech_add(n, z2, 1.0, v2z);
        for (int k = 0; k < svh; ++k)
            zgl[k] += P->ncv[kk] * efs * (p.st[kk - 1][2] * ogl[k] + ov * (v1z[k] + v2z[k]));
    }
    /* assembly, python/gradel.py:377-390 */
    const double dbl = (ii == jj) ? 2.0 : 1.0;
    for (int k = 0; k < svh; ++k) {
        tgvl[k] = dbl * (kgl[k] + erglt[k] - zgl[k]);
        tgvls[k] = dbl * ogl[k];
    }
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            tgvl[svh + 3 * i + c] = dbl * (kgs[i][c] + ergst[i][c] - zgs[i][c]);
            tgvls[svh + 3 * i + c] = dbl * ogs[i][c];
        }
    (void)skp;
    return 0;
}

/* ---- H/S build (python/outprod.py:46-60, python/necg.py:36-58) ----------------
 * Rows i = row0, row0+stride, ... (1-based, the row-cyclic split of
 * source/outprod.f90:34).  Kin/Pot may be NULL. */
int oracle_build_rows(const OracleProblem *P, const double *iv, int row0, int stride,
                      double *H, double *S, double *Kin, double *Pot) {
    const int K = P->K;
    for (int i = row0; i <= K; i += stride)
        for (int j = 1; j <= i; ++j)
            for (int stf = 1; stf <= P->nst; ++stf) {
                double o[4];
                if (oracle_matel(P, iv, stf, i, j, o)) return -1;
                const double w = P->scvv[stf - 1];
                const size_t ij = (size_t)(i - 1) * K + (j - 1);
                H[ij] += w * (o[1] + o[2] - o[3]);
                S[ij] += w * o[0];
                if (Kin) Kin[ij] += w * o[1];
                if (Pot) Pot[ij] += w * o[2];
            }
    return 0;
}

/* DH/DS columns for bra rows l (python/make_grad.py:37-55).  dh, ds are
 * (siv x K) row-major. */
int oracle_grad_rows(const OracleProblem *P, const double *iv, int row0, int stride,
                     double *dh, double *ds) {
    const int n = P->n, K = P->K, blk = n * (n + 1) / 2 + 3 * n;
    double tg[NX * (NX + 1) / 2 + 3 * NX], tgs[NX * (NX + 1) / 2 + 3 * NX];
    for (int l = row0; l <= K; l += stride)
        for (int k = 1; k <= K; ++k) {
            double acc[NX * (NX + 1) / 2 + 3 * NX] = {0}, accs[NX * (NX + 1) / 2 + 3 * NX] = {0};
            for (int stf = 1; stf <= P->nst; ++stf) {
                if (oracle_gradel(P, iv, stf, l, k, tg, tgs)) return -1;
                const double w = P->scvv[stf - 1];
                for (int i = 0; i < blk; ++i) { acc[i] += w * tg[i]; accs[i] += w * tgs[i]; }
            }
            for (int i = 0; i < blk; ++i) {
                dh[(size_t)((l - 1) * blk + i) * K + (k - 1)] = acc[i];
                ds[(size_t)((l - 1) * blk + i) * K + (k - 1)] = accs[i];
            }
        }
    return 0;
}

/* ---- python/rrms.py:21-120 ------------------------------------------------ */
/* Overlap and the full position vector st = akli ee of one (stfe, stf, ii, jj)
 * term: the symmetry maps are applied to the ket (stf) and to the bra (stfe).
 * rrms returns (ov, st[n1 - 1] ov). */
static int rrms_pair(const OracleProblem *P, const double *iv, int stfe, int stf, int ii, int jj,
                     double *ov, double st[3 * NX]) {
    const int n = P->n, svh = n * (n + 1) / 2, skp = 3 * n, blk = svh + skp;
    const int se = stfe - 1, s0 = stf - 1, i0 = ii - 1, j0 = jj - 1;
    Mat lk, ell, ak, al, t, sm, smT, tmp;
    memset(lk, 0, sizeof(Mat));
    memset(ell, 0, sizeof(Mat));
    int kk = i0 * blk, ll = j0 * blk; /* python/rrms.py:52-58 */
    for (int i = 0; i < n; ++i)
        for (int j = i; j < n; ++j) {
            lk[j][i] = iv[kk++];
            ell[j][i] = iv[ll++];
        }
    mtr(n, lk, t); mm(n, lk, t, ak); /* python/rrms.py:60-61 */
    mtr(n, ell, t); mm(n, ell, t, al);
    for (int i = 0; i < n; ++i) /* ket: al = sml^T (al sml), python/rrms.py:64-65 */
        for (int j = 0; j < n; ++j) sm[i][j] = P->sml[(size_t)s0 * n * n + i * n + j];
    mm(n, al, sm, tmp); mtr(n, sm, smT); mm(n, smT, tmp, al);
    for (int i = 0; i < n; ++i) /* bra: ak = sml_e^T (ak sml_e), python/rrms.py:68-69 */
        for (int j = 0; j < n; ++j) sm[i][j] = P->sml[(size_t)se * n * n + i * n + j];
    mm(n, ak, sm, tmp); mtr(n, sm, smT); mm(n, smT, tmp, ak);
    double s1[3 * NX], s2[3 * NX], s1t[3 * NX], s2t[3 * NX]; /* python/rrms.py:72-79 */
    for (int k = 0; k < skp; ++k) {
        s1[k] = iv[i0 * blk + svh + k];
        s2[k] = iv[j0 * blk + svh + k];
    }
    const double *Se = P->sms + (size_t)se * skp * skp, *Sk = P->sms + (size_t)s0 * skp * skp;
    for (int r = 0; r < skp; ++r) {
        double a = 0.0, b = 0.0;
        for (int c = 0; c < skp; ++c) {
            a += Sk[r * skp + c] * s2[c];
            b += Se[r * skp + c] * s1[c];
        }
        s2t[r] = a;
        s1t[r] = b;
    }
    Vec3 st1, st2, iv1, iv2, ee, stv;
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            st1[i][c] = s1t[3 * i + c];
            st2[i][c] = s2t[3 * i + c];
        }
    Mat akl, akli; /* python/rrms.py:82-90 */
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) akl[i][j] = ak[i][j] + al[i][j];
    double det;
    if (lu_inv_det(n, akl, akli, &det) != 0) return -1;
    const double dett = fabs(det);
    double pk = 1.0, pl = 1.0;
    for (int i = 0; i < n; ++i) { pk *= lk[i][i]; pl *= ell[i][i]; }
    const double detak = sqrt(fabs(pk * pk)), detal = sqrt(fabs(pl * pl));
    mv3(n, ak, st1, iv1); /* overlap, python/rrms.py:101-116 */
    const double i1 = dot3(n, st1, iv1);
    mv3(n, al, st2, iv2);
    const double i2 = dot3(n, st2, iv2);
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) ee[i][c] = iv1[i][c] + iv2[i][c];
    mv3(n, akli, ee, stv);
    const double i3 = dot3(n, ee, stv);
    const double r = detak * detal / dett;
    const double prefac = sqrt(pow(8.0, n)) * sqrt(r * r * r);
    *ov = exp(-(i1 + i2) + i3) * prefac;
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) st[3 * i + c] = stv[i][c];
    return 0;
}

int oracle_rrms(const OracleProblem *P, const double *iv, int stfe, int stf, int ii, int jj, int n1,
                double out[2]) {
    double ov, st[3 * NX];
    if (rrms_pair(P, iv, stfe, stf, ii, jj, &ov, st)) return -1;
    out[0] = ov;
    out[1] = st[n1 - 1] * ov; /* python/rrms.py:118-120 */
    return 0;
}

/* Lower triangles of the dipole matrices of python/necg.py:205-218 for bra
 * rows j = row0, row0 + stride, ...: hd[(m * K + j - 1) * K + i - 1] for each
 * component m (the loop's kk - 1) and sd[(j - 1) * K + i - 1].  The reference
 * calls rrms once per component with the same (ov, st); here one pair
 * evaluation serves every component. */
int oracle_dipole_rows(const OracleProblem *P, const double *iv, int row0, int stride, double *hd,
                       double *sd) {
    const int K = P->K, nst = P->nst, m3 = 3 * P->n;
    for (int j = row0; j <= K; j += stride)
        for (int i = 1; i <= j; ++i)
            for (int stfe = 1; stfe <= nst; ++stfe)
                for (int stf = 1; stf <= nst; ++stf) {
                    double ov, st[3 * NX];
                    if (rrms_pair(P, iv, stfe, stf, j, i, &ov, st)) return -1;
                    const double w = P->scvv[stf - 1] * P->scvv[stfe - 1];
                    const size_t ji = (size_t)(j - 1) * K + (i - 1);
                    for (int m = 0; m < m3; ++m) hd[(size_t)m * K * K + ji] += w * st[m] * ov;
                    sd[ji] += w * ov;
                }
    return 0;
}

typedef struct {
    const OracleProblem *P;
    const double *iv;
    int row0, stride, which, rc;
    double *a, *b, *c, *d;
} Job;

static void *job_run(void *arg) {
    Job *j = (Job *)arg;
    if (j->which == 0)
        j->rc = oracle_build_rows(j->P, j->iv, j->row0, j->stride, j->a, j->b, j->c, j->d);
    else if (j->which == 2)
        j->rc = oracle_dipole_rows(j->P, j->iv, j->row0, j->stride, j->a, j->b);
    else
        j->rc = oracle_grad_rows(j->P, j->iv, j->row0, j->stride, j->a, j->b);
    return NULL;
}

/* Row-cyclic threaded run of one loop; each thread owns private outputs that
 * are summed afterwards (the MPI_REDUCE of source/outprod.f90:44-45). */
static int run_threads(const OracleProblem *P, const double *iv, int which, int nthreads,
                       size_t len, double *a, double *b, double *c, double *d) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > P->K) nthreads = P->K;
    Job *jobs = (Job *)calloc(nthreads, sizeof(Job));
    pthread_t *tid = (pthread_t *)calloc(nthreads, sizeof(pthread_t));
    double **priv = (double **)calloc((size_t)nthreads * 4, sizeof(double *));
    int rc = 0;
    for (int t = 0; t < nthreads; ++t) {
        jobs[t].P = P; jobs[t].iv = iv; jobs[t].row0 = t + 1; jobs[t].stride = nthreads;
        jobs[t].which = which;
        double *outs[4] = {a, b, c, d};
        double **dst[4] = {&jobs[t].a, &jobs[t].b, &jobs[t].c, &jobs[t].d};
        for (int q = 0; q < 4; ++q) {
            if (!outs[q]) { *dst[q] = NULL; continue; }
            if (t == 0) { *dst[q] = outs[q]; continue; }
            priv[t * 4 + q] = (double *)calloc(len, sizeof(double));
            *dst[q] = priv[t * 4 + q];
        }
        if (t > 0) pthread_create(&tid[t], NULL, job_run, &jobs[t]);
    }
    job_run(&jobs[0]);
    for (int t = 1; t < nthreads; ++t) pthread_join(tid[t], NULL);
    for (int t = 0; t < nthreads; ++t) {
        if (jobs[t].rc) rc = jobs[t].rc;
        if (t == 0) continue;
        double *outs[4] = {a, b, c, d};
        for (int q = 0; q < 4; ++q) {
            if (!priv[t * 4 + q]) continue;
            for (size_t i = 0; i < len; ++i) outs[q][i] += priv[t * 4 + q][i];
            free(priv[t * 4 + q]);
        }
    }
    free(jobs); free(tid); free(priv);
    return rc;
}

/* ---- python/necg.py:36-58 ------------------------------------------------- */
int oracle_build_matrices(const OracleProblem *P, const double *iv, int nthreads, double *H,
                          double *S, double *Kin, double *Pot) {
    const int K = P->K;
    const size_t kk = (size_t)K * K;
    memset(H, 0, kk * sizeof(double));
    memset(S, 0, kk * sizeof(double));
    if (Kin) memset(Kin, 0, kk * sizeof(double));
    if (Pot) memset(Pot, 0, kk * sizeof(double));
    int rc = run_threads(P, iv, 0, nthreads, kk, H, S, Kin, Pot);
    for (int j = 0; j < K; ++j) /* python/necg.py:53-58 */
        for (int i = 0; i < j; ++i) {
            H[(size_t)i * K + j] = H[(size_t)j * K + i];
            S[(size_t)i * K + j] = S[(size_t)j * K + i];
            if (Kin) Kin[(size_t)i * K + j] = Kin[(size_t)j * K + i];
            if (Pot) Pot[(size_t)i * K + j] = Pot[(size_t)j * K + i];
        }
    return rc;
}

/* ---- python/outprod.py:20-76 + python/make_grad.py:18-90 ------------------
 * x = [iv, C] (siv + K); returns f, writes g (siv + K), H, S (K x K). */
int oracle_outprod(const OracleProblem *P, const double *x, int nthreads, double *f,
                   double *g, double *H, double *S) {
    const int n = P->n, K = P->K, blk = n * (n + 1) / 2 + 3 * n;
    const size_t siv = (size_t)K * blk;
    const double *iv = x, *C = x + siv;
    int rc = oracle_build_matrices(P, iv, nthreads, H, S, NULL, NULL);
    if (rc) return rc;
    double cHc = 0.0, cSc = 0.0; /* python/outprod.py:65-68 */
    for (int i = 0; i < K; ++i) {
        double h = 0.0, s = 0.0;
        for (int j = 0; j < K; ++j) {
            h += H[(size_t)i * K + j] * C[j];
            s += S[(size_t)i * K + j] * C[j];
        }
        cHc += C[i] * h;
        cSc += C[i] * s;
    }
    const double eng = cHc / cSc, norm = 1.0 / cSc;
    *f = eng;
    double *dh = (double *)calloc(siv * K, sizeof(double));
    double *ds = (double *)calloc(siv * K, sizeof(double));
    if (!dh || !ds) { free(dh); free(ds); return -2; }
    rc = run_threads(P, iv, 1, nthreads, siv * K, dh, ds, NULL, NULL);
    /* GRADA, python/make_grad.py:61-79 */
    for (int j = 1; j <= K; ++j)
        for (int k = 1; k <= blk; ++k) {
            const size_t ic = (size_t)(j - 1) * blk + k - 1;
            double val = 0.0;
            for (int i = 1; i <= K; ++i) {
                const double gm = norm * (dh[ic * K + (i - 1)] - eng * ds[ic * K + (i - 1)]);
                if (i != j) val += 2.0 * C[i - 1] * C[j - 1] * gm;
                else val += C[i - 1] * C[j - 1] * gm;
            }
            g[ic] = val;
        }
    /* GRADC, python/make_grad.py:85 */
    for (int i = 0; i < K; ++i) {
        double s = 0.0;
        for (int j = 0; j < K; ++j)
            s += (H[(size_t)i * K + j] - eng * S[(size_t)i * K + j]) * C[j];
        g[siv + i] = 2.0 * norm * s;
    }
    free(dh); free(ds);
    return rc;
}

/* Time-sampling helper for the CPU baseline: evaluates the listed matel and
 * gradel terms (1-based stf, ii, jj triples) and returns a checksum. */
double oracle_sample_terms(const OracleProblem *P, const double *iv, int nmat,
                           const int *mat_terms, int ngrad, const int *grad_terms) {
    double acc = 0.0, o[4];
    double tg[NX * (NX + 1) / 2 + 3 * NX], tgs[NX * (NX + 1) / 2 + 3 * NX];
    for (int t = 0; t < nmat; ++t) {
        oracle_matel(P, iv, mat_terms[3 * t], mat_terms[3 * t + 1], mat_terms[3 * t + 2], o);
        acc += o[0] + o[1];
    }
    for (int t = 0; t < ngrad; ++t) {
        oracle_gradel(P, iv, grad_terms[3 * t], grad_terms[3 * t + 1], grad_terms[3 * t + 2],
                      tg, tgs);
        acc += tg[0] + tgs[0];
    }
    return acc;
}

/* ---- python/necg.py:200-244 (dipole) --------------------------------------- */
/* comps[m] = C^T Hd_m C / C^T Sd C (0 if C^T Sd C = 0) with the matrices
 * symmetrised from their lower triangles; dip[c] = sum_i ncv[i] comps[3(i-1)+c]. */
int oracle_dipole(const OracleProblem *P, const double *iv, const double *C, int nthreads,
                  double *comps, double *dip) {
    const int K = P->K, n = P->n, m3 = 3 * n;
    const size_t kk = (size_t)K * K, len = (size_t)m3 * kk;
    double *hd = (double *)calloc(len, sizeof(double));
    double *sd = (double *)calloc(len, sizeof(double)); /* run_threads sums len entries */
    if (!hd || !sd) { free(hd); free(sd); return -2; }
    int rc = run_threads(P, iv, 2, nthreads, len, hd, sd, NULL, NULL);
    if (rc) { free(hd); free(sd); return rc; }
    for (int j = 0; j < K; ++j) /* symmetrise, python/necg.py:221-224 */
        for (int i = 0; i < j; ++i) {
            sd[(size_t)i * K + j] = sd[(size_t)j * K + i];
            for (int m = 0; m < m3; ++m) hd[m * kk + (size_t)i * K + j] = hd[m * kk + (size_t)j * K + i];
        }
    double cSc = 0.0;
    for (int a = 0; a < K; ++a) {
        double r = 0.0;
        for (int b = 0; b < K; ++b) r += sd[(size_t)a * K + b] * C[b];
        cSc += C[a] * r;
    }
    for (int c = 0; c < 3; ++c) dip[c] = 0.0;
    for (int m = 0; m < m3; ++m) {
        double cHc = 0.0;
        for (int a = 0; a < K; ++a) {
            double r = 0.0;
            for (int b = 0; b < K; ++b) r += hd[m * kk + (size_t)a * K + b] * C[b];
            cHc += C[a] * r;
        }
        comps[m] = cSc != 0.0 ? cHc / cSc : 0.0;
        dip[m % 3] += P->ncv[m / 3 + 1] * comps[m];
    }
    free(hd);
    free(sd);
    return 0;
}
