/*
 * oracle/kernel_loops.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement, in IEEE FP64 with OpenMP over target rows, of the f2py
 * Fortran loops of py-lddmm (module `kernelFunctions_fort`, source
 * py-lddmm/kernelFunctions.f90).  Only the parity tests, the smoke check and
 * the CPU-baseline / reference arm of the benchmark load this library; the
 * product path never does.
 *
 * Semantics kept from the Fortran (each function cites the lines it follows):
 *   - `ord > 4` selects the Gaussian kernel, 0..4 the Laplacian (Matern) order;
 *   - the zero-distance branch `ut < 1e-8`, where 1e-8 is a default-real
 *     (float32) literal, i.e. 9.99999993922529e-09 once promoted;
 *   - the polynomial coefficient tables c_, c1_, c2_ hold default-real
 *     literals (1./3, 0.4, 3./7, 1./15, ...), so by default they are the
 *     float32-rounded values; lddmm_oracle_set_exact_coeffs(1) switches to the
 *     exact rationals (what the dense numpy path kernelMatrixLaplacian uses);
 *   - loop order: parallel over targets k, serial over sources l, with the
 *     per-row accumulator `df` summed in source order.
 *
 * Arrays are C-ordered (row-major) exactly as numpy hands them to f2py:
 *   x[k*d + j], beta[l*dimb + c], a1[(i*n + k)*dimb + c], bmat[(k*m + l)*dimb + c].
 *
 * Deliberate deviations (documented, never silently different):
 *   - Laplacian order 0 has no derivative; the Fortran reads c1_(0,.) out of
 *     bounds.  The derivative routines here return -1 for ord == 0, and the
 *     second-derivative routines return -1 for ord in {0, 1} (c2_(ord-1,.)).
 *   - applykdiff11/12 (kernelFunctions.f90:293-428) loop over an undeclared
 *     `num_nodes_y` and a local, never-initialised array `y`; the intended
 *     meaning (y = x, the dense applyDDiffK11/12 at kernelFunctions.py:459-506)
 *     is restated.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define THRESH ((double)1e-8f) /* Fortran default-real literal 1e-8 */

static int g_exact = 0;

void lddmm_oracle_set_exact_coeffs(int exact) { g_exact = exact ? 1 : 0; }
int lddmm_oracle_get_exact_coeffs(void) { return g_exact; }

/* Kernel polynomial tables, indexed by Laplacian order.
 * P[ord][j]: row ord+1 of c_  (kernelFunctions.f90:24-26)  -> K  = P(u) e^-u
 * Q[ord][j]: row ord   of c1_ (kernelFunctions.f90:85-86)  -> K' = -Q(u) e^-u / (2 s^2)
 * R[ord][j]: row ord-1 of c2_ (kernelFunctions.f90:325)    -> K''=  R(u) e^-u / (4 s^4)
 * Both Fortran reshapes are column-major; the rows are transcribed here. */
static void tables(double P[5][5], double Q[5][4], double R[5][3]) {
    memset(P, 0, sizeof(double) * 25);
    memset(Q, 0, sizeof(double) * 20);
    memset(R, 0, sizeof(double) * 15);
    if (g_exact) {
        double p[5][5] = {{1, 0, 0, 0, 0},
                          {1, 1, 0, 0, 0},
                          {1, 1, 1.0 / 3, 0, 0},
                          {1, 1, 0.4, 1.0 / 15, 0},
                          {1, 1, 3.0 / 7, 2.0 / 21, 1.0 / 105}};
        double q[5][4] = {{0, 0, 0, 0},
                          {1, 0, 0, 0},
                          {1.0 / 3, 1.0 / 3, 0, 0},
                          {1.0 / 5, 1.0 / 5, 1.0 / 15, 0},
                          {1.0 / 7, 1.0 / 7, 2.0 / 35, 1.0 / 105}};
        double r[5][3] = {{0, 0, 0}, {0, 0, 0}, {1.0 / 3, 0, 0}, {1.0 / 15, 1.0 / 15, 0},
                          {1.0 / 35, 1.0 / 35, 1.0 / 105}};
        memcpy(P, p, sizeof p);
        memcpy(Q, q, sizeof q);
        memcpy(R, r, sizeof r);
    } else {
        /* float32 division / literal, then widened: what real(8) :: c_ receives */
        double p[5][5] = {{1, 0, 0, 0, 0},
                          {1, 1, 0, 0, 0},
                          {1, 1, (double)(1.0f / 3.0f), 0, 0},
                          {1, 1, (double)0.4f, (double)(1.0f / 15.0f), 0},
                          {1, 1, (double)(3.0f / 7.0f), (double)(2.0f / 21.0f), (double)(1.0f / 105.0f)}};
        double q[5][4] = {{0, 0, 0, 0},
                          {1, 0, 0, 0},
                          {(double)(1.0f / 3.0f), (double)(1.0f / 3.0f), 0, 0},
                          {(double)(1.0f / 5.0f), (double)(1.0f / 5.0f), (double)(1.0f / 15.0f), 0},
                          {(double)(1.0f / 7.0f), (double)(1.0f / 7.0f), (double)(2.0f / 35.0f),
                           (double)(1.0f / 105.0f)}};
        double r[5][3] = {{0, 0, 0},
                          {0, 0, 0},
                          {(double)(1.0f / 3.0f), 0, 0},
                          {(double)(1.0f / 15.0f), (double)(1.0f / 15.0f), 0},
                          {(double)(1.0f / 35.0f), (double)(1.0f / 35.0f), (double)(1.0f / 105.0f)}};
        memcpy(P, p, sizeof p);
        memcpy(Q, q, sizeof q);
        memcpy(R, r, sizeof r);
    }
}

static inline double dist(const double* a, const double* b, int d) {
    double s = 0.0;
    for (int j = 0; j < d; ++j) {
        double t = a[j] - b[j];
        s += t * t;
    }
    return sqrt(s); /* Fortran norm2 */
}

/* K(x,y): kernelFunctions.f90:33-48 */
static inline double kval(double nrm, double sig, int ord, double P[5][5]) {
    double ut = nrm / sig;
    if (ord > 4) {
        ut = ut * ut;
        if (ut < THRESH) return 1.0;
        return exp(-0.5 * ut);
    }
    if (ut < THRESH) return 1.0;
    const double* c = P[ord];
    double lpt = c[0] + c[1] * ut + c[2] * (ut * ut) + c[3] * (ut * ut * ut) + c[4] * (ut * ut * ut * ut);
    return lpt * exp(-1.0 * ut);
}

/* K'(x,y): kernelFunctions.f90:93-108 */
static inline double kdiff(double nrm, double sig, int ord, double Q[5][4]) {
    double ut = nrm / sig;
    if (ord > 4) {
        ut = ut * ut;
        if (ut < THRESH) return -1.0 / (2 * sig * sig);
        return (-1.0) * exp(-0.5 * ut) / (2 * sig * sig);
    }
    const double* c = Q[ord];
    if (ut < THRESH) return -c[0] / (2 * sig * sig);
    double lpt = c[0] + c[1] * ut + c[2] * (ut * ut) + c[3] * (ut * ut * ut);
    return -lpt * exp(-1.0 * ut) / (2 * sig * sig);
}

/* K''(x,y): kernelFunctions.f90:333-352 */
static inline double kdiff2(double nrm, double sig, int ord, double R[5][3]) {
    double ut = nrm / sig;
    double s4 = sig * sig * sig * sig;
    if (ord > 4) {
        ut = ut * ut;
        if (ut < THRESH) return 1.0 / (4 * s4);
        return exp(-0.5 * ut) / (4 * s4);
    }
    const double* c = R[ord];
    if (ut < THRESH) return c[0] / (4 * s4);
    double lpt = c[0] + c[1] * ut + c[2] * (ut * ut);
    return lpt * exp(-1.0 * ut) / (4 * s4);
}

/* applyk: kernelFunctions.f90:1-54.  f[k,:] = sum_l K(x_k, y_l) beta[l,:] */
int lddmm_oracle_applyk(const double* x, const double* y, const double* beta, double sig, int ord, int64_t n,
                        int64_t m, int d, int dimb, double* f) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord < 0) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        double df[64];
        for (int c = 0; c < dimb; ++c) df[c] = 0.0;
        for (int64_t l = 0; l < m; ++l) {
            double kh = kval(dist(x + k * d, y + l * d, d), sig, ord, P);
            for (int c = 0; c < dimb; ++c) df[c] = df[c] + kh * beta[l * dimb + c];
        }
        for (int c = 0; c < dimb; ++c) f[k * dimb + c] = df[c];
    }
    return 0;
}

/* applykdifft: kernelFunctions.f90:56-114.
 * f[k,:] = sum_l K'(x_k,y_l) * 2 (x_k - y_l) * sum_{i,c} a1[i,k,c] a2[i,l,c]
 * The Fortran `sum(a1(:,k,:)*a2(:,l,:))` walks column-major: i fastest. */
int lddmm_oracle_applykdifft(const double* x, const double* y, const double* a1, const double* a2, double sig,
                             int ord, int64_t n, int64_t m, int d, int dimb, int na, double* f) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord == 0 || ord < 0) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        double df[64];
        for (int j = 0; j < d; ++j) df[j] = 0.0;
        for (int64_t l = 0; l < m; ++l) {
            double kd = kdiff(dist(x + k * d, y + l * d, d), sig, ord, Q);
            double s = 0.0;
            for (int c = 0; c < dimb; ++c)
                for (int i = 0; i < na; ++i) s += a1[(i * n + k) * dimb + c] * a2[(i * m + l) * dimb + c];
            for (int j = 0; j < d; ++j) df[j] = df[j] + ((kd * 2) * (x[k * d + j] - y[l * d + j])) * s;
        }
        for (int j = 0; j < d; ++j) f[k * d + j] = df[j];
    }
    return 0;
}

/* applykdiff1: kernelFunctions.f90:116-172.
 * f[k,:] = sum_l K'(x_k,x_l) 2 <x_k - x_l, a1_k> a2_l */
int lddmm_oracle_applykdiff1(const double* x, const double* a1, const double* a2, double sig, int ord, int64_t n,
                             int d, double* f) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord == 0 || ord < 0) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        double df[64];
        for (int j = 0; j < d; ++j) df[j] = 0.0;
        for (int64_t l = 0; l < n; ++l) {
            double kd = kdiff(dist(x + k * d, x + l * d, d), sig, ord, Q);
            double s = 0.0;
            for (int j = 0; j < d; ++j) s += (x[k * d + j] - x[l * d + j]) * a1[k * d + j];
            for (int j = 0; j < d; ++j) df[j] = df[j] + kd * 2 * s * a2[l * d + j];
        }
        for (int j = 0; j < d; ++j) f[k * d + j] = df[j];
    }
    return 0;
}

/* applykdiff2: kernelFunctions.f90:174-230.
 * f[k,:] = -sum_l K'(x_k,x_l) 2 <x_k - x_l, a1_l> a2_l */
int lddmm_oracle_applykdiff2(const double* x, const double* a1, const double* a2, double sig, int ord, int64_t n,
                             int d, double* f) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord == 0 || ord < 0) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        double df[64];
        for (int j = 0; j < d; ++j) df[j] = 0.0;
        for (int64_t l = 0; l < n; ++l) {
            double kd = kdiff(dist(x + k * d, x + l * d, d), sig, ord, Q);
            double s = 0.0;
            for (int j = 0; j < d; ++j) s += (x[k * d + j] - x[l * d + j]) * a1[l * d + j];
            for (int j = 0; j < d; ++j) df[j] = df[j] - kd * 2 * s * a2[l * d + j];
        }
        for (int j = 0; j < d; ++j) f[k * d + j] = df[j];
    }
    return 0;
}

/* applykdiff1and2: kernelFunctions.f90:233-290.
 * f[k,:] = sum_l K'(x_k,x_l) 2 <x_k - x_l, a1_k - a1_l> a2_l */
int lddmm_oracle_applykdiff1and2(const double* x, const double* a1, const double* a2, double sig, int ord,
                                 int64_t n, int d, double* f) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord == 0 || ord < 0) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        double df[64];
        for (int j = 0; j < d; ++j) df[j] = 0.0;
        for (int64_t l = 0; l < n; ++l) {
            double kd = kdiff(dist(x + k * d, x + l * d, d), sig, ord, Q);
            double s = 0.0;
            for (int j = 0; j < d; ++j) s += (x[k * d + j] - x[l * d + j]) * (a1[k * d + j] - a1[l * d + j]);
            for (int j = 0; j < d; ++j) df[j] = df[j] + kd * 2 * s * a2[l * d + j];
        }
        for (int j = 0; j < d; ++j) f[k * d + j] = df[j];
    }
    return 0;
}

/* applykdiff11: kernelFunctions.f90:293-359 (y = x, see header).
 * f[k,:] = sum_l 4 K'' <a1_k,a2_l> <x_k-x_l, p_k> (x_k-x_l) + 2 K' <a1_k,a2_l> p_k */
int lddmm_oracle_applykdiff11(const double* x, const double* a1, const double* a2, const double* p, double sig,
                              int ord, int64_t n, int d, double* f) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord < 2) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        double df[64];
        for (int j = 0; j < d; ++j) df[j] = 0.0;
        for (int64_t l = 0; l < n; ++l) {
            double nrm = dist(x + k * d, x + l * d, d);
            double kd = kdiff(nrm, sig, ord, Q), kd2 = kdiff2(nrm, sig, ord, R);
            double aa = 0.0, xp = 0.0;
            for (int j = 0; j < d; ++j) aa += a1[k * d + j] * a2[l * d + j];
            for (int j = 0; j < d; ++j) xp += (x[k * d + j] - x[l * d + j]) * p[k * d + j];
            for (int j = 0; j < d; ++j)
                df[j] = df[j] + kd2 * 4 * aa * xp * (x[k * d + j] - x[l * d + j]) + kd * 2 * aa * p[k * d + j];
        }
        for (int j = 0; j < d; ++j) f[k * d + j] = df[j];
    }
    return 0;
}

/* applykdiff12: kernelFunctions.f90:361-428 (y = x, see header).
 * f[k,:] = -sum_l 4 K'' <a1_k,a2_l> <x_k-x_l, p_l> (x_k-x_l) - 2 K' <a1_k,a2_l> p_l */
int lddmm_oracle_applykdiff12(const double* x, const double* a1, const double* a2, const double* p, double sig,
                              int ord, int64_t n, int d, double* f) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord < 2) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        double df[64];
        for (int j = 0; j < d; ++j) df[j] = 0.0;
        for (int64_t l = 0; l < n; ++l) {
            double nrm = dist(x + k * d, x + l * d, d);
            double kd = kdiff(nrm, sig, ord, Q), kd2 = kdiff2(nrm, sig, ord, R);
            double aa = 0.0, xp = 0.0;
            for (int j = 0; j < d; ++j) aa += a1[k * d + j] * a2[l * d + j];
            for (int j = 0; j < d; ++j) xp += (x[k * d + j] - x[l * d + j]) * p[l * d + j];
            for (int j = 0; j < d; ++j)
                df[j] = df[j] - kd2 * 4 * aa * xp * (x[k * d + j] - x[l * d + j]) - kd * 2 * aa * p[l * d + j];
        }
        for (int j = 0; j < d; ++j) f[k * d + j] = df[j];
    }
    return 0;
}

/* applykdiff11and12: kernelFunctions.f90:430-496.
 * f[k,:] = sum_l 2 <a1_k,a2_l> (2 K'' <dx,dp> dx + K' dp), dx = x_k-x_l, dp = p_k-p_l */
int lddmm_oracle_applykdiff11and12(const double* x, const double* a1, const double* a2, const double* p,
                                   double sig, int ord, int64_t n, int d, double* f) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord < 2) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        double df[64], dx[64], dp[64];
        for (int j = 0; j < d; ++j) df[j] = 0.0;
        for (int64_t l = 0; l < n; ++l) {
            for (int j = 0; j < d; ++j) {
                dx[j] = x[k * d + j] - x[l * d + j];
                dp[j] = p[k * d + j] - p[l * d + j];
            }
            double nrm = dist(x + k * d, x + l * d, d);
            double kd = kdiff(nrm, sig, ord, Q), kd2 = kdiff2(nrm, sig, ord, R);
            double aa = 0.0, xp = 0.0;
            for (int j = 0; j < d; ++j) aa += a1[k * d + j] * a2[l * d + j];
            for (int j = 0; j < d; ++j) xp += dx[j] * dp[j];
            for (int j = 0; j < d; ++j) df[j] = df[j] + 2 * aa * (2 * kd2 * xp * dx[j] + kd * dp[j]);
        }
        for (int j = 0; j < d; ++j) f[k * d + j] = df[j];
    }
    return 0;
}

/* applykmat: kernelFunctions.f90:499-552.  f[k,:] = sum_l K(x_k,y_l) beta[k,l,:] */
int lddmm_oracle_applykmat(const double* x, const double* y, const double* bmat, double sig, int ord, int64_t n,
                           int64_t m, int d, int dimb, double* f) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord < 0) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        double df[64];
        for (int c = 0; c < dimb; ++c) df[c] = 0.0;
        for (int64_t l = 0; l < m; ++l) {
            double kh = kval(dist(x + k * d, y + l * d, d), sig, ord, P);
            for (int c = 0; c < dimb; ++c) df[c] = df[c] + kh * bmat[(k * m + l) * dimb + c];
        }
        for (int c = 0; c < dimb; ++c) f[k * dimb + c] = df[c];
    }
    return 0;
}

/* applykdiffmat: kernelFunctions.f90:554-610.  f[k,:] = sum_l K'(x_k,y_l) 2 (x_k-y_l) beta[k,l] */
int lddmm_oracle_applykdiffmat(const double* x, const double* y, const double* bmat, double sig, int ord,
                               int64_t n, int64_t m, int d, double* f) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord == 0 || ord < 0) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
        double df[64];
        for (int j = 0; j < d; ++j) df[j] = 0.0;
        for (int64_t l = 0; l < m; ++l) {
            double kd = kdiff(dist(x + k * d, y + l * d, d), sig, ord, Q);
            for (int j = 0; j < d; ++j) df[j] = df[j] + kd * 2 * (x[k * d + j] - y[l * d + j]) * bmat[k * m + l];
        }
        for (int j = 0; j < d; ++j) f[k * d + j] = df[j];
    }
    return 0;
}

/* Varifold data term computed per face pair, with the weights of
 * py-lddmm/surfaces.py:1200-1254 formed on the fly instead of as F x F arrays:
 *   beta_kl = (1 + <n_k,n_l>^2) a_k a_l                                  (:1216-1217, 1244-1245)
 *   u_kl    = (2 <n_k,n_l> n_l - <n_k,n_l>^2 n_k + n_k) a_l                (:1247-1250)
 * Targets k are the faces (c1, n1, a1); sources l are faces (c2, n2, a2).
 * Outputs per target: val[k] = sum_l K beta_kl,  z[k,:] = sum_l K u_kl,
 * dz[k,:] = sum_l K' 2 (c1_k - c2_l) beta_kl.  Any output pointer may be NULL.
 * This is the CPU baseline for the varifold at sizes where the numpy F x F
 * temporaries do not fit; for small F it agrees with the numpy formulas. */
int lddmm_oracle_varifold_pairs(const double* c1, const double* n1, const double* a1, int64_t nf1, const double* c2,
                                const double* n2, const double* a2, int64_t nf2, int d, double sig, int ord,
                                double* val, double* z, double* dz) {
    double P[5][5], Q[5][4], R[5][3];
    if (ord < 0 || ((dz != 0) && ord == 0)) return -1;
    tables(P, Q, R);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nf1; ++k) {
        double v = 0.0, zz[64], dd[64];
        for (int j = 0; j < d; ++j) zz[j] = dd[j] = 0.0;
        for (int64_t l = 0; l < nf2; ++l) {
            double nrm = dist(c1 + k * d, c2 + l * d, d);
            double nn = 0.0;
            for (int j = 0; j < d; ++j) nn += n1[k * d + j] * n2[l * d + j];
            double beta = (1 + nn * nn) * (a1[k] * a2[l]);
            if (val || z) {
                double kh = kval(nrm, sig, ord, P);
                if (val) v += kh * beta;
                if (z)
                    for (int j = 0; j < d; ++j)
                        zz[j] += kh * ((2 * nn * n2[l * d + j] - (nn * nn) * n1[k * d + j] + n1[k * d + j]) * a2[l]);
            }
            if (dz) {
                double kd = kdiff(nrm, sig, ord, Q);
                for (int j = 0; j < d; ++j) dd[j] += kd * 2 * (c1[k * d + j] - c2[l * d + j]) * beta;
            }
        }
        if (val) val[k] = v;
        if (z)
            for (int j = 0; j < d; ++j) z[k * d + j] = zz[j];
        if (dz)
            for (int j = 0; j < d; ++j) dz[k * d + j] = dd[j];
    }
    return 0;
}

int lddmm_oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void lddmm_oracle_set_num_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}
