/*
 * qcu_oracle.c -- CPU restatement (test infrastructure only; see qcu_oracle.h).
 *
 * The hop is written from the operator definition with explicit 4x4 Dirac
 * matrices in the DeGrand-Rossi basis, not from the reference's projector
 * tables, so that the two formulations check each other:
 *   reference projector tables  include/kernel/complex_matmul.cuh:16-227, 503-600
 *   reference gamma table        include/kernel/qcu_gamma.cuh:10-18, 70-76, 126-132, 185-191
 *   reference neighbour rule     include/point/qcu_point.cuh:16-61
 *   reference link addressing    include/point/qcu_point.cuh:68-70
 *   reference hop sum            include/kernel/su_n_m_rhs_dslash.cuh:92-105
 */
#include "qcu_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;

static int g_threads = 0;

void oracle_set_threads(int n) {
    g_threads = n;
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}

int oracle_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Dirac matrices gamma_1..gamma_4 (index mu = 0..3 for x, y, z, t), DR basis. */
static void gamma_matrix(int mu, cplx g[4][4]) {
    memset(g, 0, sizeof(cplx) * 16);
    const cplx im = _Complex_I;
    switch (mu) {
        case 0: g[0][3] = im;  g[1][2] = im;  g[2][1] = -im; g[3][0] = -im; break;
        case 1: g[0][3] = -1;  g[1][2] = 1;   g[2][1] = 1;   g[3][0] = -1;  break;
        case 2: g[0][2] = im;  g[1][3] = -im; g[2][0] = -im; g[3][1] = im;  break;
        default: g[0][2] = 1; g[1][3] = 1;  g[2][0] = 1;  g[3][1] = 1;  break;
    }
}

/* projector P = 1 + sgn * gamma_mu */
static void projector(int mu, int sgn, cplx P[4][4]) {
    cplx g[4][4];
    gamma_matrix(mu, g);
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) P[a][b] = (a == b ? 1.0 : 0.0) + sgn * g[a][b];
}

static inline long half_index(int xh, int y, int z, int t, const int L[4]) {
    return (((long)t * L[2] + z) * L[1] + y) * (L[0] / 2) + xh;
}

static inline void half_coords(long idx, const int L[4], int* xh, int* y, int* z, int* t) {
    int lxh = L[0] / 2;
    *xh = (int)(idx % lxh);
    idx /= lxh;
    *y = (int)(idx % L[1]);
    idx /= L[1];
    *z = (int)(idx % L[2]);
    *t = (int)(idx / L[2]);
}

/* neighbour of full-lattice site in direction mu, dir = +1/-1, returned as half index
 * of the opposite parity; *wrap_t set when the hop crosses the t boundary. */
static long neighbour(int x, int y, int z, int t, int mu, int dir, const int L[4], int* wrap_t) {
    int c[4] = {x, y, z, t};
    c[mu] += dir;
    *wrap_t = 0;
    if (c[mu] < 0) { c[mu] += L[mu]; if (mu == 3) *wrap_t = 1; }
    if (c[mu] >= L[mu]) { c[mu] -= L[mu]; if (mu == 3) *wrap_t = 1; }
    return half_index(c[0] / 2, c[1], c[2], c[3], L);
}

void oracle_hop_mrhs(double* out_d, const double* in_d, const double* gauge_d, const int L[4],
                     int nc, int m, int parity, int dagger, double t_sign) {
    const long vh = (long)L[0] * L[1] * L[2] * L[3] / 2;
    const cplx* in = (const cplx*)in_d;
    const cplx* gauge = (const cplx*)gauge_d;
    cplx* out = (cplx*)out_d;
    const int s = dagger ? -1 : 1;
    cplx Pf[4][4][4], Pb[4][4][4];
    for (int mu = 0; mu < 4; ++mu) {
        projector(mu, -s, Pf[mu]); /* forward:  1 - s*gamma */
        projector(mu, +s, Pb[mu]); /* backward: 1 + s*gamma */
    }
    const long site_len = 4L * nc * m;
#pragma omp parallel
    {
        cplx* proj = (cplx*)malloc(sizeof(cplx) * site_len);
        cplx* acc = (cplx*)malloc(sizeof(cplx) * site_len);
#pragma omp for schedule(static)
        for (long idx = 0; idx < vh; ++idx) {
            int xh, y, z, t;
            half_coords(idx, L, &xh, &y, &z, &t);
            const int x = 2 * xh + ((parity + y + z + t) & 1);
            memset(acc, 0, sizeof(cplx) * site_len);
            for (int mu = 0; mu < 4; ++mu) {
                for (int d = 0; d < 2; ++d) {
                    const int dir = d == 0 ? +1 : -1;
                    int wrap;
                    const long nb = neighbour(x, y, z, t, mu, dir, L, &wrap);
                    const cplx(*P)[4] = d == 0 ? Pf[mu] : Pb[mu];
                    const cplx* psi = in + nb * site_len;
                    /* projected spinor (P psi)[a][c'][r] */
                    for (int a = 0; a < 4; ++a)
                        for (int cc = 0; cc < nc; ++cc)
                            for (int r = 0; r < m; ++r) {
                                cplx v = 0;
                                for (int b = 0; b < 4; ++b)
                                    if (P[a][b] != 0) v += P[a][b] * psi[((long)b * nc + cc) * m + r];
                                proj[((long)a * nc + cc) * m + r] = v;
                            }
                    /* link: forward U_mu(x) (parity p, index idx);
                     *       backward U_mu(x-mu)^dag (parity 1-p, index nb) */
                    const cplx* U = d == 0 ? gauge + (((long)mu * 2 + parity) * vh + idx) * nc * nc
                                           : gauge + (((long)mu * 2 + (1 - parity)) * vh + nb) * nc * nc;
                    const double f = wrap ? t_sign : 1.0;
                    for (int a = 0; a < 4; ++a)
                        for (int c = 0; c < nc; ++c)
                            for (int cc = 0; cc < nc; ++cc) {
                                const cplx u = d == 0 ? U[c * nc + cc] : conj(U[cc * nc + c]);
                                const cplx fu = f * u;
                                const cplx* pr = proj + ((long)a * nc + cc) * m;
                                cplx* ac = acc + ((long)a * nc + c) * m;
                                for (int r = 0; r < m; ++r) ac[r] += fu * pr[r];
                            }
                }
            }
            memcpy(out + idx * site_len, acc, sizeof(cplx) * site_len);
        }
        free(proj);
        free(acc);
    }
}

void oracle_gather(double* mrhs_d, const double* per_rhs_d, long vh, int nc, int m) {
    cplx* mrhs = (cplx*)mrhs_d;
    const cplx* src = (const cplx*)per_rhs_d;
    const long sl = 4L * nc;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < vh; ++i)
        for (int r = 0; r < m; ++r)
            for (long e = 0; e < sl; ++e) mrhs[(i * sl + e) * m + r] = src[((long)r * vh + i) * sl + e];
}

void oracle_scatter(double* per_rhs_d, const double* mrhs_d, long vh, int nc, int m) {
    const cplx* mrhs = (const cplx*)mrhs_d;
    cplx* dst = (cplx*)per_rhs_d;
    const long sl = 4L * nc;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < vh; ++i)
        for (int r = 0; r < m; ++r)
            for (long e = 0; e < sl; ++e) dst[((long)r * vh + i) * sl + e] = mrhs[(i * sl + e) * m + r];
}

void oracle_mat(double* out_d, const double* in_d, const double* gauge, const int L[4], int nc,
                int m, double kappa, int dagger, double t_sign) {
    const long vh = (long)L[0] * L[1] * L[2] * L[3] / 2;
    const long sl = 4L * nc;
    const long half = vh * sl * m; /* complex elements of one parity, all RHS */
    double* gin = (double*)malloc(sizeof(double) * 2 * half);
    double* gout = (double*)malloc(sizeof(double) * 2 * half);
    double* tmp = (double*)malloc(sizeof(double) * 2 * half);
    const cplx* in = (const cplx*)in_d;
    cplx* out = (cplx*)out_d;
    for (int p = 0; p < 2; ++p) {
        /* gather input parity 1-p of every RHS */
        for (int r = 0; r < m; ++r)
            memcpy(tmp + 2 * (long)r * vh * sl, in + ((long)r * 2 + (1 - p)) * vh * sl,
                   sizeof(cplx) * vh * sl);
        oracle_gather(gin, tmp, vh, nc, m);
        oracle_hop_mrhs(gout, gin, gauge, L, nc, m, p, dagger, t_sign);
        oracle_scatter(tmp, gout, vh, nc, m);
        for (int r = 0; r < m; ++r) {
            const cplx* d = (const cplx*)(tmp + 2 * (long)r * vh * sl);
            const cplx* src = in + ((long)r * 2 + p) * vh * sl;
            cplx* o = out + ((long)r * 2 + p) * vh * sl;
            for (long e = 0; e < vh * sl; ++e) o[e] = src[e] - kappa * d[e];
        }
    }
    free(gin);
    free(gout);
    free(tmp);
}

void oracle_schur(double* out_d, const double* in_d, double* tmp, const double* gauge,
                  const int L[4], int nc, int m, double kappa, double t_sign) {
    const long vh = (long)L[0] * L[1] * L[2] * L[3] / 2;
    const long n = vh * 4L * nc * m;
    oracle_hop_mrhs(tmp, in_d, gauge, L, nc, m, 0, 0, t_sign);   /* tmp_e = D_eo in_o */
    oracle_hop_mrhs(out_d, tmp, gauge, L, nc, m, 1, 0, t_sign);  /* out_o = D_oe tmp_e */
    cplx* out = (cplx*)out_d;
    const cplx* in = (const cplx*)in_d;
    const double k2 = kappa * kappa;
#pragma omp parallel for schedule(static)
    for (long e = 0; e < n; ++e) out[e] = in[e] - k2 * out[e];
}

/* ---------------- multi-RHS BLAS (reference src/qcu_blas/qcu_complex_*.cu) ---------------- */

void oracle_dotc(double* res_d, const double* a_d, const double* b_d, long len, int m) {
    const cplx* a = (const cplx*)a_d;
    const cplx* b = (const cplx*)b_d;
    cplx* res = (cplx*)res_d;
    for (int j = 0; j < m; ++j) {
        double re = 0, im = 0;
#pragma omp parallel for reduction(+ : re, im) schedule(static)
        for (long i = 0; i < len; ++i) {
            const cplx v = conj(a[i * m + j]) * b[i * m + j];
            re += creal(v);
            im += cimag(v);
        }
        res[j] = re + im * _Complex_I;
    }
}

void oracle_norm(double* res, const double* a_d, long len, int m) {
    const cplx* a = (const cplx*)a_d;
    for (int j = 0; j < m; ++j) {
        double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (long i = 0; i < len; ++i) {
            const cplx v = a[i * m + j];
            s += creal(v) * creal(v) + cimag(v) * cimag(v);
        }
        res[j] = sqrt(s);
    }
}

void oracle_xsay(double* res_d, const double* x_d, const double* a_d, const double* y_d, long len, int m) {
    cplx* res = (cplx*)res_d;
    const cplx *x = (const cplx*)x_d, *a = (const cplx*)a_d, *y = (const cplx*)y_d;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < len; ++i)
        for (int j = 0; j < m; ++j) res[i * m + j] = x[i * m + j] - a[j] * y[i * m + j];
}

void oracle_xpay(double* res_d, const double* x_d, const double* a_d, const double* y_d, long len, int m) {
    cplx* res = (cplx*)res_d;
    const cplx *x = (const cplx*)x_d, *a = (const cplx*)a_d, *y = (const cplx*)y_d;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < len; ++i)
        for (int j = 0; j < m; ++j) res[i * m + j] = x[i * m + j] + a[j] * y[i * m + j];
}

void oracle_axpby(double* res_d, const double* a_d, const double* x_d, const double* b_d,
                  const double* y_d, long len, int m) {
    cplx* res = (cplx*)res_d;
    const cplx *a = (const cplx*)a_d, *x = (const cplx*)x_d, *b = (const cplx*)b_d, *y = (const cplx*)y_d;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < len; ++i)
        for (int j = 0; j < m; ++j) res[i * m + j] = a[j] * x[i * m + j] + b[j] * y[i * m + j];
}

void oracle_axpbypcz(double* res_d, const double* a_d, const double* x_d, const double* b_d,
                     const double* y_d, const double* c_d, const double* z_d, long len, int m) {
    cplx* res = (cplx*)res_d;
    const cplx *a = (const cplx*)a_d, *x = (const cplx*)x_d, *b = (const cplx*)b_d;
    const cplx *y = (const cplx*)y_d, *c = (const cplx*)c_d, *z = (const cplx*)z_d;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < len; ++i)
        for (int j = 0; j < m; ++j)
            res[i * m + j] = a[j] * x[i * m + j] + b[j] * y[i * m + j] + c[j] * z[i * m + j];
}

/* ---------------- BiCGStab, policy 1 ---------------- */

int oracle_bicgstab(double* x_d, const double* b_d, const double* gauge, const int L[4], int nc,
                    int m, double kappa, double t_sign, int max_iter, double tol, double* rel_resid) {
    const long vh = (long)L[0] * L[1] * L[2] * L[3] / 2;
    const long len = vh * 4L * nc;  /* complex elements per RHS, one parity */
    const long n = len * m;         /* complex elements, one parity, all RHS */
    const size_t bytes = sizeof(cplx) * n;
    const cplx* b = (const cplx*)b_d;
    cplx* x = (cplx*)x_d;
    const cplx* b_e = b;
    const cplx* b_o = b + n;
    cplx* x_e = x;
    cplx* x_o = x + n;

    cplx *bp = malloc(bytes), *r0 = malloc(bytes), *r = malloc(bytes), *p = malloc(bytes);
    cplx *v = malloc(bytes), *s = malloc(bytes), *t = malloc(bytes), *tmp = malloc(bytes);
    cplx* xo = malloc(bytes);
    cplx *rho = malloc(sizeof(cplx) * m), *alpha = malloc(sizeof(cplx) * m);
    cplx *omega = malloc(sizeof(cplx) * m), *beta = malloc(sizeof(cplx) * m);
    cplx *d1 = malloc(sizeof(cplx) * m), *d2 = malloc(sizeof(cplx) * m);
    cplx *kap = malloc(sizeof(cplx) * m), *one = malloc(sizeof(cplx) * m);
    double *nb = malloc(sizeof(double) * m), *nr = malloc(sizeof(double) * m);
    for (int j = 0; j < m; ++j) { kap[j] = kappa; one[j] = 1.0; }

    /* b' = b_o + kappa D_oe b_e   (bicgstab.cu:141-189) */
    oracle_hop_mrhs((double*)tmp, (const double*)b_e, gauge, L, nc, m, 1, 0, t_sign);
    oracle_xpay((double*)bp, (const double*)b_o, (const double*)kap, (const double*)tmp, len, m);
    oracle_norm(nb, (const double*)bp, len, m);

    memset(xo, 0, bytes);
    memcpy(r0, bp, bytes);
    memcpy(r, bp, bytes);
    memcpy(p, bp, bytes);

    int it, converged = 0;
    for (it = 0; it < max_iter; ++it) {
        oracle_dotc((double*)rho, (const double*)r0, (const double*)r, len, m);
        oracle_schur((double*)v, (const double*)p, (double*)tmp, gauge, L, nc, m, kappa, t_sign);
        oracle_dotc((double*)d1, (const double*)r0, (const double*)v, len, m);
        for (int j = 0; j < m; ++j) alpha[j] = rho[j] / d1[j];
        oracle_xsay((double*)s, (const double*)r, (const double*)alpha, (const double*)v, len, m);
        oracle_schur((double*)t, (const double*)s, (double*)tmp, gauge, L, nc, m, kappa, t_sign);
        oracle_dotc((double*)d1, (const double*)t, (const double*)s, len, m);
        oracle_dotc((double*)d2, (const double*)t, (const double*)t, len, m);
        for (int j = 0; j < m; ++j) omega[j] = d1[j] / d2[j];
        oracle_axpbypcz((double*)xo, (const double*)one, (const double*)xo, (const double*)alpha,
                        (const double*)p, (const double*)omega, (const double*)s, len, m);
        oracle_xsay((double*)r, (const double*)s, (const double*)omega, (const double*)t, len, m);
        oracle_norm(nr, (const double*)r, len, m);
        converged = 1;
        for (int j = 0; j < m; ++j)
            if (nr[j] / nb[j] > tol) converged = 0;
        if (converged) { ++it; break; }
        oracle_dotc((double*)d1, (const double*)r0, (const double*)r, len, m); /* rho_new */
        for (int j = 0; j < m; ++j) beta[j] = (alpha[j] * d1[j] / omega[j]) / rho[j];
        /* p = r + beta (p - omega v) */
        oracle_xsay((double*)tmp, (const double*)p, (const double*)omega, (const double*)v, len, m);
        oracle_xpay((double*)p, (const double*)r, (const double*)beta, (const double*)tmp, len, m);
    }
    if (rel_resid)
        for (int j = 0; j < m; ++j) rel_resid[j] = nr[j] / nb[j];

    /* x_o and reconstruction x_e = b_e + kappa D_eo x_o  (bicgstab_solve.cu:688-740) */
    memcpy(x_o, xo, bytes);
    oracle_hop_mrhs((double*)tmp, (const double*)x_o, gauge, L, nc, m, 0, 0, t_sign);
    oracle_xpay((double*)x_e, (const double*)b_e, (const double*)kap, (const double*)tmp, len, m);

    free(bp); free(r0); free(r); free(p); free(v); free(s); free(t); free(tmp); free(xo);
    free(rho); free(alpha); free(omega); free(beta); free(d1); free(d2); free(kap); free(one);
    free(nb); free(nr);
    return converged ? it : -1;
}

/* ---------------- even/odd reorder ---------------- */

static void reorder_sites(double* dst_d, const double* src_d, const int L[4], long site_len, int to_eo) {
    const long V = (long)L[0] * L[1] * L[2] * L[3];
    const long vh = V / 2;
    cplx* dst = (cplx*)dst_d;
    const cplx* src = (const cplx*)src_d;
#pragma omp parallel for schedule(static)
    for (long lex = 0; lex < V; ++lex) {
        long q = lex;
        const int x = (int)(q % L[0]); q /= L[0];
        const int y = (int)(q % L[1]); q /= L[1];
        const int z = (int)(q % L[2]);
        const int t = (int)(q / L[2]);
        const int par = (x + y + z + t) & 1;
        const long eo = par * vh + half_index(x / 2, y, z, t, L);
        if (to_eo)
            memcpy(dst + eo * site_len, src + lex * site_len, sizeof(cplx) * site_len);
        else
            memcpy(dst + lex * site_len, src + eo * site_len, sizeof(cplx) * site_len);
    }
}

void oracle_gauge_to_eo(double* eo, const double* lex, const int L[4], int nc) {
    const long V = (long)L[0] * L[1] * L[2] * L[3];
    const long blk = V * nc * nc;
    for (int mu = 0; mu < 4; ++mu)
        reorder_sites(eo + 2 * mu * blk, lex + 2 * mu * blk, L, (long)nc * nc, 1);
}

void oracle_gauge_from_eo(double* lex, const double* eo, const int L[4], int nc) {
    const long V = (long)L[0] * L[1] * L[2] * L[3];
    const long blk = V * nc * nc;
    for (int mu = 0; mu < 4; ++mu)
        reorder_sites(lex + 2 * mu * blk, eo + 2 * mu * blk, L, (long)nc * nc, 0);
}

void oracle_fermion_to_eo(double* eo, const double* lex, const int L[4], int nc) {
    reorder_sites(eo, lex, L, 4L * nc, 1);
}

void oracle_fermion_from_eo(double* lex, const double* eo, const int L[4], int nc) {
    reorder_sites(lex, eo, L, 4L * nc, 0);
}

/* ---------------- parallel-transport convolution (learned preconditioner layer) ----------------
 * Path k: 0 identity, 1 + 2 mu: U_mu(x) f(x + mu), 2 + 2 mu: U_mu(x - mu)^dag f(x - mu).
 * Fields are gathered full-lattice multi-RHS spinors [ch][2][Vh][4][nc][m]. */

static int ptc_opposite(int k) { return k == 0 ? 0 : (((k - 1) & 1) ? k - 1 : k + 1); }

/* (T_k f)(x) for every spin, colour and RHS of site x = (parity, idx) of one channel */
static void ptc_transport(cplx* res, const cplx* f, const cplx* gauge, const int L[4], int nc, int m,
                          int parity, long idx, int k, double t_sign) {
    const long vh = (long)L[0] * L[1] * L[2] * L[3] / 2;
    const long site_len = 4L * nc * m;
    if (k == 0) {
        memcpy(res, f + ((long)parity * vh + idx) * site_len, sizeof(cplx) * site_len);
        return;
    }
    const int mu = (k - 1) >> 1, fwd = ((k - 1) & 1) == 0;
    int xh, y, z, t;
    half_coords(idx, L, &xh, &y, &z, &t);
    const int x = 2 * xh + ((parity + y + z + t) & 1);
    int wrap;
    const long nb = neighbour(x, y, z, t, mu, fwd ? +1 : -1, L, &wrap);
    const cplx* link = fwd ? gauge + (((long)mu * 2 + parity) * vh + idx) * nc * nc
                           : gauge + (((long)mu * 2 + (1 - parity)) * vh + nb) * nc * nc;
    const cplx* src = f + ((long)(1 - parity) * vh + nb) * site_len;
    const double sg = wrap ? t_sign : 1.0;
    for (int s = 0; s < 4; ++s)
        for (int c = 0; c < nc; ++c)
            for (int r = 0; r < m; ++r) {
                cplx acc = 0;
                for (int cc = 0; cc < nc; ++cc) {
                    const cplx u = fwd ? link[c * nc + cc] : conj(link[cc * nc + c]);
                    acc += u * src[((long)s * nc + cc) * m + r];
                }
                res[((long)s * nc + c) * m + r] = sg * acc;
            }
}

void oracle_ptc_forward(double* out_d, const double* in_d, const double* w_d, const double* gauge_d,
                        const int L[4], int nc, int m, int cin, int cout, double t_sign) {
    const long vh = (long)L[0] * L[1] * L[2] * L[3] / 2;
    const long site_len = 4L * nc * m, field = 2 * vh * site_len;
    const cplx* in = (const cplx*)in_d;
    const cplx* w = (const cplx*)w_d;
    const cplx* gauge = (const cplx*)gauge_d;
    cplx* out = (cplx*)out_d;
#pragma omp parallel
    {
        cplx* tr = (cplx*)malloc(sizeof(cplx) * site_len);
#pragma omp for schedule(static)
        for (long site = 0; site < 2 * vh; ++site) {
            const int parity = (int)(site / vh);
            const long idx = site % vh;
            for (int o = 0; o < cout; ++o) memset(out + o * field + site * site_len, 0, sizeof(cplx) * site_len);
            for (int i = 0; i < cin; ++i)
                for (int k = 0; k < 9; ++k) {
                    ptc_transport(tr, in + i * field, gauge, L, nc, m, parity, idx, k, t_sign);
                    for (int o = 0; o < cout; ++o) {
                        const cplx* W = w + (((long)o * cin + i) * 9 + k) * 16;
                        cplx* dst = out + o * field + site * site_len;
                        for (int sp = 0; sp < 4; ++sp)
                            for (int s = 0; s < 4; ++s) {
                                const cplx ws = W[sp * 4 + s];
                                if (ws == 0) continue;
                                for (long e = 0; e < (long)nc * m; ++e) dst[sp * nc * m + e] += ws * tr[s * nc * m + e];
                            }
                    }
                }
        }
        free(tr);
    }
}

void oracle_ptc_adjoint(double* gin_d, const double* gout_d, const double* w_d, const double* gauge_d,
                        const int L[4], int nc, int m, int cin, int cout, double t_sign) {
    const long vh = (long)L[0] * L[1] * L[2] * L[3] / 2;
    const long site_len = 4L * nc * m, field = 2 * vh * site_len;
    const cplx* gout = (const cplx*)gout_d;
    const cplx* w = (const cplx*)w_d;
    const cplx* gauge = (const cplx*)gauge_d;
    cplx* gin = (cplx*)gin_d;
#pragma omp parallel
    {
        cplx* tr = (cplx*)malloc(sizeof(cplx) * site_len);
#pragma omp for schedule(static)
        for (long site = 0; site < 2 * vh; ++site) {
            const int parity = (int)(site / vh);
            const long idx = site % vh;
            for (int i = 0; i < cin; ++i) memset(gin + i * field + site * site_len, 0, sizeof(cplx) * site_len);
            for (int o = 0; o < cout; ++o)
                for (int k = 0; k < 9; ++k) {
                    /* T_k^dag = T_opposite(k); the spin matrix enters conjugate-transposed */
                    ptc_transport(tr, gout + o * field, gauge, L, nc, m, parity, idx, ptc_opposite(k), t_sign);
                    for (int i = 0; i < cin; ++i) {
                        const cplx* W = w + (((long)o * cin + i) * 9 + k) * 16;
                        cplx* dst = gin + i * field + site * site_len;
                        for (int s = 0; s < 4; ++s)
                            for (int sp = 0; sp < 4; ++sp) {
                                const cplx ws = conj(W[sp * 4 + s]);
                                if (ws == 0) continue;
                                for (long e = 0; e < (long)nc * m; ++e) dst[s * nc * m + e] += ws * tr[sp * nc * m + e];
                            }
                    }
                }
        }
        free(tr);
    }
}

void oracle_ptc_wgrad(double* gw_d, const double* gout_d, const double* in_d, const double* gauge_d,
                      const int L[4], int nc, int m, int cin, int cout, double t_sign) {
    const long vh = (long)L[0] * L[1] * L[2] * L[3] / 2;
    const long site_len = 4L * nc * m, field = 2 * vh * site_len;
    const cplx* gout = (const cplx*)gout_d;
    const cplx* in = (const cplx*)in_d;
    const cplx* gauge = (const cplx*)gauge_d;
    cplx* gw = (cplx*)gw_d;
    const long nw = (long)cout * cin * 9;
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nw; ++q) {
        const int k = (int)(q % 9), i = (int)((q / 9) % cin), o = (int)(q / (9L * cin));
        cplx acc[16] = {0};
        cplx* tr = (cplx*)malloc(sizeof(cplx) * site_len);
        for (long site = 0; site < 2 * vh; ++site) {
            ptc_transport(tr, in + i * field, gauge, L, nc, m, (int)(site / vh), site % vh, k, t_sign);
            const cplx* g = gout + o * field + site * site_len;
            for (int sp = 0; sp < 4; ++sp)
                for (int s = 0; s < 4; ++s) {
                    cplx a = 0;
                    for (long e = 0; e < (long)nc * m; ++e) a += g[sp * nc * m + e] * conj(tr[s * nc * m + e]);
                    acc[sp * 4 + s] += a;
                }
        }
        free(tr);
        for (int e = 0; e < 16; ++e) gw[q * 16 + e] = acc[e];
    }
}
