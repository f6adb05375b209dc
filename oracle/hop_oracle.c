/*
 * hop_oracle.c -- CPU oracle for the Wilson hopping matrix (TEST
 * INFRASTRUCTURE ONLY: used by tests/, by __graft_entry__.smoke() and by the
 * CPU-baseline leg of bench.py as the checker; never linked into the product
 * library and never on the product path).
 *
 * An independent restatement, in gather form, of the reference's plain-C
 * hopping pair:
 *   - H_eo: lib/dirac.c:35-408   (plqcd_hopping_matrix_eo_sse3_assymbly)
 *   - H_oe: lib/dirac.c:414-791  (plqcd_hopping_matrix_oe_sse3_assymbly)
 * The reference scatters projected half-spinors into phip/phim buffers and
 * then gathers them (four passes, lib/dirac.c:81-116, 143-196, 260-319,
 * 365-399). Here every output site reads its 8 neighbours directly; the
 * arithmetic per term is the same:
 *   forward  (neighbour x+mu):  chi  = U_mu(x)       * h,  h  = upper((1 -/+ ...) psi(x+mu))
 *   backward (neighbour x-mu):  chi' = U_mu(x-mu)^dag * h', h' = upper(... psi(x-mu))
 * with the projection and reconstruction signs of lib/dirac.c:95-114 and
 * 163-195 (projection), 269-311 and 371-398 (reconstruction), i.e. the
 * macros of include/su3.h:187-207, 233-254 and 298-307.
 *
 * Site order follows lib/start.c:406-433 (lexicographic x fastest, even
 * sites -- sum of coordinates even -- first) and the periodic neighbour
 * tables of lib/start.c:439-526 for a single process.
 *
 * compat=1 reproduces the reference as shipped, bug for bug:
 *   - include/su3.h:135-138 `_vector_minus_assign` is an assignment r = -s,
 *     used at lib/dirac.c:373-374 and 756-757 as if it subtracted; the lower
 *     spin components s2/s3 lose every forward contribution and restart
 *     from -chi'(mu=0).
 *   - lib/dirac.c:643 takes the forward links of odd output site j from
 *     u[4*(j-V/2)+mu] instead of u[4*j+mu].
 *
 * Field layout (the reference's API layout, include/su3.h:52-75):
 *   spinor: 12 complex doubles per site, index 3*spin + colour
 *   su3:     9 complex doubles per link, row-major c00..c22; link (i,mu)
 *            at u[4*i + mu] with i the even/odd site index.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;

/* ------------------------------------------------------------------ */
/* geometry (lib/start.c:406-526, nprocs = 1)                          */
/* ------------------------------------------------------------------ */

static long lex_of(const int L[4], const int x[4])
{
    return x[0] + (long)L[0] * (x[1] + (long)L[1] * (x[2] + (long)L[2] * x[3]));
}

static void cart_of(const int L[4], long ix, int x[4])
{
    x[0] = (int)(ix % L[0]); ix /= L[0];
    x[1] = (int)(ix % L[1]); ix /= L[1];
    x[2] = (int)(ix % L[2]); ix /= L[2];
    x[3] = (int)ix;
}

/* ipt_eo[V], ipt_lex[V], iup[4V], idn[4V] (index 4*i+mu). */
void orc_geometry(const int L[4], int *ipt_eo, int *ipt_lex, int *iup, int *idn)
{
    long V = (long)L[0] * L[1] * L[2] * L[3];
    long ce = 0, co = V / 2;
    int x[4];
    for (long ix = 0; ix < V; ix++) {
        cart_of(L, ix, x);
        int par = (x[0] + x[1] + x[2] + x[3]) & 1;
        long e = par ? co++ : ce++;
        ipt_eo[ix] = (int)e;
        ipt_lex[e] = (int)ix;
    }
    for (long i = 0; i < V; i++) {
        cart_of(L, ipt_lex[i], x);
        for (int mu = 0; mu < 4; mu++) {
            int y[4] = {x[0], x[1], x[2], x[3]};
            y[mu] = (x[mu] + 1) % L[mu];
            iup[4 * i + mu] = ipt_eo[lex_of(L, y)];
            y[mu] = (x[mu] + L[mu] - 1) % L[mu];
            idn[4 * i + mu] = ipt_eo[lex_of(L, y)];
        }
    }
}

/* ------------------------------------------------------------------ */
/* SU(3) x colour vector                                               */
/* ------------------------------------------------------------------ */

static inline void su3_mul(cplx r[3], const cplx *u, const cplx s[3])
{
    for (int a = 0; a < 3; a++)
        r[a] = u[3 * a + 0] * s[0] + u[3 * a + 1] * s[1] + u[3 * a + 2] * s[2];
}

static inline void su3_dag_mul(cplx r[3], const cplx *u, const cplx s[3])
{
    for (int a = 0; a < 3; a++)
        r[a] = conj(u[0 * 3 + a]) * s[0] + conj(u[1 * 3 + a]) * s[1] + conj(u[2 * 3 + a]) * s[2];
}

/*
 * One output site. out = 12 complex; psi indexed by even/odd site (full
 * array of V spinors); links at u[9*(4*i+mu)].
 * fwd_link_site[mu] / bwd_link_site[mu]: even/odd index of the site whose
 * link is used (normally i itself and idn[i][mu]).
 */
static void site_hop(cplx *out, const cplx *psi, const cplx *u, const int nbr_up[4],
                     const int nbr_dn[4], const long fwd_link_site[4], int compat)
{
    cplx r[4][3];
    cplx h0[3], h1[3], c0[3], c1[3];
    memset(r, 0, sizeof r);
    const cplx I_ = I;

    /* forward terms, lib/dirac.c:95-114 (projection) and 269-311 (rebuild) */
    for (int mu = 0; mu < 4; mu++) {
        const cplx *s = psi + 12 * (long)nbr_up[mu];
        const cplx *s0 = s, *s1 = s + 3, *s2 = s + 6, *s3 = s + 9;
        for (int c = 0; c < 3; c++) {
            switch (mu) {
            case 0: h0[c] = s0[c] + s2[c];       h1[c] = s1[c] + s3[c];       break;
            case 1: h0[c] = s0[c] + I_ * s3[c];  h1[c] = s1[c] + I_ * s2[c];  break;
            case 2: h0[c] = s0[c] + s3[c];       h1[c] = s1[c] - s2[c];       break;
            default: h0[c] = s0[c] + I_ * s2[c]; h1[c] = s1[c] - I_ * s3[c];  break;
            }
        }
        const cplx *U = u + 9 * (4 * fwd_link_site[mu] + mu);
        su3_mul(c0, U, h0);
        su3_mul(c1, U, h1);
        for (int c = 0; c < 3; c++) {
            r[0][c] += c0[c];
            r[1][c] += c1[c];
            switch (mu) {
            case 0: r[2][c] += c0[c];        r[3][c] += c1[c];        break;
            case 1: r[2][c] -= I_ * c1[c];   r[3][c] -= I_ * c0[c];   break;
            case 2: r[2][c] -= c1[c];        r[3][c] += c0[c];        break;
            default: r[2][c] -= I_ * c0[c];  r[3][c] += I_ * c1[c];   break;
            }
        }
    }

    /* backward terms, lib/dirac.c:163-195 (projection, U^dag) and 371-398 */
    for (int mu = 0; mu < 4; mu++) {
        const cplx *s = psi + 12 * (long)nbr_dn[mu];
        const cplx *s0 = s, *s1 = s + 3, *s2 = s + 6, *s3 = s + 9;
        for (int c = 0; c < 3; c++) {
            switch (mu) {
            case 0: h0[c] = s0[c] - s2[c];       h1[c] = s1[c] - s3[c];       break;
            case 1: h0[c] = s0[c] - I_ * s3[c];  h1[c] = s1[c] - I_ * s2[c];  break;
            case 2: h0[c] = s0[c] - s3[c];       h1[c] = s1[c] + s2[c];       break;
            default: h0[c] = s0[c] - I_ * s2[c]; h1[c] = s1[c] + I_ * s3[c];  break;
            }
        }
        const cplx *U = u + 9 * (4 * (long)nbr_dn[mu] + mu);
        su3_dag_mul(c0, U, h0);
        su3_dag_mul(c1, U, h1);
        for (int c = 0; c < 3; c++) {
            r[0][c] += c0[c];
            r[1][c] += c1[c];
            switch (mu) {
            case 0:
                if (compat) { r[2][c] = -c0[c]; r[3][c] = -c1[c]; }
                else        { r[2][c] -= c0[c]; r[3][c] -= c1[c]; }
                break;
            case 1: r[2][c] += I_ * c1[c];   r[3][c] += I_ * c0[c];   break;
            case 2: r[2][c] += c1[c];        r[3][c] -= c0[c];        break;
            default: r[2][c] += I_ * c0[c];  r[3][c] -= I_ * c1[c];   break;
            }
        }
    }
    for (int sp = 0; sp < 4; sp++)
        for (int c = 0; c < 3; c++)
            out[3 * sp + c] = r[sp][c];
}

/* Shared driver: out_parity 0 -> eo (writes [0,V/2) from odd input),
 * out_parity 1 -> oe (writes [V/2,V) from even input). */
static void hop_parity(const int L[4], const double *qin, double *qout, const double *u,
                       int out_parity, int compat, int nthreads)
{
    long V = (long)L[0] * L[1] * L[2] * L[3];
    int *ipt_eo = malloc(sizeof(int) * V), *ipt_lex = malloc(sizeof(int) * V);
    int *iup = malloc(sizeof(int) * 4 * V), *idn = malloc(sizeof(int) * 4 * V);
    orc_geometry(L, ipt_eo, ipt_lex, iup, idn);
    const cplx *psi = (const cplx *)qin;
    const cplx *uu = (const cplx *)u;
    cplx *out = (cplx *)qout;
    long base = out_parity ? V / 2 : 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (long k = 0; k < V / 2; k++) {
        long i = base + k;
        long fls[4];
        for (int mu = 0; mu < 4; mu++)
            fls[mu] = (compat && out_parity == 1) ? (i - V / 2) : i;
        site_hop(out + 12 * i, psi, uu, iup + 4 * i, idn + 4 * i, fls, compat);
    }
    (void)nthreads;
    free(ipt_eo); free(ipt_lex); free(iup); free(idn);
}

void orc_hop_eo(const int L[4], const double *qin, double *qout, const double *u, int compat, int nthreads)
{
    hop_parity(L, qin, qout, u, 0, compat, nthreads);
}

void orc_hop_oe(const int L[4], const double *qin, double *qout, const double *u, int compat, int nthreads)
{
    hop_parity(L, qin, qout, u, 1, compat, nthreads);
}

/* ------------------------------------------------------------------ */
/* Even/odd preconditioned Wilson operator and FP64 CG (no reference     */
/* counterpart: include/plqcd_global_params.h:197-201 leaves operator    */
/* and solver parameters as placeholders).                               */
/*   D = 1 - kappa H,  Mhat = 1 - kappa^2 H_eo H_oe on even sites,       */
/*   Mhat^dag = g5 Mhat g5 with g5 = diag(1,1,-1,-1).                    */
/* Even fields are V/2 spinors stored in the even half of full arrays.   */
/* ------------------------------------------------------------------ */

static void g5_half(cplx *f, long n)
{
    for (long i = 0; i < n; i++)
        for (int k = 6; k < 12; k++) f[12 * i + k] = -f[12 * i + k];
}

/* out_e = Mhat in_e (dagger: g5 Mhat g5). tmp: full-lattice scratch. */
static void mhat(const int L[4], const double *u, const cplx *in, cplx *out, cplx *tmp,
                 double kappa, int dagger, int nthreads)
{
    long V = (long)L[0] * L[1] * L[2] * L[3];
    long Vh = V / 2;
    cplx *a = tmp, *b = tmp + 12 * V;
    memcpy(a, in, sizeof(cplx) * 12 * Vh);
    if (dagger) g5_half(a, Vh);
    orc_hop_oe(L, (const double *)a, (double *)b, u, 0, nthreads);   /* b_o = H_oe a_e */
    orc_hop_eo(L, (const double *)b, (double *)a, u, 0, nthreads);   /* a_e = H_eo b_o */
    double k2 = kappa * kappa;
    /* Mhat a = a - k2 H_eo H_oe a; for the dagger a = g5 in and the result
     * is g5 (Mhat a) = in - k2 g5 (H_eo H_oe g5 in). */
    for (long i = 0; i < 12 * Vh; i++)
        out[i] = in[i] - k2 * ((dagger && (i % 12) >= 6) ? -a[i] : a[i]);
}

static double dot_re(const cplx *a, const cplx *b, long n)
{
    double s = 0;
    for (long i = 0; i < n; i++) s += creal(conj(a[i]) * b[i]);
    return s;
}

/*
 * Apply the full Wilson operator D = 1 - kappa H to a full-lattice field.
 */
void orc_wilson(const int L[4], const double *u, const double *in, double *out, double kappa, int nthreads)
{
    long V = (long)L[0] * L[1] * L[2] * L[3];
    cplx *h = malloc(sizeof(cplx) * 12 * V);
    orc_hop_eo(L, in, (double *)h, u, 0, nthreads);
    orc_hop_oe(L, in, (double *)h, u, 0, nthreads);
    const cplx *x = (const cplx *)in;
    cplx *o = (cplx *)out;
    for (long i = 0; i < 12 * V; i++) o[i] = x[i] - kappa * h[i];
    free(h);
}

/*
 * Solve D x = b (full lattice) by CG on Mhat^dag Mhat for the even part,
 * then reconstruct the odd part. Returns the iteration count; *relres gets
 * the final true relative residual |b - D x| / |b| on the full lattice.
 */
int orc_cg_solve(const int L[4], const double *u, const double *b_in, double *x_out, double kappa,
                 double tol, int maxiter, double *relres, int nthreads)
{
    long V = (long)L[0] * L[1] * L[2] * L[3];
    long Vh = V / 2, n = 12 * Vh;
    const cplx *b = (const cplx *)b_in;
    cplx *x = (cplx *)x_out;
    cplx *tmp = calloc(24 * V, sizeof(cplx));
    cplx *be = malloc(sizeof(cplx) * n), *rhs = malloc(sizeof(cplx) * n);
    cplx *r = malloc(sizeof(cplx) * n), *p = malloc(sizeof(cplx) * n);
    cplx *Ap = malloc(sizeof(cplx) * n), *t = malloc(sizeof(cplx) * n);
    cplx *hb = calloc(12 * V, sizeof(cplx));

    /* be = b_e + kappa H_eo b_o */
    orc_hop_eo(L, b_in, (double *)hb, u, 0, nthreads);
    for (long i = 0; i < n; i++) be[i] = b[i] + kappa * hb[i];
    /* rhs = Mhat^dag be */
    mhat(L, u, be, rhs, tmp, kappa, 1, nthreads);

    for (long i = 0; i < n; i++) { x[i] = 0; r[i] = rhs[i]; p[i] = rhs[i]; }
    double rr = dot_re(r, r, n), rhs2 = rr;
    int it = 0;
    while (it < maxiter) {
        mhat(L, u, p, t, tmp, kappa, 0, nthreads);
        mhat(L, u, t, Ap, tmp, kappa, 1, nthreads);
        double alpha = rr / dot_re(p, Ap, n);
        for (long i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
        double rr_new = dot_re(r, r, n);
        double beta = rr_new / rr;
        rr = rr_new;
        for (long i = 0; i < n; i++) p[i] = r[i] + beta * p[i];
        it++;
        /* stop on the true residual of the even system */
        if (rr <= tol * tol * rhs2) {
            mhat(L, u, x, t, tmp, kappa, 0, nthreads);
            double e2 = 0, b2 = dot_re(be, be, n);
            for (long i = 0; i < n; i++) { cplx d = be[i] - t[i]; e2 += creal(conj(d) * d); }
            if (e2 <= tol * tol * b2) break;
        }
    }
    /* x_o = b_o + kappa H_oe x_e */
    memset(hb, 0, sizeof(cplx) * 12 * V);
    orc_hop_oe(L, x_out, (double *)hb, u, 0, nthreads);
    for (long i = n; i < 2 * n; i++) x[i] = b[i] + kappa * hb[i];

    if (relres) {
        cplx *dx = malloc(sizeof(cplx) * 12 * V);
        orc_wilson(L, u, x_out, (double *)dx, kappa, nthreads);
        double e2 = 0, b2 = 0;
        for (long i = 0; i < 12 * V; i++) {
            cplx d = b[i] - dx[i];
            e2 += creal(conj(d) * d);
            b2 += creal(conj(b[i]) * b[i]);
        }
        *relres = sqrt(e2 / b2);
        free(dx);
    }
    free(tmp); free(be); free(rhs); free(r); free(p); free(Ap); free(t); free(hb);
    return it;
}
