/*
 * qz_oracle.c -- CPU restatement of QUANTIZER's head-node particle-mesh step.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.  Only tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py load it.
 *
 * Each routine follows the cited reference routine's arithmetic (operand order,
 * left-to-right sums, no fused multiply-add: build with -ffp-contract=off) so
 * that results match the compiled reference bit for bit; that claim is pinned
 * by tests/test_oracle_golden.py against fixtures dumped by the reference.
 * File:line citations are relative to the QUANTIZER source tree.
 */
#include "qz_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define QZ_PI 3.14159265358979323846 /* global_variables.c:223 */
static const double one_sixth = 1.0 / 6.0; /* global_variables.c:224 */

void qzo_default_params(qzo_params *p, int L)
{
    /* Defaults of global_variables.c:277, 300-341. */
    memset(p, 0, sizeof *p);
    p->L = L;
    p->G = 1.0;
    p->total_mass = 1.0;
    p->bdry = 1;
    p->solver = 0;
    p->cycle = 0;
    p->n_pre = 2;
    p->n_post = 2;
    p->n_coarse = 2;
    p->w_sor = 1.0;
    p->tol = 1.0e-10;
    p->tol2 = 1.0e-10;
    p->check_every = 5;
    p->max_iter = 5000;
    p->check_method = 0;
    p->force_stencil = 0;
    p->head_pot_method = 0;
}

long qzo_grid_points(int L)
{
    long D = (1L << L) + 3;
    return D * D * D;
}

/* initial_potential_and_acceleration_head.c:297-334: analytic point-mass
 * potential and acceleration about (0.5, 0.5, 0.5) at every box point
 * 0 .. 2^L+1 per axis (the last grid layer stays zero, as after calloc). */
static void qzo_initial_head_periodic(const qzo_params *p, double *pot, double *ax, double *ay,
                                      double *az);

void qzo_initial_head(const qzo_params *p, double *pot, double *ax, double *ay, double *az)
{
    int nc = 1 << p->L;
    int bside = nc + 2;
    int gside = bside + 1;
    double H = 1.0 / nc;
    long cap = (long)gside * gside * gside;
    memset(pot, 0, cap * sizeof(double));
    memset(ax, 0, cap * sizeof(double));
    memset(ay, 0, cap * sizeof(double));
    memset(az, 0, cap * sizeof(double));
    if (p->bdry == 0)
    {
        qzo_initial_head_periodic(p, pot, ax, ay, az);
        return;
    }
    for (int k = 0; k < bside; k++)
    {
        double ak = (k - 1) * H - 0.5;
        for (int j = 0; j < bside; j++)
        {
            double aj = (j - 1) * H - 0.5;
            for (int i = 0; i < bside; i++)
            {
                double ai = (i - 1) * H - 0.5;
                double dist = ai * ai + aj * aj + ak * ak;
                dist = sqrt(dist);
                if (dist == 0.0)
                    dist = 1.0 / (1 << p->L) * 1.0e-3;
                long g = i + (long)j * gside + (long)k * gside * gside;
                double coeff = -p->G * p->total_mass / (dist * dist * dist);
                pot[g] = -p->G * p->total_mass / dist;
                ax[g] = coeff * ai;
                ay[g] = coeff * aj;
                az[g] = coeff * ak;
            }
        }
    }
}

/* initial_potential_and_acceleration_head.c:78-296 (periodic boundaries): only
 * points with a box coordinate equal to 1 (coordinates 1 .. 2^L, k outer, i
 * inner) are written, with -G M / d, d the smallest distance from the centre
 * over the point and its images on the far faces (coordinate gl = 2^L + 1);
 * the point's acceleration -G M (a_i, a_j, a_k) / d^3 is copied to the images.
 * The image lists keep the reference's indices as written, including the ones
 * whose x coordinate is 1 where the point's own i would be expected
 * (:125-126, :178, :203, :225), so those far-face points are written from other
 * points and some stay zero. */
static void qzo_initial_head_periodic(const qzo_params *p, double *pot, double *ax, double *ay,
                                      double *az)
{
    const int nc = 1 << p->L;
    const long gs = nc + 3, gs2 = gs * gs;
    const int gl = nc + 1;
    const double H = 1.0 / nc;
    const double a0 = (gl - 1) * H - 0.5;
#define QZO_G(I, J, K) ((long)(I) + (long)(J) * gs + (long)(K) * gs2)
    for (int k = 1; k < gl; k++)
    {
        const double ak = (k - 1) * H - 0.5;
        for (int j = 1; j < gl; j++)
        {
            const double aj = (j - 1) * H - 0.5;
            for (int i = 1; i < gl; i++)
            {
                const double ai = (i - 1) * H - 0.5;
                long idx[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                double dist = 0.0, d0, d1, d2, d3;
                int cnt = 0;
                if (i == 1)
                {
                    idx[0] = QZO_G(i, j, k);
                    idx[1] = QZO_G(gl, j, k);
                    d0 = sqrt(ai * ai + aj * aj + ak * ak);
                    d1 = sqrt(a0 * a0 + aj * aj + ak * ak);
                    dist = d0 < d1 ? d0 : d1;
                    cnt++;
                }
                if (j == 1)
                {
                    if (cnt == 0)
                    {
                        idx[0] = QZO_G(i, j, k);
                        idx[1] = QZO_G(1, gl, k);
                        d0 = sqrt(ai * ai + aj * aj + ak * ak);
                        d1 = sqrt(ai * ai + a0 * a0 + ak * ak);
                        dist = d0 < d1 ? d0 : d1;
                    }
                    else
                    {
                        idx[2] = QZO_G(1, gl, k);
                        idx[3] = QZO_G(gl, gl, k);
                        d2 = sqrt(ai * ai + a0 * a0 + ak * ak);
                        d3 = sqrt(a0 * a0 + a0 * a0 + ak * ak);
                        dist = dist < d2 ? dist : d2;
                        dist = dist < d3 ? dist : d3;
                    }
                    cnt++;
                }
                if (k == 1)
                {
                    if (cnt == 0)
                    {
                        idx[0] = QZO_G(i, j, k);
                        idx[1] = QZO_G(1, j, gl);
                        d0 = sqrt(ai * ai + aj * aj + ak * ak);
                        d1 = sqrt(ai * ai + aj * aj + a0 * a0);
                        dist = d0 < d1 ? d0 : d1;
                    }
                    else if (cnt == 1)
                    {
                        if (i == 1)
                        {
                            idx[2] = QZO_G(1, j, gl);
                            idx[3] = QZO_G(gl, j, gl);
                            d2 = sqrt(ai * ai + aj * aj + a0 * a0);
                            d3 = sqrt(a0 * a0 + aj * aj + a0 * a0);
                        }
                        else
                        {
                            idx[2] = QZO_G(1, j, gl);
                            idx[3] = QZO_G(i, gl, gl);
                            d2 = sqrt(ai * ai + aj * aj + a0 * a0);
                            d3 = sqrt(ai * ai + a0 * a0 + a0 * a0);
                        }
                        dist = dist < d2 ? dist : d2;
                        dist = dist < d3 ? dist : d3;
                    }
                    else
                    {
                        idx[4] = QZO_G(1, j, gl);
                        idx[5] = QZO_G(gl, j, gl);
                        idx[6] = QZO_G(1, gl, gl);
                        idx[7] = QZO_G(gl, gl, gl);
                        const double e4 = sqrt(ai * ai + aj * aj + a0 * a0);
                        const double e5 = sqrt(a0 * a0 + aj * aj + a0 * a0);
                        const double e6 = sqrt(ai * ai + a0 * a0 + a0 * a0);
                        const double e7 = sqrt(a0 * a0 + a0 * a0 + a0 * a0);
                        dist = dist < e4 ? dist : e4;
                        dist = dist < e5 ? dist : e5;
                        dist = dist < e6 ? dist : e6;
                        dist = dist < e7 ? dist : e7;
                    }
                    cnt++;
                }
                if (cnt == 0)
                    continue;
                const double c = -p->G * p->total_mass / dist;
                for (int l = 0; l < (1 << cnt); l++)
                    pot[idx[l]] = c;
                const double c3 = -p->G * p->total_mass / (dist * dist * dist);
                ax[idx[0]] = c3 * ai;
                ay[idx[0]] = c3 * aj;
                az[idx[0]] = c3 * ak;
                for (int l = 1; l < (1 << cnt); l++)
                {
                    ax[idx[l]] = ax[idx[0]];
                    ay[idx[l]] = ay[idx[0]];
                    az[idx[l]] = az[idx[0]];
                }
            }
        }
    }
#undef QZO_G
}

/* grid_density.c:35-111 (head): CIC scatter of 4 pi G m / H^3 onto the 8
 * grid points around each particle, particles in index order. */
void qzo_deposit_head(const qzo_params *p, long n, const double *x, const double *y,
                      const double *z, const double *m, double *d)
{
    int lv = p->L;
    double H = 1.0 / (1 << lv);
    double coeff = 4.0 * p->G * QZ_PI / (H * H * H);
    long D = (1L << lv) + 3;
    long D2 = D * D;
    for (long i = 0; i < n; i++)
    {
        double px = x[i] * (1 << lv), py = y[i] * (1 << lv), pz = z[i] * (1 << lv);
        int fx = (int)px, fy = (int)py, fz = (int)pz;
        double wx1 = px - fx, wy1 = py - fy, wz1 = pz - fz;
        double wx2 = 1.0 - wx1, wy2 = 1.0 - wy1, wz2 = 1.0 - wz1;
        double w[8];
        w[0] = wx2 * wy2 * wz2;
        w[1] = wx1 * wy2 * wz2;
        w[2] = wx2 * wy1 * wz2;
        w[3] = wx1 * wy1 * wz2;
        w[4] = wx2 * wy2 * wz1;
        w[5] = wx1 * wy2 * wz1;
        w[6] = wx2 * wy1 * wz1;
        w[7] = wx1 * wy1 * wz1;
        long g = (fx + 1) + (long)(fy + 1) * D + (long)(fz + 1) * D2;
        for (int kk = 0; kk < 2; kk++)
            for (int jj = 0; jj < 2; jj++)
                for (int ii = 0; ii < 2; ii++)
                    d[g + ii + jj * D + kk * D2] += coeff * m[i] * w[ii + 2 * jj + 4 * kk];
    }
}

/* force_methods/gauss_saidel.c:29-55: lexicographic sweeps, i fastest. */
void qzo_gauss_saidel(double *phi, const double *rho, int n, int iters, double w)
{
    double H2 = (1.0 / (n - 1)) * (1.0 / (n - 1));
    long n2 = (long)n * n;
    for (int it = 0; it < iters; it++)
        for (long k = 1; k < n - 1; k++)
            for (long j = 1; j < n - 1; j++)
                for (long i = 1; i < n - 1; i++)
                {
                    long g = i + j * n + k * n2;
                    double a = one_sixth * (-H2 * rho[g] + phi[g + 1] + phi[g - 1] + phi[g + n] +
                                            phi[g - n] + phi[g + n2] + phi[g - n2]);
                    phi[g] = w * a + (1.0 - w) * phi[g];
                }
}

/* force_methods/jacobi.c:29-82: ping-pong Jacobi; an odd sweep count runs
 * one extra sweep so that the result lands in phi. */
static void jacobi_sweeps(double *old, double *nw, const double *rho, int n, int iters, double w)
{
    double C = -(1.0 / (n - 1)) * (1.0 / (n - 1));
    long n2 = (long)n * n;
    for (int it = 0; it < iters; it++)
    {
        for (long k = 1; k < n - 1; k++)
            for (long j = 1; j < n - 1; j++)
                for (long i = 1; i < n - 1; i++)
                {
                    long g = i + j * n + k * n2;
                    double a = one_sixth * (C * rho[g] + old[g + 1] + old[g - 1] + old[g + n] +
                                            old[g - n] + old[g + n2] + old[g - n2]);
                    nw[g] = w * a + (1.0 - w) * nw[g];
                }
        double *t = old;
        old = nw;
        nw = t;
    }
}

void qzo_jacobi(double *phi, const double *rho, int n, int iters, double w)
{
    long n3 = (long)n * n * n;
    double *cp = (double *)malloc(n3 * sizeof(double));
    memcpy(cp, phi, n3 * sizeof(double));
    if (iters % 2 == 0)
        jacobi_sweeps(phi, cp, rho, n, iters, w);
    else
        jacobi_sweeps(cp, phi, rho, n, iters + 1, w);
    free(cp);
}

/* conjugate_gradient_multigrid.c:29-176: r = rho + (6 phi - sum)/H^2 on the
 * interior, p = r, then up to min(iters, interior points) CG iterations with
 * lexicographic sums, leaving when rs_new / rs_old < 1e-16. */
void qzo_cg_smooth(double *phi, const double *rho, int n, int iters)
{
    double H = 1.0 / (n - 1);
    double oh2 = 1.0 / (H * H);
    long n2 = (long)n * n, n3 = n2 * n;
    double *r = calloc(n3, sizeof(double)), *p = malloc(n3 * sizeof(double)),
           *ap = malloc(n3 * sizeof(double));
    for (long k = 1; k < n - 1; k++)
        for (long j = 1; j < n - 1; j++)
            for (long i = 1; i < n - 1; i++)
            {
                long g = i + j * n + k * n2;
                r[g] = rho[g] + oh2 * (6.0 * phi[g] - phi[g + 1] - phi[g - 1] - phi[g + n] -
                                       phi[g - n] - phi[g + n2] - phi[g - n2]);
            }
    memcpy(p, r, n3 * sizeof(double));
    double rsold = 0.0;
    for (long k = 1; k < n - 1; k++)
        for (long j = 1; j < n - 1; j++)
            for (long i = 1; i < n - 1; i++)
            {
                long g = i + j * n + k * n2;
                rsold += r[g] * r[g];
            }
    long m3 = (long)(n - 2) * (n - 2) * (n - 2);
    long cycle = iters < m3 ? iters : m3;
    for (long it = 0; it < cycle; it++)
    {
        double dot = 0.0, rsnew = 0.0;
        for (long k = 1; k < n - 1; k++)
            for (long j = 1; j < n - 1; j++)
                for (long i = 1; i < n - 1; i++)
                {
                    long g = i + j * n + k * n2;
                    ap[g] = -oh2 * (6.0 * p[g] - p[g + 1] - p[g - 1] - p[g + n] - p[g - n] -
                                    p[g + n2] - p[g - n2]);
                }
        for (long k = 1; k < n - 1; k++)
            for (long j = 1; j < n - 1; j++)
                for (long i = 1; i < n - 1; i++)
                {
                    long g = i + j * n + k * n2;
                    dot += p[g] * ap[g];
                }
        double alpha = rsold / dot;
        for (long k = 1; k < n - 1; k++)
            for (long j = 1; j < n - 1; j++)
                for (long i = 1; i < n - 1; i++)
                {
                    long g = i + j * n + k * n2;
                    phi[g] += alpha * p[g];
                }
        for (long k = 1; k < n - 1; k++)
            for (long j = 1; j < n - 1; j++)
                for (long i = 1; i < n - 1; i++)
                {
                    long g = i + j * n + k * n2;
                    r[g] -= alpha * ap[g];
                }
        for (long k = 1; k < n - 1; k++)
            for (long j = 1; j < n - 1; j++)
                for (long i = 1; i < n - 1; i++)
                {
                    long g = i + j * n + k * n2;
                    rsnew += r[g] * r[g];
                }
        if (rsnew / rsold < 1.0e-16)
            break;
        for (long k = 1; k < n - 1; k++)
            for (long j = 1; j < n - 1; j++)
                for (long i = 1; i < n - 1; i++)
                {
                    long g = i + j * n + k * n2;
                    p[g] = r[g] + rsnew / rsold * p[g];
                }
        rsold = rsnew;
    }
    free(r);
    free(p);
    free(ap);
}

static void smooth(const qzo_params *p, double *phi, const double *rho, int n, int iters)
{
    if (p->solver == 0)
        qzo_gauss_saidel(phi, rho, n, iters, p->w_sor);
    else if (p->solver == 1)
        qzo_jacobi(phi, rho, n, iters, p->w_sor);
    else if (p->solver == 2)
        qzo_cg_smooth(phi, rho, n, iters);
}

/* force_methods/multigrid.c:106-229: one V/F/W cycle. */
void qzo_multigrid(const qzo_params *p, double *phi, const double *rho, int n, int type)
{
    long n2 = (long)n * n, n3 = n2 * n;
    int nc = (n + 1) / 2;
    long nc2 = (long)nc * nc, nc3 = nc2 * nc;
    double ooh2 = (double)((n - 1) * (n - 1));
    double *dphic = (double *)calloc(nc3, sizeof(double));
    double *rest = (double *)calloc(n3, sizeof(double));
    double *restc = (double *)calloc(nc3, sizeof(double));
    double *dphi = (double *)calloc(n3, sizeof(double));

    smooth(p, phi, rho, n, p->n_pre);
    /* residual, multigrid.c:140-150 */
    for (long k = 1; k < n - 1; k++)
        for (long j = 1; j < n - 1; j++)
            for (long i = 1; i < n - 1; i++)
            {
                long g = i + j * n + k * n2;
                rest[g] = rho[g] + ooh2 * (6 * phi[g] - phi[g + 1] - phi[g - 1] - phi[g + n] -
                                           phi[g - n] - phi[g + n2] - phi[g - n2]);
            }
    /* injection, multigrid.c:29-49 */
    for (long lz = 1; lz < nc - 1; lz++)
        for (long ly = 1; ly < nc - 1; ly++)
            for (long lx = 1; lx < nc - 1; lx++)
                restc[lz * nc2 + ly * nc + lx] = rest[2 * lz * n2 + 2 * ly * n + 2 * lx];
    /* coarse problem, multigrid.c:158-191 */
    if (nc < 4)
        smooth(p, phi, rho, n, p->n_coarse);
    else if (type == 0)
        qzo_multigrid(p, dphic, restc, nc, 0);
    else if (type == 1)
    {
        qzo_multigrid(p, dphic, restc, nc, 1);
        qzo_multigrid(p, dphic, restc, nc, 0);
    }
    else
    {
        qzo_multigrid(p, dphic, restc, nc, 2);
        qzo_multigrid(p, dphic, restc, nc, 2);
    }
    /* trilinear prolongation by scatter-add, multigrid.c:51-104 */
    for (long lz = 1; lz < nc - 1; lz++)
        for (long ly = 1; ly < nc - 1; ly++)
            for (long lx = 1; lx < nc - 1; lx++)
            {
                long A = 2 * lz * n2 + 2 * ly * n + 2 * lx;
                double c = dphic[lz * nc2 + ly * nc + lx];
                dphi[A] = c;
                dphi[A + 1] += 0.5 * c;
                dphi[A - 1] += 0.5 * c;
                dphi[A + n] += 0.5 * c;
                dphi[A - n] += 0.5 * c;
                dphi[A + n2] += 0.5 * c;
                dphi[A - n2] += 0.5 * c;
                dphi[A + n + 1] += 0.25 * c;
                dphi[A + n - 1] += 0.25 * c;
                dphi[A - n + 1] += 0.25 * c;
                dphi[A - n - 1] += 0.25 * c;
                dphi[A + n2 + 1] += 0.25 * c;
                dphi[A + n2 - 1] += 0.25 * c;
                dphi[A - n2 + 1] += 0.25 * c;
                dphi[A - n2 - 1] += 0.25 * c;
                dphi[A + n2 + n] += 0.25 * c;
                dphi[A + n2 - n] += 0.25 * c;
                dphi[A - n2 + n] += 0.25 * c;
                dphi[A - n2 - n] += 0.25 * c;
                dphi[A + n2 + n + 1] += 0.125 * c;
                dphi[A + n2 + n - 1] += 0.125 * c;
                dphi[A + n2 - n + 1] += 0.125 * c;
                dphi[A + n2 - n - 1] += 0.125 * c;
                dphi[A - n2 + n + 1] += 0.125 * c;
                dphi[A - n2 + n - 1] += 0.125 * c;
                dphi[A - n2 - n + 1] += 0.125 * c;
                dphi[A - n2 - n - 1] += 0.125 * c;
            }
    for (long k = 1; k < n - 1; k++)
        for (long j = 1; j < n - 1; j++)
            for (long i = 1; i < n - 1; i++)
            {
                long g = i + j * n + k * n2;
                phi[g] += dphi[g];
            }
    smooth(p, phi, rho, n, p->n_post);
    free(dphic);
    free(rest);
    free(restc);
    free(dphi);
}

/* poisson_error.c:36-133, 290-347 for the head node (type 0): the ratio test
 * against pot_old over the interior points, then the residual test; on
 * failure pot_old <- pot. */
int qzo_poisson_check_head(const qzo_params *p, double *pot, double *pot_old, const double *d,
                           double node_mass)
{
    int nc = 1 << p->L;
    long D = nc + 3, D2 = D * D, cap = D2 * D;
    int check = 1;
    double tm = 1.0 - p->tol2, tp = 1.0 + p->tol2;
    for (long k = 2; k <= nc && check; k++)
        for (long j = 2; j <= nc && check; j++)
            for (long i = 2; i <= nc; i++)
            {
                long g = i + j * D + k * D2;
                double a = pot[g] / pot_old[g];
                if ((tm > a) || (tp < a))
                {
                    check = 0;
                    break;
                }
            }
    if (check)
    {
        double H = 1.0 / (1 << p->L);
        double oh2 = 1.0 / (H * H);
        int size = nc * nc * nc;
        long nintr = (long)(nc - 1) * (nc - 1) * (nc - 1);
        double rm = 4.0 * p->G * QZ_PI * node_mass / (size * H * H * H);
        double err = 0.0;
        int ok1 = 1;
        for (long k = 2; k <= nc; k++)
            for (long j = 2; j <= nc; j++)
                for (long i = 2; i <= nc; i++)
                {
                    long g = i + j * D + k * D2;
                    double diff = d[g] + oh2 * (6.0 * pot[g] - pot[g + 1] - pot[g - 1] - pot[g + D] -
                                                pot[g - D] - pot[g + D2] - pot[g - D2]);
                    if (p->check_method == 1)
                    {
                        if (fabs(diff) / rm >= p->tol)
                            ok1 = 0;
                    }
                    else
                        err += diff * diff;
                }
        if (p->check_method == 1)
            check = ok1;
        else
        {
            err = err / nintr;
            err = sqrt(err);
            err = err / rm;
            if (p->check_method == 2)
                err = err / (cbrt((double)nintr) * cbrt((double)nintr));
            check = err < p->tol;
        }
    }
    if (!check)
        memcpy(pot_old, pot, cap * sizeof(double));
    return check;
}

/* conjugate_gradient.c:322-463 on the head (interior points of box
 * coordinates 2..2^L, lexicographic, sums in that order): r = d + lap(pot)
 * sign convention of the reference, p = r; each iteration Ap, alpha =
 * rsold / (p.Ap), pot += alpha p, r -= alpha Ap, rsnew = r.r; every
 * check_every iterations poisson_error type 1 (poisson_error.c:290-347:
 * the pot/pot_old ratio test, then conj_grad_error poisson_error.c:235-282;
 * pot_old <- pot when it fails); then p = r + rsnew/rsold p.  The cycle
 * cap is min(grid points, max_iter). */
int qzo_cg_head(const qzo_params *p, double *pot, double *pot_old, const double *d,
                double node_mass)
{
    int nc = 1 << p->L;
    long D = nc + 3, D2 = D * D, cap = D2 * D;
    long nintr = (long)(nc - 1) * (nc - 1) * (nc - 1);
    double H = 1.0 / (1 << p->L);
    double oh2 = 1.0 / (H * H);
    long *ix = (long *)malloc(nintr * sizeof(long));
    long q = 0;
    for (long k = 2; k <= nc; k++)
        for (long j = 2; j <= nc; j++)
            for (long i = 2; i <= nc; i++)
                ix[q++] = i + j * D + k * D2;
    double *r = (double *)calloc(cap, sizeof(double));
    double *pv = (double *)calloc(cap, sizeof(double));
    double *Ap = (double *)calloc(cap, sizeof(double));
    double rsold = 0.0, rsnew = 0.0;
    for (long t = 0; t < nintr; t++)
    {
        long g = ix[t];
        r[g] = d[g] + oh2 * (6.0 * pot[g] - pot[g + 1] - pot[g - 1] - pot[g + D] - pot[g - D] -
                             pot[g + D2] - pot[g - D2]);
        pv[g] = r[g];
        rsold += r[g] * r[g];
    }
    double rm = 4.0 * p->G * QZ_PI * node_mass / ((double)(nc * nc * nc) * H * H * H);
    long cycle = cap < p->max_iter ? cap : p->max_iter;
    int done = 0;
    long it;
    for (it = 0; it < cycle && !done; it++)
    {
        double pap = 0.0;
        for (long t = 0; t < nintr; t++)
        {
            long g = ix[t];
            Ap[g] = -oh2 * (6.0 * pv[g] - pv[g + 1] - pv[g - 1] - pv[g + D] - pv[g - D] -
                            pv[g + D2] - pv[g - D2]);
            pap += pv[g] * Ap[g];
        }
        double alpha = rsold / pap;
        rsnew = 0.0;
        for (long t = 0; t < nintr; t++)
        {
            long g = ix[t];
            pot[g] += alpha * pv[g];
            r[g] -= alpha * Ap[g];
            rsnew += r[g] * r[g];
        }
        if ((it + 1) % p->check_every == 0)
        {
            int check = 1;
            double tm = 1.0 - p->tol2, tp = 1.0 + p->tol2;
            for (long t = 0; t < nintr; t++)
            {
                double a = pot[ix[t]] / pot_old[ix[t]];
                if ((tm > a) || (tp < a))
                {
                    check = 0;
                    break;
                }
            }
            if (check)
            {
                if (p->check_method == 0)
                    check = rsnew < nintr * (p->tol * rm) * (p->tol * rm);
                else if (p->check_method == 1)
                {
                    for (long t = 0; t < nintr && check; t++)
                        if (fabs(r[ix[t]]) / rm >= p->tol)
                            check = 0;
                }
                else
                    check = rsnew < nintr * (p->tol * rm) * (p->tol * rm) *
                                        (cbrt((double)nintr) * cbrt((double)nintr));
            }
            if (check)
            {
                done = 1;
                break;
            }
            memcpy(pot_old, pot, cap * sizeof(double));
        }
        for (long t = 0; t < nintr; t++)
        {
            long g = ix[t];
            pv[g] = r[g] + rsnew / rsold * pv[g];
        }
        rsold = rsnew;
    }
    free(ix);
    free(r);
    free(pv);
    free(Ap);
    return done ? (int)(it + 1) : -(int)it;
}

/* potential_head_node.c:32-179: V-cycles on the solve grid (box points
 * 1..2^L+1 copied to an aux array and back), checked every check_every
 * cycles; returns the number of cycles, or -cycles when max_iter was hit.
 * With head_pot_method 1 the node conjugate gradient instead
 * (potential_head_node.c:157-171). */
int qzo_potential_head(const qzo_params *p, double *pot, double *pot_old, double *d,
                       double node_mass)
{
    if (p->head_pot_method == 1)
    {
        memcpy(pot_old, pot, qzo_grid_points(p->L) * sizeof(double));
        return qzo_cg_head(p, pot, pot_old, d, node_mass);
    }
    int nc = 1 << p->L;
    long D = nc + 3, D2 = D * D, cap = D2 * D;
    int n = nc + 1;
    long n2 = (long)n * n, n3 = n2 * n;
    double *ap = (double *)malloc(n3 * sizeof(double));
    double *ad = (double *)malloc(n3 * sizeof(double));
    memcpy(pot_old, pot, cap * sizeof(double));
    int iter = 0, check = 0;
    while (iter < p->max_iter && !check)
    {
        iter++;
        for (long k = 1; k <= n; k++)
            for (long j = 1; j <= n; j++)
                for (long i = 1; i <= n; i++)
                {
                    long g = i + j * D + k * D2, a = (i - 1) + (j - 1) * n + (k - 1) * n2;
                    ap[a] = pot[g];
                    ad[a] = d[g];
                }
        qzo_multigrid(p, ap, ad, n, p->cycle);
        for (long k = 1; k <= n; k++)
            for (long j = 1; j <= n; j++)
                for (long i = 1; i <= n; i++)
                {
                    long g = i + j * D + k * D2, a = (i - 1) + (j - 1) * n + (k - 1) * n2;
                    pot[g] = ap[a];
                    d[g] = ad[a];
                }
        if (iter % p->check_every == 0)
            check = qzo_poisson_check_head(p, pot, pot_old, d, node_mass);
    }
    free(ap);
    free(ad);
    return iter == p->max_iter ? -iter : iter;
}

/* grid_acceleration.c:36-76: 3-point central difference on the interior. */
void qzo_grid_accel_head(const qzo_params *p, const double *pot, double *ax, double *ay, double *az)
{
    int nc = 1 << p->L;
    long D = nc + 3, D2 = D * D;
    double H = 1.0 / (1 << p->L);
    double o2h = 1.0 / (2.0 * H);
    /* grid_acceleration.c:78-197 (force_stencil 1): 5-point along an axis whose
     * cells at -2 and +1 are inside the simulation, i.e. box coordinates
     * 3..2^L-1 (the head box ring of status -5 is the only missing cell) */
    double o12h = 1.0 / (12.0 * H), t3h = 2.0 / (3.0 * H);
    for (long k = 2; k <= nc; k++)
        for (long j = 2; j <= nc; j++)
            for (long i = 2; i <= nc; i++)
            {
                long g = i + j * D + k * D2;
                /* periodic (grid_acceleration.c:139-145, 159-165, 179-185): at box
                 * coordinate 2 the -2 neighbour is taken 2^L further, at 2^L the
                 * +2 neighbour 2^L back */
                const long sx[3] = {1, D, D2};
                const long c[3] = {i, j, k};
                double *out[3] = {ax, ay, az};
                for (int q = 0; q < 3; q++)
                {
                    const long s = sx[q];
                    if (p->force_stencil == 1 && c[q] >= 3 && c[q] <= nc - 1)
                        out[q][g] = (pot[g - s] - pot[g + s]) * t3h - (pot[g - 2 * s] - pot[g + 2 * s]) * o12h;
                    else if (p->force_stencil == 1 && p->bdry == 0)
                    {
                        long n7 = g + 2 * s, n8 = g - 2 * s;
                        if (c[q] == 2)
                            n8 += (long)nc * s;
                        else
                            n7 -= (long)nc * s;
                        out[q][g] = (pot[g - s] - pot[g + s]) * t3h - (pot[n8] - pot[n7]) * o12h;
                    }
                    else
                        out[q][g] = o2h * (pot[g - s] - pot[g + s]);
                }
            }
}

/* particle_acceleration.c:33-132: CIC gather, corners in kk, jj, ii order. */
void qzo_gather_head(const qzo_params *p, long n, const double *x, const double *y, const double *z,
                     const double *ax, const double *ay, const double *az,
                     double *pax, double *pay, double *paz)
{
    int lv = p->L;
    long D = (1L << lv) + 3, D2 = D * D;
    for (long i = 0; i < n; i++)
    {
        double px = x[i] * (1 << lv), py = y[i] * (1 << lv), pz = z[i] * (1 << lv);
        int fx = (int)px, fy = (int)py, fz = (int)pz;
        double wx1 = px - fx, wy1 = py - fy, wz1 = pz - fz;
        double wx2 = 1.0 - wx1, wy2 = 1.0 - wy1, wz2 = 1.0 - wz1;
        double w[8];
        w[0] = wx2 * wy2 * wz2;
        w[1] = wx1 * wy2 * wz2;
        w[2] = wx2 * wy1 * wz2;
        w[3] = wx1 * wy1 * wz2;
        w[4] = wx2 * wy2 * wz1;
        w[5] = wx1 * wy2 * wz1;
        w[6] = wx2 * wy1 * wz1;
        w[7] = wx1 * wy1 * wz1;
        long g = (fx + 1) + (long)(fy + 1) * D + (long)(fz + 1) * D2;
        for (int kk = 0; kk < 2; kk++)
            for (int jj = 0; jj < 2; jj++)
                for (int ii = 0; ii < 2; ii++)
                {
                    int a = ii + 2 * jj + 4 * kk;
                    long q = g + ii + jj * D + kk * D2;
                    pax[i] += ax[q] * w[a];
                    pay[i] += ay[q] * w[a];
                    paz[i] += az[q] * w[a];
                }
    }
}

/* particle_updating.c:39-207: kick (half dt), drift, boundary handling. */
int qzo_update_A_head(const qzo_params *p, long n, double dt, double *x, double *y, double *z,
                      double *vx, double *vy, double *vz, double *ax, double *ay, double *az)
{
    double *X[3] = {x, y, z}, *V[3] = {vx, vy, vz}, *A[3] = {ax, ay, az};
    for (long i = 0; i < n; i++)
    {
        for (int c = 0; c < 3; c++)
            V[c][i] += A[c][i] * dt * 0.5;
        for (int c = 0; c < 3; c++)
            X[c][i] += V[c][i] * dt;
        for (int c = 0; c < 3; c++)
        {
            double xc = X[c][i];
            if (xc < 0.0 || xc >= 1.0)
            {
                if (p->bdry == 0)
                    X[c][i] = xc >= 1.0 ? xc - 1.0 : 1.0 + xc;
                else if (p->bdry == 1)
                {
                    X[c][i] = xc >= 1.0 ? 2.0 - xc : -xc;
                    V[c][i] *= -1.0;
                    A[c][i] *= -1.0;
                }
                else
                    return 1; /* outflow: qzo_update_A_outflow */
            }
        }
    }
    return 0;
}

/* particle_updating.c:123-196 (outflow, head only): particles in index order;
 * one that leaves [0, 1) on any axis is removed -- the head's mass drops by
 * the mass at its slot, the count drops by one and the last particle's x, v
 * and a move into the slot (the mass array is not moved), and the loop goes
 * on with the next index, so the moved particle is not advanced in this step.
 * Returns the new count (0: none left, an error there). */
long qzo_update_A_outflow(long n, double dt, double *x, double *y, double *z, double *vx,
                          double *vy, double *vz, double *ax, double *ay, double *az,
                          const double *m, double *node_mass)
{
    double *F[9] = {x, y, z, vx, vy, vz, ax, ay, az};
    for (long i = 0; i < n; i++)
    {
        vx[i] += ax[i] * dt * 0.5;
        vy[i] += ay[i] * dt * 0.5;
        vz[i] += az[i] * dt * 0.5;
        x[i] += vx[i] * dt;
        y[i] += vy[i] * dt;
        z[i] += vz[i] * dt;
        if (x[i] < 0.0 || x[i] >= 1.0 || y[i] < 0.0 || y[i] >= 1.0 || z[i] < 0.0 || z[i] >= 1.0)
        {
            *node_mass -= m[i];
            n--;
            for (int q = 0; q < 9; q++)
                F[q][i] = F[q][n];
            if (n == 0)
                return 0;
        }
    }
    return n;
}

/* particle_updating.c:2677-2688 */
void qzo_update_B_head(long n, double dt, double *vx, double *vy, double *vz,
                       const double *ax, const double *ay, const double *az)
{
    for (long i = 0; i < n; i++)
    {
        vx[i] += ax[i] * dt * 0.5;
        vy[i] += ay[i] * dt * 0.5;
        vz[i] += az[i] * dt * 0.5;
    }
}

/* ptcl_idx_to_box_idx.c:30-139 (non-periodic geometry). */
int qzo_box_idx(int lv, int tsx, int tsy, int tsz, int dimx, int dimy, double x, double y, double z)
{
    double px = x * (1 << lv), py = y * (1 << lv), pz = z * (1 << lv);
    int fx = px < 0 ? -1 : (int)px;
    int fy = py < 0 ? -1 : (int)py;
    int fz = pz < 0 ? -1 : (int)pz;
    return (fx - tsx) + (fy - tsy) * dimx + (fz - tsz) * dimx * dimy;
}

void qzo_box_idx_batch(int lv, int tsx, int tsy, int tsz, int dimx, int dimy, long n,
                       const double *x, const double *y, const double *z, int *out)
{
    for (long i = 0; i < n; i++)
        out[i] = qzo_box_idx(lv, tsx, tsy, tsz, dimx, dimy, x[i], y[i], z[i]);
}

int qzo_sim_init(qzo_sim *s, const qzo_params *p, long n, const double *x, const double *y,
                 const double *z, const double *vx, const double *vy, const double *vz,
                 const double *m)
{
    memset(s, 0, sizeof *s);
    s->p = *p;
    s->n = n;
    long nn = n > 0 ? n : 1;
    double **pa[10] = {&s->x, &s->y, &s->z, &s->vx, &s->vy, &s->vz, &s->ax, &s->ay, &s->az, &s->m};
    for (int q = 0; q < 10; q++)
        *pa[q] = (double *)calloc(nn, sizeof(double));
    memcpy(s->x, x, n * sizeof(double));
    memcpy(s->y, y, n * sizeof(double));
    memcpy(s->z, z, n * sizeof(double));
    memcpy(s->vx, vx, n * sizeof(double));
    memcpy(s->vy, vy, n * sizeof(double));
    memcpy(s->vz, vz, n * sizeof(double));
    memcpy(s->m, m, n * sizeof(double));
    long cap = qzo_grid_points(p->L);
    double **ga[6] = {&s->pot, &s->pot_old, &s->d, &s->gax, &s->gay, &s->gaz};
    for (int q = 0; q < 6; q++)
        *ga[q] = (double *)calloc(cap, sizeof(double));
    qzo_initial_head(&s->p, s->pot, s->gax, s->gay, s->gaz);
    /* step 0: main.c:296-338 */
    qzo_deposit_head(&s->p, n, s->x, s->y, s->z, s->m, s->d);
    s->head_mass = s->p.total_mass; /* initialization.c:190 */
    int it = qzo_potential_head(&s->p, s->pot, s->pot_old, s->d, s->head_mass);
    s->last_vcycles = it;
    if (it < 0)
        return 1;
    s->vcycles_total += it;
    qzo_grid_accel_head(&s->p, s->pot, s->gax, s->gay, s->gaz);
    qzo_gather_head(&s->p, n, s->x, s->y, s->z, s->gax, s->gay, s->gaz, s->ax, s->ay, s->az);
    return 0;
}

/* main.c:375-481 with a fixed dt (timestep() replaced). */
int qzo_sim_step(qzo_sim *s, double dt)
{
    long n = s->n;
    if (s->p.bdry == 2)
    {
        n = s->n = qzo_update_A_outflow(n, dt, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay,
                                        s->az, s->m, &s->head_mass);
        if (n == 0)
            return 1;
    }
    else if (qzo_update_A_head(&s->p, n, dt, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az))
        return 1;
    long cap = qzo_grid_points(s->p.L);
    memset(s->ax, 0, n * sizeof(double));
    memset(s->ay, 0, n * sizeof(double));
    memset(s->az, 0, n * sizeof(double));
    memset(s->d, 0, cap * sizeof(double));
    qzo_deposit_head(&s->p, n, s->x, s->y, s->z, s->m, s->d);
    int it = qzo_potential_head(&s->p, s->pot, s->pot_old, s->d, s->head_mass);
    s->last_vcycles = it;
    if (it < 0)
        return 1;
    s->vcycles_total += it;
    qzo_grid_accel_head(&s->p, s->pot, s->gax, s->gay, s->gaz);
    qzo_gather_head(&s->p, n, s->x, s->y, s->z, s->gax, s->gay, s->gaz, s->ax, s->ay, s->az);
    qzo_update_B_head(n, dt, s->vx, s->vy, s->vz, s->ax, s->ay, s->az);
    return 0;
}

void qzo_sim_free(qzo_sim *s)
{
    double *a[16] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az, s->m,
                     s->pot, s->pot_old, s->d, s->gax, s->gay, s->gaz};
    for (int q = 0; q < 16; q++)
        free(a[q]);
    memset(s, 0, sizeof *s);
}

/* timestep.c:35-157 (head only): method 0 from the largest velocity
 * component, method 1 per particle and axis from velocity and acceleration. */
static double qzo_ts_axis(double v, double a, double H, double cfl, double dt)
{
    if (fabs(a) < 1.0e-16)
    {
        if (fabs(v) > 1.0e-16)
        {
            double aux = cfl * H / fabs(v);
            dt = dt < aux ? dt : aux;
        }
    }
    else
    {
        double c = v * v + 2.0 * fabs(a) * H * cfl;
        double aux;
        if (1 - v * v / c > 1.0e-8)
            aux = (-fabs(v) + sqrt(c)) / fabs(a);
        else
        {
            double eps = fabs(a * H * cfl / (v * v));
            aux = fabs(v / a) * (eps - eps * eps * 0.5);
        }
        dt = dt < aux ? dt : aux;
    }
    return dt;
}

double qzo_timestep_head(int L, int method, double cfl, double max_dt, long n, const double *vx,
                         const double *vy, const double *vz, const double *ax, const double *ay,
                         const double *az)
{
    double H = 1.0 / (1 << L);
    if (method == 1)
    {
        double dt = max_dt;
        for (long i = 0; i < n; i++)
        {
            dt = qzo_ts_axis(vx[i], ax[i], H, cfl, dt);
            dt = qzo_ts_axis(vy[i], ay[i], H, cfl, dt);
            dt = qzo_ts_axis(vz[i], az[i], H, cfl, dt);
        }
        return dt;
    }
    double vmax = 0.0;
    for (long i = 0; i < n; i++)
    {
        if (vmax < fabs(vx[i]))
            vmax = fabs(vx[i]);
        if (vmax < fabs(vy[i]))
            vmax = fabs(vy[i]);
        if (vmax < fabs(vz[i]))
            vmax = fabs(vz[i]);
    }
    double d = vmax < (cfl * H / max_dt) ? max_dt : (cfl * H / vmax);
    return max_dt > d ? d : max_dt;
}
