/*
 * pd_oracle.c -- CPU restatement of ParticleDynamics.jl's algorithms for the
 * force hot path.  TEST INFRASTRUCTURE ONLY: the checker for libpdb200's CUDA
 * path and the CPU baseline of the benchmark.  Nothing in the product links or
 * calls this file.
 *
 * Every function cites the reference file it restates (paths relative to the
 * ParticleDynamics.jl project root).  Arithmetic is FP64 except the cluster
 * list, which follows the reference's Float32 geometry operation by operation
 * (compiled with -ffp-contract=off) so that a build can be compared bit for bit.
 *
 * Build: see oracle/build.py (gcc -O2 -fopenmp -ffp-contract=off -shared).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* Packed coordinates above this value mark padding slots (the device fills them with
 * far-away, pairwise distinct points near 1e7 and zero charge). */
#define PAD_LIMIT 1.0e6f

static double mi(double d, double L) { return d - L * nearbyint(d / L); }

/* ------------------------------------------------------------------------
 * Direct pair sums (FP64).
 *   LJ / WCA: _direct_lj_reference! (test/gpu_force_reference.jl:38-80) and
 *   _reference_kernel! (test/pair_reference_gpu.jl:24-60): round-based minimum
 *   image, f/r = 24 eps s6 (2 s6 - 1) / r^2, pair energy 4 eps s6 (s6 - 1)
 *   (+ eps for WCA, + shift), half to each particle, virial 1/2 f d (x) d.
 *   Real-space Ewald Coulomb erfc(alpha r)/r inside rc_coul
 *   (test/ewald_reference.jl:69-84 restricted to the minimum image).
 * kind: 0 none, 1 LJ, 2 WCA.  ids == NULL samples every particle.
 * out: per sample 11 doubles (F xyz, E, W xx yy zz xy xz yz, count).
 * ---------------------------------------------------------------------- */
void ora_pairs_direct(int n, const double *x, const double *y, const double *z, const double *q,
                      const double box[3], int kind, double sigma, double eps, double rc_lj, double eshift_lj,
                      double C, double alpha, double rc_coul, const int *ids, int nids, double *out) {
    const double Lx = box[0], Ly = box[1], Lz = box[2];
    const double rlj2 = rc_lj * rc_lj, rco2 = rc_coul * rc_coul;
    const double two_a_sqrtpi = 2.0 * alpha / sqrt(M_PI);
#pragma omp parallel for schedule(dynamic, 16)
    for (int s = 0; s < nids; ++s) {
        const int i = ids ? ids[s] : s;
        double f[3] = {0, 0, 0}, e = 0, w[6] = {0, 0, 0, 0, 0, 0}, cnt = 0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            const double dx = mi(x[i] - x[j], Lx), dy = mi(y[i] - y[j], Ly), dz = mi(z[i] - z[j], Lz);
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (!(r2 > 0.0)) continue;
            double a = 0.0, u = 0.0;
            int hit = 0;
            if (kind && r2 < rlj2) {
                const double s6 = pow(sigma * sigma / r2, 3);
                a += 24.0 * eps * s6 * (2.0 * s6 - 1.0) / r2;
                u += 4.0 * eps * s6 * (s6 - 1.0) + (kind == 2 ? eps : 0.0) - eshift_lj;
                hit = 1;
            }
            if (C != 0.0 && q && r2 < rco2) {
                const double r = sqrt(r2);
                const double qq = C * q[i] * q[j];
                const double ec = erfc(alpha * r);
                u += qq * ec / r;
                a += qq * (ec / r + two_a_sqrtpi * exp(-alpha * alpha * r2)) / r2;
                hit = 1;
            }
            if (!hit) continue;
            f[0] += a * dx;
            f[1] += a * dy;
            f[2] += a * dz;
            e += 0.5 * u;
            w[0] += 0.5 * a * dx * dx;
            w[1] += 0.5 * a * dy * dy;
            w[2] += 0.5 * a * dz * dz;
            w[3] += 0.5 * a * dx * dy;
            w[4] += 0.5 * a * dx * dz;
            w[5] += 0.5 * a * dy * dz;
            cnt += 1.0;
        }
        double *o = out + 11 * (size_t)s;
        o[0] = f[0];
        o[1] = f[1];
        o[2] = f[2];
        o[3] = e;
        for (int k = 0; k < 6; ++k) o[4 + k] = w[k];
        o[10] = cnt;
    }
}

/* Same physics as ora_pairs_direct for every particle, with a cell grid (cells
 * >= the largest cutoff) so that large systems finish in seconds.  Each pair is
 * visited from both sides (no write races).  Used for parity at large N and as
 * the CPU baseline of the short-range part. */
void ora_pairs_cells(int n, const double *x, const double *y, const double *z, const double *q, const double box[3],
                     int kind, double sigma, double eps, double rc_lj, double eshift_lj, double C, double alpha,
                     double rc_coul, double *fx, double *fy, double *fz, double *epot, double *vir6) {
    const double L[3] = {box[0], box[1], box[2]};
    const double rmax = fmax(kind ? rc_lj : 0.0, C != 0.0 ? rc_coul : 0.0);
    int nc[3];
    for (int d = 0; d < 3; ++d) {
        nc[d] = (int)floor(L[d] / rmax);
        if (nc[d] < 3) nc[d] = 3;
    }
    const int ncell = nc[0] * nc[1] * nc[2];
    int *head = (int *)malloc(sizeof(int) * ncell), *next = (int *)malloc(sizeof(int) * n);
    int *cell = (int *)malloc(sizeof(int) * n);
    for (int c = 0; c < ncell; ++c) head[c] = -1;
    for (int i = 0; i < n; ++i) {
        const double p[3] = {x[i], y[i], z[i]};
        int ci[3];
        for (int d = 0; d < 3; ++d) {
            double u = p[d] / L[d];
            u -= floor(u);
            int k = (int)(u * nc[d]);
            if (k >= nc[d]) k = nc[d] - 1;
            if (k < 0) k = 0;
            ci[d] = k;
        }
        cell[i] = ci[0] + nc[0] * (ci[1] + nc[1] * ci[2]);
    }
    for (int i = n - 1; i >= 0; --i) {
        next[i] = head[cell[i]];
        head[cell[i]] = i;
    }
    const double rlj2 = rc_lj * rc_lj, rco2 = rc_coul * rc_coul;
    const double two_a_sqrtpi = 2.0 * alpha / sqrt(M_PI);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        const int c = cell[i];
        const int cx = c % nc[0], cy = (c / nc[0]) % nc[1], cz = c / (nc[0] * nc[1]);
        double f[3] = {0, 0, 0}, e = 0, w[6] = {0, 0, 0, 0, 0, 0};
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int cc = ((cx + dx + nc[0]) % nc[0]) + nc[0] * (((cy + dy + nc[1]) % nc[1]) +
                                                                           nc[1] * ((cz + dz + nc[2]) % nc[2]));
                    for (int j = head[cc]; j >= 0; j = next[j]) {
                        if (j == i) continue;
                        const double ddx = mi(x[i] - x[j], L[0]), ddy = mi(y[i] - y[j], L[1]),
                                     ddz = mi(z[i] - z[j], L[2]);
                        const double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        double a = 0.0, u = 0.0;
                        int hit = 0;
                        if (kind && r2 < rlj2) {
                            const double s2 = sigma * sigma / r2, s6 = s2 * s2 * s2;
                            a += 24.0 * eps * s6 * (2.0 * s6 - 1.0) / r2;
                            u += 4.0 * eps * s6 * (s6 - 1.0) + (kind == 2 ? eps : 0.0) - eshift_lj;
                            hit = 1;
                        }
                        if (C != 0.0 && q && r2 < rco2) {
                            const double r = sqrt(r2);
                            const double qq = C * q[i] * q[j];
                            const double ec = erfc(alpha * r);
                            u += qq * ec / r;
                            a += qq * (ec / r + two_a_sqrtpi * exp(-alpha * alpha * r2)) / r2;
                            hit = 1;
                        }
                        if (!hit) continue;
                        f[0] += a * ddx;
                        f[1] += a * ddy;
                        f[2] += a * ddz;
                        e += 0.5 * u;
                        w[0] += 0.5 * a * ddx * ddx;
                        w[1] += 0.5 * a * ddy * ddy;
                        w[2] += 0.5 * a * ddz * ddz;
                        w[3] += 0.5 * a * ddx * ddy;
                        w[4] += 0.5 * a * ddx * ddz;
                        w[5] += 0.5 * a * ddy * ddz;
                    }
                }
        fx[i] = f[0];
        fy[i] = f[1];
        fz[i] = f[2];
        if (epot) epot[i] = e;
        if (vir6)
            for (int k = 0; k < 6; ++k) vir6[(size_t)6 * i + k] = w[k];
    }
    free(head);
    free(next);
    free(cell);
}

/* Neighbor rows (test/neighbor_reference.jl:6-16): j != i within radius, FP64
 * minimum image.  rows must hold n*cap entries; counts[i] may exceed cap (then
 * the row is truncated).  Returns the largest count. */
int ora_neighbor_rows(int n, const double *x, const double *y, const double *z, const double box[3], double radius,
                      int cap, int *counts, int *rows) {
    int mx = 0;
#pragma omp parallel for reduction(max : mx) schedule(dynamic, 32)
    for (int i = 0; i < n; ++i) {
        int c = 0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            const double dx = mi(x[j] - x[i], box[0]), dy = mi(y[j] - y[i], box[1]), dz = mi(z[j] - z[i], box[2]);
            if (dx * dx + dy * dy + dz * dz <= radius * radius) {
                if (c < cap) rows[(size_t)i * cap + c] = j;
                ++c;
            }
        }
        counts[i] = c;
        if (c > mx) mx = c;
    }
    return mx;
}

/* ------------------------------------------------------------------------
 * Ewald sum (test/ewald_reference.jl:50-127) for an orthorhombic cell: real
 * space over images within rcut = x/alpha, reciprocal space within
 * kmax = 2 alpha x, x = sqrt(digits ln 10); self and optional uniform
 * background.  alpha <= 0 picks 3.6 / min width as the reference.
 * Outputs E, F (3n), W (9, row-major W_ab = sum r_a F_b).
 * ---------------------------------------------------------------------- */
void ora_ewald(int n, const double *R /* 3n, xyz per particle */, const double *q, const double box[3], double C,
               double alpha, double digits, int background, double *E_out, double *F, double *W) {
    const double V = box[0] * box[1] * box[2];
    const double wmin = fmin(box[0], fmin(box[1], box[2]));
    const double a = alpha > 0 ? alpha : 3.6 / wmin;
    const double xx = sqrt(digits * log(10.0));
    const double rcut = xx / a, kmax = 2.0 * a * xx;
    int nimg[3];
    for (int d = 0; d < 3; ++d) nimg[d] = (int)ceil(rcut / box[d]) + 1;
    double E = 0.0;
    double Wt[9] = {0};
    for (int k = 0; k < 3 * n; ++k) F[k] = 0.0;
    const double tap = 2.0 * a / sqrt(M_PI);
#pragma omp parallel
    {
        double El = 0.0, Wl[9] = {0};
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < n; ++i) {
            double fi[3] = {0, 0, 0};
            for (int j = 0; j < n; ++j) {
                const double qq = C * q[i] * q[j];
                if (qq == 0.0) continue;
                for (int n1 = -nimg[0]; n1 <= nimg[0]; ++n1)
                    for (int n2 = -nimg[1]; n2 <= nimg[1]; ++n2)
                        for (int n3 = -nimg[2]; n3 <= nimg[2]; ++n3) {
                            if (i == j && n1 == 0 && n2 == 0 && n3 == 0) continue;
                            const double d[3] = {R[3 * i] - R[3 * j] + box[0] * n1, R[3 * i + 1] - R[3 * j + 1] + box[1] * n2,
                                                 R[3 * i + 2] - R[3 * j + 2] + box[2] * n3};
                            const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                            if (!(r < rcut)) continue;
                            const double ec = erfc(a * r);
                            El += 0.5 * qq * ec / r;
                            const double fm = qq * (ec / r + tap * exp(-a * a * r * r)) / (r * r);
                            for (int c = 0; c < 3; ++c) fi[c] += fm * d[c];
                            for (int u = 0; u < 3; ++u)
                                for (int v = 0; v < 3; ++v) Wl[3 * u + v] += 0.5 * fm * d[u] * d[v];
                        }
            }
            for (int c = 0; c < 3; ++c) F[3 * i + c] += fi[c];
        }
#pragma omp critical
        {
            E += El;
            for (int k = 0; k < 9; ++k) Wt[k] += Wl[k];
        }
    }
    /* reciprocal space */
    int mmax[3];
    for (int d = 0; d < 3; ++d) mmax[d] = (int)ceil(kmax / (2.0 * M_PI / box[d])) + 1;
    const int n1r = 2 * mmax[0] + 1, n2r = 2 * mmax[1] + 1, n3r = 2 * mmax[2] + 1;
    const long long nk = (long long)n1r * n2r * n3r;
#pragma omp parallel
    {
        double El = 0.0, Wl[9] = {0};
        double *Fl = (double *)calloc(3 * (size_t)n, sizeof(double));
#pragma omp for schedule(dynamic, 8)
        for (long long t = 0; t < nk; ++t) {
            const int m1 = (int)(t % n1r) - mmax[0];
            const int m2 = (int)((t / n1r) % n2r) - mmax[1];
            const int m3 = (int)(t / ((long long)n1r * n2r)) - mmax[2];
            if (m1 == 0 && m2 == 0 && m3 == 0) continue;
            const double k[3] = {2.0 * M_PI * m1 / box[0], 2.0 * M_PI * m2 / box[1], 2.0 * M_PI * m3 / box[2]};
            const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
            if (!(k2 < kmax * kmax)) continue;
            const double g = 4.0 * M_PI * exp(-k2 / (4.0 * a * a)) / k2;
            double Sr = 0.0, Si = 0.0;
            for (int i = 0; i < n; ++i) {
                const double ph = k[0] * R[3 * i] + k[1] * R[3 * i + 1] + k[2] * R[3 * i + 2];
                Sr += q[i] * cos(ph);
                Si += q[i] * sin(ph);
            }
            const double Ek = C / (2.0 * V) * g * (Sr * Sr + Si * Si);
            El += Ek;
            for (int i = 0; i < n; ++i) {
                const double ph = k[0] * R[3 * i] + k[1] * R[3 * i + 1] + k[2] * R[3 * i + 2];
                /* imag(cis(ph) conj(S)) = sin(ph) Sr - cos(ph) Si */
                const double im = sin(ph) * Sr - cos(ph) * Si;
                const double s = (C / V) * g * q[i] * im;
                for (int c = 0; c < 3; ++c) Fl[3 * i + c] += s * k[c];
            }
            const double fac = 2.0 * (1.0 + k2 / (4.0 * a * a)) / k2;
            for (int u = 0; u < 3; ++u)
                for (int v = 0; v < 3; ++v) Wl[3 * u + v] += Ek * ((u == v ? 1.0 : 0.0) - fac * k[u] * k[v]);
        }
#pragma omp critical
        {
            E += El;
            for (int k = 0; k < 9; ++k) Wt[k] += Wl[k];
            for (int k = 0; k < 3 * n; ++k) F[k] += Fl[k];
        }
        free(Fl);
    }
    double q2 = 0.0, qs = 0.0;
    for (int i = 0; i < n; ++i) {
        q2 += q[i] * q[i];
        qs += q[i];
    }
    E -= C * a / sqrt(M_PI) * q2;
    if (background) {
        const double Ebg = -C * M_PI * qs * qs / (2.0 * a * a * V);
        E += Ebg;
        Wt[0] += Ebg;
        Wt[4] += Ebg;
        Wt[8] += Ebg;
    }
    *E_out = E;
    for (int k = 0; k < 9; ++k) W[k] = Wt[k];
}

/* ------------------------------------------------------------------------
 * Mesh restatement (FP64).
 * ---------------------------------------------------------------------- */

/* window_stencil(::BSplineStencil{P}, u) (src/electrostatics/Windows.jl:187-223):
 * returns k0 = floor(u) - P + 1, weights and derivatives in ascending node order. */
int ora_bspline(int P, double u, double *w, double *dw) {
    const double fl = floor(u), t = u - fl;
    double a[16], full[16];
    a[0] = t;
    a[1] = 1.0 - t;
    int len = 2;
    while (len < P - 1) { /* _bspline_step from length len to len + 1 */
        double b[16];
        for (int j = 0; j <= len; ++j) {
            const double left = j < len ? a[j] : 0.0, right = j >= 1 ? a[j - 1] : 0.0;
            b[j] = ((t + j) * left + ((double)(len + 1) - t - j) * right) / len;
        }
        ++len;
        memcpy(a, b, sizeof(double) * len);
    }
    for (int j = 0; j < P; ++j) {
        const int nn = P - 1;
        const double left = j < nn ? a[j] : 0.0, right = j >= 1 ? a[j - 1] : 0.0;
        full[j] = ((t + j) * left + ((double)(nn + 1) - t - j) * right) / nn;
    }
    for (int i = 0; i < P; ++i) {
        w[i] = full[P - 1 - i];
        const int j = P - 1 - i;
        const double left = j <= P - 2 ? a[j] : 0.0, right = j >= 1 ? a[j - 1] : 0.0;
        if (dw) dw[i] = left - right;
    }
    return (int)fl - (P - 1);
}

static double grid_coordinate(double x, double L, int K) {
    double s = x / L;
    s -= floor(s);
    double u = s * K;
    if (!isfinite(u)) return 0.0;
    return u >= K ? u - K : u;
}

static int wrapn(int n, int K) {
    n %= K;
    return n < 0 ? n + K : n;
}

/* Charge assignment (_spread_lines_kernel!, MeshKernels.jl:247-276): grid[n1 + K1 (n2 + K2 n3)] += q W. */
void ora_spread(int n, const double *x, const double *y, const double *z, const double *q, const double box[3],
                const int K[3], int P, double *grid) {
    memset(grid, 0, sizeof(double) * (size_t)K[0] * K[1] * K[2]);
    for (int i = 0; i < n; ++i) {
        if (q[i] == 0.0) continue;
        double w1[16], w2[16], w3[16];
        const int k1 = ora_bspline(P, grid_coordinate(x[i], box[0], K[0]), w1, NULL);
        const int k2 = ora_bspline(P, grid_coordinate(y[i], box[1], K[1]), w2, NULL);
        const int k3 = ora_bspline(P, grid_coordinate(z[i], box[2], K[2]), w3, NULL);
        for (int j3 = 0; j3 < P; ++j3) {
            const int n3 = wrapn(k3 + j3, K[2]);
            for (int j2 = 0; j2 < P; ++j2) {
                const int n2 = wrapn(k2 + j2, K[1]);
                for (int j1 = 0; j1 < P; ++j1)
                    grid[((size_t)n3 * K[1] + n2) * K[0] + wrapn(k1 + j1, K[0])] += q[i] * w1[j1] * w2[j2] * w3[j3];
            }
        }
    }
}

/* AD gather (_gather_ad_lines_kernel!, MeshKernels.jl:313-333): F = -q grad(phi) K/L,
 * phi_i = sum W pot (returned in phi). */
void ora_gather_ad(int n, const double *x, const double *y, const double *z, const double *q, const double box[3],
                   const int K[3], int P, const double *pot, double *F, double *phi) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double w1[16], w2[16], w3[16], d1[16], d2[16], d3[16];
        const int k1 = ora_bspline(P, grid_coordinate(x[i], box[0], K[0]), w1, d1);
        const int k2 = ora_bspline(P, grid_coordinate(y[i], box[1], K[1]), w2, d2);
        const int k3 = ora_bspline(P, grid_coordinate(z[i], box[2], K[2]), w3, d3);
        double p = 0, gx = 0, gy = 0, gz = 0;
        for (int j3 = 0; j3 < P; ++j3) {
            const int n3 = wrapn(k3 + j3, K[2]);
            for (int j2 = 0; j2 < P; ++j2) {
                const int n2 = wrapn(k2 + j2, K[1]);
                for (int j1 = 0; j1 < P; ++j1) {
                    const double c = pot[((size_t)n3 * K[1] + n2) * K[0] + wrapn(k1 + j1, K[0])];
                    p += w1[j1] * w2[j2] * w3[j3] * c;
                    gx += d1[j1] * w2[j2] * w3[j3] * c;
                    gy += w1[j1] * d2[j2] * w3[j3] * c;
                    gz += w1[j1] * w2[j2] * d3[j3] * c;
                }
            }
        }
        F[3 * i] = -q[i] * gx * (K[0] / box[0]);
        F[3 * i + 1] = -q[i] * gy * (K[1] / box[1]);
        F[3 * i + 2] = -q[i] * gz * (K[2] / box[2]);
        phi[i] = p;
    }
}

/* ik gather (_gather_ik_kernel!, MeshKernels.jl:105-147): F = q sum W E. */
void ora_gather_ik(int n, const double *x, const double *y, const double *z, const double *q, const double box[3],
                   const int K[3], int P, const double *ex, const double *ey, const double *ez, const double *pot,
                   double *F, double *phi) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double w1[16], w2[16], w3[16];
        const int k1 = ora_bspline(P, grid_coordinate(x[i], box[0], K[0]), w1, NULL);
        const int k2 = ora_bspline(P, grid_coordinate(y[i], box[1], K[1]), w2, NULL);
        const int k3 = ora_bspline(P, grid_coordinate(z[i], box[2], K[2]), w3, NULL);
        double sx = 0, sy = 0, sz = 0, p = 0;
        for (int j3 = 0; j3 < P; ++j3) {
            const int n3 = wrapn(k3 + j3, K[2]);
            for (int j2 = 0; j2 < P; ++j2) {
                const int n2 = wrapn(k2 + j2, K[1]);
                for (int j1 = 0; j1 < P; ++j1) {
                    const size_t l = ((size_t)n3 * K[1] + n2) * K[0] + wrapn(k1 + j1, K[0]);
                    const double ww = w1[j1] * w2[j2] * w3[j3];
                    sx += ww * ex[l];
                    sy += ww * ey[l];
                    sz += ww * ez[l];
                    p += ww * pot[l];
                }
            }
        }
        F[3 * i] = q[i] * sx;
        F[3 * i + 1] = q[i] * sy;
        F[3 * i + 2] = q[i] * sz;
        phi[i] = p;
    }
}

static int signed_mode(int m, int K) { return m <= K / 2 ? m : m - K; }
static int is_nyq(int m, int K) { return (K % 2 == 0) && m == K / 2; }

/* M_P at the integers (Windows.jl:265-271) and the SPME deconvolution (Windows.jl:283-308). */
static void deconvolution(int P, int K, double *D) {
    double a[16] = {0.0, 1.0};
    int len = 2;
    while (len < P) {
        double b[16];
        for (int j = 0; j <= len; ++j) {
            const double left = j < len ? a[j] : 0.0, right = j >= 1 ? a[j - 1] : 0.0;
            b[j] = ((0.0 + j) * left + ((double)(len + 1) - 0.0 - j) * right) / len;
        }
        ++len;
        memcpy(a, b, sizeof(double) * len);
    }
    for (int m = 0; m < K; ++m) {
        double re = 0, im = 0;
        for (int j = 0; j < P; ++j) {
            re += a[j] * cos(2.0 * M_PI * m * j / K);
            im += a[j] * sin(2.0 * M_PI * m * j / K);
        }
        const double den = re * re + im * im;
        D[m] = den > 1e-12 ? 1.0 / den : NAN;
    }
    for (int m = 0; m < K; ++m)
        if (isnan(D[m])) D[m] = 0.5 * (D[(m - 1 + K) % K] + D[(m + 1) % K]);
}

static void spectral_g(double alpha, double k, double *g, double *gpk) {
    const double k2 = k * k;
    *g = 4.0 * M_PI * exp(-k2 / (4.0 * alpha * alpha)) / k2;
    *gpk = *g * (-2.0 / k2 - 1.0 / (2.0 * alpha * alpha));
}

/* Influence function and virial coefficients on the R2C half spectrum
 * (src/electrostatics/Influence.jl:35-181): kind 1 SPME, 2 P3M-AD, 3 P3M-ik.
 * G[nmodes], Vc[6 * nmodes] (component-major). */
void ora_influence(int kind, int P, int nmax, const int K[3], const double box[3], double C, double alpha, double *G,
                   double *Vc) {
    const int K1 = K[0], K2 = K[1], K3 = K[2], K1h = K1 / 2 + 1;
    const long long nm = (long long)K1h * K2 * K3;
    double *D[3] = {NULL, NULL, NULL}, *U[3] = {NULL, NULL, NULL};
    const int na = 2 * nmax + 1;
    for (int d = 0; d < 3; ++d) {
        if (kind == 1) {
            D[d] = (double *)malloc(sizeof(double) * K[d]);
            deconvolution(P, K[d], D[d]);
        } else {
            U[d] = (double *)malloc(sizeof(double) * K[d] * na);
            for (int m = 0; m < K[d]; ++m)
                for (int nn = -nmax; nn <= nmax; ++nn) {
                    const double xx = M_PI * (signed_mode(m, K[d]) + (double)K[d] * nn) / K[d];
                    const double s = fabs(xx) < 1e-12 ? 1.0 : sin(xx) / xx;
                    U[d][m * na + nn + nmax] = pow(s, P);
                }
        }
    }
    const double CoverV = C / (box[0] * box[1] * box[2]);
#pragma omp parallel for schedule(static)
    for (long long idx = 0; idx < nm; ++idx) {
        const int m1 = (int)(idx % K1), dummy = 0;
        (void)dummy;
        const int mm1 = (int)(idx % K1h), rest = (int)(idx / K1h), m2 = rest % K2, m3 = rest / K2;
        (void)m1;
        const int s1 = mm1, s2 = signed_mode(m2, K2), s3 = signed_mode(m3, K3);
        const int ny1 = is_nyq(mm1, K1), ny2 = is_nyq(m2, K2), ny3 = is_nyq(m3, K3);
        const double kx = 2.0 * M_PI * s1 / box[0], ky = 2.0 * M_PI * s2 / box[1], kz = 2.0 * M_PI * s3 / box[2];
        double v[6], Gm;
        if (kind == 1) {
            if (s1 == 0 && s2 == 0 && s3 == 0) {
                G[idx] = 0;
                for (int c = 0; c < 6; ++c) Vc[c * nm + idx] = 0;
                continue;
            }
            const double k = sqrt(kx * kx + ky * ky + kz * kz);
            double g, gpk;
            spectral_g(alpha, k, &g, &gpk);
            const double Dm = D[0][mm1] * D[1][m2] * D[2][m3];
            Gm = CoverV * g * Dm;
            const double c = CoverV * Dm * gpk;
            v[0] = Gm + c * kx * kx;
            v[1] = Gm + c * ky * ky;
            v[2] = Gm + c * kz * kz;
            v[3] = c * kx * ky;
            v[4] = c * kx * kz;
            v[5] = c * ky * kz;
        } else {
            const int ik = kind == 3;
            const double dx = ny1 ? 0.0 : kx, dy = ny2 ? 0.0 : ky, dz = ny3 ? 0.0 : kz;
            const double d2 = dx * dx + dy * dy + dz * dz;
            if ((s1 == 0 && s2 == 0 && s3 == 0) || (ik && d2 == 0.0)) {
                G[idx] = 0;
                for (int c = 0; c < 6; ++c) Vc[c * nm + idx] = 0;
                continue;
            }
            double A = 0, B = 0, Cc = 0, aa[6] = {0}, cc[6] = {0};
            for (int n1 = -nmax; n1 <= nmax; ++n1) {
                const double u1 = U[0][mm1 * na + n1 + nmax], q1 = 2.0 * M_PI * (s1 + (double)K1 * n1) / box[0];
                for (int n2 = -nmax; n2 <= nmax; ++n2) {
                    const double u2 = U[1][m2 * na + n2 + nmax], q2 = 2.0 * M_PI * (s2 + (double)K2 * n2) / box[1];
                    for (int n3 = -nmax; n3 <= nmax; ++n3) {
                        const double u3 = U[2][m3 * na + n3 + nmax], q3 = 2.0 * M_PI * (s3 + (double)K3 * n3) / box[2];
                        const double U2 = (u1 * u2 * u3) * (u1 * u2 * u3);
                        B += U2;
                        const double qq = q1 * q1 + q2 * q2 + q3 * q3;
                        if (qq == 0.0) continue;
                        double g, gpk;
                        spectral_g(alpha, sqrt(qq), &g, &gpk);
                        if (ik) {
                            const double dq = dx * q1 + dy * q2 + dz * q3;
                            A += U2 * g * dq;
                            const double h = U2 * gpk * dq;
                            aa[0] += h * q1 * q1 + U2 * g * 2.0 * dx * q1;
                            aa[1] += h * q2 * q2 + U2 * g * 2.0 * dy * q2;
                            aa[2] += h * q3 * q3 + U2 * g * 2.0 * dz * q3;
                            aa[3] += h * q1 * q2 + U2 * g * (dx * q2 + q1 * dy);
                            aa[4] += h * q1 * q3 + U2 * g * (dx * q3 + q1 * dz);
                            aa[5] += h * q2 * q3 + U2 * g * (dy * q3 + q2 * dz);
                        } else {
                            A += U2 * g * qq;
                            Cc += U2 * qq;
                            const double h = U2 * (gpk * qq + 2.0 * g);
                            aa[0] += h * q1 * q1;
                            aa[1] += h * q2 * q2;
                            aa[2] += h * q3 * q3;
                            aa[3] += h * q1 * q2;
                            aa[4] += h * q1 * q3;
                            aa[5] += h * q2 * q3;
                            const double h2 = 2.0 * U2;
                            cc[0] += h2 * q1 * q1;
                            cc[1] += h2 * q2 * q2;
                            cc[2] += h2 * q3 * q3;
                            cc[3] += h2 * q1 * q2;
                            cc[4] += h2 * q1 * q3;
                            cc[5] += h2 * q2 * q3;
                        }
                    }
                }
            }
            if (ik) {
                const double den = d2 * B * B;
                Gm = CoverV * A / den;
                const double f = CoverV / den, r = CoverV * A / (B * B) * 2.0 / (d2 * d2);
                const double dd[6] = {dx * dx, dy * dy, dz * dz, dx * dy, dx * dz, dy * dz};
                for (int c = 0; c < 6; ++c) v[c] = (c < 3 ? Gm : 0.0) + f * aa[c] - r * dd[c];
            } else {
                Gm = CoverV * A / (B * Cc);
                const double f = CoverV / (B * Cc), r = CoverV * A / (B * Cc * Cc);
                for (int c = 0; c < 6; ++c) v[c] = (c < 3 ? Gm : 0.0) + f * aa[c] - r * cc[c];
            }
        }
        G[idx] = Gm;
        Vc[0 * nm + idx] = v[0];
        Vc[1 * nm + idx] = v[1];
        Vc[2 * nm + idx] = v[2];
        Vc[3 * nm + idx] = (ny1 || ny2) ? 0.0 : v[3];
        Vc[4 * nm + idx] = (ny1 || ny3) ? 0.0 : v[4];
        Vc[5 * nm + idx] = (ny2 || ny3) ? 0.0 : v[5];
    }
    for (int d = 0; d < 3; ++d) {
        free(D[d]);
        free(U[d]);
    }
}

/* ------------------------------------------------------------------------
 * Cluster list (src/clusterpairs/List.jl) in Float32 geometry, with the order
 * inside a z-bin fixed to (wrapped z, particle id).
 * ---------------------------------------------------------------------- */
static float wrapf(float x, float L) {
    const float fl = floorf(x / L);
    const float p = L * fl;
    return x - p;
}

static float micf(float d, float L) {
    const float h = 0.5f * L;
    if (d > h) d = d - L;
    if (d < -h) d = d + L;
    return d;
}

static float bbgap2f(const float *c1, const float *h1, const float *c2, const float *h2, const float *L) {
    float g[3];
    for (int d = 0; d < 3; ++d) {
        float a = fabsf(micf(c1[d] - c2[d], L[d]));
        a = a - h1[d];
        a = a - h2[d];
        g[d] = a > 0.0f ? a : 0.0f;
    }
    const float gx2 = g[0] * g[0], gy2 = g[1] * g[1], gz2 = g[2] * g[2];
    const float s = gx2 + gy2;
    return s + gz2;
}

typedef struct {
    int i;
    float z;
} zid;

static int cmp_zid(const void *a, const void *b) {
    const zid *p = (const zid *)a, *r = (const zid *)b;
    if (p->z < r->z) return -1;
    if (p->z > r->z) return 1;
    return p->i - r->i;
}

/* Geometry of setup! (List.jl:874-937).  geom[0..9] = ncx, ncy, nzb, mx, my, ncol, nbin, nsmax, nslot, ncs. */
int ora_cluster_geometry(int n, const double box[3], double rlist, int *geom) {
    const double Lx = (float)box[0], Ly = (float)box[1], Lz = (float)box[2];
    if (!(fmin(Lx, fmin(Ly, Lz)) > 2 * rlist)) return 1;
    const double rho = n / (Lx * Ly * Lz);
    const double b = cbrt(64.0 / rho);
    int ncx = (int)floor(Lx / b), ncy = (int)floor(Ly / b);
    if (ncx < 1) ncx = 1;
    if (ncy < 1) ncy = 1;
    const int ncol = ncx * ncy;
    int nzb = (int)nearbyint(Lz * rho * (Lx / ncx) * (Ly / ncy) / 4);
    if (nzb < 1) nzb = 1;
    const int nsmax = (n + 63) / 64 + ncol;
    const int mx = (int)floor(rlist / (0.98 * Lx / ncx)) + 1, my = (int)floor(rlist / (0.98 * Ly / ncy)) + 1;
    const int nxr = 2 * mx + 1 < ncx ? 2 * mx + 1 : ncx, nyr = 2 * my + 1 < ncy ? 2 * my + 1 : ncy;
    geom[0] = ncx;
    geom[1] = ncy;
    geom[2] = nzb;
    geom[3] = mx;
    geom[4] = my;
    geom[5] = ncol;
    geom[6] = ncol * nzb;
    geom[7] = nsmax;
    geom[8] = 64 * nsmax;
    geom[9] = nxr * nyr;
    return 0;
}

/* build! (List.jl:979-1051) without exclusions: clustering (_column_key_kernel!,
 * _cluster_assign_kernel!), bounding boxes (_bbox_kernel!, _super_bbox_kernel!) and
 * the outer search (_search_warp_kernel!) in serial order.
 * Outputs: perm[nslot] (-1 padding), scio[nsmax+1], cjo[necap] ((cj << 8) | imask).
 * Returns the number of super-clusters, or -(entries needed) when necap is too small. */
int ora_cluster_build(int n, const float *x, const float *y, const float *z, const double box[3], double rlist,
                      int necap, int *perm, int *scio, uint32_t *cjo) {
    int geom[10];
    if (ora_cluster_geometry(n, box, rlist, geom)) return 0;
    const int ncx = geom[0], ncy = geom[1], nzb = geom[2], mx = geom[3], my = geom[4], ncol = geom[5];
    const int nbin = geom[6], nsmax = geom[7], nslot = geom[8];
    const float L[3] = {(float)box[0], (float)box[1], (float)box[2]};
    int *bin = (int *)malloc(sizeof(int) * n), *bcnt = (int *)calloc(nbin + 1, sizeof(int));
    int *bstart = (int *)malloc(sizeof(int) * (nbin + 1));
    for (int i = 0; i < n; ++i) {
        float xw = wrapf(x[i], L[0]), yw = wrapf(y[i], L[1]), zw = wrapf(z[i], L[2]);
        if (!(isfinite(xw) && isfinite(yw) && isfinite(zw))) xw = yw = zw = 0.0f;
        int cx = (int)((xw / L[0]) * (float)ncx), cy = (int)((yw / L[1]) * (float)ncy),
            cz = (int)((zw / L[2]) * (float)nzb);
        if (cx > ncx - 1) cx = ncx - 1;
        if (cy > ncy - 1) cy = ncy - 1;
        if (cz > nzb - 1) cz = nzb - 1;
        if (cx < 0) cx = 0;
        if (cy < 0) cy = 0;
        if (cz < 0) cz = 0;
        bin[i] = (cx + ncx * cy) * nzb + cz;
        bcnt[bin[i]]++;
    }
    bstart[0] = 0;
    for (int b = 0; b < nbin; ++b) bstart[b + 1] = bstart[b] + bcnt[b];
    zid *sorted = (zid *)malloc(sizeof(zid) * (n > 0 ? n : 1));
    int *cur = (int *)malloc(sizeof(int) * nbin);
    for (int b = 0; b < nbin; ++b) cur[b] = bstart[b];
    for (int i = 0; i < n; ++i) {
        sorted[cur[bin[i]]].i = i;
        sorted[cur[bin[i]]].z = wrapf(z[i], L[2]);
        cur[bin[i]]++;
    }
    for (int b = 0; b < nbin; ++b) qsort(sorted + bstart[b], bstart[b + 1] - bstart[b], sizeof(zid), cmp_zid);
    /* columns -> super-clusters */
    int *col_sc_off = (int *)malloc(sizeof(int) * (ncol + 1)), *sc_first = (int *)malloc(sizeof(int) * nsmax);
    int *sc_n = (int *)malloc(sizeof(int) * nsmax), *sc_col = (int *)malloc(sizeof(int) * nsmax);
    int NS = 0;
    for (int c = 0; c < ncol; ++c) {
        const int c0 = bstart[c * nzb], cnt = bstart[(c + 1) * nzb] - c0;
        col_sc_off[c] = NS;
        for (int k = 0; k * 64 < cnt; ++k) {
            sc_first[NS] = c0 + 64 * k;
            sc_n[NS] = cnt - 64 * k < 64 ? cnt - 64 * k : 64;
            sc_col[NS] = c;
            ++NS;
        }
    }
    col_sc_off[ncol] = NS;
    for (int s = 0; s < nslot; ++s) perm[s] = -1;
    float *bx = (float *)malloc(sizeof(float) * nslot * 3);
    for (int s = 0; s < 3 * nslot; ++s) bx[s] = NAN;
    for (int S = 0; S < NS; ++S) {
        const int nn = sc_n[S];
        float sx[64], sy[64], sz[64];
        int hx[64], hy[64], ids[64];
        for (int t = 0; t < nn; ++t) {
            ids[t] = sorted[sc_first[S] + t].i;
            sx[t] = wrapf(x[ids[t]], L[0]);
            sy[t] = wrapf(y[ids[t]], L[1]);
            sz[t] = wrapf(z[ids[t]], L[2]);
        }
        for (int t = 0; t < nn; ++t) {
            int r = 0;
            for (int u = 0; u < nn; ++u) r += (sx[u] < sx[t]) || (sx[u] == sx[t] && u < t);
            hx[t] = r >= (nn + 1) / 2;
        }
        for (int t = 0; t < nn; ++t) {
            int m = 0, r = 0;
            for (int u = 0; u < nn; ++u)
                if (hx[u] == hx[t]) {
                    ++m;
                    r += (sy[u] < sy[t]) || (sy[u] == sy[t] && u < t);
                }
            hy[t] = r >= (m + 1) / 2;
        }
        for (int t = 0; t < nn; ++t) {
            int m = 0, r = 0;
            for (int u = 0; u < nn; ++u)
                if (hx[u] == hx[t] && hy[u] == hy[t]) {
                    ++m;
                    r += (sz[u] < sz[t]) || (sz[u] == sz[t] && u < t);
                }
            const int m0 = (m + 1) / 2, hz = r >= m0, pos = r - hz * m0;
            const int slot = 64 * S + (hx[t] * 4 + hy[t] * 2 + hz) * 8 + pos;
            perm[slot] = ids[t];
            bx[3 * slot] = sx[t];
            bx[3 * slot + 1] = sy[t];
            bx[3 * slot + 2] = sz[t];
        }
    }
    /* bounding boxes */
    const int NC = 8 * nsmax;
    float *cc = (float *)malloc(sizeof(float) * NC * 3), *ch = (float *)malloc(sizeof(float) * NC * 3);
    float *sc = (float *)malloc(sizeof(float) * nsmax * 3), *sh = (float *)malloc(sizeof(float) * nsmax * 3);
    for (int c = 0; c < NC; ++c) {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int k = 0; k < 8; ++k) {
            const int s = 8 * c + k;
            if (isnan(bx[3 * s])) continue;
            for (int d = 0; d < 3; ++d) {
                lo[d] = fminf(lo[d], bx[3 * s + d]);
                hi[d] = fmaxf(hi[d], bx[3 * s + d]);
            }
        }
        for (int d = 0; d < 3; ++d) {
            if (lo[0] == INFINITY) {
                cc[3 * c + d] = NAN;
                ch[3 * c + d] = 0.0f;
            } else {
                const float sum = lo[d] + hi[d], dif = hi[d] - lo[d];
                cc[3 * c + d] = 0.5f * sum;
                ch[3 * c + d] = 0.5f * dif;
            }
        }
    }
    for (int S = 0; S < nsmax; ++S) {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int k = 0; k < 8; ++k) {
            const int c = 8 * S + k;
            if (isnan(cc[3 * c])) continue;
            for (int d = 0; d < 3; ++d) {
                lo[d] = fminf(lo[d], cc[3 * c + d] - ch[3 * c + d]);
                hi[d] = fmaxf(hi[d], cc[3 * c + d] + ch[3 * c + d]);
            }
        }
        for (int d = 0; d < 3; ++d) {
            const float sum = lo[d] + hi[d], dif = hi[d] - lo[d];
            sc[3 * S + d] = 0.5f * sum;
            sh[3 * S + d] = 0.5f * dif;
        }
    }
    /* search in serial order: column slots (dy, dx), candidate super-clusters, j clusters */
    const float rl2 = (float)rlist * (float)rlist;
    int ne = 0;
    const int nxr = geom[9] > 0 ? (2 * mx + 1 < ncx ? 2 * mx + 1 : ncx) : 1;
    const int nyr = 2 * my + 1 < ncy ? 2 * my + 1 : ncy;
    for (int S = 0; S < NS; ++S) {
        scio[S] = ne;
        const int c = sc_col[S], cx = c % ncx, cy = c / ncx;
        const int x0 = nxr == ncx ? 0 : cx - mx, y0 = nyr == ncy ? 0 : cy - my;
        for (int k = 0; k < nxr * nyr; ++k) {
            const int dy = k / nxr, dx = k % nxr;
            const int ccx = ((x0 + dx) % ncx + ncx) % ncx, ccy = ((y0 + dy) % ncy + ncy) % ncy;
            const int col = ccx + ncx * ccy;
            int lo = col_sc_off[col];
            const int hi = col_sc_off[col + 1];
            if (lo < S) lo = S;
            for (int S2 = lo; S2 < hi; ++S2) {
                if (!(bbgap2f(sc + 3 * S, sh + 3 * S, sc + 3 * S2, sh + 3 * S2, L) < rl2)) continue;
                for (int j = 0; j < 8; ++j) {
                    const int cj = 8 * S2 + j;
                    if (isnan(cc[3 * cj])) continue;
                    uint32_t m = 0;
                    for (int a = 0; a < 8; ++a) {
                        const int ci = 8 * S + a;
                        if (cj < ci || isnan(cc[3 * ci])) continue;
                        if (bbgap2f(cc + 3 * ci, ch + 3 * ci, cc + 3 * cj, ch + 3 * cj, L) < rl2) m |= 1u << a;
                    }
                    if (m) {
                        if (ne < necap) cjo[ne] = ((uint32_t)cj << 8) | m;
                        ++ne;
                    }
                }
            }
        }
    }
    scio[NS] = ne;
    free(bin);
    free(bcnt);
    free(bstart);
    free(sorted);
    free(cur);
    free(col_sc_off);
    free(sc_first);
    free(sc_n);
    free(sc_col);
    free(bx);
    free(cc);
    free(ch);
    free(sc);
    free(sh);
    return ne > necap ? -ne : NS;
}

/* force_coordinate (src/geometry/PeriodicDisplacement.jl:21-25) in Float32. */
float ora_force_coordinate(float x, float L) {
    const float h = 0.5f * L;
    if (-h <= x && x <= h) return x;
    const float u = x / L;
    const float fl = floorf(u + 0.5f);
    const float p = L * fl;
    return x - p;
}

/* Distance-only prune of the outer list (_prune_only_kernel!, src/clusterpairs/Kernels.jl:349-394)
 * with the widened radius r_p^2 + eps (16 r_p L_max + 16 r_p^2), followed by the compaction of the
 * kept entries in list order (_compact_warp_kernel!, List.jl:719-759).  xq holds the packed force
 * coordinates and charges (4 floats per slot; padding slots above PAD_LIMIT take no part).  cjw
 * receives (cj, mask_lo | mask_hi << 8 | mark << 16) pairs at the super-cluster's outer offset; nw the
 * kept count per super-cluster.
 *
 * The periodic-path mark (bit 16) of an entry is set when its tile holds an atom within half the
 * prune buffer of a face, or when an i-atom and a j-atom lie within m = 1.01 r_p + prune buffer of
 * opposite faces of one dimension (face codes: bit 2d for +, 2d+1 for -). */
static int ora_face_code(const float *p, const float sl[3], const float wl[3]) {
    int c = 0;
    for (int k = 0; k < 3; ++k) {
        if (p[k] > sl[k]) c |= 1 << (2 * k);
        if (p[k] < -sl[k]) c |= 2 << (2 * k);
        if (fabsf(p[k]) > wl[k]) c |= 64;
    }
    return c;
}

void ora_cluster_prune(int NS, const float *xq, const int *scio, const uint32_t *cjo, const double box[3], double rp,
                       double pbuf, uint32_t *cjw, int *nw) {
    const float L[3] = {(float)box[0], (float)box[1], (float)box[2]};
    const float pb = (float)pbuf;
    const float rpf = (float)rp;
    const float rp2 = rpf * rpf;
    const float m1 = 1.01f * sqrtf(rp2);
    const float mg = m1 + pb;
    float wl[3], sl[3];
    for (int k = 0; k < 3; ++k) {
        const float hL = 0.5f * L[k], hp = 0.5f * pb;
        wl[k] = hL - hp;
        sl[k] = hL - mg;
    }
    const float iL[3] = {1.0f / L[0], 1.0f / L[1], 1.0f / L[2]};
    const float Lmax = fmaxf(L[0], fmaxf(L[1], L[2]));
    const float epsf = 1.1920929e-7f;
    const float t16 = 16.0f * sqrtf(rp2);
    const float t16L = t16 * Lmax;
    const float t16r = 16.0f * rp2;
    const float inner = t16L + t16r;
    const float rp2w = rp2 + epsf * inner;
#pragma omp parallel for schedule(dynamic, 4)
    for (int S = 0; S < NS; ++S) {
        int keep = 0;
        for (int e = scio[S]; e < scio[S + 1]; ++e) {
            const int cj = (int)(cjo[e] >> 8);
            const uint32_t imask = cjo[e] & 0xffu;
            uint32_t m[2] = {0, 0};
            int ic = 0, jc = 0;
            for (int a = 0; a < 8; ++a) {
                if (!((imask >> a) & 1u)) continue;
                for (int ti = 0; ti < 8; ++ti) {
                    const float *pi = xq + 4 * (size_t)(64 * S + 8 * a + ti);
                    if (!(pi[0] > PAD_LIMIT)) ic |= ora_face_code(pi, sl, wl);
                }
            }
            for (int tj = 0; tj < 8; ++tj) {
                const float *pj = xq + 4 * (size_t)(8 * cj + tj);
                if (!(pj[0] > PAD_LIMIT)) jc |= ora_face_code(pj, sl, wl);
            }
            int cross = 0;
            for (int k = 0; k < 3; ++k)
                if ((((ic >> (2 * k)) & 1) && ((jc >> (2 * k + 1)) & 1)) ||
                    (((ic >> (2 * k + 1)) & 1) && ((jc >> (2 * k)) & 1)))
                    cross = 1;
            const int mark = cross || ((ic | jc) & 64);
            for (int h = 0; h < 2; ++h)
                for (int a = 0; a < 8; ++a) {
                    if (!((imask >> a) & 1u)) continue;
                    int hit = 0;
                    for (int tj = 4 * h; tj < 4 * h + 4 && !hit; ++tj)
                        for (int ti = 0; ti < 8 && !hit; ++ti) {
                            const float *pi = xq + 4 * (size_t)(64 * S + 8 * a + ti);
                            const float *pj = xq + 4 * (size_t)(8 * cj + tj);
                            float d[3];
                            for (int k = 0; k < 3; ++k) {
                                const float dd = pi[k] - pj[k];
                                d[k] = fmaf(-L[k], rintf(dd * iL[k]), dd);
                            }
                            const float r2 = fmaf(d[0], d[0], fmaf(d[1], d[1], d[2] * d[2]));
                            const int real = !(pi[0] > PAD_LIMIT) && !(pj[0] > PAD_LIMIT);
                            const int ok = real && ((cj != 8 * S + a) || (tj > ti));
                            if (ok && r2 < rp2w) hit = 1;
                        }
                    if (hit) m[h] |= 1u << a;
                }
            if (m[0] | m[1]) {
                cjw[2 * (size_t)(scio[S] + keep)] = (uint32_t)cj;
                cjw[2 * (size_t)(scio[S] + keep) + 1] = m[0] | (m[1] << 8) | ((uint32_t)mark << 16);
                ++keep;
            }
        }
        nw[S] = keep;
    }
}

/* ------------------------------------------------------------------------
 * Langevin noise and BAOAB drift.
 *   Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): counter (id, stream, step low, step
 *   high), key (seed low, seed high), ten rounds with the published multipliers and Weyl key
 *   increments; four standard normals by Box-Muller of open-interval uniforms from the top 24
 *   bits (src/engine/Philox.jl:20-67).
 *   BAOAB drift B1 A1 O A2 with FP64 intermediates (_baoa_kernel!, src/engine/Langevin.jl:58-88):
 *   v1 = v + dt/(2m) f, x1 = x + dt/2 v1, c = exp(-g dt/m), r = sqrt((1-c^2)/(2 g dt m)) with the
 *   per-mass form, beta = noise * xi (Float32), v2 = c v1 + r beta, x2 = x1 + dt/2 v2, positions
 *   wrapped once into [-L/2, L/2).
 * ---------------------------------------------------------------------- */
static void ora_philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[1] = (uint32_t)p1;
        c[3] = (uint32_t)p0;
        c[0] = n0;
        c[2] = n2;
    }
}

static float ora_open01(uint32_t u) { return ((float)(u >> 8) + 0.5f) * 5.9604644775390625e-8f; }

void ora_philox_normals4(uint64_t seed, uint64_t step, uint32_t id, uint32_t stream, float *out, uint32_t *words) {
    uint32_t c[4] = {id, stream, (uint32_t)step, (uint32_t)(step >> 32)};
    ora_philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    if (words)
        for (int k = 0; k < 4; ++k) words[k] = c[k];
    for (int h = 0; h < 2; ++h) {
        const float u1 = ora_open01(c[2 * h]), u2 = ora_open01(c[2 * h + 1]);
        const float r = sqrtf(-2.0f * logf(u1));
        const double a = M_PI * (double)(2.0f * u2);
        out[2 * h] = r * (float)cos(a);
        out[2 * h + 1] = r * (float)sin(a);
    }
}

static float ora_wrap_half(float x, float L) {
    if (x >= 0.5f * L) x -= L;
    if (x < -0.5f * L) x += L;
    return x;
}

void ora_baoab_drift(int n, int dim, float *x, float *y, float *z, float *vx, float *vy, float *vz, const float *fx,
                     const float *fy, const float *fz, const float *inv_mass, float dt, float gamma, float noise,
                     uint64_t seed, uint64_t step, const double box[3]) {
    for (int i = 0; i < n; ++i) {
        float *p[3] = {x + i, y + i, dim == 3 ? z + i : NULL};
        float *v[3] = {vx + i, vy + i, dim == 3 ? vz + i : NULL};
        const float f[3] = {fx[i], fy[i], dim == 3 ? fz[i] : 0.0f};
        const double dtA = dt, imA = inv_mass[i], g = gamma;
        const double hk = dtA * imA / 2.0;
        const double c = exp(-g * dtA * imA), rr = sqrt((1.0 - c * c) * imA / (2.0 * g * dtA));
        float xi[4];
        ora_philox_normals4(seed, step, (uint32_t)(i + 1), 0u, xi, NULL);
        for (int d = 0; d < dim; ++d) {
            const double v1 = (double)*v[d] + hk * (double)f[d];
            const double x1 = (double)*p[d] + 0.5 * dtA * v1;
            const double beta = (double)(noise * xi[d]);
            const double v2 = c * v1 + rr * beta;
            *v[d] = (float)v2;
            *p[d] = ora_wrap_half((float)(x1 + 0.5 * dtA * v2), (float)box[d]);
        }
    }
}
