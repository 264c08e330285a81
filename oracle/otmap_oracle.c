/* Test infrastructure only: plain-C restatement of the reference otmap algorithm
 * (ggael/otmap, otlib/) used as the checker of the CUDA library. Each function
 * cites the reference file:line it restates. Compiled by oracle/Makefile into
 * oracle/_build/liboracle.so with -ffp-contract=off so its arithmetic matches the
 * reference's x86-64 SSE2 build operation for operation where the reference is
 * scalar. The only deliberate departure is the Laplacian solve: the reference
 * factorises the pinned pseudo-Laplacian (otsolver_2dgrid.cpp:265-360); this file
 * applies its exact pseudo-inverse through the orthonormal DCT-II basis that
 * diagonalises it (oro_poisson_dct), and keeps a dense banded Cholesky of the
 * pinned matrix (oro_poisson_pinned) for small n so the tests can check that the
 * two agree.
 */
#define _DEFAULT_SOURCE
#include "otmap_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define VID(i, j) ((j) + (i) * (n + 1))
#define FID(i, j) ((j) + (i) * n)

/* std::min / std::max semantics (NaN in the second argument yields the first) */
static double dmin(double a, double b) { return b < a ? b : a; }
static double dmax(double a, double b) { return a < b ? b : a; }

/* ------------------------------------------------------------------------- */
/* otsolver_2dgrid.cpp:47-63 */
void oro_adjust_density(int n, double* d, double max_ratio) {
  long N = (long)n * n;
  double area = 1.0 / ((double)n * (double)n); /* :97 */
  double s = 0.0;
  for (long i = 0; i < N; ++i) s += d[i];
  double I = s * area;
  for (long i = 0; i < N; ++i) d[i] /= I;
  double mn = d[0], mx = d[0];
  for (long i = 1; i < N; ++i) {
    mn = dmin(mn, d[i]);
    mx = dmax(mx, d[i]);
  }
  double ratio = dmin(max_ratio, mx / mn);
  double beta = dmax(0.0, (ratio * mn - mx) / (1.0 - ratio));
  for (long i = 0; i < N; ++i) d[i] = (d[i] + beta) / (1.0 + beta);
}

/* ------------------------------------------------------------------------- */
/* otsolver_2dgrid.cpp:362-423: interior vertices get half the sum of the two
 * adjacent face differences times n; boundary vertices the one-sided tangential
 * difference and a zero normal component; corners zero. */
void oro_vertex_gradients(int n, const double* psi, double* g) {
  double w = (double)n;
  for (int i = 1; i < n; ++i) {
    for (int j = 1; j < n; ++j) {
      double p00 = psi[FID(i - 1, j - 1)], p01 = psi[FID(i - 1, j)];
      double p10 = psi[FID(i, j - 1)], p11 = psi[FID(i, j)];
      int v = VID(i, j);
      g[2 * v + 0] = 0.5 * w * (p10 + p11 - p00 - p01);
      g[2 * v + 1] = 0.5 * w * (p01 + p11 - p00 - p10);
    }
  }
  for (int k = 1; k < n; ++k) {
    g[2 * VID(k, 0) + 0] = w * (psi[FID(k, 0)] - psi[FID(k - 1, 0)]);
    g[2 * VID(k, 0) + 1] = 0.0;
    g[2 * VID(k, n) + 0] = w * (psi[FID(k, n - 1)] - psi[FID(k - 1, n - 1)]);
    g[2 * VID(k, n) + 1] = 0.0;
    g[2 * VID(0, k) + 0] = 0.0;
    g[2 * VID(0, k) + 1] = w * (psi[FID(0, k)] - psi[FID(0, k - 1)]);
    g[2 * VID(n, k) + 0] = 0.0;
    g[2 * VID(n, k) + 1] = w * (psi[FID(n - 1, k)] - psi[FID(n - 1, k - 1)]);
  }
  int corners[4] = {VID(0, 0), VID(n, 0), VID(0, n), VID(n, n)};
  for (int c = 0; c < 4; ++c) g[2 * corners[c]] = g[2 * corners[c] + 1] = 0.0;
}

/* otsolver_2dgrid.cpp:425-447: half the cross product of the quad's diagonals */
void oro_face_areas(int n, const double* g, double* area) {
  const double e = 1.0 / (double)n;
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      int v00 = VID(i, j), v10 = VID(i + 1, j), v01 = VID(i, j + 1), v11 = VID(i + 1, j + 1);
      area[FID(i, j)] = 0.5 * ((g[2 * v11] - g[2 * v00] + e) * (g[2 * v01 + 1] - g[2 * v10 + 1] + e) -
                               (g[2 * v11 + 1] - g[2 * v00 + 1] + e) * (g[2 * v01] - g[2 * v10] - e));
    }
  }
}

/* otsolver_2dgrid.cpp:449-465 */
double oro_residual(int n, const double* psi, const double* density, double* r) {
  long N = (long)n * n;
  double area_e = 1.0 / ((double)n * (double)n);
  double* g = (double*)malloc(sizeof(double) * 2 * (size_t)(n + 1) * (n + 1));
  oro_vertex_gradients(n, psi, g);
  oro_face_areas(n, g, r);
  free(g);
  double s = 0.0;
  for (long f = 0; f < N; ++f) {
    r[f] = r[f] - area_e * density[f];
    s += r[f] * r[f];
  }
  return s / area_e;
}

/* otsolver_2dgrid.cpp:467-539: r(psi + t*dir) = r(psi) + b t + a t^2 */
void oro_line_params(int n, const double* g0, const double* gd, double* a, double* b) {
  const double e = 1.0 / (double)n;
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      int v00 = VID(i, j), v10 = VID(i + 1, j), v01 = VID(i, j + 1), v11 = VID(i + 1, j + 1);
      double diag0a_x = g0[2 * v11] - g0[2 * v00] + e;
      double diag0a_y = g0[2 * v11 + 1] - g0[2 * v00 + 1] + e;
      double diag0b_x = g0[2 * v01] - g0[2 * v10] - e;
      double diag0b_y = g0[2 * v01 + 1] - g0[2 * v10 + 1] + e;
      double dda_x = gd[2 * v11] - gd[2 * v00];
      double dda_y = gd[2 * v11 + 1] - gd[2 * v00 + 1];
      double ddb_x = gd[2 * v01] - gd[2 * v10];
      double ddb_y = gd[2 * v01 + 1] - gd[2 * v10 + 1];
      a[FID(i, j)] = 0.5 * (dda_x * ddb_y - dda_y * ddb_x);
      b[FID(i, j)] = 0.5 * (dda_x * diag0b_y - dda_y * diag0b_x + diag0a_x * ddb_y - diag0a_y * ddb_x);
    }
  }
}

/* ------------------------------------------------------------------------- */
/* Real roots of w3 t^3 + w2 t^2 + w1 t + w0 (the companion-matrix eigenproblem of
 * otsolver_2dgrid.cpp:563-572), by the closed form for a depressed cubic and two
 * Newton polishing steps. Returns the number of real roots (1 or 3). */
static double cubic_eval(const double c[4], double t) { return ((c[3] * t + c[2]) * t + c[1]) * t + c[0]; }
static double cubic_deriv(const double c[4], double t) { return (3.0 * c[3] * t + 2.0 * c[2]) * t + c[1]; }

static int cubic_real_roots(const double w[4], double roots[3]) {
  double a = w[2] / w[3], b = w[1] / w[3], c = w[0] / w[3];
  if (!isfinite(a) || !isfinite(b) || !isfinite(c)) return 0;
  double p = b - a * a / 3.0;
  double q = 2.0 * a * a * a / 27.0 - a * b / 3.0 + c;
  double disc = 0.25 * q * q + p * p * p / 27.0;
  int m;
  if (disc > 0.0) {
    double sq = sqrt(disc);
    double u = cbrt(-0.5 * q + (q <= 0.0 ? sq : -sq));
    double y = (u != 0.0) ? u - p / (3.0 * u) : 0.0;
    roots[0] = y - a / 3.0;
    m = 1;
  } else {
    double r = sqrt(dmax(0.0, -p / 3.0));
    if (r == 0.0) {
      roots[0] = roots[1] = roots[2] = -a / 3.0;
    } else {
      double arg = dmax(-1.0, dmin(1.0, -0.5 * q / (r * r * r)));
      double phi = acos(arg) / 3.0;
      for (int k = 0; k < 3; ++k) roots[k] = 2.0 * r * cos(phi - 2.0943951023931954923 * k) - a / 3.0;
    }
    m = 3;
  }
  double cc[4] = {c, b, a, 1.0};
  for (int k = 0; k < m; ++k) {
    for (int it = 0; it < 2; ++it) {
      double f = cubic_eval(cc, roots[k]), df = cubic_deriv(cc, roots[k]);
      if (df != 0.0 && isfinite(f / df)) roots[k] -= f / df;
    }
  }
  return m;
}

/* otsolver_2dgrid.cpp:563-595: among the real roots of e'(t) in [-10,10] pick the
 * one with the least quartic e(t); otherwise alpha = 0.5. */
int oro_pick_step(const double z[5], double* alpha, double* emin) {
  double w[4] = {z[1], 2.0 * z[2], 3.0 * z[3], 4.0 * z[4]};
  double roots[3];
  int m = cubic_real_roots(w, roots);
  int found = 0;
  double best_t = 0.0, rmin = 0.0;
  for (int k = 0; k < m; ++k) {
    double t = roots[k];
    if (t >= -10.0 && t <= 10.0) {
      double r = z[0] + t * (z[1] + t * (z[2] + t * (z[3] + t * z[4])));
      if (!found || r < rmin) {
        found = 1;
        best_t = t;
        rmin = r;
      }
    }
  }
  if (!found) {
    best_t = 0.5;
    rmin = z[0] + best_t * (z[1] + best_t * (z[2] + best_t * (z[3] + best_t * z[4])));
  }
  *alpha = best_t;
  *emin = rmin;
  return found;
}

/* ------------------------------------------------------------------------- */
/* otsolver_2dgrid.cpp:284-311: M = -L, 2 on the diagonal and -1/2 at each of the
 * four diagonal neighbours, indices clamped at the border (duplicates summed). */
void oro_laplacian_apply(int n, const double* x, double* y) {
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      int i1 = i == 0 ? i : i - 1, j1 = j == 0 ? j : j - 1;
      int i2 = i == n - 1 ? i : i + 1, j2 = j == n - 1 ? j : j + 1;
      y[FID(i, j)] = 2.0 * x[FID(i, j)] - 0.5 * (x[FID(i1, j1)] + x[FID(i1, j2)] + x[FID(i2, j1)] + x[FID(i2, j2)]);
    }
  }
}

/* Orthonormal DCT-II basis C[k*n+i] = s_k cos(pi (i+1/2) k / n). */
static double* dct_basis(int n) {
  double* C = (double*)malloc(sizeof(double) * (size_t)n * n);
  for (int k = 0; k < n; ++k) {
    double s = k == 0 ? sqrt(1.0 / n) : sqrt(2.0 / n);
    for (int i = 0; i < n; ++i) C[(size_t)k * n + i] = s * cos(M_PI * (i + 0.5) * k / n);
  }
  return C;
}

void oro_poisson_dct(int n, const double* r, double* d) {
  size_t N = (size_t)n * n;
  double* C = dct_basis(n);
  double* T = (double*)calloc(N, sizeof(double));
  double* U = (double*)calloc(N, sizeof(double));
  /* T[k][j] = sum_i C[k][i] r[i][j] */
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < n; ++i) {
      double c = C[(size_t)k * n + i];
      for (int j = 0; j < n; ++j) T[(size_t)k * n + j] += c * r[(size_t)i * n + j];
    }
  /* U[k][l] = sum_j T[k][j] C[l][j], divided by lambda_kl */
  for (int k = 0; k < n; ++k)
    for (int l = 0; l < n; ++l) {
      double s = 0.0;
      for (int j = 0; j < n; ++j) s += T[(size_t)k * n + j] * C[(size_t)l * n + j];
      double lam = 2.0 - 2.0 * cos(M_PI * k / n) * cos(M_PI * l / n);
      U[(size_t)k * n + l] = (k == 0 && l == 0) ? 0.0 : s / lam;
    }
  /* T[i][l] = sum_k C[k][i] U[k][l] */
  memset(T, 0, N * sizeof(double));
  for (int k = 0; k < n; ++k)
    for (int i = 0; i < n; ++i) {
      double c = C[(size_t)k * n + i];
      for (int l = 0; l < n; ++l) T[(size_t)i * n + l] += c * U[(size_t)k * n + l];
    }
  /* d[i][j] = sum_l T[i][l] C[l][j] */
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int l = 0; l < n; ++l) s += T[(size_t)i * n + l] * C[(size_t)l * n + j];
      d[(size_t)i * n + j] = s;
    }
  /* mean projection, otsolver_2dgrid.cpp:179 */
  double mean = 0.0;
  for (size_t f = 0; f < N; ++f) mean += d[f];
  mean /= (double)N;
  for (size_t f = 0; f < N; ++f) d[f] -= mean;
  free(C);
  free(T);
  free(U);
}

/* Dense banded Cholesky of the pinned matrix (otsolver_2dgrid.cpp:321: M(0,0) += |M(0,0)|*1e4),
 * bandwidth n+1 in the face ordering, then the mean projection of :179. */
int oro_poisson_pinned(int n, const double* r, double* d) {
  long N = (long)n * n, bw = n + 1;
  double* L = (double*)calloc((size_t)N * (bw + 1), sizeof(double)); /* L[i][i-k], k=0..bw */
#define LB(i, k) L[(size_t)(i) * (bw + 1) + (k)]
  double* e = (double*)calloc((size_t)N, sizeof(double));
  double* col = (double*)calloc((size_t)N, sizeof(double));
  /* fill lower band of M column by column via M e_c */
  for (long c = 0; c < N; ++c) {
    e[c] = 1.0;
    oro_laplacian_apply(n, e, col);
    e[c] = 0.0;
    for (long i = c; i < N && i - c <= bw; ++i) LB(i, i - c) = col[i];
  }
  LB(0, 0) += fabs(LB(0, 0)) * 1e4;
  for (long i = 0; i < N; ++i) {
    for (long k = bw; k >= 0; --k) {
      long j = i - k;
      if (j < 0) continue;
      double s = LB(i, k);
      for (long m = (j - bw > i - bw ? j - bw : i - bw); m < j; ++m) {
        if (m < 0) continue;
        s -= LB(i, i - m) * LB(j, j - m);
      }
      if (k == 0) {
        if (s <= 0.0) {
          free(L);
          free(e);
          free(col);
          return -1;
        }
        LB(i, 0) = sqrt(s);
      } else {
        LB(i, k) = s / LB(j, 0);
      }
    }
  }
  for (long i = 0; i < N; ++i) {
    double s = r[i];
    for (long m = (i - bw > 0 ? i - bw : 0); m < i; ++m) s -= LB(i, i - m) * d[m];
    d[i] = s / LB(i, 0);
  }
  for (long i = N - 1; i >= 0; --i) {
    double s = d[i];
    for (long m = i + 1; m < N && m - i <= bw; ++m) s -= LB(m, m - i) * d[m];
    d[i] = s / LB(i, 0);
  }
#undef LB
  double mean = 0.0;
  for (long f = 0; f < N; ++f) mean += d[f];
  mean /= (double)N;
  for (long f = 0; f < N; ++f) d[f] -= mean;
  free(L);
  free(e);
  free(col);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* otsolver_2dgrid.cpp:106-245 (the quasi-Newton loop) with
 * compute_conjugate_jacobian_beta (:248-261) and solve_1D_problem (:541-606). */
int oro_solve(int n, const double* density_in, const oro_options* opt, double* psi_out, double* fwd_xy,
              double* density_out, double* trace, int trace_cap, double* residual_out) {
  size_t N = (size_t)n * n, V = (size_t)(n + 1) * (n + 1);
  const double area_e = 1.0 / ((double)n * (double)n);
  double* rho = (double*)malloc(N * sizeof(double));
  memcpy(rho, density_in, N * sizeof(double));
  oro_adjust_density(n, rho, opt->max_ratio);

  double* xk = (double*)calloc(N, sizeof(double));
  double* xkp1 = (double*)calloc(N, sizeof(double));
  double* rkm1 = (double*)calloc(N, sizeof(double));
  double* rk = (double*)calloc(N, sizeof(double));
  double* rkp1 = (double*)calloc(N, sizeof(double));
  double* d_hat = (double*)calloc(N, sizeof(double));
  double* d = (double*)calloc(N, sizeof(double));
  double* a = (double*)calloc(N, sizeof(double));
  double* b = (double*)calloc(N, sizeof(double));
  double* tmp = (double*)calloc(N, sizeof(double));
  double* reps = (double*)calloc(N, sizeof(double));
  double* g0 = (double*)calloc(2 * V, sizeof(double)); /* :126, gradients at psi = 0 */
  double* gd = (double*)calloc(2 * V, sizeof(double));

  double beta = 0.0, alpha = 0.0;
  double residual = oro_residual(n, xk, rho, rkp1); /* :146 */
  int it = 0;
  while (it < opt->max_iter && residual > opt->threshold) { /* :160 */
    double* t;
    t = rkm1; rkm1 = rk; rk = rkp1; rkp1 = t; /* :167-168 */

    oro_poisson_dct(n, rk, d_hat); /* :175-179 */
    double nd = 0.0;
    for (size_t f = 0; f < N; ++f) nd += d_hat[f] * d_hat[f];
    if (sqrt(nd) <= 2.0 * DBL_MIN) break; /* :182-183 */

    if (it < 1 || !opt->beta_cj) { /* :191-200 */
      memcpy(d, d_hat, N * sizeof(double));
    } else {
      double eps = alpha / 2.0; /* :255-260 */
      for (size_t f = 0; f < N; ++f) tmp[f] = xk[f] - eps * d_hat[f];
      oro_residual(n, tmp, rho, reps);
      double num = 0.0, den = 0.0;
      for (size_t f = 0; f < N; ++f) {
        double jd = rk[f] - rkm1[f];
        num += jd * (reps[f] - rk[f]);
        den += jd * jd;
      }
      beta = dmax(-1.0, num / den / eps * alpha);
      for (size_t f = 0; f < N; ++f) d[f] = d_hat[f] + beta * d[f];
    }

    /* solve_1D_problem */
    oro_vertex_gradients(n, d, gd);
    oro_line_params(n, g0, gd, a, b);
    double z[5] = {residual * area_e, 0, 0, 0, 0};
    double s_br = 0, s_bb = 0, s_ar = 0, s_ab = 0, s_aa = 0;
    for (size_t f = 0; f < N; ++f) {
      s_br += b[f] * rk[f];
      s_bb += b[f] * b[f];
      s_ar += a[f] * rk[f];
      s_ab += a[f] * b[f];
      s_aa += a[f] * a[f];
    }
    z[1] = 2.0 * s_br;
    z[2] = s_bb + 2 * s_ar;
    z[3] = 2.0 * s_ab;
    z[4] = s_aa;
    double rmin;
    oro_pick_step(z, &alpha, &rmin);
    for (size_t f = 0; f < N; ++f) xkp1[f] = xk[f] + alpha * d[f];       /* :599 */
    for (size_t v = 0; v < 2 * V; ++v) g0[v] += alpha * gd[v];           /* :603 */
    for (size_t f = 0; f < N; ++f) rkp1[f] = a[f] * (alpha * alpha) + b[f] * alpha + rk[f]; /* :604 */
    residual = rmin / area_e;                                            /* :605 */
    t = xk; xk = xkp1; xkp1 = t;                                         /* :214 */

    if (trace && it < trace_cap) {
      double dn = 0.0, linf = -INFINITY;
      for (size_t f = 0; f < N; ++f) {
        dn += d[f] * d[f];
        linf = dmax(linf, rkp1[f]);
      }
      trace[5 * it + 0] = alpha;
      trace[5 * it + 1] = beta;
      trace[5 * it + 2] = sqrt(dn);
      trace[5 * it + 3] = residual;
      trace[5 * it + 4] = linf / area_e;
    }
    ++it;
  }

  if (fwd_xy) { /* :222-227 */
    double* g = (double*)malloc(2 * V * sizeof(double));
    oro_vertex_gradients(n, xk, g);
    for (int i = 0; i <= n; ++i)
      for (int j = 0; j <= n; ++j) {
        int v = VID(i, j);
        fwd_xy[2 * v] = (double)i * (1.0 / (double)n) + g[2 * v];
        fwd_xy[2 * v + 1] = (double)j * (1.0 / (double)n) + g[2 * v + 1];
      }
    free(g);
  }
  if (psi_out) memcpy(psi_out, xk, N * sizeof(double));
  if (density_out) memcpy(density_out, rho, N * sizeof(double));
  if (residual_out) *residual_out = residual;
  free(rho); free(xk); free(xkp1); free(rkm1); free(rk); free(rkp1); free(d_hat); free(d);
  free(a); free(b); free(tmp); free(reps); free(g0); free(gd);
  return it;
}

/* ------------------------------------------------------------------------- */
/* utils/eigen_addons.h:15-22 */
static double cross2(double ax, double ay, double bx, double by) { return ax * by - ay * bx; }
static double signed_area3(const double* a, const double* b, const double* c) {
  return 0.5 * cross2(b[0] - a[0], b[1] - a[1], c[0] - a[0], c[1] - a[1]);
}

/* utils/mesh_utils.h:18-25 */
static void bary_in_triangle(const double* q, const double* p0, const double* p1, const double* p2, double* uv) {
  double q2x = q[0] - p2[0], q2y = q[1] - p2[1];
  double eux = p1[0] - p2[0], euy = p1[1] - p2[1];
  double evx = p0[0] - p2[0], evy = p0[1] - p2[1];
  double area2 = cross2(evx, evy, eux, euy);
  uv[0] = cross2(q2x, q2y, eux, euy) / area2;
  uv[1] = cross2(evx, evy, q2x, q2y) / area2;
}

/* utils/mesh_utils.cpp:18-59 */
int oro_bilinear_in_quad(const double q[2], const double p[8], double* pu, double* pv) {
  const double *p0 = p, *p1 = p + 2, *p2 = p + 4, *p3 = p + 6;
  double A0 = signed_area3(q, p0, p1);
  double A1 = signed_area3(q, p1, p2);
  double A2 = signed_area3(q, p2, p3);
  double A3 = signed_area3(q, p3, p0);
  double B0 = signed_area3(q, p3, p1);
  double B1 = signed_area3(q, p0, p2);
  double B3 = signed_area3(q, p2, p0);
  double D = B0 * B0 + B1 * B1 + 2 * A0 * A2 + 2 * A1 * A3;
  if (D < 0) return 0;
  double E0 = 2 * A0 - B0 - B1 + sqrt(D);
  double E3 = 2 * A3 - B3 - B0 + sqrt(D);
  double zero = 4 * DBL_MIN;
  double v = fabs(A0) <= zero ? 0 : 2 * A0 / E0;
  double u = fabs(A3) <= zero ? 0 : 2 * A3 / E3;
  double E0p = 2 * A0 - B0 - B1 - sqrt(D);
  double E3p = 2 * A3 - B3 - B0 - sqrt(D);
  double v_alt = fabs(A0) <= zero ? 0 : 2 * A0 / E0p;
  double u_alt = fabs(A3) <= zero ? 0 : 2 * A3 / E3p;
  double eps = sqrt(DBL_EPSILON);
  if (fabs(u) < eps) u = 0;
  if (fabs(v) < eps) v = 0;
  if (fabs(u - 1.) < eps) u = 1;
  if (fabs(v - 1.) < eps) v = 1;
  if (fabs(u_alt) < eps) u_alt = 0;
  if (fabs(v_alt) < eps) v_alt = 0;
  if (fabs(u_alt - 1.) < eps) u_alt = 1;
  if (fabs(v_alt - 1.) < eps) v_alt = 1;
  if ((u < 0 || v < 0 || u > 1 || v > 1) && (u_alt >= 0 && v_alt >= 0 && u_alt <= 1 && v_alt <= 1)) {
    double t = u; u = u_alt; u_alt = t;
    t = v; v = v_alt; v_alt = t;
  }
  *pu = u;
  *pv = v;
  return 1;
}

/* utils/mesh_utils.cpp:76-88 */
int oro_bilinear_weights(const double q[2], const double p[8], double w[4]) {
  double eps = 4 * DBL_EPSILON;
  double u, v;
  if (!oro_bilinear_in_quad(q, p, &u, &v)) return 0;
  w[0] = (1. - u) * (1 - v);
  w[1] = (u) * (1. - v);
  w[2] = (u) * (v);
  w[3] = (1. - u) * (v);
  for (int k = 0; k < 4; ++k) {
    if (fabs(w[k]) <= eps) w[k] = 0;
    else if (fabs(w[k] - 1.) <= eps) w[k] = 1;
  }
  return 1;
}

/* utils/mesh_utils.cpp:62-74 */
int oro_inside_quad(const double q[2], const double p[8]) {
  double eps = 1e-8, uv[2];
  bary_in_triangle(q, p, p + 2, p + 4, uv);
  if (uv[0] >= -eps && uv[1] >= -eps && uv[0] + uv[1] <= 1. + eps) return 1;
  bary_in_triangle(q, p, p + 4, p + 6, uv);
  if (uv[0] >= -eps && uv[1] >= -eps && uv[0] + uv[1] <= 1. + eps) return 1;
  return 0;
}

/* Quad corners of face f = j + i*n: (i,j), (i+1,j), (i+1,j+1), (i,j+1)
 * (utils/mesh_utils.cpp:110-121, face vertex order of Surface_mesh::add_quad). */
static void face_corners(int n, const double* xy, int f, double p[8], int vid[4]) {
  int i = f / n, j = f % n;
  int v[4] = {VID(i, j), VID(i + 1, j), VID(i + 1, j + 1), VID(i, j + 1)};
  for (int k = 0; k < 4; ++k) {
    p[2 * k] = xy[2 * v[k]];
    p[2 * k + 1] = xy[2 * v[k] + 1];
    if (vid) vid[k] = v[k];
  }
}

/* ------------------------------------------------------------------------- */
/* utils/bvh2d.h:31-39, bvh2d.cpp:29-64, 167-242 */
typedef struct {
  double mn[2], mx[2];
  int first; /* first child (inner) or first face slot (leaf) */
  int nb;
  int leaf;
} oro_node;

struct oro_bvh {
  int n;
  const double* xy;
  double* cen; /* centroids, permuted together with faces */
  int* faces;
  oro_node* nodes;
  int nnodes, cap;
};

static int bvh_split(oro_bvh* b, int start, int end, int dim, float split_value) {
  int l = start, r = end - 1;
  while (l < r) {
    while (l < end && b->cen[2 * l + dim] < split_value) ++l;
    while (r >= start && b->cen[2 * r + dim] >= split_value) --r;
    if (l >= r) break;
    double c0 = b->cen[2 * l], c1 = b->cen[2 * l + 1];
    b->cen[2 * l] = b->cen[2 * r];
    b->cen[2 * l + 1] = b->cen[2 * r + 1];
    b->cen[2 * r] = c0;
    b->cen[2 * r + 1] = c1;
    int tf = b->faces[l];
    b->faces[l] = b->faces[r];
    b->faces[r] = tf;
    ++l;
    --r;
  }
  /* when l == end both branches below return end; the read past the range is avoided */
  if (l >= end) return end;
  return b->cen[2 * l + dim] <= split_value ? (end < l + 1 ? end : l + 1) : l;
}

static void bvh_node(oro_bvh* b, int id, int start, int end, int level, int target, int max_depth) {
  double mn[2] = {INFINITY, INFINITY}, mx[2] = {-INFINITY, -INFINITY};
  for (int i = start; i < end; ++i) {
    double p[8];
    face_corners(b->n, b->xy, b->faces[i], p, NULL);
    for (int k = 0; k < 4; ++k)
      for (int c = 0; c < 2; ++c) {
        mn[c] = dmin(mn[c], p[2 * k + c]);
        mx[c] = dmax(mx[c], p[2 * k + c]);
      }
  }
  oro_node* nd = &b->nodes[id];
  double diag[2] = {mx[0] - mn[0], mx[1] - mn[1]};
  for (int c = 0; c < 2; ++c) {
    double en = diag[c] * (2. * DBL_EPSILON) + DBL_EPSILON;
    nd->mn[c] = mn[c] - en;
    nd->mx[c] = mx[c] + en;
  }
  if (end - start <= target || level >= max_depth) {
    nd->leaf = 1;
    nd->first = start;
    nd->nb = end - start > 0 ? end - start : 0;
    return;
  }
  nd->leaf = 0;
  int dim = diag[1] > diag[0] ? 1 : 0;
  float split_value = (float)(0.5 * (nd->mx[dim] + nd->mn[dim]));
  int mid = bvh_split(b, start, end, dim, split_value);
  if (mid == start || mid == end) {
    nd->leaf = 1;
    nd->first = start;
    nd->nb = end - start > 0 ? end - start : 0;
    return;
  }
  if (b->nnodes + 2 > b->cap) {
    b->cap = b->cap * 2 + 2;
    b->nodes = (oro_node*)realloc(b->nodes, sizeof(oro_node) * (size_t)b->cap);
  }
  int child = b->nnodes;
  b->nodes[id].first = child;
  b->nnodes += 2;
  bvh_node(b, child, start, mid, level + 1, target, max_depth);
  bvh_node(b, child + 1, mid, end, level + 1, target, max_depth);
}

oro_bvh* oro_bvh_build(int n, const double* fwd_xy) {
  oro_bvh* b = (oro_bvh*)calloc(1, sizeof(oro_bvh));
  int N = n * n;
  b->n = n;
  b->xy = fwd_xy;
  b->cen = (double*)malloc(sizeof(double) * 2 * (size_t)N);
  b->faces = (int*)malloc(sizeof(int) * (size_t)N);
  for (int f = 0; f < N; ++f) {
    double p[8];
    face_corners(n, fwd_xy, f, p, NULL);
    double cx = 0, cy = 0;
    for (int k = 0; k < 4; ++k) {
      cx += p[2 * k];
      cy += p[2 * k + 1];
    }
    b->cen[2 * f] = cx / 4;
    b->cen[2 * f + 1] = cy / 4;
    b->faces[f] = f;
  }
  b->cap = 1024;
  b->nodes = (oro_node*)malloc(sizeof(oro_node) * (size_t)b->cap);
  b->nnodes = 1;
  bvh_node(b, 0, 0, N, 0, 4, 24);
  return b;
}

/* The face order the build leaves in its face array (bvh2d.cpp:167-242) and, per face,
 * the enlarged box of its leaf: faces_out[pos] = face, leaf_box[4 f .. 4 f + 3]. */
void oro_bvh_order(int n, const double* fwd_xy, int* faces_out, double* leaf_box) {
  oro_bvh* b = oro_bvh_build(n, fwd_xy);
  int N = n * n;
  for (int p = 0; p < N; ++p) faces_out[p] = b->faces[p];
  for (int k = 0; k < b->nnodes; ++k) {
    const oro_node* nd = &b->nodes[k];
    if (!nd->leaf) continue;
    for (int p = nd->first; p < nd->first + nd->nb; ++p) {
      int f = b->faces[p];
      leaf_box[4 * f] = nd->mn[0];
      leaf_box[4 * f + 1] = nd->mn[1];
      leaf_box[4 * f + 2] = nd->mx[0];
      leaf_box[4 * f + 3] = nd->mx[1];
    }
  }
  oro_bvh_free(b);
}

void oro_bvh_free(oro_bvh* b) {
  if (!b) return;
  free(b->cen);
  free(b->faces);
  free(b->nodes);
  free(b);
}

static int box_contains(const oro_node* nd, const double* q) {
  return nd->mn[0] <= q[0] && nd->mn[1] <= q[1] && q[0] <= nd->mx[0] && q[1] <= nd->mx[1];
}

/* bvh2d.cpp:94-162 with stop_at_first = false */
static void bvh_intersect(const oro_bvh* b, int id, const double* q, int cap, int* count, int* faces, double* bary) {
  const oro_node* nd = &b->nodes[id];
  if (nd->leaf) {
    for (int i = nd->first; i < nd->first + nd->nb; ++i) {
      double p[8], w[4];
      face_corners(b->n, b->xy, b->faces[i], p, NULL);
      if (oro_inside_quad(q, p) && oro_bilinear_weights(q, p, w)) {
        if (w[0] <= 1.0f && w[1] <= 1.0f && w[2] <= 1.0f && w[3] <= 1.0f && w[0] >= 0.0f && w[1] >= 0.0f &&
            w[2] >= 0.0f && w[3] >= 0.0f) {
          if (*count < cap) {
            faces[*count] = b->faces[i];
            for (int k = 0; k < 4; ++k) bary[4 * *count + k] = w[k];
          }
          ++*count;
        }
      }
    }
  } else {
    int c1 = nd->first, c2 = nd->first + 1;
    if (box_contains(&b->nodes[c1], q)) bvh_intersect(b, c1, q, cap, count, faces, bary);
    if (box_contains(&b->nodes[c2], q)) bvh_intersect(b, c2, q, cap, count, faces, bary);
  }
}

int oro_bvh_query_all(const oro_bvh* b, const double q[2], int cap, int* faces, double* bary) {
  int count = 0;
  if (box_contains(&b->nodes[0], q)) bvh_intersect(b, 0, q, cap, &count, faces, bary);
  return count;
}

/* transport_map.cpp:50-102 (fast_mode = false) and :105-128 */
long oro_apply_inverse(int n, const double* fwd_xy, const double* density, double* pts, long P, int* face_out,
                       int* nhits_out) {
  enum { CAP = 16 };
  oro_bvh* b = oro_bvh_build(n, fwd_xy);
  long missing = 0;
  for (long i = 0; i < P; ++i) {
    double q[2] = {dmin(dmax(pts[2 * i], 0.), 1.), dmin(dmax(pts[2 * i + 1], 0.), 1.)}; /* :53 */
    int faces[CAP];
    double bary[4 * CAP];
    int nh = oro_bvh_query_all(b, q, CAP, faces, bary);
    if (nhits_out) nhits_out[i] = nh;
    if (nh == 0) {
      /* the reference reads hits[0] of an empty list here (transport_map.cpp:67-70) */
      ++missing;
      if (face_out) face_out[i] = -1;
      pts[2 * i] = NAN;
      pts[2 * i + 1] = NAN;
      continue;
    }
    int f = faces[0];
    const double* w = bary; /* weights always from the first hit (:81) */
    if (nh > 1) {
      double best_area = density[f];
      for (int k = 1; k < nh && k < CAP; ++k) {
        if (density[faces[k]] > best_area) {
          f = faces[k];
          best_area = density[faces[k]] > best_area; /* becomes 0/1 (:82) */
        }
      }
    }
    double p[8];
    int vid[4];
    face_corners(n, fwd_xy, f, p, vid);
    /* origin mesh vertex v = (i/n, j/n) */
    double rx = 0, ry = 0;
    for (int k = 0; k < 4; ++k) {
      int vi = vid[k] / (n + 1), vj = vid[k] % (n + 1);
      double ox = (double)vi * (1.0 / (double)n), oy = (double)vj * (1.0 / (double)n);
      if (k == 0) {
        rx = w[0] * ox;
        ry = w[0] * oy;
      } else {
        rx += w[k] * ox;
        ry += w[k] * oy;
      }
    }
    pts[2 * i] = rx;
    pts[2 * i + 1] = ry;
    if (face_out) face_out[i] = f;
  }
  oro_bvh_free(b);
  return missing;
}

/* ------------------------------------------------------------------------- */
/* utils/rasterizer.cpp:162-209 (quad rasterize_face) and :188-236 (PerFace branch).
 * A pixel whose bilinear solve has D < 0 counts as outside (the reference leaves the
 * weights uninitialised there). */
void oro_rasterize(int n, const double* xy, const double* density, int rows, int cols, int stale_weights,
                   double* img) {
  float scale = (float)(1. / (double)((long)n * n));
  double stale[4] = {0, 0, 0, 0};
  memset(img, 0, sizeof(double) * (size_t)rows * cols);
  for (int f = 0; f < n * n; ++f) {
    double p[8];
    face_corners(n, xy, f, p, NULL);
    double in_mass = scale * (density ? density[f] : 1.0);
    double area = fabs(signed_area3(p, p + 2, p + 4) + signed_area3(p, p + 4, p + 6));
    double ulx = dmin(dmin(dmin(p[0], p[2]), p[4]), p[6]);
    double uly = dmin(dmin(dmin(p[1], p[3]), p[5]), p[7]);
    double lrx = dmax(dmax(dmax(p[0], p[2]), p[4]), p[6]);
    double lry = dmax(dmax(dmax(p[1], p[3]), p[5]), p[7]);
    int x0 = (int)(ulx * (double)cols), y0 = (int)(uly * (double)rows);
    if (x0 < 0) x0 = 0;
    if (y0 < 0) y0 = 0;
    int x1 = (int)(lrx * (double)cols) + 1, y1 = (int)(lry * (double)rows) + 1;
    if (x1 > cols) x1 = cols;
    if (y1 > rows) y1 = rows;
    for (int y = y0; y < y1; ++y)
      for (int x = x0; x < x1; ++x) {
        double q[2] = {((double)x + 0.5) / (double)cols, ((double)y + 0.5) / (double)rows};
        double w[4];
        if (oro_bilinear_weights(q, p, w)) {
          memcpy(stale, w, sizeof w);
        } else {
          if (!stale_weights) continue;
          memcpy(w, stale, sizeof w);
        }
        if (w[0] <= 1.0f && w[1] <= 1.0f && w[2] <= 1.0f && w[3] <= 1.0f && w[0] >= 0.0f && w[1] >= 0.0f &&
            w[2] >= 0.0f && w[3] >= 0.0f)
          img[(size_t)y * cols + x] = in_mass / area;
      }
  }
}

/* ------------------------------------------------------------------------- */
/* rasterize_image on an indexed face set of triangles and quads, both options
 * (rasterizer.cpp:36-58 BarycentricTransform, 86-185 rasterize_face, 188-302).
 * mode 0 = RIO_PerVertexDensity, 1 = RIO_PerFaceDensity. Faces in index order, the
 * last face covering a pixel wins. PerVertex: per-vertex float accumulation of
 * 1/|area| in face order, value = float(scale) * value / count, and the fragment
 * value is the float sum of (vertex 0's value * float(weight)) over the corners
 * (the reference's interpolation loop reads verts[0] each time). */
static void tri_bary(const double q[2], const double p[8], double w[4]) {
  double m00 = p[0] - p[4], m10 = p[1] - p[5]; /* column s1 - s3 */
  double m01 = p[2] - p[4], m11 = p[3] - p[5]; /* column s2 - s3 */
  double invdet = 1.0 / (m00 * m11 - m10 * m01);
  double t00 = m11 * invdet, t10 = -m10 * invdet, t01 = -m01 * invdet, t11 = m00 * invdet;
  double vx = q[0] - p[4], vy = q[1] - p[5];
  double b0 = t00 * vx + t01 * vy, b1 = t10 * vx + t11 * vy;
  w[0] = b0;
  w[1] = b1;
  w[2] = 1.0 - b0 - b1;
  w[3] = 0.0;
}

static int load_mesh_face(const double* xy, const int* start, const int* idx, int f, double p[8], int vid[4]) {
  int c = start[f + 1] - start[f];
  for (int k = 0; k < 4; ++k) {
    int v = idx[start[f] + (k < c ? k : c - 1)];
    vid[k] = v;
    p[2 * k] = xy[2 * v];
    p[2 * k + 1] = xy[2 * v + 1];
  }
  return c;
}

static double mesh_face_area(const double p[8], int c) {
  if (c == 3) return fabs(signed_area3(p, p + 2, p + 4));
  return fabs(signed_area3(p, p + 2, p + 4) + signed_area3(p, p + 4, p + 6));
}

void oro_rasterize_mesh(int nv, const double* xy, int nf, const int* start, const int* idx, const double* density,
                        int cells, int rows, int cols, int mode, int stale_weights, double* img) {
  float scale = (float)(1. / (double)(density ? cells : nf));
  float* value = NULL;
  double stale[4] = {0, 0, 0, 0};
  memset(img, 0, sizeof(double) * (size_t)rows * cols);
  if (mode == 0) {
    value = (float*)calloc((size_t)(nv > 0 ? nv : 1), sizeof(float));
    double* div = (double*)calloc((size_t)(nv > 0 ? nv : 1), sizeof(double));
    for (int f = 0; f < nf; ++f) {
      double p[8];
      int vid[4];
      int c = load_mesh_face(xy, start, idx, f, p, vid);
      double area = mesh_face_area(p, c);
      for (int k = start[f]; k < start[f + 1]; ++k) {
        value[idx[k]] = (float)((double)value[idx[k]] + 1. / area);
        div[idx[k]] += 1.;
      }
    }
    for (int v = 0; v < nv; ++v) value[v] = (float)((double)(scale * value[v]) / div[v]);
    free(div);
  }
  for (int f = 0; f < nf; ++f) {
    double p[8];
    int vid[4];
    int c = load_mesh_face(xy, start, idx, f, p, vid);
    double in_mass = scale * (density ? density[f] : 1.0);
    double fvalue = in_mass / mesh_face_area(p, c);
    double ulx = dmin(dmin(dmin(p[0], p[2]), p[4]), p[6]);
    double uly = dmin(dmin(dmin(p[1], p[3]), p[5]), p[7]);
    double lrx = dmax(dmax(dmax(p[0], p[2]), p[4]), p[6]);
    double lry = dmax(dmax(dmax(p[1], p[3]), p[5]), p[7]);
    int x0 = (int)(ulx * (double)cols), y0 = (int)(uly * (double)rows);
    if (x0 < 0) x0 = 0;
    if (y0 < 0) y0 = 0;
    int x1 = (int)(lrx * (double)cols) + 1, y1 = (int)(lry * (double)rows) + 1;
    if (x1 > cols) x1 = cols;
    if (y1 > rows) y1 = rows;
    for (int y = y0; y < y1; ++y)
      for (int x = x0; x < x1; ++x) {
        double q[2] = {((double)x + 0.5) / (double)cols, ((double)y + 0.5) / (double)rows};
        double w[4];
        if (c == 3) {
          tri_bary(q, p, w);
        } else if (oro_bilinear_weights(q, p, w)) {
          memcpy(stale, w, sizeof w);
        } else {
          if (!stale_weights) continue;
          memcpy(w, stale, sizeof w);
        }
        if (!(w[0] <= 1.0f && w[1] <= 1.0f && w[2] <= 1.0f && w[3] <= 1.0f && w[0] >= 0.0f && w[1] >= 0.0f &&
              w[2] >= 0.0f && w[3] >= 0.0f))
          continue;
        if (mode == 0) {
          float v0 = value[vid[0]], acc = 0.0f;
          for (int k = 0; k < c; ++k) acc = acc + v0 * (float)w[k];
          img[(size_t)y * cols + x] = (double)acc;
        } else {
          img[(size_t)y * cols + x] = fvalue;
        }
      }
  }
  free(value);
}

void oro_grid_faces(int n, int* start, int* idx) {
  for (int f = 0; f < n * n; ++f) {
    int i = f / n, j = f % n;
    start[f] = 4 * f;
    idx[4 * f] = VID(i, j);
    idx[4 * f + 1] = VID(i + 1, j);
    idx[4 * f + 2] = VID(i + 1, j + 1);
    idx[4 * f + 3] = VID(i, j + 1);
  }
  start[n * n] = 4 * n * n;
}

/* interpolate (apps/barycenters.cpp:250-276): out = sum_k w_k mesh_k, left to right. */
void oro_mesh_blend(long V2, int count, const double* const* meshes, const double* w, double* out) {
  for (long t = 0; t < V2; ++t) {
    double acc = w[0] * meshes[0][t];
    for (int k = 1; k < count; ++k) acc = acc + w[k] * meshes[k][t];
    out[t] = acc;
  }
}

/* prune_empty_faces (mesh_utils.cpp:124-141) followed by Surface_mesh's
 * garbage_collection (Surface_mesh.cpp:1975-2110): faces with zero density are
 * removed, then every vertex left without a face; survivors are compacted by the
 * two-cursor exchange of garbage_collection (vertices and faces separately). A
 * triangulated grid (nf = 2 cells) reads cell f/2 for face f. */
static int compact(int count, const char* dead_in, int* newpos) {
  char* dead = (char*)malloc((size_t)(count > 0 ? count : 1));
  int* at = (int*)malloc(sizeof(int) * (size_t)(count > 0 ? count : 1));
  for (int i = 0; i < count; ++i) {
    dead[i] = dead_in[i];
    at[i] = i;
    newpos[i] = -1;
  }
  int kept = 0;
  if (count > 0) {
    int i0 = 0, i1 = count - 1;
    for (;;) {
      while (!dead[i0] && i0 < i1) ++i0;
      while (dead[i1] && i0 < i1) --i1;
      if (i0 >= i1) break;
      char td = dead[i0];
      dead[i0] = dead[i1];
      dead[i1] = td;
      int ta = at[i0];
      at[i0] = at[i1];
      at[i1] = ta;
    }
    kept = dead[i0] ? i0 : i0 + 1;
  }
  for (int pos = 0; pos < kept; ++pos) newpos[at[pos]] = pos;
  free(dead);
  free(at);
  return kept;
}

int oro_prune_empty_faces(int nv, const double* xy, int nf, const int* start, const int* idx, const double* density,
                          int cells, int* nv_out, double* xy_out, int* nf_out, int* start_out, int* idx_out) {
  char* fdead = (char*)calloc((size_t)(nf > 0 ? nf : 1), 1);
  char* touched = (char*)calloc((size_t)(nv > 0 ? nv : 1), 1);
  char* live = (char*)calloc((size_t)(nv > 0 ? nv : 1), 1);
  char* vdead = (char*)calloc((size_t)(nv > 0 ? nv : 1), 1);
  int* fpos = (int*)malloc(sizeof(int) * (size_t)(nf > 0 ? nf : 1));
  int* vpos = (int*)malloc(sizeof(int) * (size_t)(nv > 0 ? nv : 1));
  int* from = (int*)malloc(sizeof(int) * (size_t)(nf > 0 ? nf : 1));
  const int pairs = (nf == 2 * cells);
  for (int f = 0; f < nf; ++f) {
    fdead[f] = density[pairs ? f / 2 : f] == 0;
    for (int k = start[f]; k < start[f + 1]; ++k) {
      if (fdead[f])
        touched[idx[k]] = 1;
      else
        live[idx[k]] = 1;
    }
  }
  for (int v = 0; v < nv; ++v) vdead[v] = touched[v] && !live[v];
  *nv_out = compact(nv, vdead, vpos);
  *nf_out = compact(nf, fdead, fpos);
  for (int v = 0; v < nv; ++v)
    if (vpos[v] >= 0) {
      xy_out[2 * vpos[v]] = xy[2 * v];
      xy_out[2 * vpos[v] + 1] = xy[2 * v + 1];
    }
  for (int f = 0; f < nf; ++f)
    if (fpos[f] >= 0) from[fpos[f]] = f;
  int k = 0;
  start_out[0] = 0;
  for (int q = 0; q < *nf_out; ++q) {
    int f = from[q];
    for (int t = start[f]; t < start[f + 1]; ++t) idx_out[k++] = vpos[idx[t]];
    start_out[q + 1] = k;
  }
  free(from);
  free(fdead);
  free(touched);
  free(live);
  free(vdead);
  free(fpos);
  free(vpos);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* sample_transportmap_to_image (stochastic_rasterizer.cpp:19-88) with the library's
 * counter-based generator in place of std::rand(): the splitmix64 output function
 * (Steele, Lea & Flood, OOPSLA 2014) of a (seed, face, sample, draw) key. */
static unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

static double splat_uniform(unsigned long long key, long sample, int draw) {
  unsigned long long x = mix64(key + (unsigned long long)(2 * sample + draw + 1) * 0x9e3779b97f4a7c15ULL);
  return (double)(x >> 11) * 0x1.0p-53;
}

void oro_sample_image(int nv, const double* xy, int nf, const int* start, const int* idx, const int* spf,
                      unsigned long long seed, int rows, int cols, double* img) {
  (void)nv;
  memset(img, 0, sizeof(double) * (size_t)rows * cols);
  const double dx = 1. / (double)cols, dy = 1. / (double)rows;
  for (int f = 0; f < nf; ++f) {
    double p[8];
    int vid[4];
    int c = load_mesh_face(xy, start, idx, f, p, vid);
    unsigned long long key = mix64(seed ^ mix64((unsigned long long)(f + 1) * 0xd1b54a32d192ed03ULL));
    for (long s = 0; s < spf[f]; ++s) {
      double px, py;
      if (c == 3) {
        double r1 = sqrt(splat_uniform(key, s, 0)), r2 = splat_uniform(key, s, 1);
        double b0 = 1. - r1, b1 = r1 * (1. - r2), b2 = r1 * r2;
        px = b0 * p[0] + b1 * p[2] + b2 * p[4];
        py = b0 * p[1] + b1 * p[3] + b2 * p[5];
      } else {
        double u = splat_uniform(key, s, 0), v = splat_uniform(key, s, 1);
        double w0 = (1. - u) * (1 - v), w1 = (u) * (1 - v), w2 = (u) * (v), w3 = (1. - u) * (v);
        px = w0 * p[0] + w1 * p[2] + w2 * p[4] + w3 * p[6];
        py = w0 * p[1] + w1 * p[3] + w2 * p[5] + w3 * p[7];
      }
      if (!(px >= 0 && py >= 0 && px <= 1 && py <= 1)) continue;
      int pi = (int)(py / dy), pj = (int)(px / dx);
      if (pi < rows && pj < cols) img[(size_t)pi * cols + pj] += 1.0;
    }
  }
}

/* ------------------------------------------------------------------------- */
/* GridBasedTransportSolver::compute_transport_cost (otsolver_2dgrid.cpp:608-640) on
 * vertex displacements g (V x 2 AoS); returns the sequential sum of the per-face costs. */
double oro_grid_transport_cost(int n, const double* g, const double* density, double* per_face) {
  const double e2 = 1.0 / ((double)n * (double)n);
  const double z1 = sqrt(1. / 3.) / 2. + 0.5, z2 = -sqrt(1. / 3.) / 2. + 0.5;
  const double zu[4] = {z1, z1, z2, z2}, zv[4] = {z1, z2, z2, z1};
  double total = 0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      int c[4] = {VID(i, j), VID(i + 1, j), VID(i + 1, j + 1), VID(i, j + 1)};
      double acc = 0;
      for (int q = 0; q < 4; ++q) {
        double u = zu[q], v = zv[q];
        double a0 = (1 - u) * (1 - v), a1 = u * (1 - v), a2 = u * v, a3 = (1 - u) * v;
        double x = a0 * g[2 * c[0]] + a1 * g[2 * c[1]] + a2 * g[2 * c[2]] + a3 * g[2 * c[3]];
        double y = a0 * g[2 * c[0] + 1] + a1 * g[2 * c[1] + 1] + a2 * g[2 * c[2] + 1] + a3 * g[2 * c[3] + 1];
        acc = q == 0 ? x * x + y * y : acc + (x * x + y * y);
      }
      int f = j + i * n;
      double cost = density[f] * e2 * acc / 4.;
      if (per_face) per_face[f] = cost;
      total += cost;
    }
  return total;
}

/* ------------------------------------------------------------------------- */
/* transport_map.cpp:131-215 for a quad grid mesh: the face count equals the
 * density size, so the reference takes its per-triangle branch (:184-199) on the
 * first three vertices of each face's circulation, which for a Surface_mesh quad
 * (v0,v1,v2,v3) starting at its last halfedge are (v3, v0, v1). */
double oro_transport_cost(int n, const double* src_xy, const double* dst_xy, const double* density,
                          double* per_face) {
  int N = n * n;
  double res = 0, integral = 0;
  for (int f = 0; f < N; ++f) {
    int vid[4];
    double p[8];
    face_corners(n, src_xy, f, p, vid);
    int t[3] = {vid[3], vid[0], vid[1]};
    double s1[2] = {src_xy[2 * t[0]], src_xy[2 * t[0] + 1]};
    double s2[2] = {src_xy[2 * t[1]], src_xy[2 * t[1] + 1]};
    double s3[2] = {src_xy[2 * t[2]], src_xy[2 * t[2] + 1]};
    double face_area = signed_area3(s1, s2, s3);
    double dx[3], dy[3];
    for (int k = 0; k < 3; ++k) {
      dx[k] = dst_xy[2 * t[k]] - src_xy[2 * t[k]];
      dy[k] = dst_xy[2 * t[k] + 1] - src_xy[2 * t[k] + 1];
    }
#define DIST2(l1, l2, l3)                                             \
  ((l1 * dx[0] + l2 * dx[1] + l3 * dx[2]) * (l1 * dx[0] + l2 * dx[1] + l3 * dx[2]) + \
   (l1 * dy[0] + l2 * dy[1] + l3 * dy[2]) * (l1 * dy[0] + l2 * dy[1] + l3 * dy[2]))
    double face_cost = (DIST2(0.5, 0.5, 0) + DIST2(0, 0.5, 0.5) + DIST2(0.5, 0, 0.5)) / 3.0;
#undef DIST2
    integral += density[f] * face_area;
    face_cost = density[f] * face_area * face_cost;
    res += face_cost;
    if (per_face) per_face[f] = face_cost;
  }
  if (per_face)
    for (int f = 0; f < N; ++f) per_face[f] /= integral;
  return res / integral;
}
