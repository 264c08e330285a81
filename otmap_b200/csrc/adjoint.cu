// Implicit adjoint of a converged transport map with respect to its input density.
//
// The reference has no derivative; this follows from its equations. The solve drives
// the area residual F(psi, rho~) = A(psi) - e^2 rho~ to zero (otsolver_2dgrid.cpp:449-465)
// where A(psi) is the area of each quad of the grid displaced by the vertex gradients
// g = G psi (otsolver_2dgrid.cpp:362-447) and rho~ = adjust(rho) (otsolver_2dgrid.cpp:47-63).
// For a loss L(fwd) of the forward mesh fwd = grid + g, with q = dL/dfwd (per vertex):
//   dL/dpsi   = G^T q
//   J^T lambda = G^T q,  J = dA/dpsi = (dA/dg) G      (mean-zero subspace: J 1 = 0, 1^T J = 0)
//   dL/drho~  = e^2 lambda
//   dL/drho   = (lambda - (lambda . rho) / S) / S,  S = sum(rho)   (ratio clamp inactive)
// J^T is applied matrix-free: k_adj_vertex forms h_v = sum_c lambda_c dA_c/dg_v over the four
// cells around each vertex (dA_c/dD1 = (D2y, -D2x)/2, dA_c/dD2 = (-D1y, D1x)/2 with the
// cell diagonals D1 = g11 - g00 + (e,e), D2 = g01 - g10 + (-e,e)), and k_adj_cells gathers
// (G^T h)_f over every vertex whose clamped gradient stencil touches cell f. Both are
// deterministic gathers. lambda solves J^T lambda = b by restarted GMRES right-
// preconditioned with the pseudo-inverse of M (the reference's pseudo-Laplacian; J = -M at
// psi = 0), using the same cosine-transform Poisson solve as the forward loop; the
// one-step mode stops at lambda = -M^+ b (one Poisson solve). For strongly deformed maps
// J departs far from -M (a plain preconditioned fixed-point iteration diverges there),
// hence the Krylov method.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.cuh"

namespace otm {

__device__ __forceinline__ int clampv(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

// Device state of one restart cycle of the Krylov solve. The cycle's Arnoldi steps run on
// the device (a CUDA graph with a WHILE node, or the same kernels launched one step at a
// time): every step kernel reads the step index j here instead of taking it as a launch
// argument, and the Givens kernel advances it and decides whether the cycle goes on.
struct AdjCtl {
  int j;       // the step being taken: basis vectors 0..j are orthonormal
  int go;      // the cycle takes another step
  int m;       // restart length
  int budget;  // steps allowed in this cycle (the call's cap on Poisson solves)
  double bnorm, tol;
};

// Displacement g of vertex (i, j) from the forward mesh.
__device__ __forceinline__ double2 disp(const double* fwd, int n, int i, int j) {
  const size_t v = (size_t)j + (size_t)i * (n + 1);
  const double dx = 1.0 / (double)n;
  return make_double2(fwd[2 * v] - (double)i * dx, fwd[2 * v + 1] - (double)j * dx);
}

// Diagonals of cell (ci, cj).
__device__ __forceinline__ void cell_diags(const double* fwd, int n, int ci, int cj, double2& D1, double2& D2) {
  const double e = 1.0 / (double)n;
  double2 g00 = disp(fwd, n, ci, cj), g10 = disp(fwd, n, ci + 1, cj), g01 = disp(fwd, n, ci, cj + 1),
          g11 = disp(fwd, n, ci + 1, cj + 1);
  D1 = make_double2(g11.x - g00.x + e, g11.y - g00.y + e);
  D2 = make_double2(g01.x - g10.x - e, g01.y - g10.y + e);
}

// h_v = sum over the cells c around vertex v of lambda_c dA_c / dg_v.
__global__ void k_adj_vertex(int n, const double* fwd, const double* lambda, double* h) {
  const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long V = (long)(n + 1) * (n + 1);
  if (v >= V) return;
  const int vi = (int)(v / (n + 1)), vj = (int)(v % (n + 1));
  double hx = 0.0, hy = 0.0;
  double2 D1, D2;
  if (vi < n && vj < n) {  // v00 of cell (vi, vj): -dA/dD1
    cell_diags(fwd, n, vi, vj, D1, D2);
    const double l = 0.5 * lambda[(size_t)vi * n + vj];
    hx += l * -D2.y;
    hy += l * D2.x;
  }
  if (vi > 0 && vj < n) {  // v10 of cell (vi-1, vj): -dA/dD2
    cell_diags(fwd, n, vi - 1, vj, D1, D2);
    const double l = 0.5 * lambda[(size_t)(vi - 1) * n + vj];
    hx += l * D1.y;
    hy += l * -D1.x;
  }
  if (vi < n && vj > 0) {  // v01 of cell (vi, vj-1): dA/dD2
    cell_diags(fwd, n, vi, vj - 1, D1, D2);
    const double l = 0.5 * lambda[(size_t)vi * n + vj - 1];
    hx += l * -D1.y;
    hy += l * D1.x;
  }
  if (vi > 0 && vj > 0) {  // v11 of cell (vi-1, vj-1): dA/dD1
    cell_diags(fwd, n, vi - 1, vj - 1, D1, D2);
    const double l = 0.5 * lambda[(size_t)(vi - 1) * n + vj - 1];
    hx += l * D2.y;
    hy += l * -D2.x;
  }
  h[2 * v] = hx;
  h[2 * v + 1] = hy;
}

// (G^T h)_f: vertex (vi, vj) reads cells (clamp(vi-1+a), clamp(vj-1+b)), a, b in {0, 1},
// with gx coefficient (2a-1) n/2 and gy coefficient (2b-1) n/2
// (otsolver_2dgrid.cpp:379-422 with clamped indices). Cell (i, j) collects every
// (vertex, a, b) whose clamped position is (i, j); out = scale * G^T h (+ add).
__global__ void k_adj_cells(int n, const double* h, double scale, const double* add, double* out,
                            const AdjCtl* ctl, long ld) {
  if (ctl) out += (size_t)(ctl->j + 1) * ld;  // the new basis vector of the step
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= (long)n * n) return;
  const int i = (int)(f / n), j = (int)(f % n);
  // row choices: (vi, a) with clamp(vi - 1 + a) == i
  int ri[3], ra[3], nr = 0;
  ri[nr] = i + 1; ra[nr++] = 0;
  ri[nr] = i; ra[nr++] = 1;
  if (i == 0) { ri[nr] = 0; ra[nr++] = 0; }
  if (i == n - 1) { ri[nr] = n; ra[nr++] = 1; }
  int cj[3], cb[3], nc = 0;
  cj[nc] = j + 1; cb[nc++] = 0;
  cj[nc] = j; cb[nc++] = 1;
  if (j == 0) { cj[nc] = 0; cb[nc++] = 0; }
  if (j == n - 1) { cj[nc] = n; cb[nc++] = 1; }
  const double hw = 0.5 * (double)n;
  double acc = 0.0;
  for (int p = 0; p < nr; ++p)
    for (int q = 0; q < nc; ++q) {
      const size_t v = (size_t)cj[q] + (size_t)ri[p] * (n + 1);
      acc += hw * ((2 * ra[p] - 1) * h[2 * v] + (2 * cb[q] - 1) * h[2 * v + 1]);
    }
  out[f] = scale * acc + (add ? add[f] : 0.0);
}

// partial[b * (m+1) + i] = sum over this block's cells of w . V_i, i < m (basis vectors
// stored contiguously with stride `ld`), and partial[b * (m+1) + m] = w . w. The dot
// products are formed DOT_CHUNK at a time in one pass over the cells (w read once per
// chunk), each a per-thread FMA chain over the grid-stride cells, then reduced together.
// With ctl: w is basis vector j + 1 and m = j + 1 (or 0: w . w alone, for norm_only).
constexpr int DOT_CHUNK = 8;
__global__ void k_adj_multidot(long N, const double* w, const double* V, long ld, int m, double* partial,
                               const AdjCtl* ctl, int norm_only) {
  __shared__ double red[32 * DOT_CHUNK];
  if (ctl) {
    w = V + (size_t)(ctl->j + 1) * ld;
    m = norm_only ? 0 : ctl->j + 1;
  }
  const int P = m + 1;
  for (int i0 = 0; i0 < P; i0 += DOT_CHUNK) {
    double s[DOT_CHUNK];
#pragma unroll
    for (int c = 0; c < DOT_CHUNK; ++c) s[c] = 0.0;
    for (long f = (long)blockIdx.x * blockDim.x + threadIdx.x; f < N; f += (long)gridDim.x * blockDim.x) {
      const double wf = w[f];
#pragma unroll
      for (int c = 0; c < DOT_CHUNK; ++c) {
        const int i = i0 + c;
        if (i < P) s[c] = fma(wf, i < m ? V[(size_t)i * ld + f] : wf, s[c]);
      }
    }
    block_sum<DOT_CHUNK>(s, red);
    if (threadIdx.x == 0)
#pragma unroll
      for (int c = 0; c < DOT_CHUNK; ++c)
        if (i0 + c < P) partial[(size_t)blockIdx.x * P + i0 + c] = s[c];
  }
}

// The block partials of k_adj_multidot summed in block order (thread i: entry i).
__device__ __forceinline__ double sum_partials(const double* partial, int nblocks, int P, int i) {
  double t = 0.0;
  for (int b = 0; b < nblocks; ++b) t += partial[(size_t)b * P + i];
  return t;
}

// Gram-Schmidt pass over basis vectors 0..j: c_i = <w, v_i> (for the combine) and the
// Hessenberg column entry H_ij accumulated over the two passes (pass 0 sets it).
__global__ void k_adj_orth_reduce(const double* partial, int nblocks, int j, int pass, double* hcol, double* c,
                                  const AdjCtl* ctl) {
  if (ctl) j = ctl->j;
  const int i = threadIdx.x;
  if (i > j) return;
  const double d = sum_partials(partial, nblocks, j + 2, i);
  c[i] = d;
  hcol[i] = (pass ? hcol[i] : 0.0) + d;
}

// |w| after the passes: H_{j+1,j} and the factor that normalises w (0 when |w| = 0).
__global__ void k_adj_norm_reduce(const double* partial, int nblocks, int j, double* hcol, double* inv,
                                  const AdjCtl* ctl) {
  if (threadIdx.x != 0) return;
  if (ctl) j = ctl->j;
  const double hn = sqrt(sum_partials(partial, nblocks, 1, 0));
  hcol[j + 1] = hn;
  *inv = hn > 0 ? 1.0 / hn : 1.0;
}

__global__ void k_adj_scale_by(long N, double* v, const double* a, const AdjCtl* ctl, long ld) {
  if (ctl) v += (size_t)(ctl->j + 1) * ld;
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f < N) v[f] *= *a;
}

// w = a * w - sum_i c_i V_i (i < m); c in device memory; with ctl, w = V_{j+1} and m = j + 1
__global__ void k_adj_combine(long N, double* w, double a, const double* V, long ld, int m, const double* c,
                              const AdjCtl* ctl) {
  if (ctl) {
    w = const_cast<double*>(V) + (size_t)(ctl->j + 1) * ld;
    m = ctl->j + 1;
  }
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= N) return;
  double x = a * w[f];
  for (int i = 0; i < m; ++i) x = fma(-c[i], V[(size_t)i * ld + f], x);
  w[f] = x;
}

// Every Poisson record of the workspace ready for a new call: a bounded wait that gave up in
// an earlier call stopped its record and flagged it.
__global__ void k_adj_reset_recs(Inst* recs, int count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < count) {
    recs[k].active = 1;
    recs[k].fault = 0;
  }
}

// The Poisson record of the step reads basis vector j.
__global__ void k_adj_set_src(Inst* rec, double* V, long ld, const AdjCtl* ctl) {
  if (threadIdx.x == 0) rec->r[0] = V + (size_t)ctl->j * ld;
}

// Start of a restart cycle: residual norm rnorm in g_0.
__global__ void k_adj_cycle_init(AdjCtl* ctl, double* gv, int m, double rnorm, double bnorm, double tol, int budget) {
  if (threadIdx.x != 0) return;
  ctl->j = 0;
  ctl->go = budget > 0 ? 1 : 0;
  ctl->m = m;
  ctl->budget = budget;
  ctl->bnorm = bnorm;
  ctl->tol = tol;
  gv[0] = rnorm;
  for (int i = 1; i <= m; ++i) gv[i] = 0.0;
}

// End of Arnoldi step j (one thread): the new Hessenberg column, the previous Givens
// rotations applied to it, the rotation that zeroes H_{j+1,j}, the updated residual
// estimate |g_{j+1}|, and the loop test: go on while it is above tol * |b|, the new basis
// vector is non-zero, the cycle has room and the call's budget is not spent. H is
// (m+1) x m, row-major.
__global__ void k_adj_givens(AdjCtl* ctl, const double* hcol, double* H, double* cs, double* sn, double* gv,
                             cudaGraphConditionalHandle handle, int in_graph) {
  if (threadIdx.x != 0) return;
  const int j = ctl->j, m = ctl->m;
  auto Hs = [&](int i, int c) -> double& { return H[(size_t)i * m + c]; };
  for (int i = 0; i <= j + 1; ++i) Hs(i, j) = hcol[i];
  const double hn = hcol[j + 1];
  for (int i = 0; i < j; ++i) {
    const double t = cs[i] * Hs(i, j) + sn[i] * Hs(i + 1, j);
    Hs(i + 1, j) = -sn[i] * Hs(i, j) + cs[i] * Hs(i + 1, j);
    Hs(i, j) = t;
  }
  const double den = hypot(Hs(j, j), Hs(j + 1, j));
  cs[j] = den > 0 ? Hs(j, j) / den : 1.0;
  sn[j] = den > 0 ? Hs(j + 1, j) / den : 0.0;
  Hs(j, j) = den;
  Hs(j + 1, j) = 0.0;
  gv[j + 1] = -sn[j] * gv[j];
  gv[j] = cs[j] * gv[j];
  const int k = j + 1;
  const int go = (fabs(gv[k]) / ctl->bnorm > ctl->tol) && hn != 0 && k < m && k < ctl->budget;
  ctl->j = k;
  ctl->go = go;
  if (in_graph) cudaGraphSetConditional(handle, go ? 1u : 0u);
}

// H y = g for the k = j steps of the cycle (back substitution, one thread): y into c.
__global__ void k_adj_trisolve(const AdjCtl* ctl, const double* H, const double* gv, double* y) {
  if (threadIdx.x != 0) return;
  const int k = ctl->j, m = ctl->m;
  for (int i = k - 1; i >= 0; --i) {
    double t = gv[i];
    for (int l = i + 1; l < k; ++l) t -= H[(size_t)i * m + l] * y[l];
    y[i] = t / H[(size_t)i * m + i];
  }
}

// out = sum_i c_i V_i (i < m; with ctl, the cycle's step count)
__global__ void k_adj_span(long N, double* out, const double* V, long ld, int m, const double* c, const AdjCtl* ctl) {
  if (ctl) m = ctl->j;
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= N) return;
  double x = 0.0;
  for (int i = 0; i < m; ++i) x = fma(c[i], V[(size_t)i * ld + f], x);
  out[f] = x;
}

// v = b - v
__global__ void k_adj_resid(long N, const double* b, double* v) {
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f < N) v[f] = b[f] - v[f];
}

__global__ void k_adj_scale(long N, double* v, double a) {
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f < N) v[f] *= a;
}

__global__ void k_adj_neg(long N, const double* z, double* lambda) {
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f < N) lambda[f] = -z[f];
}

__global__ void k_adj_add(long N, const double* z, double* lambda) {
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f < N) lambda[f] += z[f];
}

// lambda += -z
__global__ void k_adj_axpy(long N, const double* z, double* lambda) {
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f < N) lambda[f] -= z[f];
}

// sums[0] = lambda . rho, sums[1] = sum rho, reduced in a fixed order by one block
__global__ void k_adj_rho_sums(long N, const double* lambda, const double* rho, double* sums) {
  __shared__ double red[64];
  double v[2] = {0.0, 0.0};
  for (long f = threadIdx.x; f < N; f += blockDim.x) {
    v[0] = fma(lambda[f], rho[f], v[0]);
    v[1] += rho[f];
  }
  block_sum<2>(v, red);
  if (threadIdx.x == 0) {
    sums[0] = v[0];
    sums[1] = v[1];
  }
}

__global__ void k_adj_finish(long N, const double* lambda, const double* sums, double* out) {
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f < N) out[f] = (lambda[f] - sums[0] / sums[1]) / sums[1];
}

}  // namespace otm

using namespace otm;

namespace otm {
void dense_poisson(otm_context* ctx, Inst* d_inst, const int* gemm_inst, int G);

// Adjoint workspace of one grid size, kept by the context: device vectors, the Krylov
// basis and one Poisson record per (source, destination) pair the solver uses, so a call
// allocates nothing and uploads nothing but its inputs' pointers.
struct AdjointWs : otm_context::Erased {
  int n = 0, m = 0;
  size_t N = 0, V = 0, ld = 0;
  DevBuf buf, recs, lists;
  double *b, *lam, *z, *h, *t1, *t2, *Vb, *c, *part, *sums, *hcol, *inv;
  double *fwdc, *H, *cs, *sn, *gv;  // the forward mesh of the call; the cycle's Hessenberg state
  AdjCtl* ctl = nullptr;
  int G = 0, rows = 0, cols = 0, reg = 0, fft = 0;
  // the Arnoldi step as a graph with a WHILE node (built on first use) and its kernel count
  cudaGraphExec_t step_graph = nullptr;
  long step_kernels = 0;
  ~AdjointWs() override {
    if (step_graph) cudaGraphExecDestroy(step_graph);
  }
  // record k: src = basis vector k (k < m+1); record m+1: src = b; record m+2: src = h;
  // record m+3: src = the basis vector of the current step (set on the device); dst = z
  Inst* rec(int k) { return recs.as<Inst>() + k; }
};

static AdjointWs* adjoint_ws(otm_context* ctx, int n, int m) {
  auto& slot = ctx->adjoint[n];
  if (slot && static_cast<AdjointWs*>(slot.get())->m >= m) return static_cast<AdjointWs*>(slot.get());
  auto* W = new AdjointWs;
  W->n = n;
  W->m = m;
  W->N = (size_t)n * n;
  W->V = (size_t)(n + 1) * (n + 1);
  W->ld = (W->N + 31) / 32 * 32;
  const int nred = 256;
  const size_t words = W->ld * 6 + 2 * W->V + (size_t)(m + 1) * W->ld + (m + 2) + (size_t)nred * (m + 2) + (m + 3) + 64 +
                       16 + 2 * W->V + (size_t)(m + 1) * m + 3 * (size_t)m + 1;
  W->buf.reserve(sizeof(double) * words);
  double* p = W->buf.as<double>();
  W->b = p; p += W->ld;
  W->lam = p; p += W->ld;
  W->z = p; p += W->ld;
  W->t1 = p; p += W->ld;
  W->t2 = p; p += W->ld;
  W->h = p; p += 2 * W->V + W->ld;
  W->Vb = p; p += (size_t)(m + 1) * W->ld;
  W->c = p; p += m + 2;
  W->sums = p; p += 2;
  W->part = p; p += (size_t)nred * (m + 2);
  W->hcol = p; p += m + 2;  // the current Hessenberg column
  W->inv = p; p += 8;
  W->ctl = reinterpret_cast<AdjCtl*>(p); p += 8;
  W->fwdc = p; p += 2 * W->V;
  W->H = p; p += (size_t)(m + 1) * m;
  W->cs = p; p += m;
  W->sn = p; p += m;
  W->gv = p;
  SizeTables* T = ctx->tables.at(n).get();
  Inst base;
  std::memset(&base, 0, sizeof(base));
  base.n = n;
  base.active = 1;
  base.t1 = W->t1;
  base.t2 = W->t2;
  base.C = T->C.as<double>();
  base.cosk = T->cosk.as<double>();
  base.tw = T->tw.as<double2>();
  base.pt = T->pt.as<double2>();
  base.fft = (ctx->poisson_mode != OTM_POISSON_DENSE && fft_eligible(n)) ? 1 : 0;
  W->fft = base.fft;
  int items;
  if (base.fft) {
    int lg = 0;
    while ((1 << lg) < n) ++lg;
    base.logn = lg;
    W->reg = dct_reg_supported(n) ? 1 : 0;
    const int per = W->reg ? dct_reg_lines_per_block(n) : fft_lines(n);
    const int cper = W->reg ? dct_reg_cols_per_block(n) : fft_lines(n);
    base.nrow = n / per;
    base.ncol = n / cper;
    W->rows = base.nrow;
    W->cols = base.ncol;
    items = std::max(W->rows, W->cols);
  } else {
    int t = (n + 63) / 64;
    base.ngemm = W->G = items = t * t;
  }
  std::vector<Inst> recs(m + 4, base);
  for (int k = 0; k <= m; ++k) recs[k].r[0] = W->Vb + (size_t)k * W->ld;
  recs[m + 1].r[0] = W->b;
  recs[m + 2].r[0] = W->h;
  recs[m + 3].r[0] = W->Vb;
  for (auto& r : recs) r.dhat = W->z;
  W->recs.reserve(sizeof(Inst) * recs.size());
  W->lists.reserve(sizeof(int) * items);
  std::vector<int> zeros(items, 0);
  OTM_CUDA(cudaMemcpyAsync(W->recs.p, recs.data(), sizeof(Inst) * recs.size(), cudaMemcpyHostToDevice, ctx->stream));
  OTM_CUDA(cudaMemcpyAsync(W->lists.p, zeros.data(), sizeof(int) * items, cudaMemcpyHostToDevice, ctx->stream));
  OTM_CUDA(cudaStreamSynchronize(ctx->stream));
  slot.reset(W);
  return W;
}

// z = M^+ (source of record k)
static void poisson_rec(otm_context* ctx, AdjointWs* W, int k) {
  Inst* d = W->rec(k);
  const int* L = W->lists.as<int>();
  if (W->fft) {
    if (W->reg)
      dct_reg_run(ctx, W->n, false, d, L, 0, W->rows, L, 0, W->cols);
    else
      poisson_fft(ctx, d, L, 0, W->rows, L, 0, W->cols);
  } else {
    dense_poisson(ctx, d, L, W->G);
  }
}

// One Arnoldi step j of the cycle (j read on the device): z = M^+ v_j, w = J^T z into
// v_{j+1}, two classical Gram-Schmidt passes and the normalisation (reductions in block
// order on the device), then the Givens kernel, which advances j and sets the loop test.
static void arnoldi_step(otm_context* ctx, AdjointWs* W, int n, cudaGraphConditionalHandle handle, int in_graph) {
  const long N = (long)W->N, ld = (long)W->ld;
  const int RB = 256, nred = 256;
  const unsigned gN = (unsigned)((W->N + RB - 1) / RB), gV = (unsigned)((W->V + RB - 1) / RB);
  const AdjCtl* ctl = W->ctl;
  launch(ctx, "adj_set_src", k_adj_set_src, 1, 32, W->rec(W->m + 3), W->Vb, ld, ctl);
  poisson_rec(ctx, W, W->m + 3);
  launch(ctx, "adj_vertex", k_adj_vertex, gV, RB, n, (const double*)W->fwdc, (const double*)W->z, W->h);
  launch(ctx, "adj_cells", k_adj_cells, gN, RB, n, (const double*)W->h, 1.0, (const double*)nullptr, W->Vb, ctl, ld);
  const unsigned rt = (unsigned)((W->m + 1 + 31) / 32 * 32);
  for (int pass = 0; pass < 2; ++pass) {
    launch(ctx, "adj_dot", k_adj_multidot, nred, RB, N, (const double*)nullptr, (const double*)W->Vb, ld, 0, W->part,
           ctl, 0);
    launch(ctx, "adj_reduce", k_adj_orth_reduce, 1, rt, (const double*)W->part, nred, 0, pass, W->hcol, W->c, ctl);
    launch(ctx, "adj_combine", k_adj_combine, gN, RB, N, W->Vb, 1.0, (const double*)W->Vb, ld, 0, (const double*)W->c,
           ctl);
  }
  launch(ctx, "adj_dot", k_adj_multidot, nred, RB, N, (const double*)nullptr, (const double*)W->Vb, ld, 0, W->part, ctl,
         1);
  launch(ctx, "adj_reduce", k_adj_norm_reduce, 1, 32, (const double*)W->part, nred, 0, W->hcol, W->inv, ctl);
  launch(ctx, "adj_scale", k_adj_scale_by, gN, RB, N, W->Vb, (const double*)W->inv, ctl, ld);
  launch(ctx, "adj_givens", k_adj_givens, 1, 32, W->ctl, (const double*)W->hcol, W->H, W->cs, W->sn, W->gv, handle,
         in_graph);
}

// The cycle's steps as a graph: a WHILE node whose body is one Arnoldi step, its condition
// set by the Givens kernel (at most m bodies per launch).
static void build_step_graph(otm_context* ctx, AdjointWs* W, int n) {
  cudaStream_t st = ctx->stream;
  dct_reg_attrs(ctx->device);
  poisson_fft_attrs(ctx->device);
  cudaGraph_t g = nullptr;
  OTM_CUDA(cudaGraphCreate(&g, 0));
  try {
    cudaGraphConditionalHandle handle;
    OTM_CUDA(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    OTM_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &params));
    cudaGraph_t body = params.conditional.phGraph_out[0];
    const long before = ctx->launches;
    OTM_CUDA(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
      arnoldi_step(ctx, W, n, handle, 1);
    } catch (...) {
      cudaGraph_t dummy;
      cudaStreamEndCapture(st, &dummy);
      throw;
    }
    OTM_CUDA(cudaStreamEndCapture(st, &body));
    W->step_kernels = ctx->launches - before;
    ctx->launches = before;  // captured, not executed
    OTM_CUDA(cudaGraphInstantiate(&W->step_graph, g, 0));
  } catch (...) {
    cudaGraphDestroy(g);
    throw;
  }
  cudaGraphDestroy(g);
}

}  // namespace otm

extern "C" void otm_default_adjoint_options(otm_adjoint_options* o) {
  if (!o) return;
  o->mode = OTM_ADJOINT_KRYLOV;
  o->tol = 1e-10;
  o->max_iter = 2000;
  o->restart = 40;
}

extern "C" int otm_adjoint(otm_context* ctx, int n, const double* density, const double* fwd_xy,
                           const double* grad_fwd, const otm_adjoint_options* opt, double* grad_density,
                           otm_adjoint_stats* stats) {
  return guarded([&] {
    if (!ctx || !density || !fwd_xy || !grad_fwd || !grad_density) throw BadArg{"otm_adjoint: null argument"};
    if (n < 1 || n > 16384) throw BadArg{"otm_adjoint: grid size out of range"};
    otm_adjoint_options o;
    otm_default_adjoint_options(&o);
    if (opt) o = *opt;
    if (o.mode != OTM_ADJOINT_ONE_STEP && o.mode != OTM_ADJOINT_KRYLOV) throw BadArg{"otm_adjoint: unknown mode"};
    make_current(ctx);
    if (otm_init(ctx, n) != OTM_OK) throw BadArg{std::string("otm_adjoint: ") + otm_last_error()};
    cudaStream_t st = ctx->stream;
    const int m = o.mode == OTM_ADJOINT_KRYLOV ? std::max(1, std::min(o.restart, 200)) : 1;
    AdjointWs* W = adjoint_ws(ctx, n, m);
    launch(ctx, "adj_reset", k_adj_reset_recs, 1, 256, W->rec(0), W->m + 4);
    const size_t N = W->N, V = W->V, ld = W->ld;
    const int RB = 256, nred = 256;
    // inputs: used in place when they are device memory, else staged into the workspace
    auto stage = [&](const double* src, double* tmp, size_t words) -> const double* {
      if (is_device_ptr(src)) return src;
      copy_in(ctx, tmp, src, sizeof(double) * words);
      return tmp;
    };
    if (!is_device_ptr(fwd_xy) || !is_device_ptr(grad_fwd) || !is_device_ptr(density)) {
      ctx->staging.reserve(sizeof(double) * (4 * V + N));
    }
    double* stg = ctx->staging.as<double>();
    const double* d_fwd = stage(fwd_xy, stg, 2 * V);
    const double* d_q = stage(grad_fwd, stg + 2 * V, 2 * V);
    const double* d_rho = stage(density, stg + 4 * V, N);
    const unsigned gN = (unsigned)((N + RB - 1) / RB), gV = (unsigned)((V + RB - 1) / RB);
    double* d_b = W->b;
    double* d_lam = W->lam;
    double* d_z = W->z;
    double* d_h = W->h;
    double* d_V = W->Vb;
    double* d_c = W->c;
    double* d_part = W->part;
    // b = G^T q
    launch(ctx, "adj_cells", k_adj_cells, gN, RB, n, d_q, 1.0, (const double*)nullptr, d_b, (const AdjCtl*)nullptr, 0L);
    std::vector<double> hp;
    auto multidot = [&](const double* w, int k, std::vector<double>& out) {
      launch(ctx, "adj_dot", k_adj_multidot, nred, RB, (long)N, w, (const double*)d_V, (long)ld, k, d_part,
             (const AdjCtl*)nullptr, 0);
      hp.resize((size_t)nred * (k + 1));
      OTM_CUDA(cudaMemcpyAsync(hp.data(), d_part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, st));
      OTM_CUDA(cudaStreamSynchronize(st));
      out.assign(k + 1, 0.0);
      for (int blk = 0; blk < nred; ++blk)
        for (int i = 0; i <= k; ++i) out[i] += hp[(size_t)blk * (k + 1) + i];
    };
    auto apply_jt = [&](const double* x, double* out) {
      launch(ctx, "adj_vertex", k_adj_vertex, gV, RB, n, d_fwd, x, d_h);
      launch(ctx, "adj_cells", k_adj_cells, gN, RB, n, (const double*)d_h, 1.0, (const double*)nullptr, out,
             (const AdjCtl*)nullptr, 0L);
    };
    int solves = 0;
    double rel = -1.0;
    if (o.mode == OTM_ADJOINT_ONE_STEP) {
      // lambda = -M^+ b: the solve writes z, lambda = -z
      poisson_rec(ctx, W, W->m + 1);
      ++solves;
      launch(ctx, "adj_scale", k_adj_neg, gN, RB, (long)N, (const double*)d_z, d_lam);
    } else {
      OTM_CUDA(cudaMemsetAsync(d_lam, 0, sizeof(double) * N, st));
      // Restarted GMRES(m) on J^T lambda = b, right-preconditioned: J^T M^+ y = b, lambda = M^+ y.
      // A cycle's Arnoldi steps run on the device (classical Gram-Schmidt applied twice,
      // Givens rotations and the loop test in one-thread kernels) as one graph launch with a
      // WHILE node -- or, in the host-driven loop mode and under the profiler, the same
      // kernels one step at a time; the host reads the cycle's step count once per restart,
      // forms the true residual and decides whether to restart.
      std::vector<double> dots;
      OTM_CUDA(cudaMemcpyAsync(d_V, d_b, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
      OTM_CUDA(cudaMemcpyAsync(W->fwdc, d_fwd, sizeof(double) * 2 * V, cudaMemcpyDeviceToDevice, st));
      multidot(d_V, 0, dots);
      const double bnorm = std::sqrt(dots[0]);
      const bool graph = ctx->loop_mode == OTM_LOOP_GRAPH && !ctx->prof.on;
      rel = bnorm > 0 ? 1.0 : 0.0;
      bool first = true;
      while (bnorm > 0) {
        double* v0 = d_V;
        double rnorm;
        if (first) {
          rnorm = bnorm;
          first = false;
        } else {
          apply_jt(d_lam, v0);
          launch(ctx, "adj_resid", k_adj_resid, gN, RB, (long)N, (const double*)d_b, v0);
          multidot(v0, 0, dots);
          rnorm = std::sqrt(dots[0]);
        }
        rel = rnorm / bnorm;
        if (!(rel > o.tol) || solves >= o.max_iter) break;
        launch(ctx, "adj_scale", k_adj_scale, gN, RB, (long)N, v0, 1.0 / rnorm);
        launch(ctx, "adj_cycle", k_adj_cycle_init, 1, 32, W->ctl, W->gv, m, rnorm, bnorm, o.tol, o.max_iter - solves);
        if (graph) {
          if (!W->step_graph) build_step_graph(ctx, W, n);
          OTM_CUDA(cudaGraphLaunch(W->step_graph, st));
        } else {
          AdjCtl hc;
          do {
            arnoldi_step(ctx, W, n, (cudaGraphConditionalHandle)0, 0);
            OTM_CUDA(cudaMemcpyAsync(&hc, W->ctl, sizeof(hc), cudaMemcpyDeviceToHost, st));
            OTM_CUDA(cudaStreamSynchronize(st));
            ctx->prof.flush();
          } while (hc.go);
        }
        // lambda += M^+ (V y), H y = g solved on the device
        launch(ctx, "adj_trisolve", k_adj_trisolve, 1, 32, (const AdjCtl*)W->ctl, (const double*)W->H,
               (const double*)W->gv, d_c);
        launch(ctx, "adj_span", k_adj_span, gN, RB, (long)N, d_h, (const double*)d_V, (long)ld, 0, (const double*)d_c,
               (const AdjCtl*)W->ctl);
        poisson_rec(ctx, W, W->m + 2);  // z = M^+ h
        launch(ctx, "adj_add", k_adj_add, gN, RB, (long)N, (const double*)d_z, d_lam);
        AdjCtl hc;
        OTM_CUDA(cudaMemcpyAsync(&hc, W->ctl, sizeof(hc), cudaMemcpyDeviceToHost, st));
        OTM_CUDA(cudaStreamSynchronize(st));
        if (graph) ctx->launches += W->step_kernels * (long)hc.j;
        solves += hc.j + 1;
        if (hc.j == 0) break;  // no step was possible: nothing changes by restarting
      }
    }
    // chain through the density normalisation, reduced and applied on the device
    launch(ctx, "adj_rho_sums", k_adj_rho_sums, 1, 1024, (long)N, (const double*)d_lam, d_rho, W->sums);
    bool odev = is_device_ptr(grad_density);
    double* out = odev ? grad_density : d_z;
    launch(ctx, "adj_finish", k_adj_finish, gN, RB, (long)N, (const double*)d_lam, (const double*)W->sums, out);
    OTM_CUDA(cudaGetLastError());
    if (!odev) copy_out(ctx, grad_density, out, sizeof(double) * N);
    // a bounded wait inside a transform that gave up flags its record
    std::vector<Inst> recs_h((size_t)W->m + 4);
    OTM_CUDA(cudaMemcpyAsync(recs_h.data(), W->rec(0), sizeof(Inst) * recs_h.size(), cudaMemcpyDeviceToHost, st));
    OTM_CUDA(cudaStreamSynchronize(st));
    ctx->prof.flush();
    for (const Inst& r : recs_h)
      if (r.fault) throw DeviceTimeout{"otm_adjoint: a bounded device-side wait gave up"};
    if (stats) {
      stats->iterations = solves;
      stats->relative_residual = rel;
    }
    return (int)OTM_OK;
  });
}
