// Device-resident restarted GMRES (CGS2 Arnoldi, Givens rotations on the
// device) and FP64 iterative refinement around an FP32-valued inner GMRES.
//
// Reference: examples/iterative/gmres.cu:468-771 (left-preconditioned GMRES(m)
// with MGS and host-side Givens; its bugs are fixed here: dot length nvars,
// m+1 basis vectors, restarts). Host round trips happen only every
// `check_every` Arnoldi steps and at restarts; every kernel of a step reads
// the step index and a done flag from device memory, so steps queued after
// convergence are no-ops.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "gf_internal.h"

struct gf_precond;

namespace gf {

gf_status precond_apply_impl(gf_precond* p, const double* r, double* z, cudaStream_t st);
template <class VT>
gf_status spmv_impl(int n, const int32_t* rowp, const int32_t* cols, const VT* A,
                    const double* x, double alpha, double beta, double* y, cudaStream_t st);
gf_status precond_status(gf_precond* p, cudaStream_t st, int* bits);
int* precond_status_ptr(gf_precond* p);

constexpr int kRedBlocks = 296;  // 2 x 148 SMs
constexpr int kRedThreads = 256;

struct GmState {
  int j;        // Arnoldi index within the cycle
  int done;     // 1 converged / breakdown / step limit: later steps are no-ops
  int pad0, pad1;
  double target;
  double hn;
  double rel;   // last true relative residual
  double bnorm;
};

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += sh[k];
  __syncthreads();
  return s;
}

// partial[i * kRedBlocks + bx] = sum over block slice of V_i . w  for i <= j
__global__ void dots_kernel(const double* __restrict__ V, const double* __restrict__ w, size_t N,
                            const GmState* st, int fixed_count, double* partial) {
  __shared__ double sh[32];
  if (st && st->done) return;
  const int cnt = fixed_count > 0 ? fixed_count : st->j + 1;
  const size_t chunk = (N + gridDim.x - 1) / gridDim.x;
  const size_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  for (int i = 0; i < cnt; i++) {
    const double* v = V + (size_t)i * N;
    double acc = 0.0;
    for (size_t t = lo + threadIdx.x; t < hi; t += blockDim.x) acc = fma(v[t], w[t], acc);
    const double s = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[(size_t)i * gridDim.x + blockIdx.x] = s;
  }
}

// h_i = sum_b partial[i][b]; H[i][j] (+)= h_i
__global__ void reduce_dots_kernel(const double* partial, int nb, GmState* st, int m, double* H,
                                   double* h, int accumulate) {
  if (st->done) return;
  const int j = st->j;
  for (int i = threadIdx.x; i <= j; i += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nb; b++) s += partial[(size_t)i * nb + b];
    h[i] = s;
    if (accumulate)
      H[(size_t)i * m + j] += s;
    else
      H[(size_t)i * m + j] = s;
  }
}

// w -= sum_{i<=j} h_i V_i ; optionally partial sums of |w|^2
__global__ void update_kernel(const double* __restrict__ V, double* __restrict__ w, size_t N,
                              const GmState* st, const double* __restrict__ h, double* partial) {
  __shared__ double sh[32];
  __shared__ double hs[1024];
  if (st->done) return;
  const int cnt = st->j + 1;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) hs[i] = h[i];
  __syncthreads();
  const size_t chunk = (N + gridDim.x - 1) / gridDim.x;
  const size_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  double acc = 0.0;
  for (size_t t = lo + threadIdx.x; t < hi; t += blockDim.x) {
    double s = w[t];
    for (int i = 0; i < cnt; i++) s = fma(-hs[i], V[(size_t)i * N + t], s);
    w[t] = s;
    acc = fma(s, s, acc);
  }
  if (partial) {
    const double b = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = b;
  }
}

// hn = sqrt(sum partial); H[j+1][j] = hn
__global__ void norm_finish_kernel(const double* partial, int nb, GmState* st, int m,
                                   double* H) {
  if (st->done) return;
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += partial[b];
  st->hn = sqrt(s);
  H[(size_t)(st->j + 1) * m + st->j] = st->hn;
}

__global__ void normalize_kernel(const double* __restrict__ w, double* __restrict__ vnext,
                                 size_t N, const GmState* st) {
  if (st->done) return;
  const double inv = st->hn > 0.0 ? 1.0 / st->hn : 0.0;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < N;
       t += (size_t)gridDim.x * blockDim.x)
    vnext[t] = w[t] * inv;
}

// Givens update for column j (examples/iterative/gmres.cu:672-699) and the
// convergence test |g[j+1]| <= target.
__global__ void givens_kernel(GmState* st, int m, double* H, double* g, double* cs, double* ss,
                              int step_limit) {
  if (st->done) return;
  const int j = st->j;
  for (int i = 0; i < j; i++) {
    const double a = H[(size_t)i * m + j], c = H[(size_t)(i + 1) * m + j];
    H[(size_t)i * m + j] = cs[i] * a + ss[i] * c;
    H[(size_t)(i + 1) * m + j] = -ss[i] * a + cs[i] * c;
  }
  const double a = H[(size_t)j * m + j], c = H[(size_t)(j + 1) * m + j];
  const double hyp = sqrt(a * a + c * c);
  cs[j] = hyp > 0.0 ? a / hyp : 1.0;
  ss[j] = hyp > 0.0 ? c / hyp : 0.0;
  H[(size_t)j * m + j] = cs[j] * a + ss[j] * c;
  H[(size_t)(j + 1) * m + j] = 0.0;
  g[j + 1] = -ss[j] * g[j];
  g[j] = cs[j] * g[j];
  st->j = j + 1;
  if (fabs(g[j + 1]) <= st->target || st->hn == 0.0 || !isfinite(g[j + 1]) ||
      st->j >= step_limit)
    st->done = 1;
}

// y = H^{-1} g over the first j columns
__global__ void backsolve_kernel(const GmState* st, int m, const double* H, const double* g,
                                 double* y) {
  const int j = st->j;
  for (int i = j - 1; i >= 0; i--) {
    double s = g[i];
    for (int k = i + 1; k < j; k++) s -= H[(size_t)i * m + k] * y[k];
    y[i] = s / H[(size_t)i * m + i];
  }
}

// out = sum_{i<j} y_i V_i
__global__ void combine_kernel(const double* __restrict__ V, size_t N, const GmState* st,
                               const double* __restrict__ y, double* __restrict__ out) {
  __shared__ double ys[1024];
  const int j = st->j;
  for (int i = threadIdx.x; i < j; i += blockDim.x) ys[i] = y[i];
  __syncthreads();
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < N;
       t += (size_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < j; i++) s = fma(ys[i], V[(size_t)i * N + t], s);
    out[t] = s;
  }
}

__global__ void axpy_kernel(double a, const double* __restrict__ x, double* __restrict__ y,
                            size_t N) {
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < N;
       t += (size_t)gridDim.x * blockDim.x)
    y[t] += a * x[t];
}

// V0 = src / ||src|| using partial norm sums; g[0] = beta; resets the cycle
__global__ void cycle_init_kernel(const double* partial, int nb, GmState* st, double* g,
                                  double* H, int m) {
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += partial[b];
  const double beta = sqrt(s);
  st->hn = beta;
  st->j = 0;
  st->done = (beta == 0.0) ? 1 : 0;
  g[0] = beta;
  for (int i = 1; i <= m; i++) g[i] = 0.0;
}
__global__ void scale_kernel(const double* __restrict__ src, double* __restrict__ dst, size_t N,
                             const GmState* st) {
  const double inv = st->hn > 0.0 ? 1.0 / st->hn : 0.0;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < N;
       t += (size_t)gridDim.x * blockDim.x)
    dst[t] = src[t] * inv;
}
__global__ void set_target_kernel(GmState* st, const double* partial, int nb, double rtol,
                                  int use_partial, double value) {
  double s = 0.0;
  if (use_partial)
    for (int b = 0; b < nb; b++) s += partial[b];
  st->target = use_partial ? rtol * sqrt(s) : value;
}
__global__ void sumsq_kernel(const double* __restrict__ w, size_t N, double* partial) {
  __shared__ double sh[32];
  const size_t chunk = (N + gridDim.x - 1) / gridDim.x;
  const size_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  double acc = 0.0;
  for (size_t t = lo + threadIdx.x; t < hi; t += blockDim.x) acc = fma(w[t], w[t], acc);
  const double b = block_sum(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = b;
}
__global__ void finish_sum_kernel(const double* partial, int nb, double* out) {
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += partial[b];
  *out = sqrt(s);
}
template <class T2>
__global__ void cvt_kernel(size_t n, const double* __restrict__ in, T2* __restrict__ out) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = (T2)in[t];
}
__global__ void permute2_kernel(const int32_t* perm, int nnodes, const double* in, double* out,
                                int dir) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 6 * nnodes) return;
  const int i = t / 6, k = t % 6;
  if (dir == 0)
    out[6 * (size_t)perm[i] + k] = in[t];
  else
    out[t] = in[6 * (size_t)perm[i] + k];
}

// Workspace cached per (assembler, m).
struct GmWork {
  int m = 0, n = 0;
  DevBuf<double> V, H, g, cs, ss, y, h, partial, w, t, r, x, b, d, e, scal;
  DevBuf<GmState> st;
  DevBuf<float> A32;
  size_t a32_n = 0;
};

static gf_status ensure_work(GmWork& W, int m, int n, size_t nnz36, bool mixed) {
  const size_t N = (size_t)6 * n;
  if (W.m != m || W.n != n) {
    cudaError_t e = cudaSuccess;
    auto al = [&](cudaError_t x) {
      if (e == cudaSuccess) e = x;
    };
    al(W.V.alloc((size_t)(m + 1) * N));
    al(W.H.alloc((size_t)(m + 1) * m));
    al(W.g.alloc(m + 1));
    al(W.cs.alloc(m));
    al(W.ss.alloc(m));
    al(W.y.alloc(m));
    al(W.h.alloc(m + 1));
    al(W.partial.alloc((size_t)(m + 2) * kRedBlocks));
    al(W.w.alloc(N));
    al(W.t.alloc(N));
    al(W.r.alloc(N));
    al(W.x.alloc(N));
    al(W.b.alloc(N));
    al(W.d.alloc(N));
    al(W.e.alloc(N));
    al(W.scal.alloc(4));
    al(W.st.alloc(1));
    if (e != cudaSuccess) {
      set_last_error("gmres workspace", e);
      W.m = 0;
      return e == cudaErrorMemoryAllocation ? GF_OOM : GF_CUDA_ERROR;
    }
    W.m = m;
    W.n = n;
  }
  if (mixed && W.a32_n != nnz36) {
    GF_CUDA(W.A32.alloc(nnz36));
    W.a32_n = nnz36;
  }
  return GF_OK;
}

// One GMRES(m) solve of A x = b in the solver ordering, in place on x.
// VT selects the SpMV value type (double for FP64, float for the inner
// solve of the mixed mode).
template <class VT>
static gf_status gmres_core(gf_assembler* a, const VT* Avals, gf_precond* p, GmWork& W,
                            const double* b, double* x, int m, int max_it, double rtol,
                            int side, int check_every, cudaStream_t st, int* iters,
                            int* restarts, double* rel_out, bool* converged) {
  const int n = a->nnodes;
  const size_t N = (size_t)6 * n;
  const int vb = 592, vt = 256;
  GmState* S = W.st.p;
  double* part = W.partial.p;
  auto spmv = [&](const double* in, double alpha, double beta, double* out) {
    return spmv_impl<VT>(n, a->d_rowp.p, a->d_cols.p, Avals, in, alpha, beta, out, st);
  };
  // bnorm and the inner target
  GmState h0{};
  GF_CUDA(cudaMemcpyAsync(S, &h0, sizeof(GmState), cudaMemcpyHostToDevice, st));
  sumsq_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(b, N, part);
  finish_sum_kernel<<<1, 1, 0, st>>>(part, kRedBlocks, W.scal.p);
  double bnorm = 0.0;
  GF_CUDA(cudaMemcpyAsync(&bnorm, W.scal.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  GF_CUDA(cudaStreamSynchronize(st));
  if (bnorm == 0.0) bnorm = 1.0;
  if (side == 0) {
    gf_status s = precond_apply_impl(p, b, W.t.p, st);
    if (s != GF_OK) return s;
    sumsq_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(W.t.p, N, part);
    set_target_kernel<<<1, 1, 0, st>>>(S, part, kRedBlocks, rtol, 1, 0.0);
  } else {
    set_target_kernel<<<1, 1, 0, st>>>(S, part, kRedBlocks, rtol, 0, rtol * bnorm);
  }
  GF_CHECK_LAUNCH();
  int it_total = 0, nrest = 0;
  double rel = 1.0;
  *converged = false;
  while (true) {
    // r = b - A x ; rel
    GF_CUDA(cudaMemcpyAsync(W.r.p, b, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    gf_status s = spmv(x, -1.0, 1.0, W.r.p);
    if (s != GF_OK) return s;
    sumsq_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(W.r.p, N, part);
    finish_sum_kernel<<<1, 1, 0, st>>>(part, kRedBlocks, W.scal.p);
    double rn = 0.0;
    GF_CUDA(cudaMemcpyAsync(&rn, W.scal.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    GF_CUDA(cudaStreamSynchronize(st));
    rel = rn / bnorm;
    if (!std::isfinite(rel)) {
      *iters = it_total;
      *restarts = nrest;
      *rel_out = rel;
      return GF_NAN;
    }
    if (rel <= rtol) {
      *converged = true;
      break;
    }
    if (it_total >= max_it) break;
    if (nrest > 0 || it_total > 0) nrest++;
    // V0
    const double* src = W.r.p;
    if (side == 0) {
      s = precond_apply_impl(p, W.r.p, W.t.p, st);
      if (s != GF_OK) return s;
      src = W.t.p;
    }
    sumsq_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(src, N, part);
    cycle_init_kernel<<<1, 1, 0, st>>>(part, kRedBlocks, S, W.g.p, W.H.p, m);
    scale_kernel<<<vb, vt, 0, st>>>(src, W.V.p, N, S);
    GF_CHECK_LAUNCH();
    const int steps = std::min(m, max_it - it_total);
    int done_steps = 0;
    while (done_steps < steps) {
      const int batch = std::min(check_every, steps - done_steps);
      for (int k = 0; k < batch; k++) {
        // the step index lives on the device; host-side k only bounds the queue
        const int jj = done_steps + k;
        const double* vj = W.V.p + (size_t)jj * N;
        if (side == 0) {
          s = spmv(vj, 1.0, 0.0, W.t.p);
          if (s == GF_OK) s = precond_apply_impl(p, W.t.p, W.w.p, st);
        } else {
          s = precond_apply_impl(p, vj, W.t.p, st);
          if (s == GF_OK) s = spmv(W.t.p, 1.0, 0.0, W.w.p);
        }
        if (s != GF_OK) return s;
        dots_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(W.V.p, W.w.p, N, S, 0, part);
        reduce_dots_kernel<<<1, 256, 0, st>>>(part, kRedBlocks, S, m, W.H.p, W.h.p, 0);
        update_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(W.V.p, W.w.p, N, S, W.h.p, nullptr);
        dots_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(W.V.p, W.w.p, N, S, 0, part);
        reduce_dots_kernel<<<1, 256, 0, st>>>(part, kRedBlocks, S, m, W.H.p, W.h.p, 1);
        update_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(W.V.p, W.w.p, N, S, W.h.p,
                                                          part + (size_t)(m + 1) * kRedBlocks);
        norm_finish_kernel<<<1, 1, 0, st>>>(part + (size_t)(m + 1) * kRedBlocks, kRedBlocks, S,
                                            m, W.H.p);
        normalize_kernel<<<vb, vt, 0, st>>>(W.w.p, W.V.p + (size_t)(jj + 1) * N, N, S);
        givens_kernel<<<1, 1, 0, st>>>(S, m, W.H.p, W.g.p, W.cs.p, W.ss.p, steps);
        GF_CHECK_LAUNCH();
      }
      done_steps += batch;
      GmState hs;
      GF_CUDA(cudaMemcpyAsync(&hs, S, sizeof(GmState), cudaMemcpyDeviceToHost, st));
      GF_CUDA(cudaStreamSynchronize(st));
      if (hs.done) break;
    }
    GmState hs;
    GF_CUDA(cudaMemcpyAsync(&hs, S, sizeof(GmState), cudaMemcpyDeviceToHost, st));
    GF_CUDA(cudaStreamSynchronize(st));
    int bits = 0;
    precond_status(p, st, &bits);
    if (bits & 1) return GF_TIMEOUT;
    // x += V y  (left)  or  M^{-1} V y  (right)
    backsolve_kernel<<<1, 1, 0, st>>>(S, m, W.H.p, W.g.p, W.y.p);
    combine_kernel<<<vb, vt, 0, st>>>(W.V.p, N, S, W.y.p, W.w.p);
    GF_CHECK_LAUNCH();
    if (side == 1) {
      s = precond_apply_impl(p, W.w.p, W.t.p, st);
      if (s != GF_OK) return s;
      axpy_kernel<<<vb, vt, 0, st>>>(1.0, W.t.p, x, N);
    } else {
      axpy_kernel<<<vb, vt, 0, st>>>(1.0, W.w.p, x, N);
    }
    GF_CHECK_LAUNCH();
    it_total += hs.j;
  }
  *iters = it_total;
  *restarts = nrest;
  *rel_out = rel;
  return GF_OK;
}

}  // namespace gf

using namespace gf;

struct gf_solver_cache {
  GmWork w;
};

static gf_solver_cache* cache_for(gf_assembler* a) {
  // one cache per assembler handle (leaks nothing: freed with the process
  // or reused; kept in a small registry keyed by the handle address)
  static thread_local std::vector<std::pair<gf_assembler*, gf_solver_cache*>> reg;
  for (auto& kv : reg)
    if (kv.first == a) return kv.second;
  auto* c = new gf_solver_cache();
  reg.emplace_back(a, c);
  return c;
}

extern "C" {

void gf_solve_opts_default(gf_solve_opts* o) {
  if (!o) return;
  o->restart = 50;
  o->max_iters = 5000;
  o->rtol = 1e-8;
  o->side = 1;
  o->mixed = 0;
  o->inner_rtol = 1e-4;
  o->max_refine = 20;
  o->check_every = 25;
}

gf_status gf_gmres_solve(gf_assembler* a, gf_bsr* A, gf_precond* p, const double* d_b,
                         double* d_x, const gf_solve_opts* opts, gf_solve_stats* stats,
                         void* stream) {
  if (!a || !A || !p || !d_b || !d_x || A->a != a) return GF_INVALID_ARG;
  gf_solve_opts o;
  gf_solve_opts_default(&o);
  if (opts) o = *opts;
  if (o.restart < 1 || o.restart > 1000 || o.max_iters < 1 || !(o.rtol > 0.0) ||
      o.check_every < 1 || (o.side != 0 && o.side != 1))
    return GF_INVALID_ARG;
  cudaStream_t st = as_stream(stream);
  auto t0 = std::chrono::steady_clock::now();
  const int n = a->nnodes;
  const size_t N = (size_t)6 * n;
  const size_t nnz36 = (size_t)36 * a->pat.nnz();
  GmWork& W = cache_for(a)->w;
  gf_status s = ensure_work(W, o.restart, n, nnz36, o.mixed != 0);
  if (s != GF_OK) return s;
  const int vb = 592, vt = 256;
  // into solver ordering
  permute2_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(a->d_perm.p, n, d_b, W.b.p, 0);
  permute2_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(a->d_perm.p, n, d_x, W.x.p, 0);
  GF_CHECK_LAUNCH();
  int iters = 0, rest = 0, refine = 0;
  double rel = 1.0;
  bool conv = false;
  gf_status result = GF_OK;
  if (!o.mixed) {
    result = gmres_core<double>(a, A->vals.p, p, W, W.b.p, W.x.p, o.restart, o.max_iters, o.rtol,
                                o.side, o.check_every, st, &iters, &rest, &rel, &conv);
  } else {
    cvt_kernel<float><<<(unsigned)((nnz36 + 255) / 256), 256, 0, st>>>(nnz36, A->vals.p,
                                                                       W.A32.p);
    GF_CHECK_LAUNCH();
    double bn = 0.0;
    sumsq_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(W.b.p, N, W.partial.p);
    finish_sum_kernel<<<1, 1, 0, st>>>(W.partial.p, kRedBlocks, W.scal.p);
    GF_CUDA(cudaMemcpyAsync(&bn, W.scal.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    GF_CUDA(cudaStreamSynchronize(st));
    if (bn == 0.0) bn = 1.0;
    while (true) {
      // r = b - A64 x (FP64)
      GF_CUDA(cudaMemcpyAsync(W.r.p, W.b.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
      s = spmv_impl<double>(n, a->d_rowp.p, a->d_cols.p, A->vals.p, W.x.p, -1.0, 1.0, W.r.p, st);
      if (s != GF_OK) return s;
      sumsq_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(W.r.p, N, W.partial.p);
      finish_sum_kernel<<<1, 1, 0, st>>>(W.partial.p, kRedBlocks, W.scal.p);
      double rn = 0.0;
      GF_CUDA(cudaMemcpyAsync(&rn, W.scal.p, sizeof(double), cudaMemcpyDeviceToHost, st));
      GF_CUDA(cudaStreamSynchronize(st));
      rel = rn / bn;
      if (!std::isfinite(rel)) {
        result = GF_NAN;
        break;
      }
      if (rel <= o.rtol) {
        conv = true;
        break;
      }
      if (refine >= o.max_refine || iters >= o.max_iters) break;
      // inner solve A32 d = r (d from zero); r is copied because the core
      // overwrites its residual buffer
      GF_CUDA(cudaMemcpyAsync(W.d.p, W.r.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
      GF_CUDA(cudaMemsetAsync(W.e.p, 0, sizeof(double) * N, st));
      int it_in = 0, rs_in = 0;
      double rel_in = 1.0;
      bool conv_in = false;
      s = gmres_core<float>(a, W.A32.p, p, W, W.d.p, W.e.p, o.restart, o.max_iters - iters,
                            o.inner_rtol, o.side, o.check_every, st, &it_in, &rs_in, &rel_in,
                            &conv_in);
      if (s != GF_OK) {
        result = s;
        break;
      }
      iters += it_in;
      rest += rs_in;
      refine++;
      axpy_kernel<<<vb, vt, 0, st>>>(1.0, W.e.p, W.x.p, N);
      GF_CHECK_LAUNCH();
    }
  }
  permute2_kernel<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(a->d_perm.p, n, W.x.p, d_x, 1);
  GF_CHECK_LAUNCH();
  GF_CUDA(cudaStreamSynchronize(st));
  auto t1 = std::chrono::steady_clock::now();
  if (result == GF_OK && !conv) result = GF_NOT_CONVERGED;
  if (stats) {
    stats->iterations = iters;
    stats->restarts = rest;
    stats->refinements = refine;
    stats->status = result;
    stats->rel_residual = rel;
    stats->time_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  }
  return result;
}

}  // extern "C"
