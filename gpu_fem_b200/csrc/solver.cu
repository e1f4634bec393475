// BSR SpMV, block ILU(k) numeric factorization, level-ordered triangular
// solves and the device-resident GMRES / iterative-refinement driver.
//
// Reference: cusparseDbsrmv, cusparseDbsrilu02 and cusparseDbsrsv2_solve as
// called by examples/iterative/gmres.cu:374-771, and the GMRES loop there.
//
// Triangular dependencies (factorization and both solves) are handled in
// one persistent launch per sweep: warps take rows in level order from an
// atomic counter and wait on per-row ready flags of the rows they depend on.
// Every row a warp waits for was taken earlier by a running warp, so the
// sweep cannot deadlock; every wait is bounded (kSpinLimit polls) and a wait
// that runs out sets an error bit in the status word instead of hanging.
// Flags carry an epoch read from device memory, so the same launch
// sequence can be captured in a CUDA graph and replayed.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "gf_internal.h"

namespace gf {

constexpr long long kSpinLimit = 1ll << 26;
enum { ST_TIMEOUT = 1, ST_ZERO_PIVOT = 2, ST_NAN = 4 };

struct SweepCtl {
  int epoch;     // incremented before every sweep
  int counter;   // work counter, reset with the epoch
  int status;    // error bits
  int pivot;     // first zero-pivot row + 1
};

// ------------------------------------------------------------------ SpMV
// y = alpha A x + beta y. One warp per block row; 4 groups of 6 lanes, lane
// (g, r) handles row r of block 4k+g; 6-lane groups are reduced with two
// shuffles.
template <class VT>
__global__ void spmv_kernel(int n, const int32_t* __restrict__ rowp,
                            const int32_t* __restrict__ cols, const VT* __restrict__ A,
                            const double* __restrict__ x, double alpha, double beta,
                            double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  const int g = lane / 6, r = lane % 6;
  double acc = 0.0;
  if (g < 4) {
    const int b0 = rowp[row], b1 = rowp[row + 1];
    for (int blk = b0 + g; blk < b1; blk += 4) {
      const VT* a = A + 36 * (size_t)blk + 6 * r;
      const double* xx = x + 6 * (size_t)cols[blk];
#pragma unroll
      for (int c = 0; c < 6; c++) acc = fma((double)a[c], xx[c], acc);
    }
  }
  acc += __shfl_down_sync(0xffffffffu, acc, 12);
  acc += __shfl_down_sync(0xffffffffu, acc, 6);
  if (lane < 6) {
    double* yy = y + 6 * (size_t)row + lane;
    *yy = (beta == 0.0) ? alpha * acc : alpha * acc + beta * (*yy);
  }
}

// ------------------------------------------------------------ sweep control
__global__ void sweep_begin(SweepCtl* c) {
  c->epoch += 1;
  c->counter = 0;
}

__device__ __forceinline__ int fetch_row(SweepCtl* c, int lane) {
  int idx = 0;
  if (lane == 0) idx = atomicAdd(&c->counter, 1);
  return __shfl_sync(0xffffffffu, idx, 0);
}

__device__ __forceinline__ void wait_flag(const int* flags, int k, int epoch, SweepCtl* c) {
  long long spins = 0;
  while (*((volatile const int*)&flags[k]) != epoch) {
    if (++spins > kSpinLimit) {
      atomicOr(&c->status, ST_TIMEOUT);
      break;
    }
  }
  __threadfence();
}

__device__ __forceinline__ void publish(int* flags, int i, int epoch, int lane) {
  __threadfence();
  __syncwarp();
  if (lane == 0) *((volatile int*)&flags[i]) = epoch;
}

// ----------------------------------------------------- block ILU factorization
// IKJ block ILU on the given pattern (FP64, in place). Lower blocks become
// L_ik = A_ik U_kk^{-1}; the diagonal block is replaced by U_ii^{-1}.
__device__ void inv6_warp(double* M, double* Inv, int lane, SweepCtl* ctl, int row) {
  // Gauss-Jordan with partial pivoting on a 6x6 block held in shared memory;
  // lane t < 36 owns one entry of the augmented right half via two passes.
  if (lane < 32) {
    for (int t = lane; t < 36; t += 32) Inv[t] = (t / 6 == t % 6) ? 1.0 : 0.0;
  }
  __syncwarp();
  for (int c = 0; c < 6; c++) {
    int p = c;
    double best = fabs(M[6 * c + c]);
    for (int r = c + 1; r < 6; r++) {
      const double v = fabs(M[6 * r + c]);
      if (v > best) {
        best = v;
        p = r;
      }
    }
    if (!(best > 0.0) || !isfinite(best)) {
      if (lane == 0) {
        atomicOr(&ctl->status, ST_ZERO_PIVOT);
        atomicCAS(&ctl->pivot, 0, row + 1);
      }
    }
    __syncwarp();
    if (p != c && lane < 12) {
      double* src = lane < 6 ? M : Inv;
      const int k = lane % 6;
      const double t0 = src[6 * p + k];
      src[6 * p + k] = src[6 * c + k];
      src[6 * c + k] = t0;
    }
    __syncwarp();
    const double piv = 1.0 / M[6 * c + c];
    __syncwarp();
    if (lane < 12) {
      double* dst = lane < 6 ? M : Inv;
      dst[6 * c + lane % 6] *= piv;
    }
    __syncwarp();
    // eliminate column c from other rows: lanes cover (row, col) of both halves
    double f[6];
    for (int r = 0; r < 6; r++) f[r] = M[6 * r + c];
    __syncwarp();
    for (int t = lane; t < 72; t += 32) {
      const int half = t / 36, rr = (t % 36) / 6, k = t % 6;
      if (rr == c) continue;
      double* dst = half ? Inv : M;
      dst[6 * rr + k] -= f[rr] * dst[6 * c + k];
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(128) ilu_factor_kernel(
    int n, const int32_t* __restrict__ rowp, const int32_t* __restrict__ cols,
    const int32_t* __restrict__ diag, const int32_t* __restrict__ order, double* LU, int* flags,
    SweepCtl* ctl) {
  __shared__ double sm[4][3][36];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* Lb = sm[warp][0];
  double* M = sm[warp][1];
  double* Inv = sm[warp][2];
  const int epoch = ctl->epoch;
  while (true) {
    const int idx = fetch_row(ctl, lane);
    if (idx >= n) break;
    const int i = order[idx];
    const int r0 = rowp[i], r1 = rowp[i + 1], di = diag[i];
    for (int kp = r0; kp < di; kp++) {
      const int k = cols[kp];
      if (lane == 0) wait_flag(flags, k, epoch, ctl);
      __syncwarp();
      // L_ik = A_ik * U_kk^{-1}
      const double* Ukk = LU + 36 * (size_t)diag[k];
      const double* Aik = LU + 36 * (size_t)kp;
      for (int t = lane; t < 36; t += 32) {
        const int r = t / 6, c = t % 6;
        double s = 0.0;
#pragma unroll
        for (int m = 0; m < 6; m++) s = fma(Aik[6 * r + m], __ldcg(&Ukk[6 * m + c]), s);
        Lb[t] = s;
      }
      __syncwarp();
      for (int t = lane; t < 36; t += 32) LU[36 * (size_t)kp + t] = Lb[t];
      // A_ij -= L_ik U_kj for j > k in row k that are present in row i
      int tp = kp + 1;
      const int k1 = rowp[k + 1];
      for (int jp = diag[k] + 1; jp < k1; jp++) {
        const int j = cols[jp];
        while (tp < r1 && cols[tp] < j) tp++;
        if (tp >= r1) break;
        if (cols[tp] != j) continue;
        const double* Ukj = LU + 36 * (size_t)jp;
        double* Aij = LU + 36 * (size_t)tp;
        for (int t = lane; t < 36; t += 32) {
          const int r = t / 6, c = t % 6;
          double s = 0.0;
#pragma unroll
          for (int m = 0; m < 6; m++) s = fma(Lb[6 * r + m], __ldcg(&Ukj[6 * m + c]), s);
          Aij[t] -= s;
        }
      }
      __syncwarp();
    }
    // invert the updated diagonal block in place
    double* Dii = LU + 36 * (size_t)di;
    for (int t = lane; t < 36; t += 32) M[t] = Dii[t];
    __syncwarp();
    inv6_warp(M, Inv, lane, ctl, i);
    for (int t = lane; t < 36; t += 32) {
      const double v = Inv[t];
      if (!isfinite(v)) {
        atomicOr(&ctl->status, ST_ZERO_PIVOT);
        atomicCAS(&ctl->pivot, 0, i + 1);
      }
      Dii[t] = v;
    }
    publish(flags, i, epoch, lane);
  }
}

// --------------------------------------------------------- triangular solves
// Lower: y_i = r_i - sum_{k<i} L_ik y_k (unit block diagonal).
// Upper: x_i = Uinv_ii (y_i - sum_{j>i} U_ij x_j).
template <class VT, bool UPPER>
__global__ void __launch_bounds__(128) trisolve_kernel(
    int n, const int32_t* __restrict__ rowp, const int32_t* __restrict__ cols,
    const int32_t* __restrict__ diag, const int32_t* __restrict__ order,
    const VT* __restrict__ LU, const double* __restrict__ rhs, double* out, int* flags,
    SweepCtl* ctl) {
  const int lane = threadIdx.x & 31;
  const int g = lane / 6, r = lane % 6;
  const int epoch = ctl->epoch;
  while (true) {
    const int idx = fetch_row(ctl, lane);
    if (idx >= n) break;
    const int i = order[idx];
    const int di = diag[i];
    const int b0 = UPPER ? di + 1 : rowp[i];
    const int b1 = UPPER ? rowp[i + 1] : di;
    double acc = 0.0;
    if (g < 4) {
      for (int blk = b0 + g; blk < b1; blk += 4) {
        const int k = cols[blk];
        VT a[6];
#pragma unroll
        for (int c = 0; c < 6; c++) a[c] = LU[36 * (size_t)blk + 6 * r + c];
        wait_flag(flags, k, epoch, ctl);
        const double* xk = out + 6 * (size_t)k;
#pragma unroll
        for (int c = 0; c < 6; c++) acc = fma((double)a[c], __ldcg(&xk[c]), acc);
      }
    }
    acc += __shfl_down_sync(0xffffffffu, acc, 12);
    acc += __shfl_down_sync(0xffffffffu, acc, 6);
    const double t = (lane < 6 ? rhs[6 * (size_t)i + lane] : 0.0) - acc;
    if (!UPPER) {
      if (lane < 6) __stcg(&out[6 * (size_t)i + lane], t);
    } else {
      double v = 0.0;
#pragma unroll
      for (int c = 0; c < 6; c++) {
        const double tc = __shfl_sync(0xffffffffu, t, c);
        if (lane < 6) v = fma((double)LU[36 * (size_t)di + 6 * lane + c], tc, v);
      }
      if (lane < 6) __stcg(&out[6 * (size_t)i + lane], v);
    }
    publish(flags, i, epoch, lane);
  }
}

// ------------------------------------------------------------ small kernels
__global__ void scatter_values_kernel(int nA, const int32_t* __restrict__ map,
                                      const double* __restrict__ A, double* __restrict__ LU) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)nA * 36) return;
  LU[36 * (size_t)map[t / 36] + t % 36] = A[t];
}
template <class T2>
__global__ void convert_kernel(size_t n, const double* __restrict__ in, T2* __restrict__ out) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = (T2)in[t];
}

}  // namespace gf

using namespace gf;

struct gf_precond {
  gf_assembler* a = nullptr;
  int fill = 0, prec = GF_PREC_FP64;
  Pattern pat;
  int nlevL = 0, nlevU = 0;
  DevBuf<int32_t> d_rowp, d_cols, d_diag, d_orderL, d_orderU, d_amap, d_flags;
  DevBuf<double> d_lu;
  DevBuf<float> d_lu32;
  DevBuf<double> d_tmp;
  DevBuf<SweepCtl> d_ctl;
};

namespace gf {
gf_status precond_apply_impl(gf_precond* p, const double* r, double* z, cudaStream_t st);
}

extern "C" {

gf_status gf_precond_create(gf_assembler* a, int32_t fill_level, int32_t precision,
                            gf_precond** out) {
  if (!a || !out || fill_level < 0 || (precision != GF_PREC_FP64 && precision != GF_PREC_FP32))
    return GF_INVALID_ARG;
  gf_precond* p = new gf_precond();
  p->a = a;
  p->fill = fill_level;
  p->prec = precision;
  p->pat = fill_level == 0 ? a->pat : iluk_pattern(a->pat, fill_level);
  const int n = a->nnodes;
  std::vector<int32_t> diag(n), lvL, lvU, ordL(n), ordU(n), amap(a->pat.nnz());
  for (int i = 0; i < n; i++) {
    const int32_t* b0 = p->pat.cols.data() + p->pat.rowp[i];
    const int32_t* b1 = p->pat.cols.data() + p->pat.rowp[i + 1];
    diag[i] = (int32_t)(std::lower_bound(b0, b1, i) - p->pat.cols.data());
    for (int jp = a->pat.rowp[i]; jp < a->pat.rowp[i + 1]; jp++) {
      const int32_t* f = std::lower_bound(b0, b1, a->pat.cols[jp]);
      amap[jp] = (int32_t)(f - p->pat.cols.data());
    }
  }
  p->nlevL = levels(p->pat, true, lvL);
  p->nlevU = levels(p->pat, false, lvU);
  for (int i = 0; i < n; i++) ordL[i] = ordU[i] = i;
  std::stable_sort(ordL.begin(), ordL.end(), [&](int x, int y) { return lvL[x] < lvL[y]; });
  std::stable_sort(ordU.begin(), ordU.end(), [&](int x, int y) { return lvU[x] < lvU[y]; });
  cudaError_t e = cudaSuccess;
  auto up = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  up(p->d_rowp.upload(p->pat.rowp));
  up(p->d_cols.upload(p->pat.cols));
  up(p->d_diag.upload(diag));
  up(p->d_orderL.upload(ordL));
  up(p->d_orderU.upload(ordU));
  up(p->d_amap.upload(amap));
  up(p->d_flags.alloc(n));
  if (e == cudaSuccess) up(cudaMemset(p->d_flags.p, 0, sizeof(int32_t) * n));
  up(p->d_lu.alloc((size_t)36 * p->pat.nnz()));
  if (precision == GF_PREC_FP32) up(p->d_lu32.alloc((size_t)36 * p->pat.nnz()));
  up(p->d_tmp.alloc((size_t)6 * n));
  up(p->d_ctl.alloc(1));
  if (e == cudaSuccess) up(cudaMemset(p->d_ctl.p, 0, sizeof(SweepCtl)));
  if (e != cudaSuccess) {
    set_last_error("gf_precond_create", e);
    delete p;
    return e == cudaErrorMemoryAllocation ? GF_OOM : GF_CUDA_ERROR;
  }
  *out = p;
  return GF_OK;
}

gf_status gf_precond_destroy(gf_precond* p) {
  delete p;
  return GF_OK;
}

gf_status gf_precond_info(const gf_precond* p, int32_t* nnzb, int32_t* nl, int32_t* nu) {
  if (!p) return GF_INVALID_ARG;
  if (nnzb) *nnzb = p->pat.nnz();
  if (nl) *nl = p->nlevL;
  if (nu) *nu = p->nlevU;
  return GF_OK;
}

gf_status gf_precond_get(const gf_precond* p, int32_t* rowPtr, int32_t* colPtr,
                         double* h_values) {
  if (!p) return GF_INVALID_ARG;
  if (rowPtr) std::copy(p->pat.rowp.begin(), p->pat.rowp.end(), rowPtr);
  if (colPtr) std::copy(p->pat.cols.begin(), p->pat.cols.end(), colPtr);
  if (h_values)
    GF_CUDA(cudaMemcpy(h_values, p->d_lu.p, sizeof(double) * 36 * p->pat.nnz(),
                       cudaMemcpyDeviceToHost));
  return GF_OK;
}

static int persistent_blocks() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms * 8;
}

gf_status gf_precond_factor(gf_precond* p, gf_bsr* A, void* stream) {
  if (!p || !A || A->a != p->a) return GF_INVALID_ARG;
  cudaStream_t st = as_stream(stream);
  const int n = p->a->nnodes;
  const size_t nv = (size_t)36 * p->pat.nnz();
  GF_CUDA(cudaMemsetAsync(p->d_lu.p, 0, sizeof(double) * nv, st));
  const size_t na = (size_t)36 * p->a->pat.nnz();
  scatter_values_kernel<<<(unsigned)((na + 255) / 256), 256, 0, st>>>(p->a->pat.nnz(),
                                                                      p->d_amap.p, A->vals.p,
                                                                      p->d_lu.p);
  GF_CHECK_LAUNCH();
  GF_CUDA(cudaMemsetAsync(&p->d_ctl.p->status, 0, 2 * sizeof(int), st));
  sweep_begin<<<1, 1, 0, st>>>(p->d_ctl.p);
  GF_CHECK_LAUNCH();
  const int nb = std::min(persistent_blocks(), (n + 3) / 4);
  ilu_factor_kernel<<<nb, 128, 0, st>>>(n, p->d_rowp.p, p->d_cols.p, p->d_diag.p,
                                        p->d_orderL.p, p->d_lu.p, p->d_flags.p, p->d_ctl.p);
  GF_CHECK_LAUNCH();
  if (p->prec == GF_PREC_FP32) {
    convert_kernel<float><<<(unsigned)((nv + 255) / 256), 256, 0, st>>>(nv, p->d_lu.p,
                                                                        p->d_lu32.p);
    GF_CHECK_LAUNCH();
  }
  SweepCtl h;
  GF_CUDA(cudaMemcpyAsync(&h, p->d_ctl.p, sizeof(SweepCtl), cudaMemcpyDeviceToHost, st));
  GF_CUDA(cudaStreamSynchronize(st));
  if (h.status & ST_TIMEOUT) return GF_TIMEOUT;
  if (h.status & ST_ZERO_PIVOT) return GF_ZERO_PIVOT;
  return GF_OK;
}

gf_status gf_precond_apply(gf_precond* p, const double* d_r, double* d_z, void* stream) {
  if (!p || !d_r || !d_z) return GF_INVALID_ARG;
  return precond_apply_impl(p, d_r, d_z, as_stream(stream));
}

}  // extern "C"

namespace gf {

gf_status precond_apply_impl(gf_precond* p, const double* r, double* z, cudaStream_t st) {
  const int n = p->a->nnodes;
  const int nb = std::min(persistent_blocks(), (n + 3) / 4);
  sweep_begin<<<1, 1, 0, st>>>(p->d_ctl.p);
  if (p->prec == GF_PREC_FP32) {
    trisolve_kernel<float, false><<<nb, 128, 0, st>>>(n, p->d_rowp.p, p->d_cols.p, p->d_diag.p,
                                                      p->d_orderL.p, p->d_lu32.p, r,
                                                      p->d_tmp.p, p->d_flags.p, p->d_ctl.p);
    sweep_begin<<<1, 1, 0, st>>>(p->d_ctl.p);
    trisolve_kernel<float, true><<<nb, 128, 0, st>>>(n, p->d_rowp.p, p->d_cols.p, p->d_diag.p,
                                                     p->d_orderU.p, p->d_lu32.p, p->d_tmp.p, z,
                                                     p->d_flags.p, p->d_ctl.p);
  } else {
    trisolve_kernel<double, false><<<nb, 128, 0, st>>>(n, p->d_rowp.p, p->d_cols.p, p->d_diag.p,
                                                       p->d_orderL.p, p->d_lu.p, r, p->d_tmp.p,
                                                       p->d_flags.p, p->d_ctl.p);
    sweep_begin<<<1, 1, 0, st>>>(p->d_ctl.p);
    trisolve_kernel<double, true><<<nb, 128, 0, st>>>(n, p->d_rowp.p, p->d_cols.p, p->d_diag.p,
                                                      p->d_orderU.p, p->d_lu.p, p->d_tmp.p, z,
                                                      p->d_flags.p, p->d_ctl.p);
  }
  GF_CHECK_LAUNCH();
  return GF_OK;
}

template <class VT>
gf_status spmv_impl(int n, const int32_t* rowp, const int32_t* cols, const VT* A,
                    const double* x, double alpha, double beta, double* y, cudaStream_t st) {
  const int threads = 256, rows_per_block = threads / 32;
  spmv_kernel<VT><<<(n + rows_per_block - 1) / rows_per_block, threads, 0, st>>>(
      n, rowp, cols, A, x, alpha, beta, y);
  GF_CHECK_LAUNCH();
  return GF_OK;
}
template gf_status spmv_impl<double>(int, const int32_t*, const int32_t*, const double*,
                                     const double*, double, double, double*, cudaStream_t);
template gf_status spmv_impl<float>(int, const int32_t*, const int32_t*, const float*,
                                    const double*, double, double, double*, cudaStream_t);

gf_status precond_status(gf_precond* p, cudaStream_t st, int* bits) {
  SweepCtl h;
  GF_CUDA(cudaMemcpyAsync(&h, p->d_ctl.p, sizeof(SweepCtl), cudaMemcpyDeviceToHost, st));
  GF_CUDA(cudaStreamSynchronize(st));
  *bits = h.status;
  return GF_OK;
}

int* precond_status_ptr(gf_precond* p) { return &p->d_ctl.p->status; }

}  // namespace gf

extern "C" gf_status gf_bsr_spmv(gf_bsr* m, double alpha, const double* d_x, double beta,
                                 double* d_y, void* stream) {
  if (!m || !d_x || !d_y) return GF_INVALID_ARG;
  return spmv_impl<double>(m->a->nnodes, m->a->d_rowp.p, m->a->d_cols.p, m->vals.p, d_x, alpha,
                           beta, d_y, as_stream(stream));
}
