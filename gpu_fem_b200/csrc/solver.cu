// Batched solver engine: BSR SpMV, block ILU(k) factorization, block
// triangular sweeps and restarted GMRES / iterative refinement over a batch
// of independent problems (a single problem is a batch of one).
//
// Reference: cusparseDbsrmv, cusparseDbsrilu02 and cusparseDbsrsv2_solve as
// called by examples/iterative/gmres.cu:374-771, and the GMRES loop there
// (left-preconditioned GMRES(m), MGS, host Givens; bugs fixed: dot length
// nvars, m+1 basis vectors, restarts).
//
// Batch layout: every problem keeps its own pattern / values / factor
// buffers; a device table of ProbDev descriptors gives each kernel the
// problem of a global block row (row_prob), its offset in the batch vector
// space and its triangular level structure.
//  * SpMV and the GMRES vector work run over all rows / chunks of the batch.
//  * Triangular work (the factorization and both sweeps) runs one CTA per
//    problem: the CTA walks the problem's levels and separates them with
//    __syncthreads(), so a dependency costs a block barrier (tens of ns)
//    instead of a device-wide round trip; the problems of a batch run on
//    different SMs at once.
//
// GMRES reductions are segmented per problem over fixed 4096-entry chunks
// aligned to each problem's own vector, with per-problem Arnoldi states, so
// a problem's iterates are bitwise identical alone and inside any batch.
#include <algorithm>
#include <atomic>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <thread>
#include <type_traits>

#include "gf_internal.h"

namespace gf {

enum { ST_TIMEOUT = 1, ST_ZERO_PIVOT = 2, ST_NAN = 4 };
constexpr int kChunk = 4096;
constexpr int kRedThreads = 256;

struct SweepCtl {
  int status;
  int pivot;
};

// ------------------------------------------------ barriers and bulk copies
constexpr unsigned long long kWaitNs = 2000000000ull;  // default bound of every device-side wait
constexpr int kSweepCta = 2;  // CTAs (one thread-block cluster) per problem for triangular work

// Bound (ns) of the waits that end when a bulk copy lands or when the
// partner CTA of a cluster arrives (gf_test_set_waits changes it). The waits
// that drain a CTA's own copies in flight before it leaves always use kWaitNs.
__device__ unsigned long long g_wait_ns = kWaitNs;
// Failure-injection knob for tests (gf_test_set_waits): when non-zero, CTA
// rank 1 of a split problem never arrives on its partner's meeting barriers,
// so the partner's bounded wait runs out and the launch reports ST_TIMEOUT.
// Every wait stays bounded and both CTAs still meet on the final cluster
// barrier, so nothing hangs.
__device__ int g_skip_meet = 0;

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// as mbar_try_wait, but the thread may be suspended (not spinning on issue
// slots) until the phase completes or about hint_ns have passed
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, unsigned parity,
                                                    unsigned hint_ns) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}
// bounded wait; returns false if limit_ns passed first
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                          unsigned long long limit_ns) {
  // the timer is read only once the first test fails (reading it is slow)
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  unsigned n = 0;
  while (!mbar_try_wait(bar, parity)) {
    if ((++n & 255u) == 0u && gtimer() - t0 > limit_ns) return false;
  }
  return true;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// address of the same shared-memory location in CTA `rank` of the cluster
__device__ __forceinline__ unsigned cluster_map(unsigned addr, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_store(unsigned addr, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}
// arrive on an mbarrier of another CTA of the cluster (releases this CTA's
// earlier writes at cluster scope)
__device__ __forceinline__ void mbar_arrive_remote(unsigned addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(addr)
               : "memory");
}
// bounded wait with acquire at cluster scope; false if limit_ns passed first
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, unsigned parity,
                                                  unsigned long long limit_ns) {
  unsigned long long t0 = 0;
  unsigned n = 0;
  while (true) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    if (n == 0) t0 = gtimer();  // read only once the first test fails (reading it is slow)
    if ((++n & 255u) == 0u && gtimer() - t0 > limit_ns) return false;
  }
}
// all threads of all CTAs of the cluster
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;" :::
                   "memory");
}


// ------------------------------------------------------------------ SpMV
// y = alpha A x + beta y over all rows of live problems; one warp per block
// row, 4 groups of 6 lanes (group g takes blocks g, g+4, ...).
template <class VT>
__global__ void bspmv_kernel(int nrows, const int32_t* __restrict__ row_prob,
                             const ProbDev* __restrict__ P, const int* __restrict__ live,
                             const double* __restrict__ x, double alpha, double beta,
                             double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int grow = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (grow >= nrows) return;
  const int p = row_prob[grow];
  if (live && !live[p]) return;
  const ProbDev& d = P[p];
  const int i = grow - d.off;
  const VT* A = sizeof(VT) == 8 ? (const VT*)d.A64 : (const VT*)d.A32;
  const double* xb = x + 6 * (size_t)d.off;
  const int g = lane / 6, r = lane % 6;
  double acc = 0.0;
  if (g < 4) {
    const int b0 = d.rowp[i], b1 = d.rowp[i + 1];
    for (int blk = b0 + g; blk < b1; blk += 4) {
      const VT* a = A + 36 * (size_t)blk + 6 * r;
      const double* xx = xb + 6 * (size_t)d.cols[blk];
#pragma unroll
      for (int c = 0; c < 6; c++) acc = fma((double)a[c], xx[c], acc);
    }
  }
  acc += __shfl_down_sync(0xffffffffu, acc, 12);
  acc += __shfl_down_sync(0xffffffffu, acc, 6);
  if (lane < 6) {
    double* yy = y + 6 * (size_t)grow + lane;
    *yy = (beta == 0.0) ? alpha * acc : alpha * acc + beta * (*yy);
  }
}

// ----------------------------------------------------- block ILU factorization
__device__ void inv6_warp(double* M, double* Inv, int lane, SweepCtl* ctl, int row) {
  for (int t = lane; t < 36; t += 32) Inv[t] = (t / 6 == t % 6) ? 1.0 : 0.0;
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

// IKJ block ILU on each problem's ILU pattern (FP64, in place): lower blocks
// become L_ik = A_ik U_kk^{-1}, the diagonal block is replaced by U_ii^{-1}.
// One warp factors one row. The row's values are staged in the warp's slice
// of shared memory (rows up to kFacVals blocks; longer rows are updated in
// global memory), so the read-modify-writes of the sequential steps cost a
// shared-memory latency, and the row is written back whole when it is final.
// Within a row the steps k (its lower blocks, ascending) are sequential; a
// step's updates A_ij -= L_ik U_kj over j in U(k) are spread over the lanes
// (lane = block slot b < 5, column c < 6; 2 slot batches in flight). The
// column lists and U_kj values of a step's first batch (final rows in
// global memory) are loaded together with U_kk^{-1}. Each row's column
// indices are staged for the searches j -> slot.
//
// Scheduling is dataflow, not level-synchronous: the warps of the CTAs a
// problem is given take its rows in factorization order (ascending lower
// level) from a per-problem counter, and step k of row i waits only until
// row k is final (its flag done[k] equals the launch's epoch, stored with
// release after all of row k's values). Rows of later levels therefore run
// while the rows they do not read are still being factored, and a row's
// early steps overlap the end of the rows it reads last. Every row that a
// warp waits for has a lower level, so it was taken earlier by a warp that
// is running; the waits end whatever the CTAs' residency. Each wait is still
// bounded: the first that runs out sets ST_TIMEOUT, which ends the others.
constexpr int kFacWarps = 8;
constexpr int kFacRow = 256;    // row blocks whose columns are staged in shared memory
constexpr int kFacVals = 80;    // row blocks whose values are staged in shared memory
constexpr int kFacPass = 6;     // passes of 5 U(k) blocks loaded at the start of a step
constexpr int kFacBatch = 2;    // passes of 5 blocks in flight per lane beyond those
constexpr int kFacMap = 1024;   // column span of a row whose column -> slot map is kept
// per warp: values, L_ik, the diagonal block and its inverse, columns, map
// and the row's step order
constexpr size_t kFacWarpSmem = sizeof(double) * (36 * kFacVals + 3 * 36) +
                                sizeof(int32_t) * kFacRow + sizeof(int16_t) * (kFacMap + kFacRow);
constexpr size_t kFacSmem = kFacWarps * kFacWarpSmem;

__device__ __forceinline__ int find_col(const int32_t* c, int lo, int hi, int j) {
  const int end = hi;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (c[mid] < j)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < end && c[lo] == j) ? lo : -1;
}

__device__ __forceinline__ int ld_relaxed_gpu(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Waits (bounded) until *flag == want, then acquires what its writer
// released. False when the bound ran out (ST_TIMEOUT set here) or another
// wait already ran out.
__device__ bool wait_flag(const int* flag, int want, unsigned long long limit, SweepCtl* ctl) {
  if (ld_relaxed_gpu(flag) == want) {
    fence_acq_rel_gpu();
    return true;
  }
  const unsigned long long t0 = gtimer();
  while (true) {
    if (ld_relaxed_gpu(flag) == want) {
      fence_acq_rel_gpu();
      return true;
    }
    if (ld_relaxed_gpu(&ctl->status) & ST_TIMEOUT) return false;
    if (gtimer() - t0 > limit) {
      atomicOr(&ctl->status, ST_TIMEOUT);
      return false;
    }
  }
}

// cta_prob[blockIdx.x]: the problem a CTA works on; grab[p]: problem p's row
// counter (zero at launch).
__global__ void __launch_bounds__(kFacWarps * 32) bfactor_df(const ProbDev* __restrict__ P,
                                                            const int32_t* __restrict__ cta_prob,
                                                            int* __restrict__ grab, int epoch,
                                                            SweepCtl* ctl) {
  extern __shared__ __align__(16) unsigned char fsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* ws = fsm + (size_t)warp * kFacWarpSmem;
  double* sR = reinterpret_cast<double*>(ws);  // staged row values
  double* Lb = sR + 36 * kFacVals;             // L_ik of the current step
  double* sM = Lb + 36;                        // diagonal block (pivoting copy)
  double* sI = sM + 36;                        // its inverse
  int32_t* sC = reinterpret_cast<int32_t*>(sI + 36);
  int16_t* sMap = reinterpret_cast<int16_t*>(sC + kFacRow);  // column - base -> slot - r0, or -1
  int16_t* sOrd = sMap + kFacMap;                              // step t -> slot - r0
  for (int t = lane; t < kFacMap; t += 32) sMap[t] = -1;
  __syncwarp();
  const int b = lane / 6, c = lane % 6;  // update slot and column (lanes 30, 31 idle)
  const int prob = cta_prob[blockIdx.x];
  const ProbDev d = P[prob];
  int* counter = grab + prob;
  int* done = d.done;
  const unsigned long long wlim = g_wait_ns;
  const bool skip_first = g_skip_meet != 0;  // failure injection: row 0 of the order never published
  const int32_t* rowp = d.prowp;
  const int32_t* cols = d.pcols;
  const int32_t* diag = d.pdiag;
  double* LU = d.LU64;
  int idx = lane == 0 ? atomicAdd(counter, 1) : 0;
  idx = __shfl_sync(0xffffffffu, idx, 0);
  bool live = true;
  while (idx < d.n && live) {
    const int nidx = lane == 0 ? atomicAdd(counter, 1) : 0;  // the next row, in flight meanwhile
    const int i = d.levLrows[idx];
    const int r0 = rowp[i], r1 = rowp[i + 1], di = diag[i], len = r1 - r0;
    const bool cstaged = len <= kFacRow;
    const bool vstaged = len <= kFacVals;
    const int32_t* rc = cstaged ? sC - r0 : cols;  // rc[kp] = column of slot kp
    double* R = vstaged ? sR - 36 * (size_t)r0 : LU;  // R[36 kp + e] = entry e of slot kp
    if (cstaged) {
      for (int t = lane; t < len; t += 32) sC[t] = cols[r0 + t];
      for (int t = lane; t < di - r0; t += 32) sOrd[t] = (int16_t)(d.pord[r0 + t] - r0);
    }
    // slot of the row's step t (r0 <= t < di)
    auto step_slot = [&](int t) { return cstaged ? r0 + sOrd[t - r0] : d.pord[t]; };
    // column -> slot map of the row when its column span fits (binary
    // searches otherwise)
    const int cbase = cols[r0], span = cols[r1 - 1] - cbase + 1;
    const bool mapped = span <= kFacMap;
    if (mapped)
      for (int t = lane; t < len; t += 32) sMap[cols[r0 + t] - cbase] = (int16_t)t;
    if (vstaged) {
      // eight loads in flight per lane
      const double* src = LU + 36 * (size_t)r0;
      const int nv = 36 * len;
      for (int t0 = 0; t0 < nv; t0 += 256) {
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const int t = t0 + 32 * q + lane;
          v[q] = t < nv ? src[t] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const int t = t0 + 32 * q + lane;
          if (t < nv) sR[t] = v[q];
        }
      }
    }
    __syncwarp();
    unsigned ready = 0;  // bit s: the row of step (window start + s) is final
    for (int st = r0; st < di; st++) {
      const int kp = step_slot(st);
      const int s = (st - r0) & 31;
      if (s == 0) {
        // the flags of the next 32 steps, one per lane; a lane that sees
        // its row final acquires it for the warp (the warp barrier below
        // orders that acquire before every lane's later loads)
        const int q = st + lane;
        const int f = q < di ? (ld_relaxed_gpu(done + rc[step_slot(q)]) == epoch) : 1;
        fence_acq_rel_gpu();
        ready = __ballot_sync(0xffffffffu, f);
        __syncwarp();
      }
      const int k = rc[kp];
      if (!((ready >> s) & 1u)) {
        int ok = lane == 0 ? (int)wait_flag(done + k, epoch, wlim, ctl) : 0;
        ok = __shfl_sync(0xffffffffu, ok, 0);
        __syncwarp();
        if (!ok) {
          live = false;
          break;
        }
      }
      const int u0 = diag[k] + 1, u1 = rowp[k + 1];
      // loads that do not depend on this row's earlier steps, all in flight
      // together: the first kFacPass x 5 blocks of U(k) (columns and values)
      // and U_kk^{-1}
      int jc[kFacPass];
      double u[kFacPass][6];
#pragma unroll
      for (int q = 0; q < kFacPass; q++) {
        const int jp = u0 + 5 * q + b;
        const bool in = lane < 30 && jp < u1;
        jc[q] = in ? cols[jp] : -1;
#pragma unroll
        for (int m = 0; m < 6; m++) u[q][m] = in ? LU[36 * (size_t)jp + 6 * m + c] : 0.0;
      }
      const double* Ukk = LU + 36 * (size_t)diag[k];
      double* Aik = R + 36 * (size_t)kp;
      double s0 = 0.0, s1 = 0.0;
      {
        const int r = lane / 6, cc = lane % 6;
#pragma unroll
        for (int m = 0; m < 6; m++) s0 = fma(Aik[6 * r + m], Ukk[6 * m + cc], s0);
        if (lane < 4) {
          const int r2 = (lane + 32) / 6, c2 = (lane + 32) % 6;
#pragma unroll
          for (int m = 0; m < 6; m++) s1 = fma(Aik[6 * r2 + m], Ukk[6 * m + c2], s1);
        }
      }
      __syncwarp();
      Lb[lane] = s0;
      Aik[lane] = s0;
      if (lane < 4) {
        Lb[32 + lane] = s1;
        Aik[32 + lane] = s1;
      }
      __syncwarp();
      {
        // targets of the prefetched blocks (distinct slots of this row), then
        // all their reads before any write
        int tp[kFacPass];
#pragma unroll
        for (int q = 0; q < kFacPass; q++) {
          if (mapped) {
            const int off = jc[q] - cbase;
            const int m = (jc[q] >= 0 && off < span) ? sMap[off] : -1;
            tp[q] = m >= 0 ? r0 + m : -1;
          } else {
            tp[q] = jc[q] >= 0 ? find_col(rc, kp + 1, r1, jc[q]) : -1;
          }
        }
        double lb[36];  // L_ik in registers for the updates
#pragma unroll
        for (int t = 0; t < 36; t++) lb[t] = Lb[t];
        double a[kFacPass][6];
#pragma unroll
        for (int q = 0; q < kFacPass; q++)
#pragma unroll
          for (int r = 0; r < 6; r++) a[q][r] = tp[q] >= 0 ? R[36 * (size_t)tp[q] + 6 * r + c] : 0.0;
#pragma unroll
        for (int q = 0; q < kFacPass; q++)
          if (tp[q] >= 0) {
#pragma unroll
            for (int r = 0; r < 6; r++) {
              double sacc = 0.0;
#pragma unroll
              for (int m = 0; m < 6; m++) sacc = fma(lb[6 * r + m], u[q][m], sacc);
              R[36 * (size_t)tp[q] + 6 * r + c] = a[q][r] - sacc;
            }
          }
      }
      // the rest of U(k) (rows longer than the prefetch), kFacBatch passes at a time
      for (int jb = u0 + 5 * kFacPass; jb < u1; jb += 5 * kFacBatch) {
        int jt[kFacBatch];
        double v[kFacBatch][6];
#pragma unroll
        for (int q = 0; q < kFacBatch; q++) {
          const int jp = jb + 5 * q + b;
          const bool in = lane < 30 && jp < u1;
          jt[q] = in ? cols[jp] : -1;
#pragma unroll
          for (int m = 0; m < 6; m++) v[q][m] = in ? LU[36 * (size_t)jp + 6 * m + c] : 0.0;
        }
        int tp[kFacBatch];
#pragma unroll
        for (int q = 0; q < kFacBatch; q++) {
          if (mapped) {
            const int off = jt[q] - cbase;
            const int m = (jt[q] >= 0 && off < span) ? sMap[off] : -1;
            tp[q] = m >= 0 ? r0 + m : -1;
          } else {
            tp[q] = jt[q] >= 0 ? find_col(rc, kp + 1, r1, jt[q]) : -1;
          }
        }
        double a[kFacBatch][6];
#pragma unroll
        for (int q = 0; q < kFacBatch; q++)
#pragma unroll
          for (int r = 0; r < 6; r++) a[q][r] = tp[q] >= 0 ? R[36 * (size_t)tp[q] + 6 * r + c] : 0.0;
#pragma unroll
        for (int q = 0; q < kFacBatch; q++)
          if (tp[q] >= 0) {
#pragma unroll
            for (int r = 0; r < 6; r++) {
              double sacc = 0.0;
#pragma unroll
              for (int m = 0; m < 6; m++) sacc = fma(Lb[6 * r + m], v[q][m], sacc);
              R[36 * (size_t)tp[q] + 6 * r + c] = a[q][r] - sacc;
            }
          }
      }
      __syncwarp();
    }
    if (!live) break;
    double* Dii = R + 36 * (size_t)di;
    for (int t = lane; t < 36; t += 32) sM[t] = Dii[t];
    __syncwarp();
    inv6_warp(sM, sI, lane, ctl, d.off + i);
    for (int t = lane; t < 36; t += 32) {
      const double v = sI[t];
      if (!isfinite(v)) {
        atomicOr(&ctl->status, ST_ZERO_PIVOT);
        atomicCAS(&ctl->pivot, 0, d.off + i + 1);
      }
      Dii[t] = v;
    }
    __syncwarp();
    if (vstaged) {
      double* dst = LU + 36 * (size_t)r0;
      for (int t = lane; t < 36 * len; t += 32) dst[t] = sR[t];
    }
    if (mapped)
      for (int t = lane; t < len; t += 32) sMap[cols[r0 + t] - cbase] = -1;
    // publish: every lane's stores of the row reach device scope before the
    // flag (release) says the row is final
    __threadfence();
    __syncwarp();
    if (lane == 0 && !(skip_first && idx == 0)) st_release_gpu(done + i, epoch);
    idx = __shfl_sync(0xffffffffu, nidx, 0);
  }
}

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


// ------------------------------------------- prefetched level-major sweeps
// A thread-block cluster of kSweepCta CTAs per problem walks the chunks of
// one triangle in level-major order (a chunk holds rows of one level); each
// CTA solves its half of every chunk's rows from its own stream, and the
// CTAs meet once per chunk on a pair of mbarriers (bounded waits, release /
// acquire at cluster scope). A ring of kStages shared-memory stages
// is filled by 1D bulk copies (cp.async.bulk, completion counted on an
// mbarrier) kStages-1 chunks ahead of the chunk being solved. The x
// entries a chunk multiplies come from two places:
//  - near: rows solved by the previous chunk, kept in a shared-memory ring
//    that both CTAs write (their own and, through distributed shared
//    memory, the partner's);
//  - far: rows solved two or more chunks earlier, loaded from global memory
//    one chunk ahead (issued right after the barrier that ends chunk c-1,
//    consumed by chunk c+1), together with chunk c+1's right-hand sides;
// so a chunk's critical path is two block barriers, shared-memory copies and
// its rows' 6x6 products. x / y live in global memory, written and re-read
// by the problem's cluster only.
constexpr int kSweepThreads = 512;
constexpr int kStages = 2;
constexpr size_t kSweepSmemMax = 220 * 1024;  // dynamic; the static part is < 1 KB

// Dynamic shared memory of one sweep: kStages staging buffers of `stage`
// bytes; two buffers (this chunk, next chunk) of gathered x (capb x 6
// doubles) and right-hand sides (capr x 6); the ring of the two latest
// chunks' results (2 slots x kSweepCta capr rows x 6).
__host__ __device__ inline size_t sweep_smem_bytes(int stage, int capb, int capr) {
  return kStages * (size_t)stage + 96 * ((size_t)capb + capr) + 96 * (size_t)kSweepCta * capr;
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Row r of a 6x6 block (6 consecutive values) times 6 x entries, with
// vector shared-memory loads and two partial sums.
__device__ __forceinline__ double dot6(const double* a, const double* x) {
  const double2 a0 = reinterpret_cast<const double2*>(a)[0], a1 = reinterpret_cast<const double2*>(a)[1],
                a2 = reinterpret_cast<const double2*>(a)[2];
  const double2 x0 = reinterpret_cast<const double2*>(x)[0], x1 = reinterpret_cast<const double2*>(x)[1],
                x2 = reinterpret_cast<const double2*>(x)[2];
  double s0 = a0.x * x0.x, s1 = a0.y * x0.y;
  s0 = fma(a1.x, x1.x, s0);
  s1 = fma(a1.y, x1.y, s1);
  s0 = fma(a2.x, x2.x, s0);
  s1 = fma(a2.y, x2.y, s1);
  return s0 + s1;
}
__device__ __forceinline__ double dot6(const float* a, const double* x) {
  const float2 a0 = reinterpret_cast<const float2*>(a)[0], a1 = reinterpret_cast<const float2*>(a)[1],
               a2 = reinterpret_cast<const float2*>(a)[2];
  const double2 x0 = reinterpret_cast<const double2*>(x)[0], x1 = reinterpret_cast<const double2*>(x)[1],
                x2 = reinterpret_cast<const double2*>(x)[2];
  double s0 = (double)a0.x * x0.x, s1 = (double)a0.y * x0.y;
  s0 = fma((double)a1.x, x1.x, s0);
  s1 = fma((double)a1.y, x1.y, s1);
  s0 = fma((double)a2.x, x2.x, s0);
  s1 = fma((double)a2.y, x2.y, s1);
  return s0 + s1;
}

template <class VT, bool UPPER>
__global__ void __launch_bounds__(kSweepThreads) bsweep_tma(const ProbDev* __restrict__ P,
                                                           const int* __restrict__ live,
                                                           const double* __restrict__ rhs,
                                                           double* out, SweepCtl* ctl,
                                                           unsigned long long* bytes_ctr) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar[kStages];
  __shared__ uint64_t xbar[2];  // the partner's "chunk done" arrivals, alternating
  __shared__ int abort_flag;
  const int p = blockIdx.x / kSweepCta;
  const unsigned rank = cluster_rank(), partner = rank ^ 1u;
  if (live && !live[p]) return;  // the same for every CTA of the cluster
  if ((UPPER ? P[p].U.kind : P[p].L.kind) != TRI_LEVEL) return;  // solved by bsweep_df
  const bool split = (UPPER ? P[p].U.nsplit : P[p].L.nsplit) > 1;
  if (!split && rank != 0) return;  // one CTA solves the whole chunk; no cluster traffic
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  const int g = lane / 6, r = lane % 6;
  const ProbDev& d = P[p];
  const TriDesc T = UPPER ? d.U : d.L;
  // xbuf[h]: gathered x (capb x 6) then right-hand sides (capr x 6) of the
  // chunks with parity h
  double* xbuf = reinterpret_cast<double*>(smem + (size_t)kStages * T.stage);
  const size_t xstride = 6 * ((size_t)T.capb + T.capr);
  const int ringrows = kSweepCta * T.capr;
  double* ring = xbuf + 2 * xstride;  // 2 x ringrows x 6
  const unsigned pring = cluster_map(smem_u32(ring), partner);
  const unsigned pxbar = cluster_map(smem_u32(xbar), partner);
  const int64_t* offs = T.off + (size_t)rank * (T.nch + 1);  // this CTA's half chunks
  const unsigned long long wlim = g_wait_ns;
  const bool arrive = !(g_skip_meet && rank == 1);
  const double* rb = rhs + 6 * (size_t)d.off;
  double* ob = out + 6 * (size_t)d.off;
  if (tid == 0) {
    for (int s = 0; s < kStages; s++) mbar_init(&bar[s], 1);
    mbar_init(&xbar[0], 1);
    mbar_init(&xbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  if (split)
    cluster_barrier();  // both CTAs' barriers exist before any remote arrival
  else
    __syncthreads();
  // chunk byte ranges are read one issue ahead so tid 0 never waits on them
  long long lo = 0, hi = 0;
  const int producer = kSweepThreads - 32;  // lane 0 of the last warp issues every copy
  if (tid == producer) {
    lo = offs[0];
    hi = offs[1];
  }
  auto issue = [&](int c) {  // producer only; lo/hi hold chunk c's range
    uint64_t* b = &bar[c % kStages];
    mbar_expect_tx(b, (unsigned)(hi - lo));
    bulk_g2s(smem + (size_t)(c % kStages) * T.stage, T.stream + lo, (unsigned)(hi - lo), b);
    lo = hi;
    if (c + 2 <= T.nch) hi = offs[c + 2];
  };
  if (tid == producer)
    for (int c = 0; c < kStages - 1 && c < T.nch; c++) issue(c);
  int issued = min(kStages - 1, T.nch);
  // chunk 0 has no earlier rows: only its right-hand sides
  if (!mbar_wait(&bar[0], 0u, wlim)) abort_flag = 1;
  __syncthreads();
  // 6-double rows of x and of the right-hand side move as three 16-byte
  // pieces when both vectors are 16-byte aligned, else as six 8-byte ones
  const bool a16 = ((reinterpret_cast<uintptr_t>(rb) | reinterpret_cast<uintptr_t>(ob)) & 15) == 0;
  // pieces per row as a compile-time constant (3 or 6): the index splits
  // below then compile to multiplications instead of divisions
  auto with_pw = [&](auto fn) {
    if (a16)
      fn(std::integral_constant<int, 3>{});
    else
      fn(std::integral_constant<int, 6>{});
  };
  auto copy_piece = [](auto pwc, double* dst, const double* src, int piece) {
    if (decltype(pwc)::value == 3)
      cp_async16(dst + 2 * piece, src + 2 * piece);
    else
      cp_async8(dst + piece, src + piece);
  };
  if (!abort_flag) {
    const int nr0 = reinterpret_cast<const int4*>(smem)->x;
    const int4* ri0 = reinterpret_cast<const int4*>(smem + 32);
    with_pw([&](auto pwc) {
      constexpr int pw = decltype(pwc)::value;
      for (int t = tid; t < pw * nr0; t += kSweepThreads)
        copy_piece(pwc, xbuf + 6 * T.capb + 6 * (t / pw), rb + 6 * (size_t)ri0[t / pw].x, t % pw);
    });
    cp_async_commit();
  }
  int c = 0;
  for (; c < T.nch; c++) {
    const int s = c % kStages;
    if (c > 0 && !mbar_wait(&bar[s], (unsigned)((c / kStages) & 1), wlim)) abort_flag = 1;
    cp_async_wait_all();  // this thread's copies for chunk c have landed
    __syncthreads();      // this CTA's half of chunk c-1 solved; its stage and xbuf[(c+1)&1] are free
    if (c > 0 && split) {
      // meet the partner: its half of chunk c-1 (global x, ring rows in
      // this CTA) is complete and visible once its arrival is seen
      if (tid == 0) {
        const unsigned slot = (unsigned)((c - 1) & 1);
        if (arrive) mbar_arrive_remote(pxbar + 8u * slot);
        if (!mbar_wait_cluster(&xbar[slot], (unsigned)(((c - 1) >> 1) & 1), wlim)) abort_flag = 1;
      }
      __syncthreads();
    }
    if (abort_flag) break;
    const unsigned char* st = smem + (size_t)s * T.stage;
    const int4 h0 = reinterpret_cast<const int4*>(st)[0];
    const int4 h1 = reinterpret_cast<const int4*>(st)[1];
    const int nr = h0.x, nb = h0.y, nn = h0.z, nf1 = h1.x, nr1 = h1.y;
    const int4* ri = reinterpret_cast<const int4*>(st + 32);
    const int2* nearl = reinterpret_cast<const int2*>(ri + nr);
    const int2* far1 = nearl + nn;
    const int32_t* rows1 = reinterpret_cast<const int32_t*>(far1 + nf1);
    const size_t voff = (32 + 16 * (size_t)nr + 8 * (size_t)(nn + nf1) + 4 * (size_t)nr1 + 15) &
                        ~(size_t)15;
    const VT* sv = reinterpret_cast<const VT*>(st + voff);
    double* xs = xbuf + xstride * (c & 1);
    double* rs = xs + 6 * (size_t)T.capb;
    // asynchronous copies for chunk c+1 (waited for one chunk later): far x
    // entries (rows solved by chunks <= c-1, complete at the barrier above)
    // and right-hand sides, into the gather area chunk c-1 used. When the
    // chunk has fewer rows than the CTA has warps, the warps without a row
    // issue them while the others solve theirs; otherwise every thread
    // issues them first.
    auto issue_next = [&](int t0, int stride) {
      double* xn = xbuf + xstride * ((c + 1) & 1);
      with_pw([&](auto pwc) {
        constexpr int pw = decltype(pwc)::value;
        for (int t = t0; t < pw * (nf1 + nr1); t += stride) {
          if (t < pw * nf1) {
            const int2 f = far1[t / pw];
            copy_piece(pwc, xn + 6 * f.x, ob + 6 * (size_t)f.y, t % pw);
          } else {
            const int t2 = t - pw * nf1;
            copy_piece(pwc, xn + 6 * T.capb + 6 * (t2 / pw), rb + 6 * (size_t)rows1[t2 / pw],
                       t2 % pw);
          }
        }
      });
    };
    const bool idle_issue = nr < nw;
    if (!idle_issue) issue_next(tid, kSweepThreads);
    // near entries: results of chunk c-1 from the ring
    {
      const double2* rp =
          reinterpret_cast<const double2*>(ring + 6 * (size_t)ringrows * ((c + 1) & 1));
      double2* xs2 = reinterpret_cast<double2*>(xs);
      for (int t = tid; t < 3 * nn; t += kSweepThreads) {
        const int2 q = nearl[t / 3];
        xs2[3 * q.x + t % 3] = rp[3 * q.y + t % 3];
      }
    }
    __syncthreads();
    // the producer warp (the last) refills the stage chunk c-1 used, then
    // solves rows like the others (it is given a row only when a chunk has
    // as many rows as the CTA has warps)
    if (issued < T.nch) {
      if (tid == producer) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(issued);
      }
      issued++;
    }
    if (idle_issue && warp >= nr) issue_next(tid - 32 * nr, 32 * (nw - nr));
    cp_async_commit();
    double* wp = ring + 6 * (size_t)ringrows * (c & 1);
    const unsigned pwp = pring + 8u * 6u * (unsigned)ringrows * (unsigned)(c & 1);
    for (int k = warp; k < nr; k += nw) {
      const int4 row = ri[k];
      const int i = row.x, rbeg = row.y, rcnt = row.z, gk = row.w;
      const int first = UPPER ? 1 : 0;  // U rows start with U_ii^{-1}
      // row `lane` of U_ii^{-1} (lanes 0..5), loaded while the products run
      double di[6];
      if (UPPER) {
        const VT* Di = sv + (size_t)rbeg * 36 + 6 * (lane < 6 ? lane : 0);
#pragma unroll
        for (int cc = 0; cc < 6; cc++) di[cc] = (double)Di[cc];
      }
      double acc = 0.0;
      if (g < 4) {
        double acc1 = 0.0;
        int j = first + g;
        for (; j + 4 < rcnt; j += 8) {
          acc += dot6(sv + (size_t)(rbeg + j) * 36 + 6 * r, xs + 6 * (rbeg + j));
          acc1 += dot6(sv + (size_t)(rbeg + j + 4) * 36 + 6 * r, xs + 6 * (rbeg + j + 4));
        }
        if (j < rcnt) acc += dot6(sv + (size_t)(rbeg + j) * 36 + 6 * r, xs + 6 * (rbeg + j));
        acc += acc1;
      }
      acc += __shfl_down_sync(0xffffffffu, acc, 12);
      acc += __shfl_down_sync(0xffffffffu, acc, 6);
      const double t = (lane < 6 ? rs[6 * k + lane] : 0.0) - acc;
      double v = t;
      if (UPPER) {
        double tc[6];
#pragma unroll
        for (int cc = 0; cc < 6; cc++) tc[cc] = __shfl_sync(0xffffffffu, t, cc);
        v = fma(di[4], tc[4], fma(di[2], tc[2], di[0] * tc[0])) +
            fma(di[5], tc[5], fma(di[3], tc[3], di[1] * tc[1]));
      }
      if (lane < 6) {
        ob[6 * (size_t)i + lane] = v;
        wp[6 * gk + lane] = v;
        if (split) cluster_store(pwp + 8u * (unsigned)(6 * gk + lane), v);
      }
    }
  }
  cp_async_wait_all();  // no copy may land after the kernel ends
  if (!abort_flag && tid == 0 && rank == 0 && bytes_ctr)
    atomicAdd(bytes_ctr, (unsigned long long)T.abytes);
  if (abort_flag && tid == producer) {
    atomicOr(&ctl->status, ST_TIMEOUT);
    // chunks c .. issued-1 may still be in flight: let them land (bounded)
    for (int q = c; q < issued; q++)
      mbar_wait(&bar[q % kStages], (unsigned)((q / kStages) & 1), kWaitNs);
  }
  // neither CTA leaves while the other may still write into its shared
  // memory; every path of both CTAs of a split problem reaches this point
  if (split) cluster_barrier();
}

// One sweep of a batch: a cluster of kSweepCta CTAs per problem.
template <class VT, bool UPPER>
static cudaError_t launch_sweep(int np, size_t smem, cudaStream_t st, const ProbDev* desc,
                                const int* live, const double* rhs, double* out, SweepCtl* ctl,
                                unsigned long long* ctr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(np * kSweepCta));
  cfg.blockDim = dim3(kSweepThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kSweepCta;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ::gf::count_launch();
  return cudaLaunchKernelEx(&cfg, bsweep_tma<VT, UPPER>, desc, live, rhs, out, ctl, ctr);
}

// ------------------------------------------------------ dataflow sweeps
// One CTA per problem walks one triangle row by row in level order without
// block barriers: compute warp w solves the rows of every chunk whose
// chunk-local index is w mod kDfWarps, and a row waits only for the rows it
// multiplies. A solved row's x entries go to global memory (the result) and
// to a shared-memory ring of the latest `ring` positions; every ring slot
// has an mbarrier whose phase k completes when position slot + k ring is
// written, so a consumer waits (bounded, suspended in hardware rather than
// spinning) on the phase of exactly the position it reads, with release /
// acquire ordering at CTA scope. A row's blocks are ordered by the position
// they depend on, so the lane groups multiply the long-solved rows while the
// latest ones finish.
// Flow control keeps the phases unambiguous: before overwriting a slot with
// position p a warp waits until every warp has moved past p - ring + maxdist
// (so all readers of the slot's previous position are done), using the
// positions the warps publish in wpos[]. Every position below min(wpos) is
// solved, so the warp holding that minimum can always proceed: nothing
// waits in a cycle.
// The factor stream arrives through kDfStages shared-memory stages filled by
// 1D bulk copies, which a producer warp issues as the compute warps release
// stages (full / empty mbarriers), and a gather warp copies each chunk's
// right-hand sides into the chunk's stage with cp.async (completion counted
// on a third mbarrier), so no row waits on a global load. The compute warps
// store nothing to global memory: a writer warp copies every solved row from
// the ring to the result vector in position order (it waits on the same
// slot barriers and takes part in the flow control), so the release
// operations of the compute warps order shared-memory writes only and never
// wait for global stores to complete. All waits are bounded; on a timeout
// the CTA records ST_TIMEOUT and ends after its copies in flight have landed.
constexpr int kDfThreads = 576;
constexpr int kDfWarps = kDfThreads / 32 - 3;  // compute warps
constexpr int kDfProducer = kDfWarps;          // issues the stage copies
constexpr int kDfGather = kDfWarps + 1;        // gathers the right-hand sides
constexpr int kDfWriter = kDfWarps + 2;        // writes results to global memory
constexpr int kDfStages = 4;
constexpr int kDfRows = 64;                    // rows per chunk at most
constexpr int kDfWriteBatch = 64;              // positions the writer reports at once

// dynamic shared memory of a dataflow sweep: the stages, their right-hand
// sides, the ring's x entries (6 doubles), row indices and mbarriers
__host__ __device__ inline size_t df_smem_bytes(int stage, int ring) {
  return kDfStages * ((size_t)stage + 48 * (size_t)kDfRows) + (size_t)ring * (48 + 8 + 4);
}
__device__ __forceinline__ void mbar_arrive_local(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ int ld_acquire_s32(const int* p) {
  int v;
  asm volatile("ld.acquire.cta.shared.b32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_s32(int* p, int v) {
  asm volatile("st.release.cta.shared.b32 [%0], %1;" ::"r"(smem_u32(p)), "r"(v) : "memory");
}
// arrive on `bar` once all of this thread's earlier cp.async copies have
// landed (the arrival is not counted in advance)
__device__ __forceinline__ void cp_async_arrive(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void cp_async8_df(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}

template <class VT, bool UPPER>
__global__ void __launch_bounds__(kDfThreads) bsweep_df(const ProbDev* __restrict__ P,
                                                       const int* __restrict__ live,
                                                       const double* __restrict__ rhs,
                                                       double* out, SweepCtl* ctl,
                                                       unsigned long long* bytes_ctr) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t full[kDfStages], empty[kDfStages], rhsb[kDfStages];
  // every position below wpos[w] that compute warp w owns is solved; every
  // position below wpos[kDfWarps] has been written out by the writer warp
  __shared__ int wpos[kDfWarps + 1];
  __shared__ volatile int abort_flag;
  const int p = blockIdx.x;
  if (live && !live[p]) return;
  const ProbDev& d = P[p];
  const TriDesc T = UPPER ? d.U : d.L;
  if (T.kind != TRI_DATAFLOW) return;  // solved by bsweep_tma
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int rmask = T.ring - 1, rlog = __ffs(T.ring) - 1;
  // layout: stages | right-hand sides of the stages | ring x | ring mbarriers
  double* srhs = reinterpret_cast<double*>(smem + (size_t)kDfStages * T.stage);
  double* rx = srhs + (size_t)kDfStages * 6 * kDfRows;
  uint64_t* rbar = reinterpret_cast<uint64_t*>(rx + 6 * (size_t)T.ring);
  int* ridx = reinterpret_cast<int*>(rbar + T.ring);  // row index of each slot's position
  for (int t = tid; t < T.ring; t += kDfThreads) mbar_init(&rbar[t], 1);
  if (tid <= kDfWarps) wpos[tid] = 0;
  if (tid == 0) {
    for (int s = 0; s < kDfStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kDfWarps);
      mbar_init(&rhsb[s], 32);
    }
    abort_flag = 0;
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();
  const unsigned long long wlim = g_wait_ns;
  // bounded wait that also gives up once another warp has aborted
  // Waiting warps sleep in the barrier test instead of spinning, so the warps
  // that have work get the issue slots; the timer is read only once the
  // first test fails.
  auto wait_bar = [&](uint64_t* bar, unsigned par) {
    if (mbar_try_wait(bar, par)) return true;
    const unsigned long long t0 = gtimer();
    unsigned n = 0;
    while (!mbar_try_wait_sleep(bar, par, 2000u))
      if ((++n & 15u) == 0u && (abort_flag || gtimer() - t0 > wlim)) return false;
    return true;
  };
  auto fail = [&]() {
    if (!abort_flag) {
      abort_flag = 1;
      atomicOr(&ctl->status, ST_TIMEOUT);
    }
  };
  if (warp == kDfProducer) {
    if (lane == 0) {
      int issued = 0;
      for (int c = 0; c < T.nch; c++) {
        const int s = c % kDfStages;
        // the compute warps have released chunk c - kDfStages
        if (c >= kDfStages && !wait_bar(&empty[s], (unsigned)(((c / kDfStages) - 1) & 1))) {
          fail();
          break;
        }
        const long long lo = T.off[c], hi = T.off[c + 1];
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&full[s], (unsigned)(hi - lo));
        bulk_g2s(smem + (size_t)s * T.stage, T.stream + lo, (unsigned)(hi - lo), &full[s]);
        issued = c + 1;
      }
      // no copy may land after the CTA ends: the last stages' copies (all
      // earlier ones were consumed before their stages were reused)
      for (int q = max(0, issued - kDfStages); q < issued; q++)
        mbar_wait(&full[q % kDfStages], (unsigned)((q / kDfStages) & 1), kWaitNs);
    }
    return;
  }
  if (warp == kDfGather) {
    // the right-hand sides of each chunk's rows into the chunk's stage, as
    // soon as the chunk's records have landed
    const double* rb = rhs + 6 * (size_t)d.off;
    for (int c = 0; c < T.nch; c++) {
      const int s = c % kDfStages;
      if (!wait_bar(&full[s], (unsigned)((c / kDfStages) & 1))) {
        if (lane == 0) fail();
        break;
      }
      const unsigned char* st = smem + (size_t)s * T.stage;
      const int nr = reinterpret_cast<const int4*>(st)->x;
      const int4* rec = reinterpret_cast<const int4*>(st + 16);
      double* dst = srhs + (size_t)s * 6 * kDfRows;
      for (int t = lane; t < 6 * nr; t += 32)
        cp_async8_df(dst + t, rb + 6 * (size_t)rec[t / 6].x + t % 6);
      cp_async_arrive(&rhsb[s]);
    }
    cp_async_wait_all();  // no copy may land after the CTA ends
    return;
  }
  double* ob = out + 6 * (size_t)d.off;
  const int n = d.n;
  if (warp == kDfWriter) {
    // lane group g5 (5 groups of 6 lanes) writes position q0 + g5
    const int g5 = lane / 6, r6 = lane % 6;
    bool okw = true;
    for (int q0 = 0; q0 < n && okw; q0 += 5) {
      const int q = q0 + g5;
      if (lane < 30 && q < n) {
        if (!wait_bar(&rbar[q & rmask], (unsigned)((q >> rlog) & 1))) {
          fail();
          okw = false;
        } else {
          const int slot = q & rmask;
          ob[6 * (size_t)ridx[slot] + r6] = rx[6 * slot + r6];
        }
      }
      if (__any_sync(0xffffffffu, !okw)) break;
      const int next = q0 + 5;
      // report progress every kDfWriteBatch positions; the release makes the
      // slot reads above complete before any warp may overwrite the slots
      if (next % kDfWriteBatch == 0 || next >= n) {
        __syncwarp();
        if (lane == 0) st_release_s32(&wpos[kDfWarps], next >= n ? 0x7fffffff : next);
      }
    }
    return;
  }
  const int g = lane / 6, r = lane % 6;
  // failure-injection knob for tests: warp 0 never publishes its rows
  const bool publish = !(g_skip_meet && warp == 0);
  int seen_min = 0;  // a lower bound of min(wpos)
  bool ok = true;
  for (int c = 0; c < T.nch && ok; c++) {
    const int s = c % kDfStages;
    const unsigned par = (unsigned)((c / kDfStages) & 1);
    if (!wait_bar(&full[s], par) || !wait_bar(&rhsb[s], par)) {
      fail();
      ok = false;
    }
    if (__any_sync(0xffffffffu, !ok)) break;
    const unsigned char* st = smem + (size_t)s * T.stage;
    const int4 h = *reinterpret_cast<const int4*>(st);
    const int nr = h.x, nb = h.y, p0 = h.z;
    const int4* rec = reinterpret_cast<const int4*>(st + 16);
    const int* dep = reinterpret_cast<const int*>(rec + nr);
    const VT* val = reinterpret_cast<const VT*>(
        st + ((16 + 16 * (size_t)nr + 4 * (size_t)nb + 15) & ~(size_t)15));
    const double* crhs = srhs + (size_t)s * 6 * kDfRows;
    for (int k = warp; k < nr; k += kDfWarps) {
      const int pos = p0 + k;
      if (lane == 0) st_release_s32(&wpos[warp], pos);
      const int4 row = rec[k];
      const int i = row.x, b0 = row.y, cnt = row.z;
      const double rv = lane < 6 ? crhs[6 * k + lane] : 0.0;
      double acc = 0.0;
      if (g < 4) {
        for (int j = (UPPER ? 1 : 0) + g; j < cnt; j += 4) {
          const int q = dep[b0 + j];
          if (!wait_bar(&rbar[q & rmask], (unsigned)((q >> rlog) & 1))) {
            fail();
            ok = false;
            break;
          }
          acc += dot6(val + (size_t)(b0 + j) * 36 + 6 * r, rx + 6 * (size_t)(q & rmask));
        }
      }
      if (__any_sync(0xffffffffu, !ok)) {
        ok = false;
        break;
      }
      acc += __shfl_down_sync(0xffffffffu, acc, 12);
      acc += __shfl_down_sync(0xffffffffu, acc, 6);
      const double t = rv - acc;
      double v = t;
      if (UPPER) {
        const VT* Di = val + (size_t)b0 * 36;
        v = 0.0;
#pragma unroll
        for (int cc = 0; cc < 6; cc++) {
          const double tc = __shfl_sync(0xffffffffu, t, cc);
          if (lane < 6) v = fma((double)Di[6 * lane + cc], tc, v);
        }
      }
      // flow control: the slot's previous position (pos - ring) is read
      // only by rows at positions <= pos - ring + maxdist
      const int slot = pos & rmask;
      const int lim = pos - T.ring + T.maxdist;
      if (lim >= seen_min) {
        unsigned long long t0 = 0;
        for (int it = 0;; it++) {
          int m = lane <= kDfWarps ? ld_acquire_s32(&wpos[lane]) : 0x7fffffff;
          m = __reduce_min_sync(0xffffffffu, m);
          seen_min = m;
          if (m > lim) break;
          if (it == 0) t0 = gtimer();
          const int stop =
              __shfl_sync(0xffffffffu, lane == 0 && (abort_flag || gtimer() - t0 > wlim), 0);
          if (stop) {
            if (lane == 0) fail();
            ok = false;
            break;
          }
        }
        if (!ok) break;
      }
      if (lane < 6) rx[6 * slot + lane] = v;
      if (lane == 0) ridx[slot] = i;
      __syncwarp();
      if (lane == 0 && publish) mbar_arrive_local(&rbar[slot]);
    }
    if (!ok) break;
    __syncwarp();
    if (lane == 0) {
      mbar_arrive_local(&empty[s]);
      st_release_s32(&wpos[warp], p0 + nr + warp);  // its first position in the next chunk
    }
  }
  if (lane == 0) st_release_s32(&wpos[warp], 0x7fffffff);
  if (ok && tid == 0 && bytes_ctr) atomicAdd(bytes_ctr, (unsigned long long)T.abytes);
}

// Factor values into a chunk stream: block slot q of the triangle takes
// the 6x6 block src[map[q]] (zero for padding, map < 0) at element offset
// vpos[q] of the stream viewed as VT.
template <class VT>
__global__ void repack_kernel(size_t nslots, const int32_t* __restrict__ map,
                              const int64_t* __restrict__ vpos, const double* __restrict__ src,
                              VT* __restrict__ dst) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nslots * 36) return;
  const size_t q = t / 36, e = t % 36;
  const int m = map[q];
  dst[vpos[q] + e] = m >= 0 ? (VT)src[36 * (size_t)m + e] : (VT)0;
}

// ------------------------------------------------- segmented vector kernels
struct Chunks {
  int n;                   // number of chunks
  const int32_t* prob;     // chunk -> problem
  const int64_t* lo;       // chunk start (doubles, batch space)
  const int64_t* hi;       // chunk end
  const int32_t* pstart;   // problem -> first chunk, [np + 1]
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

// partial[i * C.n + c] = V_i . w over chunk c, i = 0..jj, for running problems.
// w stays in registers; eight basis vectors at a time are read with all
// their loads in flight and reduced together (the same summation order as
// one vector at a time: per thread in element order, then the warp tree,
// then the warps in order).
constexpr int kDotGroup = 8;
__global__ void __launch_bounds__(kRedThreads) seg_dots(const double* __restrict__ V,
                                                        const double* __restrict__ w, size_t N,
                                                        int jj, Chunks C,
                                                        const int* __restrict__ run,
                                                        double* partial) {
  constexpr int E = kChunk / kRedThreads;  // elements per thread
  __shared__ double sh[kDotGroup][kRedThreads / 32];
  const int c = blockIdx.x;
  if (!run[C.prob[c]]) return;
  const int64_t lo = C.lo[c], hi = C.hi[c];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double wr[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int64_t t = lo + threadIdx.x + (int64_t)e * kRedThreads;
    wr[e] = t < hi ? w[t] : 0.0;
  }
  for (int i0 = 0; i0 <= jj; i0 += kDotGroup) {
    double acc[kDotGroup];
#pragma unroll
    for (int q = 0; q < kDotGroup; q++) {
      acc[q] = 0.0;
      if (i0 + q <= jj) {
        const double* v = V + (size_t)(i0 + q) * N;
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int64_t t = lo + threadIdx.x + (int64_t)e * kRedThreads;
          if (t < hi) acc[q] = fma(v[t], wr[e], acc[q]);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kDotGroup; q++)
      for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], o);
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < kDotGroup; q++) sh[q][warp] = acc[q];
    __syncthreads();
    if (threadIdx.x < kDotGroup && i0 + (int)threadIdx.x <= jj) {
      double s = 0.0;
      for (int k = 0; k < kRedThreads / 32; k++) s += sh[threadIdx.x][k];
      partial[(size_t)(i0 + threadIdx.x) * C.n + c] = s;
    }
    __syncthreads();
  }
}

struct GmArrays {
  double* H;       // np * (m+1) * m
  double* g;       // np * (m+1)
  double* cs;      // np * m
  double* ss;      // np * m
  double* y;       // np * m
  double* h;       // np * (m+1)
  double* hn;      // np
  double* target;  // np
  int* jcnt;       // np
  int* run;        // np
  int* live;       // np
};

// h_p[i] = sum over p's chunks; H_p[i][jj] (+)= h_p[i]
__global__ void seg_reduce_dots(const double* partial, Chunks C, int jj, int m, GmArrays G,
                                int acc) {
  const int p = blockIdx.x;
  if (!G.run[p]) return;
  for (int i = threadIdx.x; i <= jj; i += blockDim.x) {
    double s = 0.0;
    for (int c = C.pstart[p]; c < C.pstart[p + 1]; c++) s += partial[(size_t)i * C.n + c];
    G.h[(size_t)p * (m + 1) + i] = s;
    double* Hij = &G.H[(size_t)p * (m + 1) * m + (size_t)i * m + jj];
    *Hij = acc ? *Hij + s : s;
  }
}
// w -= sum_{i<=jj} h_p[i] V_i over chunk c; optional per-chunk |w|^2
__global__ void seg_update(const double* __restrict__ V, double* __restrict__ w, size_t N,
                           int jj, int m, Chunks C, GmArrays G, double* pnorm) {
  __shared__ double sh[32];
  __shared__ double hs[1024];
  const int c = blockIdx.x;
  const int p = C.prob[c];
  if (!G.run[p]) return;
  for (int i = threadIdx.x; i <= jj; i += blockDim.x) hs[i] = G.h[(size_t)p * (m + 1) + i];
  __syncthreads();
  const int64_t lo = C.lo[c], hi = C.hi[c];
  double acc = 0.0;
  for (int64_t t = lo + threadIdx.x; t < hi; t += blockDim.x) {
    double s = w[t];
#pragma unroll 8
    for (int i = 0; i <= jj; i++) s = fma(-hs[i], V[(size_t)i * N + t], s);
    w[t] = s;
    acc = fma(s, s, acc);
  }
  if (pnorm) {
    const double b = block_sum(acc, sh);
    if (threadIdx.x == 0) pnorm[c] = b;
  }
}
// per-chunk sum of squares over problems with mask[p] (all when mask is null)
__global__ void seg_sumsq(const double* __restrict__ v, Chunks C, const int* __restrict__ mask,
                          double* pnorm) {
  __shared__ double sh[32];
  const int c = blockIdx.x;
  if (mask && !mask[C.prob[c]]) return;
  double acc = 0.0;
  for (int64_t t = C.lo[c] + threadIdx.x; t < C.hi[c]; t += blockDim.x)
    acc = fma(v[t], v[t], acc);
  const double b = block_sum(acc, sh);
  if (threadIdx.x == 0) pnorm[c] = b;
}
__global__ void seg_norm_out(const double* pnorm, Chunks C, int np, const int* mask,
                             double* out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  if (mask && !mask[p]) return;
  double s = 0.0;
  for (int c = C.pstart[p]; c < C.pstart[p + 1]; c++) s += pnorm[c];
  out[p] = sqrt(s);
}
__global__ void seg_norm_finish(const double* pnorm, Chunks C, int np, int jj, int m,
                                GmArrays G) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np || !G.run[p]) return;
  double s = 0.0;
  for (int c = C.pstart[p]; c < C.pstart[p + 1]; c++) s += pnorm[c];
  G.hn[p] = sqrt(s);
  G.H[(size_t)p * (m + 1) * m + (size_t)(jj + 1) * m + jj] = G.hn[p];
}
__global__ void seg_scale(const double* __restrict__ src, double* __restrict__ dst, Chunks C,
                          const int* __restrict__ run, const double* __restrict__ hn) {
  const int c = blockIdx.x;
  const int p = C.prob[c];
  if (!run[p]) return;
  const double inv = hn[p] > 0.0 ? 1.0 / hn[p] : 0.0;
  for (int64_t t = C.lo[c] + threadIdx.x; t < C.hi[c]; t += blockDim.x) dst[t] = src[t] * inv;
}
// Givens update of column jj (examples/iterative/gmres.cu:672-699) per problem
__global__ void bgivens(int np, int jj, int m, int step_limit, GmArrays G) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np || !G.run[p]) return;
  double* H = G.H + (size_t)p * (m + 1) * m;
  double* g = G.g + (size_t)p * (m + 1);
  double* cs = G.cs + (size_t)p * m;
  double* ss = G.ss + (size_t)p * m;
  for (int i = 0; i < jj; i++) {
    const double a = H[(size_t)i * m + jj], c = H[(size_t)(i + 1) * m + jj];
    H[(size_t)i * m + jj] = cs[i] * a + ss[i] * c;
    H[(size_t)(i + 1) * m + jj] = -ss[i] * a + cs[i] * c;
  }
  const double a = H[(size_t)jj * m + jj], c = H[(size_t)(jj + 1) * m + jj];
  const double hyp = sqrt(a * a + c * c);
  cs[jj] = hyp > 0.0 ? a / hyp : 1.0;
  ss[jj] = hyp > 0.0 ? c / hyp : 0.0;
  H[(size_t)jj * m + jj] = cs[jj] * a + ss[jj] * c;
  H[(size_t)(jj + 1) * m + jj] = 0.0;
  g[jj + 1] = -ss[jj] * g[jj];
  g[jj] = cs[jj] * g[jj];
  G.jcnt[p] = jj + 1;
  if (fabs(g[jj + 1]) <= G.target[p] || G.hn[p] == 0.0 || !isfinite(g[jj + 1]) ||
      jj + 1 >= step_limit)
    G.run[p] = 0;
}
__global__ void bbacksolve(int np, int m, GmArrays G) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np || !G.live[p]) return;
  const int j = G.jcnt[p];
  const double* H = G.H + (size_t)p * (m + 1) * m;
  const double* g = G.g + (size_t)p * (m + 1);
  double* y = G.y + (size_t)p * m;
  for (int i = j - 1; i >= 0; i--) {
    double s = g[i];
    for (int k = i + 1; k < j; k++) s -= H[(size_t)i * m + k] * y[k];
    y[i] = s / H[(size_t)i * m + i];
  }
}
// out = sum_{i < jcnt_p} y_p[i] V_i over live problems (zero otherwise)
__global__ void seg_combine(const double* __restrict__ V, size_t N, int m, Chunks C, GmArrays G,
                            double* __restrict__ out) {
  __shared__ double ys[1024];
  const int c = blockIdx.x;
  const int p = C.prob[c];
  const int j = G.live[p] ? G.jcnt[p] : 0;
  for (int i = threadIdx.x; i < j; i += blockDim.x) ys[i] = G.y[(size_t)p * m + i];
  __syncthreads();
  for (int64_t t = C.lo[c] + threadIdx.x; t < C.hi[c]; t += blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < j; i++) s = fma(ys[i], V[(size_t)i * N + t], s);
    out[t] = s;
  }
}
// cycle start: beta_p = ||src_p||, g_p = (beta, 0, ...), run_p = live_p
// tfac (may be null): target = tfac[p] * beta, the Arnoldi residual
// reduction this cycle must reach.
__global__ void bcycle_init(const double* pnorm, Chunks C, int np, int m, GmArrays G,
                            const double* tfac) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  double s = 0.0;
  if (G.live[p])
    for (int c = C.pstart[p]; c < C.pstart[p + 1]; c++) s += pnorm[c];
  const double beta = sqrt(s);
  G.hn[p] = beta;
  if (tfac && G.live[p]) G.target[p] = tfac[p] * beta;
  G.jcnt[p] = 0;
  G.run[p] = (G.live[p] && beta > 0.0) ? 1 : 0;
  double* g = G.g + (size_t)p * (m + 1);
  g[0] = beta;
  for (int i = 1; i <= m; i++) g[i] = 0.0;
}
// y += a * x over problems with mask[p] (all when mask is null)
__global__ void seg_axpy(double a, const double* __restrict__ x, double* __restrict__ y,
                         Chunks C, const int* __restrict__ mask) {
  const int c = blockIdx.x;
  if (mask && !mask[C.prob[c]]) return;
  for (int64_t t = C.lo[c] + threadIdx.x; t < C.hi[c]; t += blockDim.x) y[t] += a * x[t];
}
__global__ void seg_copy(const double* __restrict__ x, double* __restrict__ y, Chunks C,
                         const int* __restrict__ mask) {
  const int c = blockIdx.x;
  if (mask && !mask[C.prob[c]]) return;
  for (int64_t t = C.lo[c] + threadIdx.x; t < C.hi[c]; t += blockDim.x) y[t] = x[t];
}
__global__ void set_target(int np, const double* norms, double rtol, GmArrays G) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < np) G.target[p] = rtol * norms[p];
}
// natural <-> batch-space permutation, one problem per blockIdx.y
struct PermEntry {
  const int32_t* perm;
  int n, off;
  const double* in;
  double* out;
};
__global__ void bpermute(const PermEntry* E, int dir) {
  const PermEntry e = E[blockIdx.y];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 6 * e.n; t += gridDim.x * blockDim.x) {
    const int i = t / 6, k = t % 6;
    if (dir == 0)
      e.out[6 * ((size_t)e.off + e.perm[i]) + k] = e.in[t];
    else
      e.out[t] = e.in[6 * ((size_t)e.off + e.perm[i]) + k];
  }
}

}  // namespace gf

using namespace gf;

// ---------------------------------------------------------------- handles
struct gf_precond {
  gf_assembler* a = nullptr;
  int fill = 0, prec = GF_PREC_FP64;
  Pattern pat;
  int nlevL = 0, nlevU = 0;
  std::vector<int32_t> lvL, lvU;
  DevBuf<int32_t> d_rowp, d_cols, d_diag, d_amap;
  DevBuf<int32_t> d_levLptr, d_levLrows;  // factorization order
  DevBuf<int32_t> d_done;                  // per row: epoch of the factorization that finished it
  DevBuf<int32_t> d_ord;                   // per row: the order of its factorization steps
  long long fwork = 0;                     // block updates of one factorization
  int sym_gpu = 0;                         // ILU(k) pattern computed on the GPU
  double sym_ms = 0.0, setup_ms = 0.0;     // host wall time of the pattern / of the whole setup
  DevBuf<double> d_lu;
  struct Tri {
    int nch = 0, stage = 0, capb = 0, capr = 0, nsplit = 1;
    int kind = TRI_LEVEL, ring = 0, maxdist = 0;
    size_t nslots = 0;
    long long abytes = 0;
    DevBuf<int64_t> off, vpos;
    DevBuf<int32_t> map;
    DevBuf<unsigned char> stream;
  } tri[2];  // 0 = L, 1 = U
  gf_batch* self = nullptr;  // batch of one, built on first use
};

namespace gf {
// Chunk stream of one triangle (layout described at TriDesc).
static cudaError_t build_tri(gf_precond* p, const std::vector<int32_t>& diag, bool upper) {
  const Pattern& P = p->pat;
  const int n = P.n;
  const std::vector<int32_t>& lv = upper ? p->lvU : p->lvL;
  const int nlev = upper ? p->nlevU : p->nlevL;
  const size_t vs = p->prec == GF_PREC_FP32 ? 4 : 8;
  auto cnt = [&](int i) { return upper ? P.rowp[i + 1] - diag[i] : diag[i] - P.rowp[i]; };
  std::vector<int32_t> ptr(nlev + 1, 0), rows(n);
  for (int i = 0; i < n; i++) ptr[lv[i] + 1]++;
  for (int l = 0; l < nlev; l++) ptr[l + 1] += ptr[l];
  {
    std::vector<int32_t> f(ptr.begin(), ptr.end() - 1);
    for (int i = 0; i < n; i++) rows[f[lv[i]]++] = i;
  }
  int maxc = 0;
  long long real = 0;
  for (int i = 0; i < n; i++) {
    maxc = std::max(maxc, cnt(i));
    real += cnt(i);
  }
  const int mc4 = (maxc + 3) & ~3;
  const int base = p->prec == GF_PREC_FP32 ? 416 : 208;
  const int capr = 128;
  // One CTA or the two CTAs of the problem's cluster per chunk, whichever
  // the chunk model of B200 clock64 traces makes cheaper: a chunk costs
  // ~1,000 cycles of copies and barriers plus ~1,900 cycles per round of
  // rows over the 16 warps of a CTA (a row's latency), and splitting it
  // adds ~1,450 cycles for the two CTAs' meeting. Splitting pays when levels
  // have more rows than one CTA's warps or more blocks than its stage.
  auto model = [&](int ns) {
    const int cb = ns > 1 ? ns * (std::max(base, ((3 * mc4 + 1) / 2 + 3) & ~3) - mc4)
                          : std::max(base, mc4);
    const int cr = ns * capr, warps = kSweepThreads / 32;
    double cyc = 0.0;
    int cur = 0, nr = 0;
    auto close = [&]() {
      const int per_cta = (nr + ns - 1) / ns;
      cyc += 1000.0 + (ns > 1 ? 1450.0 : 0.0) + 1900.0 * ((per_cta + warps - 1) / warps);
      cur = nr = 0;
    };
    for (int l = 0; l < nlev; l++) {
      for (int k = ptr[l]; k < ptr[l + 1]; k++) {
        const int c = cnt(rows[k]);
        if (nr > 0 && (cur + c > cb || nr == cr)) close();
        cur += c;
        nr++;
      }
      if (nr > 0) close();
    }
    return cyc;
  };
  const int nsplit = model(kSweepCta) < model(1) ? kSweepCta : 1;
  // per CTA: blocks of one half chunk. Split chunks are bounded so that
  // giving each row to the lighter half leaves every half within capb (a
  // half exceeds the mean by at most half a row) and a longest row fits.
  const int capb = nsplit > 1 ? std::max(base, ((3 * mc4 + 1) / 2 + 3) & ~3) : std::max(base, mc4);
  const int gcapb = nsplit > 1 ? nsplit * (capb - mc4) : capb, gcapr = nsplit * capr;
  // pass 1: chunk boundaries (row ranges of `rows`); a chunk never spans two levels
  std::vector<int32_t> ck{0};
  {
    int cur = 0, nr = 0;
    for (int l = 0; l < nlev; l++) {
      for (int k = ptr[l]; k < ptr[l + 1]; k++) {
        const int c = cnt(rows[k]);
        if (nr > 0 && (cur + c > gcapb || nr == gcapr)) {
          ck.push_back(k);
          cur = nr = 0;
        }
        cur += c;
        nr++;
      }
      if (nr > 0) {
        ck.push_back(ptr[l + 1]);
        cur = nr = 0;
      }
    }
  }
  const int nch = (int)ck.size() - 1;
  // split every chunk's rows over the CTAs: each row goes to the half with
  // fewer blocks so far (ties: fewer rows), within capr rows a half
  std::vector<int32_t> half(n), chunk_of(n), grow(n);
  std::vector<std::vector<int32_t>> hrows((size_t)kSweepCta * nch);  // [h * nch + c]
  for (int c = 0; c < nch; c++) {
    int hb[kSweepCta] = {0}, hr[kSweepCta] = {0};
    for (int k = ck[c]; k < ck[c + 1]; k++) {
      const int i = rows[k];
      int h = 0;
      for (int q = 1; q < nsplit; q++)
        if (hr[h] == capr || (hr[q] < capr && (hb[q] < hb[h] || (hb[q] == hb[h] && hr[q] < hr[h]))))
          h = q;
      half[i] = h;
      chunk_of[i] = c;
      grow[i] = k - ck[c];
      hb[h] += cnt(i);
      hr[h]++;
      hrows[(size_t)h * nch + c].push_back(i);
    }
    for (int h = 0; h < kSweepCta; h++)
      if (hb[h] > capb || hr[h] > capr) return cudaErrorInvalidValue;
  }
  // per half chunk: stored blocks (padded), and where each block's x comes
  // from. Near: row solved by the previous chunk (either CTA; ring position
  // = its row index within that chunk); far: solved earlier (global row).
  // U's diagonal block U_ii^{-1} multiplies no x; padding is unused.
  const size_t HC = (size_t)kSweepCta * nch;
  std::vector<int32_t> nbp(HC);
  std::vector<std::vector<int32_t>> nearl(HC), farl(HC);  // pairs (slot, source)
  for (int h = 0; h < kSweepCta; h++)
    for (int c = 0; c < nch; c++) {
      const size_t hc = (size_t)h * nch + c;
      int b = 0;
      auto src = [&](int slot, int j) {
        if (chunk_of[j] == c - 1) {
          nearl[hc].push_back(slot);
          nearl[hc].push_back(grow[j]);
        } else {
          farl[hc].push_back(slot);
          farl[hc].push_back(j);
        }
      };
      for (int i : hrows[hc]) {
        if (upper) {
          b++;  // U_ii^{-1}
          for (int jp = diag[i] + 1; jp < P.rowp[i + 1]; jp++) src(b++, P.cols[jp]);
        } else {
          for (int jp = P.rowp[i]; jp < diag[i]; jp++) src(b++, P.cols[jp]);
        }
      }
      nbp[hc] = std::max(4, (b + 3) & ~3);
    }
  for (int h = 0; h < kSweepCta; h++)
    if (!farl[(size_t)h * nch].empty() || !nearl[(size_t)h * nch].empty())
      return cudaErrorInvalidValue;  // level 0 depends on nothing
  // byte layout of half chunk (h, c): two int4 headers, row records {row,
  // first block, blocks, row index in the chunk}, the near list, the far
  // list and rows of half chunk (h, c+1), then (16-byte aligned) values.
  // Half h's chunks are contiguous; off[h * (nch + 1) + c] is their start.
  auto pre = [&](int h, int c) {
    const size_t hc = (size_t)h * nch + c;
    const int64_t nr = (int64_t)hrows[hc].size();
    const int64_t nf1 = c + 1 < nch ? (int64_t)farl[hc + 1].size() / 2 : 0;
    const int64_t nr1 = c + 1 < nch ? (int64_t)hrows[hc + 1].size() : 0;
    return (32 + 16 * nr + 4 * (int64_t)nearl[hc].size() + 8 * nf1 + 4 * nr1 + 15) & ~(int64_t)15;
  };
  std::vector<int64_t> off((size_t)kSweepCta * (nch + 1), 0);
  size_t nslots = 0;
  int stage = 0;
  int64_t pos = 0;
  for (int h = 0; h < kSweepCta; h++)
    for (int c = 0; c <= nch; c++) {
      off[(size_t)h * (nch + 1) + c] = pos;
      if (c == nch) break;
      const int64_t bytes = pre(h, c) + 36 * (int64_t)vs * nbp[(size_t)h * nch + c];
      pos += bytes;
      stage = (int)std::max<int64_t>(stage, bytes);
      nslots += nbp[(size_t)h * nch + c];
    }
  std::vector<unsigned char> bytes(pos, 0);
  std::vector<int32_t> map(nslots, -1);
  std::vector<int64_t> vpos(nslots);
  size_t q = 0;
  for (int h = 0; h < kSweepCta; h++)
    for (int c = 0; c < nch; c++) {
      const size_t hc = (size_t)h * nch + c;
      const int64_t o = off[(size_t)h * (nch + 1) + c];
      int32_t* w = reinterpret_cast<int32_t*>(bytes.data() + o);
      const int nr = (int)hrows[hc].size(), nb = nbp[hc];
      const int nn = (int)nearl[hc].size() / 2;
      const int nf1 = c + 1 < nch ? (int)farl[hc + 1].size() / 2 : 0;
      const int nr1 = c + 1 < nch ? (int)hrows[hc + 1].size() : 0;
      w[0] = nr;
      w[1] = nb;
      w[2] = nn;
      w[4] = nf1;
      w[5] = nr1;
      int32_t* rec = w + 8;
      int b = 0;
      for (int k = 0; k < nr; k++) {
        const int i = hrows[hc][k];
        rec[4 * k + 0] = i;
        rec[4 * k + 1] = b;
        rec[4 * k + 2] = cnt(i);
        rec[4 * k + 3] = grow[i];
        if (upper) {
          map[q + b++] = diag[i];
          for (int jp = diag[i] + 1; jp < P.rowp[i + 1]; jp++) map[q + b++] = jp;
        } else {
          for (int jp = P.rowp[i]; jp < diag[i]; jp++) map[q + b++] = jp;
        }
      }
      int32_t* lists = rec + 4 * nr;
      std::copy(nearl[hc].begin(), nearl[hc].end(), lists);
      lists += nearl[hc].size();
      if (c + 1 < nch) {
        std::copy(farl[hc + 1].begin(), farl[hc + 1].end(), lists);
        lists += farl[hc + 1].size();
        for (int i : hrows[hc + 1]) *lists++ = i;
      }
      const int64_t v0 = (o + pre(h, c)) / (int64_t)vs;
      for (int k = 0; k < nb; k++) vpos[q + k] = v0 + 36 * (int64_t)k;
      q += nb;
    }
  // algorithmic bytes of one sweep (compulsory unique traffic): per stored
  // block its values and column index; per row a row pointer, its
  // right-hand side and its result (each x entry is read once, however many
  // blocks multiply it)
  gf_precond::Tri& t = p->tri[upper ? 1 : 0];
  t.nsplit = nsplit;
  t.abytes = real * (36 * (long long)vs + 4) + (long long)n * (4 + 48 + 48) + 4;
  t.nch = nch;
  t.stage = stage;
  t.capb = capb;
  t.capr = capr;
  t.nslots = nslots;
  cudaError_t e = cudaSuccess;
  auto up = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  up(t.off.upload(off));
  up(t.vpos.upload(vpos));
  up(t.map.upload(map));
  up(t.stream.upload(bytes));
  return e;
}
// Stream of one triangle for the dataflow sweep (layout described at
// TriDesc). Returns cudaSuccess with *used = false, building nothing, when
// the triangle's ring and stages do not fit one CTA's shared memory.
static cudaError_t build_df(gf_precond* p, const std::vector<int32_t>& diag, bool upper,
                            bool* used) {
  const Pattern& P = p->pat;
  const int n = P.n;
  const std::vector<int32_t>& lv = upper ? p->lvU : p->lvL;
  const int nlev = upper ? p->nlevU : p->nlevL;
  const size_t vs = p->prec == GF_PREC_FP32 ? 4 : 8;
  *used = false;
  // positions: rows by level, ties by row index
  std::vector<int32_t> ptr(nlev + 1, 0), order(n), pos(n);
  for (int i = 0; i < n; i++) ptr[lv[i] + 1]++;
  for (int l = 0; l < nlev; l++) ptr[l + 1] += ptr[l];
  {
    std::vector<int32_t> f(ptr.begin(), ptr.end() - 1);
    for (int i = 0; i < n; i++) order[f[lv[i]]++] = i;
  }
  for (int k = 0; k < n; k++) pos[order[k]] = k;
  // a row's blocks: (position multiplied, factor block), U_ii^{-1} first in U
  auto blocks = [&](int i, std::vector<std::pair<int32_t, int32_t>>& out) {
    out.clear();
    if (upper) {
      for (int jp = diag[i] + 1; jp < P.rowp[i + 1]; jp++) out.emplace_back(pos[P.cols[jp]], jp);
    } else {
      for (int jp = P.rowp[i]; jp < diag[i]; jp++) out.emplace_back(pos[P.cols[jp]], jp);
    }
    std::sort(out.begin(), out.end());
    if (upper) out.insert(out.begin(), std::make_pair(-1, diag[i]));
  };
  std::vector<std::pair<int32_t, int32_t>> bl;
  int maxdist = 1, maxcnt = 0;
  long long real = 0;
  for (int i = 0; i < n; i++) {
    blocks(i, bl);
    maxcnt = std::max(maxcnt, (int)bl.size());
    real += (long long)bl.size();
    for (auto& b : bl)
      if (b.first >= 0) maxdist = std::max(maxdist, pos[i] - b.first);
  }
  // the ring holds every position a row may still need (maxdist back) plus
  // the lag of the progress the warps report (a chunk's rows for the compute
  // warps, a report batch for the writer), so flow control never waits on a
  // warp that is itself waiting
  int ring = 64;
  while (ring < 2 * (maxdist + 1) || ring < maxdist + 2 * kDfRows + kDfWriteBatch + 8) ring *= 2;
  const int capb = std::max(vs == 4 ? 224 : 112, maxcnt), capr = kDfRows;
  // chunks: consecutive positions, at most capb blocks and capr rows
  std::vector<int32_t> ck{0};
  {
    int cb = 0, cr = 0;
    for (int k = 0; k < n; k++) {
      const int cnt = upper ? P.rowp[order[k] + 1] - diag[order[k]] : diag[order[k]] - P.rowp[order[k]];
      if (cr > 0 && (cb + cnt > capb || cr == capr)) {
        ck.push_back(k);
        cb = cr = 0;
      }
      cb += cnt;
      cr++;
    }
    ck.push_back(n);
  }
  const int nch = (int)ck.size() - 1;
  std::vector<int64_t> off(nch + 1, 0);
  auto head = [&](int c, int nb) {
    return (16 + 16 * (int64_t)(ck[c + 1] - ck[c]) + 4 * (int64_t)nb + 15) & ~(int64_t)15;
  };
  std::vector<int32_t> nbc(nch, 0);
  int stage = 0;
  for (int c = 0; c < nch; c++) {
    for (int k = ck[c]; k < ck[c + 1]; k++) {
      const int i = order[k];
      nbc[c] += upper ? P.rowp[i + 1] - diag[i] : diag[i] - P.rowp[i];
    }
    const int64_t bytes = head(c, nbc[c]) + 36 * (int64_t)vs * nbc[c];
    off[c + 1] = off[c] + bytes;
    stage = (int)std::max<int64_t>(stage, bytes);
  }
  if (df_smem_bytes(stage, ring) > kSweepSmemMax) return cudaSuccess;
  std::vector<unsigned char> bytes(off[nch], 0);
  const size_t nslots = (size_t)real;
  std::vector<int32_t> map(nslots);
  std::vector<int64_t> vpos(nslots);
  size_t q = 0;
  for (int c = 0; c < nch; c++) {
    int32_t* w = reinterpret_cast<int32_t*>(bytes.data() + off[c]);
    const int nr = ck[c + 1] - ck[c];
    w[0] = nr;
    w[1] = nbc[c];
    w[2] = ck[c];
    int32_t* rec = w + 4;
    int32_t* dep = rec + 4 * nr;
    const int64_t v0 = (off[c] + head(c, nbc[c])) / (int64_t)vs;
    int b = 0;
    for (int k = 0; k < nr; k++) {
      const int i = order[ck[c] + k];
      blocks(i, bl);
      rec[4 * k + 0] = i;
      rec[4 * k + 1] = b;
      rec[4 * k + 2] = (int)bl.size();
      for (auto& e : bl) {
        dep[b] = e.first;
        map[q] = e.second;
        vpos[q] = v0 + 36 * (int64_t)b;
        q++;
        b++;
      }
    }
  }
  gf_precond::Tri& t = p->tri[upper ? 1 : 0];
  t.kind = TRI_DATAFLOW;
  t.nsplit = 1;
  t.ring = ring;
  t.maxdist = maxdist;
  t.nch = nch;
  t.stage = stage;
  t.capb = capb;
  t.capr = capr;
  t.nslots = nslots;
  t.abytes = real * (36 * (long long)vs + 4) + (long long)n * (4 + 48 + 48) + 4;
  cudaError_t e = cudaSuccess;
  auto up = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  up(t.off.upload(off));
  up(t.vpos.upload(vpos));
  up(t.map.upload(map));
  up(t.stream.upload(bytes));
  if (e == cudaSuccess) *used = true;
  return e;
}
static TriDesc tri_desc(const gf_precond* p, int which) {
  const gf_precond::Tri& t = p->tri[which];
  return TriDesc{t.nch,    t.stage,  t.capb, t.capr, t.off.p,   t.stream.p,
                 t.abytes, t.nsplit, t.kind, t.ring, t.maxdist};
}
static size_t sweep_smem(const gf_precond* p, int which) {
  const gf_precond::Tri& t = p->tri[which];
  return t.kind == TRI_DATAFLOW ? df_smem_bytes(t.stage, t.ring)
                                : sweep_smem_bytes(t.stage, t.capb, t.capr);
}
}  // namespace gf

struct gf_batch {
  int np = 0, nrows = 0, maxlevL = 0, maxlevU = 0;
  size_t smemL = 0, smemU = 0;  // dynamic shared memory of the level-synchronous sweeps
  size_t dfL = 0, dfU = 0;      // ... and of the dataflow sweeps
  int nlevelL = 0, nlevelU = 0, ndfL = 0, ndfU = 0;  // problems solved by each kind
  int pprec = GF_PREC_FP64;      // factor precision shared by the batch's preconditioners
  size_t N = 0;  // doubles in batch space
  std::vector<gf_assembler*> asms;
  std::vector<gf_bsr*> mats;
  std::vector<gf_precond*> pcs;
  std::vector<int> offs;
  DevBuf<ProbDev> d_desc;
  DevBuf<int32_t> d_row_prob;
  DevBuf<SweepCtl> d_ctl;
  DevBuf<double> d_tmp, d_b, d_x;
  int nchunks = 0;
  DevBuf<int32_t> d_cprob, d_pstart;
  int fac_grid = 0;                  // CTAs of the dataflow factorization
  DevBuf<int32_t> d_fcta, d_fgrab;   // problem of each CTA; per-problem row counters
  DevBuf<int64_t> d_clo, d_chi;
  DevBuf<PermEntry> d_perm_b, d_perm_x, d_perm_out;
  int m = 0;
  DevBuf<double> V, H, g, cs, ss, y, h, hn, target, partial, pnorm, w, t, r, d, e, norms, bnorm;
  DevBuf<double> tfac;
  DevBuf<int> jcnt, run, live, live2;
  gf::BatchAsm* basm = nullptr;  // launch data of the batched assembly
  int scatter = 0;               // 0: coloured, GF_ASSEMBLE_ATOMIC: atomic
  Chunks chunks() const { return Chunks{nchunks, d_cprob.p, d_clo.p, d_chi.p, d_pstart.p}; }
  ~gf_batch() { gf::batch_asm_free(basm); }
};

namespace gf {

static int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// Order of the factorization steps of every row (ord[r0 .. di) = slots of
// the row's lower blocks in the order they are taken). Step k must follow
// every step k' whose row k' has column k in its upper part (k' updates
// A_ik), and nothing else; among the steps whose predecessors are done the
// one whose row k has the lowest lower level goes first (ties: lower
// column). Rows finish roughly in level order in the dataflow
// factorization, so the steps that wait for the last-finishing rows move to
// the end of the row and the steps after them shrink to those that really
// depend on them. Rows longer than kOrderMax lower blocks keep ascending
// order (complete factors: there every step depends on the previous one).
constexpr int kOrderMax = 128;
static void step_order_rows(const Pattern& P, const std::vector<int32_t>& diag,
                            const std::vector<int32_t>& lv, std::vector<int32_t>& ord, int i0,
                            int i1) {
  std::vector<int32_t> indeg, head, nxt, to, heap;
  for (int i = i0; i < i1; i++) {
    const int r0 = P.rowp[i], di = diag[i], m = di - r0;
    if (m <= 1 || m > kOrderMax) {
      for (int t = r0; t < di; t++) ord[t] = t;
      continue;
    }
    indeg.assign(m, 0);
    head.assign(m, -1);
    nxt.clear();
    to.clear();
    for (int a = 0; a < m; a++) {
      const int k = P.cols[r0 + a];
      // columns of U(k) that are lower columns of row i after a (both ascending)
      int u = diag[k] + 1;
      const int u1 = P.rowp[k + 1];
      int b = a + 1;
      while (u < u1 && b < m) {
        const int cu = P.cols[u], cb = P.cols[r0 + b];
        if (cu < cb) {
          u++;
        } else if (cb < cu) {
          b++;
        } else {
          to.push_back(b);
          nxt.push_back(head[a]);
          head[a] = (int)to.size() - 1;
          indeg[b]++;
          u++;
          b++;
        }
      }
    }
    // Kahn's algorithm with a min-heap on (level, column) = (lv, local index)
    auto key = [&](int a) { return ((long long)lv[P.cols[r0 + a]] << 32) | (unsigned)a; };
    auto cmp = [&](int x, int y) { return key(x) > key(y); };
    heap.clear();
    for (int a = 0; a < m; a++)
      if (indeg[a] == 0) heap.push_back(a);
    std::make_heap(heap.begin(), heap.end(), cmp);
    int t = r0;
    while (!heap.empty()) {
      std::pop_heap(heap.begin(), heap.end(), cmp);
      const int a = heap.back();
      heap.pop_back();
      ord[t++] = r0 + a;
      for (int e = head[a]; e >= 0; e = nxt[e])
        if (--indeg[to[e]] == 0) {
          heap.push_back(to[e]);
          std::push_heap(heap.begin(), heap.end(), cmp);
        }
    }
  }
}
// Length of the factorization's dependency chain in step units when every
// row takes its steps in the order `ord` (null: ascending) and finishing a
// row costs two steps: a row's step k starts once its previous step and
// row k are done.
static double step_chain(const Pattern& P, const std::vector<int32_t>& diag,
                         const std::vector<int32_t>* ord) {
  std::vector<double> done(P.n, 0.0);
  double longest = 0.0;
  for (int i = 0; i < P.n; i++) {
    double t = 0.0;
    for (int s = P.rowp[i]; s < diag[i]; s++) {
      const int k = P.cols[ord ? (*ord)[s] : s];
      t = std::max(t, done[k]) + 1.0;
    }
    done[i] = t + 2.0;
    longest = std::max(longest, done[i]);
  }
  return longest;
}

// Rows are independent: host threads take contiguous row ranges. The order
// is kept only where it shortens the dependency chain by 15 % or more
// (natural-ordered grids, where a row's last-finishing dependency otherwise
// sits before its same-line steps: 18-24 % on plates, a 1.5-3x faster
// factorization); elsewhere (RCM orders: 0-9 %) the steps stay ascending,
// the order of the host and reference factorizations. The summation order
// matters on ill-conditioned shells: on the jittered 100x50 cantilever
// (RCM, ILU(8), factor entries up to 3e8) the two orders give factors with
// the same backward error, 6e-16, but right-preconditioned GMRES needs 59
// steps with the ascending one and 118 with the reordered one.
static void step_order(const Pattern& P, const std::vector<int32_t>& diag,
                       const std::vector<int32_t>& lv, std::vector<int32_t>& ord) {
  const int n = P.n;
  ord.assign(P.nnz(), 0);
  const int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (nt == 1 || n < 4096) {
    step_order_rows(P, diag, lv, ord, 0, n);
  } else {
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++) {
      const int i0 = (int)((long long)n * t / nt), i1 = (int)((long long)n * (t + 1) / nt);
      th.emplace_back([&, i0, i1] { step_order_rows(P, diag, lv, ord, i0, i1); });
    }
    for (auto& x : th) x.join();
  }
  if (step_chain(P, diag, &ord) * 1.15 > step_chain(P, diag, nullptr))
    for (int i = 0; i < n; i++)
      for (int t = P.rowp[i]; t < diag[i]; t++) ord[t] = t;
}

// CTAs of the dataflow factorization for one problem given `budget` CTAs for
// it: at least one, at most one per 32 rows (four rows per warp) and 128.
static int fac_ctas_cap(const gf_precond* p, int budget) {
  return std::max(1, std::min({budget, 128, p->pat.n / (4 * kFacWarps)}));
}
// A preconditioner factored alone gets the whole GPU (one CTA per SM).
static int fac_ctas_alone(const gf_precond* p) { return fac_ctas_cap(p, sm_count()); }

// Spreads one CTA per SM over the batch's problems in proportion to their
// block updates to the power 0.7 (largest remainders first), within each
// problem's cap: the small problems' dependency chains need a few CTAs more
// than their share of the updates (64-plate batch on B200, factorization
// ms by exponent: 0.5 43.3, 0.6 40.1, 0.7 38.0, 0.85 39.2, 1 41.4, 1.5 56.6);
// fills cta_prob with the problem of every CTA.
static void fac_plan(const std::vector<gf_precond*>& pcs, std::vector<int>& ctas,
                     std::vector<int32_t>& cta_prob) {
  const int np = (int)pcs.size(), total = std::max(sm_count(), np);
  double W = 0.0;
  for (auto* p : pcs) W += std::pow((double)std::max<long long>(p->fwork, 1), 0.7);
  ctas.assign(np, 1);
  std::vector<std::pair<double, int>> rem;
  int used = 0;
  for (int k = 0; k < np; k++) {
    const double want = total * std::pow((double)std::max<long long>(pcs[k]->fwork, 1), 0.7) / W;
    const int cap = fac_ctas_cap(pcs[k], total);
    ctas[k] = std::max(1, std::min(cap, (int)want));
    used += ctas[k];
    if (ctas[k] < cap) rem.push_back({want - ctas[k], k});
  }
  std::sort(rem.begin(), rem.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  for (size_t q = 0; q < rem.size() && used < total; q++) {
    ctas[rem[q].second]++;
    used++;
  }
  cta_prob.clear();
  for (int k = 0; k < np; k++)
    for (int c = 0; c < ctas[k]; c++) cta_prob.push_back(k);
}

// Descriptor table (rebuilt when a buffer such as the FP32 matrix copy is
// allocated).
static gf_status upload_desc(gf_batch* B) {
  std::vector<ProbDev> h(B->np);
  for (int k = 0; k < B->np; k++) {
    gf_assembler* a = B->asms[k];
    gf_precond* p = B->pcs[k];
    ProbDev& d = h[k];
    d.n = a->nnodes;
    d.off = B->offs[k];
    d.rowp = a->d_rowp.p;
    d.cols = a->d_cols.p;
    d.A64 = B->mats[k]->vals.p;
    d.A32 = B->mats[k]->vals32.p;
    d.prowp = p->d_rowp.p;
    d.pcols = p->d_cols.p;
    d.pdiag = p->d_diag.p;
    d.LU64 = p->d_lu.p;
    d.nlevL = p->nlevL;
    d.done = p->d_done.p;
    d.pord = p->d_ord.p;
    d.nlevU = p->nlevU;
    d.levLptr = p->d_levLptr.p;
    d.levLrows = p->d_levLrows.p;
    d.L = tri_desc(p, 0);
    d.U = tri_desc(p, 1);
  }
  GF_CUDA(cudaMemcpy(B->d_desc.p, h.data(), sizeof(ProbDev) * B->np, cudaMemcpyHostToDevice));
  return GF_OK;
}

static gf_status batch_build(gf_batch* B) {
  const int np = B->np;
  B->offs.resize(np + 1);
  B->offs[0] = 0;
  for (int k = 0; k < np; k++) B->offs[k + 1] = B->offs[k] + B->asms[k]->nnodes;
  B->nrows = B->offs[np];
  B->N = (size_t)6 * B->nrows;
  std::vector<int32_t> row_prob(B->nrows);
  B->pprec = B->pcs[0]->prec;
  for (int k = 0; k < np; k++) {
    if (B->pcs[k]->prec != B->pprec) return GF_INVALID_ARG;  // one factor precision per batch
    for (int w = 0; w < 2; w++) {
      const bool df = B->pcs[k]->tri[w].kind == TRI_DATAFLOW;
      size_t& sm = df ? (w ? B->dfU : B->dfL) : (w ? B->smemU : B->smemL);
      sm = std::max(sm, sweep_smem(B->pcs[k], w));
      (df ? (w ? B->ndfU : B->ndfL) : (w ? B->nlevelU : B->nlevelL))++;
    }
    for (int i = 0; i < B->asms[k]->nnodes; i++) row_prob[B->offs[k] + i] = k;
    B->maxlevL = std::max(B->maxlevL, B->pcs[k]->nlevL);
    B->maxlevU = std::max(B->maxlevU, B->pcs[k]->nlevU);
  }
  // reduction chunks aligned to each problem
  std::vector<int32_t> cprob, pstart(np + 1);
  std::vector<int64_t> clo, chi;
  for (int k = 0; k < np; k++) {
    pstart[k] = (int32_t)cprob.size();
    const int64_t lo = 6ll * B->offs[k], hi = 6ll * B->offs[k + 1];
    for (int64_t s = lo; s < hi; s += kChunk) {
      cprob.push_back(k);
      clo.push_back(s);
      chi.push_back(std::min(hi, s + (int64_t)kChunk));
    }
  }
  pstart[np] = (int32_t)cprob.size();
  B->nchunks = (int)cprob.size();
  cudaError_t e = cudaSuccess;
  auto up = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  up(B->d_desc.alloc(np));
  {
    std::vector<int> ctas;
    std::vector<int32_t> cta_prob;
    fac_plan(B->pcs, ctas, cta_prob);
    B->fac_grid = (int)cta_prob.size();
    up(B->d_fcta.upload(cta_prob));
    up(B->d_fgrab.alloc(np));
  }
  up(B->d_row_prob.upload(row_prob));
  up(B->d_ctl.alloc(1));
  if (e == cudaSuccess) up(cudaMemset(B->d_ctl.p, 0, sizeof(SweepCtl)));
  up(B->d_tmp.alloc(B->N));
  up(B->d_b.alloc(B->N));
  up(B->d_x.alloc(B->N));
  up(B->d_cprob.upload(cprob));
  up(B->d_pstart.upload(pstart));
  up(B->d_clo.upload(clo));
  up(B->d_chi.upload(chi));
  up(B->d_perm_b.alloc(np));
  up(B->d_perm_x.alloc(np));
  up(B->d_perm_out.alloc(np));
  up(B->norms.alloc(np));
  up(B->bnorm.alloc(np));
  up(B->live2.alloc(np));
  if (e != cudaSuccess) {
    set_last_error("batch build", e);
    return e == cudaErrorMemoryAllocation ? GF_OOM : GF_CUDA_ERROR;
  }
  return upload_desc(B);
}

static gf_status ensure_gmres(gf_batch* B, int m) {
  if (B->m == m) return GF_OK;
  const int np = B->np;
  cudaError_t e = cudaSuccess;
  auto al = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  al(B->V.alloc((size_t)(m + 1) * B->N));
  al(B->H.alloc((size_t)np * (m + 1) * m));
  al(B->g.alloc((size_t)np * (m + 1)));
  al(B->cs.alloc((size_t)np * m));
  al(B->ss.alloc((size_t)np * m));
  al(B->y.alloc((size_t)np * m));
  al(B->h.alloc((size_t)np * (m + 1)));
  al(B->hn.alloc(np));
  al(B->target.alloc(np));
  al(B->tfac.alloc(np));
  al(B->partial.alloc((size_t)(m + 1) * B->nchunks));
  al(B->pnorm.alloc(B->nchunks));
  al(B->w.alloc(B->N));
  al(B->t.alloc(B->N));
  al(B->r.alloc(B->N));
  al(B->d.alloc(B->N));
  al(B->e.alloc(B->N));
  al(B->jcnt.alloc(np));
  al(B->run.alloc(np));
  al(B->live.alloc(np));
  if (e != cudaSuccess) {
    set_last_error("gmres workspace", e);
    B->m = 0;
    return e == cudaErrorMemoryAllocation ? GF_OOM : GF_CUDA_ERROR;
  }
  GF_CUDA(cudaMemset(B->H.p, 0, sizeof(double) * B->H.n));
  B->m = m;
  return GF_OK;
}

static GmArrays arrays(gf_batch* B) {
  return GmArrays{B->H.p,  B->g.p,      B->cs.p,   B->ss.p,  B->y.p,   B->h.p,
                  B->hn.p, B->target.p, B->jcnt.p, B->run.p, B->live.p};
}


// Sweep timing for benchmarks (gf_timing_enable / gf_timing_read): CUDA
// events bracket the two sweep launches of every preconditioner apply on the
// launching stream, and the sweeps add their algorithmic bytes to a device
// counter. Off by default; the events come from a pool that is drained
// (synchronised and summed) when it runs full.
namespace {
struct Timing {
  std::mutex mu;
  bool on = false;
  unsigned long long* d_bytes = nullptr;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
  size_t used = 0;
  double ms = 0.0;
  long long launches = 0;
};
Timing g_timing;
constexpr size_t kTimingPool = 8192;
cudaError_t timing_drain_locked() {
  for (size_t k = 0; k < g_timing.used; k++) {
    float t = 0.f;
    cudaError_t e = cudaEventSynchronize(g_timing.pool[k].second);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, g_timing.pool[k].first, g_timing.pool[k].second);
    if (e != cudaSuccess) return e;
    g_timing.ms += t;
  }
  g_timing.used = 0;
  return cudaSuccess;
}
}  // namespace
// Records the opening event of one sweep pair when timing is on; *e1 gets
// the closing event to record after the second launch.
static gf_status timing_begin(cudaStream_t st, unsigned long long** ctr, cudaEvent_t* e1) {
  std::lock_guard<std::mutex> lk(g_timing.mu);
  if (!g_timing.on) return GF_OK;
  if (g_timing.used == g_timing.pool.size()) {
    if (g_timing.pool.size() < kTimingPool) {
      cudaEvent_t a, b;
      GF_CUDA(cudaEventCreate(&a));
      GF_CUDA(cudaEventCreate(&b));
      g_timing.pool.emplace_back(a, b);
    } else {
      GF_CUDA(timing_drain_locked());
    }
  }
  auto& pr = g_timing.pool[g_timing.used++];
  GF_CUDA(cudaEventRecord(pr.first, st));
  *e1 = pr.second;
  *ctr = g_timing.d_bytes;
  g_timing.launches += 2;
  return GF_OK;
}

// z = U^{-1} L^{-1} r for problems with live[p] (all when live is null).
// The factor values are in the preconditioners' precision (one per batch),
// independent of the precision of the Krylov loop that calls this.
// One triangle of every problem of the batch: the dataflow kernel for the
// problems whose triangle has a dataflow stream, the level-synchronous
// kernel for the others (each kernel skips the other kind's problems).
template <class VT, bool UPPER>
static cudaError_t launch_tri(gf_batch* B, cudaStream_t st, const int* live, const double* rhs,
                              double* out, unsigned long long* ctr) {
  // the same caps for every batch: threads launching batches with different
  // footprints concurrently must not lower them under each other
  cudaError_t e = cudaSuccess;
  if (UPPER ? B->ndfU : B->ndfL) {
    e = cudaFuncSetAttribute(bsweep_df<VT, UPPER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSweepSmemMax);
    if (e != cudaSuccess) return e;
    ::gf::count_launch();
    bsweep_df<VT, UPPER><<<B->np, kDfThreads, UPPER ? B->dfU : B->dfL, st>>>(
        B->d_desc.p, live, rhs, out, B->d_ctl.p, ctr);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (UPPER ? B->nlevelU : B->nlevelL) {
    e = cudaFuncSetAttribute(bsweep_tma<VT, UPPER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kSweepSmemMax);
    if (e != cudaSuccess) return e;
    e = launch_sweep<VT, UPPER>(B->np, UPPER ? B->smemU : B->smemL, st, B->d_desc.p, live, rhs,
                                out, B->d_ctl.p, ctr);
  }
  return e;
}

static bool sweeps_fit(const gf_batch* B) {
  return B->smemL <= kSweepSmemMax && B->smemU <= kSweepSmemMax && B->dfL <= kSweepSmemMax &&
         B->dfU <= kSweepSmemMax;
}

// y = L^{-1} r into tmp, z = U^{-1} y, for the problems with live[p].
template <class VT>
static gf_status bsweeps(gf_batch* B, const int* live, const double* r, double* tmp, double* z,
                         cudaStream_t st, bool timed) {
  unsigned long long* ctr = nullptr;
  cudaEvent_t e1 = nullptr;
  if (timed && timing_begin(st, &ctr, &e1) != GF_OK) return GF_CUDA_ERROR;
  GF_CUDA((launch_tri<VT, false>(B, st, live, r, tmp, ctr)));
  GF_CUDA((launch_tri<VT, true>(B, st, live, tmp, z, ctr)));
  GF_CHECK_LAUNCH();
  if (e1) GF_CUDA(cudaEventRecord(e1, st));
  return GF_OK;
}
template <class VT>
static gf_status bprecond(gf_batch* B, const int* live, const double* r, double* z,
                          cudaStream_t st) {
  if (!sweeps_fit(B)) return GF_INVALID_ARG;
  return B->pprec == GF_PREC_FP32 ? bsweeps<float>(B, live, r, B->d_tmp.p, z, st, true)
                                  : bsweeps<double>(B, live, r, B->d_tmp.p, z, st, true);
}

template <class VT>
static gf_status bspmv(gf_batch* B, const int* live, const double* x, double alpha, double beta,
                       double* y, cudaStream_t st) {
  bspmv_kernel<VT><<<(B->nrows + 7) / 8, 256, 0, st>>>(B->nrows, B->d_row_prob.p, B->d_desc.p,
                                                       live, x, alpha, beta, y); ::gf::count_launch();
  GF_CHECK_LAUNCH();
  return GF_OK;
}

// Reads and clears the status flags that the batch's kernels have recorded
// since the last read (timeouts of bounded waits, zero pivots). Flags are
// cleared only here, after they have been read, so a flag set by a launch
// whose caller did not wait (gf_precond_apply) is reported by the next call
// that reads them.
static gf_status read_ctl(gf_batch* B, cudaStream_t st, SweepCtl* h) {
  GF_CUDA(cudaMemcpyAsync(h, B->d_ctl.p, sizeof(SweepCtl), cudaMemcpyDeviceToHost, st));
  GF_CUDA(cudaMemsetAsync(B->d_ctl.p, 0, sizeof(SweepCtl), st));
  GF_CUDA(cudaStreamSynchronize(st));
  return GF_OK;
}
static gf_status ctl_status(const SweepCtl& h) {
  if (h.status & ST_TIMEOUT) {
    set_last_error_text("a bounded device-side wait ran out (a stalled copy or partner CTA)");
    return GF_TIMEOUT;
  }
  if (h.status & ST_ZERO_PIVOT) {
    set_last_error_text("singular diagonal block in block row " + std::to_string(h.pivot - 1) +
                        " (batch space)");
    return GF_ZERO_PIVOT;
  }
  return GF_OK;
}

static gf_status batch_factor(gf_batch* B, cudaStream_t st) {
  for (int k = 0; k < B->np; k++) {
    gf_precond* p = B->pcs[k];
    const size_t nv = (size_t)36 * p->pat.nnz();
    GF_CUDA(cudaMemsetAsync(p->d_lu.p, 0, sizeof(double) * nv, st));
    const size_t na = (size_t)36 * p->a->pat.nnz();
    scatter_values_kernel<<<(unsigned)((na + 255) / 256), 256, 0, st>>>(
        p->a->pat.nnz(), p->d_amap.p, B->mats[k]->vals.p, p->d_lu.p); ::gf::count_launch();
  }
  GF_CHECK_LAUNCH();
  {
    // a fresh epoch per launch: flags left by earlier factorizations (of any
    // batch holding these preconditioners) never equal it
    static std::atomic<int> epochs{0};
    int epoch = ++epochs;
    if (epoch <= 0) {
      epochs = 1;
      epoch = 1;
    }
    GF_CUDA(cudaMemsetAsync(B->d_fgrab.p, 0, sizeof(int32_t) * B->np, st));
    ::gf::count_launch();
    GF_CUDA(cudaFuncSetAttribute(bfactor_df, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kFacSmem));
    bfactor_df<<<(unsigned)B->fac_grid, kFacWarps * 32, kFacSmem, st>>>(
        B->d_desc.p, B->d_fcta.p, B->d_fgrab.p, epoch, B->d_ctl.p);
  }
  GF_CHECK_LAUNCH();
  for (int k = 0; k < B->np; k++) {
    gf_precond* p = B->pcs[k];
    for (int w = 0; w < 2; w++) {
      gf_precond::Tri& t = p->tri[w];
      const unsigned nb = (unsigned)((t.nslots * 36 + 255) / 256);
      if (t.nslots == 0) continue;
      if (p->prec == GF_PREC_FP32)
        repack_kernel<float><<<nb, 256, 0, st>>>(t.nslots, t.map.p, t.vpos.p, p->d_lu.p,
                                                  reinterpret_cast<float*>(t.stream.p));
      else
        repack_kernel<double><<<nb, 256, 0, st>>>(t.nslots, t.map.p, t.vpos.p, p->d_lu.p,
                                                   reinterpret_cast<double*>(t.stream.p));
      ::gf::count_launch();
    }
  }
  GF_CHECK_LAUNCH();
  SweepCtl h;
  gf_status s = read_ctl(B, st, &h);
  if (s != GF_OK) return s;
  return ctl_status(h);
}

// Batched restarted GMRES on A x = b (batch space) for problems with
// live0[p] != 0. side 1: right preconditioning (Givens residual = true
// residual); side 0: left (the reference's choice). Per-problem outputs:
// iters, restarts, rel (true ||b - A x|| / ||b||).
template <class VT>
static gf_status bgmres(gf_batch* B, const double* b, double* x, int m, int max_it, double rtol,
                        int side, int check_every, const std::vector<int>& live0,
                        std::vector<int>& iters, std::vector<int>& restarts,
                        std::vector<double>& rel, cudaStream_t st) {
  const int np = B->np;
  gf_status s = ensure_gmres(B, m);
  if (s != GF_OK) return s;
  const Chunks C = B->chunks();
  const GmArrays G = arrays(B);
  const int nc = B->nchunks;
  const int pb = (np + 127) / 128;
  std::vector<double> bn(np, 1.0), rn(np);
  GF_CUDA(cudaMemcpyAsync(B->live.p, live0.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st));
  seg_sumsq<<<nc, kRedThreads, 0, st>>>(b, C, nullptr, B->pnorm.p); ::gf::count_launch();
  seg_norm_out<<<pb, 128, 0, st>>>(B->pnorm.p, C, np, nullptr, B->bnorm.p); ::gf::count_launch();
  GF_CUDA(cudaMemcpyAsync(bn.data(), B->bnorm.p, sizeof(double) * np, cudaMemcpyDeviceToHost, st));
  if (side != 0) set_target<<<pb, 128, 0, st>>>(np, B->bnorm.p, rtol, G), ::gf::count_launch();
  GF_CHECK_LAUNCH();
  GF_CUDA(cudaStreamSynchronize(st));
  for (int p = 0; p < np; p++)
    if (bn[p] == 0.0) bn[p] = 1.0;
  std::vector<int> live = live0, jc(np), runh(np);
  SweepCtl ctlh{};
  std::vector<double> tf(np, 0.0);
  iters.assign(np, 0);
  restarts.assign(np, 0);
  rel.assign(np, 0.0);
  int steps_total = 0;
  bool first = true;
  while (true) {
    // r = b - A x and the true relative residual of every live problem
    seg_copy<<<nc, kRedThreads, 0, st>>>(b, B->r.p, C, B->live.p); ::gf::count_launch();
    s = bspmv<VT>(B, B->live.p, x, -1.0, 1.0, B->r.p, st);
    if (s != GF_OK) return s;
    seg_sumsq<<<nc, kRedThreads, 0, st>>>(B->r.p, C, B->live.p, B->pnorm.p); ::gf::count_launch();
    seg_norm_out<<<pb, 128, 0, st>>>(B->pnorm.p, C, np, B->live.p, B->norms.p); ::gf::count_launch();
    GF_CUDA(cudaMemcpyAsync(rn.data(), B->norms.p, sizeof(double) * np, cudaMemcpyDeviceToHost,
                            st));
    GF_CUDA(cudaStreamSynchronize(st));
    bool any = false, bad = false;
    for (int p = 0; p < np; p++) {
      if (!live[p]) continue;
      rel[p] = rn[p] / bn[p];
      if (!std::isfinite(rel[p])) {
        bad = true;
        live[p] = 0;
      } else if (rel[p] <= rtol) {
        live[p] = 0;
      } else {
        any = true;
        if (!first) restarts[p]++;
      }
    }
    first = false;
    if (bad) return GF_NAN;
    if (!any || steps_total >= max_it) break;
    GF_CUDA(cudaMemcpyAsync(B->live.p, live.data(), sizeof(int) * np, cudaMemcpyHostToDevice,
                            st));
    const double* src = B->r.p;
    if (side == 0) {
      s = bprecond<VT>(B, B->live.p, B->r.p, B->t.p, st);
      if (s != GF_OK) return s;
      src = B->t.p;
      // Left preconditioning minimises ||M^-1 r||, which can sit far from
      // ||r|| when M is ill-conditioned: every cycle asks the preconditioned
      // residual to drop by the factor the true residual still needs (with
      // a margin of 2 after the first cycle).
      for (int p = 0; p < np; p++)
        tf[p] = live[p] ? (restarts[p] ? 0.5 : 1.0) * rtol * bn[p] / rn[p] : 0.0;
      GF_CUDA(cudaMemcpyAsync(B->tfac.p, tf.data(), sizeof(double) * np, cudaMemcpyHostToDevice,
                              st));
    }
    seg_sumsq<<<nc, kRedThreads, 0, st>>>(src, C, B->live.p, B->pnorm.p); ::gf::count_launch();
    bcycle_init<<<pb, 128, 0, st>>>(B->pnorm.p, C, np, m, G, side == 0 ? B->tfac.p : nullptr);
    ::gf::count_launch();
    seg_scale<<<nc, kRedThreads, 0, st>>>(src, B->V.p, C, B->run.p, B->hn.p); ::gf::count_launch();
    GF_CHECK_LAUNCH();
    const int steps = std::min(m, max_it - steps_total);
    int jj = 0;
    while (jj < steps) {
      const int batch = std::min(check_every, steps - jj);
      for (int k = 0; k < batch; k++, jj++) {
        const double* vj = B->V.p + (size_t)jj * B->N;
        if (side == 0) {
          s = bspmv<VT>(B, B->run.p, vj, 1.0, 0.0, B->t.p, st);
          if (s == GF_OK) s = bprecond<VT>(B, B->run.p, B->t.p, B->w.p, st);
        } else {
          s = bprecond<VT>(B, B->run.p, vj, B->t.p, st);
          if (s == GF_OK) s = bspmv<VT>(B, B->run.p, B->t.p, 1.0, 0.0, B->w.p, st);
        }
        if (s != GF_OK) return s;
        seg_dots<<<nc, kRedThreads, 0, st>>>(B->V.p, B->w.p, B->N, jj, C, B->run.p,
                                              B->partial.p); ::gf::count_launch();
        seg_reduce_dots<<<np, 128, 0, st>>>(B->partial.p, C, jj, m, G, 0); ::gf::count_launch();
        seg_update<<<nc, kRedThreads, 0, st>>>(B->V.p, B->w.p, B->N, jj, m, C, G, nullptr); ::gf::count_launch();
        seg_dots<<<nc, kRedThreads, 0, st>>>(B->V.p, B->w.p, B->N, jj, C, B->run.p,
                                              B->partial.p); ::gf::count_launch();
        seg_reduce_dots<<<np, 128, 0, st>>>(B->partial.p, C, jj, m, G, 1); ::gf::count_launch();
        seg_update<<<nc, kRedThreads, 0, st>>>(B->V.p, B->w.p, B->N, jj, m, C, G, B->pnorm.p); ::gf::count_launch();
        seg_norm_finish<<<pb, 128, 0, st>>>(B->pnorm.p, C, np, jj, m, G); ::gf::count_launch();
        seg_scale<<<nc, kRedThreads, 0, st>>>(B->w.p, B->V.p + (size_t)(jj + 1) * B->N, C,
                                               B->run.p, B->hn.p); ::gf::count_launch();
        bgivens<<<pb, 128, 0, st>>>(np, jj, m, steps, G); ::gf::count_launch();
        GF_CHECK_LAUNCH();
      }
      GF_CUDA(cudaMemcpyAsync(runh.data(), B->run.p, sizeof(int) * np, cudaMemcpyDeviceToHost,
                              st));
      GF_CUDA(cudaMemcpyAsync(&ctlh, B->d_ctl.p, sizeof(SweepCtl), cudaMemcpyDeviceToHost, st));
      GF_CUDA(cudaStreamSynchronize(st));
      // a sweep whose bounded wait ran out left a partial z: stop (the
      // caller reads and clears the flag)
      if (ctlh.status & ST_TIMEOUT) return GF_TIMEOUT;
      if (std::all_of(runh.begin(), runh.end(), [](int v) { return v == 0; })) break;
    }
    bbacksolve<<<pb, 128, 0, st>>>(np, m, G); ::gf::count_launch();
    seg_combine<<<nc, kRedThreads, 0, st>>>(B->V.p, B->N, m, C, G, B->w.p); ::gf::count_launch();
    GF_CHECK_LAUNCH();
    if (side == 1) {
      s = bprecond<VT>(B, B->live.p, B->w.p, B->t.p, st);
      if (s != GF_OK) return s;
      seg_axpy<<<nc, kRedThreads, 0, st>>>(1.0, B->t.p, x, C, B->live.p); ::gf::count_launch();
    } else {
      seg_axpy<<<nc, kRedThreads, 0, st>>>(1.0, B->w.p, x, C, B->live.p); ::gf::count_launch();
    }
    GF_CHECK_LAUNCH();
    GF_CUDA(cudaMemcpyAsync(jc.data(), B->jcnt.p, sizeof(int) * np, cudaMemcpyDeviceToHost, st));
    GF_CUDA(cudaStreamSynchronize(st));
    int mx = 0;
    for (int p = 0; p < np; p++)
      if (live[p]) {
        iters[p] += jc[p];
        mx = std::max(mx, jc[p]);
      }
    steps_total += mx;
  }
  return GF_OK;
}

// Full solve of the batch (vectors in batch space): FP64 GMRES, or FP64
// iterative refinement around an FP32-valued inner GMRES (FP32 SpMV + FP32
// ILU apply with FP64 vectors and accumulation).
static gf_status batch_solve_space(gf_batch* B, const gf_solve_opts& o,
                                   std::vector<gf_solve_stats>& S, cudaStream_t st) {
  const int np = B->np;
  auto t0 = std::chrono::steady_clock::now();
  std::vector<int> live(np, 1), iters, rest;
  std::vector<double> rel;
  S.assign(np, gf_solve_stats{});
  gf_status result = GF_OK;
  if (!o.mixed) {
    result = bgmres<double>(B, B->d_b.p, B->d_x.p, o.restart, o.max_iters, o.rtol, o.side,
                            o.check_every, live, iters, rest, rel, st);
    for (int p = 0; p < np && !iters.empty(); p++) {
      S[p].iterations = iters[p];
      S[p].restarts = rest[p];
      S[p].rel_residual = rel[p];
    }
  } else {
    for (int k = 0; k < np; k++) {
      gf_bsr* A = B->mats[k];
      const size_t n36 = (size_t)36 * A->a->pat.nnz();
      if (A->vals32.n != n36) {
        GF_CUDA(A->vals32.alloc(n36));
        gf_status s2 = upload_desc(B);
        if (s2 != GF_OK) return s2;
      }
      convert_kernel<float><<<(unsigned)((n36 + 255) / 256), 256, 0, st>>>(n36, A->vals.p,
                                                                           A->vals32.p); ::gf::count_launch();
    }
    GF_CHECK_LAUNCH();
    gf_status s = ensure_gmres(B, o.restart);
    if (s != GF_OK) return s;
    const Chunks C = B->chunks();
    const int nc = B->nchunks, pb = (np + 127) / 128;
    std::vector<double> bn(np), rn(np);
    seg_sumsq<<<nc, kRedThreads, 0, st>>>(B->d_b.p, C, nullptr, B->pnorm.p); ::gf::count_launch();
    seg_norm_out<<<pb, 128, 0, st>>>(B->pnorm.p, C, np, nullptr, B->bnorm.p); ::gf::count_launch();
    GF_CUDA(cudaMemcpyAsync(bn.data(), B->bnorm.p, sizeof(double) * np, cudaMemcpyDeviceToHost,
                            st));
    GF_CUDA(cudaStreamSynchronize(st));
    for (int p = 0; p < np; p++)
      if (bn[p] == 0.0) bn[p] = 1.0;
    std::vector<int> tot_it(np, 0), tot_rs(np, 0), nref(np, 0);
    std::vector<double> relv(np, 1.0);
    int refine = 0;
    while (true) {
      GF_CUDA(cudaMemcpyAsync(B->live2.p, live.data(), sizeof(int) * np, cudaMemcpyHostToDevice,
                              st));
      seg_copy<<<nc, kRedThreads, 0, st>>>(B->d_b.p, B->d.p, C, B->live2.p); ::gf::count_launch();
      s = bspmv<double>(B, B->live2.p, B->d_x.p, -1.0, 1.0, B->d.p, st);
      if (s != GF_OK) return s;
      seg_sumsq<<<nc, kRedThreads, 0, st>>>(B->d.p, C, B->live2.p, B->pnorm.p); ::gf::count_launch();
      seg_norm_out<<<pb, 128, 0, st>>>(B->pnorm.p, C, np, B->live2.p, B->norms.p); ::gf::count_launch();
      GF_CUDA(cudaMemcpyAsync(rn.data(), B->norms.p, sizeof(double) * np,
                              cudaMemcpyDeviceToHost, st));
      GF_CUDA(cudaStreamSynchronize(st));
      bool any = false;
      for (int p = 0; p < np; p++) {
        if (!live[p]) continue;
        relv[p] = rn[p] / bn[p];
        if (!std::isfinite(relv[p])) {
          result = GF_NAN;
          live[p] = 0;
        } else if (relv[p] <= o.rtol) {
          live[p] = 0;
        } else {
          any = true;
        }
      }
      if (!any || refine >= o.max_refine) break;
      int maxit = 0;
      for (int p = 0; p < np; p++)
        if (live[p]) maxit = std::max(maxit, o.max_iters - tot_it[p]);
      if (maxit <= 0) break;
      // inner solve A32 e = r from zero
      GF_CUDA(cudaMemsetAsync(B->e.p, 0, sizeof(double) * B->N, st));
      s = bgmres<float>(B, B->d.p, B->e.p, o.restart, maxit, o.inner_rtol, o.side,
                        o.check_every, live, iters, rest, rel, st);
      if (s != GF_OK) {
        result = s;
        break;
      }
      GF_CUDA(cudaMemcpyAsync(B->live2.p, live.data(), sizeof(int) * np, cudaMemcpyHostToDevice,
                              st));
      seg_axpy<<<nc, kRedThreads, 0, st>>>(1.0, B->e.p, B->d_x.p, C, B->live2.p); ::gf::count_launch();
      GF_CHECK_LAUNCH();
      for (int p = 0; p < np; p++)
        if (live[p]) {
          tot_it[p] += iters[p];
          tot_rs[p] += rest[p];
          nref[p]++;
        }
      refine++;
    }
    for (int p = 0; p < np; p++) {
      S[p].iterations = tot_it[p];
      S[p].restarts = tot_rs[p];
      S[p].refinements = nref[p];
      S[p].rel_residual = relv[p];
    }
  }
  const double ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  for (int p = 0; p < np; p++) {
    S[p].time_ms = ms;
    // hard failures (NaN, CUDA, timeout) mark every problem; otherwise each
    // problem's status is its own convergence
    gf_status sp = result;
    if (sp == GF_OK || sp == GF_NOT_CONVERGED)
      sp = (S[p].rel_residual <= o.rtol) ? GF_OK : GF_NOT_CONVERGED;
    S[p].status = sp;
    if (result == GF_OK && sp != GF_OK) result = sp;
  }
  return result;
}

static gf_status batch_create_impl(int n, gf_assembler* const* asms, gf_bsr* const* mats,
                                   gf_precond* const* pcs, gf_batch** out) {
  gf_batch* B = new gf_batch();
  B->np = n;
  B->asms.assign(asms, asms + n);
  B->mats.assign(mats, mats + n);
  B->pcs.assign(pcs, pcs + n);
  gf_status s = batch_build(B);
  if (s != GF_OK) {
    delete B;
    return s;
  }
  *out = B;
  return GF_OK;
}

static gf_status self_batch(gf_precond* p, gf_bsr* A) {
  if (p->self && p->self->mats[0] == A) return GF_OK;
  if (p->self) {
    delete p->self;
    p->self = nullptr;
  }
  gf_assembler* a = p->a;
  return batch_create_impl(1, &a, &A, &p, &p->self);
}

static bool opts_ok(const gf_solve_opts& o) {
  return o.restart >= 1 && o.restart <= 1000 && o.max_iters >= 1 && o.rtol > 0.0 &&
         o.check_every >= 1 && (o.side == 0 || o.side == 1) && o.max_refine >= 0 &&
         (!o.mixed || o.inner_rtol > 0.0);
}

}  // namespace gf

// ------------------------------------------------------------------ C ABI
extern "C" {

gf_status gf_precond_create(gf_assembler* a, int32_t fill_level, int32_t precision,
                            gf_precond** out) {
  return gf_precond_create_ex(a, fill_level, precision, GF_SWEEP_AUTO, out);
}

gf_status gf_precond_create_ex(gf_assembler* a, int32_t fill_level, int32_t precision,
                               int32_t sweep, gf_precond** out) {
  if (!a || !out || fill_level < 0 || (precision != GF_PREC_FP64 && precision != GF_PREC_FP32) ||
      sweep < GF_SWEEP_AUTO || sweep > GF_SWEEP_LEVEL)
    return GF_INVALID_ARG;
  const auto t_setup = std::chrono::steady_clock::now();
  gf_precond* p = new gf_precond();
  p->a = a;
  p->fill = fill_level;
  p->prec = precision;
  {
    const auto t0 = std::chrono::steady_clock::now();
    if (fill_level == 0) {
      p->pat = a->pat;
    } else {
      p->sym_gpu = iluk_pattern_gpu(a->pat, fill_level, p->pat) ? 1 : 0;
      if (!p->sym_gpu) p->pat = iluk_pattern(a->pat, fill_level);
    }
    p->sym_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  const int n = a->nnodes;
  std::vector<int32_t> diag(n), amap(a->pat.nnz());
  for (int i = 0; i < n; i++) {
    const int32_t* b0 = p->pat.cols.data() + p->pat.rowp[i];
    const int32_t* b1 = p->pat.cols.data() + p->pat.rowp[i + 1];
    diag[i] = (int32_t)(std::lower_bound(b0, b1, i) - p->pat.cols.data());
    for (int jp = a->pat.rowp[i]; jp < a->pat.rowp[i + 1]; jp++) {
      const int32_t* f = std::lower_bound(b0, b1, a->pat.cols[jp]);
      amap[jp] = (int32_t)(f - p->pat.cols.data());
    }
  }
  p->nlevL = levels(p->pat, true, p->lvL);
  p->nlevU = levels(p->pat, false, p->lvU);
  auto group = [n](const std::vector<int32_t>& lv, int nl, std::vector<int32_t>& ptr,
                   std::vector<int32_t>& rows) {
    ptr.assign(nl + 1, 0);
    for (int i = 0; i < n; i++) ptr[lv[i] + 1]++;
    for (int l = 0; l < nl; l++) ptr[l + 1] += ptr[l];
    rows.resize(n);
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int i = 0; i < n; i++) rows[fill[lv[i]]++] = i;
  };
  std::vector<int32_t> lptr, lrows;
  group(p->lvL, p->nlevL, lptr, lrows);
  cudaError_t e = cudaSuccess;
  auto up = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  up(p->d_rowp.upload(p->pat.rowp));
  up(p->d_cols.upload(p->pat.cols));
  up(p->d_diag.upload(diag));
  up(p->d_amap.upload(amap));
  up(p->d_levLptr.upload(lptr));
  up(p->d_levLrows.upload(lrows));
  up(p->d_lu.alloc((size_t)36 * p->pat.nnz()));
  up(p->d_done.alloc((size_t)n));
  {
    std::vector<int32_t> ord;
    step_order(p->pat, diag, p->lvL, ord);
    up(p->d_ord.upload(ord));
  }
  if (e == cudaSuccess) up(cudaMemset(p->d_done.p, 0, sizeof(int32_t) * (size_t)n));
  // block updates of one factorization: per step (i, k) the block L_ik and
  // one update per block of U(k)
  p->fwork = 0;
  for (int i = 0; i < n; i++)
    for (int kp = p->pat.rowp[i]; kp < diag[i]; kp++) {
      const int k = p->pat.cols[kp];
      p->fwork += p->pat.rowp[k + 1] - diag[k];
    }
  for (int w = 0; w < 2 && e == cudaSuccess; w++) {
    bool df = false;
    if (sweep == GF_SWEEP_DATAFLOW) e = build_df(p, diag, w == 1, &df);
    if (e == cudaSuccess && !df) {
      if (sweep == GF_SWEEP_DATAFLOW) {
        set_last_error_text("gf_precond_create_ex: the dataflow sweep's ring and stages of this "
                            "factor do not fit one CTA's shared memory");
        delete p;
        return GF_INVALID_ARG;
      }
      e = build_tri(p, diag, w == 1);
    }
  }
  auto fits = [&](int w) {
    return sweep_smem(p, w) <= kSweepSmemMax;
  };
  if (e == cudaSuccess && !(fits(0) && fits(1))) {
    set_last_error_text("gf_precond_create: the ILU(" + std::to_string(fill_level) +
                        ") factor has rows too long for the triangular sweep's "
                        "shared-memory stage; use a lower fill level");
    delete p;
    return GF_INVALID_ARG;  // a factor row longer than one staging buffer
  }
  if (e != cudaSuccess) {
    set_last_error("gf_precond_create", e);
    delete p;
    return e == cudaErrorMemoryAllocation ? GF_OOM : GF_CUDA_ERROR;
  }
  p->setup_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_setup).count();
  *out = p;
  return GF_OK;
}

gf_status gf_precond_destroy(gf_precond* p) {
  if (p && p->self) delete p->self;
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

gf_status gf_precond_setup_info(const gf_precond* p, int32_t* symbolic_on_gpu, double* symbolic_ms,
                                double* setup_ms) {
  if (!p) return GF_INVALID_ARG;
  if (symbolic_on_gpu) *symbolic_on_gpu = p->sym_gpu;
  if (symbolic_ms) *symbolic_ms = p->sym_ms;
  if (setup_ms) *setup_ms = p->setup_ms;
  return GF_OK;
}

gf_status gf_precond_layout(const gf_precond* p, int32_t* nsplit_L, int32_t* nsplit_U,
                            int32_t* fac_ctas, int32_t* chunks_L, int32_t* chunks_U) {
  if (!p) return GF_INVALID_ARG;
  if (nsplit_L) *nsplit_L = p->tri[0].nsplit;
  if (nsplit_U) *nsplit_U = p->tri[1].nsplit;
  if (fac_ctas) *fac_ctas = fac_ctas_alone(p);
  if (chunks_L) *chunks_L = p->tri[0].nch;
  if (chunks_U) *chunks_U = p->tri[1].nch;
  return GF_OK;
}

gf_status gf_precond_sweeps(const gf_precond* p, int32_t* kind_L, int32_t* kind_U,
                            int32_t* ring_L, int32_t* ring_U) {
  if (!p) return GF_INVALID_ARG;
  auto kind = [](const gf_precond::Tri& t) {
    return t.kind == TRI_DATAFLOW ? GF_SWEEP_DATAFLOW : GF_SWEEP_LEVEL;
  };
  if (kind_L) *kind_L = kind(p->tri[0]);
  if (kind_U) *kind_U = kind(p->tri[1]);
  if (ring_L) *ring_L = p->tri[0].ring;
  if (ring_U) *ring_U = p->tri[1].ring;
  return GF_OK;
}

gf_status gf_precond_status(gf_precond* p, void* stream) {
  if (!p) return GF_INVALID_ARG;
  if (!p->self) return GF_OK;  // nothing has run
  SweepCtl h;
  gf_status s = read_ctl(p->self, as_stream(stream), &h);
  if (s != GF_OK) return s;
  return ctl_status(h);
}

gf_status gf_test_set_waits(unsigned long long wait_ns, int32_t skip_meetings) {
  const unsigned long long w = wait_ns ? wait_ns : kWaitNs;
  const int k = skip_meetings ? 1 : 0;
  GF_CUDA(cudaMemcpyToSymbol(g_wait_ns, &w, sizeof(w)));
  GF_CUDA(cudaMemcpyToSymbol(g_skip_meet, &k, sizeof(k)));
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

gf_status gf_precond_factor(gf_precond* p, gf_bsr* A, void* stream) {
  if (!p || !A || A->a != p->a) return GF_INVALID_ARG;
  gf_status s = self_batch(p, A);
  if (s != GF_OK) return s;
  return batch_factor(p->self, as_stream(stream));
}

gf_status gf_precond_apply(gf_precond* p, const double* d_r, double* d_z, void* stream) {
  if (!p || !d_r || !d_z || !p->self) return GF_INVALID_ARG;
  cudaStream_t st = as_stream(stream);
  gf_batch* B = p->self;
  gf_status s = bprecond<double>(B, nullptr, d_r, B->d_x.p, st);
  if (s != GF_OK) return s;
  GF_CUDA(cudaMemcpyAsync(d_z, B->d_x.p, sizeof(double) * B->N, cudaMemcpyDeviceToDevice, st));
  return GF_OK;
}

// ---- preconditioner apply without allocation --------------------------
// The intermediate vector of gf_precond_apply_noalloc. One array per device
// for the whole process; its address on a device is looked up once, by the
// first call made with that device current.
static __device__ __align__(256) double g_noalloc_y[GF_NOALLOC_MAX_DOUBLES];
static constexpr int kNoAllocDevices = 64;
static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[kNoAllocDevices] = {};

gf_status gf_precond_apply_noalloc(gf_precond* p, const double* d_r, double* d_z, void* stream) {
  if (!p || !d_r || !d_z || !p->self) return GF_INVALID_ARG;
  gf_batch* B = p->self;
  const size_t need = (size_t)6 * p->pat.n;
  if (need > (size_t)GF_NOALLOC_MAX_DOUBLES) {
    set_last_error_text("gf_precond_apply_noalloc: the problem needs " + std::to_string(need) +
                        " doubles of scratch, more than the fixed " +
                        std::to_string(GF_NOALLOC_MAX_DOUBLES));
    return GF_INVALID_ARG;
  }
  int dev = 0;
  GF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocDevices) {
    set_last_error_text("gf_precond_apply_noalloc: device index " + std::to_string(dev) +
                        " is above the " + std::to_string(kNoAllocDevices) +
                        " devices this entry point supports");
    return GF_INVALID_ARG;
  }
  double* y = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* a = nullptr;
      GF_CUDA(cudaGetSymbolAddress(&a, g_noalloc_y));
      g_noalloc_ptr[dev] = static_cast<double*>(a);
    }
    y = g_noalloc_ptr[dev];
  }
  if (!sweeps_fit(B)) {
    set_last_error_text("gf_precond_apply_noalloc: the sweeps need more shared memory than a "
                        "CTA has");
    return GF_INVALID_ARG;
  }
  // the same two sweeps as gf_precond_apply; y in the fixed array and z
  // written straight into d_z (a batch of one starts at offset 0)
  const gf_status s = p->prec == GF_PREC_FP32
                          ? bsweeps<float>(B, nullptr, d_r, y, d_z, as_stream(stream), false)
                          : bsweeps<double>(B, nullptr, d_r, y, d_z, as_stream(stream), false);
  return s;
}

gf_status gf_timing_enable(int32_t enable) {
  std::lock_guard<std::mutex> lk(g_timing.mu);
  GF_CUDA(timing_drain_locked());
  g_timing.ms = 0.0;
  g_timing.launches = 0;
  if (enable && !g_timing.d_bytes) {
    void* p = nullptr;
    GF_CUDA(cudaMalloc(&p, sizeof(unsigned long long)));
    g_timing.d_bytes = static_cast<unsigned long long*>(p);
  }
  if (g_timing.d_bytes) GF_CUDA(cudaMemset(g_timing.d_bytes, 0, sizeof(unsigned long long)));
  g_timing.on = enable != 0;
  return GF_OK;
}

gf_status gf_timing_read(double* sweep_ms, long long* sweep_launches, double* sweep_bytes) {
  std::lock_guard<std::mutex> lk(g_timing.mu);
  GF_CUDA(timing_drain_locked());
  unsigned long long b = 0;
  if (g_timing.d_bytes)
    GF_CUDA(cudaMemcpy(&b, g_timing.d_bytes, sizeof(b), cudaMemcpyDeviceToHost));
  if (sweep_ms) *sweep_ms = g_timing.ms;
  if (sweep_launches) *sweep_launches = g_timing.launches;
  if (sweep_bytes) *sweep_bytes = (double)b;
  return GF_OK;
}

void gf_solve_opts_default(gf_solve_opts* o) {
  if (!o) return;
  o->restart = 50;
  o->max_iters = 5000;
  o->rtol = 1e-8;
  o->side = 1;
  o->mixed = 0;
  o->inner_rtol = 1e-4;
  o->max_refine = 30;
  o->check_every = 25;
}

gf_status gf_batch_create(int32_t n, gf_assembler* const* asms, gf_bsr* const* mats,
                          gf_precond* const* pcs, gf_batch** out) {
  if (n <= 0 || !asms || !mats || !pcs || !out) return GF_INVALID_ARG;
  for (int k = 0; k < n; k++)
    if (!asms[k] || !mats[k] || !pcs[k] || mats[k]->a != asms[k] || pcs[k]->a != asms[k])
      return GF_INVALID_ARG;
  return batch_create_impl(n, asms, mats, pcs, out);
}

gf_status gf_batch_destroy(gf_batch* b) {
  delete b;
  return GF_OK;
}

gf_status gf_batch_assemble(gf_batch* B, void* stream) {
  return gf_batch_assemble_ex(B, nullptr, stream);
}

gf_status gf_batch_assemble_ex(gf_batch* B, const double* const* d_thick, void* stream) {
  if (!B) return GF_INVALID_ARG;
  std::vector<double*> values(B->np);
  for (int k = 0; k < B->np; k++) values[k] = B->mats[k]->vals.p;
  return batch_assemble(B->basm, B->asms, values, d_thick, GF_ASSEMBLE_FUSE_BCS | B->scatter,
                        as_stream(stream));
}

gf_status gf_batch_set_scatter(gf_batch* B, int32_t flags) {
  if (!B || (flags != 0 && flags != GF_ASSEMBLE_ATOMIC)) return GF_INVALID_ARG;
  B->scatter = flags;
  return GF_OK;
}

gf_status gf_batch_factor(gf_batch* B, void* stream) {
  if (!B) return GF_INVALID_ARG;
  return batch_factor(B, as_stream(stream));
}

gf_status gf_batch_solve(gf_batch* B, const double* const* d_b, double* const* d_x,
                         const gf_solve_opts* opts, gf_solve_stats* stats, void* stream) {
  if (!B || !d_b || !d_x) return GF_INVALID_ARG;
  gf_solve_opts o;
  gf_solve_opts_default(&o);
  if (opts) o = *opts;
  if (!opts_ok(o)) return GF_INVALID_ARG;
  for (int k = 0; k < B->np; k++)
    if (!d_b[k] || !d_x[k]) return GF_INVALID_ARG;
  cudaStream_t st = as_stream(stream);
  std::vector<PermEntry> eb(B->np), ex(B->np), eo(B->np);
  int maxn = 0;
  for (int k = 0; k < B->np; k++) {
    gf_assembler* a = B->asms[k];
    eb[k] = PermEntry{a->d_perm.p, a->nnodes, B->offs[k], d_b[k], B->d_b.p};
    ex[k] = PermEntry{a->d_perm.p, a->nnodes, B->offs[k], d_x[k], B->d_x.p};
    eo[k] = PermEntry{a->d_perm.p, a->nnodes, B->offs[k], B->d_x.p, d_x[k]};
    maxn = std::max(maxn, a->nnodes);
  }
  GF_CUDA(cudaMemcpyAsync(B->d_perm_b.p, eb.data(), sizeof(PermEntry) * B->np,
                          cudaMemcpyHostToDevice, st));
  GF_CUDA(cudaMemcpyAsync(B->d_perm_x.p, ex.data(), sizeof(PermEntry) * B->np,
                          cudaMemcpyHostToDevice, st));
  GF_CUDA(cudaMemcpyAsync(B->d_perm_out.p, eo.data(), sizeof(PermEntry) * B->np,
                          cudaMemcpyHostToDevice, st));
  const dim3 grid((unsigned)std::max(1, std::min(64, (6 * maxn + 255) / 256)), (unsigned)B->np);
  bpermute<<<grid, 256, 0, st>>>(B->d_perm_b.p, 0); ::gf::count_launch();
  bpermute<<<grid, 256, 0, st>>>(B->d_perm_x.p, 0); ::gf::count_launch();
  GF_CHECK_LAUNCH();
  std::vector<gf_solve_stats> S;
  gf_status s = batch_solve_space(B, o, S, st);
  bpermute<<<grid, 256, 0, st>>>(B->d_perm_out.p, 1); ::gf::count_launch();
  GF_CHECK_LAUNCH();
  // every sweep of the solve has run: read and clear the device status
  SweepCtl h;
  gf_status sc = read_ctl(B, st, &h);
  if (sc == GF_OK) sc = ctl_status(h);
  if (sc != GF_OK) {
    s = sc;
    for (auto& x : S) x.status = sc;
  }
  if (stats)
    for (int k = 0; k < B->np && k < (int)S.size(); k++) stats[k] = S[k];
  return s;
}

gf_status gf_gmres_solve(gf_assembler* a, gf_bsr* A, gf_precond* p, const double* d_b,
                         double* d_x, const gf_solve_opts* opts, gf_solve_stats* stats,
                         void* stream) {
  if (!a || !A || !p || !d_b || !d_x || A->a != a || p->a != a) return GF_INVALID_ARG;
  gf_status s = self_batch(p, A);
  if (s != GF_OK) return s;
  return gf_batch_solve(p->self, &d_b, &d_x, opts, stats, stream);
}

gf_status gf_direct_solve(gf_assembler* a, gf_bsr* A, const double* d_b, double* d_x,
                          gf_solve_stats* stats, void* stream) {
  if (!a || !A || !d_b || !d_x || A->a != a) return GF_INVALID_ARG;
  gf_precond* p = nullptr;
  gf_status s = gf_precond_create(a, GF_FILL_FULL, GF_PREC_FP64, &p);
  if (s != GF_OK) return s;
  s = gf_precond_factor(p, A, stream);
  gf_solve_stats st{};
  if (s == GF_OK) {
    // x = (LU)^{-1} b is the first step of right-preconditioned GMRES from
    // x = 0 with the complete factor; the further steps are FP64 iterative
    // refinement, run until the residual stops falling (at most 4 steps)
    const size_t n = (size_t)6 * a->nnodes;
    cudaError_t e = cudaMemsetAsync(d_x, 0, sizeof(double) * n, as_stream(stream));
    if (e != cudaSuccess) {
      set_last_error("gf_direct_solve", e);
      s = GF_CUDA_ERROR;
    } else {
      gf_solve_opts o;
      gf_solve_opts_default(&o);
      o.restart = 4;
      o.max_iters = 4;
      o.rtol = 1e-15;
      o.side = 1;
      s = gf_gmres_solve(a, A, p, d_b, d_x, &o, &st, stream);
      if (s == GF_NOT_CONVERGED) s = GF_OK;  // a direct solve has no tolerance to miss
      st.status = s;
    }
  }
  if (stats) *stats = st;
  gf_precond_destroy(p);
  return s;
}

gf_status gf_bsr_spmv(gf_bsr* m, double alpha, const double* d_x, double beta, double* d_y,
                      void* stream) {
  if (!m || !d_x || !d_y) return GF_INVALID_ARG;
  gf_assembler* a = m->a;
  cudaStream_t st = as_stream(stream);
  if (!m->desc.p) {
    ProbDev d{};
    d.n = a->nnodes;
    d.off = 0;
    d.rowp = a->d_rowp.p;
    d.cols = a->d_cols.p;
    d.A64 = m->vals.p;
    GF_CUDA(m->desc.upload(&d, 1));
    GF_CUDA(m->rowprob.alloc(a->nnodes));
    GF_CUDA(cudaMemset(m->rowprob.p, 0, sizeof(int32_t) * a->nnodes));
  }
  bspmv_kernel<double><<<(a->nnodes + 7) / 8, 256, 0, st>>>(a->nnodes, m->rowprob.p, m->desc.p,
                                                            nullptr, d_x, alpha, beta, d_y); ::gf::count_launch();
  GF_CHECK_LAUNCH();
  return GF_OK;
}

}  // extern "C"
