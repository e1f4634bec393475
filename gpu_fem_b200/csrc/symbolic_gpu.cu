// ILU(k) symbolic factorization on the GPU: the level-of-fill rule of
// computeILUk (include/linalg/bsr_utils.h:678-807), one warp per row, rows
// scheduled as a dataflow (a row waits only for the rows whose final
// pattern it merges).
//
// Row i keeps the levels of its candidate columns in a dense byte window of
// shared memory over [lo_i, hi_i]: lo_i is the first column of A's row i (or
// i), and hi_i = max(last column of A's row i, i, hi_k for lo_i <= k < i)
// bounds every column the fill can reach (fill into row i comes from the
// upper part of rows k in [lo_i, i), whose columns are bounded by hi_k).
// Starting from A's entries and the diagonal at level 0, the warp takes the
// row's lower columns k in ascending order (a ballot over 32 window entries
// finds the next one at level <= k_fill), waits until row k's pattern is
// final, and for every upper entry (j, lev_kj) of row k lowers the level of
// column j to lev_ik + lev_kj + 1 when that is <= k_fill (adding j when it
// was absent): exactly the host rule, where an existing entry takes the
// minimum and a new one enters only within the fill level. The row's
// entries are then compacted in column order into its output slot (columns,
// levels, count, position of the diagonal) and published with a release
// flag. Rows are taken in index order, so every row a warp waits for was
// taken earlier by a running warp; each wait is bounded.
#include <algorithm>
#include <vector>

#include "gf_internal.h"

namespace gf {

namespace {

constexpr int kSymWarps = 8;
constexpr int kSymWin = 4096;  // window bytes per warp
constexpr unsigned long long kSymWaitNs = 2000000000ull;

__device__ __forceinline__ unsigned long long sym_timer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ int sym_ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__global__ void __launch_bounds__(kSymWarps * 32)
    iluk_sym_kernel(int n, const int32_t* __restrict__ arowp, const int32_t* __restrict__ acols,
                    const int32_t* __restrict__ lo, const int32_t* __restrict__ hi,
                    const int64_t* __restrict__ off, int32_t* ocols, uint8_t* olev, int32_t* ocnt,
                    int32_t* odiag, int* done, int* counter, int fill, int* status) {
  __shared__ uint8_t swin[kSymWarps][kSymWin];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t* L = swin[warp];
  for (int t = lane; t < kSymWin; t += 32) L[t] = 255;
  __syncwarp();
  const int fill8 = fill < 254 ? fill : 254;  // levels above 254 only occur with fill >= 254
  int i = lane == 0 ? atomicAdd(counter, 1) : 0;
  i = __shfl_sync(0xffffffffu, i, 0);
  while (i < n) {
    const int inext = lane == 0 ? atomicAdd(counter, 1) : 0;
    const int l0 = lo[i], win = hi[i] - l0 + 1;
    for (int t = arowp[i] + lane; t < arowp[i + 1]; t += 32) L[acols[t] - l0] = 0;
    if (lane == 0) L[i - l0] = 0;
    __syncwarp();
    bool ok = true;
    for (int pos = l0; pos < i;) {
      const int c = pos + lane;
      const bool cand = c < i && L[c - l0] <= fill8;
      const unsigned m = __ballot_sync(0xffffffffu, cand);
      if (!m) {
        pos += 32;
        continue;
      }
      const int k = pos + __ffs(m) - 1;
      const int clev = L[k - l0];
      int rdy = 1;
      if (lane == 0) {
        if (sym_ld_relaxed(done + k) != 1) {
          const unsigned long long t0 = sym_timer();
          while (sym_ld_relaxed(done + k) != 1) {
            if (sym_ld_relaxed(status) != 0 || sym_timer() - t0 > kSymWaitNs) {
              atomicOr(status, 1);
              rdy = 0;
              break;
            }
          }
        }
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
      }
      rdy = __shfl_sync(0xffffffffu, rdy, 0);
      __syncwarp();
      if (!rdy) {
        ok = false;
        break;
      }
      const int64_t ko = off[k];
      const int kd = odiag[k], kc = ocnt[k];
      for (int t = kd + 1 + lane; t < kc; t += 32) {
        const int j = ocols[ko + t];
        const int nl = clev + (int)olev[ko + t] + 1;
        if (nl <= fill) {
          const uint8_t v = (uint8_t)(nl < 254 ? nl : 254);
          if (v < L[j - l0]) L[j - l0] = v;
        }
      }
      __syncwarp();
      pos = k + 1;
    }
    if (!ok) break;
    // compact the row in column order, resetting the window behind
    int cnt = 0, dpos = -1;
    const int64_t oi = off[i];
    for (int base = 0; base < win; base += 32) {
      const int t = base + lane;
      const uint8_t v = t < win ? L[t] : (uint8_t)255;
      const bool present = v != 255;
      const unsigned m = __ballot_sync(0xffffffffu, present);
      const int at = cnt + __popc(m & ((1u << lane) - 1u));
      if (present) {
        ocols[oi + at] = l0 + t;
        olev[oi + at] = v;
      }
      const unsigned dm = __ballot_sync(0xffffffffu, present && l0 + t == i);
      if (dm) dpos = cnt + __popc(m & ((1u << (__ffs(dm) - 1)) - 1u));
      cnt += __popc(m);
      if (t < win) L[t] = 255;
    }
    if (lane == 0) {
      ocnt[i] = cnt;
      odiag[i] = dpos;
    }
    __threadfence();
    __syncwarp();
    if (lane == 0) asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(done + i), "r"(1) : "memory");
    i = __shfl_sync(0xffffffffu, inext, 0);
  }
}

// one warp per row: the row's entries from its slot into the compact array
__global__ void iluk_sym_compact(int n, const int64_t* __restrict__ off,
                                 const int32_t* __restrict__ rowp, const int32_t* __restrict__ ocols,
                                 int32_t* cols) {
  const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int c = rowp[i + 1] - rowp[i];
  for (int t = lane; t < c; t += 32) cols[rowp[i] + t] = ocols[off[i] + t];
}

// ---- node pattern and elemIndMap
// (get_row_col_ptrs, include/linalg/bsr_utils.h:430-476; get_elem_ind_map,
// include/linalg/bsr_utils.h:809-870)
constexpr int kNodeCand = 256;  // candidate neighbours of a node (4 per incident element)

__global__ void node_incidence(int nelem, const int32_t* __restrict__ conn, int32_t* cnt) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nelem) return;
  for (int a = 0; a < 4; a++) atomicAdd(&cnt[conn[4 * e + a]], 1);
}

__global__ void node_elements(int nelem, const int32_t* __restrict__ conn,
                              const int32_t* __restrict__ start, int32_t* cursor, int32_t* elems) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nelem) return;
  for (int a = 0; a < 4; a++) {
    const int v = conn[4 * e + a];
    elems[start[v] + atomicAdd(&cursor[v], 1)] = e;
  }
}

// One warp per node: the nodes of its elements, deduplicated and sorted by
// rank (a candidate's position is the number of distinct smaller ones).
// rowp == nullptr: count only.
__global__ void __launch_bounds__(256)
    node_rows(int nnodes, const int32_t* __restrict__ conn, const int32_t* __restrict__ start,
              const int32_t* __restrict__ elems, int32_t* cnt, const int32_t* __restrict__ rowp,
              int32_t* cols) {
  __shared__ int32_t cand[8][kNodeCand];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * 8 + warp;
  if (i >= nnodes) return;
  int32_t* cd = cand[warp];
  const int e0 = start[i], m = 4 * (start[i + 1] - e0);
  for (int t = lane; t < m; t += 32) cd[t] = conn[4 * elems[e0 + t / 4] + t % 4];
  __syncwarp();
  int nuniq = 0;
  for (int t0 = 0; t0 < m; t0 += 32) {
    const int t = t0 + lane;
    bool first = t < m;
    int pos = 0;
    if (first) {
      const int v = cd[t];
      for (int s = 0; s < t && first; s++) first = cd[s] != v;
      if (first && rowp)
        for (int s = 0; s < m; s++) {
          const int w = cd[s];
          if (w < v) {
            bool f2 = true;
            for (int u = 0; u < s && f2; u++) f2 = cd[u] != w;
            pos += f2 ? 1 : 0;
          }
        }
      if (first && rowp) cols[rowp[i] + pos] = v;
    }
    nuniq += __popc(__ballot_sync(0xffffffffu, first));
  }
  if (lane == 0 && !rowp) cnt[i] = nuniq;
}

// 16 entries per element: slot of block (perm[node a], perm[node b]).
__global__ void elem_map_kernel(int nelem, const int32_t* __restrict__ conn,
                                const int32_t* __restrict__ perm, const int32_t* __restrict__ rowp,
                                const int32_t* __restrict__ cols, int32_t* map) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)16 * nelem) return;
  const int e = (int)(t / 16), a = (int)(t % 16) / 4, b = (int)(t % 4);
  const int r = perm[conn[4 * e + a]], c = perm[conn[4 * e + b]];
  int lo = rowp[r], hi = rowp[r + 1];
  const int end = hi;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (cols[mid] < c)
      lo = mid + 1;
    else
      hi = mid;
  }
  map[t] = (lo < end && cols[lo] == c) ? lo : -1;
}

}  // namespace

bool pattern_from_conn_gpu(int nelem, int nnodes, const int32_t* conn, Pattern& out) {
  if (nelem <= 0 || nnodes <= 0) return false;
  DevBuf<int32_t> d_conn, d_cnt, d_start, d_cursor, d_elems, d_rows, d_rowp, d_cols;
  cudaError_t e = cudaSuccess;
  auto up = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  up(d_conn.upload(conn, (size_t)4 * nelem));
  up(d_cnt.alloc(nnodes));
  if (e == cudaSuccess) up(cudaMemset(d_cnt.p, 0, sizeof(int32_t) * nnodes));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const unsigned eb = (unsigned)((nelem + 255) / 256), nb = (unsigned)((nnodes + 7) / 8);
  count_launch();
  node_incidence<<<eb, 256>>>(nelem, d_conn.p, d_cnt.p);
  std::vector<int32_t> cnt(nnodes), start(nnodes + 1, 0);
  up(cudaMemcpy(cnt.data(), d_cnt.p, sizeof(int32_t) * nnodes, cudaMemcpyDeviceToHost));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  for (int i = 0; i < nnodes; i++) {
    if (4 * cnt[i] > kNodeCand) return false;  // the host handles such meshes
    start[i + 1] = start[i] + cnt[i];
  }
  up(d_start.upload(start));
  up(d_cursor.alloc(nnodes));
  up(d_elems.alloc((size_t)start[nnodes]));
  if (e == cudaSuccess) up(cudaMemset(d_cursor.p, 0, sizeof(int32_t) * nnodes));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  count_launch();
  node_elements<<<eb, 256>>>(nelem, d_conn.p, d_start.p, d_cursor.p, d_elems.p);
  count_launch();
  node_rows<<<nb, 256>>>(nnodes, d_conn.p, d_start.p, d_elems.p, d_cnt.p, nullptr, nullptr);
  up(cudaMemcpy(cnt.data(), d_cnt.p, sizeof(int32_t) * nnodes, cudaMemcpyDeviceToHost));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  out.n = nnodes;
  out.rowp.assign(nnodes + 1, 0);
  for (int i = 0; i < nnodes; i++) out.rowp[i + 1] = out.rowp[i] + cnt[i];
  up(d_rowp.upload(out.rowp));
  up(d_cols.alloc((size_t)out.rowp[nnodes]));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  count_launch();
  node_rows<<<nb, 256>>>(nnodes, d_conn.p, d_start.p, d_elems.p, d_cnt.p, d_rowp.p, d_cols.p);
  out.cols.resize(out.rowp[nnodes]);
  up(cudaGetLastError());
  up(cudaMemcpy(out.cols.data(), d_cols.p, sizeof(int32_t) * out.cols.size(),
                cudaMemcpyDeviceToHost));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return true;
}

bool elem_ind_map_gpu(int nelem, const int32_t* conn, const Pattern& p,
                      const std::vector<int32_t>& perm, std::vector<int32_t>& map) {
  DevBuf<int32_t> d_conn, d_perm, d_rowp, d_cols, d_map;
  cudaError_t e = cudaSuccess;
  auto up = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  up(d_conn.upload(conn, (size_t)4 * nelem));
  up(d_perm.upload(perm));
  up(d_rowp.upload(p.rowp));
  up(d_cols.upload(p.cols));
  up(d_map.alloc((size_t)16 * nelem));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  count_launch();
  elem_map_kernel<<<(unsigned)(((size_t)16 * nelem + 255) / 256), 256>>>(nelem, d_conn.p, d_perm.p,
                                                                       d_rowp.p, d_cols.p, d_map.p);
  map.resize((size_t)16 * nelem);
  up(cudaGetLastError());
  up(cudaMemcpy(map.data(), d_map.p, sizeof(int32_t) * map.size(), cudaMemcpyDeviceToHost));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return true;
}

bool iluk_pattern_gpu(const Pattern& a, int fill, Pattern& out) {
  const int n = a.n;
  if (n == 0) return false;
  // windows [lo_i, hi_i] (range maxima of hi over [lo_i, i) by a segment tree)
  std::vector<int32_t> lo(n), hi(n);
  int size = 1;
  while (size < n) size <<= 1;
  std::vector<int32_t> seg(2 * (size_t)size, -1);
  auto query = [&](int l, int r) {  // max over [l, r)
    int res = -1;
    for (l += size, r += size; l < r; l >>= 1, r >>= 1) {
      if (l & 1) res = std::max(res, seg[l++]);
      if (r & 1) res = std::max(res, seg[--r]);
    }
    return res;
  };
  std::vector<int64_t> off(n + 1, 0);
  for (int i = 0; i < n; i++) {
    const int r0 = a.rowp[i], r1 = a.rowp[i + 1];
    lo[i] = r1 > r0 ? std::min(a.cols[r0], i) : i;
    int h = r1 > r0 ? std::max(a.cols[r1 - 1], i) : i;
    if (lo[i] < i) h = std::max(h, query(lo[i], i));
    hi[i] = h;
    for (int p = i + size; p >= 1; p >>= 1) seg[p] = std::max(seg[p], h);
    if (hi[i] - lo[i] + 1 > kSymWin) return false;  // the host computes such patterns
    off[i + 1] = off[i] + (hi[i] - lo[i] + 1);
  }
  if (off[n] > (int64_t)1 << 31) return false;  // output slots beyond 10 GB: host
  DevBuf<int32_t> d_rowp, d_cols, d_lo, d_hi, d_ocols, d_cnt, d_diag, d_done, d_ctr, d_status;
  DevBuf<int64_t> d_off;
  DevBuf<uint8_t> d_olev;
  cudaError_t e = cudaSuccess;
  auto up = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  up(d_rowp.upload(a.rowp));
  up(d_cols.upload(a.cols));
  up(d_lo.upload(lo));
  up(d_hi.upload(hi));
  up(d_off.upload(off));
  up(d_ocols.alloc((size_t)off[n]));
  up(d_olev.alloc((size_t)off[n]));
  up(d_cnt.alloc(n));
  up(d_diag.alloc(n));
  up(d_done.alloc(n));
  up(d_ctr.alloc(1));
  up(d_status.alloc(1));
  if (e == cudaSuccess) up(cudaMemset(d_done.p, 0, sizeof(int32_t) * n));
  if (e == cudaSuccess) up(cudaMemset(d_ctr.p, 0, sizeof(int32_t)));
  if (e == cudaSuccess) up(cudaMemset(d_status.p, 0, sizeof(int32_t)));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::max(1, std::min(2 * sms, (n + kSymWarps - 1) / kSymWarps));
  count_launch();
  iluk_sym_kernel<<<grid, kSymWarps * 32>>>(n, d_rowp.p, d_cols.p, d_lo.p, d_hi.p, d_off.p,
                                            d_ocols.p, d_olev.p, d_cnt.p, d_diag.p, d_done.p,
                                            d_ctr.p, fill, d_status.p);
  std::vector<int32_t> cnt(n);
  int st = 0;
  up(cudaGetLastError());
  up(cudaMemcpy(&st, d_status.p, sizeof(int), cudaMemcpyDeviceToHost));
  up(cudaMemcpy(cnt.data(), d_cnt.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
  if (e != cudaSuccess || st != 0) {
    cudaGetLastError();
    return false;
  }
  out.n = n;
  out.rowp.assign(n + 1, 0);
  for (int i = 0; i < n; i++) out.rowp[i + 1] = out.rowp[i] + cnt[i];
  DevBuf<int32_t> d_prow, d_pcols;
  up(d_prow.upload(out.rowp));
  up(d_pcols.alloc((size_t)out.rowp[n]));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  count_launch();
  iluk_sym_compact<<<(unsigned)(((size_t)n * 32 + 255) / 256), 256>>>(n, d_off.p, d_prow.p,
                                                                      d_ocols.p, d_pcols.p);
  out.cols.resize(out.rowp[n]);
  up(cudaGetLastError());
  up(cudaMemcpy(out.cols.data(), d_pcols.p, sizeof(int32_t) * out.cols.size(),
                cudaMemcpyDeviceToHost));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return true;
}

}  // namespace gf
