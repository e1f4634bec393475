// CPU ORACLE — test infrastructure only. Imported by tests/, by
// __graft_entry__.smoke() as the checker, and by bench.py's CPU-baseline leg.
// The product (gpu_fem_b200) never links or calls anything in this file.
//
// C entry points over the element restatement in shell_oracle.hpp plus the
// sparse host algorithms of the reference's hot path:
//   pattern        include/linalg/bsr_utils.h:430-476 (get_row_col_ptrs)
//   RCM            include/linalg/reordering_utils.h:189-291
//   elemIndMap     include/linalg/bsr_utils.h:809-870
//   scatter        include/linalg/bsr_mat.h:195-226
//   BCs            include/linalg/bsr_mat.cuh:1-104, include/linalg/vec.h:59-65
//   ILU(k) pattern include/linalg/bsr_utils.h:678-807 (levFill = 0 keeps A's pattern)
//   block ILU(0)   cusparseDbsrilu02 as called at examples/iterative/gmres.cu:426-457
//   trisolves      cusparseDbsrsv2_solve, examples/iterative/gmres.cu:522-532
//   SpMV           cusparseDbsrmv, examples/iterative/gmres.cu:498-509
//   GMRES(m)       examples/iterative/gmres.cu:468-771 with its bugs fixed
//                  (dot length nvars, m+1 basis vectors, restarts).
// Plus restatements of this project's own deterministic scheduling
// (element chunks, chunk/element colouring, first-touch masks, level sets),
// which the CUDA path must reproduce bit-exactly.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "shell_oracle.hpp"

using oracle::ShellData;
using cplx = std::complex<double>;

extern "C" {

// ------------------------------------------------------------- elements
void orc_element_residual(const double* X, const double* u, const ShellData* d, double* res) {
  for (int i = 0; i < 24; i++) res[i] = 0.0;
  oracle::element_residual<double>(*d, X, u, res);
}
void orc_element_jacobian(const double* X, const double* u, const ShellData* d, double* res,
                          double* K) {
  for (int i = 0; i < 24; i++) res[i] = 0.0;
  oracle::element_jacobian<double>(*d, X, u, res, K);
}
double orc_element_energy(const double* X, const double* u, const ShellData* d) {
  return oracle::element_energy<double>(*d, X, u);
}
// Complex-step variants: u = u_re + i u_im (X real).
void orc_element_energy_cs(const double* X, const double* u_re, const double* u_im,
                           const ShellData* d, double* out_re, double* out_im) {
  cplx Xc[12], uc[24];
  for (int i = 0; i < 12; i++) Xc[i] = X[i];
  for (int i = 0; i < 24; i++) uc[i] = cplx(u_re[i], u_im[i]);
  cplx U = oracle::element_energy<cplx>(*d, Xc, uc);
  *out_re = U.real();
  *out_im = U.imag();
}
void orc_element_residual_cs(const double* X, const double* u_re, const double* u_im,
                             const ShellData* d, double* r_re, double* r_im) {
  cplx Xc[12], uc[24], rc[24];
  for (int i = 0; i < 12; i++) Xc[i] = X[i];
  for (int i = 0; i < 24; i++) {
    uc[i] = cplx(u_re[i], u_im[i]);
    rc[i] = 0.0;
  }
  oracle::element_residual<cplx>(*d, Xc, uc, rc);
  for (int i = 0; i < 24; i++) {
    r_re[i] = rc[i].real();
    r_im[i] = rc[i].imag();
  }
}

// ------------------------------------------------------------- pattern
// Block pattern = node adjacency through shared elements, columns ascending,
// diagonal included (get_row_col_ptrs, bsr_utils.h:430-476). Pass colPtr =
// NULL to count only. Returns nnzb.
int orc_bsr_pattern(int nelem, int nnodes, const int* conn, int* rowPtr, int* colPtr) {
  std::vector<std::vector<int>> adj(nnodes);
  for (int e = 0; e < nelem; e++)
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) adj[conn[4 * e + a]].push_back(conn[4 * e + b]);
  int nnz = 0;
  if (rowPtr) rowPtr[0] = 0;
  for (int i = 0; i < nnodes; i++) {
    auto& v = adj[i];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    if (colPtr)
      for (int c : v) colPtr[nnz++] = c;
    else
      nnz += (int)v.size();
    if (rowPtr) rowPtr[i + 1] = nnz;
  }
  return nnz;
}

// TacsComputeRCMLevSetOrder / TacsComputeRCMOrder (reordering_utils.h:189-291):
// BFS level sets from `root`, neighbours in colPtr order, then reversed.
// rcm_vars[old] = new.
int orc_rcm(int n, const int* rowp, const int* cols, int root, int n_iters, int* rcm_vars) {
  if (n_iters < 1) n_iters = 1;
  std::vector<int> levset(n);
  int rvars = 0;
  for (int it = 0; it < n_iters; it++) {
    int start = 0, end = 0;
    for (int k = 0; k < n; k++) rcm_vars[k] = -1;
    int var_num = 0;
    bool done = false;
    while (var_num < n && !done) {
      if (end - start == 0) {
        if (rcm_vars[root] >= 0) {
          int i = 0;
          for (; i < n; i++)
            if (rcm_vars[i] < 0) {
              root = i;
              break;
            }
          if (i >= n) {
            done = true;
            break;
          }
        }
        levset[end] = root;
        rcm_vars[root] = var_num++;
        end++;
      }
      while (start < end) {
        int next = end;
        for (int cur = start; cur < end; cur++) {
          int node = levset[cur];
          for (int j = rowp[node]; j < rowp[node + 1]; j++) {
            int nn = cols[j];
            if (rcm_vars[nn] < 0) {
              rcm_vars[nn] = var_num++;
              levset[next++] = nn;
            }
          }
        }
        start = end;
        end = next;
      }
    }
    for (int i = 0; i < var_num; i++) rcm_vars[levset[i]] = var_num - 1 - i;
    rvars = var_num;
    if (rvars != n) return rvars;
    root = rcm_vars[0];
  }
  return rvars;
}

// Deterministic q-ordering on an RCM order rcm[old] = new (the intent of
// examples/iterative/gmres.cu:159-215 with a fixed seed): bandwidth b =
// max |i - j| of the RCM-ordered pattern (getBandWidth,
// include/linalg/bsr_utils.h:655-670); windows of w = floor(b / pfac)
// consecutive new positions; in each window, positions hi-1 down to lo+1
// each swap their node with position lo + x mod (i - lo + 1), x the next
// output of one std::mt19937_64(seed). out[old] = new.
void orc_qorder(int n, const int* rowp, const int* cols, const int* rcm, double pfac,
                unsigned long long seed, int* out) {
  int bw = 0;
  for (int i = 0; i < n; i++)
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) {
      const int d = rcm[i] - rcm[cols[jp]];
      bw = std::max(bw, d < 0 ? -d : d);
    }
  const double pp = pfac > 0.0 ? pfac : 1.0;
  const int w = std::max(1, (int)((double)bw / pp));
  std::vector<int> at(n);
  for (int i = 0; i < n; i++) at[rcm[i]] = i;
  std::mt19937_64 gen(seed);
  for (int lo = 0; lo < n; lo += w) {
    const int hi = std::min(n, lo + w);
    for (int i = hi - 1; i > lo; i--) {
      const unsigned long long x = gen();
      const int j = lo + (int)(x % (unsigned long long)(i - lo + 1));
      const int t = at[i];
      at[i] = at[j];
      at[j] = t;
    }
  }
  for (int k = 0; k < n; k++) out[at[k]] = k;
}

// Permuted pattern P A P^T with ascending columns; perm[old] = new.
void orc_permute_pattern(int n, const int* rowp, const int* cols, const int* perm,
                         int* rowp2, int* cols2) {
  std::vector<int> iperm(n);
  for (int i = 0; i < n; i++) iperm[perm[i]] = i;
  rowp2[0] = 0;
  int nz = 0;
  for (int I = 0; I < n; I++) {
    int i = iperm[I];
    int s = nz;
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) cols2[nz++] = perm[cols[jp]];
    std::sort(cols2 + s, cols2 + nz);
    rowp2[I + 1] = nz;
  }
}

// get_elem_ind_map (bsr_utils.h:809-870): map[16 e + 4 a + b] = block index
// of (perm[conn[e,a]], perm[conn[e,b]]).
void orc_elem_ind_map(int nelem, const int* conn, const int* rowp, const int* cols,
                      const int* perm, int* map) {
  for (int e = 0; e < nelem; e++)
    for (int a = 0; a < 4; a++) {
      int r = perm[conn[4 * e + a]];
      for (int b = 0; b < 4; b++) {
        int c = perm[conn[4 * e + b]];
        int found = -1;
        for (int jp = rowp[r]; jp < rowp[r + 1]; jp++)
          if (cols[jp] == c) {
            found = jp;
            break;
          }
        map[16 * e + 4 * a + b] = found;
      }
    }
}

// ------------------------------------------------------------- assembly
static void gather_elem(int e, const int* conn, const double* xpts, const double* vars,
                        double X[12], double u[24]) {
  for (int a = 0; a < 4; a++) {
    int n = conn[4 * e + a];
    for (int k = 0; k < 3; k++) X[3 * a + k] = xpts[3 * n + k];
    for (int k = 0; k < 6; k++) u[6 * a + k] = vars ? vars[6 * n + k] : 0.0;
  }
}

// add_jacobian_cpu (base/elem_group.h:121-181) + addElementMatrixValues
// (bsr_mat.h:195-226): values[36 map + 6r + c] += K[24(6a+r) + 6b + c].
// res (natural node order) += R_e. Element matrices are computed in parallel
// (nthreads), then scattered serially in element order.
void orc_assemble_jacobian(int nelem, const int* conn, const double* xpts, const double* vars,
                           const ShellData* data, const int* elem_ind_map, double* values,
                           double* res, int nthreads) {
  const int chunk = 4096;
  std::vector<double> Ks((size_t)chunk * 576), Rs((size_t)chunk * 24);
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#endif
  for (int e0 = 0; e0 < nelem; e0 += chunk) {
    int ne = std::min(chunk, nelem - e0);
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static)
#endif
    for (int k = 0; k < ne; k++) {
      double X[12], u[24];
      gather_elem(e0 + k, conn, xpts, vars, X, u);
      double* R = &Rs[(size_t)k * 24];
      for (int i = 0; i < 24; i++) R[i] = 0.0;
      oracle::element_jacobian<double>(data[e0 + k], X, u, R, &Ks[(size_t)k * 576]);
    }
    for (int k = 0; k < ne; k++) {
      int e = e0 + k;
      const double* K = &Ks[(size_t)k * 576];
      for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
          double* v = &values[36 * (size_t)elem_ind_map[16 * e + 4 * a + b]];
          for (int r = 0; r < 6; r++)
            for (int c = 0; c < 6; c++) v[6 * r + c] += K[24 * (6 * a + r) + 6 * b + c];
        }
      if (res)
        for (int a = 0; a < 4; a++) {
          int n = conn[4 * e + a];
          for (int k2 = 0; k2 < 6; k2++) res[6 * n + k2] += Rs[(size_t)k * 24 + 6 * a + k2];
        }
    }
  }
}

// add_residual_cpu (base/elem_group.h:40-79), natural node order.
void orc_assemble_residual(int nelem, const int* conn, const double* xpts, const double* vars,
                           const ShellData* data, double* res) {
  for (int e = 0; e < nelem; e++) {
    double X[12], u[24], R[24];
    gather_elem(e, conn, xpts, vars, X, u);
    for (int i = 0; i < 24; i++) R[i] = 0.0;
    oracle::element_residual<double>(data[e], X, u, R);
    for (int a = 0; a < 4; a++) {
      int n = conn[4 * e + a];
      for (int k = 0; k < 6; k++) res[6 * n + k] += R[6 * a + k];
    }
  }
}

double orc_assemble_energy(int nelem, const int* conn, const double* xpts, const double* vars,
                           const ShellData* data) {
  double U = 0.0;
  for (int e = 0; e < nelem; e++) {
    double X[12], u[24];
    gather_elem(e, conn, xpts, vars, X, u);
    U += oracle::element_energy<double>(data[e], X, u);
  }
  return U;
}

// ------------------------------------------------------------- BCs
// Dirichlet row/column elimination (apply_mat_bcs_rows_kernel /
// apply_mat_bcs_cols_kernel, bsr_mat.cuh:1-104): the BC row and column
// become the identity row/column. bcs are natural DOF indices; the node is
// mapped through perm[old] = new.
void orc_apply_bcs_mat(int nnodes, const int* rowp, const int* cols, const int* perm, int nbcs,
                       const int* bcs, double* values) {
  for (int ib = 0; ib < nbcs; ib++) {
    int dof = bcs[ib];
    int brow = perm[dof / 6], ir = dof % 6;
    int grow = 6 * brow + ir;
    for (int jp = rowp[brow]; jp < rowp[brow + 1]; jp++)
      for (int c = 0; c < 6; c++)
        values[36 * (size_t)jp + 6 * ir + c] = (6 * cols[jp] + c == grow) ? 1.0 : 0.0;
  }
  for (int ib = 0; ib < nbcs; ib++) {
    int dof = bcs[ib];
    int bcol = perm[dof / 6], ic = dof % 6;
    int gcol = 6 * bcol + ic;
    for (int i = 0; i < nnodes; i++)
      for (int jp = rowp[i]; jp < rowp[i + 1]; jp++)
        if (cols[jp] == bcol)
          for (int r = 0; r < 6; r++)
            values[36 * (size_t)jp + 6 * r + ic] = (6 * i + r == gcol) ? 1.0 : 0.0;
  }
}
void orc_apply_bcs_vec(int nbcs, const int* bcs, double* vec) {
  for (int i = 0; i < nbcs; i++) vec[bcs[i]] = 0.0;
}

// Symbolic full LU fill (no reordering) of a block pattern — the known-answer
// check of examples/basic_shell/test_fill_in.cu:24-29 (28 -> 32 blocks).
int orc_full_fill_count(int n, const int* rowp, const int* cols) {
  std::vector<std::vector<int>> rows(n);
  for (int i = 0; i < n; i++) rows[i].assign(cols + rowp[i], cols + rowp[i + 1]);
  // right-looking symbolic elimination on the symmetric structure
  for (int k = 0; k < n; k++) {
    std::vector<int> up;
    for (int c : rows[k])
      if (c > k) up.push_back(c);
    for (int i : up) {
      std::vector<int> merged;
      std::set_union(rows[i].begin(), rows[i].end(), up.begin(), up.end(),
                     std::back_inserter(merged));
      rows[i] = merged;
    }
  }
  int nz = 0;
  for (int i = 0; i < n; i++) nz += (int)rows[i].size();
  return nz;
}

// ------------------------------------------------------------- ILU(0)
static void blk_inv6(const double* A, double* Ai) {
  double M[36], I[36];
  for (int i = 0; i < 36; i++) {
    M[i] = A[i];
    I[i] = (i % 7 == 0) ? 1.0 : 0.0;
  }
  for (int c = 0; c < 6; c++) {
    int p = c;
    for (int r = c + 1; r < 6; r++)
      if (std::fabs(M[6 * r + c]) > std::fabs(M[6 * p + c])) p = r;
    if (p != c)
      for (int k = 0; k < 6; k++) {
        std::swap(M[6 * p + k], M[6 * c + k]);
        std::swap(I[6 * p + k], I[6 * c + k]);
      }
    double piv = 1.0 / M[6 * c + c];
    for (int k = 0; k < 6; k++) {
      M[6 * c + k] *= piv;
      I[6 * c + k] *= piv;
    }
    for (int r = 0; r < 6; r++)
      if (r != c) {
        double f = M[6 * r + c];
        if (f != 0.0)
          for (int k = 0; k < 6; k++) {
            M[6 * r + k] -= f * M[6 * c + k];
            I[6 * r + k] -= f * I[6 * c + k];
          }
      }
  }
  for (int i = 0; i < 36; i++) Ai[i] = I[i];
}
static void blk_mm(const double* A, const double* B, double* C) {  // C = A B
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      double s = 0.0;
      for (int k = 0; k < 6; k++) s += A[6 * i + k] * B[6 * k + j];
      C[6 * i + j] = s;
    }
}

// Block ILU(0) on A's own pattern, in place: lower blocks hold L (unit block
// diagonal implied), upper blocks and the diagonal hold U. Diagonal blocks
// are left as U_ii (not inverted). Returns 0, or 1 + the first block row
// whose diagonal block is singular.
int orc_ilu0_factor(int n, const int* rowp, const int* cols, double* vals) {
  std::vector<int> diag(n, -1);
  for (int i = 0; i < n; i++)
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++)
      if (cols[jp] == i) diag[i] = jp;
  std::vector<double> Uinv((size_t)n * 36);
  std::vector<int> pos(n, -1);
  for (int i = 0; i < n; i++) {
    if (diag[i] < 0) return i + 1;
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) pos[cols[jp]] = jp;
    for (int kp = rowp[i]; kp < rowp[i + 1] && cols[kp] < i; kp++) {
      int k = cols[kp];
      double L[36];
      blk_mm(&vals[36 * (size_t)kp], &Uinv[36 * (size_t)k], L);
      std::memcpy(&vals[36 * (size_t)kp], L, sizeof(L));
      for (int jp = diag[k] + 1; jp < rowp[k + 1]; jp++) {
        int j = cols[jp];
        int tp = pos[j];
        if (tp < 0) continue;
        double P[36];
        blk_mm(L, &vals[36 * (size_t)jp], P);
        for (int t = 0; t < 36; t++) vals[36 * (size_t)tp + t] -= P[t];
      }
    }
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) pos[cols[jp]] = -1;
    const double* D = &vals[36 * (size_t)diag[i]];
    blk_inv6(D, &Uinv[36 * (size_t)i]);
    for (int t = 0; t < 36; t++)
      if (!std::isfinite(Uinv[36 * (size_t)i + t])) return i + 1;
  }
  return 0;
}

// z = U^{-1} L^{-1} r on the factored values.
void orc_ilu0_apply(int n, const int* rowp, const int* cols, const double* LU, const double* r,
                    double* z) {
  std::vector<double> y((size_t)6 * n);
  for (int i = 0; i < n; i++) {
    double s[6];
    for (int k = 0; k < 6; k++) s[k] = r[6 * i + k];
    for (int jp = rowp[i]; jp < rowp[i + 1] && cols[jp] < i; jp++) {
      const double* B = &LU[36 * (size_t)jp];
      const double* x = &y[6 * (size_t)cols[jp]];
      for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) s[a] -= B[6 * a + b] * x[b];
    }
    for (int k = 0; k < 6; k++) y[6 * i + k] = s[k];
  }
  for (int i = n - 1; i >= 0; i--) {
    double s[6];
    int dp = -1;
    for (int k = 0; k < 6; k++) s[k] = y[6 * (size_t)i + k];
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) {
      if (cols[jp] == i) dp = jp;
      if (cols[jp] <= i) continue;
      const double* B = &LU[36 * (size_t)jp];
      const double* x = &z[6 * (size_t)cols[jp]];
      for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) s[a] -= B[6 * a + b] * x[b];
    }
    double Di[36];
    blk_inv6(&LU[36 * (size_t)dp], Di);
    for (int a = 0; a < 6; a++) {
      double t = 0.0;
      for (int b = 0; b < 6; b++) t += Di[6 * a + b] * s[b];
      z[6 * (size_t)i + a] = t;
    }
  }
}

// z = U^{-1} L^{-1} r on factor values whose diagonal blocks hold U_ii^{-1}
// (the layout the CUDA factorization produces): the same two block
// triangular solves as orc_ilu0_apply, multiplying by the stored inverse
// instead of inverting U_ii.
void orc_ilu_apply_dinv(int n, const int* rowp, const int* cols, const double* LU,
                        const double* r, double* z) {
  std::vector<double> y((size_t)6 * n);
  for (int i = 0; i < n; i++) {
    double s[6];
    for (int k = 0; k < 6; k++) s[k] = r[6 * (size_t)i + k];
    for (int jp = rowp[i]; jp < rowp[i + 1] && cols[jp] < i; jp++) {
      const double* B = &LU[36 * (size_t)jp];
      const double* x = &y[6 * (size_t)cols[jp]];
      for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) s[a] -= B[6 * a + b] * x[b];
    }
    for (int k = 0; k < 6; k++) y[6 * (size_t)i + k] = s[k];
  }
  for (int i = n - 1; i >= 0; i--) {
    double s[6];
    int dp = -1;
    for (int k = 0; k < 6; k++) s[k] = y[6 * (size_t)i + k];
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) {
      if (cols[jp] == i) dp = jp;
      if (cols[jp] <= i) continue;
      const double* B = &LU[36 * (size_t)jp];
      const double* x = &z[6 * (size_t)cols[jp]];
      for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) s[a] -= B[6 * a + b] * x[b];
    }
    const double* Di = &LU[36 * (size_t)dp];
    for (int a = 0; a < 6; a++) {
      double t = 0.0;
      for (int b = 0; b < 6; b++) t += Di[6 * a + b] * s[b];
      z[6 * (size_t)i + a] = t;
    }
  }
}

// Backward error of a block ILU factor on its own pattern, without forming
// dense matrices: (L U)_ij = sum_{k <= min(i,j)} L_ik U_kj with L_ii = I,
// compared with A_ij for every (i, j) of the pattern (ILU(k) is defined by
// (L U)_ij = A_ij there). LU holds L below the diagonal, U above it and
// U_ii^{-1} on it (the CUDA layout; dinv = 1) or U_ii (dinv = 0). A is
// given on the same pattern. out[0] = max |(L U - A)_ij|, out[1] = max |A|.
void orc_ilu_backward_error(int n, const int* rowp, const int* cols, const double* LU,
                            const double* A, int dinv, double* out) {
  std::vector<int> diag(n, -1);
  for (int i = 0; i < n; i++)
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++)
      if (cols[jp] == i) diag[i] = jp;
  std::vector<double> U((size_t)36 * n);  // U_ii
  for (int i = 0; i < n; i++) {
    const double* D = &LU[36 * (size_t)diag[i]];
    if (dinv)
      blk_inv6(D, &U[36 * (size_t)i]);
    else
      std::memcpy(&U[36 * (size_t)i], D, 36 * sizeof(double));
  }
  double emax = 0.0, amax = 0.0;
#ifdef _OPENMP
#pragma omp parallel reduction(max : emax, amax)
#endif
  {
    std::vector<int> pos(n, -1);
    std::vector<double> acc;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
    for (int i = 0; i < n; i++) {
      const int r0 = rowp[i], r1 = rowp[i + 1];
      acc.assign((size_t)36 * (r1 - r0), 0.0);
      for (int jp = r0; jp < r1; jp++) pos[cols[jp]] = jp - r0;
      auto add = [&](const double* Lik, int k) {  // acc[i, j] += L_ik U_kj, j in U(k)
        for (int jp = diag[k]; jp < rowp[k + 1]; jp++) {
          const int t = pos[cols[jp]];
          if (t < 0) continue;
          const double* Ukj = jp == diag[k] ? &U[36 * (size_t)k] : &LU[36 * (size_t)jp];
          double* C = &acc[36 * (size_t)t];
          if (!Lik) {
            for (int q = 0; q < 36; q++) C[q] += Ukj[q];
          } else {
            for (int a = 0; a < 6; a++)
              for (int b = 0; b < 6; b++) {
                double sum = 0.0;
                for (int m = 0; m < 6; m++) sum += Lik[6 * a + m] * Ukj[6 * m + b];
                C[6 * a + b] += sum;
              }
          }
        }
      };
      for (int kp = r0; kp < diag[i]; kp++) add(&LU[36 * (size_t)kp], cols[kp]);
      add(nullptr, i);
      for (int jp = r0; jp < r1; jp++) {
        const double* a = &A[36 * (size_t)jp];
        const double* c = &acc[36 * (size_t)(jp - r0)];
        for (int q = 0; q < 36; q++) {
          emax = std::max(emax, std::fabs(c[q] - a[q]));
          amax = std::max(amax, std::fabs(a[q]));
        }
      }
      for (int jp = r0; jp < r1; jp++) pos[cols[jp]] = -1;
    }
  }
  out[0] = emax;
  out[1] = amax;
}

// Copy A's blocks into a pattern that contains A's (copyValuesTo,
// include/linalg/bsr_mat.h:145-193); other blocks of out are zeroed.
// Returns 0, or 1 + the first row with a block missing from the pattern.
int orc_scatter_to_pattern(int n, const int* rowp, const int* cols, const double* vals,
                           const int* rowp2, const int* cols2, double* out) {
  std::memset(out, 0, sizeof(double) * 36 * (size_t)rowp2[n]);
  for (int i = 0; i < n; i++) {
    int q = rowp2[i];
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) {
      while (q < rowp2[i + 1] && cols2[q] < cols[jp]) q++;
      if (q == rowp2[i + 1] || cols2[q] != cols[jp]) return i + 1;
      std::memcpy(&out[36 * (size_t)q], &vals[36 * (size_t)jp], 36 * sizeof(double));
    }
  }
  return 0;
}

// y = A x (BSR 6x6 row-major blocks)
void orc_spmv(int n, const int* rowp, const int* cols, const double* A, const double* x,
              double* y) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (int i = 0; i < n; i++) {
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) {
      const double* B = &A[36 * (size_t)jp];
      const double* xx = &x[6 * (size_t)cols[jp]];
      for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) s[a] += B[6 * a + b] * xx[b];
    }
    for (int a = 0; a < 6; a++) y[6 * (size_t)i + a] = s[a];
  }
}

// Level sets of the lower (lower=1) or upper (lower=0) triangular solve DAG:
// level[i] = 1 + max level over dependencies (0 if none). Returns #levels.
int orc_levels(int n, const int* rowp, const int* cols, int lower, int* level) {
  int nl = 0;
  if (lower) {
    for (int i = 0; i < n; i++) {
      int l = 0;
      for (int jp = rowp[i]; jp < rowp[i + 1] && cols[jp] < i; jp++)
        l = std::max(l, level[cols[jp]] + 1);
      level[i] = l;
      nl = std::max(nl, l + 1);
    }
  } else {
    for (int i = n - 1; i >= 0; i--) {
      int l = 0;
      for (int jp = rowp[i]; jp < rowp[i + 1]; jp++)
        if (cols[jp] > i) l = std::max(l, level[cols[jp]] + 1);
      level[i] = l;
      nl = std::max(nl, l + 1);
    }
  }
  return nl;
}

// ------------------------------------------------------------- GMRES
// GMRES(m) with modified Gram-Schmidt and Givens rotations
// (examples/iterative/gmres.cu:468-771; c = a/h, s = b/h as at :684-693),
// restarted. A is on (rowp, cols); the block ILU factor LU is on its own
// pattern (prowp, pcols) with U_ii^{-1} in its diagonal blocks. side = 0:
// left preconditioning M^{-1} A x = M^{-1} b (the reference's choice);
// side = 1: right preconditioning A M^{-1} y = b. The inner loop stops when
// the Givens residual estimate reaches rtol times its initial value;
// convergence is declared on the true relative residual ||b - A x|| / ||b||
// <= rtol, checked at every restart. Vector work runs on nthreads threads.
int orc_gmres_k(int n, const int* rowp, const int* cols, const double* A, const int* prowp,
                const int* pcols, const double* LU, const double* b, double* x, int m,
                double rtol, int maxit, int side, int nthreads, int* iters, double* relres) {
  const size_t N = (size_t)6 * n;
  const long long NN = (long long)N;
  if (nthreads < 1) nthreads = 1;
  std::vector<std::vector<double>> V(m + 1, std::vector<double>(N));
  std::vector<double> H((size_t)(m + 1) * m), g(m + 1), cs(m), ss(m), w(N), t(N), r(N),
      bb(b, b + N), xx(x, x + N);
  auto dot = [&](const std::vector<double>& a, const std::vector<double>& c) {
    double s = 0.0;
#ifdef _OPENMP
#pragma omp parallel for reduction(+ : s) num_threads(nthreads) if (nthreads > 1)
#endif
    for (long long k = 0; k < NN; k++) s += a[k] * c[k];
    return s;
  };
  auto axpy = [&](double a, const std::vector<double>& xv, std::vector<double>& yv) {
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) if (nthreads > 1)
#endif
    for (long long k = 0; k < NN; k++) yv[k] += a * xv[k];
  };
  auto spmv = [&](const double* in, double* out) {
#ifdef _OPENMP
#pragma omp parallel for num_threads(nthreads) schedule(static) if (nthreads > 1)
#endif
    for (int i = 0; i < n; i++) {
      double s[6] = {0, 0, 0, 0, 0, 0};
      for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) {
        const double* B = &A[36 * (size_t)jp];
        const double* xv = &in[6 * (size_t)cols[jp]];
        for (int a = 0; a < 6; a++)
          for (int c = 0; c < 6; c++) s[a] += B[6 * a + c] * xv[c];
      }
      for (int a = 0; a < 6; a++) out[6 * (size_t)i + a] = s[a];
    }
  };
  auto prec = [&](const double* in, double* out) {
    orc_ilu_apply_dinv(n, prowp, pcols, LU, in, out);
  };
  double bnorm = std::sqrt(dot(bb, bb));
  if (bnorm == 0.0) bnorm = 1.0;
  int it = 0;
  auto true_res = [&]() {
    spmv(xx.data(), t.data());
    for (size_t i = 0; i < N; i++) r[i] = bb[i] - t[i];
    return std::sqrt(dot(r, r)) / bnorm;
  };
  double rel = true_res();
  while (rel > rtol && it < maxit) {
    if (side == 0)
      prec(r.data(), V[0].data());
    else
      V[0] = r;
    double beta = std::sqrt(dot(V[0], V[0]));
    if (!(beta > 0.0) || !std::isfinite(beta)) break;
    for (size_t i = 0; i < N; i++) V[0][i] /= beta;
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    const double target = rtol * (side == 0 ? beta / rel : bnorm);
    int j = 0;
    for (; j < m && it < maxit; j++, it++) {
      if (side == 0) {
        spmv(V[j].data(), t.data());
        prec(t.data(), w.data());
      } else {
        prec(V[j].data(), t.data());
        spmv(t.data(), w.data());
      }
      for (int i = 0; i <= j; i++) {
        const double h = dot(w, V[i]);
        H[(size_t)i * m + j] = h;
        axpy(-h, V[i], w);
      }
      const double hn = std::sqrt(dot(w, w));
      H[(size_t)(j + 1) * m + j] = hn;
      if (hn != 0.0)
        for (size_t k = 0; k < N; k++) V[j + 1][k] = w[k] / hn;
      for (int i = 0; i < j; i++) {
        const double a = H[(size_t)i * m + j], c = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + ss[i] * c;
        H[(size_t)(i + 1) * m + j] = -ss[i] * a + cs[i] * c;
      }
      const double a = H[(size_t)j * m + j], c = H[(size_t)(j + 1) * m + j];
      const double hyp = std::sqrt(a * a + c * c);
      cs[j] = hyp > 0.0 ? a / hyp : 1.0;
      ss[j] = hyp > 0.0 ? c / hyp : 0.0;
      H[(size_t)j * m + j] = cs[j] * a + ss[j] * c;
      H[(size_t)(j + 1) * m + j] = 0.0;
      g[j + 1] = -ss[j] * g[j];
      g[j] = cs[j] * g[j];
      if (std::fabs(g[j + 1]) <= target || hn == 0.0) {
        j++;
        it++;
        break;
      }
    }
    // y = H^{-1} g (upper triangular), x += V y (left) or M^{-1} V y (right)
    std::vector<double> y(j);
    for (int i = j - 1; i >= 0; i--) {
      double s = g[i];
      for (int k = i + 1; k < j; k++) s -= H[(size_t)i * m + k] * y[k];
      y[i] = s / H[(size_t)i * m + i];
    }
    std::fill(w.begin(), w.end(), 0.0);
    for (int i = 0; i < j; i++) axpy(y[i], V[i], w);
    if (side == 1) {
      prec(w.data(), t.data());
      w.swap(t);
    }
    for (size_t k = 0; k < N; k++) xx[k] += w[k];
    rel = true_res();
    if (!std::isfinite(rel)) break;
  }
  for (size_t i = 0; i < N; i++) x[i] = xx[i];
  *iters = it;
  *relres = rel;
  return rel <= rtol ? 0 : 1;
}

// Dense LU with partial pivoting; solves A x = b in place (A row-major n x n,
// overwritten). Returns 0 on success.
int orc_dense_solve(int n, double* A, double* b) {
  std::vector<int> piv(n);
  for (int k = 0; k < n; k++) {
    int p = k;
    for (int i = k + 1; i < n; i++)
      if (std::fabs(A[(size_t)i * n + k]) > std::fabs(A[(size_t)p * n + k])) p = i;
    if (A[(size_t)p * n + k] == 0.0) return k + 1;
    if (p != k) {
      for (int j = 0; j < n; j++) std::swap(A[(size_t)p * n + j], A[(size_t)k * n + j]);
      std::swap(b[p], b[k]);
    }
    double inv = 1.0 / A[(size_t)k * n + k];
    for (int i = k + 1; i < n; i++) {
      double f = A[(size_t)i * n + k] * inv;
      if (f == 0.0) continue;
      A[(size_t)i * n + k] = f;
      for (int j = k + 1; j < n; j++) A[(size_t)i * n + j] -= f * A[(size_t)k * n + j];
      b[i] -= f * b[k];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = b[i];
    for (int j = i + 1; j < n; j++) s -= A[(size_t)i * n + j] * b[j];
    b[i] = s / A[(size_t)i * n + i];
  }
  return 0;
}

}  // extern "C"

extern "C" {
// Symbolic ILU(k) (computeILUk, include/linalg/bsr_utils.h:678-807): level of
// fill of entry (i,j) = min over k of lev(i,k) + lev(k,j) + 1; entries with
// level <= levFill are kept, original entries have level 0 and a missing
// diagonal is added. Pass cols_out = NULL to count. Returns nnz.
int orc_iluk_pattern(int n, const int* rowp, const int* cols, int levFill, int* rowp_out,
                     int* cols_out) {
  std::vector<int> rp(n + 1, 0), cl, lv, diag(n);
  std::vector<int> rcols, rlevs;
  for (int i = 0; i < n; i++) {
    rcols.assign(cols + rowp[i], cols + rowp[i + 1]);
    rlevs.assign(rcols.size(), 0);
    if (!std::binary_search(rcols.begin(), rcols.end(), i)) {
      auto it = std::lower_bound(rcols.begin(), rcols.end(), i);
      rlevs.insert(rlevs.begin() + (it - rcols.begin()), 0);
      rcols.insert(it, i);
    }
    size_t j = 0;
    for (; rcols[j] < i; j++) {
      int k = rcols[j], clev = rlevs[j];
      size_t p = j + 1;
      for (int kk = diag[k] + 1; kk < rp[k + 1]; kk++) {
        while (p < rcols.size() && rcols[p] < cl[kk]) p++;
        int nl = clev + lv[kk] + 1;
        if (p < rcols.size() && rcols[p] == cl[kk]) {
          if (rlevs[p] > nl) rlevs[p] = nl;
        } else if (nl <= levFill) {
          rcols.insert(rcols.begin() + p, cl[kk]);
          rlevs.insert(rlevs.begin() + p, nl);
        }
      }
    }
    diag[i] = rp[i] + (int)j;
    cl.insert(cl.end(), rcols.begin(), rcols.end());
    lv.insert(lv.end(), rlevs.begin(), rlevs.end());
    rp[i + 1] = (int)cl.size();
  }
  if (rowp_out)
    for (int i = 0; i <= n; i++) rowp_out[i] = rp[i];
  if (cols_out)
    for (size_t k = 0; k < cl.size(); k++) cols_out[k] = cl[k];
  return (int)cl.size();
}

// The same Dirichlet elimination as orc_apply_bcs_mat in one pass over the
// blocks, with a per-DOF mask instead of a scan of every block per BC DOF
// (identical values: every entry of a BC row or column is assigned 0 or 1).
void orc_apply_bcs_mat_fast(int nnodes, const int* rowp, const int* cols, const int* perm,
                            int nbcs, const int* bcs, double* values) {
  std::vector<unsigned char> mask(nnodes, 0);  // solver-order node -> constrained DOF bits
  for (int ib = 0; ib < nbcs; ib++) mask[perm[bcs[ib] / 6]] |= (unsigned char)(1u << (bcs[ib] % 6));
  for (int i = 0; i < nnodes; i++)
    for (int jp = rowp[i]; jp < rowp[i + 1]; jp++) {
      const int j = cols[jp];
      if (!mask[i] && !mask[j]) continue;
      double* v = &values[36 * (size_t)jp];
      for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++)
          if (((mask[i] >> r) & 1) || ((mask[j] >> c) & 1))
            v[6 * r + c] = (i == j && r == c) ? 1.0 : 0.0;
    }
}

// One CPU solve of a shell problem along the path the GPU runs, for the
// timed CPU baseline: block pattern (get_row_col_ptrs) in the given node
// ordering (perm[old] = new), element assembly of K (add_jacobian_cpu,
// elements on nthreads threads) and the Dirichlet elimination, symbolic
// ILU(fill) (computeILUk), numeric block ILU, and right-preconditioned
// GMRES(restart) to ||b - A x|| / ||b|| <= rtol (examples/iterative/gmres.cu
// steps, FP64 throughout). x_out gets the displacements in natural order.
// t[0..3]: seconds of pattern + symbolic ILU (set-up the GPU path keeps
// resident between steps), assembly + BCs, numeric factorization, GMRES.
// Returns 0 when converged, 1 when not, 2 on a singular pivot.
int orc_solve_problem(int nelem, int nnodes, const int* conn, const double* xpts,
                      const ShellData* data, int nbcs, const int* bcs, const double* loads,
                      const int* perm, int fill, int restart, double rtol, int maxit,
                      int nthreads, double* x_out, int* iters, double* relres, double* t) {
  using clk = std::chrono::steady_clock;
  auto sec = [](clk::time_point a, clk::time_point b) {
    return std::chrono::duration<double>(b - a).count();
  };
  const auto t0 = clk::now();
  const int nnz0 = orc_bsr_pattern(nelem, nnodes, conn, nullptr, nullptr);
  std::vector<int> rowp0(nnodes + 1), cols0(nnz0), rowp(nnodes + 1), cols(nnz0),
      emap((size_t)16 * nelem);
  orc_bsr_pattern(nelem, nnodes, conn, rowp0.data(), cols0.data());
  orc_permute_pattern(nnodes, rowp0.data(), cols0.data(), perm, rowp.data(), cols.data());
  orc_elem_ind_map(nelem, conn, rowp.data(), cols.data(), perm, emap.data());
  std::vector<int> prowp(nnodes + 1);
  const int nnzp = orc_iluk_pattern(nnodes, rowp.data(), cols.data(), fill, prowp.data(), nullptr);
  std::vector<int> pcols(nnzp);
  orc_iluk_pattern(nnodes, rowp.data(), cols.data(), fill, prowp.data(), pcols.data());
  const auto t1 = clk::now();
  std::vector<double> A((size_t)36 * nnz0, 0.0);
  orc_assemble_jacobian(nelem, conn, xpts, nullptr, data, emap.data(), A.data(), nullptr,
                        nthreads);
  orc_apply_bcs_mat_fast(nnodes, rowp.data(), cols.data(), perm, nbcs, bcs, A.data());
  const auto t2 = clk::now();
  std::vector<double> LU((size_t)36 * nnzp);
  orc_scatter_to_pattern(nnodes, rowp.data(), cols.data(), A.data(), prowp.data(), pcols.data(),
                         LU.data());
  const int piv = orc_ilu0_factor(nnodes, prowp.data(), pcols.data(), LU.data());
  if (piv) return 2;
  for (int i = 0; i < nnodes; i++)
    for (int jp = prowp[i]; jp < prowp[i + 1]; jp++)
      if (pcols[jp] == i) {
        double Di[36];
        blk_inv6(&LU[36 * (size_t)jp], Di);
        std::memcpy(&LU[36 * (size_t)jp], Di, sizeof(Di));
      }
  const auto t3 = clk::now();
  const size_t N = (size_t)6 * nnodes;
  std::vector<double> b(N), x(N, 0.0);
  for (int i = 0; i < nnodes; i++)
    for (int k = 0; k < 6; k++) b[6 * (size_t)perm[i] + k] = loads[6 * (size_t)i + k];
  const int st = orc_gmres_k(nnodes, rowp.data(), cols.data(), A.data(), prowp.data(),
                             pcols.data(), LU.data(), b.data(), x.data(), restart, rtol, maxit, 1,
                             nthreads, iters, relres);
  const auto t4 = clk::now();
  for (int i = 0; i < nnodes; i++)
    for (int k = 0; k < 6; k++) x_out[6 * (size_t)i + k] = x[6 * (size_t)perm[i] + k];
  if (t) {
    t[0] = sec(t0, t1);
    t[1] = sec(t1, t2);
    t[2] = sec(t2, t3);
    t[3] = sec(t3, t4);
  }
  return st;
}
}  // extern "C"
