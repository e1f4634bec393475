// Shell residual / Jacobian / energy assembly kernels and their C ABI.
//
// Reference: add_residual_gpu / add_jacobian_gpu (include/base/elem_group.cuh:17-211)
// launch one thread per (element, quadrature point[, Jacobian column]) and
// scatter with FP64 atomicAdd (include/linalg/vec.h:278-293,
// include/linalg/bsr_mat.h:229-276).
//
// Here a warp owns a chunk of up to eight neighbouring elements:
//   * coordinates and DOFs of the chunk are gathered into the warp's shared
//     memory slot and the per-element geometry (normals, nodal frames, the
//     four quadrature-point frames, the tying-point vectors) is computed by
//     8 x 4 lanes at once;
//   * per element, lane l < 24 builds column l of the four 9x24 strain
//     matrices B_q and of D B_q; each of the 32 lanes then owns a 3x6 tile of
//     K_e = sum_q B_q^T D B_q (144 contiguous bytes of one 6x6 BSR block) and
//     writes it with 16-byte stores; R_e = K_e u_e follows from the tiles;
//   * the scatter follows the coloured schedule built on the host: chunks of
//     one colour share no node and run concurrently (one launch per colour);
//     inside a chunk the warp handles its elements in order. The first
//     toucher of a block stores, later touchers read-modify-write; there are
//     no atomics and the result is bitwise reproducible;
//   * with GF_ASSEMBLE_ATOMIC the colours are ignored: the outputs are zeroed
//     and one launch over all chunks adds with FP64 atomics (the reference's
//     scatter; sums in arrival order, so not bitwise reproducible);
//   * a batch of problems runs each colour of all its problems in one launch
//     (work items = (problem, chunk) per warp), or all chunks of all
//     problems in one launch with atomics.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "gf_internal.h"

namespace gf {

constexpr int kAsmWarps = 2;     // warps (= chunks) per CTA
constexpr int kEPW = 8;          // elements per chunk; geometry spread over 8 x 4 lanes
constexpr int kChunkSize = kEPW;

struct WarpSlot {
  double X[kEPW][12];
  double U[kEPW][24];
  ElemGeom g[kEPW];
  double Bt[36][24];   // B_q[k][l] of the current element, row qk = 9q + k
  double DBt[36][24];  // (D B_q)[k][l]
  double E[36];
  double S[36];
};

struct AsmParams {
  const double* xpts;
  const double* vars;
  const uint8_t* bcmask;
  const int32_t* sconn;
  const int32_t* semap;
  const uint32_t* sft;
  const double* sthick;
  const int32_t* smat;
  const Material* mats;
  const int32_t* chunk_start;
  const double* thick_nat;   // optional per-call thickness (natural element order)
  const int32_t* sorder;     // schedule position -> element
  int chunk_base, chunk_end;
  double* values;
  double* res;
  double* energy_part;
  int flags;
};

enum { MODE_JAC = 0, MODE_RES = 1, MODE_ENERGY = 2 };

// Geometry of up to kEPW elements (schedule positions s0 .. s0+cnt-1).
__device__ void batch_geometry(int s0, int cnt, WarpSlot& w, const AsmParams& P, int lane) {
  for (int t = lane; t < cnt * 12; t += 32) {
    const int k = t / 12, i = t % 12;
    const int node = P.sconn[4 * (s0 + k) + i / 3];
    w.X[k][i] = P.xpts[3 * node + i % 3];
  }
  for (int t = lane; t < cnt * 24; t += 32) {
    const int k = t / 24, i = t % 24;
    const int node = P.sconn[4 * (s0 + k) + i / 6];
    w.U[k][i] = P.vars ? P.vars[6 * node + i % 6] : 0.0;
  }
  __syncwarp();
  const int k = lane >> 2, n = lane & 3;
  const bool on = k < cnt;
  Material m;
  if (on) m = P.mats[P.smat ? P.smat[s0 + k] : 0];
  if (on) geom_normal(w.X[k], n, &w.g[k].fn[3 * n]);
  __syncwarp();
  if (on) {
    geom_node(m, w.X[k], w.g[k].fn, n, w.g[k].Tn01[n], w.g[k].XTn[n], w.g[k].tcross[n]);
    geom_quad(m, w.X[k], w.g[k].fn, n, w.g[k].T[n], w.g[k].A[n], w.g[k].Az[n],
              w.g[k].scale[n]);
  }
  for (int t = lane; t < cnt * 5; t += 32) geom_tying(w.X[t / 5], w.g[t / 5].fn, t % 5, w.g[t / 5]);
  __syncwarp();
}

template <int MODE>
__device__ void process_element(int s, int k, WarpSlot& w, const AsmParams& P, int lane,
                                double& energy_acc) {
  const Material m = P.mats[P.smat ? P.smat[s] : 0];
  const double t = P.thick_nat ? P.thick_nat[P.sorder[s]] : P.sthick[s];
  const ElemGeom& g = w.g[k];
  if (lane < 24) {
    double Bc[36];
    bmat_column(g, lane, Bc);
#pragma unroll
    for (int qk = 0; qk < 36; qk++) w.Bt[qk][lane] = Bc[qk];
    if (MODE == MODE_JAC) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        double Sq[9];
        stress(m, t, g.scale[q], &Bc[9 * q], Sq);
#pragma unroll
        for (int kk = 0; kk < 9; kk++) w.DBt[9 * q + kk][lane] = Sq[kk];
      }
    }
  }
  __syncwarp();
  const int4 cn = reinterpret_cast<const int4*>(P.sconn)[s];
  const int nodes[4] = {cn.x, cn.y, cn.z, cn.w};
  const bool fuse = (P.flags & GF_ASSEMBLE_FUSE_BCS) != 0;
  const bool add = (P.flags & GF_ASSEMBLE_ADD) != 0;
  const uint32_t ft = P.sft[s];

  if (MODE == MODE_JAC) {
    // lane (I, J): rows 3I..3I+2, columns 6J..6J+5 of K_e (one block row slice)
    const int I = lane >> 2, J = lane & 3;
    double acc[3][6];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 6; c++) acc[r][c] = 0.0;
#pragma unroll 4
    for (int qk = 0; qk < 36; qk++) {
      const double b0 = w.Bt[qk][3 * I], b1 = w.Bt[qk][3 * I + 1], b2 = w.Bt[qk][3 * I + 2];
      const double2* dp = reinterpret_cast<const double2*>(&w.DBt[qk][6 * J]);
      const double2 d01 = dp[0], d23 = dp[1], d45 = dp[2];
      const double d[6] = {d01.x, d01.y, d23.x, d23.y, d45.x, d45.y};
#pragma unroll
      for (int c = 0; c < 6; c++) {
        acc[0][c] = fma(b0, d[c], acc[0][c]);
        acc[1][c] = fma(b1, d[c], acc[1][c]);
        acc[2][c] = fma(b2, d[c], acc[2][c]);
      }
    }
    const int a = I >> 1, r0 = 3 * (I & 1), b = J;
    // residual part for rows 3I..3I+2 over columns of node b
    double rp[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
      double s_ = 0.0;
#pragma unroll
      for (int c = 0; c < 6; c++) s_ = fma(acc[r][c], w.U[k][6 * b + c], s_);
      rp[r] = s_;
    }
    if (P.values) {
      const uint32_t bca = fuse ? P.bcmask[nodes[a]] : 0u;
      const uint32_t bcb = fuse ? P.bcmask[nodes[b]] : 0u;
      const bool first = (ft >> (4 * a + b)) & 1;
      const int blk = P.semap[16 * s + 4 * a + b];
      double* dst = P.values + 36 * (size_t)blk + 6 * r0;
      double v[18];
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 6; c++) {
          double x = acc[r][c];
          if (fuse && (((bca >> (r0 + r)) & 1) || ((bcb >> c) & 1)))
            x = (a == b && r0 + r == c && first) ? 1.0 : 0.0;
          v[6 * r + c] = x;
        }
      double2* d2 = reinterpret_cast<double2*>(dst);
      if (P.flags & GF_ASSEMBLE_ATOMIC) {
#pragma unroll
        for (int h = 0; h < 18; h++) atomicAdd(dst + h, v[h]);
      } else if (first && !add) {
#pragma unroll
        for (int h = 0; h < 9; h++) d2[h] = make_double2(v[2 * h], v[2 * h + 1]);
      } else {
#pragma unroll
        for (int h = 0; h < 9; h++) {
          const double2 o = d2[h];
          d2[h] = make_double2(o.x + v[2 * h], o.y + v[2 * h + 1]);
        }
      }
    }
    // R rows 3I..3I+2: sum the four column slices (lanes J = 0..3 of row group I)
#pragma unroll
    for (int r = 0; r < 3; r++) {
      rp[r] += __shfl_xor_sync(0xffffffffu, rp[r], 1);
      rp[r] += __shfl_xor_sync(0xffffffffu, rp[r], 2);
    }
    if (P.res && J < 3) {
      const int r = r0 + J;  // lanes J = 0,1,2 store rows r0, r0+1, r0+2
      double val = rp[J == 0 ? 0 : (J == 1 ? 1 : 2)];
      if (fuse && ((P.bcmask[nodes[a]] >> r) & 1)) val = 0.0;
      double* dst = P.res + 6 * (size_t)nodes[a] + r;
      const bool first = (ft >> (16 + a)) & 1;
      if (P.flags & GF_ASSEMBLE_ATOMIC)
        atomicAdd(dst, val);
      else if (first && !add)
        *dst = val;
      else
        *dst += val;
    }
  } else {
    // E_q = B_q u, S_q = D E_q, R = sum_q B_q^T S_q
    double e0 = 0.0, e1 = 0.0;
#pragma unroll
    for (int l = 0; l < 24; l++) {
      e0 = fma(w.Bt[lane][l], w.U[k][l], e0);
      if (lane < 4) e1 = fma(w.Bt[32 + lane][l], w.U[k][l], e1);
    }
    double* E = w.E;
    E[lane] = e0;
    if (lane < 4) E[32 + lane] = e1;
    __syncwarp();
    if (lane < 4) stress(m, t, g.scale[lane], &E[9 * lane], &w.S[9 * lane]);
    __syncwarp();
    if (MODE == MODE_ENERGY) {
      if (lane == 0) {
        double U = 0.0;
        for (int q = 0; q < 36; q++) U += 0.5 * E[q] * w.S[q];
        energy_acc += U;
      }
    } else if (lane < 24) {
      double rj = 0.0;
#pragma unroll
      for (int qk = 0; qk < 36; qk++) rj = fma(w.Bt[qk][lane], w.S[qk], rj);
      if (P.res) {
        const int b = lane / 6, c = lane % 6;
        if (fuse && ((P.bcmask[nodes[b]] >> c) & 1)) rj = 0.0;
        double* dst = P.res + 6 * (size_t)nodes[b] + c;
        const bool first = (ft >> (16 + b)) & 1;
        if (P.flags & GF_ASSEMBLE_ATOMIC)
          atomicAdd(dst, rj);
        else if (first && !add)
          *dst = rj;
        else
          *dst += rj;
      }
    }
  }
  __syncwarp();
}

template <int MODE>
__global__ void __launch_bounds__(kAsmWarps * 32)
    assemble_kernel(AsmParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSlot* slots = reinterpret_cast<WarpSlot*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int li = P.chunk_base + blockIdx.x * kAsmWarps + warp;  // this warp's chunk
  if (li >= P.chunk_end) return;
  const int s0 = P.chunk_start[li], cnt = P.chunk_start[li + 1] - s0;
  WarpSlot& w = slots[warp];
  double energy_acc = 0.0;
  batch_geometry(s0, cnt, w, P, lane);
  for (int k = 0; k < cnt; k++) process_element<MODE>(s0 + k, k, w, P, lane, energy_acc);
  if (MODE == MODE_ENERGY && lane == 0) P.energy_part[li] = energy_acc;
}

// Batched form: warp w of the launch works on chunk work[w].y of problem
// work[w].x, whose parameters are copied to shared memory first.
template <int MODE>
__global__ void __launch_bounds__(kAsmWarps * 32)
    assemble_batch_kernel(const AsmParams* __restrict__ PP, const int2* __restrict__ work,
                          int nwork) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSlot* slots = reinterpret_cast<WarpSlot*>(smem_raw);
  __shared__ AsmParams sp[kAsmWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wi = blockIdx.x * kAsmWarps + warp;
  if (wi >= nwork) return;
  const int2 it = work[wi];
  if (lane == 0) sp[warp] = PP[it.x];
  __syncwarp();
  const AsmParams& P = sp[warp];
  const int s0 = P.chunk_start[it.y], cnt = P.chunk_start[it.y + 1] - s0;
  WarpSlot& w = slots[warp];
  double energy_acc = 0.0;
  batch_geometry(s0, cnt, w, P, lane);
  for (int k = 0; k < cnt; k++) process_element<MODE>(s0 + k, k, w, P, lane, energy_acc);
}

__global__ void sum_kernel(const double* part, int n, double* out) {
  // deterministic single-thread-per-lane tree over a fixed partition
  __shared__ double s[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += part[i];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

// Dirichlet rows and columns (apply_mat_bcs_rows_kernel /
// apply_mat_bcs_cols_kernel, include/linalg/bsr_mat.cuh:1-104) in one pass
// over a precomputed entry list: (block, block row, is_column, inner index).
__global__ void bc_mat_kernel(const int32_t* entries, int n, const int32_t* cols,
                              double* values) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int4 e = reinterpret_cast<const int4*>(entries)[t];
  const int blk = e.x, brow = e.y, is_col = e.z, inner = e.w;
  const int bcol = cols[blk];
  double* v = values + 36 * (size_t)blk;
  for (int k = 0; k < 6; k++) {
    const int r = is_col ? k : inner, c = is_col ? inner : k;
    v[6 * r + c] = (6 * brow + r == 6 * bcol + c) ? 1.0 : 0.0;
  }
}

__global__ void gather_thickness(const int32_t* order, int n, const double* in, double* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = in[order[t]];
}

__global__ void bc_vec_kernel(const int32_t* bcs, int n, double* vec) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) vec[bcs[t]] = 0.0;
}

__global__ void permute_kernel(const int32_t* perm, int nnodes, const double* in, double* out,
                               int dir) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 6 * nnodes) return;
  const int i = t / 6, k = t % 6;
  if (dir == 0)
    out[6 * (size_t)perm[i] + k] = in[t];
  else
    out[t] = in[6 * (size_t)perm[i] + k];
}

template <int MODE>
static gf_status launch_assembly(gf_assembler* a, double* values, double* res, int flags,
                                 cudaStream_t st, const double* thick_nat = nullptr) {
  AsmParams P;
  P.xpts = a->d_xpts.p;
  P.vars = a->d_vars.p;
  P.bcmask = a->d_bcmask.p;
  P.sconn = a->d_sconn.p;
  P.semap = a->d_semap.p;
  P.sft = a->d_sft.p;
  P.sthick = a->d_sthick.p;
  P.smat = a->d_smat.p;
  P.mats = a->d_mats.p;
  P.chunk_start = a->d_chunk_start.p;
  P.thick_nat = thick_nat;
  P.sorder = a->d_sorder.p;
  P.values = values;
  P.res = res;
  P.energy_part = a->d_energy_part.p;
  P.flags = flags;
  const size_t smem = sizeof(WarpSlot) * kAsmWarps;
  // per device and constant, so setting it on every call is race-free
  GF_CUDA(cudaFuncSetAttribute(assemble_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  const Schedule& s = a->sched;
  if (flags & GF_ASSEMBLE_ATOMIC) {
    if (!(flags & GF_ASSEMBLE_ADD)) {
      if (values) GF_CUDA(cudaMemsetAsync(values, 0, sizeof(double) * 36 * (size_t)a->pat.nnz(), st));
      if (res) GF_CUDA(cudaMemsetAsync(res, 0, sizeof(double) * 6 * (size_t)a->nnodes, st));
    }
    P.chunk_base = 0;
    P.chunk_end = s.nchunks;
    const int nblk = (s.nchunks + kAsmWarps - 1) / kAsmWarps;
    if (nblk > 0) {
      assemble_kernel<MODE><<<nblk, kAsmWarps * 32, smem, st>>>(P); ::gf::count_launch();
      GF_CHECK_LAUNCH();
    }
    return GF_OK;
  }
  for (int cc = 0; cc < s.ncc; cc++) {
    const int nch = s.cc_start[cc + 1] - s.cc_start[cc];
    if (nch == 0) continue;
    const int nblk = (nch + kAsmWarps - 1) / kAsmWarps;
    P.chunk_base = s.cc_start[cc];
    P.chunk_end = s.cc_start[cc + 1];
    assemble_kernel<MODE><<<nblk, kAsmWarps * 32, smem, st>>>(P); ::gf::count_launch();
    GF_CHECK_LAUNCH();
  }
  return GF_OK;
}

// Cached launch data of a batch's assembly: per-problem parameters (rebuilt
// when a problem's thickness pointer or the flags change) and the work lists.
struct BatchAsm {
  std::vector<AsmParams> host;
  DevBuf<AsmParams> d_params;
  DevBuf<int2> d_work;
  std::vector<int> off;  // work ranges: per colour (coloured) or one (atomic)
  int flags = -1;
};

void batch_asm_free(BatchAsm* b) { delete b; }

gf_status batch_assemble(BatchAsm*& cache, const std::vector<gf_assembler*>& asms,
                         const std::vector<double*>& values, const double* const* thick,
                         int flags, cudaStream_t st) {
  const int np = (int)asms.size();
  if (!cache) cache = new BatchAsm();
  BatchAsm& B = *cache;
  std::vector<AsmParams> h(np);
  for (int k = 0; k < np; k++) {
    gf_assembler* a = asms[k];
    AsmParams& P = h[k];
    std::memset(&P, 0, sizeof(P));
    P.xpts = a->d_xpts.p;
    P.vars = a->d_vars.p;
    P.bcmask = a->d_bcmask.p;
    P.sconn = a->d_sconn.p;
    P.semap = a->d_semap.p;
    P.sft = a->d_sft.p;
    P.sthick = a->d_sthick.p;
    P.smat = a->d_smat.p;
    P.mats = a->d_mats.p;
    P.chunk_start = a->d_chunk_start.p;
    P.thick_nat = thick ? thick[k] : nullptr;
    P.sorder = a->d_sorder.p;
    P.values = values[k];
    P.res = nullptr;
    P.energy_part = a->d_energy_part.p;
    P.flags = flags;
  }
  const bool atomic = (flags & GF_ASSEMBLE_ATOMIC) != 0;
  if (B.flags != flags || B.host.size() != h.size() ||
      std::memcmp(B.host.data(), h.data(), sizeof(AsmParams) * h.size()) != 0) {
    // work items: (problem, chunk), colour by colour, or all chunks at once
    std::vector<int2> work;
    B.off.assign(1, 0);
    if (atomic) {
      for (int k = 0; k < np; k++)
        for (int c = 0; c < asms[k]->sched.nchunks; c++) work.push_back(make_int2(k, c));
      B.off.push_back((int)work.size());
    } else {
      int ncc = 0;
      for (auto* a : asms) ncc = std::max(ncc, a->sched.ncc);
      for (int cc = 0; cc < ncc; cc++) {
        for (int k = 0; k < np; k++) {
          const Schedule& s = asms[k]->sched;
          if (cc >= s.ncc) continue;
          for (int c = s.cc_start[cc]; c < s.cc_start[cc + 1]; c++) work.push_back(make_int2(k, c));
        }
        B.off.push_back((int)work.size());
      }
    }
    GF_CUDA(B.d_work.alloc(work.size()));
    GF_CUDA(B.d_params.alloc(h.size()));
    GF_CUDA(cudaMemcpyAsync(B.d_work.p, work.data(), sizeof(int2) * work.size(),
                            cudaMemcpyHostToDevice, st));
    GF_CUDA(cudaMemcpyAsync(B.d_params.p, h.data(), sizeof(AsmParams) * h.size(),
                            cudaMemcpyHostToDevice, st));
    GF_CUDA(cudaStreamSynchronize(st));  // the host copies are reused
    B.host = h;
    B.flags = flags;
  }
  if (atomic && !(flags & GF_ASSEMBLE_ADD))
    for (int k = 0; k < np; k++)
      GF_CUDA(cudaMemsetAsync(values[k], 0, sizeof(double) * 36 * (size_t)asms[k]->pat.nnz(), st));
  const size_t smem = sizeof(WarpSlot) * kAsmWarps;
  GF_CUDA(cudaFuncSetAttribute(assemble_batch_kernel<MODE_JAC>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (size_t r = 0; r + 1 < B.off.size(); r++) {
    const int nwork = B.off[r + 1] - B.off[r];
    if (nwork == 0) continue;
    assemble_batch_kernel<MODE_JAC><<<(nwork + kAsmWarps - 1) / kAsmWarps, kAsmWarps * 32, smem,
                                      st>>>(B.d_params.p, B.d_work.p + B.off[r], nwork);
    ::gf::count_launch();
    GF_CHECK_LAUNCH();
  }
  return GF_OK;
}

}  // namespace gf

using namespace gf;

// ------------------------------------------------------------------ C ABI
extern "C" {

gf_status gf_assembler_create(const gf_mesh_desc* d, gf_assembler** out) {
  if (!d || !out || d->num_nodes <= 0 || d->num_elements <= 0 || !d->conn || !d->xpts ||
      !d->data || (d->num_bcs > 0 && !d->bcs))
    return GF_INVALID_ARG;
  *out = nullptr;
  const int nn = d->num_nodes, ne = d->num_elements;
  for (size_t i = 0; i < (size_t)4 * ne; i++)
    if (d->conn[i] < 0 || d->conn[i] >= nn) return GF_INVALID_ARG;
  for (int e = 0; e < ne; e++)
    for (int x = 0; x < 4; x++)
      for (int y = x + 1; y < 4; y++)
        if (d->conn[4 * e + x] == d->conn[4 * e + y]) return GF_INVALID_ARG;
  for (int i = 0; i < d->num_bcs; i++)
    if (d->bcs[i] < 0 || d->bcs[i] >= 6 * nn) return GF_INVALID_ARG;
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return GF_NO_DEVICE;

  gf_assembler* a = new gf_assembler();
  a->nnodes = nn;
  a->nelem = ne;
  a->nbcs = d->num_bcs;
  a->conn.assign(d->conn, d->conn + 4 * (size_t)ne);
  a->bcs.assign(d->bcs, d->bcs + d->num_bcs);
  if (pattern_from_conn_gpu(ne, nn, d->conn, a->pat0))
    a->sym_flags |= 1;
  else
    a->pat0 = pattern_from_conn(ne, nn, d->conn);
  order_nodes(a->pat0, d, a->perm);
  a->iperm.resize(nn);
  for (int i = 0; i < nn; i++) a->iperm[a->perm[i]] = i;
  a->pat = permute_pattern(a->pat0, a->perm);
  if (elem_ind_map_gpu(ne, d->conn, a->pat, a->perm, a->emap))
    a->sym_flags |= 2;
  else
    elem_ind_map(ne, d->conn, a->pat, a->perm, a->emap);
  if (build_schedule(ne, nn, d->conn, a->emap, a->pat.nnz(), kChunkSize, a->sched) != 0) {
    delete a;
    return GF_INVALID_ARG;
  }
  // materials: dedupe (E, nu, tOffset, refAxis) per element; thickness per element
  std::vector<int32_t> emat(ne);
  std::vector<double> thick(ne);
  for (int e = 0; e < ne; e++) {
    const gf_shell_data& sd = d->data[e];
    thick[e] = sd.thick;
    Material m{sd.E, sd.nu, sd.tOffset, {sd.refAxis[0], sd.refAxis[1], sd.refAxis[2]},
               sd.has_ref_axis ? 1 : 0, 0};
    int found = -1;
    for (size_t k = 0; k < a->mats.size(); k++) {
      const Material& o = a->mats[k];
      if (o.E == m.E && o.nu == m.nu && o.tOffset == m.tOffset &&
          o.has_ref_axis == m.has_ref_axis && o.refAxis[0] == m.refAxis[0] &&
          o.refAxis[1] == m.refAxis[1] && o.refAxis[2] == m.refAxis[2]) {
        found = (int)k;
        break;
      }
    }
    if (found < 0) {
      found = (int)a->mats.size();
      a->mats.push_back(m);
    }
    emat[e] = found;
  }
  const Schedule& s = a->sched;
  std::vector<int32_t> sconn((size_t)4 * ne), semap((size_t)16 * ne), smat(ne);
  std::vector<uint32_t> sft(ne);
  std::vector<double> sthick(ne);
  for (int k = 0; k < ne; k++) {
    const int e = s.order[k];
    for (int x = 0; x < 4; x++) sconn[4 * k + x] = d->conn[4 * e + x];
    for (int x = 0; x < 16; x++) semap[16 * k + x] = a->emap[16 * e + x];
    sft[k] = s.first_touch[e];
    sthick[k] = thick[e];
    smat[k] = emat[e];
  }
  std::vector<uint8_t> bcmask(nn, 0);
  for (int i = 0; i < d->num_bcs; i++) bcmask[d->bcs[i] / 6] |= (uint8_t)(1u << (d->bcs[i] % 6));
  // BC entry list (solver order): rows of constrained DOFs and the matching columns
  std::vector<int32_t> ent;
  const Pattern& P = a->pat;
  for (int i = 0; i < d->num_bcs; i++) {
    const int node = a->perm[d->bcs[i] / 6], inner = d->bcs[i] % 6;
    for (int jp = P.rowp[node]; jp < P.rowp[node + 1]; jp++) {
      ent.insert(ent.end(), {jp, node, 0, inner});
      const int j = P.cols[jp];  // symmetric pattern: block (j, node) exists
      const int32_t* b0 = P.cols.data() + P.rowp[j];
      const int32_t* b1 = P.cols.data() + P.rowp[j + 1];
      const int32_t* f = std::lower_bound(b0, b1, node);
      ent.insert(ent.end(), {(int32_t)(f - P.cols.data()), j, 1, inner});
    }
  }
  a->nbc_entries = (int)(ent.size() / 4);
  std::vector<int32_t> diag(nn);
  for (int i = 0; i < nn; i++) {
    const int32_t* b0 = P.cols.data() + P.rowp[i];
    const int32_t* b1 = P.cols.data() + P.rowp[i + 1];
    diag[i] = (int32_t)(std::lower_bound(b0, b1, i) - P.cols.data());
  }
  gf_status st = GF_OK;
  auto up = [&](cudaError_t e) {
    if (e != cudaSuccess && st == GF_OK) {
      set_last_error("gf_assembler_create upload", e);
      st = (e == cudaErrorMemoryAllocation) ? GF_OOM : GF_CUDA_ERROR;
    }
  };
  up(a->d_xpts.upload(d->xpts, (size_t)3 * nn));
  up(a->d_vars.alloc((size_t)6 * nn));
  if (st == GF_OK) up(cudaMemset(a->d_vars.p, 0, sizeof(double) * 6 * nn));
  up(a->d_perm.upload(a->perm));
  up(a->d_bcs.upload(a->bcs));
  up(a->d_bcmask.upload(bcmask));
  up(a->d_sconn.upload(sconn));
  up(a->d_semap.upload(semap));
  up(a->d_smat.upload(smat));
  up(a->d_sft.upload(sft));
  up(a->d_sthick.upload(sthick));
  up(a->d_sorder.upload(s.order));
  up(a->d_chunk_start.upload(s.chunk_start));
  up(a->d_mats.upload(a->mats));
  up(a->d_rowp.upload(P.rowp));
  up(a->d_cols.upload(P.cols));
  up(a->d_bc_entries.upload(ent));
  up(a->d_energy_part.alloc(s.nchunks + 1));
  up(a->d_diag.upload(diag));
  if (st != GF_OK) {
    delete a;
    return st;
  }
  *out = a;
  return GF_OK;
}

gf_status gf_assembler_destroy(gf_assembler* a) {
  delete a;
  return GF_OK;
}

int32_t gf_assembler_num_nodes(const gf_assembler* a) { return a ? a->nnodes : 0; }
int32_t gf_assembler_num_elements(const gf_assembler* a) { return a ? a->nelem : 0; }
int32_t gf_assembler_num_vars(const gf_assembler* a) { return a ? 6 * a->nnodes : 0; }
int32_t gf_assembler_nnzb(const gf_assembler* a) { return a ? a->pat.nnz() : 0; }

gf_status gf_assembler_get_pattern(const gf_assembler* a, int32_t* rowPtr, int32_t* colPtr,
                                   int32_t* perm, int32_t* elemIndMap) {
  if (!a) return GF_INVALID_ARG;
  if (rowPtr) std::copy(a->pat.rowp.begin(), a->pat.rowp.end(), rowPtr);
  if (colPtr) std::copy(a->pat.cols.begin(), a->pat.cols.end(), colPtr);
  if (perm) std::copy(a->perm.begin(), a->perm.end(), perm);
  if (elemIndMap) std::copy(a->emap.begin(), a->emap.end(), elemIndMap);
  return GF_OK;
}

gf_status gf_assembler_get_schedule(const gf_assembler* a, int32_t* elem_chunk,
                                    int32_t* chunk_color, int32_t* elem_color,
                                    uint32_t* first_touch, int32_t* num_chunk_colors,
                                    int32_t* num_chunks) {
  if (!a) return GF_INVALID_ARG;
  const Schedule& s = a->sched;
  if (elem_chunk) std::copy(s.elem_chunk.begin(), s.elem_chunk.end(), elem_chunk);
  if (chunk_color) std::copy(s.chunk_color.begin(), s.chunk_color.end(), chunk_color);
  if (elem_color) std::copy(s.elem_color.begin(), s.elem_color.end(), elem_color);
  if (first_touch) std::copy(s.first_touch.begin(), s.first_touch.end(), first_touch);
  if (num_chunk_colors) *num_chunk_colors = s.ncc;
  if (num_chunks) *num_chunks = s.nchunks;
  return GF_OK;
}

gf_status gf_set_variables(gf_assembler* a, const double* d_vars, void* stream) {
  if (!a || !d_vars) return GF_INVALID_ARG;
  GF_CUDA(cudaMemcpyAsync(a->d_vars.p, d_vars, sizeof(double) * 6 * a->nnodes,
                          cudaMemcpyDeviceToDevice, as_stream(stream)));
  return GF_OK;
}

gf_status gf_add_residual(gf_assembler* a, double* d_res, int32_t flags, void* stream) {
  if (!a || !d_res) return GF_INVALID_ARG;
  return launch_assembly<MODE_RES>(a, nullptr, d_res, flags, as_stream(stream));
}

gf_status gf_assembler_setup_info(const gf_assembler* a, int32_t* pattern_on_gpu,
                                  int32_t* elem_map_on_gpu) {
  if (!a) return GF_INVALID_ARG;
  if (pattern_on_gpu) *pattern_on_gpu = (a->sym_flags & 1) ? 1 : 0;
  if (elem_map_on_gpu) *elem_map_on_gpu = (a->sym_flags & 2) ? 1 : 0;
  return GF_OK;
}

gf_status gf_add_jacobian(gf_assembler* a, double* d_res, gf_bsr* mat, int32_t flags,
                          void* stream) {
  if (!a || !mat || mat->a != a) return GF_INVALID_ARG;
  return launch_assembly<MODE_JAC>(a, mat->vals.p, d_res, flags, as_stream(stream));
}

gf_status gf_add_jacobian_thick(gf_assembler* a, const double* d_thick, double* d_res,
                                gf_bsr* mat, int32_t flags, void* stream) {
  if (!a || !mat || mat->a != a || !d_thick) return GF_INVALID_ARG;
  return launch_assembly<MODE_JAC>(a, mat->vals.p, d_res, flags, as_stream(stream), d_thick);
}

gf_status gf_add_energy(gf_assembler* a, double* h_energy, void* stream) {
  if (!a || !h_energy) return GF_INVALID_ARG;
  cudaStream_t st = as_stream(stream);
  gf_status s = launch_assembly<MODE_ENERGY>(a, nullptr, nullptr, 0, st);
  if (s != GF_OK) return s;
  sum_kernel<<<1, 256, 0, st>>>(a->d_energy_part.p, a->sched.nchunks,
                                a->d_energy_part.p + a->sched.nchunks); ::gf::count_launch();
  GF_CHECK_LAUNCH();
  GF_CUDA(cudaMemcpyAsync(h_energy, a->d_energy_part.p + a->sched.nchunks, sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  GF_CUDA(cudaStreamSynchronize(st));
  return GF_OK;
}

gf_status gf_assembler_set_thickness(gf_assembler* a, const double* d_thick, void* stream) {
  if (!a || !d_thick) return GF_INVALID_ARG;
  gather_thickness<<<(a->nelem + 255) / 256, 256, 0, as_stream(stream)>>>(
      a->d_sorder.p, a->nelem, d_thick, a->d_sthick.p); ::gf::count_launch();
  GF_CHECK_LAUNCH();
  return GF_OK;
}

gf_status gf_apply_bcs_vec(gf_assembler* a, double* d_vec, void* stream) {
  if (!a || !d_vec) return GF_INVALID_ARG;
  if (a->nbcs == 0) return GF_OK;
  bc_vec_kernel<<<(a->nbcs + 255) / 256, 256, 0, as_stream(stream)>>>(a->d_bcs.p, a->nbcs,
                                                                      d_vec); ::gf::count_launch();
  GF_CHECK_LAUNCH();
  return GF_OK;
}

gf_status gf_apply_bcs_mat(gf_assembler* a, gf_bsr* mat, void* stream) {
  if (!a || !mat || mat->a != a) return GF_INVALID_ARG;
  if (a->nbc_entries == 0) return GF_OK;
  bc_mat_kernel<<<(a->nbc_entries + 127) / 128, 128, 0, as_stream(stream)>>>(
      a->d_bc_entries.p, a->nbc_entries, a->d_cols.p, mat->vals.p); ::gf::count_launch();
  GF_CHECK_LAUNCH();
  return GF_OK;
}

gf_status gf_bsr_create(gf_assembler* a, gf_bsr** out) {
  if (!a || !out) return GF_INVALID_ARG;
  gf_bsr* m = new gf_bsr();
  m->a = a;
  cudaError_t e = m->vals.alloc((size_t)36 * a->pat.nnz());
  if (e == cudaSuccess) e = cudaMemset(m->vals.p, 0, sizeof(double) * 36 * a->pat.nnz());
  if (e != cudaSuccess) {
    set_last_error("gf_bsr_create", e);
    delete m;
    return e == cudaErrorMemoryAllocation ? GF_OOM : GF_CUDA_ERROR;
  }
  *out = m;
  return GF_OK;
}

gf_status gf_bsr_destroy(gf_bsr* m) {
  delete m;
  return GF_OK;
}

double* gf_bsr_values(gf_bsr* m) { return m ? m->vals.p : nullptr; }

gf_status gf_bsr_zero(gf_bsr* m, void* stream) {
  if (!m) return GF_INVALID_ARG;
  GF_CUDA(cudaMemsetAsync(m->vals.p, 0, sizeof(double) * m->vals.n, as_stream(stream)));
  return GF_OK;
}

gf_status gf_permute_vec(gf_assembler* a, const double* d_in, double* d_out, int32_t dir,
                         void* stream) {
  if (!a || !d_in || !d_out || d_in == d_out || (dir != 0 && dir != 1)) return GF_INVALID_ARG;
  const int n = 6 * a->nnodes;
  permute_kernel<<<(n + 255) / 256, 256, 0, as_stream(stream)>>>(a->d_perm.p, a->nnodes, d_in,
                                                                  d_out, dir); ::gf::count_launch();
  GF_CHECK_LAUNCH();
  return GF_OK;
}

}  // extern "C"
