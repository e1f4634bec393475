// Shell residual / Jacobian / energy assembly kernels and their C ABI.
//
// Reference: add_residual_gpu / add_jacobian_gpu (include/base/elem_group.cuh:17-211)
// launch one thread per (element, quadrature point[, Jacobian column]) and
// scatter with FP64 atomicAdd (include/linalg/vec.h:278-293,
// include/linalg/bsr_mat.h:229-276).
//
// Here one warp owns one element:
//   * node coordinates and DOFs are gathered once into the warp's shared
//     memory slot, the per-element geometry (normals, nodal frames, the four
//     quadrature-point frames, the tying-point vectors) is spread over lanes;
//   * lane l < 24 builds column l of the four 9x24 strain matrices B_q and
//     keeps D B_q[:, l] in registers; column l of K_e = sum_q B_q^T D B_q is
//     a 36-term product against the shared B (broadcast reads);
//   * the scatter follows the coloured schedule built on the host: one CTA
//     per chunk, chunks of one colour per launch, element colours separated
//     by __syncthreads(). The first toucher of a block stores, later touchers
//     read-modify-write; there are no atomics and the result is bitwise
//     reproducible.
#include <cstdio>

#include "gf_internal.h"

namespace gf {

constexpr int kAsmWarps = 4;

struct WarpSlot {
  double X[12];
  double U[24];
  ElemGeom g;
  double Bt[36][24];
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
  const int32_t* ec_off;
  int chunk_base;
  double* values;
  double* res;
  double* energy_part;
  int flags;
};

enum { MODE_JAC = 0, MODE_RES = 1, MODE_ENERGY = 2 };

template <int MODE>
__device__ void process_element(int s, WarpSlot& w, const AsmParams& P, int lane,
                                double& energy_acc) {
  const int4 cn = reinterpret_cast<const int4*>(P.sconn)[s];
  const int nodes[4] = {cn.x, cn.y, cn.z, cn.w};
  if (lane < 12) w.X[lane] = P.xpts[3 * nodes[lane / 3] + lane % 3];
  if (lane < 24) w.U[lane] = P.vars ? P.vars[6 * nodes[lane / 6] + lane % 6] : 0.0;
  const Material m = P.mats[P.smat ? P.smat[s] : 0];
  const double t = P.sthick[s];
  __syncwarp();
  if (lane < 4) geom_normal(w.X, lane, &w.g.fn[3 * lane]);
  __syncwarp();
  if (lane < 4) {
    geom_node(m, w.X, w.g.fn, lane, w.g.Tn01[lane], w.g.XTn[lane], w.g.tcross[lane]);
  } else if (lane < 8) {
    const int q = lane - 4;
    geom_quad(m, w.X, w.g.fn, q, w.g.T[q], w.g.A[q], w.g.Az[q], w.g.scale[q]);
  } else if (lane < 13) {
    geom_tying(w.X, w.g.fn, lane - 8, w.g);
  }
  __syncwarp();
  double Bc[36];
  if (lane < 24) {
    bmat_column(w.g, lane, Bc);
#pragma unroll
    for (int k = 0; k < 36; k++) w.Bt[k][lane] = Bc[k];
  }
  __syncwarp();

  const bool fuse = (P.flags & GF_ASSEMBLE_FUSE_BCS) != 0;
  const bool add = (P.flags & GF_ASSEMBLE_ADD) != 0;
  const uint32_t ft = P.sft[s];
  uint32_t bcm[4] = {0, 0, 0, 0};
  if (fuse)
    for (int a = 0; a < 4; a++) bcm[a] = P.bcmask[nodes[a]];

  double rj = 0.0;  // residual entry of DOF `lane`
  if (MODE == MODE_JAC) {
    if (lane < 24) {
      // D B_q[:, lane] in place
#pragma unroll
      for (int q = 0; q < 4; q++) {
        double Sq[9];
        stress(m, t, w.g.scale[q], &Bc[9 * q], Sq);
#pragma unroll
        for (int k = 0; k < 9; k++) Bc[9 * q + k] = Sq[k];
      }
      double acc[24];
#pragma unroll
      for (int i = 0; i < 24; i++) acc[i] = 0.0;
#pragma unroll 4
      for (int qk = 0; qk < 36; qk++) {
        const double d = Bc[qk];
        const double2* row = reinterpret_cast<const double2*>(&w.Bt[qk][0]);
#pragma unroll
        for (int i = 0; i < 12; i++) {
          const double2 b = row[i];
          acc[2 * i] = fma(b.x, d, acc[2 * i]);
          acc[2 * i + 1] = fma(b.y, d, acc[2 * i + 1]);
        }
      }
      // acc[i] = K[i][lane] = K[lane][i]
#pragma unroll
      for (int i = 0; i < 24; i++) rj = fma(acc[i], w.U[i], rj);
      if (P.values) {
        const int b = lane / 6, c = lane % 6;
        const bool cbc = (bcm[b] >> c) & 1;
#pragma unroll
        for (int a = 0; a < 4; a++) {
          const int blk = P.semap[16 * s + 4 * a + b];
          double* dst = P.values + 36 * (size_t)blk + c;
          const bool first = (ft >> (4 * a + b)) & 1;
#pragma unroll
          for (int r = 0; r < 6; r++) {
            double v = acc[6 * a + r];
            if (fuse && (cbc || ((bcm[a] >> r) & 1))) v = (a == b && r == c && first) ? 1.0 : 0.0;
            if (first && !add)
              dst[6 * r] = v;
            else
              dst[6 * r] += v;
          }
        }
      }
    }
  } else {
    // E_q = B_q u (36 entries over 32 lanes), S_q = D E_q, R = sum_q B_q^T S_q
    for (int k = lane; k < 36; k += 32) {
      double e = 0.0;
#pragma unroll
      for (int l = 0; l < 24; l++) e = fma(w.Bt[k][l], w.U[l], e);
      w.E[k] = e;
    }
    __syncwarp();
    if (lane < 4) stress(m, t, w.g.scale[lane], &w.E[9 * lane], &w.S[9 * lane]);
    __syncwarp();
    if (MODE == MODE_ENERGY) {
      if (lane == 0) {
        double U = 0.0;
        for (int k = 0; k < 36; k++) U += 0.5 * w.E[k] * w.S[k];
        energy_acc += U;
      }
    } else if (lane < 24) {
#pragma unroll
      for (int k = 0; k < 36; k++) rj = fma(w.Bt[k][lane], w.S[k], rj);
    }
  }
  if (MODE != MODE_ENERGY && P.res && lane < 24) {
    const int b = lane / 6, c = lane % 6;
    if (fuse && ((bcm[b] >> c) & 1)) rj = 0.0;
    double* dst = P.res + 6 * (size_t)nodes[b] + c;
    const bool first = (ft >> (16 + b)) & 1;
    if (first && !add)
      *dst = rj;
    else
      *dst += rj;
  }
  __syncwarp();
}

template <int MODE>
__global__ void __launch_bounds__(kAsmWarps * 32)
    assemble_kernel(AsmParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSlot* slots = reinterpret_cast<WarpSlot*>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int li = P.chunk_base + blockIdx.x;
  const int s0 = P.chunk_start[li];
  const int32_t* off = &P.ec_off[(size_t)li * (kMaxEC + 1)];
  double energy_acc = 0.0;
  for (int col = 0; col < kMaxEC; col++) {
    const int b = off[col], e = off[col + 1];
    if (b == e) continue;
    for (int k = b + warp; k < e; k += kAsmWarps)
      process_element<MODE>(s0 + k, slots[warp], P, lane, energy_acc);
    __syncthreads();
  }
  if (MODE == MODE_ENERGY) {
    __shared__ double part[kAsmWarps];
    if (lane == 0) part[warp] = energy_acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double sum = 0.0;
      for (int w = 0; w < kAsmWarps; w++) sum += part[w];
      P.energy_part[li] = sum;
    }
  }
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
                                 cudaStream_t st) {
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
  P.ec_off = a->d_ec_off.p;
  P.values = values;
  P.res = res;
  P.energy_part = a->d_energy_part.p;
  P.flags = flags;
  const size_t smem = sizeof(WarpSlot) * kAsmWarps;
  static bool attr_set[3] = {false, false, false};
  if (!attr_set[MODE]) {
    GF_CUDA(cudaFuncSetAttribute(assemble_kernel<MODE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set[MODE] = true;
  }
  const Schedule& s = a->sched;
  for (int cc = 0; cc < s.ncc; cc++) {
    const int nblk = s.cc_start[cc + 1] - s.cc_start[cc];
    if (nblk == 0) continue;
    P.chunk_base = s.cc_start[cc];
    assemble_kernel<MODE><<<nblk, kAsmWarps * 32, smem, st>>>(P);
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
  a->pat0 = pattern_from_conn(ne, nn, d->conn);
  if (d->ordering == GF_ORDER_RCM) {
    rcm_order(a->pat0, d->rcm_root, 1, a->perm);
  } else {
    a->perm.resize(nn);
    for (int i = 0; i < nn; i++) a->perm[i] = i;
  }
  a->iperm.resize(nn);
  for (int i = 0; i < nn; i++) a->iperm[a->perm[i]] = i;
  a->pat = permute_pattern(a->pat0, a->perm);
  elem_ind_map(ne, d->conn, a->pat, a->perm, a->emap);
  if (build_schedule(ne, nn, d->conn, a->emap, a->pat.nnz(), 32, a->sched) != 0) {
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
  up(a->d_chunk_start.upload(s.chunk_start));
  up(a->d_ec_off.upload(s.ec_off));
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

gf_status gf_add_jacobian(gf_assembler* a, double* d_res, gf_bsr* mat, int32_t flags,
                          void* stream) {
  if (!a || !mat || mat->a != a) return GF_INVALID_ARG;
  return launch_assembly<MODE_JAC>(a, mat->vals.p, d_res, flags, as_stream(stream));
}

gf_status gf_add_energy(gf_assembler* a, double* h_energy, void* stream) {
  if (!a || !h_energy) return GF_INVALID_ARG;
  cudaStream_t st = as_stream(stream);
  gf_status s = launch_assembly<MODE_ENERGY>(a, nullptr, nullptr, 0, st);
  if (s != GF_OK) return s;
  sum_kernel<<<1, 256, 0, st>>>(a->d_energy_part.p, a->sched.nchunks,
                                a->d_energy_part.p + a->sched.nchunks);
  GF_CHECK_LAUNCH();
  GF_CUDA(cudaMemcpyAsync(h_energy, a->d_energy_part.p + a->sched.nchunks, sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  GF_CUDA(cudaStreamSynchronize(st));
  return GF_OK;
}

gf_status gf_apply_bcs_vec(gf_assembler* a, double* d_vec, void* stream) {
  if (!a || !d_vec) return GF_INVALID_ARG;
  if (a->nbcs == 0) return GF_OK;
  bc_vec_kernel<<<(a->nbcs + 255) / 256, 256, 0, as_stream(stream)>>>(a->d_bcs.p, a->nbcs,
                                                                      d_vec);
  GF_CHECK_LAUNCH();
  return GF_OK;
}

gf_status gf_apply_bcs_mat(gf_assembler* a, gf_bsr* mat, void* stream) {
  if (!a || !mat || mat->a != a) return GF_INVALID_ARG;
  if (a->nbc_entries == 0) return GF_OK;
  bc_mat_kernel<<<(a->nbc_entries + 127) / 128, 128, 0, as_stream(stream)>>>(
      a->d_bc_entries.p, a->nbc_entries, a->d_cols.p, mat->vals.p);
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
                                                                  d_out, dir);
  GF_CHECK_LAUNCH();
  return GF_OK;
}

}  // extern "C"
