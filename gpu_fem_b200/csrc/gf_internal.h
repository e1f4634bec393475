// Internal definitions shared by the libgpufem translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/gpufem.h"
#include "shell_element.cuh"

namespace gf {

// Thread-local text of the last CUDA error seen by the library.
void set_last_error(const char* where, cudaError_t e);
void set_last_error_text(const std::string& text);
// Process-wide count of kernels this library has launched.
void count_launch();

#define GF_CUDA(call)                                  \
  do {                                                 \
    cudaError_t _e = (call);                           \
    if (_e != cudaSuccess) {                           \
      ::gf::set_last_error(#call, _e);                 \
      return _e == cudaErrorMemoryAllocation ? GF_OOM : GF_CUDA_ERROR; \
    }                                                  \
  } while (0)

#define GF_CHECK_LAUNCH()                              \
  do {                                                 \
    cudaError_t _e = cudaGetLastError();               \
    if (_e != cudaSuccess) {                           \
      ::gf::set_last_error("kernel launch", _e);       \
      return GF_CUDA_ERROR;                            \
    }                                                  \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Device buffer that frees itself.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    release();
    n = count;
    if (count == 0) return cudaSuccess;
    return cudaMalloc(&p, count * sizeof(T));
  }
  cudaError_t upload(const T* h, size_t count) {
    cudaError_t e = alloc(count);
    if (e != cudaSuccess || count == 0) return e;
    return cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice);
  }
  cudaError_t upload(const std::vector<T>& v) { return upload(v.data(), v.size()); }
};

// ---------------------------------------------------------------- symbolic
struct Pattern {
  int n = 0;
  std::vector<int32_t> rowp, cols;
  int nnz() const { return rowp.empty() ? 0 : rowp[n]; }
};

// Node adjacency through shared elements (get_row_col_ptrs,
// include/linalg/bsr_utils.h:430-476).
Pattern pattern_from_conn(int nelem, int nnodes, const int32_t* conn);
// TacsComputeRCMOrder (include/linalg/reordering_utils.h:189-291): rcm[old] = new.
void rcm_order(const Pattern& p, int root, int iters, std::vector<int32_t>& rcm);
Pattern permute_pattern(const Pattern& p, const std::vector<int32_t>& perm);
int bandwidth(const Pattern& p);
// deterministic q-ordering on top of an RCM order (examples/iterative/gmres.cu:159-215)
void qorder(const Pattern& p, const std::vector<int32_t>& rcm, double pfac, uint64_t seed,
            std::vector<int32_t>& out);
// node ordering of a mesh description (GF_ORDER_*): perm[old] = new
void order_nodes(const Pattern& p, const gf_mesh_desc* d, std::vector<int32_t>& perm);
// get_elem_ind_map (include/linalg/bsr_utils.h:809-870); -1 if not found.
void elem_ind_map(int nelem, const int32_t* conn, const Pattern& p,
                  const std::vector<int32_t>& perm, std::vector<int32_t>& map);
// computeILUk (include/linalg/bsr_utils.h:678-807).
Pattern iluk_pattern(const Pattern& a, int lev);
// The same pattern computed on the GPU (symbolic_gpu.cu); false when a row's
// column window exceeds the kernel's or the device fails, and the caller
// then uses iluk_pattern.
bool iluk_pattern_gpu(const Pattern& a, int lev, Pattern& out);
// The node pattern and elemIndMap computed on the GPU (symbolic_gpu.cu):
// false when a node has more than 64 elements or the device fails, and the
// caller then uses pattern_from_conn / elem_ind_map.
bool pattern_from_conn_gpu(int nelem, int nnodes, const int32_t* conn, Pattern& out);
bool elem_ind_map_gpu(int nelem, const int32_t* conn, const Pattern& p,
                      const std::vector<int32_t>& perm, std::vector<int32_t>& map);
// Level sets of the lower / upper triangular DAG.
int levels(const Pattern& p, bool lower, std::vector<int32_t>& level);

// Coloured scatter schedule (this project's design; restated in the oracle).
struct Schedule {
  int chunk_size = 0;
  int nchunks = 0, ncc = 0;      // chunks, chunk colours
  int max_ec = 0;                // element colours (max over chunks)
  std::vector<int32_t> elem_chunk, chunk_color, elem_color;
  std::vector<uint32_t> first_touch;  // bits 0-15 blocks (4a+b), 16-19 nodes
  // execution order
  std::vector<int32_t> order;         // schedule position -> element
  std::vector<int32_t> chunk_list;    // chunks sorted by (colour, id)
  std::vector<int32_t> cc_start;      // [ncc+1] offsets into chunk_list
  std::vector<int32_t> chunk_start;   // [nchunks+1] schedule offsets (in chunk_list order)
};
constexpr int kMaxEC = 15;

// Level-major chunk stream of one triangle (L or U) of a block ILU factor.
// Rows are grouped by level and cut into chunks (a chunk never spans two
// levels; at most capb blocks and capr rows). Chunk c is one contiguous,
// 16-byte aligned byte range [off[c], off[c+1]) of `stream`:
//   int4 header {nrows, nblocks, 0, 0}
//   nrows x int4 {row, first block (chunk-local), blocks, 0}
//   nblocks x int32 column (problem-local block row)
//   nblocks x 36 values (row-major 6x6, factor precision)
// so one bulk copy brings everything a chunk's solve needs into shared
// memory. nblocks is a non-zero multiple of 4 (zero padding blocks). For U
// every row starts with its U_ii^{-1} block.
//
// A triangle solved by the dataflow sweep (kind TRI_DATAFLOW) has a simpler
// stream: rows in level order (position p = 0..n-1) cut into chunks of
// consecutive positions (at most capb blocks and capr rows), chunk c being
//   int4 header {nrows, nblocks, first position, 0}
//   nrows x int4 {row, first block (chunk-local), blocks, 0}
//   nblocks x int32 position of the row each block multiplies (-1 for U's
//     leading U_ii^{-1} block and for padding), ascending within a row
//   (16-byte aligned) nblocks x 36 values
// and a row's x entries come from a shared-memory ring of the latest `ring`
// positions' results (ring > 2 maxdist, maxdist = the largest position
// distance between a row and a row it multiplies).
enum { TRI_LEVEL = 0, TRI_DATAFLOW = 1 };
struct TriDesc {
  int nch;                       // chunks
  int stage;                     // bytes of the largest chunk (staging buffer size)
  int capb, capr;                // blocks / rows per chunk at most
  const int64_t* off;            // level: [2 (nch+1)] byte offsets of the two halves'
                                 // chunks; dataflow: [nch+1]
  const unsigned char* stream;
  long long abytes;              // algorithmic bytes of one sweep (for timing)
  int nsplit;                    // level: CTAs that share each chunk's rows (1 or 2)
  int kind;                      // TRI_LEVEL or TRI_DATAFLOW
  int ring, maxdist;             // dataflow: ring slots (a power of two), dependency reach
};

// Per-problem descriptor used by the batched solver kernels: block rows,
// offset of the problem in the batch vector space (in block rows), the
// matrix pattern and values (FP64 and the FP32 copy of the mixed mode), the
// ILU pattern and factor values, and the factor's chunk streams.
struct ProbDev {
  int n, off;
  const int32_t* rowp;
  const int32_t* cols;
  const double* A64;
  const float* A32;
  const int32_t* prowp;
  const int32_t* pcols;
  const int32_t* pdiag;
  double* LU64;              // factor in ILU-pattern order (FP64)
  int nlevL, nlevU;          // triangular levels
  int32_t* done;             // per row: epoch of the factorization that finished it
  const int32_t* pord;       // per row: slots of its lower blocks in factorization-step order
  const int32_t* levLptr;    // rows grouped by lower level (factorization order)
  const int32_t* levLrows;
  TriDesc L, U;              // chunk streams of the factor for the sweeps
};
// Batched Jacobian assembly with fused BCs (assembly.cu): one launch per
// colour over all problems, or one launch with GF_ASSEMBLE_ATOMIC; `cache`
// holds the launch data between calls (batch_asm_free releases it).
struct BatchAsm;
void batch_asm_free(BatchAsm* b);
int build_schedule(int nelem, int nnodes, const int32_t* conn, const std::vector<int32_t>& emap,
                   int nnzb, int chunk_size, Schedule& s);

}  // namespace gf

// ------------------------------------------------------------------ handles
struct gf_assembler {
  int nnodes = 0, nelem = 0, nbcs = 0;
  int sym_flags = 0;                // bit 0: node pattern, bit 1: elemIndMap computed on the GPU
  gf::Pattern pat0;                 // natural pattern
  gf::Pattern pat;                  // solver-order pattern
  std::vector<int32_t> perm, iperm;
  std::vector<int32_t> conn;        // natural
  std::vector<int32_t> bcs;
  std::vector<int32_t> emap;        // natural element order
  gf::Schedule sched;
  std::vector<gf::Material> mats;
  // device: natural-order mesh
  gf::DevBuf<double> d_xpts, d_vars;
  gf::DevBuf<int32_t> d_perm, d_bcs;
  gf::DevBuf<uint8_t> d_bcmask;     // per natural node, bit r = DOF r constrained
  // device: schedule-ordered element data
  gf::DevBuf<int32_t> d_sconn, d_semap, d_smat;
  gf::DevBuf<uint32_t> d_sft;
  gf::DevBuf<double> d_sthick;
  gf::DevBuf<int32_t> d_sorder;     // schedule position -> element
  gf::DevBuf<int32_t> d_chunk_list, d_chunk_start;
  gf::DevBuf<gf::Material> d_mats;
  // device: pattern (solver order) and BC entry list
  gf::DevBuf<int32_t> d_rowp, d_cols;
  gf::DevBuf<int32_t> d_bc_entries;  // 4 ints per entry: blk, row node, is_col, inner
  int nbc_entries = 0;
  gf::DevBuf<double> d_energy_part;
  gf::DevBuf<int32_t> d_diag;        // solver-order diagonal block index per row
};

struct gf_bsr {
  gf_assembler* a = nullptr;
  gf::DevBuf<double> vals;
  gf::DevBuf<float> vals32;           // FP32 copy for the mixed-precision SpMV
  gf::DevBuf<gf::ProbDev> desc;       // one-entry table for gf_bsr_spmv
  gf::DevBuf<int32_t> rowprob;
};

namespace gf {
gf_status batch_assemble(BatchAsm*& cache, const std::vector<gf_assembler*>& asms,
                         const std::vector<double*>& values, const double* const* thick, int flags,
                         cudaStream_t st);
}  // namespace gf
