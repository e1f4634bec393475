// C++ facade over the C ABI (include/gpufem.h) that keeps the reference's
// class templates, method names and argument orders, so driver code written
// against smdogroup/gpu_fem ports by adding `using namespace gpufem;`:
//   element-group composition   examples/plate_demo/linear_static.cu:17-27
//     (QuadLinearQuadrature, LinearizedRotation, ShellQuadBasis,
//      ShellIsotropicData, IsotropicShell, ShellElementGroup: type tags that
//      select the library's MITC4 linear shell, include/shell/*)
//   ElementAssembler<T, ElemGroup, Vec, Mat>   include/assembler.h:14-322
//   BsrData (host copy)          include/linalg/bsr_utils.h:43-404
//   BsrMat<Vec>, createBsrMat    include/linalg/bsr_mat.h:9-357
//   DeviceVec, HostVec, VecType  include/linalg/vec.h:146-394
//   ILUk_Preconditioner          include/linalg/precond.h:5-55
//   CUSPARSE::direct_LU_solve_old  include/linalg/solvers/cusparse.h:16-192
//   gmres_solve                  examples/iterative/gmres.cu:468-771 (driver code)
// Differences: errors throw gpufem::Error instead of calling exit();
// handles own their memory (the reference's destructors are commented out,
// vec.h:180-186); vectors at the boundary are in natural node order and the
// solver ordering is applied inside; can_print flags are accepted and print
// nothing; TACSMeshLoader reads the 4-node shell subset of BDF input.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../gpufem.h"

namespace gpufem {

struct Error : std::runtime_error {
  gf_status status;
  Error(gf_status s, const std::string& where)
      : std::runtime_error(where + ": " + gf_status_string(s) + " " + gf_last_error()),
        status(s) {}
};
inline void check(gf_status s, const char* where) {
  if (s != GF_OK) throw Error(s, where);
}

template <typename T>
class DeviceVec;

template <typename T>
class HostVec {
 public:
  HostVec() = default;
  explicit HostVec(int n, const T* data = nullptr) : v_(n) {
    if (data) std::copy(data, data + n, v_.begin());
  }
  T* getPtr() { return v_.data(); }
  const T* getPtr() const { return v_.data(); }
  int getSize() const { return (int)v_.size(); }
  T& operator[](int i) { return v_[i]; }
  const T& operator[](int i) const { return v_[i]; }
  void zeroValues() { std::fill(v_.begin(), v_.end(), T(0)); }
  void copyValuesTo(HostVec& o) const { std::copy(v_.begin(), v_.end(), o.getPtr()); }
  // values uniform in [0, 1) from a fixed-seed generator (HostVec::randomize)
  void randomize() {
    uint64_t s = 0x9E3779B97F4A7C15ull;
    for (auto& x : v_) {
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      x = T((double)(s >> 11) * (1.0 / 9007199254740992.0));
    }
  }
  // createDeviceVec (include/linalg/vec.h:351-368), defined after DeviceVec
  DeviceVec<T> createDeviceVec(bool memset = true, bool can_print = false) const;

 private:
  std::vector<T> v_;
};

template <typename T>
class DeviceVec {
 public:
  DeviceVec() = default;
  explicit DeviceVec(int n) : n_(n) {
    T* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * (n > 0 ? n : 1)) != cudaSuccess)
      throw Error(GF_OOM, "DeviceVec");
    cudaMemset(p, 0, sizeof(T) * n);
    p_.reset(p, [](T* q) { cudaFree(q); });
  }
  explicit DeviceVec(const HostVec<T>& h) : DeviceVec(h.getSize()) {
    cudaMemcpy(p_.get(), h.getPtr(), sizeof(T) * n_, cudaMemcpyHostToDevice);
  }
  T* getPtr() { return p_.get(); }
  const T* getPtr() const { return p_.get(); }
  int getSize() const { return n_; }
  void zeroValues() { cudaMemset(p_.get(), 0, sizeof(T) * n_); }
  void copyValuesTo(DeviceVec& o) const {
    cudaMemcpy(o.getPtr(), p_.get(), sizeof(T) * n_, cudaMemcpyDeviceToDevice);
  }
  HostVec<T> createHostVec() const {
    HostVec<T> h(n_);
    cudaMemcpy(h.getPtr(), p_.get(), sizeof(T) * n_, cudaMemcpyDeviceToHost);
    return h;
  }

 private:
  int n_ = 0;
  std::shared_ptr<T> p_;
};

template <typename T>
DeviceVec<T> HostVec<T>::createDeviceVec(bool, bool) const {
  return DeviceVec<T>(*this);
}

// the reference's vector type of GPU builds (include/linalg/vec.h:391)
template <typename T>
using VecType = DeviceVec<T>;

// ---- element composition (type tags; the shell math is in the library)
template <typename T>
struct QuadLinearQuadrature {};  // 2x2 Gauss, include/shell/quadrature.h:4-19
template <typename T>
struct LinearizedRotation {};    // include/shell/director.h:28-137
template <typename T, class Quad, int order>
struct ShellQuadBasis {          // include/shell/basis.h:7-289
  struct Geo {
    static constexpr int num_nodes = 4, spatial_dim = 3;
  };
  static constexpr int num_nodes = 4;
};
// ShellIsotropicData<T, has_ref_axis> (include/shell/data.h:8-47)
template <typename T, bool kRefAxis>
struct ShellIsotropicData : gf_shell_data {
  ShellIsotropicData() : gf_shell_data{} {}
  ShellIsotropicData(T E_, T nu_, T thick_, T tOffset_ = T(0)) : gf_shell_data{} {
    E = E_;
    nu = nu_;
    thick = thick_;
    tOffset = tOffset_;
  }
  ShellIsotropicData(T E_, T nu_, T thick_, T tOffset_, const T refAxis_[3])
      : ShellIsotropicData(E_, nu_, thick_, tOffset_) {
    static_assert(kRefAxis, "a reference axis needs has_ref_axis = true");
    for (int i = 0; i < 3; i++) refAxis[i] = refAxis_[i];
    has_ref_axis = 1;
  }
};
template <typename T, class Data_>
struct IsotropicShell {          // include/shell/physics.h:6-350
  using Data = Data_;
  static constexpr int vars_per_node = 6;
};
template <typename T, class Director_, class Basis_, class Phys_>
struct ShellElementGroup {       // include/shell/elem_group.h:13
  using Director = Director_;
  using Basis = Basis_;
  using Geo = typename Basis_::Geo;
  using Phys = Phys_;
};
static_assert(sizeof(ShellIsotropicData<double, false>) == sizeof(gf_shell_data),
              "ShellIsotropicData must have gf_shell_data's layout");

// BsrData (include/linalg/bsr_utils.h:43-404): the block pattern in the
// solver ordering with its permutation (perm[natural node] = solver row,
// iperm its inverse) and elemIndMap (16 block slots per element). Host
// copies; the device copies stay inside the library. `fill_level` is the ILU
// fill this pattern stands for when a preconditioner is built from it
// (0: A's own pattern, GF_FILL_FULL: complete LU).
struct BsrData {
  int nnodes = 0, nnzb = 0, block_dim = 6;
  int fill_level = 0;
  HostVec<int> rowPtr, colPtr, perm, iperm, elemIndMap;
  gf_assembler* assembler = nullptr;  // the library handle the pattern belongs to
};

template <class Vec>
class BsrMat;

// TACSMeshLoader<T> (include/mesh/TACSMeshLoader.h:138-225), the part the
// shell path uses: scanBDFFile reads GRID / CQUAD4 / SPC entries
// (gf_bdf_read) and getAssemblerCreatorData hands them to createFromBDF.
template <typename T>
class TACSMeshLoader {
 public:
  TACSMeshLoader() = default;
  TACSMeshLoader(const TACSMeshLoader&) = delete;
  TACSMeshLoader& operator=(const TACSMeshLoader&) = delete;
  ~TACSMeshLoader() {
    if (m_) gf_bdf_free(m_);
  }
  int scanBDFFile(const char* file_name) {
    if (m_) gf_bdf_free(m_);
    m_ = nullptr;
    check(gf_bdf_read(file_name, &m_), "scanBDFFile");
    return 0;
  }
  int getNumNodes() const { return m_ ? m_->num_nodes : 0; }
  int getNumElements() const { return m_ ? m_->num_elements : 0; }
  const gf_bdf_mesh* data() const { return m_; }

 private:
  gf_bdf_mesh* m_ = nullptr;
};

// ElementAssembler<T, ElemGroup, Vec, Mat> (include/assembler.h:14-322).
// Geo and vars connectivity must be identical for the shell element. The
// node ordering of the solver (RCM by default here; the reference reorders
// in symbolic_factorization) is fixed at construction.
template <typename T_, class ElemGroup, template <typename> class Vec,
          template <typename> class Mat_>
class ElementAssembler {
 public:
  using T = T_;
  using Geo = typename ElemGroup::Geo;
  using Basis = typename ElemGroup::Basis;
  using Phys = typename ElemGroup::Phys;
  using Data = typename Phys::Data;
  using Mat = Mat_<Vec<T>>;
  static constexpr int32_t geo_nodes_per_elem = Geo::num_nodes;
  static constexpr int32_t vars_nodes_per_elem = Basis::num_nodes;
  static constexpr int32_t spatial_dim = Geo::spatial_dim;
  static constexpr int32_t vars_per_node = Phys::vars_per_node;

  // ElementAssembler(num_geo_nodes, num_vars_nodes, num_elements, geo_conn,
  // vars_conn, xpts, bcs, physData) (include/assembler.h:31-34)
  ElementAssembler(int32_t num_geo_nodes, int32_t num_vars_nodes, int32_t num_elements,
                   HostVec<int32_t>& geo_conn, HostVec<int32_t>& vars_conn, HostVec<T>& xpts,
                   HostVec<int>& bcs, HostVec<Data>& physData, int ordering = GF_ORDER_RCM) {
    if (num_geo_nodes != num_vars_nodes) throw Error(GF_INVALID_ARG, "ElementAssembler");
    (void)vars_conn;
    gf_mesh_desc d{};
    d.num_nodes = num_geo_nodes;
    d.num_elements = num_elements;
    d.conn = geo_conn.getPtr();
    d.xpts = xpts.getPtr();
    d.bcs = bcs.getPtr();
    d.num_bcs = bcs.getSize();
    d.data = physData.getPtr();
    d.ordering = ordering;
    gf_assembler* a = nullptr;
    check(gf_assembler_create(&d, &a), "gf_assembler_create");
    h_.reset(a, [](gf_assembler* x) { gf_assembler_destroy(x); });
    xpts_ = xpts;
    conn_ = geo_conn;
  }
  // createFromBDF(mesh_loader, single_data) (include/assembler.h:92-115):
  // every element gets the same material data
  static ElementAssembler createFromBDF(TACSMeshLoader<T>& mesh_loader, Data single_data,
                                        int ordering = GF_ORDER_RCM) {
    const gf_bdf_mesh* m = mesh_loader.data();
    if (!m) throw Error(GF_INVALID_ARG, "createFromBDF: no mesh scanned");
    HostVec<int32_t> conn(4 * m->num_elements, m->conn);
    HostVec<int> bcs(m->num_bcs, m->bcs);
    HostVec<T> xpts(3 * m->num_nodes, m->xpts);
    HostVec<Data> data(m->num_elements);
    for (int e = 0; e < m->num_elements; e++) data[e] = single_data;
    return ElementAssembler(m->num_nodes, m->num_nodes, m->num_elements, conn, conn, xpts, bcs,
                            data, ordering);
  }
  // symbolic_factorization(fill, print) (include/assembler.h:76-81). The
  // reference widens the matrix pattern to the full LU fill here, for
  // CUSPARSE::direct_LU_solve_old; in this library the pattern and ordering
  // are built by the constructor and the direct solve builds the fill
  // itself, so this only records that a direct solve is intended.
  void symbolic_factorization(double fill_factor = 10.0, bool print = false) {
    (void)fill_factor;
    (void)print;
    full_fill_ = true;
  }
  BsrData getBsrData() const {
    BsrData b;
    b.nnodes = get_num_nodes();
    b.assembler = h_.get();
    b.fill_level = full_fill_ ? GF_FILL_FULL : 0;
    b.rowPtr = HostVec<int>(b.nnodes + 1);
    check(gf_assembler_get_pattern(h_.get(), b.rowPtr.getPtr(), nullptr, nullptr, nullptr),
          "getBsrData");
    b.nnzb = b.rowPtr[b.nnodes];
    b.colPtr = HostVec<int>(b.nnzb);
    b.perm = HostVec<int>(b.nnodes);
    b.iperm = HostVec<int>(b.nnodes);
    b.elemIndMap = HostVec<int>(16 * get_num_elements());
    check(gf_assembler_get_pattern(h_.get(), nullptr, b.colPtr.getPtr(), b.perm.getPtr(),
                                   b.elemIndMap.getPtr()),
          "getBsrData");
    for (int i = 0; i < b.nnodes; i++) b.iperm[b.perm[i]] = i;
    return b;
  }
  HostVec<T>& getXpts() { return xpts_; }
  HostVec<int32_t>& getConn() { return conn_; }
  int get_num_xpts() const { return 3 * get_num_nodes(); }
  int get_num_vars() const { return gf_assembler_num_vars(h_.get()); }
  int get_num_nodes() const { return gf_assembler_num_nodes(h_.get()); }
  int get_num_elements() const { return gf_assembler_num_elements(h_.get()); }
  // createVarsVec(data, randomize, can_print) (include/assembler.h:169-189)
  Vec<T> createVarsVec(T* data = nullptr, bool randomize = false, bool can_print = false) {
    (void)can_print;
    HostVec<T> h(get_num_vars(), data);
    if (randomize) h.randomize();
    return h.createDeviceVec();
  }
  // set_variables (include/assembler.h:191-195); copied, not referenced
  void set_variables(Vec<T>& v) {
    check(gf_set_variables(h_.get(), v.getPtr(), nullptr), "set_variables");
  }
  // add_energy(U, can_print) (include/assembler.h:198): U += strain energy
  void add_energy(T& Uenergy, bool can_print = false) {
    (void)can_print;
    double U = 0.0;
    check(gf_add_energy(h_.get(), &U, nullptr), "add_energy");
    Uenergy += U;
  }
  // add_residual(res, can_print) (include/assembler.h:232): res += R(u)
  void add_residual(Vec<T>& res, bool can_print = false) {
    (void)can_print;
    check(gf_add_residual(h_.get(), res.getPtr(), GF_ASSEMBLE_ADD, nullptr), "add_residual");
  }
  // add_jacobian(res, mat, can_print) (include/assembler.h:267): res += R(u),
  // mat += K(u)
  void add_jacobian(Vec<T>& res, Mat& mat, bool can_print = false) {
    (void)can_print;
    check(gf_add_jacobian(h_.get(), res.getPtr(), mat.handle(), GF_ASSEMBLE_ADD, nullptr),
          "add_jacobian");
  }
  // apply_bcs(vec / mat, can_print) (include/assembler.h:119-154)
  void apply_bcs(Vec<T>& v, bool can_print = false) {
    (void)can_print;
    check(gf_apply_bcs_vec(h_.get(), v.getPtr(), nullptr), "apply_bcs(vec)");
  }
  void apply_bcs(Mat& mat, bool can_print = false) {
    (void)can_print;
    check(gf_apply_bcs_mat(h_.get(), mat.handle(), nullptr), "apply_bcs(mat)");
  }
  gf_assembler* handle() const { return h_.get(); }

 private:
  std::shared_ptr<gf_assembler> h_;
  HostVec<T> xpts_;
  HostVec<int32_t> conn_;
  bool full_fill_ = false;
};

// BsrMat<Vec> (include/linalg/bsr_mat.h:9-352): 6x6-block values on the
// device in the solver ordering, with a host copy of its BsrData.
template <class Vec>
class BsrMat {
 public:
  using T = double;
  explicit BsrMat(const BsrData& bsr_data) : bsr_(bsr_data) {
    if (!bsr_.assembler) throw Error(GF_INVALID_ARG, "BsrMat");
    gf_bsr* m = nullptr;
    check(gf_bsr_create(bsr_.assembler, &m), "gf_bsr_create");
    h_.reset(m, [](gf_bsr* x) { gf_bsr_destroy(x); });
  }
  BsrData getBsrData() const { return bsr_; }
  int* getPerm() { return bsr_.perm.getPtr(); }
  int* getIPerm() { return bsr_.iperm.getPtr(); }
  int* getRowPtr() { return bsr_.rowPtr.getPtr(); }
  int* getColPtr() { return bsr_.colPtr.getPtr(); }
  int get_nnz() const { return 36 * bsr_.nnzb; }
  double* getPtr() { return gf_bsr_values(h_.get()); }
  void zeroValues() { check(gf_bsr_zero(h_.get(), nullptr), "zeroValues"); }
  // host copy of the values (createHostVec, bsr_mat.h:30)
  HostVec<T> createHostVec() {
    HostVec<T> h(get_nnz());
    if (cudaMemcpy(h.getPtr(), getPtr(), sizeof(T) * (size_t)get_nnz(),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
      throw Error(GF_CUDA_ERROR, "createHostVec");
    return h;
  }
  // device-to-device copy of the values into a matrix of the same pattern
  void copyValuesTo(BsrMat& o) const {
    if (o.bsr_.assembler != bsr_.assembler) throw Error(GF_INVALID_ARG, "copyValuesTo");
    if (cudaMemcpy(o.getPtr(), gf_bsr_values(h_.get()), sizeof(T) * 36 * (size_t)bsr_.nnzb,
                   cudaMemcpyDeviceToDevice) != cudaSuccess)
      throw Error(GF_CUDA_ERROR, "copyValuesTo");
  }
  gf_bsr* handle() const { return h_.get(); }
  gf_assembler* assembler() const { return bsr_.assembler; }

 private:
  BsrData bsr_;
  std::shared_ptr<gf_bsr> h_;
};

// createBsrMat<Assembler, Vec>(assembler) (include/linalg/bsr_mat.h:354-357)
template <class Assembler, class Vec>
BsrMat<Vec> createBsrMat(Assembler& assembler) {
  return BsrMat<Vec>(assembler.getBsrData());
}

// ILUk_Preconditioner (include/linalg/precond.h:5-55). The reference holds
// a preconditioner matrix with the ILU(k) pattern and copies A's values into
// it (copyValues); here the factor and its pattern live in the library: the
// fill level comes from precond_mat's BsrData (fill_level), or is given.
template <class Vec = DeviceVec<double>>
class ILUk_Preconditioner {
 public:
  ILUk_Preconditioner(BsrMat<Vec>& precond_mat, BsrMat<Vec>& orig_mat, bool print = false)
      : ILUk_Preconditioner(orig_mat, precond_mat.getBsrData().fill_level, GF_PREC_FP64) {
    (void)print;
  }
  ILUk_Preconditioner(BsrMat<Vec>& orig_mat, int fill_level, int precision = GF_PREC_FP64,
                      int sweep = GF_SWEEP_AUTO)
      : mat_(&orig_mat) {
    gf_precond* p = nullptr;
    check(gf_precond_create_ex(orig_mat.assembler(), fill_level, precision, sweep, &p),
          "gf_precond_create");
    h_.reset(p, [](gf_precond* x) { gf_precond_destroy(x); });
  }
  // copyValues + numeric factorization (precond.h:35-44; cusparseDbsrilu02)
  void copyValues() {}  // the factorization reads A's values itself
  void factor() { check(gf_precond_factor(h_.get(), mat_->handle(), nullptr), "factor"); }
  // z = (LU)^{-1} r, r and z in the solver ordering (gf_precond_apply)
  void apply(Vec& r, Vec& z) {
    check(gf_precond_apply(h_.get(), r.getPtr(), z.getPtr(), nullptr), "apply");
  }
  gf_precond* handle() const { return h_.get(); }
  BsrMat<Vec>& matrix() { return *mat_; }

 private:
  BsrMat<Vec>* mat_;
  std::shared_ptr<gf_precond> h_;
};

// GMRES driver of examples/iterative/gmres.cu:468-771 as a function; rhs and
// soln in natural order (soln is the initial guess on entry).
template <class Assembler, class Vec>
gf_solve_stats gmres_solve(Assembler& a, BsrMat<Vec>& A, ILUk_Preconditioner<Vec>& P, Vec& rhs,
                           Vec& soln, const gf_solve_opts* opts = nullptr) {
  gf_solve_stats st{};
  gf_status s = gf_gmres_solve(a.handle(), A.handle(), P.handle(), rhs.getPtr(), soln.getPtr(),
                               opts, &st, nullptr);
  if (s != GF_OK && s != GF_NOT_CONVERGED) throw Error(s, "gmres_solve");
  return st;
}

namespace CUSPARSE {
// direct_LU_solve_old (include/linalg/solvers/cusparse.h:16-192): complete
// block LU of mat and two triangular solves, rhs and soln in natural order.
template <typename T>
gf_solve_stats direct_LU_solve_old(BsrMat<DeviceVec<T>>& mat, DeviceVec<T>& rhs,
                                   DeviceVec<T>& soln, bool can_print = false) {
  (void)can_print;
  gf_solve_stats st{};
  check(gf_direct_solve(mat.assembler(), mat.handle(), rhs.getPtr(), soln.getPtr(), &st, nullptr),
        "direct_LU_solve_old");
  return st;
}
}  // namespace CUSPARSE

}  // namespace gpufem
