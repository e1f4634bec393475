// C++ facade over the C ABI (include/gpufem.h) that keeps the reference's
// class and method names so driver code written against smdogroup/gpu_fem
// ports with few edits:
//   ElementAssembler      include/assembler.h:14-322
//   BsrData (host copy)   include/linalg/bsr_utils.h:43-404
//   BsrMat, createBsrMat  include/linalg/bsr_mat.h:9-357
//   DeviceVec, HostVec    include/linalg/vec.h:146-371
//   ILUk_Preconditioner   include/linalg/precond.h:5-55
//   gmres_solve           examples/iterative/gmres.cu:468-771 (driver code)
// Differences: errors throw gpufem::Error instead of calling exit();
// handles own their memory (the reference's destructors are commented out,
// vec.h:180-186); vectors at the boundary are in natural node order and the
// solver ordering (RCM) is applied inside.
#pragma once
#include <cuda_runtime.h>

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
  // createDeviceVec (include/linalg/vec.h), defined after DeviceVec
  DeviceVec<T> createDeviceVec() const;

 private:
  std::vector<T> v_;
};

template <typename T>
class DeviceVec {
 public:
  DeviceVec() = default;
  explicit DeviceVec(int n) : n_(n) {
    T* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * n) != cudaSuccess) throw Error(GF_OOM, "DeviceVec");
    cudaMemset(p, 0, sizeof(T) * n);
    p_.reset(p, [](T* q) { cudaFree(q); });
  }
  explicit DeviceVec(const HostVec<T>& h) : DeviceVec(h.getSize()) {
    cudaMemcpy(p_.get(), h.getPtr(), sizeof(T) * n_, cudaMemcpyHostToDevice);
  }
  T* getPtr() { return p_.get(); }
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
DeviceVec<T> HostVec<T>::createDeviceVec() const {
  return DeviceVec<T>(*this);
}

// BsrData (include/linalg/bsr_utils.h:43-404): the block pattern in the
// solver ordering with its permutation (perm[natural node] = solver row,
// iperm its inverse) and elemIndMap (16 block slots per element). Host
// copies; the device copies stay inside the library.
struct BsrData {
  int nnodes = 0, nnzb = 0;
  HostVec<int> rowPtr, colPtr, perm, iperm, elemIndMap;
};

// ShellIsotropicData<double, has_ref_axis> (include/shell/data.h:8-47)
inline gf_shell_data ShellIsotropicData(double E, double nu, double thick,
                                        double tOffset = 0.0) {
  gf_shell_data d{};
  d.E = E;
  d.nu = nu;
  d.thick = thick;
  d.tOffset = tOffset;
  return d;
}

class BsrMat;

class ElementAssembler {
 public:
  // ElementAssembler(num_geo_nodes, num_vars_nodes, num_elements, geo_conn,
  // vars_conn, xpts, bcs, physData) (include/assembler.h:31-34); geo and
  // vars connectivity must be identical for the shell element.
  ElementAssembler(int num_geo_nodes, int num_vars_nodes, int num_elements,
                   HostVec<int>& geo_conn, HostVec<int>& vars_conn, HostVec<double>& xpts,
                   HostVec<int>& bcs, HostVec<gf_shell_data>& physData,
                   int ordering = GF_ORDER_NATURAL) {
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
  // The pattern, ordering and elemIndMap are built by the constructor; the
  // reference's symbolic_factorization(fill, print) (assembler.h:76-81)
  // is kept for drivers that call it and changes nothing.
  void symbolic_factorization(double fill = 100.0, bool print = false) {
    (void)fill;
    (void)print;
  }
  BsrData getBsrData() const {
    BsrData b;
    b.nnodes = get_num_nodes();
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
  const HostVec<double>& getXpts() const { return xpts_; }
  const HostVec<int>& getConn() const { return conn_; }
  int get_num_vars() const { return gf_assembler_num_vars(h_.get()); }
  int get_num_nodes() const { return gf_assembler_num_nodes(h_.get()); }
  int get_num_elements() const { return gf_assembler_num_elements(h_.get()); }
  DeviceVec<double> createVarsVec() const { return DeviceVec<double>(get_num_vars()); }
  void set_variables(DeviceVec<double>& v) {
    check(gf_set_variables(h_.get(), v.getPtr(), nullptr), "set_variables");
  }
  void add_residual(DeviceVec<double>& res) {
    check(gf_add_residual(h_.get(), res.getPtr(), GF_ASSEMBLE_ADD, nullptr), "add_residual");
  }
  inline void add_jacobian(DeviceVec<double>& res, BsrMat& mat);
  double add_energy() {
    double U = 0.0;
    check(gf_add_energy(h_.get(), &U, nullptr), "add_energy");
    return U;
  }
  void apply_bcs(DeviceVec<double>& v) {
    check(gf_apply_bcs_vec(h_.get(), v.getPtr(), nullptr), "apply_bcs(vec)");
  }
  inline void apply_bcs(BsrMat& mat);
  gf_assembler* handle() const { return h_.get(); }

 private:
  std::shared_ptr<gf_assembler> h_;
  HostVec<double> xpts_;
  HostVec<int> conn_;
};

class BsrMat {
  static int nnzb(const gf_assembler* a) {
    std::vector<int> rp(gf_assembler_num_nodes(a) + 1);
    check(gf_assembler_get_pattern(a, rp.data(), nullptr, nullptr, nullptr), "nnzb");
    return rp.back();
  }

 public:
  explicit BsrMat(ElementAssembler& a) : a_(a.handle()) {
    gf_bsr* m = nullptr;
    check(gf_bsr_create(a_, &m), "gf_bsr_create");
    h_.reset(m, [](gf_bsr* x) { gf_bsr_destroy(x); });
  }
  double* getPtr() { return gf_bsr_values(h_.get()); }
  void zeroValues() { check(gf_bsr_zero(h_.get(), nullptr), "zeroValues"); }
  // device-to-device copy of the 36 nnzb values into a matrix of the same pattern
  void copyValuesTo(BsrMat& o) const {
    if (o.a_ != a_) throw Error(GF_INVALID_ARG, "copyValuesTo");
    const int nnzb = BsrMat::nnzb(a_);
    if (cudaMemcpy(o.getPtr(), gf_bsr_values(h_.get()), sizeof(double) * 36 * (size_t)nnzb,
                   cudaMemcpyDeviceToDevice) != cudaSuccess)
      throw Error(GF_CUDA_ERROR, "copyValuesTo");
  }
  gf_bsr* handle() const { return h_.get(); }

 private:
  gf_assembler* a_;
  std::shared_ptr<gf_bsr> h_;
};

// add_jacobian keeps the reference's additive semantics on a zeroed matrix.
void ElementAssembler::add_jacobian(DeviceVec<double>& res, BsrMat& mat) {
  check(gf_add_jacobian(h_.get(), res.getPtr(), mat.handle(), GF_ASSEMBLE_ADD, nullptr),
        "add_jacobian");
}
void ElementAssembler::apply_bcs(BsrMat& mat) {
  check(gf_apply_bcs_mat(h_.get(), mat.handle(), nullptr), "apply_bcs(mat)");
}

inline BsrMat createBsrMat(ElementAssembler& a) { return BsrMat(a); }

class ILUk_Preconditioner {
 public:
  ILUk_Preconditioner(ElementAssembler& a, int fill_level = 0, int precision = GF_PREC_FP64) {
    gf_precond* p = nullptr;
    check(gf_precond_create(a.handle(), fill_level, precision, &p), "gf_precond_create");
    h_.reset(p, [](gf_precond* x) { gf_precond_destroy(x); });
  }
  // copyValues + factor (include/linalg/precond.h:35-44)
  void factor(BsrMat& A) { check(gf_precond_factor(h_.get(), A.handle(), nullptr), "factor"); }
  gf_precond* handle() const { return h_.get(); }

 private:
  std::shared_ptr<gf_precond> h_;
};

// GMRES driver of examples/iterative/gmres.cu:468-771 as a function.
inline gf_solve_stats gmres_solve(ElementAssembler& a, BsrMat& A, ILUk_Preconditioner& P,
                                  DeviceVec<double>& rhs, DeviceVec<double>& soln,
                                  const gf_solve_opts* opts = nullptr) {
  gf_solve_stats st{};
  gf_status s = gf_gmres_solve(a.handle(), A.handle(), P.handle(), rhs.getPtr(), soln.getPtr(),
                               opts, &st, nullptr);
  if (s != GF_OK && s != GF_NOT_CONVERGED) throw Error(s, "gmres_solve");
  return st;
}

}  // namespace gpufem
