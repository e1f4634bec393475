// CPU ORACLE — test infrastructure only, never part of the product path.
//
// A plain C++ restatement of the reference's linear MITC4 shell element
// (smdogroup/gpu_fem, include/shell/*), templated on the scalar type so the
// reference's complex-step checks (tests/shell_res/res_cs.cu,
// tests/shell_jac/jac-cs.cu) can be re-run with T = std::complex<double>.
//
// The reference builds on the external A2D library (smdogroup/a2d, no pinned
// version, not vendored). Its primitives used on this path are restated here
// from their mathematics: 3x3 inverse/determinant, 3x3 products with transpose
// flags, cross/dot/normalise, and the symmetric-matrix packing
// (11, 12, 13, 22, 23, 33). The AD stacks of include/shell/physics.h:41-92 are
// restated as explicit forward / reverse code.
//
// Intended-math fixes relative to the reference snapshot (each is a bug in the
// snapshot, not a design choice):
//  * ShellComputeDispGradSens (include/shell/basis.h:566-567) overwrites
//    u0d_bar^T with the u1x_bar term instead of adding it. Here it adds. For
//    the linear strain u0x_bar is identically zero, so results are unchanged.
//  * add_element_quadpt_jacobian_col (include/shell/elem_group.h:286-289)
//    sends the disp-grad Hessian reverse into `res` instead of `matCol`. Here it
//    goes into the Jacobian column, so K is the exact Hessian of the energy and
//    R(u) = K u (pinned by the complex-step tests).
//
// Parity unpinned by reference outputs: the reference cannot be built here
// (A2D and sparse-utils are absent) and its tests store no expected values.
// What the restatement is checked against instead: complex-step
// residual/energy and Jacobian/residual identities on the reference's
// one-element fixture, the 2-element fill-in known answer,
// linearity/symmetry/rigid-body properties, and the Navier plate solution
// (see tests/).
#pragma once
#include <cmath>
#include <complex>
#include <cstring>

namespace oracle {

using std::sqrt;

// Per-element material data; mirrors ShellIsotropicData
// (include/shell/data.h:8-47): shear correction 5/6, drilling regularisation
// 10, natural transform unless has_ref_axis.
struct ShellData {
  double E, nu, thick, tOffset;
  double refAxis[3];
  int has_ref_axis;
};

constexpr double kShearCorrection = 5.0 / 6.0;  // data.h:11
constexpr double kDrillReg = 10.0;              // data.h:12
constexpr double kRt3 = 0.577350269189626;      // quadrature.h:9 (literal)

// ---------------------------------------------------------------- quadrature
// QuadLinearQuadrature::getQuadraturePoint (include/shell/quadrature.h:11-18)
template <class T>
inline double quad_point(int iq, T pt[2]) {
  const double p[2] = {-kRt3, kRt3};
  pt[0] = p[iq % 2];
  pt[1] = p[iq / 2];
  return 1.0;
}

// ------------------------------------------------------------------- basis
// ShellQuadBasis, order 2 (include/shell/basis.h:56-142)
template <class T>
inline void lag1(const T& u, T N[2]) {
  N[0] = 0.5 * (1.0 - u);
  N[1] = 0.5 * (1.0 + u);
}
template <class T>
inline void lag2(const T pt[2], T N[4]) {
  T na[2], nb[2];
  lag1(pt[0], na);
  lag1(pt[1], nb);
  for (int j = 0; j < 2; j++)
    for (int i = 0; i < 2; i++) N[2 * j + i] = na[i] * nb[j];
}
template <class T>
inline void lag2grad(const T pt[2], T N[4], T Nxi[4], T Neta[4]) {
  T na[2], nb[2];
  lag1(pt[0], na);
  lag1(pt[1], nb);
  const double dn[2] = {-0.5, 0.5};
  for (int j = 0; j < 2; j++)
    for (int i = 0; i < 2; i++) {
      N[2 * j + i] = na[i] * nb[j];
      Nxi[2 * j + i] = dn[i] * nb[j];
      Neta[2 * j + i] = na[i] * dn[j];
    }
}
// getNodePoint (basis.h:138-142): tensor-product node order.
template <class T>
inline void node_point(int n, T pt[2]) {
  pt[0] = -1.0 + 2.0 * (n % 2);
  pt[1] = -1.0 + 2.0 * (n / 2);
}
// interpFields (basis.h:144-156)
template <int VPN, int NF, class T>
inline void interp(const T pt[2], const T* vals, T* out) {
  T N[4];
  lag2(pt, N);
  for (int f = 0; f < NF; f++) {
    out[f] = 0.0;
    for (int n = 0; n < 4; n++) out[f] += N[n] * vals[n * VPN + f];
  }
}
// interpFieldsGrad (basis.h:158-172)
template <int VPN, int NF, class T>
inline void interp_grad(const T pt[2], const T* vals, T* dxi, T* deta) {
  T N[4], Nx[4], Ne[4];
  lag2grad(pt, N, Nx, Ne);
  for (int f = 0; f < NF; f++) {
    dxi[f] = 0.0;
    deta[f] = 0.0;
    for (int n = 0; n < 4; n++) {
      dxi[f] += Nx[n] * vals[n * VPN + f];
      deta[f] += Ne[n] * vals[n * VPN + f];
    }
  }
}
// interpFieldsTranspose (basis.h:174-187), additive
template <int VPN, int NF, class T>
inline void interp_T(const T pt[2], const T* bar, T* vals_bar) {
  T N[4];
  lag2(pt, N);
  for (int f = 0; f < NF; f++)
    for (int n = 0; n < 4; n++) vals_bar[n * VPN + f] += bar[f] * N[n];
}
// interpFieldsGradTranspose (basis.h:189-203), additive
template <int VPN, int NF, class T>
inline void interp_grad_T(const T pt[2], const T* dxi_bar, const T* deta_bar,
                          T* vals_bar) {
  T N[4], Nx[4], Ne[4];
  lag2grad(pt, N, Nx, Ne);
  for (int f = 0; f < NF; f++)
    for (int n = 0; n < 4; n++)
      vals_bar[n * VPN + f] += dxi_bar[f] * Nx[n] + deta_bar[f] * Ne[n];
}

// MITC tying points (basis.h:205-235) and their interpolation
// (basis.h:237-287). Components: 0 g11, 1 g22, 2 g12, 3 g23, 4 g13; offsets
// (basis.h:30-36) 0, 2, 4, 5, 7; 9 tying values in total.
constexpr int kTyOff[5] = {0, 2, 4, 5, 7};
constexpr int kTyNum[5] = {2, 2, 1, 2, 2};
template <class T>
inline void tying_point(int icomp, int n, T pt[2]) {
  const double red = 0.0, full[2] = {-1.0, 1.0};
  if (icomp == 0 || icomp == 4) {
    pt[0] = red;
    pt[1] = full[n];
  } else if (icomp == 1 || icomp == 3) {
    pt[0] = full[n % 2];
    pt[1] = red;
  } else {
    pt[0] = red;
    pt[1] = red;
  }
}
template <class T>
inline void tying_interp(int icomp, const T pt[2], T* N) {
  T na[2], nb[2];
  lag1(pt[0], na);
  lag1(pt[1], nb);
  if (icomp == 0 || icomp == 4) {
    N[0] = nb[0];
    N[1] = nb[1];
  } else if (icomp == 1 || icomp == 3) {
    N[0] = na[0];
    N[1] = na[1];
  } else {
    N[0] = 1.0;
  }
}
// interpTyingStrain (basis.h:314-368): gty packed (11,12,13,22,23,33).
template <class T>
inline void interp_tying(const T pt[2], const T ety[9], T gty[6]) {
  const int slot[5] = {0, 3, 1, 4, 2};  // g11->11, g22->22, g12->12, g23->23, g13->13
  for (int c = 0; c < 5; c++) {
    T N[2];
    tying_interp(c, pt, N);
    T s = 0.0;
    for (int k = 0; k < kTyNum[c]; k++) s += N[k] * ety[kTyOff[c] + k];
    gty[slot[c]] = s;
  }
  gty[5] = 0.0;
}
// interpTyingStrainTranspose (basis.h:370-425), additive
template <class T>
inline void interp_tying_T(const T pt[2], const T gty_bar[6], T ety_bar[9]) {
  const int slot[5] = {0, 3, 1, 4, 2};
  for (int c = 0; c < 5; c++) {
    T N[2];
    tying_interp(c, pt, N);
    for (int k = 0; k < kTyNum[c]; k++) ety_bar[kTyOff[c] + k] += gty_bar[slot[c]] * N[k];
  }
}

// ------------------------------------------------- small dense helpers (A2D)
template <class T>
inline void cross(const T a[3], const T b[3], T c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
template <class T>
inline T dot3(const T a[3], const T b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
// columns a, b, c -> row-major frame (basis.h:120-127)
template <class T>
inline void frame(const T a[3], const T b[3], const T c[3], T F[9]) {
  for (int i = 0; i < 3; i++) {
    F[3 * i] = a[i];
    F[3 * i + 1] = b[i];
    F[3 * i + 2] = c[i];
  }
}
template <class T>
inline T det3(const T A[9]) {
  return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
         A[2] * (A[3] * A[7] - A[4] * A[6]);
}
template <class T>
inline void inv3(const T A[9], T B[9]) {
  T d = det3(A);
  T id = 1.0 / d;
  B[0] = (A[4] * A[8] - A[5] * A[7]) * id;
  B[1] = -(A[1] * A[8] - A[2] * A[7]) * id;
  B[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  B[3] = -(A[3] * A[8] - A[5] * A[6]) * id;
  B[4] = (A[0] * A[8] - A[2] * A[6]) * id;
  B[5] = -(A[0] * A[5] - A[2] * A[3]) * id;
  B[6] = (A[3] * A[7] - A[4] * A[6]) * id;
  B[7] = -(A[0] * A[7] - A[1] * A[6]) * id;
  B[8] = (A[0] * A[4] - A[1] * A[3]) * id;
}
// C = op(A) op(B); ta/tb select the transpose.
template <class T>
inline void mm3(const T A[9], const T B[9], T C[9], bool ta = false, bool tb = false) {
  T R[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      T s = 0.0;
      for (int k = 0; k < 3; k++) {
        T a = ta ? A[3 * k + i] : A[3 * i + k];
        T b = tb ? B[3 * j + k] : B[3 * k + j];
        s += a * b;
      }
      R[3 * i + j] = s;
    }
  for (int i = 0; i < 9; i++) C[i] = R[i];
}

// ---------------------------------------------------------------- geometry
// ShellComputeNodeNormals (basis.h:292-311)
template <class T>
inline void node_normals(const T X[12], T fn[12]) {
  for (int n = 0; n < 4; n++) {
    T pt[2];
    node_point(n, pt);
    T xi[3], eta[3], c[3];
    interp_grad<3, 3>(pt, X, xi, eta);
    cross(xi, eta, c);
    T nrm = sqrt(dot3(c, c));
    for (int i = 0; i < 3; i++) fn[3 * n + i] = (1.0 / nrm) * c[i];
  }
}
// ShellComputeTransform (shell_utils.h:4-40)
template <class T>
inline void shell_transform(const ShellData& d, const T Xxi[3], const T n0[3], T Tm[9]) {
  T nn = sqrt(dot3(n0, n0));
  T nhat[3] = {n0[0] / nn, n0[1] / nn, n0[2] / nn};
  T t1[3];
  for (int i = 0; i < 3; i++) t1[i] = d.has_ref_axis ? T(d.refAxis[i]) : Xxi[i];
  T dd = dot3(nhat, t1);
  T tmp[3];
  for (int i = 0; i < 3; i++) tmp[i] = t1[i] - dd * nhat[i];
  T tn = sqrt(dot3(tmp, tmp));
  T t1h[3] = {tmp[0] / tn, tmp[1] / tn, tmp[2] / tn};
  T t2h[3];
  cross(nhat, t1h, t2h);
  for (int i = 0; i < 3; i++) {
    Tm[3 * i] = t1h[i];
    Tm[3 * i + 1] = t2h[i];
    Tm[3 * i + 2] = nhat[i];
  }
}

// ---------------------------------------------------------------- director
// LinearizedRotation (director.h:28-137): C = I - skew(q); d = q x n
template <class T>
inline void rotation_mat(const T q[3], T C[9]) {
  C[0] = 1.0; C[1] = q[2];  C[2] = -q[1];
  C[3] = -q[2]; C[4] = 1.0; C[5] = q[0];
  C[6] = q[1]; C[7] = -q[0]; C[8] = 1.0;
}
template <class T>
inline void rotation_mat_sens(const T Cb[9], T qb[3]) {
  qb[0] += -(Cb[7] - Cb[5]);
  qb[1] += -(Cb[2] - Cb[6]);
  qb[2] += -(Cb[3] - Cb[1]);
}
template <class T>
inline void director(const T* vars, const T fn[12], T d[12]) {
  for (int n = 0; n < 4; n++) cross(&vars[6 * n + 3], &fn[3 * n], &d[3 * n]);
}
template <class T>
inline void director_sens(const T fn[12], const T d_bar[12], T* res) {
  for (int n = 0; n < 4; n++) {
    T c[3];
    cross(&fn[3 * n], &d_bar[3 * n], c);
    for (int i = 0; i < 3; i++) res[6 * n + 3 + i] += c[i];
  }
}

// ------------------------------------------------------------- drill strain
// ShellComputeDrillStrain (shell_utils.h:42-105)
template <class T>
inline void drill_strain(const T qpt[2], const ShellData& dat, const T X[12], const T* vars,
                         const T fn[12], T& et) {
  T etn[4];
  for (int n = 0; n < 4; n++) {
    T pt[2];
    node_point(n, pt);
    T xi[3], eta[3], Xd[9], Tm[9];
    interp_grad<3, 3>(pt, X, xi, eta);
    frame(xi, eta, &fn[3 * n], Xd);
    shell_transform(dat, xi, &fn[3 * n], Tm);
    T uxi[3], ueta[3], zero[3] = {0.0, 0.0, 0.0}, u0xn[9];
    interp_grad<6, 3>(pt, vars, uxi, ueta);
    frame(uxi, ueta, zero, u0xn);
    T C[9], tmp[9];
    rotation_mat(&vars[6 * n + 3], C);
    mm3(Tm, C, tmp, true, false);
    mm3(tmp, Tm, C);
    T XdinvT[9];
    inv3(Xd, tmp);
    mm3(tmp, Tm, XdinvT);
    mm3(u0xn, XdinvT, tmp);
    mm3(Tm, tmp, u0xn, true, false);
    etn[n] = 0.5 * (C[3] + u0xn[3] - C[1] - u0xn[1]);
  }
  T e[1];
  interp<1, 1>(qpt, etn, e);
  et = e[0];
}
// ShellComputeDrillStrainSens (shell_utils.h:116-179), additive into res
template <class T>
inline void drill_strain_sens(const T qpt[2], const ShellData& dat, const T X[12],
                              const T fn[12], const T& et_bar, T* res) {
  T etn_bar[4] = {0.0, 0.0, 0.0, 0.0};
  T eb[1] = {et_bar};
  interp_T<1, 1>(qpt, eb, etn_bar);
  for (int n = 0; n < 4; n++) {
    T pt[2];
    node_point(n, pt);
    T xi[3], eta[3], Xd[9], Tm[9];
    interp_grad<3, 3>(pt, X, xi, eta);
    frame(xi, eta, &fn[3 * n], Xd);
    shell_transform(dat, xi, &fn[3 * n], Tm);
    T ub[9], Cb[9];
    for (int i = 0; i < 9; i++) ub[i] = Cb[i] = 0.0;
    ub[1] = -0.5 * etn_bar[n];
    ub[3] = 0.5 * etn_bar[n];
    Cb[1] = -0.5 * etn_bar[n];
    Cb[3] = 0.5 * etn_bar[n];
    T tmp[9];
    mm3(Tm, Cb, tmp);
    mm3(tmp, Tm, Cb, false, true);
    rotation_mat_sens(Cb, &res[6 * n + 3]);
    T XdinvT[9];
    inv3(Xd, tmp);
    mm3(tmp, Tm, XdinvT);
    mm3(XdinvT, ub, tmp, false, true);
    mm3(tmp, Tm, ub, false, true);
    interp_grad_T<6, 3>(pt, &ub[0], &ub[3], res);
  }
}

// ----------------------------------------------------------- tying strains
// IsotropicShell::computeTyingStrain (physics.h:94-209)
template <class T>
inline void tying_strain(const T X[12], const T fn[12], const T* vars, const T d[12],
                         T ety[9]) {
  for (int c = 0; c < 5; c++)
    for (int k = 0; k < kTyNum[c]; k++) {
      T pt[2];
      tying_point(c, k, pt);
      T Xxi[3], Xeta[3], Uxi[3], Ueta[3];
      interp_grad<3, 3>(pt, X, Xxi, Xeta);
      interp_grad<6, 3>(pt, vars, Uxi, Ueta);
      T v;
      if (c == 0) {
        v = dot3(Uxi, Xxi);
      } else if (c == 1) {
        v = dot3(Ueta, Xeta);
      } else if (c == 2) {
        v = 0.5 * (dot3(Uxi, Xeta) + dot3(Ueta, Xxi));
      } else {
        T d0[3], n0[3];
        interp<3, 3>(pt, d, d0);
        interp<3, 3>(pt, fn, n0);
        if (c == 3)
          v = 0.5 * (dot3(Xeta, d0) + dot3(n0, Ueta));
        else
          v = 0.5 * (dot3(Xxi, d0) + dot3(n0, Uxi));
      }
      ety[kTyOff[c] + k] = v;
    }
}
// computeTyingStrainSens (physics.h:220-339), additive into res and d_bar
template <class T>
inline void tying_strain_sens(const T X[12], const T fn[12], const T ety_bar[9], T* res,
                              T d_bar[12]) {
  for (int c = 0; c < 5; c++)
    for (int k = 0; k < kTyNum[c]; k++) {
      T pt[2];
      tying_point(c, k, pt);
      T Xxi[3], Xeta[3];
      interp_grad<3, 3>(pt, X, Xxi, Xeta);
      T eb = ety_bar[kTyOff[c] + k];
      T ub_xi[3] = {0.0, 0.0, 0.0}, ub_eta[3] = {0.0, 0.0, 0.0}, db[3] = {0.0, 0.0, 0.0};
      if (c == 0) {
        for (int i = 0; i < 3; i++) ub_xi[i] = eb * Xxi[i];
      } else if (c == 1) {
        for (int i = 0; i < 3; i++) ub_eta[i] = eb * Xeta[i];
      } else if (c == 2) {
        for (int i = 0; i < 3; i++) {
          ub_eta[i] = 0.5 * eb * Xxi[i];
          ub_xi[i] = 0.5 * eb * Xeta[i];
        }
      } else {
        T n0[3];
        interp<3, 3>(pt, fn, n0);
        if (c == 3) {
          for (int i = 0; i < 3; i++) {
            db[i] = 0.5 * eb * Xeta[i];
            ub_eta[i] = 0.5 * eb * n0[i];
          }
        } else {
          for (int i = 0; i < 3; i++) {
            db[i] = 0.5 * eb * Xxi[i];
            ub_xi[i] = 0.5 * eb * n0[i];
          }
        }
      }
      interp_grad_T<6, 3>(pt, ub_xi, ub_eta, res);
      if (c >= 3) interp_T<3, 3>(pt, db, d_bar);
    }
}

// ------------------------------------------------------ displacement grads
// e0ty = A^T G A for symmetric packed G (a2dsymmatrotateframe.h:241-249)
template <class T>
inline void sym_rotate(const T A[9], const T g[6], T e[6]) {
  T G[9] = {g[0], g[1], g[2], g[1], g[3], g[4], g[2], g[4], g[5]};
  T tmp[9], R[9];
  mm3(A, G, tmp, true, false);
  mm3(tmp, A, R);
  e[0] = R[0]; e[1] = R[1]; e[2] = R[2]; e[3] = R[4]; e[4] = R[5]; e[5] = R[8];
}
// Adjoint of sym_rotate w.r.t. the packed entries of G
// (SymMat3x3RotateFrameReverse, a2dsymmatrotateframe.h:262-290).
template <class T>
inline void sym_rotate_T(const T A[9], const T eb[6], T gb[6]) {
  // L = sum_{a<=b} eb_ab e_ab = sum_ab U_ab e_ab with U upper-triangular.
  T U[9] = {eb[0], eb[1], eb[2], 0.0, eb[3], eb[4], 0.0, 0.0, eb[5]};
  T tmp[9], M[9];
  mm3(A, U, tmp);
  mm3(tmp, A, M, false, true);  // M = A U A^T = dL/dG (full)
  gb[0] = M[0];
  gb[1] = M[1] + M[3];
  gb[2] = M[2] + M[6];
  gb[3] = M[4];
  gb[4] = M[5] + M[7];
  gb[5] = M[8];
}

// ShellComputeDispGrad (basis.h:427-502); returns detXd
template <class T>
inline T disp_grad(const T pt[2], const ShellData& dat, const T X[12], const T* vars,
                   const T fn[12], const T d[12], const T ety[9], T u0x[9], T u1x[9],
                   T e0ty[6]) {
  T Tm[9], Xd[9], Xdz[9];
  {
    T Xxi[3], Xeta[3], nxi[3], neta[3], n0[3], zero[3] = {0.0, 0.0, 0.0};
    interp<3, 3>(pt, fn, n0);
    interp_grad<3, 3>(pt, X, Xxi, Xeta);
    interp_grad<3, 3>(pt, fn, nxi, neta);
    frame(Xxi, Xeta, n0, Xd);
    frame(nxi, neta, zero, Xdz);
    shell_transform(dat, Xxi, n0, Tm);
  }
  {
    T d0[3], d0xi[3], d0eta[3], uxi[3], ueta[3], zero[3] = {0.0, 0.0, 0.0};
    interp<3, 3>(pt, d, d0);
    interp_grad<3, 3>(pt, d, d0xi, d0eta);
    interp_grad<6, 3>(pt, vars, uxi, ueta);
    frame(uxi, ueta, d0, u0x);
    frame(d0xi, d0eta, zero, u1x);
  }
  T XdinvT[9], detXd;
  {
    T Xdinv[9], tmp[9], XdinvzT[9];
    inv3(Xd, Xdinv);
    detXd = det3(Xd);
    mm3(Xdinv, Tm, XdinvT);
    mm3(Xdinv, Xdz, tmp);
    for (int i = 0; i < 9; i++) tmp[i] = -tmp[i];
    mm3(tmp, XdinvT, XdinvzT);
    T a[9], b[9];
    mm3(u1x, XdinvT, a);
    mm3(u0x, XdinvzT, b);
    for (int i = 0; i < 9; i++) a[i] += b[i];
    mm3(Tm, a, u1x, true, false);
    mm3(u0x, XdinvT, a);
    mm3(Tm, a, u0x, true, false);
  }
  {
    T gty[6];
    interp_tying(pt, ety, gty);
    sym_rotate(XdinvT, gty, e0ty);
  }
  return detXd;
}
// ShellComputeDispGradSens (basis.h:514-595), additive into res/d_bar/ety_bar
template <class T>
inline void disp_grad_sens(const T pt[2], const ShellData& dat, const T X[12], const T fn[12],
                           const T u0xb[9], const T u1xb[9], const T e0tyb[6], T* res,
                           T d_bar[12], T ety_bar[9]) {
  T Tm[9], Xd[9], Xdz[9];
  {
    T Xxi[3], Xeta[3], nxi[3], neta[3], n0[3], zero[3] = {0.0, 0.0, 0.0};
    interp<3, 3>(pt, fn, n0);
    interp_grad<3, 3>(pt, X, Xxi, Xeta);
    interp_grad<3, 3>(pt, fn, nxi, neta);
    frame(Xxi, Xeta, n0, Xd);
    frame(nxi, neta, zero, Xdz);
    shell_transform(dat, Xxi, n0, Tm);
  }
  T XdinvT[9];
  {
    T Xdinv[9], tmp[9], XdinvzT[9];
    inv3(Xd, Xdinv);
    mm3(Xdinv, Tm, XdinvT);
    mm3(Xdinv, Xdz, tmp);
    for (int i = 0; i < 9; i++) tmp[i] = -tmp[i];
    mm3(tmp, XdinvT, XdinvzT);
    // u0d_bar^T = XdinvT u0x_bar^T T^T + XdinvzT u1x_bar^T T^T
    T u0dT[9], a[9];
    mm3(XdinvT, u0xb, tmp, false, true);
    mm3(tmp, Tm, u0dT, false, true);
    mm3(XdinvzT, u1xb, tmp, false, true);
    mm3(tmp, Tm, a, false, true);
    for (int i = 0; i < 9; i++) u0dT[i] += a[i];
    interp_T<3, 3>(pt, &u0dT[6], d_bar);
    interp_grad_T<6, 3>(pt, &u0dT[0], &u0dT[3], res);
    // u1d_bar^T = XdinvT u1x_bar^T T^T
    T u1dT[9];
    mm3(XdinvT, u1xb, tmp, false, true);
    mm3(tmp, Tm, u1dT, false, true);
    interp_grad_T<3, 3>(pt, &u1dT[0], &u1dT[3], d_bar);
  }
  {
    T gb[6];
    sym_rotate_T(XdinvT, e0tyb, gb);
    interp_tying_T(pt, gb, ety_bar);
  }
}

// ------------------------------------------------------- strain and stress
// LinearShellStrainCore / Reverse (a2d/a2dshellstrain.h:13-70)
template <class T>
inline void shell_strain(const T u1x[9], const T e0ty[6], const T& et, T E[9]) {
  E[0] = e0ty[0];
  E[1] = e0ty[3];
  E[2] = 2.0 * e0ty[1];
  E[3] = u1x[0];
  E[4] = u1x[4];
  E[5] = u1x[1] + u1x[3];
  E[6] = 2.0 * e0ty[4];
  E[7] = 2.0 * e0ty[2];
  E[8] = et;
}
template <class T>
inline void shell_strain_T(const T Eb[9], T u1xb[9], T e0tyb[6], T& etb) {
  e0tyb[0] += Eb[0];
  e0tyb[3] += Eb[1];
  e0tyb[1] += 2.0 * Eb[2];
  u1xb[0] += Eb[3];
  u1xb[4] += Eb[4];
  u1xb[1] += Eb[5];
  u1xb[3] += Eb[5];
  e0tyb[4] += 2.0 * Eb[6];
  e0tyb[2] += 2.0 * Eb[7];
  etb += Eb[8];
}
// IsotropicShellStressCore (a2d/a2disotropicshellstress.h:12-51): S = D E.
// D is symmetric, so the reverse (lines 53-90, overwrite semantics) is the
// same map applied to the stress seed.
template <class T>
inline void symv3(double s, const double C[6], const T* x, T* y, bool add) {
  T r0 = C[0] * x[0] + C[1] * x[1] + C[2] * x[2];
  T r1 = C[1] * x[0] + C[3] * x[1] + C[4] * x[2];
  T r2 = C[2] * x[0] + C[4] * x[1] + C[5] * x[2];
  if (add) {
    y[0] += s * r0; y[1] += s * r1; y[2] += s * r2;
  } else {
    y[0] = s * r0; y[1] = s * r1; y[2] = s * r2;
  }
}
template <class T>
inline void shell_stress(const ShellData& d, const T E[9], T S[9]) {
  const double Dm = d.E / (1.0 - d.nu * d.nu);
  const double C[6] = {Dm, d.nu * Dm, 0.0, Dm, 0.0, d.E / 2.0 / (1.0 + d.nu)};
  const double t = d.thick, to = d.tOffset;
  symv3(t, C, &E[0], &S[0], false);
  symv3(-t * t * to, C, &E[3], &S[0], true);
  symv3(-t * t * to, C, &E[0], &S[3], false);
  symv3(t * t * t / 12.0, C, &E[3], &S[3], true);
  symv3(t * t * t * to * to, C, &E[3], &S[3], true);
  const double As = kShearCorrection * t * C[5];
  S[6] = As * E[6];
  S[7] = As * E[7];
  S[8] = kDrillReg * As * E[8];
}

// ----------------------------------------------- per-quadrature-point ops
template <class T>
struct QuadFwd {
  T fn[12], d[12], ety[9], u0x[9], u1x[9], e0ty[6], et, detXd, scale, pt[2];
};
template <class T>
inline void quad_forward(int iq, const ShellData& dat, const T X[12], const T* vars,
                         QuadFwd<T>& f) {
  double w = quad_point(iq, f.pt);
  node_normals(X, f.fn);
  drill_strain(f.pt, dat, X, vars, f.fn, f.et);
  director(vars, f.fn, f.d);
  tying_strain(X, f.fn, vars, f.d, f.ety);
  f.detXd = disp_grad(f.pt, dat, X, vars, f.fn, f.d, f.ety, f.u0x, f.u1x, f.e0ty);
  f.scale = f.detXd * w;
}
// Backpropagate strain seed Eb to the element DOFs (reverse chain of
// elem_group.h:155-175).
template <class T>
inline void quad_reverse(const QuadFwd<T>& f, const ShellData& dat, const T X[12],
                         const T Eb[9], T* out) {
  T u0xb[9], u1xb[9], e0tyb[6], etb = 0.0;
  for (int i = 0; i < 9; i++) u0xb[i] = u1xb[i] = 0.0;
  for (int i = 0; i < 6; i++) e0tyb[i] = 0.0;
  shell_strain_T(Eb, u1xb, e0tyb, etb);
  T d_bar[12], ety_bar[9];
  for (int i = 0; i < 12; i++) d_bar[i] = 0.0;
  for (int i = 0; i < 9; i++) ety_bar[i] = 0.0;
  disp_grad_sens(f.pt, dat, X, f.fn, u0xb, u1xb, e0tyb, out, d_bar, ety_bar);
  drill_strain_sens(f.pt, dat, X, f.fn, etb, out);
  tying_strain_sens(X, f.fn, ety_bar, out, d_bar);
  director_sens(f.fn, d_bar, out);
}

// add_element_quadpt_energy (shell/elem_group.h:41-95): U += 0.5 scale E.S
template <class T>
inline T element_energy(const ShellData& dat, const T X[12], const T vars[24]) {
  T U = 0.0;
  for (int q = 0; q < 4; q++) {
    QuadFwd<T> f;
    quad_forward(q, dat, X, vars, f);
    T E[9], S[9];
    shell_strain(f.u1x, f.e0ty, f.et, E);
    shell_stress(dat, E, S);
    T es = 0.0;
    for (int i = 0; i < 9; i++) es += E[i] * S[i];
    U += 0.5 * f.scale * es;
  }
  return U;
}

// add_element_quadpt_residual (shell/elem_group.h:98-180): res += B^T scale D E
template <class T>
inline void element_residual(const ShellData& dat, const T X[12], const T vars[24],
                             T res[24]) {
  for (int q = 0; q < 4; q++) {
    QuadFwd<T> f;
    quad_forward(q, dat, X, vars, f);
    T E[9], S[9], Eb[9];
    shell_strain(f.u1x, f.e0ty, f.et, E);
    T Es[9];
    for (int i = 0; i < 9; i++) Es[i] = f.scale * E[i];
    shell_stress(dat, Es, Eb);  // overwrite semantics: Eb = D (scale E)
    (void)S;
    quad_reverse(f, dat, X, Eb, res);
  }
}

// add_element_quadpt_jacobian_col (shell/elem_group.h:183-303), looped over
// the 24 columns and 4 quadrature points exactly as add_jacobian_cpu
// (base/elem_group.h:121-181) does: per (column, quadrature point) a forward
// pass, a unit-seed forward pass, the first-order reverse into the residual
// and the second-order reverse into the column. K is stored row-major with
// K[24*i + j]; it is symmetric. The residual collects 24 copies and is
// scaled by 1/24 (base/elem_group.h:174).
template <class T>
inline void element_jacobian(const ShellData& dat, const T X[12], const T vars[24], T res[24],
                             T K[576]) {
  T racc[24];
  for (int i = 0; i < 24; i++) racc[i] = 0.0;
  for (int iv = 0; iv < 24; iv++) {
    T col[24];
    for (int i = 0; i < 24; i++) col[i] = 0.0;
    T p[24];
    for (int i = 0; i < 24; i++) p[i] = 0.0;
    p[iv] = 1.0;
    for (int q = 0; q < 4; q++) {
      QuadFwd<T> f, pf;
      quad_forward(q, dat, X, vars, f);
      // hforward: the maps are linear, so the seed pass is a forward pass on p
      quad_forward(q, dat, X, p, pf);
      T E[9], Es[9], Eb[9];
      shell_strain(f.u1x, f.e0ty, f.et, E);
      for (int i = 0; i < 9; i++) Es[i] = f.scale * E[i];
      shell_stress(dat, Es, Eb);
      quad_reverse(f, dat, X, Eb, racc);
      T pE[9], pEs[9], hb[9];
      shell_strain(pf.u1x, pf.e0ty, pf.et, pE);
      for (int i = 0; i < 9; i++) pEs[i] = f.scale * pE[i];
      shell_stress(dat, pEs, hb);
      quad_reverse(f, dat, X, hb, col);
    }
    for (int i = 0; i < 24; i++) K[24 * iv + i] = col[i];
  }
  for (int i = 0; i < 24; i++) res[i] += racc[i] * (1.0 / 24.0);
}

}  // namespace oracle
