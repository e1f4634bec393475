// Linear MITC4 shell element in explicit strain-displacement form.
//
// The reference evaluates the element with A2D forward/reverse sweeps per
// (element, quadrature point, Jacobian column)
// (include/shell/elem_group.h:98-303). Every map on that path is linear in
// the DOFs, so this file writes the same strains as E_q = B_q u with the
// 9 x 24 matrix B_q built column by column from per-element geometry that is
// computed once:
//   membrane/shear rows  e0ty = (Xd^-1 T)^T gty (Xd^-1 T) from the MITC tying
//                        strains (include/shell/physics.h:94-209,
//                        include/shell/basis.h:314-502)
//   bending rows         u1x = T^T (u1d Xd^-1 T + u0d XdinvzT)
//                        (include/shell/basis.h:452-493)
//   drilling row         nodal drill strains interpolated to the point
//                        (include/shell/shell_utils.h:42-105)
// with the strain vector of LinearShellStrainCore
// (include/shell/a2d/a2dshellstrain.h:13-30) and the isotropic ABD stress of
// IsotropicShellStressCore (include/shell/a2d/a2disotropicshellstress.h:12-51).
// Then K_e = sum_q w_q detXd_q B_q^T D B_q and R_e = K_e u_e, which is the
// Hessian / gradient of the energy U = 1/2 sum_q w_q detXd_q E.S
// (include/shell/physics.h:19-37).
//
// Everything here is __host__ __device__ so the same code can be compiled
// for the CPU when checking the algebra.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define GF_HD __host__ __device__ __forceinline__
#else
#define GF_HD inline
#endif

namespace gf {

constexpr double kRt3 = 0.577350269189626;    // include/shell/quadrature.h:9
constexpr double kShear = 5.0 / 6.0;          // include/shell/data.h:11
constexpr double kDrill = 10.0;               // include/shell/data.h:12

// Material entry; per-element thickness is stored separately.
struct Material {
  double E, nu, tOffset;
  double refAxis[3];
  int has_ref_axis;
  int pad;
};

// Node sign pattern of the tensor-product basis: node a sits at
// (xi_a, eta_a) = (-1 + 2 (a % 2), -1 + 2 (a / 2))  (basis.h:138-142).
GF_HD double node_xi(int a) { return (a & 1) ? 1.0 : -1.0; }
GF_HD double node_eta(int a) { return (a & 2) ? 1.0 : -1.0; }

// Bilinear shape function and its parametric derivatives at (xi, eta).
GF_HD void shape(int a, double xi, double eta, double& N, double& Nx, double& Ne) {
  const double sa = node_xi(a), ta = node_eta(a);
  const double fx = 0.5 * (1.0 + sa * xi), fe = 0.5 * (1.0 + ta * eta);
  N = fx * fe;
  Nx = 0.5 * sa * fe;
  Ne = 0.5 * ta * fx;
}

GF_HD void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
GF_HD double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// Interpolated value and gradients of a 3-vector nodal field f[4][3].
GF_HD void interp3(const double* f, double xi, double eta, double* v, double* dxi,
                   double* deta) {
  for (int k = 0; k < 3; k++) v[k] = dxi[k] = deta[k] = 0.0;
  for (int a = 0; a < 4; a++) {
    double N, Nx, Ne;
    shape(a, xi, eta, N, Nx, Ne);
    for (int k = 0; k < 3; k++) {
      v[k] += N * f[3 * a + k];
      dxi[k] += Nx * f[3 * a + k];
      deta[k] += Ne * f[3 * a + k];
    }
  }
}

// 3x3 inverse (row-major) and determinant.
GF_HD double inv3(const double* A, double* B) {
  const double c0 = A[4] * A[8] - A[5] * A[7];
  const double c1 = A[3] * A[8] - A[5] * A[6];
  const double c2 = A[3] * A[7] - A[4] * A[6];
  const double det = A[0] * c0 - A[1] * c1 + A[2] * c2;
  const double id = 1.0 / det;
  B[0] = c0 * id;
  B[1] = -(A[1] * A[8] - A[2] * A[7]) * id;
  B[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  B[3] = -c1 * id;
  B[4] = (A[0] * A[8] - A[2] * A[6]) * id;
  B[5] = -(A[0] * A[5] - A[2] * A[3]) * id;
  B[6] = c2 * id;
  B[7] = -(A[0] * A[7] - A[1] * A[6]) * id;
  B[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return det;
}
GF_HD void mm3(const double* A, const double* B, double* C) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

// ShellComputeTransform (include/shell/shell_utils.h:4-40): columns
// (t1, n x t1, n) with t1 = refAxis or dX/dxi projected off the normal.
GF_HD void shell_transform(const Material& m, const double* Xxi, const double* n0, double* T) {
  const double nn = sqrt(dot3(n0, n0));
  const double nh[3] = {n0[0] / nn, n0[1] / nn, n0[2] / nn};
  double t1[3];
  for (int i = 0; i < 3; i++) t1[i] = m.has_ref_axis ? m.refAxis[i] : Xxi[i];
  const double d = dot3(nh, t1);
  double tmp[3];
  for (int i = 0; i < 3; i++) tmp[i] = t1[i] - d * nh[i];
  const double tn = sqrt(dot3(tmp, tmp));
  const double t1h[3] = {tmp[0] / tn, tmp[1] / tn, tmp[2] / tn};
  double t2h[3];
  cross3(nh, t1h, t2h);
  for (int i = 0; i < 3; i++) {
    T[3 * i] = t1h[i];
    T[3 * i + 1] = t2h[i];
    T[3 * i + 2] = nh[i];
  }
}

// Per-element geometry shared by all 24 DOF columns.
struct ElemGeom {
  double fn[12];        // unit node normals (ShellComputeNodeNormals, basis.h:292-311)
  // drill strain, per node n: rows c of T_n (first two columns), rows 0/1 of
  // Xd_n^-1 T_n, and t0 x t1 of T_n
  double Tn01[4][6];    // [c*2 + i] = T_n[c][i], i in {0,1}
  double XTn[4][6];     // [r*3 + j] = (Xd_n^-1 T_n)[r][j], r in {0,1}
  double tcross[4][3];  // T_n[:,0] x T_n[:,1]
  // quadrature points
  double T[4][9];       // shell transform
  double A[4][9];       // Xd^-1 T
  double Az[4][9];      // XdinvzT = -Xd^-1 Xdz Xd^-1 T
  double scale[4];      // detXd * weight
  // tying points: g11/g13 at (0, -1), (0, 1); g22/g23 at (-1, 0), (1, 0); g12 at (0, 0)
  double Xxi_t[2][3], n0_xi_t[2][3];    // at (0, eta_j)
  double Xeta_t[2][3], n0_eta_t[2][3];  // at (xi_i, 0)
  double Xxi_c[3], Xeta_c[3];           // at (0, 0)
};

GF_HD void quad_point(int q, double& xi, double& eta) {
  xi = (q & 1) ? kRt3 : -kRt3;
  eta = (q & 2) ? kRt3 : -kRt3;
}

// ---- geometry pieces (each independent, so warps can spread them over lanes)
GF_HD void geom_normal(const double* X, int n, double* fn_n) {
  double v[3], xi[3], eta[3], c[3];
  interp3(X, node_xi(n), node_eta(n), v, xi, eta);
  cross3(xi, eta, c);
  const double nrm = sqrt(dot3(c, c));
  for (int k = 0; k < 3; k++) fn_n[k] = (1.0 / nrm) * c[k];
}
GF_HD void geom_node(const Material& m, const double* X, const double* fn, int n,
                     double* Tn01, double* XTn, double* tc) {
  double v[3], xi[3], eta[3];
  interp3(X, node_xi(n), node_eta(n), v, xi, eta);
  const double* f = &fn[3 * n];
  double Xd[9], Xdi[9], T[9], XT[9];
  for (int i = 0; i < 3; i++) {
    Xd[3 * i] = xi[i];
    Xd[3 * i + 1] = eta[i];
    Xd[3 * i + 2] = f[i];
  }
  shell_transform(m, xi, f, T);
  inv3(Xd, Xdi);
  mm3(Xdi, T, XT);
  for (int c = 0; c < 3; c++) {
    Tn01[2 * c] = T[3 * c];
    Tn01[2 * c + 1] = T[3 * c + 1];
  }
  for (int j = 0; j < 6; j++) XTn[j] = XT[j];
  const double t0[3] = {T[0], T[3], T[6]}, t1[3] = {T[1], T[4], T[7]};
  cross3(t0, t1, tc);
}
GF_HD void geom_quad(const Material& m, const double* X, const double* fn, int q, double* T,
                     double* A, double* Az, double& scale) {
  double xi, eta;
  quad_point(q, xi, eta);
  double xv[3], Xxi[3], Xeta[3], n0[3], nxi[3], neta[3];
  interp3(X, xi, eta, xv, Xxi, Xeta);
  interp3(fn, xi, eta, n0, nxi, neta);
  double Xd[9], Xdz[9], Xdi[9];
  for (int i = 0; i < 3; i++) {
    Xd[3 * i] = Xxi[i];
    Xd[3 * i + 1] = Xeta[i];
    Xd[3 * i + 2] = n0[i];
    Xdz[3 * i] = nxi[i];
    Xdz[3 * i + 1] = neta[i];
    Xdz[3 * i + 2] = 0.0;
  }
  shell_transform(m, Xxi, n0, T);
  const double det = inv3(Xd, Xdi);
  mm3(Xdi, T, A);
  double tmp[9];
  mm3(Xdi, Xdz, tmp);
  mm3(tmp, A, Az);
  for (int i = 0; i < 9; i++) Az[i] = -Az[i];
  scale = det;  // quadrature weight is 1 (quadrature.h:13-17)
}
// k in 0..4: 0,1 -> (0, -1), (0, 1); 2,3 -> (-1, 0), (1, 0); 4 -> (0, 0)
GF_HD void geom_tying(const double* X, const double* fn, int k, ElemGeom& g) {
  double xi = 0.0, eta = 0.0;
  if (k < 2) eta = k ? 1.0 : -1.0;
  else if (k < 4) xi = (k == 3) ? 1.0 : -1.0;
  double xv[3], Xxi[3], Xeta[3], n0[3], d1[3], d2[3];
  interp3(X, xi, eta, xv, Xxi, Xeta);
  interp3(fn, xi, eta, n0, d1, d2);
  for (int i = 0; i < 3; i++) {
    if (k < 2) {
      g.Xxi_t[k][i] = Xxi[i];
      g.n0_xi_t[k][i] = n0[i];
    } else if (k < 4) {
      g.Xeta_t[k - 2][i] = Xeta[i];
      g.n0_eta_t[k - 2][i] = n0[i];
    } else {
      g.Xxi_c[i] = Xxi[i];
      g.Xeta_c[i] = Xeta[i];
    }
  }
}

GF_HD void compute_geom(const Material& m, const double* X, ElemGeom& g) {
  for (int n = 0; n < 4; n++) geom_normal(X, n, &g.fn[3 * n]);
  for (int n = 0; n < 4; n++) geom_node(m, X, g.fn, n, g.Tn01[n], g.XTn[n], g.tcross[n]);
  for (int q = 0; q < 4; q++) geom_quad(m, X, g.fn, q, g.T[q], g.A[q], g.Az[q], g.scale[q]);
  for (int k = 0; k < 5; k++) geom_tying(X, g.fn, k, g);
}

// Column l = 6a + c of B_q for all four quadrature points: Bc[q*9 + k].
GF_HD void bmat_column(const ElemGeom& g, int l, double* Bc) {
  const int a = l / 6, c = l % 6;
  const bool rot = c >= 3;
  double v[3] = {0.0, 0.0, 0.0};  // director sensitivity e_k x fn_a (director.h:98-107)
  if (rot) {
    const int k = c - 3;
    const double e[3] = {k == 0 ? 1.0 : 0.0, k == 1 ? 1.0 : 0.0, k == 2 ? 1.0 : 0.0};
    cross3(e, &g.fn[3 * a], v);
  }
  // MITC tying strain sensitivities (physics.h:94-209), order
  // g11(2) g22(2) g12(1) g23(2) g13(2)
  double ety[9];
  for (int j = 0; j < 2; j++) {  // points (0, eta_j)
    const double eta = j ? 1.0 : -1.0;
    double N, Nx, Ne;
    shape(a, 0.0, eta, N, Nx, Ne);
    if (!rot) {
      ety[0 + j] = Nx * g.Xxi_t[j][c];
      ety[7 + j] = 0.5 * g.n0_xi_t[j][c] * Nx;
    } else {
      ety[0 + j] = 0.0;
      ety[7 + j] = 0.5 * dot3(g.Xxi_t[j], v) * N;
    }
  }
  for (int i = 0; i < 2; i++) {  // points (xi_i, 0)
    const double xi = i ? 1.0 : -1.0;
    double N, Nx, Ne;
    shape(a, xi, 0.0, N, Nx, Ne);
    if (!rot) {
      ety[2 + i] = Ne * g.Xeta_t[i][c];
      ety[5 + i] = 0.5 * g.n0_eta_t[i][c] * Ne;
    } else {
      ety[2 + i] = 0.0;
      ety[5 + i] = 0.5 * dot3(g.Xeta_t[i], v) * N;
    }
  }
  {
    double N, Nx, Ne;
    shape(a, 0.0, 0.0, N, Nx, Ne);
    ety[4] = rot ? 0.0 : 0.5 * (Nx * g.Xeta_c[c] + Ne * g.Xxi_c[c]);
  }
  // nodal drill strains (shell_utils.h:42-105): translations act through the
  // in-plane displacement gradient at every node, rotations through
  // C = I - skew(theta) at their own node.
  double etn[4];
  for (int n = 0; n < 4; n++) {
    if (!rot) {
      double N, Nx, Ne;
      shape(a, node_xi(n), node_eta(n), N, Nx, Ne);
      const double w0 = g.Tn01[n][2 * c], w1 = g.Tn01[n][2 * c + 1];
      const double s0 = Nx * g.XTn[n][0] + Ne * g.XTn[n][3];
      const double s1 = Nx * g.XTn[n][1] + Ne * g.XTn[n][4];
      etn[n] = 0.5 * (w1 * s0 - w0 * s1);
    } else {
      etn[n] = (n == a) ? -g.tcross[n][c - 3] : 0.0;
    }
  }
  for (int q = 0; q < 4; q++) {
    double xi, eta;
    quad_point(q, xi, eta);
    const double na0 = 0.5 * (1.0 - xi), na1 = 0.5 * (1.0 + xi);
    const double nb0 = 0.5 * (1.0 - eta), nb1 = 0.5 * (1.0 + eta);
    // interpTyingStrain (basis.h:314-368): packed (11, 12, 13, 22, 23, 33)
    const double g11 = nb0 * ety[0] + nb1 * ety[1];
    const double g22 = na0 * ety[2] + na1 * ety[3];
    const double g12 = ety[4];
    const double g23 = na0 * ety[5] + na1 * ety[6];
    const double g13 = nb0 * ety[7] + nb1 * ety[8];
    const double G[9] = {g11, g12, g13, g12, g22, g23, g13, g23, 0.0};
    const double* A = g.A[q];
    double H[9];  // H = G A
    mm3(G, A, H);
    // e_ab = sum_i A_ia H_ib
    double e00 = 0, e11 = 0, e01 = 0, e12 = 0, e02 = 0;
    for (int i = 0; i < 3; i++) {
      e00 += A[3 * i] * H[3 * i];
      e11 += A[3 * i + 1] * H[3 * i + 1];
      e01 += A[3 * i] * H[3 * i + 1];
      e12 += A[3 * i + 1] * H[3 * i + 2];
      e02 += A[3 * i] * H[3 * i + 2];
    }
    // bending: u1x = w r^T
    double N, Nx, Ne;
    shape(a, xi, eta, N, Nx, Ne);
    const double* T = g.T[q];
    const double* Az = g.Az[q];
    double w[2], r[2];
    if (!rot) {
      w[0] = T[3 * c];
      w[1] = T[3 * c + 1];
      r[0] = Nx * Az[0] + Ne * Az[3];
      r[1] = Nx * Az[1] + Ne * Az[4];
    } else {
      w[0] = T[0] * v[0] + T[3] * v[1] + T[6] * v[2];
      w[1] = T[1] * v[0] + T[4] * v[1] + T[7] * v[2];
      r[0] = Nx * A[0] + Ne * A[3] + N * Az[6];
      r[1] = Nx * A[1] + Ne * A[4] + N * Az[7];
    }
    double et = 0.0;
    for (int n = 0; n < 4; n++) {
      double Nn, dx, de;
      shape(n, xi, eta, Nn, dx, de);
      et += Nn * etn[n];
    }
    double* E = &Bc[9 * q];
    E[0] = e00;
    E[1] = e11;
    E[2] = 2.0 * e01;
    E[3] = w[0] * r[0];
    E[4] = w[1] * r[1];
    E[5] = w[0] * r[1] + w[1] * r[0];
    E[6] = 2.0 * e12;
    E[7] = 2.0 * e02;
    E[8] = et;
  }
}

// S = D E for the isotropic shell (a2disotropicshellstress.h:12-51), scaled.
GF_HD void stress(const Material& m, double t, double s, const double* E, double* S) {
  const double Dm = m.E / (1.0 - m.nu * m.nu);
  const double C0 = Dm, C1 = m.nu * Dm, C5 = m.E / 2.0 / (1.0 + m.nu);
  const double to = m.tOffset;
  const double a = s * t, b = -s * t * t * to, d = s * (t * t * t / 12.0 + t * t * t * to * to);
  const double m0 = C0 * E[0] + C1 * E[1], m1 = C1 * E[0] + C0 * E[1], m2 = C5 * E[2];
  const double k0 = C0 * E[3] + C1 * E[4], k1 = C1 * E[3] + C0 * E[4], k2 = C5 * E[5];
  S[0] = a * m0 + b * k0;
  S[1] = a * m1 + b * k1;
  S[2] = a * m2 + b * k2;
  S[3] = b * m0 + d * k0;
  S[4] = b * m1 + d * k1;
  S[5] = b * m2 + d * k2;
  const double As = kShear * t * C5;
  S[6] = s * As * E[6];
  S[7] = s * As * E[7];
  S[8] = s * kDrill * As * E[8];
}

}  // namespace gf
