// Driver written against the C++ facade the way the reference's drivers are
// written (examples/plate_demo/linear_static.cu:12-73 and the ILU-GMRES of
// examples/iterative/gmres.cu): template composition of the shell element,
// ElementAssembler, createBsrMat, add_jacobian, apply_bcs, the direct LU
// solve, ILUk_Preconditioner with GMRES, add_energy.
// Usage: linear_static <mesh.bin> <output prefix> [mesh.bdf]
// mesh.bin (little-endian): int32 nn, ne, nbc; float64 E, nu; int32 conn[4 ne];
// float64 xpts[3 nn]; int32 bcs[nbc]; float64 thick[ne]; float64 loads[6 nn].
// Writes <prefix>.pattern (int32 nn, nnzb, rowPtr, colPtr, perm),
// <prefix>.K (36 nnzb float64), <prefix>.x_direct / .x_gmres (6 nn float64,
// natural order) and <prefix>.info (float64 energy, direct residual, GMRES
// residual, GMRES steps).
#include <cstdio>
#include <vector>

#include "gpufem/gpufem.hpp"
using namespace gpufem;

template <class V>
static bool rd(FILE* f, V* p, size_t n) {
  return fread(p, sizeof(V), n, f) == n;
}
template <class V>
static void wr(const std::string& path, const V* p, size_t n) {
  FILE* f = fopen(path.c_str(), "wb");
  fwrite(p, sizeof(V), n, f);
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  using T = double;
  using Quad = QuadLinearQuadrature<T>;
  using Director = LinearizedRotation<T>;
  using Basis = ShellQuadBasis<T, Quad, 2>;
  constexpr bool has_ref_axis = false;
  using Data = ShellIsotropicData<T, has_ref_axis>;
  using Physics = IsotropicShell<T, Data>;
  using ElemGroup = ShellElementGroup<T, Director, Basis, Physics>;
  using Assembler = ElementAssembler<T, ElemGroup, VecType, BsrMat>;

  FILE* f = fopen(argv[1], "rb");
  if (!f) return 3;
  int32_t nn, ne, nbc;
  double E, nu;
  bool ok = rd(f, &nn, 1) && rd(f, &ne, 1) && rd(f, &nbc, 1) && rd(f, &E, 1) && rd(f, &nu, 1);
  std::vector<int32_t> conn(4 * (size_t)ne), bcv(nbc);
  std::vector<double> xp(3 * (size_t)nn), th(ne), ld(6 * (size_t)nn);
  ok = ok && rd(f, conn.data(), conn.size()) && rd(f, xp.data(), xp.size()) &&
       rd(f, bcv.data(), bcv.size()) && rd(f, th.data(), th.size()) &&
       rd(f, ld.data(), ld.size());
  fclose(f);
  if (!ok) return 4;
  const std::string out = argv[2];
  try {
    HostVec<int32_t> geo_conn(4 * ne, conn.data());
    HostVec<T> xpts(3 * nn, xp.data());
    HostVec<int> bcs(nbc, bcv.data());
    HostVec<Data> physData(ne);
    for (int e = 0; e < ne; e++) physData[e] = Data(E, nu, th[e]);
    Assembler assembler(nn, nn, ne, geo_conn, geo_conn, xpts, bcs, physData);
    if (argc > 3) {  // the same mesh from a BDF file: same counts
      TACSMeshLoader<T> loader;
      loader.scanBDFFile(argv[3]);
      Assembler from_bdf = Assembler::createFromBDF(loader, physData[0]);
      if (from_bdf.get_num_nodes() != nn || from_bdf.get_num_elements() != ne) return 6;
    }

    bool print = false;
    assembler.symbolic_factorization(10.0, print);
    auto vars = assembler.createVarsVec();
    assembler.set_variables(vars);
    auto res = assembler.createVarsVec();
    auto soln = assembler.createVarsVec();
    auto kmat = createBsrMat<Assembler, VecType<T>>(assembler);
    assembler.add_jacobian(res, kmat, print);
    assembler.apply_bcs(res, print);
    assembler.apply_bcs(kmat, print);
    auto loads = assembler.createVarsVec(ld.data());
    assembler.apply_bcs(loads, true);
    gf_solve_stats sd = CUSPARSE::direct_LU_solve_old<T>(kmat, loads, soln, true);

    // ILU(2)-GMRES on the same system (the preconditioner matrix's BsrData
    // carries the fill level, as the reference's ILU pattern would)
    BsrData pbd = kmat.getBsrData();
    pbd.fill_level = 2;
    BsrMat<VecType<T>> precond_mat(pbd);
    ILUk_Preconditioner<VecType<T>> precond(precond_mat, kmat);
    precond.copyValues();
    precond.factor();
    auto x_gmres = assembler.createVarsVec();
    gf_solve_opts opts;
    gf_solve_opts_default(&opts);
    opts.restart = 200;
    opts.max_iters = 4000;
    opts.rtol = 1e-10;
    gf_solve_stats sg = gmres_solve(assembler, kmat, precond, loads, x_gmres, &opts);

    // strain energy at the solution: U = 1/2 u^T K u = 1/2 b^T u
    assembler.set_variables(soln);
    T U = 0.0;
    assembler.add_energy(U);

    BsrData bd = assembler.getBsrData();
    std::vector<int32_t> pat;
    pat.push_back(bd.nnodes);
    pat.push_back(bd.nnzb);
    pat.insert(pat.end(), kmat.getRowPtr(), kmat.getRowPtr() + bd.nnodes + 1);
    pat.insert(pat.end(), kmat.getColPtr(), kmat.getColPtr() + bd.nnzb);
    pat.insert(pat.end(), kmat.getPerm(), kmat.getPerm() + bd.nnodes);
    wr(out + ".pattern", pat.data(), pat.size());
    HostVec<T> hk = kmat.createHostVec();
    wr(out + ".K", hk.getPtr(), (size_t)hk.getSize());
    HostVec<T> hd = soln.createHostVec(), hg = x_gmres.createHostVec();
    wr(out + ".x_direct", hd.getPtr(), (size_t)hd.getSize());
    wr(out + ".x_gmres", hg.getPtr(), (size_t)hg.getSize());
    double info[4] = {U, sd.rel_residual, sg.rel_residual, (double)sg.iterations};
    wr(out + ".info", info, 4);
  } catch (const Error& e) {
    fprintf(stderr, "%s\n", e.what());
    return 5;
  }
  return 0;
}
