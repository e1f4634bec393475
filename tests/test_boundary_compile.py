"""The drop-in boundary builds: a C++ driver written against the facade
(include/gpufem/gpufem.hpp) and a C program written against the C ABI
(include/gpufem.h), both shaped like the examples in INTEGRATION.md, compile
and link against libgpufem.so. Nothing is run (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
LIB_DIR = os.path.join(ROOT, "gpu_fem_b200")

CPP_DRIVER = r"""
#include "gpufem/gpufem.hpp"
using namespace gpufem;

int run(int nn, int ne, const int* conn_ptr, const double* xpts_ptr, int nbc,
        const int* bcs_ptr, const double* loads) {
  HostVec<int> conn(4 * ne, conn_ptr), bcs(nbc, bcs_ptr);
  HostVec<double> xpts(3 * nn, xpts_ptr);
  HostVec<gf_shell_data> data(ne);
  for (int e = 0; e < ne; e++) data[e] = ShellIsotropicData(70e9, 0.3, 0.005);
  ElementAssembler assembler(nn, nn, ne, conn, conn, xpts, bcs, data, GF_ORDER_RCM);
  auto kmat = createBsrMat(assembler);
  auto res = assembler.createVarsVec();
  assembler.add_jacobian(res, kmat);
  assembler.apply_bcs(res);
  assembler.apply_bcs(kmat);
  ILUk_Preconditioner precond(assembler, 2);
  precond.factor(kmat);
  DeviceVec<double> rhs(HostVec<double>(6 * nn, loads)), soln(6 * nn);
  gf_solve_opts opts;
  gf_solve_opts_default(&opts);
  opts.rtol = 1e-8;
  gf_solve_stats st = gmres_solve(assembler, kmat, precond, rhs, soln, &opts);
  // the rest of the reference surface the facade keeps
  assembler.symbolic_factorization();
  BsrData bd = assembler.getBsrData();
  auto kcopy = createBsrMat(assembler);
  kmat.copyValuesTo(kcopy);
  HostVec<double> hx = soln.createHostVec();
  DeviceVec<double> dx = hx.createDeviceVec();
  return st.iterations + bd.nnzb + assembler.getXpts().getSize() + dx.getSize();
}

int main() { return 0; }
"""

C_DRIVER = r"""
#include <stddef.h>
#include "gpufem.h"

int run(int nn, int ne, const int* conn, const double* xpts, const int* bcs, int nbc,
        const gf_shell_data* data, const double* d_loads, double* d_x, void* stream) {
  gf_mesh_desc d = {0};
  d.num_nodes = nn;
  d.num_elements = ne;
  d.conn = conn;
  d.xpts = xpts;
  d.bcs = bcs;
  d.num_bcs = nbc;
  d.data = data;
  d.ordering = GF_ORDER_NATURAL;
  gf_assembler* a;
  if (gf_assembler_create(&d, &a) != GF_OK) return -1;
  gf_bsr* K;
  gf_bsr_create(a, &K);
  gf_add_jacobian(a, NULL, K, GF_ASSEMBLE_FUSE_BCS, stream);
  gf_precond* P;
  gf_precond_create(a, 6, GF_PREC_FP32, &P);
  gf_precond_factor(P, K, stream);
  gf_solve_opts o;
  gf_solve_opts_default(&o);
  o.side = 1;
  o.rtol = 1e-8;
  gf_solve_stats s;
  gf_status st = gf_gmres_solve(a, K, P, d_loads, d_x, &o, &s, stream);
  gf_precond_destroy(P);
  gf_bsr_destroy(K);
  gf_assembler_destroy(a);
  return (int)st;
}

int main(void) { return 0; }
"""


def _need(tool):
    if shutil.which(tool) is None:
        pytest.skip(f"{tool} not available")
    if not os.path.exists(os.path.join(CUDA, "include", "cuda_runtime.h")):
        pytest.skip("CUDA headers not available")
    if not os.path.exists(os.path.join(LIB_DIR, "libgpufem.so")):
        pytest.skip("libgpufem.so not built")


def _build(compiler, src, suffix, std, tmp_path):
    path = tmp_path / f"driver{suffix}"
    path.write_text(src)
    out = tmp_path / "driver"
    cmd = [compiler, std, str(path), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), "-L", LIB_DIR, "-lgpufem",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_facade_driver_compiles_and_links(tmp_path):
    _need("g++")
    _build("g++", CPP_DRIVER, ".cpp", "-std=c++17", tmp_path)


def test_c_abi_driver_compiles_and_links(tmp_path):
    _need("gcc")
    _build("gcc", C_DRIVER, ".c", "-std=c11", tmp_path)
