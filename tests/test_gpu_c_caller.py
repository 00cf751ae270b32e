"""The library used from a plain C program, the way the reference's compiled
caller uses it: no Python in the process, only include/eafcg.h and
libeafcg.so. The program reads a system written by the test, solves it with
eaf_cg_solve_f64 and writes phi back; the result must equal the solve of the
same system through the Python binding bit for bit (same library, same
launch), and the program's argument errors must come back as status codes."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gen, pkg

pytestmark = pytest.mark.gpu

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "eafcg.h"

static double* read_array(const char* dir, const char* name, size_t n) {
  char path[4096];
  snprintf(path, sizeof(path), "%s/%s.bin", dir, name);
  FILE* f = fopen(path, "rb");
  if (!f) return NULL;
  double* a = (double*)malloc(n * sizeof(double));
  size_t got = a ? fread(a, sizeof(double), n, f) : 0;
  fclose(f);
  if (got != n) { free(a); return NULL; }
  return a;
}

int main(int argc, char** argv) {
  if (argc != 7) return 64;
  const char* dir = argv[1];
  const int nr = atoi(argv[2]), nth = atoi(argv[3]), nz = atoi(argv[4]);
  const int max_iter = atoi(argv[5]);
  const double tol = atof(argv[6]);
  const size_t n = (size_t)(nr + 4) * (nth + 4) * (nz + 4);
  const char* names[9] = {"aW", "aE", "aS", "aN", "aB", "aT", "aP", "Su", "phi"};
  double* a[9];
  for (int i = 0; i < 9; ++i)
    if (!(a[i] = read_array(dir, names[i], n))) return 65;
  eaf_cg_t h;
  if (eaf_cg_create(NULL, nr, nth, nz, 0) != EAF_EINVAL) return 66;
  int st = eaf_cg_create(&h, nr, nth, nz, 0);
  if (st != EAF_OK) { fprintf(stderr, "create: %s\n", eaf_last_error()); return 67; }
  double res = 0.0;
  int it = 0;
  if (eaf_cg_solve_f64(h, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], NULL,
                       max_iter, tol, &res, &it) != EAF_EINVAL) return 68;
  st = eaf_cg_solve_f64(h, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8],
                        max_iter, tol, &res, &it);
  eaf_cg_destroy(h);
  char path[4096];
  snprintf(path, sizeof(path), "%s/phi_out.bin", dir);
  FILE* f = fopen(path, "wb");
  if (!f || fwrite(a[8], sizeof(double), n, f) != n) return 69;
  fclose(f);
  printf("%d %d %a %s\n", st, it, res, eaf_status_string(st));
  return 0;
}
"""


@pytest.mark.parametrize("dims,seed", [((12, 24, 16), 0), ((35, 70, 50), 2)])
def test_c_program_matches_python_binding(tmp_path, dims, seed):
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    eaf = pkg()
    g = gen()
    libdir = os.path.dirname(eaf._lib.LIB_PATH)
    src = tmp_path / "caller.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "caller"
    subprocess.run(["gcc", "-std=c99", "-O2", "-I", os.path.join(ROOT, "include"), str(src),
                    "-L", libdir, "-leafcg", "-Wl,-rpath," + libdir, "-o", str(exe)],
                   check=True)
    s = g.make_system(*dims, seed=seed)
    phi0 = g.zeros_phi(*dims)
    for name, arr in zip(g.COEF_NAMES + ("phi",), s.arrays() + [phi0]):
        np.ascontiguousarray(arr, dtype=np.float64).tofile(tmp_path / f"{name}.bin")
    r = subprocess.run([str(exe), str(tmp_path), *map(str, dims), "200000", "1e-8"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stderr)
    st_c, it_c, res_hex, name = r.stdout.split()
    phi_c = np.fromfile(tmp_path / "phi_out.bin", dtype=np.float64).reshape(phi0.shape)
    phi_p = phi0.copy()
    with eaf.CGSolver(*dims) as cg:
        res_p, it_p, st_p = cg.solve(s.arrays(), phi_p, 200000, 1e-8)
    assert int(st_c) == st_p == 0 and name == "EAF_OK"
    assert int(it_c) == it_p and float.fromhex(res_hex) == res_p
    assert np.array_equal(phi_c, phi_p)
