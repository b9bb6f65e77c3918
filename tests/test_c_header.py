"""The boundary from C: include/hodlr_gpu.h compiles as plain C99 (the
language a cgo / JNI / FFI binding sees), a C program links the library,
and the host-only and argument-checking paths answer as documented.  Runs
without a GPU: compute entry points report HODLR_ERR_CUDA there."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "fastsolver_b200")

C_SOURCE = r"""
#include <stdio.h>
#include <stdlib.h>
#include "hodlr_gpu.h"

int main(int argc, char **argv) {
  int N = atoi(argv[1]), m = atoi(argv[2]), r = atoi(argv[3]), t = atoi(argv[4]);
  int cap = 4096;
  int *nodes = (int *)malloc(sizeof(int) * 10 * cap);
  int nn = hodlr_build_tree(N, m, r, t, nodes, cap);
  if (nn <= 0) return 2;
  for (int i = 0; i < nn * 10; ++i) printf("%d%c", nodes[i], (i % 10 == 9) ? '\n' : ' ');
  /* argument errors are reported before any device use */
  hodlr_system h = 0;
  fprintf(stderr, "create_null %d\n", hodlr_create(NULL, N, m, r, t));
  fprintf(stderr, "solve_null %d\n", hodlr_solve(NULL, NULL));
  fprintf(stderr, "status %s\n", hodlr_status_string(HODLR_ERR_NOCONV));
  hodlr_schedule s;
  fprintf(stderr, "sched_null %d\n", hodlr_get_schedule(NULL, &s));
  (void)h;
  free(nodes);
  return 0;
}
"""


@pytest.fixture(scope="module")
def c_program(tmp_path_factory, fs):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    d = tmp_path_factory.mktemp("cabi")
    src = d / "prog.c"
    src.write_text(C_SOURCE)
    exe = d / "prog"
    subprocess.check_call([cc, "-std=c99", "-Wall", "-Werror", "-pedantic",
                           "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                           "-L", LIBDIR, "-lhodlr_b200", f"-Wl,-rpath,{LIBDIR}"])
    return str(exe)


@pytest.mark.parametrize("N,m,r,t", [(480, 2, 30, 60), (3001, 5, 12, 200), (262144, 16, 64, 512)])
def test_c_program_builds_the_same_tree(fs, c_program, N, m, r, t):
    out = subprocess.run([c_program, str(N), str(m), str(r), str(t)], capture_output=True,
                         text=True, check=True)
    rows = np.array([[int(v) for v in line.split()] for line in out.stdout.splitlines()])
    np.testing.assert_array_equal(rows, fs.build_tree(N, m, r, t))
    err = dict(line.split(" ", 1) for line in out.stderr.splitlines())
    assert int(err["create_null"]) == -1
    assert int(err["solve_null"]) == -1
    assert int(err["sched_null"]) == -1
    assert err["status"] == "refinement did not reach the tolerance"
