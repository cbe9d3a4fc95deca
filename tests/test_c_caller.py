"""A plain C99 caller compiled against each public header and linked against
its library, as a code that used the reference's C API would be: the headers
compile on their own (-std=c99 -Wall -Werror), every declared name links, and
the argument checks and workspace queries answer without a GPU."""
import os
import shutil
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "bsofi_b200")

CALLER = textwrap.dedent("""
    #include <stdio.h>
    #include "%(header)s"
    int main(void) {
      %(real)s A[64] = {0}, tau[8] = {0}, w[1] = {0};
      int info = 0, h[10] = {0}, n = 0, L = 4, lda = 0;
      double t0[2], t1[2];
      /* illegal sizes are rejected before any device call */
      lapackXbsof(0, 2, A, 8, tau, w, 1, &info);
      if (info != -1) return 1;
      lapackXbsof(4, 2, A, 8, tau, w, -1, &info);   /* workspace query */
      if (info != 0 || w[0] < 1) return 2;
      if (hybridxinith_(h, &n, &L, &lda) != -1) return 3;
      if (lapackXbsofiLWork(4, 2, 8) < 1) return 4;
      fgetwalltime_(t0);
      fgetwalltime_(t1);
      if (felapsed_(t1, t0) < 0.0) return 5;
      /* every declared function links */
      void *fns[] = {%(fns)s};
      for (unsigned i = 0; i < sizeof(fns) / sizeof(fns[0]); i++)
        if (!fns[i]) return 6;
      printf("ok\\n");
      return 0;
    }
""")


@pytest.mark.parametrize("which", ["fp64", "fp32"])
def test_c_caller_compiles_links_and_runs(tmp_path, which):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    sys.path.insert(0, ROOT)
    from bsofi_b200 import _lib, fp32
    if which == "fp64":
        header, lib, real, names = "bsofi_b200.h", "bsofi_b200", "double", _lib.declared_symbols()
    else:
        header, lib, real, names = "bsofi_b200_fp32.h", "bsofi_b200_fp32", "float", fp32.declared()
    src = tmp_path / "caller.c"
    src.write_text(CALLER % {"header": header, "real": real,
                             "fns": ", ".join("(void *)%s" % f for f in names)})
    exe = tmp_path / "caller"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-Wno-pedantic",
                    "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", PKG, "-l" + lib, "-Wl,-rpath," + PKG], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stderr)
    assert out.stdout.strip() == "ok"
