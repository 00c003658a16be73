"""A C host written against each library's public header compiles with gcc,
links against the library and runs: configuration, context creation (which on
a machine without a usable GPU returns a context carrying an error message)
and teardown.  This is the link surface a Futhark-generated library's host
uses."""
import os
import shutil
import subprocess

import pytest

from conftest import REPO

PKG = os.path.join(REPO, "futhark-benchmarks_b200")

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "%(header)s"

int main(void) {
  struct futhark_context_config *cfg = futhark_context_config_new();
  if (!cfg) return 1;
  futhark_context_config_set_device(cfg, "#0");
  struct futhark_context *ctx = futhark_context_new(cfg);
  futhark_context_config_free(cfg);
  if (!ctx) return 2;
  char *err = futhark_context_get_error(ctx);
  int rc = 0;
  if (err) {            /* no usable GPU: the calls after this must fail cleanly */
    %(failing_call)s
    free(err);
    err = futhark_context_get_error(ctx);
    if (!err) rc = 4;   /* the failure left a message */
    free(err);
  } else {              /* a usable GPU: a tiny entry-point call */
    %(working_call)s
  }
  futhark_context_free(ctx);
  printf("ok %%d\n", rc);
  return rc;
}
"""

CASES = {
    "liblvc.so": dict(
        header="LocVolCalib.h",
        failing_call="if (futhark_context_sync(ctx) == 0) rc = 3;",
        working_call="struct futhark_f32_1d *out = NULL;"
                     " if (futhark_entry_main(ctx, &out, 2, 8, 8, 4, 0.03f, 5.0f, 0.2f, 0.6f, 0.5f)) rc = 5;"
                     " else futhark_free_f32_1d(ctx, out);"),
    "libtke.so": dict(
        header="tke.h",
        failing_call="if (futhark_new_f32_1d(ctx, NULL, 4) != NULL) rc = 3;",
        working_call="struct futhark_f32_1d *a = futhark_new_f32_1d(ctx, NULL, 4);"
                     " if (!a) rc = 5; else futhark_free_f32_1d(ctx, a);"),
    "libop.so": dict(
        header="op.h",
        failing_call="if (futhark_new_f32_1d(ctx, NULL, 4) != NULL) rc = 3;",
        working_call="struct futhark_f32_1d *a = futhark_new_f32_1d(ctx, NULL, 4);"
                     " if (!a) rc = 5; else futhark_free_f32_1d(ctx, a);"),
}


@pytest.mark.parametrize("lib", sorted(CASES))
def test_c_host_compiles_links_and_runs(tmp_path, lib):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    case = CASES[lib]
    src = tmp_path / "host.c"
    src.write_text(PROGRAM % case)
    exe = tmp_path / "host"
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"), str(src), "-o",
                    str(exe), "-L", PKG, f"-l:{lib}", f"-Wl,-rpath,{PKG}"], check=True)
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, (run.stdout, run.stderr)
    assert run.stdout.strip() == "ok 0"
