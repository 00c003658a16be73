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


PRICING_HOST = r"""
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "LocVolCalib.h"

/* The nine scalars of a LocVolCalib dataset (.in) file: Futhark text
   values, "--" comments to the end of the line, an optional type suffix. */
static int read_inputs(const char *path, double v[9]) {
  FILE *f = fopen(path, "r");
  if (!f) return -1;
  char line[512];
  int n = 0;
  while (n < 9 && fgets(line, sizeof line, f)) {
    char *c = strstr(line, "--");
    if (c) *c = 0;
    char *p = line;
    while (n < 9) {
      char *end;
      double x = strtod(p, &end);
      if (end == p) break;
      v[n++] = x;
      p = end;
      while (*p && *p != ' ' && *p != '\t' && *p != '\n') p++;  /* type suffix */
    }
  }
  fclose(f);
  return n == 9 ? 0 : -2;
}

int main(int argc, char **argv) {
  double v[9];
  if (argc < 2 || read_inputs(argv[1], v)) return 1;
  struct futhark_context_config *cfg = futhark_context_config_new();
  struct futhark_context *ctx = futhark_context_new(cfg);
  char *err = futhark_context_get_error(ctx);
  if (err) { fprintf(stderr, "%s\n", err); free(err); return 2; }
  struct futhark_f32_1d *out = NULL;
  if (futhark_entry_main(ctx, &out, (int32_t)v[0], (int32_t)v[1], (int32_t)v[2], (int32_t)v[3],
                         (float)v[4], (float)v[5], (float)v[6], (float)v[7], (float)v[8])) {
    err = futhark_context_get_error(ctx);
    fprintf(stderr, "%s\n", err ? err : "?");
    free(err);
    return 3;
  }
  const int64_t *shape = futhark_shape_f32_1d(ctx, out);
  int64_t n = shape[0];
  float *prices = malloc(sizeof(float) * (n > 0 ? n : 1));
  if (futhark_values_f32_1d(ctx, out, prices) || futhark_context_sync(ctx)) return 4;
  for (int64_t i = 0; i < n; i++) printf("%.9g\n", prices[i]);
  free(prices);
  futhark_free_f32_1d(ctx, out);
  futhark_context_free(ctx);
  futhark_context_config_free(cfg);
  return 0;
}
"""


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small", "medium"])
def test_c_host_prices_reference_dataset_on_gpu(tmp_path, name):
    """A C host prices a reference dataset through futhark_entry_main and
    futhark_values_f32_1d on the GPU; its prices match the dataset's .out file
    (finpar/LocVolCalib-data) within 5e-6 absolute."""
    import gzip

    import numpy as np

    from conftest import read_dataset, DATASETS
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "price.c"
    src.write_text(PRICING_HOST)
    exe = tmp_path / "price"
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"), str(src), "-o",
                    str(exe), "-L", PKG, "-l:liblvc.so", f"-Wl,-rpath,{PKG}"], check=True)
    data = tmp_path / f"{name}.in"
    with gzip.open(os.path.join(DATASETS, "finpar", "LocVolCalib-data", f"{name}.in.gz")) as f:
        data.write_bytes(f.read())
    run = subprocess.run([str(exe), str(data)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, (run.stdout, run.stderr)
    got = np.array([float(x) for x in run.stdout.split()])
    (want,) = read_dataset(f"finpar/LocVolCalib-data/{name}.out")
    assert got.shape == want.shape
    assert np.max(np.abs(got - want.astype(np.float64))) <= 5e-6
