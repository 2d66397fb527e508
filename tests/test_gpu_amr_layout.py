"""The state boundary in the reference driver's own array layout
(300riemann_module_3d.f:495-530): a C program, compiled here against
include/cubesphere_b200.h and linked to the library, fills Fortran-order
module arrays U_amr(1-G:N+G, 1-G:N+G, 1-G:nr+G, ncomp, 6),
entropygr_amr(1-G:N+G, 1-G:N+G, 1-G:nr+G, 6) and Bxf/Byf/Bzf_amr(0-G:N+G,
0-G:N+G, 0-G:nr+G, 6) from the library's panel-box state, hands them to
cs_state_put_amr unchanged, steps, and reads them back with
cs_state_get_amr; every value must agree with the panel-box path and the
extra species component must come back untouched."""
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT, has_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]

PROGRAM = r"""
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "cubesphere_b200.h"

/* Fortran column-major offsets with the reference's lower bounds */
#define ZO(i, j, k, c, p) ((((long)(p) * NC + (c)) * NKZ + ((k) + G - 1)) * NJZ * NIZ + (long)((j) + G - 1) * NIZ + ((i) + G - 1))
#define EO(i, j, k, p) ((((long)(p)) * NKZ + ((k) + G - 1)) * NJZ * NIZ + (long)((j) + G - 1) * NIZ + ((i) + G - 1))
#define FO(i, j, k, p) ((((long)(p)) * NK + ((k) + G)) * NJ * NI + (long)((j) + G) * NI + ((i) + G))
#define BO(c, p, i, j, k) ((((long)(c) * 6 + (p)) * NK + ((k) + G)) * NJ * NI + (long)((j) + G) * NI + ((i) + G))

static int N = 16, NR = 8, G = 4, NC = 9;
static long NI, NJ, NK, NIZ, NJZ, NKZ;

static int fail(const char* what, cs_ctx* c) {
  fprintf(stderr, "%s: %s\n", what, c ? cs_last_error(c) : "");
  return 1;
}

int main(void) {
  cs_params p;
  memset(&p, 0, sizeof p);
  p.ntp = N; p.nr = NR; p.nghost = G; p.radial_mesh = CS_RADIAL_STRETCHED; p.rmin = 1.0; p.rmax = 2.0;
  p.radial_ratio = 1.02; p.gamma = 5.0 / 3.0; p.rhofloor = 1e-12; p.prsfloor = 1e-9; p.smallnum = 1e-12;
  p.cfl_coef = 0.4; p.flatten_coef = 0.4; p.prs_flatten_coef = 1.5; p.gm = 1.0; p.bc_lower = 2; p.bc_upper = 2;
  p.rk_scheme = CS_IMEX_RK2; p.flags = 0;
  cs_ctx *a = NULL, *b = NULL;
  if (cs_create(&p, &a) || cs_create(&p, &b)) return fail("cs_create", a);
  if (cs_mesh_build(a) || cs_mesh_build(b)) return fail("cs_mesh_build", a);
  cs_init_desc d = {2025, 1, 4, 0.05, 0.05, 0.0, 0.05};
  if (cs_init_problem(a, &d)) return fail("cs_init_problem", a);
  NI = NJ = N + 2 * G + 1; NK = NR + 2 * G + 1; NIZ = NJZ = N + 2 * G; NKZ = NR + 2 * G;
  long S6 = 6 * NI * NJ * NK, Z = NIZ * NJZ * NKZ;
  double *U = malloc(8 * S6 * sizeof(double)), *ent = malloc(S6 * sizeof(double));
  double *bx = malloc(S6 * sizeof(double)), *by = malloc(S6 * sizeof(double)), *bz = malloc(S6 * sizeof(double));
  double *Ua = malloc(NC * 6 * Z * sizeof(double)), *ea = malloc(6 * Z * sizeof(double));
  double *bxa = malloc(S6 * sizeof(double)), *bya = malloc(S6 * sizeof(double)), *bza = malloc(S6 * sizeof(double));
  if (cs_state_get(a, U, ent, bx, by, bz)) return fail("cs_state_get", a);
  /* the driver's arrays, filled element by element in Fortran order */
  for (int q = 0; q < 6; ++q)
    for (int k = 1 - G; k <= NR + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) {
          for (int c = 0; c < 8; ++c) Ua[ZO(i, j, k, c, q)] = U[BO(c, q, i, j, k)];
          Ua[ZO(i, j, k, 8, q)] = 7.0;  /* a passive species the library ignores */
          ea[EO(i, j, k, q)] = ent[BO(0, q, i, j, k)];
        }
  for (int q = 0; q < 6; ++q)
    for (int k = -G; k <= NR + G; ++k)
      for (int j = -G; j <= N + G; ++j)
        for (int i = -G; i <= N + G; ++i) {
          bxa[FO(i, j, k, q)] = bx[BO(0, q, i, j, k)];
          bya[FO(i, j, k, q)] = by[BO(0, q, i, j, k)];
          bza[FO(i, j, k, q)] = bz[BO(0, q, i, j, k)];
        }
  if (cs_state_put_amr(b, NC, Ua, ea, bxa, bya, bza)) return fail("cs_state_put_amr", b);
  double dta = 0, dtb = 0;
  if (cs_evaluate_timestep(a, 1e30, &dta) || cs_evaluate_timestep(b, 1e30, &dtb)) return fail("cfl", a);
  if (dta != dtb) { fprintf(stderr, "dt %g %g\n", dta, dtb); return 1; }
  if (cs_step(a, dta, &dta) || cs_step(b, dtb, &dtb)) return fail("cs_step", a);
  if (dta != dtb) { fprintf(stderr, "dt after step %g %g\n", dta, dtb); return 1; }
  if (cs_state_get(a, U, ent, bx, by, bz)) return fail("cs_state_get", a);
  if (cs_state_get_amr(b, NC, Ua, ea, bxa, bya, bza)) return fail("cs_state_get_amr", b);
  long bad = 0;
  for (int q = 0; q < 6; ++q)
    for (int k = 1 - G; k <= NR + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) {
          for (int c = 0; c < 8; ++c) bad += Ua[ZO(i, j, k, c, q)] != U[BO(c, q, i, j, k)];
          bad += Ua[ZO(i, j, k, 8, q)] != 7.0;
          bad += ea[EO(i, j, k, q)] != ent[BO(0, q, i, j, k)];
        }
  for (int q = 0; q < 6; ++q)
    for (int k = -G; k <= NR + G; ++k)
      for (int j = -G; j <= N + G; ++j)
        for (int i = -G; i <= N + G; ++i)
          bad += bxa[FO(i, j, k, q)] != bx[BO(0, q, i, j, k)] || bya[FO(i, j, k, q)] != by[BO(0, q, i, j, k)] ||
                 bza[FO(i, j, k, q)] != bz[BO(0, q, i, j, k)];
  if (bad) { fprintf(stderr, "%ld values differ\n", bad); return 1; }
  if (cs_state_put_amr(b, 7, Ua, ea, bxa, bya, bza) != CS_ERR_ARG) return fail("ncomp check", b);
  printf("ok\n");
  cs_destroy(a);
  cs_destroy(b);
  return 0;
}
"""


def test_driver_arrays_pass_through_the_c_abi_unchanged(tmp_path):
    src = tmp_path / "amr.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "amr"
    lib = ROOT / "cubesphere_b200"
    r = subprocess.run(["gcc", "-O1", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe),
                        "-L", str(lib), "-lcubesphere_b200", f"-Wl,-rpath,{lib}", "-lm"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
