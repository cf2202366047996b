"""The generated bicubic coefficient map (csrc/bicubic_gen.cuh) against the
reference's dense loop (bcucof_opt.c:55-61: xx += wt[i][k] * x[k], k = 0..15,
from xx = 0), bit for bit on random inputs, compiled on the host with no
contraction (CPU only)."""
from __future__ import annotations

import subprocess
import sys

import pytest

from conftest import ROOT

CSRC = ROOT / "dns-solvers-with-grid-embedding_b200" / "csrc"


def test_generated_map_is_the_dense_loop_bitwise(tmp_path):
    sys.path.insert(0, str(CSRC))
    import gen_bicubic

    W = gen_bicubic.weights()
    rows = ",\n".join("{" + ", ".join(f"{w}.0" for w in row) + "}" for row in W)
    src = f'''
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "{CSRC / "bicubic_gen.cuh"}"
static const double wt[16][16] = {{{rows}}};
int main(void) {{
  srand(7);
  long bad = 0;
  for (int it = 0; it < 400000; it++) {{
    double x[16], a[16], b[16];
    for (int k = 0; k < 16; k++) {{
      x[k] = ((double)rand() / RAND_MAX - 0.5) * pow(10.0, -(rand() % 12));
      if (rand() % 13 == 0) x[k] = 0.0;
    }}
    for (int i = 0; i < 16; i++) {{
      double xx = 0.;
      for (int k = 0; k < 16; k++) xx += wt[i][k] * x[k];
      a[i] = xx;
    }}
    DNS_BICUBIC_COEFFS(b, x);
    for (int i = 0; i < 16; i++)
      if (a[i] != b[i]) bad++;   /* values (a zero may differ in sign only) */
  }}
  printf("%ld\\n", bad);
  return 0;
}}
'''
    (tmp_path / "chk.c").write_text(src)
    exe = tmp_path / "chk"
    r = subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), str(tmp_path / "chk.c"), "-lm"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip(f"no host C compiler: {r.stderr[:200]}")
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.strip()
    assert out == "0"
