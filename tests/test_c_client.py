"""The C ABI from plain C (CPU): a C99 program that includes only
include/ngap_b200.h compiles with -pedantic -Werror, links
libngap_b200.so and runs its host-only entry points on the apple example
(README.md:156-186 of the reference: reports 0x400000005, 0x40000002f,
0x400000040, 0x40000004b)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")

C_SOURCE = r"""
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "ngap_b200.h"

static int fail(const char* what) {
  char msg[256];
  ngap_last_error(msg, sizeof(msg));
  fprintf(stderr, "%s: %s\n", what, msg);
  return 1;
}

int main(int argc, char** argv) {
  ngap_nfa* nfa = NULL;
  ngap_groups* groups = NULL;
  ngap_group_opts gopts;
  ngap_table_opts topts;
  ngap_tile_desc tile;
  FILE* f;
  uint8_t input[4096];
  uint64_t reports[64];
  uint32_t ids[64], reps[64];
  int64_t off[2], roff[2];
  size_t len;
  int64_t i, n;
  int ntiles = 0;
  if (argc != 3) return 2;
  if (ngap_nfa_load_anml(argv[1], &nfa) != NGAP_OK) return fail("load");
  gopts.group_num = 1;
  gopts.max_nfa_size = -1; /* no size limit */
  gopts.quit_degree = 1;
  gopts.remove_degree = 0;
  if (ngap_groups_build(nfa, &gopts, &groups) != NGAP_OK) return fail("groups");
  memset(&topts, 0, sizeof(topts));
  topts.precompute_depth = 2;
  topts.precompute_cutoff = -1;
  if (ngap_tiles_describe(groups, &topts, &tile, 1, &ntiles) != NGAP_OK) return fail("tiles");
  if (ngap_tiles_lookup(groups, &topts, 0, (const uint8_t*)"ap", 1, 2, ids, off, reps, roff, 64)
      != NGAP_OK)
    return fail("lookup");
  f = fopen(argv[2], "rb");
  if (!f) return 3;
  len = fread(input, 1, sizeof(input), f);
  fclose(f);
  n = ngap_cpu_validate_reference(groups, input, 1, (int64_t)len, 0, reports, 64, NULL);
  if (n < 0) return fail("validate");
  printf("states %lld edges %lld groups %d tiles %d depth %d lookup %lld\n",
         (long long)ngap_nfa_num_states(nfa), (long long)ngap_nfa_num_edges(nfa),
         ngap_groups_count(groups), ntiles, tile.depth, (long long)off[1]);
  for (i = 0; i < n; i++) printf("0x%llx\n", (unsigned long long)reports[i]);
  ngap_groups_destroy(groups);
  ngap_nfa_destroy(nfa);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_plain_c_client(built, tmp_path):
    src = tmp_path / "client.c"
    src.write_text(C_SOURCE)
    exe = tmp_path / "client"
    libdir = os.path.join(ROOT, "ngap_b200")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lngap_b200", "-Wl,-rpath," + libdir],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe), os.path.join(GOLD, "apple.anml"),
                        os.path.join(GOLD, "apple_input.txt")],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.split()
    head = r.stdout.splitlines()[0]
    assert head == "states 5 edges 4 groups 1 tiles 1 depth 2 lookup 1", head
    assert lines[-4:] == ["0x400000005", "0x40000002f", "0x400000040", "0x40000004b"]
