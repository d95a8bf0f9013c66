"""The boundary from plain C: a C11 program that includes include/rsx.h and links librsx.so, as a native caller of
the reference's host API would, built with gcc and run without a GPU.  It checks the layout queries, the synthetic
world and start states, a V3 arena dump round trip, and that asking for a device on a machine without one returns
RSX_E_NODEV with a message instead of crashing."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "rocketsim-cuda_b200")
CUDA_LIB = "/usr/local/cuda/lib64"

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "rsx.h"

int main(void) {
  if (rsx_arena_words() != 2784 || rsx_tick_words() != 2567 || rsx_static_words() != 317895) return 10;
  uint32_t* sd = calloc(rsx_static_words(), 4);
  uint32_t* st = calloc(2 * rsx_arena_words(), 4);
  uint32_t* back = calloc(rsx_arena_words(), 4);
  if (!sd || !st || !back) return 11;
  if (rsx_build_static(sd, 7, 2, 5) <= 0) return 12;  /* the triangle count */
  const float mix[5] = {0.2f, 0.5f, 0.15f, 0.1f, 0.05f};
  if (rsx_make_states(sd, st, 2, 3, mix) != RSX_OK) return 13;
  rsx_v3_template t;
  if (rsx_v3_template_init(sd, &t) != RSX_OK) return 14;
  size_t len = 0;
  if (rsx_v3_write_arena(st, sd, &t, NULL, 0, &len) != RSX_E_ARG || len < RSX_V3_ARENA_HEADER_LEN) return 15;
  uint8_t* buf = malloc(len);
  if (rsx_v3_write_arena(st, sd, &t, buf, len, &len) != RSX_OK) return 16;
  rsx_v3_template t2;
  if (rsx_v3_parse_arena(buf, len, sd, back, &t2) != RSX_OK) return 17;
  if (memcmp(back, st, rsx_tick_words() * 4) != 0) return 18;
  buf[0] ^= 1;  /* a broken magic is refused with the reference's message */
  if (rsx_v3_parse_arena(buf, len, sd, back, &t2) != RSX_E_FORMAT || strstr(rsx_last_error(), "magic") == NULL) return 19;
  rsx_device* dev = NULL;
  int rc = rsx_device_create(0, &dev);
  printf("device_create %d %s\n", rc, rc == RSX_OK ? "" : rsx_last_error());
  if (rc == RSX_OK) rsx_device_destroy(dev);
  else if (rc != RSX_E_NODEV) return 20;
  free(buf); free(back); free(st); free(sd);
  printf("ok\n");
  return 0;
}
"""


def test_c_program_links_and_runs(tmp_path, rsx):
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    src = tmp_path / "abi.c"
    exe = tmp_path / "abi"
    src.write_text(PROGRAM)
    cmd = ["gcc", "-std=c11", "-Wall", "-Werror", "-O1", str(src), "-I", os.path.join(ROOT, "include"), "-L", LIBDIR, "-lrsx",
           f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)]
    if os.path.isdir(CUDA_LIB):
        cmd[-2:-2] = ["-L", CUDA_LIB, f"-Wl,-rpath,{CUDA_LIB}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert out.stdout.strip().endswith("ok")
