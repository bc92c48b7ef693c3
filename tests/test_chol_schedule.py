"""Host-side work list of the persistent dataflow Cholesky (engine.cuh: chol_schedule,
chol_schedule_valid), compiled on the CPU.

The factorisation kernel hands tile tasks out by ticket; its critical path (every POTRF(k),
TRSM(k, k+1) and the update of tile (k+1, k+1)) is one chain item, ticket 0, that waits on the
other items' trailing updates.  The schedule cannot deadlock when nothing that waits on a chain
step precedes what that step needs, which chol_schedule_valid checks by replaying the list.
Here: the lists built for every tile count up to 200 (m up to 12 800) pass, and (up to 12
tiles, every item in turn) lists with an item moved ahead of its inputs, a missing item or a
duplicated item are rejected.
"""
import pathlib
import shutil
import subprocess

import pytest

CSRC = pathlib.Path(__file__).resolve().parents[1] / "sdpx.rs_b200" / "csrc"

HARNESS = r"""
#include <cstdio>
#include <utility>
#include "engine.cuh"
using namespace sdpxg;
int main() {
  for (int nt = 1; nt <= 200; ++nt) {
    std::vector<unsigned> it = chol_schedule(nt);
    if (!chol_schedule_valid(it, nt)) { std::printf("rejected nt=%d\n", nt); return 1; }
    if (nt >= 2 && nt <= 12) {
      // every item moved to the front (before the chain's first step produced its inputs)
      for (size_t t = 1; t < it.size(); ++t) {
        std::vector<unsigned> bad = it;
        std::swap(bad[1], bad[t]);
        const unsigned c = it[t];
        const int type = (int)(c >> 30), k = (int)((c >> 20) & 1023u);
        if (k > 0 && chol_schedule_valid(bad, nt)) {  // inputs from step k-1 cannot exist yet
          std::printf("accepted early item nt=%d t=%zu\n", nt, t); return 1;
        }
        (void)type;
      }
      std::vector<unsigned> miss(it.begin(), it.end() - 1);
      if (chol_schedule_valid(miss, nt)) { std::printf("accepted missing item nt=%d\n", nt); return 1; }
      std::vector<unsigned> dup = it;
      dup.push_back(it.back());
      if (chol_schedule_valid(dup, nt)) { std::printf("accepted duplicate nt=%d\n", nt); return 1; }
    }
  }
  std::printf("ok\n");
  return 0;
}
"""


def test_dataflow_schedules_valid_and_checked(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not pathlib.Path(nvcc).exists():
        pytest.skip("nvcc not available")
    src = tmp_path / "sched.cu"
    src.write_text(HARNESS)
    exe = tmp_path / "sched"
    subprocess.run([nvcc, "-std=c++17", "-O1", f"-I{CSRC}", str(src), "-o", str(exe)], check=True,
                   capture_output=True, timeout=600)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
