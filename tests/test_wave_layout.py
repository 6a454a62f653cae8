"""Host-side layout checks (no device).  The wave-synchronous inversion state:
the buffer that gm::wave_buffers carves for a chunk -- LM records, staging
blocks, wave counters, three pixel lists -- must hold every region inside
gm::wave_buffer_bytes, disjoint and aligned, for every grid size and
iteration limit.  A small host program is compiled against the engine's
headers and linked to the engine library; it only does pointer arithmetic
on a made-up base address.  The normal equations' compile-time entry
table: alpha's packed upper triangle, then beta, each operand pair once,
with the stray-light factor of each entry."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "g-milos_b200")
LIB = os.path.join(PKG, "gmilos_b200", "libgmilos.so")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"

PROGRAM = r"""
#include <cstdio>
#include <cstdint>
#include "gm_kernels.cuh"

static int bad = 0;
static void expect(bool ok, const char* what, int nl, int miter, long chunk) {
  if (!ok) { std::printf("FAIL %s nl=%d miter=%d chunk=%ld\n", what, nl, miter, chunk); ++bad; }
}

int main() {
  static_assert(sizeof(gm::PixLM) == 576, "record size");
  static_assert(sizeof(gm::PixLM) % 16 == 0, "records keep 16-byte alignment");
  static_assert(gm::stage_floats_for(1) == 28 * 32 && gm::stage_floats_for(2) == 55 * 32, "staging rows");
  const int nls[] = {1, 12, 30, 32, 33, 45, 64};
  const int miters[] = {0, 1, 50, 200};
  const long chunks[] = {1, 3, 1000, 16384, 1 << 20};
  char* base = reinterpret_cast<char*>(uintptr_t(1) << 32);
  for (int nl : nls)
    for (int miter : miters)
      for (long chunk : chunks) {
        const size_t total = gm::wave_buffer_bytes(nl, miter, chunk);
        const gm::WaveBuffers b = gm::wave_buffers(base, nl, miter, chunk);
        const int lpl = nl <= 32 ? 1 : 2;
        const int waves = 1 + (miter > 1 ? miter : 1);
        struct R { const char* name; const char* lo; size_t bytes; size_t align; } r[] = {
            {"state", reinterpret_cast<const char*>(b.w.state), sizeof(gm::PixLM) * (size_t)chunk, 16},
            {"stage", reinterpret_cast<const char*>(b.w.stage), sizeof(float) * gm::stage_floats_for(lpl) * (size_t)chunk, 16},
            {"cnt", reinterpret_cast<const char*>(b.w.cnt), sizeof(gm::WaveCounters) * (size_t)waves, 16},
            {"act0", reinterpret_cast<const char*>(b.w.act0), sizeof(uint32_t) * (size_t)chunk, 4},
            {"act1", reinterpret_cast<const char*>(b.w.act1), sizeof(uint32_t) * (size_t)chunk, 4},
            {"accl", reinterpret_cast<const char*>(b.w.accl), sizeof(uint32_t) * (size_t)chunk, 4}};
        expect(b.chunk == chunk, "chunk", nl, miter, chunk);
        for (const R& x : r) {
          expect(x.lo >= base && x.lo + x.bytes <= base + total, x.name, nl, miter, chunk);
          expect(((uintptr_t)x.lo % x.align) == 0, x.name, nl, miter, chunk);
        }
        for (const R& x : r)
          for (const R& y : r)
            if (&x < &y) expect(x.lo + x.bytes <= y.lo || y.lo + y.bytes <= x.lo, "overlap", nl, miter, chunk);
      }
  std::printf(bad ? "FAILED %d\n" : "OK\n", bad);
  return bad ? 1 : 0;
}
"""


@pytest.mark.skipif(not os.path.exists(LIB), reason="engine library not built")
def test_wave_buffers_fit_and_do_not_overlap(tmp_path):
    src = tmp_path / "layout.cu"
    exe = tmp_path / "layout"
    src.write_text(PROGRAM)
    cmd = [NVCC, "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "csrc"), str(src),
           "-o", str(exe), "-L", os.path.dirname(LIB), "-lgmilos", "-Xlinker", "-rpath=" + os.path.dirname(LIB)]
    build = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert build.returncode == 0, build.stderr[-2000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0 and run.stdout.strip().endswith("OK"), run.stdout[-2000:] + run.stderr[-500:]


NE_PROGRAM = r"""
#include <cstdio>
#include "gm_device.cuh"

// The normal equations' entry table (host-evaluated constexpr functions):
// alpha's packed upper triangle in upk order, then beta, every operand pair
// once; the stray-light factor bits count the scaled rows of each entry.
template <int NT>
int check() {
  int bad = 0;
  constexpr int NE = gm::ne_entries<NT>(), NA = NT * (NT + 1) / 2;
  static_assert(NE == NA + NT, "entries");
  int seen[16][16] = {};
  for (int e = 0; e < NE; ++e) {
    const int ab = gm::ne_entry<NT>(e), a = ab >> 4, b = ab & 15;
    if (!(a >= 0 && a < NT && b >= a && b <= NT)) { std::printf("FAIL range NT=%d e=%d\n", NT, e); ++bad; continue; }
    if (e < NA && (b == NT || gm::upk<NT>(a, b) != e)) { std::printf("FAIL alpha NT=%d e=%d\n", NT, e); ++bad; }
    if (e >= NA && (b != NT || a != e - NA)) { std::printf("FAIL beta NT=%d e=%d\n", NT, e); ++bad; }
    if (seen[a][b]++) { std::printf("FAIL twice NT=%d e=%d\n", NT, e); ++bad; }
    const int f = (int)((gm::ne_alfa_bits<NT>(e / 32) >> (2 * (e % 32))) & 3u);
    if (f != (a < NT - 1) + (b < NT - 1)) { std::printf("FAIL alfa NT=%d e=%d\n", NT, e); ++bad; }
  }
  return bad;
}

int main() {
  const int bad = check<10>() + check<11>();
  std::printf(bad ? "FAILED %d\n" : "OK\n", bad);
  return bad ? 1 : 0;
}
"""


def test_normal_equation_entry_table(tmp_path):
    src = tmp_path / "ne.cu"
    exe = tmp_path / "ne"
    src.write_text(NE_PROGRAM)
    cmd = [NVCC, "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "csrc"), str(src),
           "-o", str(exe)]
    build = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert build.returncode == 0, build.stderr[-2000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0 and run.stdout.strip().endswith("OK"), run.stdout[-2000:] + run.stderr[-500:]
