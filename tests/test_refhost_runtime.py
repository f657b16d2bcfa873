"""The CUDA-thread emulator under the host build of the reference
(oracle/refhost): barrier semantics and the launch rewrite, on the CPU.

A small program is compiled with rh_cuda_shim.h and rh_fiber.cpp:
  * a 1024-thread tree reduction through __shared__ memory with a barrier
    per level (the reference's bin_reduc pattern), over a multi-block grid;
  * threads of a block that return before others reach their barriers (the
    reference's last chunks leave whole warps out of the barrier-laden
    branch; exited threads no longer hold a barrier back);
  * each block's __shared__ data private to the block while blocks run on
    several OS threads.
It must print the sums a sequential loop gives."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RH = os.path.join(ROOT, "oracle", "refhost")
sys.path.insert(0, RH)
from launch_rewrite import rewrite  # noqa: E402

PROG = r"""
#include <cstdio>
__global__ void tree(const double *in, double *out, int n) {
  __shared__ double s[1024];
  int t = threadIdx.x, b = blockIdx.x + gridDim.x * blockIdx.y;
  s[t] = (t < n) ? in[b * n + t] : 0.0;
  __syncthreads();
  for (int h = 512; h > 0; h >>= 1) {
    if (t < h) s[t] += s[t + h];
    __syncthreads();
  }
  if (t == 0) out[b] = s[0];
}
__global__ void early(double *out, int live) {
  __shared__ double s[128];
  int t = threadIdx.x;
  if (t >= live) return;            // these threads never reach a barrier
  s[t] = t + 1.0 + blockIdx.x;
  __syncthreads();
  double v = 0.0;
  for (int k = 0; k < live; k++) v += s[k];
  __syncthreads();
  s[t] = v;
  __syncthreads();
  if (t == 0) out[blockIdx.x] = s[live - 1];
}
int main() {
  const int nb = 12, n = 1000;
  double *in = new double[nb * n], *out = new double[nb], *out2 = new double[nb];
  for (int i = 0; i < nb * n; i++) in[i] = (i % 97) * 0.5 + 1.0 / (1 + i % 13);
  tree<<<dim3(4, 3, 1), 1024, 0, 0>>>(in, out, n);
  early<<<nb, 128>>>(out2, 96);
  for (int b = 0; b < nb; b++) {
    double ref = 0.0, ref2 = 0.0;
    for (int i = 0; i < n; i++) ref += in[b * n + i];
    for (int k = 0; k < 96; k++) ref2 += k + 1.0 + b;
    std::printf("%d %.17g %.17g %.17g %.17g\n", b, out[b], ref, out2[b], ref2);
  }
  return 0;
}
"""


def test_launch_rewrite():
    src = "  k<<< set[n].g , 128 , 0 , set[n].s >>>\n     (a, f(b, c), d);\n  q<<<1, 2>>>(x);"
    out, n = rewrite(src)
    assert n == 2
    assert "RH_LAUNCH(dim3(set[n].g), dim3(128), [&] { k(a, f(b, c), d); })" in out
    assert "RH_LAUNCH(dim3(1), dim3(2), [&] { q(x); })" in out
    assert "<<<" not in out


def test_fiber_barriers_and_shared_memory(tmp_path):
    cu = tmp_path / "prog.cu"
    cu.write_text(PROG)
    cpp = tmp_path / "prog.cpp"
    txt, n = rewrite(PROG)
    assert n == 2
    cpp.write_text(txt)
    exe = tmp_path / "prog"
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-include", os.path.join(RH, "rh_cuda_shim.h"),
                        f"-I{RH}", "-o", str(exe), str(cpp), os.path.join(RH, "rh_fiber.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=dict(os.environ, OMP_NUM_THREADS="4"),
                       timeout=120)
    assert r.returncode == 0, r.stderr
    rows = [ln.split() for ln in r.stdout.strip().splitlines()]
    assert len(rows) == 12
    for b, got, ref, got2, ref2 in rows:
        assert abs(float(got) - float(ref)) <= 1e-9 * abs(float(ref)), (b, got, ref)
        assert float(got2) == float(ref2), (b, got2, ref2)
