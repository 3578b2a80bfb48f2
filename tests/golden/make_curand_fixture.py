"""Record raw words of cuRAND's Philox4_32_10 generator -- the generator of
the reference's predict/resampling kernels (src/particle_filter/predict.cu:14-20,
resampling.cu:183-205) -- so the project's own Philox can be pinned to it.

Needs a GPU and nvcc: python tests/golden/make_curand_fixture.py
Writes tests/golden/curand_philox.json.
"""
from __future__ import annotations

import json
import subprocess
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent

SRC = r"""
#include <cstdio>
#include <curand_kernel.h>
__global__ void draw(unsigned long long seed, unsigned long long subseq, unsigned* out, int n4) {
  curandStatePhilox4_32_10_t st;
  curand_init(seed, subseq, 0, &st);
  for (int i = 0; i < n4; ++i) {
    uint4 v = curand4(&st);
    out[4 * i] = v.x; out[4 * i + 1] = v.y; out[4 * i + 2] = v.z; out[4 * i + 3] = v.w;
  }
}
int main() {
  const unsigned long long seeds[3] = {42ull, 12345ull, 0x123456789abcdefull};
  const unsigned long long subs[3] = {0ull, 7ull, 1000003ull};
  unsigned *d, h[16];
  cudaMalloc(&d, sizeof(h));
  printf("[");
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      draw<<<1, 1>>>(seeds[a], subs[b], d, 4);
      cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
      printf("%s{\"seed\": %llu, \"subsequence\": %llu, \"words\": [", (a || b) ? ", " : "", seeds[a], subs[b]);
      for (int i = 0; i < 16; ++i) printf("%s%u", i ? ", " : "", h[i]);
      printf("]}");
    }
  printf("]\n");
  cudaFree(d);
  return cudaGetLastError() != cudaSuccess;
}
"""


def main():
    with tempfile.TemporaryDirectory() as td:
        cu = Path(td) / "curand_words.cu"
        exe = Path(td) / "curand_words"
        cu.write_text(SRC)
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", str(cu), "-o", str(exe)],
                       check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    recs = json.loads(out)
    (HERE / "curand_philox.json").write_text(json.dumps({
        "source": "cuRAND curandStatePhilox4_32_10_t, curand_init(seed, subsequence, 0) then curand4() x4",
        "records": recs}, indent=1))
    print("wrote", HERE / "curand_philox.json")


if __name__ == "__main__":
    main()
