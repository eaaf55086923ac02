// Host driver for chase.cuh, used by tests/test_two_stage.py: reads a band
// matrix in compact lower storage, runs the chase sweep by sweep on the host
// and writes the result and the reflectors.
//   chase_harness n b band.bin out.bin refl.bin
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "chase.cuh"

int main(int argc, char** argv) {
  if (argc != 6) return 2;
  const int n = atoi(argv[1]), b = atoi(argv[2]);
  const size_t ld = 2 * (size_t)b + 1;
  std::vector<cplx> ab(ld * n);
  FILE* f = fopen(argv[3], "rb");
  if (!f || fread(ab.data(), sizeof(cplx), ab.size(), f) != ab.size()) return 3;
  fclose(f);
  BandView B{ab.data(), n, b};
  std::vector<cplx> v(b), work(2 * b), refl;
  for (int i = 0; i < n - 2; ++i) {
    int col = i, lo = i + 1;
    while (lo < n - 1) {
      const int hi = (lo + b < n) ? lo + b : n;
      if (hi - lo < 2) break;
      cplx tau;
      chase_task(B, col, lo, hi, v.data(), &tau, work.data());
      // record: (i, lo, len) as doubles, tau, v[0..len)
      refl.push_back(cmk(i, lo));
      refl.push_back(cmk(hi - lo, 0.0));
      refl.push_back(tau);
      for (int t = 0; t < hi - lo; ++t) refl.push_back(v[t]);
      col = lo;
      lo += b;
    }
  }
  f = fopen(argv[4], "wb");
  fwrite(ab.data(), sizeof(cplx), ab.size(), f);
  fclose(f);
  f = fopen(argv[5], "wb");
  fwrite(refl.data(), sizeof(cplx), refl.size(), f);
  fclose(f);
  return 0;
}
