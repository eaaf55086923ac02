// Host driver for exciting_b200/csrc/specfun.cuh, used by tests/test_specfun.py.
//   specfun_harness in.txt out.bin
// in.txt lines:  Y lmax theta phi        -> (lmax+1)^2 complex values
//                J m lmax x              -> lmax+1 values of d^m j_l(x)
//                P m np x x_0..x_np-1 y_0..y_np-1 -> one value
// Results are appended to out.bin as doubles in input order.
#include <cstdio>
#include <vector>

#include "specfun.cuh"

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  FILE* in = fopen(argv[1], "r");
  FILE* out = fopen(argv[2], "wb");
  if (!in || !out) return 3;
  char kind;
  while (fscanf(in, " %c", &kind) == 1) {
    if (kind == 'Y') {
      int lmax;
      double th, ph;
      if (fscanf(in, "%d %lf %lf", &lmax, &th, &ph) != 3) return 4;
      std::vector<cplx> y((lmax + 1) * (lmax + 1));
      sf_ylm(lmax, th, ph, y.data(), 1);
      fwrite(y.data(), sizeof(cplx), y.size(), out);
    } else if (kind == 'J') {
      int m, lmax;
      double x;
      if (fscanf(in, "%d %d %lf", &m, &lmax, &x) != 3) return 4;
      std::vector<double> d(lmax + 1);
      sf_sbessel_deriv(m, lmax, x, d.data());
      fwrite(d.data(), sizeof(double), d.size(), out);
    } else if (kind == 'P') {
      int m, np;
      double x;
      if (fscanf(in, "%d %d %lf", &m, &np, &x) != 3) return 4;
      std::vector<double> xa(np), ya(np);
      for (int i = 0; i < np; ++i) if (fscanf(in, "%lf", &xa[i]) != 1) return 4;
      for (int i = 0; i < np; ++i) if (fscanf(in, "%lf", &ya[i]) != 1) return 4;
      const double v = sf_polynom_deriv(m, np, xa.data(), ya.data(), x);
      fwrite(&v, sizeof(double), 1, out);
    } else {
      return 5;
    }
  }
  fclose(in);
  fclose(out);
  return 0;
}
