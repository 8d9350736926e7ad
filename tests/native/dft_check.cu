// Host check of the register DFTs in lf_fft.cuh (dft2 .. dft32, forward and
// inverse, float and double) against a direct float64 DFT.  Prints one line
// per case: "R inv type max_rel_err"; exit status 1 if any error exceeds the
// bound given on the command line for its type.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../../cmblensing_b200/csrc/lf_fft.cuh"

using namespace lf;

template <int R, typename T, bool INV>
double check(std::mt19937_64& rng) {
  std::normal_distribution<double> nd;
  double worst = 0.0;
  for (int trial = 0; trial < 200; ++trial) {
    double xr[R], xi[R];
    c2<T> a[R];
    for (int j = 0; j < R; ++j) {
      xr[j] = nd(rng);
      xi[j] = nd(rng);
      a[j] = mk<T>(T(xr[j]), T(xi[j]));
      xr[j] = double(a[j].x);  // the rounded inputs are the reference's inputs
      xi[j] = double(a[j].y);
    }
    dft<R, T, INV>(a);
    double num = 0.0, den = 0.0;
    for (int k = 0; k < R; ++k) {
      double sr = 0.0, si = 0.0;
      for (int j = 0; j < R; ++j) {
        const double ang = (INV ? 2.0 : -2.0) * M_PI * double((j * k) % R) / double(R);
        sr += xr[j] * std::cos(ang) - xi[j] * std::sin(ang);
        si += xr[j] * std::sin(ang) + xi[j] * std::cos(ang);
      }
      num += (double(a[k].x) - sr) * (double(a[k].x) - sr) + (double(a[k].y) - si) * (double(a[k].y) - si);
      den += sr * sr + si * si;
    }
    worst = std::fmax(worst, std::sqrt(num / den));
  }
  return worst;
}

template <int R>
bool run(std::mt19937_64& rng, double tol32, double tol64) {
  bool ok = true;
  const double e[4] = {check<R, float, false>(rng), check<R, float, true>(rng), check<R, double, false>(rng),
                       check<R, double, true>(rng)};
  const char* names[4] = {"fwd f32", "inv f32", "fwd f64", "inv f64"};
  for (int i = 0; i < 4; ++i) {
    const double tol = i < 2 ? tol32 : tol64;
    std::printf("%d %s %.3e\n", R, names[i], e[i]);
    ok = ok && e[i] < tol;
  }
  return ok;
}

int main(int argc, char** argv) {
  const double tol32 = argc > 1 ? std::atof(argv[1]) : 1e-6;
  const double tol64 = argc > 2 ? std::atof(argv[2]) : 1e-14;
  std::mt19937_64 rng(12345);
  bool ok = run<2>(rng, tol32, tol64);
  ok = run<4>(rng, tol32, tol64) && ok;
  ok = run<8>(rng, tol32, tol64) && ok;
  ok = run<16>(rng, tol32, tol64) && ok;
  ok = run<32>(rng, tol32, tol64) && ok;
  return ok ? 0 : 1;
}
