// Seeded synthetic workload fields shared by every consumer of the solver:
// the benchmark, the tests and the CPU oracle all evaluate the right-hand side
// and the coefficients through this one definition, so a hierarchy built from
// the same seed is bit-identical everywhere (same std::exp, same operation
// order, host double precision).
//
//   rhs(x)  = sum_{i<16} A_i * exp(-|x - c_i|^2 / (2 w_i^2))
//             c_i ~ U[0.2,0.8]^3, w_i ~ U[0.02,0.1], A_i = +-U[0.5,2] (sign p=1/2)
//   coef(x) = exp(ln(10) * g(x)),  g = sum_{m<8} c_m cos(2 pi k_m.x + phi_m) / sum|c_m|
//             k_m in {-4..4}^3 \ {0}, c_m ~ U[-1,1], phi_m ~ U[0,2 pi)
//   coef lies in [0.1, 10].  a(x) uses the first mode set (cell centres), b(x)
//   the second (face centres).
//
// Random stream: std::mt19937_64(seed); u = (draw >> 11) * 2^-53; draw order
// bumps, then a-modes, then b-modes.
#ifndef CMG_SYNTHETIC_H
#define CMG_SYNTHETIC_H

#include <cmath>
#include <cstdint>
#include <random>

namespace cmg_synth {

struct Stream {
  std::mt19937_64 g;
  explicit Stream(uint64_t seed) : g(seed) {}
  double u() { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Bumps {
  double cx[16], cy[16], cz[16], w2x2[16], amp[16];
  void draw(Stream& s) {
    for (int i = 0; i < 16; ++i) {
      cx[i] = 0.2 + 0.6 * s.u();
      cy[i] = 0.2 + 0.6 * s.u();
      cz[i] = 0.2 + 0.6 * s.u();
      double w = 0.02 + 0.08 * s.u();
      double a = 0.5 + 1.5 * s.u();
      amp[i] = (s.u() < 0.5) ? -a : a;
      w2x2[i] = 2.0 * w * w;
    }
  }
  double eval(double x, double y, double z) const {
    double v = 0.0;
    for (int i = 0; i < 16; ++i) {
      double dx = x - cx[i], dy = y - cy[i], dz = z - cz[i];
      double r2 = dx * dx + dy * dy + dz * dz;
      v += amp[i] * std::exp(-r2 / w2x2[i]);
    }
    return v;
  }
};

struct Modes {
  double kx[8], ky[8], kz[8], c[8], ph[8], norm;
  void draw(Stream& s) {
    norm = 0.0;
    for (int m = 0; m < 8; ++m) {
      int k[3];
      do {
        for (int d = 0; d < 3; ++d) {
          int v = (int)(9.0 * s.u());
          if (v > 8) v = 8;
          k[d] = v - 4;
        }
      } while (k[0] == 0 && k[1] == 0 && k[2] == 0);
      kx[m] = k[0];
      ky[m] = k[1];
      kz[m] = k[2];
      c[m] = 2.0 * s.u() - 1.0;
      ph[m] = 6.283185307179586 * s.u();
      norm += std::fabs(c[m]);
    }
  }
  double eval(double x, double y, double z) const {
    double g = 0.0;
    for (int m = 0; m < 8; ++m)
      g += c[m] * std::cos(6.283185307179586 * (kx[m] * x + ky[m] * y + kz[m] * z) + ph[m]);
    g = g / norm;
    return std::exp(2.302585092994046 * g);
  }
};

struct Problem {
  Bumps bumps;
  Modes acoef, bcoef;
  explicit Problem(uint64_t seed) {
    Stream s(seed);
    bumps.draw(s);
    acoef.draw(s);
    bcoef.draw(s);
  }
};

}  // namespace cmg_synth

#endif
