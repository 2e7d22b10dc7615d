// Device evaluation of the seeded synthetic fields of synthetic.H: the same
// formulas and operation order, with exp and cos of the CUDA math library,
// so values agree with the host generator to within their last bits.
#ifndef CMG_SYNTHDEV_H
#define CMG_SYNTHDEV_H

#include "synthetic.H"

namespace cmg {

__device__ __forceinline__ double devBumps(const cmg_synth::Bumps& B, double x, double y, double z) {
  double v = 0.0;
  for (int i = 0; i < 16; ++i) {
    double dx = x - B.cx[i], dy = y - B.cy[i], dz = z - B.cz[i];
    double r2 = dx * dx + dy * dy + dz * dz;
    v += B.amp[i] * exp(-r2 / B.w2x2[i]);
  }
  return v;
}

__device__ __forceinline__ double devModes(const cmg_synth::Modes& M, double x, double y, double z) {
  double g = 0.0;
  for (int m = 0; m < 8; ++m)
    g += M.c[m] * cos(6.283185307179586 * (M.kx[m] * x + M.ky[m] * y + M.kz[m] * z) + M.ph[m]);
  g = g / M.norm;
  return exp(2.302585092994046 * g);
}

}  // namespace cmg

#endif
