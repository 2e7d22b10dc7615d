// ORACLE — test infrastructure only. Nothing in the product links this file.
//
// C++ restatement of the ChomboFortran (.ChF) leaf kernels that sit on the
// AMRMultiGrid / AMRPoissonOp / VCAMRPoissonOp2 V-cycle.  The reference builds
// these from Fortran via its chfpp preprocessor; this image has no Fortran
// compiler, so each kernel is restated here in plain C++ with the same loop
// nest (k outer, j, i inner), the same expression association order and the
// same argument list that the chfpp-generated prototype expands to in 3D
// (data pointer, lo0..lo2, hi0..hi2[, ncomp]) so that the reference's own C++
// call sites (FORT_* macros) link against it unchanged.  Build with
// -ffp-contract=off: gfortran on x86-64 does not contract a*b+c into an FMA.
//
// Every function cites the .ChF file:line (paths relative to the Chombo
// lib/src tree) that it restates.

#include <cmath>
#include <cstdlib>
#include <cstdio>

typedef double Real;

namespace {

// BaseFab layout: component-major, x fastest (BaseFabImplem.H:291-312).
struct Fab {
  Real* p;
  int lo0, lo1, lo2, hi0, hi1, hi2, nc;
  long nx, ny, nz;
  Fab(const Real* d, const int* l0, const int* l1, const int* l2,
      const int* h0, const int* h1, const int* h2, const int* n)
      : p(const_cast<Real*>(d)), lo0(*l0), lo1(*l1), lo2(*l2),
        hi0(*h0), hi1(*h1), hi2(*h2), nc(n ? *n : 1) {
    nx = hi0 - lo0 + 1;
    ny = hi1 - lo1 + 1;
    nz = hi2 - lo2 + 1;
  }
  Real& operator()(int i, int j, int k, int n = 0) const {
    return p[(i - lo0) + nx * ((j - lo1) + ny * ((k - lo2) + nz * (long)n))];
  }
};

inline void mayday(const char* what) {
  std::fprintf(stderr, "ChF oracle MAYDAYERROR in %s\n", what);
  std::abort();
}

// Fortran integer division truncates toward zero, as C++ does.
inline int fdiv(int a, int b) { return a / b; }

}  // namespace

#define FAB(name) const Real* name, const int* i##name##lo0, const int* i##name##lo1, \
    const int* i##name##lo2, const int* i##name##hi0, const int* i##name##hi1,          \
    const int* i##name##hi2, const int* n##name##comp
#define FAB1(name) const Real* name, const int* i##name##lo0, const int* i##name##lo1, \
    const int* i##name##lo2, const int* i##name##hi0, const int* i##name##hi1,           \
    const int* i##name##hi2
#define BOX(name) const int* i##name##lo0, const int* i##name##lo1, const int* i##name##lo2, \
    const int* i##name##hi0, const int* i##name##hi1, const int* i##name##hi2
#define MKFAB(name) Fab F_##name(name, i##name##lo0, i##name##lo1, i##name##lo2, \
    i##name##hi0, i##name##hi1, i##name##hi2, n##name##comp)
#define MKFAB1(name) Fab F_##name(name, i##name##lo0, i##name##lo1, i##name##lo2, \
    i##name##hi0, i##name##hi1, i##name##hi2, nullptr)
#define BLO(name, d) (*i##name##lo##d)
#define BHI(name, d) (*i##name##hi##d)

extern "C" {

// AMRPoissonOpF.ChF:9-49 (gsmcamrpop): point relaxation on a coloured box.
void gsmcamrpop_(FAB1(phi), FAB1(rhs), BOX(coloredbox), const Real* dx,
                 const Real* alpha, const Real* beta) {
  MKFAB1(phi);
  MKFAB1(rhs);
  Real dxinv = 1.0 / ((*dx) * (*dx));
  Real sum_b = 0.0;
  for (int idir = 0; idir < 3; ++idir) sum_b = sum_b + 2.0 * dxinv;
  Real lambda = 1.0 / (*alpha - *beta * sum_b);
  for (int k = BLO(coloredbox, 2); k <= BHI(coloredbox, 2); k += 2)
    for (int j = BLO(coloredbox, 1); j <= BHI(coloredbox, 1); j += 2)
      for (int i = BLO(coloredbox, 0); i <= BHI(coloredbox, 0); i += 2) {
        Real lphi = (F_phi(i + 1, j, k) + F_phi(i - 1, j, k) - 2.0 * F_phi(i, j, k)) +
                    (F_phi(i, j + 1, k) + F_phi(i, j - 1, k) - 2.0 * F_phi(i, j, k)) +
                    (F_phi(i, j, k + 1) + F_phi(i, j, k - 1) - 2.0 * F_phi(i, j, k));
        lphi = lphi * dxinv;
        F_phi(i, j, k) = F_phi(i, j, k) + lambda * (F_rhs(i, j, k) - lphi);
      }
}

// AMRPoissonOpF.ChF:51-118 (GSRBHELMHOLTZ): one colour of red-black GS for
// alpha*phi + beta*Lap(phi) = rhs.
void gsrbhelmholtz_(FAB(phi), FAB(rhs), BOX(region), const Real* dx, const Real* alpha,
                    const Real* beta, const int* redBlack) {
  MKFAB(phi);
  MKFAB(rhs);
  Real dxinv = 1.0 / ((*dx) * (*dx));
  Real sum_b = 0.0;
  for (int idir = 0; idir < 3; ++idir) sum_b = sum_b + 2.0 * dxinv;
  Real lambda = -1.0 / (*alpha - *beta * sum_b);
  int ncomp = F_phi.nc;
  if (ncomp != F_rhs.nc) mayday("GSRBHELMHOLTZ");
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j) {
        int imin = BLO(region, 0);
        int indtot = imin + j + k;
        imin = imin + std::abs((indtot + *redBlack) % 2);
        int imax = BHI(region, 0);
        for (int i = imin; i <= imax; i += 2) {
          Real lphi = (F_phi(i + 1, j, k, n) + F_phi(i - 1, j, k, n) + F_phi(i, j + 1, k, n) +
                       F_phi(i, j - 1, k, n) + F_phi(i, j, k + 1, n) + F_phi(i, j, k - 1, n) -
                       2.0 * 3 * F_phi(i, j, k, n)) *
                      dxinv;
          Real helmop = *alpha * F_phi(i, j, k, n) + *beta * lphi;
          F_phi(i, j, k, n) = F_phi(i, j, k, n) + lambda * (helmop - F_rhs(i, j, k, n));
        }
      }
}

// AMRPoissonOpF.ChF:120-198 (GSRBLAPLACIAN): one colour of red-black GS for
// Lap(phi) = rhs (alpha = 0, beta = 1), the active (#else) branch.
void gsrblaplacian_(FAB(phi), FAB(rhs), BOX(region), const Real* dx, const int* redBlack) {
  MKFAB(phi);
  MKFAB(rhs);
  Real dxinv = 1.0 / ((*dx) * (*dx));
  Real sum_b = 0.0;
  for (int idir = 0; idir < 3; ++idir) sum_b = sum_b + 2.0 * dxinv;
  Real lambda = -1.0 / sum_b;
  int ncomp = F_phi.nc;
  if (ncomp != F_rhs.nc) mayday("GSRBLAPLACIAN");
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j) {
        int imin = BLO(region, 0);
        int indtot = imin + j + k;
        imin = imin + std::abs((indtot + *redBlack) % 2);
        int imax = BHI(region, 0);
        for (int i = imin; i <= imax; i += 2) {
          Real lphi = (F_phi(i + 1, j, k, n) + F_phi(i - 1, j, k, n) + F_phi(i, j + 1, k, n) +
                       F_phi(i, j - 1, k, n) + F_phi(i, j, k + 1, n) + F_phi(i, j, k - 1, n)) *
                      dxinv;
          F_phi(i, j, k, n) = lambda * (F_rhs(i, j, k, n) - lphi);
        }
      }
}

// AMRPoissonOpF.ChF:200-232 (gsrblazy).
void gsrblazy_(FAB1(phi), FAB1(lphi), FAB1(rhs), BOX(coloredbox), const Real* alpha,
               const Real* beta, const Real* dx) {
  MKFAB1(phi);
  MKFAB1(lphi);
  MKFAB1(rhs);
  Real dxinv = 1.0 / ((*dx) * (*dx));
  Real sum_b = 0.0;
  for (int idir = 0; idir < 3; ++idir) sum_b = sum_b + 2.0 * dxinv;
  Real lambda = -1.0 / (*alpha - *beta * sum_b);
  for (int k = BLO(coloredbox, 2); k <= BHI(coloredbox, 2); k += 2)
    for (int j = BLO(coloredbox, 1); j <= BHI(coloredbox, 1); j += 2)
      for (int i = BLO(coloredbox, 0); i <= BHI(coloredbox, 0); i += 2)
        F_phi(i, j, k) = F_phi(i, j, k) - lambda * (F_rhs(i, j, k) - F_lphi(i, j, k));
}

// AMRPoissonOpF.ChF:287-324 (OPERATORLAP): lofphi = alpha*phi + beta*Lap(phi).
void operatorlap_(FAB(lofphi), FAB(phi), BOX(region), const Real* dx, const Real* alpha,
                  const Real* beta) {
  MKFAB(lofphi);
  MKFAB(phi);
  int ncomp = F_phi.nc;
  if (ncomp != F_lofphi.nc) mayday("OPERATORLAP");
  Real dxinv = 1.0 / ((*dx) * (*dx));
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j)
        for (int i = BLO(region, 0); i <= BHI(region, 0); ++i) {
          Real lap = (F_phi(i + 1, j, k, n) + F_phi(i - 1, j, k, n) + F_phi(i, j + 1, k, n) +
                      F_phi(i, j - 1, k, n) + F_phi(i, j, k + 1, n) + F_phi(i, j, k - 1, n) -
                      (Real)(2 * 3) * F_phi(i, j, k, n)) *
                     dxinv;
          F_lofphi(i, j, k, n) = *alpha * F_phi(i, j, k, n) + *beta * lap;
        }
}

// AMRPoissonOpF.ChF:341-377 (OPERATORLAPRES): r = rhs - (alpha*phi + beta*Lap(phi)),
// evaluated as -alpha*phi - beta*lap + rhs.
void operatorlapres_(FAB(r), FAB(phi), FAB(rhs), BOX(region), const Real* dx,
                     const Real* alpha, const Real* beta) {
  MKFAB(r);
  MKFAB(phi);
  MKFAB(rhs);
  int ncomp = F_phi.nc;
  Real dxinv = 1.0 / ((*dx) * (*dx));
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j)
        for (int i = BLO(region, 0); i <= BHI(region, 0); ++i) {
          Real lap = (F_phi(i + 1, j, k, n) + F_phi(i - 1, j, k, n) + F_phi(i, j + 1, k, n) +
                      F_phi(i, j - 1, k, n) + F_phi(i, j, k + 1, n) + F_phi(i, j, k - 1, n) -
                      (Real)(2 * 3) * F_phi(i, j, k, n)) *
                     dxinv;
          F_r(i, j, k, n) = -(*alpha * F_phi(i, j, k, n)) - *beta * lap + F_rhs(i, j, k, n);
        }
}

// AMRPoissonOpF.ChF:394-438 (RESTRICTRES): res[i/2] += (rhs - L phi)/8, in fine
// k-j-i order.
void restrictres_(FAB(res), FAB(phi), FAB(rhs), const Real* alpha, const Real* beta,
                  BOX(region), const Real* dx) {
  MKFAB(res);
  MKFAB(phi);
  MKFAB(rhs);
  int ncomp = F_phi.nc;
  Real dxinv = 1.0 / ((*dx) * (*dx));
  Real denom = 2 * 2 * 2;
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j)
        for (int i = BLO(region, 0); i <= BHI(region, 0); ++i) {
          int ii = fdiv(i, 2), jj = fdiv(j, 2), kk = fdiv(k, 2);
          Real lofphi = *alpha * F_phi(i, j, k, n) +
                        *beta *
                            (F_phi(i + 1, j, k, n) + F_phi(i - 1, j, k, n) + F_phi(i, j + 1, k, n) +
                             F_phi(i, j - 1, k, n) + F_phi(i, j, k + 1, n) + F_phi(i, j, k - 1, n) -
                             F_phi(i, j, k, n) * 2 * 3) *
                            dxinv;
          F_res(ii, jj, kk, n) = F_res(ii, jj, kk, n) + (F_rhs(i, j, k, n) - lofphi) / denom;
        }
}

// AMRPoissonOpF.ChF:453-478 (PROLONG): piecewise-constant phi[i] += coarse[i/m].
void prolong_(FAB(phi), FAB(coarse), BOX(region), const int* m) {
  MKFAB(phi);
  MKFAB(coarse);
  int ncomp = F_phi.nc;
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j)
        for (int i = BLO(region, 0); i <= BHI(region, 0); ++i)
          F_phi(i, j, k, n) = F_phi(i, j, k, n) + F_coarse(fdiv(i, *m), fdiv(j, *m), fdiv(k, *m), n);
}

// AMRPoissonOpF.ChF:492-555 (PROLONG_2): trilinear-like prolongation (ratio 2).
void prolong_2_(FAB(phi), FAB(coarse), BOX(region), const int* m) {
  MKFAB(phi);
  MKFAB(coarse);
  Real den = 1.0 / (Real)(4 * 4 * 4);
  Real fx[3];
  fx[0] = 3.0 * den;
  fx[1] = 9.0 * den;
  fx[2] = 27.0 * den;
  Real f0 = 1.0 * den;
  int ncomp = F_phi.nc;
  for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
    for (int j = BLO(region, 1); j <= BHI(region, 1); ++j)
      for (int i = BLO(region, 0); i <= BHI(region, 0); ++i) {
        int ic = fdiv(i, *m), jc = fdiv(j, *m), kc = fdiv(k, *m);
        int o0 = 2 * (i % 2) - 1, o1 = 2 * (j % 2) - 1, o2 = 2 * (k % 2) - 1;
        for (int n = 0; n < ncomp; ++n) {
          F_phi(i, j, k, n) = F_phi(i, j, k, n) + fx[2] * F_coarse(ic, jc, kc, n) +
                              f0 * F_coarse(ic + o0, jc + o1, kc + o2, n);
          F_phi(i, j, k, n) = F_phi(i, j, k, n) +
                              fx[1] * (F_coarse(ic + o0, jc, kc, n) + F_coarse(ic, jc + o1, kc, n) +
                                       F_coarse(ic, jc, kc + o2, n));
          F_phi(i, j, k, n) = F_phi(i, j, k, n) +
                              fx[0] * (F_coarse(ic + o0, jc + o1, kc, n) +
                                       F_coarse(ic, jc + o1, kc + o2, n) +
                                       F_coarse(ic + o0, jc, kc + o2, n));
        }
      }
}

// AMRPoissonOpF.ChF:557-586 (NEWGETFLUX): flux = (phi[i] - phi[i - e_dir]) * beta_dx.
void newgetflux_(FAB(flux), FAB(phi), BOX(box), const Real* beta_dx, const int* a_idir) {
  MKFAB(flux);
  MKFAB(phi);
  int ii = (*a_idir == 0), jj = (*a_idir == 1), kk = (*a_idir == 2);
  int ncomp = F_phi.nc;
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(box, 2); k <= BHI(box, 2); ++k)
      for (int j = BLO(box, 1); j <= BHI(box, 1); ++j)
        for (int i = BLO(box, 0); i <= BHI(box, 0); ++i)
          F_flux(i, j, k, n) = (F_phi(i, j, k, n) - F_phi(i - ii, j - jj, k - kk, n)) * (*beta_dx);
}

// VCAMRPoissonOpF.ChF:57-125 (GSRBHELMHOLTZVC3D): one colour of red-black GS for
// alpha*a*phi - beta*div(b grad phi) = rhs with precomputed lambda.
void gsrbhelmholtzvc3d_(FAB(phi), FAB(rhs), BOX(region), const Real* dx, const Real* alpha,
                        FAB(aCoef), const Real* beta, FAB(bCoef0), FAB(bCoef1), FAB(bCoef2),
                        FAB(lambda), const int* redBlack) {
  MKFAB(phi);
  MKFAB(rhs);
  MKFAB(aCoef);
  MKFAB(bCoef0);
  MKFAB(bCoef1);
  MKFAB(bCoef2);
  MKFAB(lambda);
  int ncomp = F_phi.nc;
  if (ncomp != F_rhs.nc) mayday("GSRBHELMHOLTZVC");
  if (ncomp != F_bCoef0.nc || ncomp != F_bCoef1.nc || ncomp != F_bCoef2.nc)
    mayday("GSRBHELMHOLTZVC");
  Real dxinv = 1.0 / ((*dx) * (*dx));
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j) {
        int imin = BLO(region, 0);
        int indtot = imin + j + k;
        imin = imin + std::abs((indtot + *redBlack) % 2);
        int imax = BHI(region, 0);
        for (int i = imin; i <= imax; i += 2) {
          Real p = F_phi(i, j, k, n);
          Real lofphi =
              *alpha * F_aCoef(i, j, k, n) * p -
              *beta *
                  (F_bCoef0(i + 1, j, k, n) * (F_phi(i + 1, j, k, n) - p) -
                   F_bCoef0(i, j, k, n) * (p - F_phi(i - 1, j, k, n)) +
                   F_bCoef1(i, j + 1, k, n) * (F_phi(i, j + 1, k, n) - p) -
                   F_bCoef1(i, j, k, n) * (p - F_phi(i, j - 1, k, n)) +
                   F_bCoef2(i, j, k + 1, n) * (F_phi(i, j, k + 1, n) - p) -
                   F_bCoef2(i, j, k, n) * (p - F_phi(i, j, k - 1, n))) *
                  dxinv;
          F_phi(i, j, k, n) = p - F_lambda(i, j, k, n) * (lofphi - F_rhs(i, j, k, n));
        }
      }
}

// VCAMRPoissonOpF.ChF:148-216 (VCCOMPUTEOP3D).
void vccomputeop3d_(FAB(lofphi), FAB(phi), const Real* alpha, FAB(aCoef), const Real* beta,
                    FAB(bCoef0), FAB(bCoef1), FAB(bCoef2), BOX(region), const Real* dx) {
  MKFAB(lofphi);
  MKFAB(phi);
  MKFAB(aCoef);
  MKFAB(bCoef0);
  MKFAB(bCoef1);
  MKFAB(bCoef2);
  int ncomp = F_phi.nc;
  if (ncomp != F_lofphi.nc) mayday("VCCOMPUTEOP");
  if (ncomp != F_bCoef0.nc || ncomp != F_bCoef1.nc || ncomp != F_bCoef2.nc)
    mayday("VCCOMPUTEOP");
  Real dxinv = 1.0 / ((*dx) * (*dx));
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j)
        for (int i = BLO(region, 0); i <= BHI(region, 0); ++i) {
          Real p = F_phi(i, j, k, n);
          F_lofphi(i, j, k, n) =
              *alpha * F_aCoef(i, j, k, n) * p -
              *beta *
                  (F_bCoef0(i + 1, j, k, n) * (F_phi(i + 1, j, k, n) - p) -
                   F_bCoef0(i, j, k, n) * (p - F_phi(i - 1, j, k, n)) +
                   F_bCoef1(i, j + 1, k, n) * (F_phi(i, j + 1, k, n) - p) -
                   F_bCoef1(i, j, k, n) * (p - F_phi(i, j - 1, k, n)) +
                   F_bCoef2(i, j, k + 1, n) * (F_phi(i, j, k + 1, n) - p) -
                   F_bCoef2(i, j, k, n) * (p - F_phi(i, j, k - 1, n))) *
                  dxinv;
        }
}

// VCAMRPoissonOpF.ChF:241-312 (VCCOMPUTERES3D): res = rhs - (alpha a phi - beta div b grad phi).
void vccomputeres3d_(FAB(res), FAB(phi), FAB(rhs), const Real* alpha, FAB(aCoef),
                     const Real* beta, FAB(bCoef0), FAB(bCoef1), FAB(bCoef2), BOX(region),
                     const Real* dx) {
  MKFAB(res);
  MKFAB(phi);
  MKFAB(rhs);
  MKFAB(aCoef);
  MKFAB(bCoef0);
  MKFAB(bCoef1);
  MKFAB(bCoef2);
  int ncomp = F_phi.nc;
  if (ncomp != F_res.nc) mayday("VCCOMPUTERES");
  if (ncomp != F_bCoef0.nc || ncomp != F_bCoef1.nc || ncomp != F_bCoef2.nc)
    mayday("VCCOMPUTERES");
  Real dxinv = 1.0 / ((*dx) * (*dx));
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j)
        for (int i = BLO(region, 0); i <= BHI(region, 0); ++i) {
          Real p = F_phi(i, j, k, n);
          F_res(i, j, k, n) =
              F_rhs(i, j, k, n) -
              (*alpha * F_aCoef(i, j, k, n) * p -
               *beta *
                   (F_bCoef0(i + 1, j, k, n) * (F_phi(i + 1, j, k, n) - p) -
                    F_bCoef0(i, j, k, n) * (p - F_phi(i - 1, j, k, n)) +
                    F_bCoef1(i, j + 1, k, n) * (F_phi(i, j + 1, k, n) - p) -
                    F_bCoef1(i, j, k, n) * (p - F_phi(i, j - 1, k, n)) +
                    F_bCoef2(i, j, k + 1, n) * (F_phi(i, j, k + 1, n) - p) -
                    F_bCoef2(i, j, k, n) * (p - F_phi(i, j, k - 1, n))) *
                   dxinv);
        }
}

// VCAMRPoissonOpF.ChF:337-413 (RESTRICTRESVC3D).
void restrictresvc3d_(FAB(res), FAB(phi), FAB(rhs), const Real* alpha, FAB(aCoef),
                      const Real* beta, FAB(bCoef0), FAB(bCoef1), FAB(bCoef2), BOX(region),
                      const Real* dx) {
  MKFAB(res);
  MKFAB(phi);
  MKFAB(rhs);
  MKFAB(aCoef);
  MKFAB(bCoef0);
  MKFAB(bCoef1);
  MKFAB(bCoef2);
  int ncomp = F_phi.nc;
  Real dxinv = 1.0 / ((*dx) * (*dx));
  Real denom = 2 * 2 * 2;
  for (int n = 0; n < ncomp; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j)
        for (int i = BLO(region, 0); i <= BHI(region, 0); ++i) {
          int ii = fdiv(i, 2), jj = fdiv(j, 2), kk = fdiv(k, 2);
          Real p = F_phi(i, j, k, n);
          Real lofphi =
              *alpha * F_aCoef(i, j, k, n) * p -
              *beta *
                  (F_bCoef0(i + 1, j, k, n) * (F_phi(i + 1, j, k, n) - p) -
                   F_bCoef0(i, j, k, n) * (p - F_phi(i - 1, j, k, n)) +
                   F_bCoef1(i, j + 1, k, n) * (F_phi(i, j + 1, k, n) - p) -
                   F_bCoef1(i, j, k, n) * (p - F_phi(i, j - 1, k, n)) +
                   F_bCoef2(i, j, k + 1, n) * (F_phi(i, j, k + 1, n) - p) -
                   F_bCoef2(i, j, k, n) * (p - F_phi(i, j, k - 1, n))) *
                  dxinv;
          F_res(ii, jj, kk, n) = F_res(ii, jj, kk, n) + (F_rhs(i, j, k, n) - lofphi) / denom;
        }
}

// VCAMRPoissonOpF.ChF:498-525 (SUMFACES): lhs += scale*beta*(b[i+e_dir] + b[i]).
void sumfaces_(FAB(lhs), const Real* beta, FAB(bCoefs), BOX(box), const int* dir,
               const Real* scale) {
  MKFAB(lhs);
  MKFAB(bCoefs);
  int ii = (*dir == 0), jj = (*dir == 1), kk = (*dir == 2);
  for (int n = 0; n < F_lhs.nc; ++n)
    for (int k = BLO(box, 2); k <= BHI(box, 2); ++k)
      for (int j = BLO(box, 1); j <= BHI(box, 1); ++j)
        for (int i = BLO(box, 0); i <= BHI(box, 0); ++i) {
          Real sumVal = F_bCoefs(i + ii, j + jj, k + kk, n) + F_bCoefs(i, j, k, n);
          F_lhs(i, j, k, n) = F_lhs(i, j, k, n) + *scale * *beta * sumVal;
        }
}

// AverageF.ChF:9-163 (average): arithmetic mean over the refRatio^3 fine cells.
// Ratio 2 and 4 use the unrolled, fixed summation order of the .ChF.
void average_(FAB(coarse), FAB(fine), BOX(box), const int* refRatio, BOX(bref)) {
  MKFAB(coarse);
  MKFAB(fine);
  int r = *refRatio;
  Real refScale = 1.0 / (Real)(r * r * r);
  for (int var = 0; var < F_coarse.nc; ++var)
    for (int k = BLO(box, 2); k <= BHI(box, 2); ++k)
      for (int j = BLO(box, 1); j <= BHI(box, 1); ++j)
        for (int i = BLO(box, 0); i <= BHI(box, 0); ++i) {
          int p0 = i * r, p1 = j * r, p2 = k * r;
          Real s = 0.0;
          if (r == 2) {
            s = F_fine(p0, p1, p2, var) + F_fine(p0 + 1, p1, p2, var) +
                F_fine(p0, p1 + 1, p2, var) + F_fine(p0 + 1, p1 + 1, p2, var) +
                F_fine(p0, p1, p2 + 1, var) + F_fine(p0 + 1, p1, p2 + 1, var) +
                F_fine(p0, p1 + 1, p2 + 1, var) + F_fine(p0 + 1, p1 + 1, p2 + 1, var);
            F_coarse(i, j, k, var) = refScale * s;
          } else if (r == 4) {
            bool first = true;
            for (int c = 0; c < 4; ++c)
              for (int b = 0; b < 4; ++b)
                for (int a = 0; a < 4; ++a) {
                  Real v = F_fine(p0 + a, p1 + b, p2 + c, var);
                  s = first ? v : s + v;
                  first = false;
                }
            F_coarse(i, j, k, var) = refScale * s;
          } else {
            Real coarseSum = 0;
            for (int c = BLO(bref, 2); c <= BHI(bref, 2); ++c)
              for (int b = BLO(bref, 1); b <= BHI(bref, 1); ++b)
                for (int a = BLO(bref, 0); a <= BHI(bref, 0); ++a)
                  coarseSum = coarseSum + F_fine(p0 + a, p1 + b, p2 + c, var);
            F_coarse(i, j, k, var) = coarseSum * refScale;
          }
        }
}

// AverageF.ChF:166-318 (averageharmonic).
void averageharmonic_(FAB(coarse), FAB(fine), BOX(box), const int* refRatio, BOX(bref)) {
  MKFAB(coarse);
  MKFAB(fine);
  int r = *refRatio;
  Real refScale = 1.0 / (Real)(r * r * r);
  for (int var = 0; var < F_coarse.nc; ++var)
    for (int k = BLO(box, 2); k <= BHI(box, 2); ++k)
      for (int j = BLO(box, 1); j <= BHI(box, 1); ++j)
        for (int i = BLO(box, 0); i <= BHI(box, 0); ++i) {
          int p0 = i * r, p1 = j * r, p2 = k * r;
          if (r == 2 || r == 4) {
            Real s = 0.0;
            bool first = true;
            for (int c = 0; c < r; ++c)
              for (int b = 0; b < r; ++b)
                for (int a = 0; a < r; ++a) {
                  Real v = 1.0 / F_fine(p0 + a, p1 + b, p2 + c, var);
                  s = first ? v : s + v;
                  first = false;
                }
            F_coarse(i, j, k, var) = refScale * s;
            F_coarse(i, j, k, var) = 1.0 / F_coarse(i, j, k, var);
          } else {
            Real coarseSum = 0;
            for (int c = BLO(bref, 2); c <= BHI(bref, 2); ++c)
              for (int b = BLO(bref, 1); b <= BHI(bref, 1); ++b)
                for (int a = BLO(bref, 0); a <= BHI(bref, 0); ++a)
                  coarseSum = coarseSum + 1.0 / F_fine(p0 + a, p1 + b, p2 + c, var);
            F_coarse(i, j, k, var) = 1.0 / (coarseSum * refScale);
          }
        }
}

// AverageFaceF.ChF:22-66 (AVERAGEFACE): sum over the refBox fine faces times
// (1/refFactor)^(D-1).
void averageface_(FAB(coarse), FAB(fine), BOX(crseBox), const int* dir, const int* nRef,
                  const int* refFactor, BOX(refBox)) {
  MKFAB(coarse);
  MKFAB(fine);
  (void)dir;
  Real base = 1.0 / (Real)(*refFactor);
  Real ref_scale = base * base;
  int r = *nRef;
  for (int var = 0; var < F_coarse.nc; ++var)
    for (int k = BLO(crseBox, 2); k <= BHI(crseBox, 2); ++k)
      for (int j = BLO(crseBox, 1); j <= BHI(crseBox, 1); ++j)
        for (int i = BLO(crseBox, 0); i <= BHI(crseBox, 0); ++i) {
          Real crseSum = 0;
          for (int c = BLO(refBox, 2); c <= BHI(refBox, 2); ++c)
            for (int b = BLO(refBox, 1); b <= BHI(refBox, 1); ++b)
              for (int a = BLO(refBox, 0); a <= BHI(refBox, 0); ++a)
                crseSum = crseSum + F_fine(i * r + a, j * r + b, k * r + c, var);
          F_coarse(i, j, k, var) = ref_scale * crseSum;
        }
}

// AverageFaceF.ChF:84-128 (AVERAGEFACEHARMONIC).
void averagefaceharmonic_(FAB(coarse), FAB(fine), BOX(crseBox), const int* dir,
                          const int* nRef, const int* refFactor, BOX(refBox)) {
  MKFAB(coarse);
  MKFAB(fine);
  (void)dir;
  Real base = 1.0 / (Real)(*refFactor);
  Real ref_scale = base * base;
  int r = *nRef;
  for (int var = 0; var < F_coarse.nc; ++var)
    for (int k = BLO(crseBox, 2); k <= BHI(crseBox, 2); ++k)
      for (int j = BLO(crseBox, 1); j <= BHI(crseBox, 1); ++j)
        for (int i = BLO(crseBox, 0); i <= BHI(crseBox, 0); ++i) {
          Real crseSum = 0;
          for (int c = BLO(refBox, 2); c <= BHI(refBox, 2); ++c)
            for (int b = BLO(refBox, 1); b <= BHI(refBox, 1); ++b)
              for (int a = BLO(refBox, 0); a <= BHI(refBox, 0); ++a)
                crseSum = crseSum + 1.0 / F_fine(i * r + a, j * r + b, k * r + c, var);
          F_coarse(i, j, k, var) = 1.0 / (ref_scale * crseSum);
        }
}

// InterpF.ChF:435-464 (INTERPHOMO): homogeneous quadratic coarse-fine ghost,
// ghost = c1*phi[+1 inward] + c2*phi[+2 inward].  The .ChF negates its ihilo
// argument in place; the callers pass a fresh local, so the side effect is kept.
void interphomo_(FAB(phi), BOX(region), const Real* x1, const Real* dxCrse, const int* idir,
                 const int* ihilo) {
  MKFAB(phi);
  Real c1 = 2.0 * (*dxCrse - *x1) / (*dxCrse + *x1);
  Real c2 = -(*dxCrse - *x1) / (*dxCrse + 3.0 * *x1);
  int* hl = const_cast<int*>(ihilo);
  *hl = *hl * (-1);
  int s = *hl;
  int d0 = (*idir == 0) * s, d1 = (*idir == 1) * s, d2 = (*idir == 2) * s;
  for (int n = 0; n < F_phi.nc; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j)
        for (int i = BLO(region, 0); i <= BHI(region, 0); ++i) {
          Real pa = F_phi(i + d0, j + d1, k + d2, n);
          Real pb = F_phi(i + 2 * d0, j + 2 * d1, k + 2 * d2, n);
          F_phi(i, j, k, n) = c1 * pa + c2 * pb;
        }
}

// InterpF.ChF:466-494 (INTERPHOMOLINEAR).
void interphomolinear_(FAB(phi), BOX(region), const Real* x1, const Real* dxCrse,
                       const int* idir, const int* ihilo) {
  MKFAB(phi);
  int* hl = const_cast<int*>(ihilo);
  *hl = *hl * (-1);
  int s = *hl;
  int d0 = (*idir == 0) * s, d1 = (*idir == 1) * s, d2 = (*idir == 2) * s;
  Real factor = 1.0 - 2.0 * *x1 / (*x1 + *dxCrse);
  for (int n = 0; n < F_phi.nc; ++n)
    for (int k = BLO(region, 2); k <= BHI(region, 2); ++k)
      for (int j = BLO(region, 1); j <= BHI(region, 1); ++j)
        for (int i = BLO(region, 0); i <= BHI(region, 0); ++i) {
          Real pa = F_phi(i + d0, j + d1, k + d2, n);
          F_phi(i, j, k, n) = factor * pa;
        }
}

// InterpF.ChF:12-44 (interpconstant): every fine cell of the refined box of
// each coarse cell of b takes the coarse value.
void interpconstant_(FAB(fine), FAB(coarse), BOX(b), const int* refRatio, BOX(bref)) {
  MKFAB(fine);
  MKFAB(coarse);
  const int r = *refRatio;
  for (int var = 0; var < F_coarse.nc; ++var)
    for (int k = BLO(b, 2); k <= BHI(b, 2); ++k)
      for (int j = BLO(b, 1); j <= BHI(b, 1); ++j)
        for (int i = BLO(b, 0); i <= BHI(b, 0); ++i)
          for (int kk = BLO(bref, 2); kk <= BHI(bref, 2); ++kk)
            for (int jj = BLO(bref, 1); jj <= BHI(bref, 1); ++jj)
              for (int ii = BLO(bref, 0); ii <= BHI(bref, 0); ++ii)
                F_fine(i * r + ii, j * r + jj, k * r + kk, var) = F_coarse(i, j, k, var);
}

// InterpF.ChF:48-71 (interpcentralslope): half * (state[+1] - state[-1]).
void interpcentralslope_(FAB(slope), FAB(state), BOX(b), const int* dir) {
  MKFAB(slope);
  MKFAB(state);
  const int d0 = *dir == 0, d1 = *dir == 1, d2 = *dir == 2;
  for (int var = 0; var < F_state.nc; ++var)
    for (int k = BLO(b, 2); k <= BHI(b, 2); ++k)
      for (int j = BLO(b, 1); j <= BHI(b, 1); ++j)
        for (int i = BLO(b, 0); i <= BHI(b, 0); ++i)
          F_slope(i, j, k, var) = 0.5 * (F_state(i + d0, j + d1, k + d2, var) - F_state(i - d0, j - d1, k - d2, var));
}

// InterpF.ChF:76-100 (interphisideslope): state[+1] - state.
void interphisideslope_(FAB(slope), FAB(state), BOX(b), const int* dir) {
  MKFAB(slope);
  MKFAB(state);
  const int d0 = *dir == 0, d1 = *dir == 1, d2 = *dir == 2;
  for (int var = 0; var < F_state.nc; ++var)
    for (int k = BLO(b, 2); k <= BHI(b, 2); ++k)
      for (int j = BLO(b, 1); j <= BHI(b, 1); ++j)
        for (int i = BLO(b, 0); i <= BHI(b, 0); ++i)
          F_slope(i, j, k, var) = F_state(i + d0, j + d1, k + d2, var) - F_state(i, j, k, var);
}

// InterpF.ChF:104-126 (interplosideslope): state - state[-1].
void interplosideslope_(FAB(slope), FAB(state), BOX(b), const int* dir) {
  MKFAB(slope);
  MKFAB(state);
  const int d0 = *dir == 0, d1 = *dir == 1, d2 = *dir == 2;
  for (int var = 0; var < F_state.nc; ++var)
    for (int k = BLO(b, 2); k <= BHI(b, 2); ++k)
      for (int j = BLO(b, 1); j <= BHI(b, 1); ++j)
        for (int i = BLO(b, 0); i <= BHI(b, 0); ++i)
          F_slope(i, j, k, var) = F_state(i, j, k, var) - F_state(i - d0, j - d1, k - d2, var);
}

// InterpF.ChF:135-312 (interplimit): multidimensional limiter.  statemax /
// statemin over the neighbours (bn) inside the state FAB; deltasum = half *
// (|islope| + |jslope| + |kslope|); eta = min(statemax - state, state -
// statemin), zero when eta <= 1.e-9 * |statemax|, else eta / deltasum when
// deltasum > eta, else one; every slope scaled by eta.  The literal 1.e-9 is
// a default-kind (single precision) Fortran constant in the reference's GNU
// build (no real-8 promotion flag), so it enters as (double)1.0e-9f.
void interplimit_(FAB(islope), FAB(jslope), FAB(kslope), FAB(state), BOX(bcoarse), BOX(bn), BOX(physdomain)) {
  MKFAB(islope);
  MKFAB(jslope);
  MKFAB(kslope);
  MKFAB(state);
  (void)iphysdomainlo0; (void)iphysdomainlo1; (void)iphysdomainlo2;
  (void)iphysdomainhi0; (void)iphysdomainhi1; (void)iphysdomainhi2;
  const Real tiny = (Real)1.0e-9f;
  for (int var = 0; var < F_islope.nc; ++var)
    for (int k = BLO(bcoarse, 2); k <= BHI(bcoarse, 2); ++k)
      for (int j = BLO(bcoarse, 1); j <= BHI(bcoarse, 1); ++j)
        for (int i = BLO(bcoarse, 0); i <= BHI(bcoarse, 0); ++i) {
          const Real s = F_state(i, j, k, var);
          Real smax = s, smin = s;
          for (int kk = BLO(bn, 2); kk <= BHI(bn, 2); ++kk)
            for (int jj = BLO(bn, 1); jj <= BHI(bn, 1); ++jj)
              for (int ii = BLO(bn, 0); ii <= BHI(bn, 0); ++ii) {
                const int a = i + ii, b = j + jj, c = k + kk;
                if (a >= F_state.lo0 && a <= F_state.hi0 && b >= F_state.lo1 && b <= F_state.hi1 &&
                    c >= F_state.lo2 && c <= F_state.hi2) {
                  const Real v = F_state(a, b, c, var);
                  smax = std::fmax(smax, v);
                  smin = std::fmin(smin, v);
                }
              }
          const Real deltasum = 0.5 * (std::fabs(F_islope(i, j, k, var)) + std::fabs(F_jslope(i, j, k, var)) +
                                       std::fabs(F_kslope(i, j, k, var)));
          Real eta = std::fmin(smax - s, s - smin);
          if (eta <= tiny * std::fabs(smax)) {
            eta = 0.0;
          } else if (deltasum > eta) {
            eta = eta / deltasum;
          } else {
            eta = 1.0;
          }
          F_islope(i, j, k, var) = eta * F_islope(i, j, k, var);
          F_jslope(i, j, k, var) = eta * F_jslope(i, j, k, var);
          F_kslope(i, j, k, var) = eta * F_kslope(i, j, k, var);
        }
}

// InterpF.ChF:318-369 (interplinear): fine += dxf * slope over the refined
// box of each coarse cell, dxf = -half + (id + half) / ref_ratio with id the
// fine offset in direction dir.
void interplinear_(FAB(fine), FAB(slope), BOX(b), const int* dir, const int* refRatio, BOX(bref)) {
  MKFAB(fine);
  MKFAB(slope);
  const int r = *refRatio, d = *dir;
  for (int var = 0; var < F_fine.nc; ++var)
    for (int k = BLO(b, 2); k <= BHI(b, 2); ++k)
      for (int j = BLO(b, 1); j <= BHI(b, 1); ++j)
        for (int i = BLO(b, 0); i <= BHI(b, 0); ++i)
          for (int kk = BLO(bref, 2); kk <= BHI(bref, 2); ++kk)
            for (int jj = BLO(bref, 1); jj <= BHI(bref, 1); ++jj)
              for (int ii = BLO(bref, 0); ii <= BHI(bref, 0); ++ii) {
                const int id = d == 0 ? ii : (d == 1 ? jj : kk);
                const Real dxf = -0.5 + ((id + 0.5) / r);
                Real& f = F_fine(i * r + ii, j * r + jj, k * r + kk, var);
                f = f + dxf * F_slope(i, j, k, var);
              }
}

// QuadCFInterpF.ChF:9-48 (quadinterp): quadratic through phistar and two
// interior fine cells.
void quadinterp_(FAB(phi), FAB(phistar), BOX(box), const int* ihilo, const Real* h,
                 const int* idir, const int* scomp, const int* ecomp, const int* nref) {
  MKFAB(phi);
  MKFAB(phistar);
  int nr = *nref;
  Real frac = 2.0 / ((*h) * (*h));
  Real denom = (Real)(nr * nr + 4 * nr + 3);
  Real mult = frac / denom;
  Real invh = 1.0 / *h;
  Real x = 2.0 * *h;
  Real xsquared = 4.0 * (*h) * (*h);
  int s = *ihilo;
  int d0 = (*idir == 0) * s, d1 = (*idir == 1) * s, d2 = (*idir == 2) * s;
  for (int n = *scomp; n <= *ecomp; ++n)
    for (int k = BLO(box, 2); k <= BHI(box, 2); ++k)
      for (int j = BLO(box, 1); j <= BHI(box, 1); ++j)
        for (int i = BLO(box, 0); i <= BHI(box, 0); ++i) {
          Real pa = F_phi(i - 2 * d0, j - 2 * d1, k - 2 * d2, n);
          Real pb = F_phi(i - d0, j - d1, k - d2, n);
          Real ps = F_phistar(i + d0, j + d1, k + d2, n);
          Real a = mult * (2.0 * ps + (Real)(nr + 1) * pa - (Real)(nr + 3) * pb);
          Real b = (pb - pa) * invh - a * *h;
          F_phi(i, j, k, n) = xsquared * a + b * x + pa;
        }
}

// QuadCFInterpF.ChF:50-126 (PHISTAR): coarse value extrapolated tangentially to
// the fine ghost location, aa + update1 + update2 + update3.
void phistar_(FAB(fPhiStar), BOX(region), FAB(phic), FAB(coarslope), FAB(coarcurva),
              FAB(coarmixed), const Real* dxf, const int* ivar, const int* dir, const int* sign,
              const int* nRef) {
  MKFAB(fPhiStar);
  MKFAB(phic);
  MKFAB(coarslope);
  MKFAB(coarcurva);
  MKFAB(coarmixed);
  static const int YOU[2][3] = {{1, 0, 0}, {2, 2, 1}};
  int nr = *nRef;
  Real dxc = nr * *dxf;
  int you1 = YOU[0][*dir], you2 = YOU[1][*dir];
  int s = *sign;
  int d[3] = {(*dir == 0) * s, (*dir == 1) * s, (*dir == 2) * s};
  for (int r2 = BLO(region, 2); r2 <= BHI(region, 2); ++r2)
    for (int r1 = BLO(region, 1); r1 <= BHI(region, 1); ++r1)
      for (int r0 = BLO(region, 0); r0 <= BHI(region, 0); ++r0) {
        int ic[3] = {fdiv(r0, nr), fdiv(r1, nr), fdiv(r2, nr)};
        int ivf[3] = {r0, r1, r2};
        Real xf1 = (ivf[you1] + 0.5) * *dxf;
        Real xc1 = (ic[you1] + 0.5) * dxc;
        Real xf2 = (ivf[you2] + 0.5) * *dxf;
        Real xc2 = (ic[you2] + 0.5) * dxc;
        Real x1 = xf1 - xc1;
        Real x2 = xf2 - xc2;
        Real aa = F_phic(ic[0], ic[1], ic[2], *ivar);
        Real update1 = x1 * F_coarslope(ic[0], ic[1], ic[2], you1) +
                       0.5 * x1 * x1 * F_coarcurva(ic[0], ic[1], ic[2], you1);
        Real update2 = x2 * F_coarslope(ic[0], ic[1], ic[2], you2) +
                       0.5 * x2 * x2 * F_coarcurva(ic[0], ic[1], ic[2], you2);
        Real update3 = x1 * x2 * F_coarmixed(ic[0], ic[1], ic[2], 0);
        F_fPhiStar(r0 + d[0], r1 + d[1], r2 + d[2], *ivar) = aa + update1 + update2 + update3;
      }
}

// LevelFluxRegisterF.ChF:9-44 (INCREMENTFINE): cFine[i/nRef] += scale * fine[i].
void incrementfine_(FAB(fine), FAB(cFine), BOX(fineBox), const int* nRef, const Real* scale,
                    const int* srcStart, const int* destStart, const int* ncomp) {
  MKFAB(fine);
  MKFAB(cFine);
  for (int var = 0; var < *ncomp; ++var) {
    int srcComp = *srcStart + var;
    int destComp = *destStart + var;
    for (int k = BLO(fineBox, 2); k <= BHI(fineBox, 2); ++k)
      for (int j = BLO(fineBox, 1); j <= BHI(fineBox, 1); ++j)
        for (int i = BLO(fineBox, 0); i <= BHI(fineBox, 0); ++i) {
          int i0 = fdiv(i, nRef[0]), i1 = fdiv(j, nRef[1]), i2 = fdiv(k, nRef[2]);
          F_cFine(i0, i1, i2, destComp) =
              F_cFine(i0, i1, i2, destComp) + *scale * F_fine(i, j, k, srcComp);
        }
  }
}

}  // extern "C"

// The ChF flop counter is a Fortran COMMON block (BaseTools/CH_Counters.H:23-32,
// defined in BaseTools/CH_CountersF.f); the restatements do not count flops,
// but the reference C++ references the block, so it is defined here.
extern "C" {
struct {
  long long ch_flops;
} ch_timer_ = {0};
}
