// Field-wise hash of every host plan table (ghost lists, face rules, per-chunk
// ghosts, coarse-fine stencils, flux registers, copy items, chunks) of three
// synthetic hierarchies: a regression check that the plan builders produce the
// tables the device solve was verified with.
#include <cstdio>
#include <cstdint>
#include <cstring>
#include "geom.H"
#include "plan.H"
#include "meshrefine.H"
#include "hostpool.H"
using namespace cmg;
struct H {
  uint64_t h = 1469598103934665603ULL;
  void add(const void* p, size_t n) { const unsigned char* c = (const unsigned char*)p; for (size_t i = 0; i < n; ++i) { h ^= c[i]; h *= 1099511628211ULL; } }
  template <class T> void v(const T& x) { add(&x, sizeof(T)); }
};
static void hashLevel(H& h, const LevelPlan& L) {
  for (auto& g : L.gcells) { h.v(g.dst); h.v(g.s1); h.v(g.s2); }
  for (int p = 0; p < 2; ++p) { h.v(L.gcStart[p]); h.v(L.gcExch[p]); h.v(L.gcCF[p]); }
  for (auto& r : L.faceRules) { h.v(r.src); h.v(r.kind); }
  for (int x : L.faceOff) h.v(x);
  for (int c = 0; c < 2; ++c) { for (auto& g : L.chunkGhost[c]) { h.v(g.dst); h.v(g.s1); h.v(g.s2); } for (int x : L.chunkGhostStart[c]) h.v(x); }
  for (auto& e : L.cfCoarse) { h.v(e.cc); for (int k = 0; k < 2; ++k) { h.v(e.d1[k].kind); h.v(e.d1[k].n); h.v(e.d1[k].start); h.v(e.d2[k].kind); h.v(e.d2[k].n); h.v(e.d2[k].start); } h.v(e.mx.kind); h.v(e.mx.n); h.v(e.mx.start); }
  for (auto& f : L.cfFine) { h.v(f.g); h.v(f.pa); h.v(f.pb); h.v(f.x1); h.v(f.x2); h.v(f.coarse); h.v(f.packed); }
  for (double w : L.cfW) h.v(w);
  for (int64_t o : L.cfOff) h.v(o);
  for (auto& c : L.rfCells) { h.v(c.c); h.v(c.nco); h.v(c.nfi); h.v(c.start); h.v(c.fstart); }
  for (auto& t : L.rfCoarse) { h.v(t.hi); h.v(t.lo); h.v(t.bface); h.v(t.dir); h.v(t.sgn); }
  for (auto& g : L.rfFine) { for (int k = 0; k < 4; ++k) { h.v(g.hi[k]); h.v(g.lo[k]); h.v(g.bface[k]); } h.v(g.dir); h.v(g.scale); }
  for (auto& t : L.ghost) { h.v(t.kind); h.v(t.dst); h.v(t.src); h.v(t.dir); h.v(t.side); for (int k = 0; k < 3; ++k) { h.v(t.lo[k]); h.v(t.hi[k]); h.v(t.shift[k]); } }
  for (auto& c : L.toCoarse) { h.v(c.cbox); h.v(c.fbox); for (int k = 0; k < 3; ++k) { h.v(c.lo[k]); h.v(c.hi[k]); } }
  for (auto& c : L.chunksColor[0]) { h.v(c.box); h.v(c.start); }
}
int main() {
  struct Case { int n0, nl; } cases[] = {{32, 3}, {64, 3}, {128, 3}};
  for (auto cs : cases) {
    auto boxes = syntheticHierarchy(cs.n0, cs.nl, 32, 8, 0.75, 20261203, 0.1);
    const int nl = (int)boxes.size();
    std::vector<LevelPlan> amr(nl);
    Box dom(IV(0, 0, 0), IV(cs.n0 - 1, cs.n0 - 1, cs.n0 - 1));
    double dx = 1.0 / cs.n0;
    std::vector<Box> doms(nl, dom);
    std::vector<double> dxs(nl, dx);
    for (int l = 1; l < nl; ++l) {
      doms[l] = doms[l - 1].refine(2);
      dxs[l] = dxs[l - 1] / 2;
    }
    // levels, then level pairs, as items of the host pool (the solver's
    // order), each item looping over its boxes on the same pool
    hostParallel(nl, [&](size_t l) {
      buildLevel(amr[l], Layout(boxes[l]), doms[l], dxs[l], l ? dxs[l - 1] : 0.0, nullptr, nullptr);
      ensureChunkGhosts(amr[l]);
      ensureFaceRules(amr[l]);
    });
    hostParallel(nl - 1, [&](size_t i) {
      const int l = (int)i + 1;
      buildQuadCF(amr[l], amr[l - 1]);
      buildCoarseFine(amr[l], amr[l - 1]);
      buildReflux(amr[l - 1], amr[l], true);
    });
    H h;
    for (auto& L : amr) hashLevel(h, L);
    printf("n0 %d levels %d hash %016llx\n", cs.n0, nl, (unsigned long long)h.h);
  }
  // one periodic level (64^3 in 64 boxes of 16^3, periodic in x and y) with
  // its multigrid depths and the bottom plan of the deepest
  {
    const bool per[3] = {true, true, false};
    const int bc[6] = {0, 0, 0, 0, 1, 0};
    Box dom(IV(0, 0, 0), IV(63, 63, 63));
    Layout g0(domainSplit(dom, 16, 8));
    H h;
    LevelPlan L0;
    buildLevel(L0, g0, dom, 1.0 / 64, 0.0, bc, per);
    ensureChunkGhosts(L0);
    ensureFaceRules(L0);
    hashLevel(h, L0);
    LevelPlan last;
    int depths = 0;
    for (int c = 2; g0.coarsenable(c * 2); c *= 2, ++depths) {
      LevelPlan M;
      buildLevel(M, g0.coarsen(c), dom.coarsen(c), c / 64.0, 0.0, bc, per);
      ensureChunkGhosts(M);
      ensureFaceRules(M);
      hashLevel(h, M);
      last = M;
    }
    BottomPlan B;
    buildBottom(depths ? last : L0, B);
    h.v(B.nv);
    h.v(B.ng);
    for (int x : B.fab) h.v(x);
    for (int x : B.nb) h.v(x);
    for (int c = 0; c < 2; ++c)
      for (int x : B.color[c]) h.v(x);
    for (int x : B.boxStart) h.v(x);
    for (int x : B.gsrc) h.v(x);
    for (int x : B.gkind) h.v(x);
    for (int x : B.nbv) h.v(x);
    printf("periodic64 depths %d hash %016llx\n", depths, (unsigned long long)h.h);
  }
  return 0;
}
