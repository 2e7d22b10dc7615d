// Plan construction.  Each builder cites the reference code whose data it
// reproduces; the kernels then apply these tables without any geometry logic.
#include "plan.H"

#include "hostpool.H"

#include <atomic>
#include <exception>
#include <thread>
#include <algorithm>
#include <map>
#include <stdexcept>
#include <unordered_map>

namespace cmg {

namespace {

void chunkCounts(std::vector<Chunk>& out, int box, int64_t n) {
  for (int64_t s = 0; s < n; s += CHUNK) out.push_back(Chunk{box, (int)s});
}

// Fine cell set on the face (d, side) of box b: the ghost layer inside the
// domain minus every box of the level (CFIVS / CFStencil definitions,
// AMRTools/CFIVS.cpp:330-390, AMRTools/CFStencil.cpp:240-326).
bool faceCFSet(const LevelPlan& L, const Box& b, int d, int side, CellSet& out) {
  Box edge = b.adjCell(d, side, 1) & L.domain;
  if (edge.empty()) return false;
  std::vector<int> hits;
  L.index.query(L.grids.boxes, edge, hits);
  // The boxes of a level are disjoint: the layer is covered (no cell set
  // needed) when their overlaps with it add up to its size.
  int64_t covered = 0;
  for (int k : hits) covered += (L.grids[k] & edge).numPts();
  if (covered == edge.numPts()) return false;
  out.define(edge, true);
  for (int k : hits) out.subtract(L.grids[k]);
  return !out.empty();
}

// Greedy cover of a cell set by disjoint boxes: from the first remaining cell
// (x-fastest order) extend along x, then y, then z while every cell is in the
// set.  Used for coarse-fine faces that are not a single box; the per-cell
// formula does not depend on the grouping.
std::vector<Box> coverByBoxes(const CellSet& s) {
  CellSet left = s;
  std::vector<Box> out;
  for (const IV& p : s.cells()) {
    if (!left.contains(p)) continue;
    Box b(p, p);
    while (left.contains(IV(b.hi[0] + 1, p[1], p[2]))) b.hi[0]++;
    for (;;) {
      Box nb = b;
      nb.hi[1]++;
      Box row(IV(b.lo[0], nb.hi[1], b.lo[2]), IV(b.hi[0], nb.hi[1], b.hi[2]));
      if (!left.containsBox(row)) break;
      b = nb;
    }
    for (;;) {
      Box nb = b;
      nb.hi[2]++;
      Box slab(IV(b.lo[0], b.lo[1], nb.hi[2]), IV(b.hi[0], b.hi[1], nb.hi[2]));
      if (!left.containsBox(slab)) break;
      b = nb;
    }
    left.subtract(b);
    out.push_back(b);
  }
  return out;
}

}  // namespace

// Index of a face-ghost cell g of box b in its face table, or -1 when g is
// not a face ghost (inside the box, or outside in more than one direction).
static int64_t faceSlot(const LevelPlan& L, size_t b, const IV& g, int& dir, int& side) {
  const Box& bx = L.grids[b];
  int n = 0;
  for (int d = 0; d < 3; ++d) {
    if (g[d] < bx.lo[d]) dir = d, side = -1, ++n;
    else if (g[d] > bx.hi[d]) dir = d, side = 1, ++n;
  }
  if (n != 1 || g[dir] != (side < 0 ? bx.lo[dir] - 1 : bx.hi[dir] + 1)) return -1;
  const int t0 = dir == 0 ? 1 : 0, t1 = dir == 2 ? 1 : 2;
  return L.faceOff[6 * b + 2 * dir + (side > 0)] + (g[t0] - bx.lo[t0]) +
         (int64_t)bx.size(t0) * (g[t1] - bx.lo[t1]);
}

// Runs fn(i) for every i in [0, n) on the host thread pool; the items must
// write disjoint data.
template <class F>
void parallelItems(size_t n, F fn) {
  hostParallel(n, [&](size_t i) { fn(i); });
}

void buildDeferred(LevelPlan& L);
void buildChunkGhosts(LevelPlan& L);

bool ensureFaceRules(LevelPlan& L) {
  if (!L.faceOff.empty() || L.grids.size() == 0) return false;
  buildFaceRules(L);
  return true;
}

// Rules of every face-ghost cell from the level's ghost tasks (the fill with
// coarse-fine values that precedes each relaxation pass).
void buildFaceRules(LevelPlan& L) {
  L.faceOff.assign(6 * L.grids.size() + 1, 0);
  int64_t off = 0;
  for (size_t b = 0; b < L.grids.size(); ++b) {
    const Box& bx = L.grids[b];
    for (int d = 0; d < 3; ++d) {
      const int t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
      for (int s = 0; s < 2; ++s) {
        L.faceOff[6 * b + 2 * d + s] = (int)off;
        off += (int64_t)bx.size(t0) * bx.size(t1);
      }
    }
  }
  L.faceOff[6 * L.grids.size()] = (int)off;
  L.faceRules.assign((size_t)off, FaceRule{0, FR_FAB});
  // Boxes write their own slots, and ghost tasks disjoint ghost regions, so
  // both loops run on host threads.
  parallelItems(L.grids.size(), [&](size_t b) {
    const Box& bx = L.grids[b];
    for (int d = 0; d < 3; ++d) {
      const int t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
      for (int s = 0; s < 2; ++s)
        for (int v = bx.lo[t1]; v <= bx.hi[t1]; ++v)
          for (int u = bx.lo[t0]; u <= bx.hi[t0]; ++u) {
            IV g;
            g[d] = s ? bx.hi[d] + 1 : bx.lo[d] - 1;
            g[t0] = u;
            g[t1] = v;
            int dd, ss;
            L.faceRules[faceSlot(L, b, g, dd, ss)].src = (int)cellOf(L, (int)b, g);
          }
    }
  });
  parallelItems(L.ghost.size(), [&](size_t ti) {
    const GhostTask& t = L.ghost[ti];
    for (int k = t.lo[2]; k <= t.hi[2]; ++k)
      for (int j = t.lo[1]; j <= t.hi[1]; ++j)
        for (int i = t.lo[0]; i <= t.hi[0]; ++i) {
          IV g(i, j, k);
          int d = 0, side = 0;
          int64_t q = faceSlot(L, t.dst, g, d, side);
          if (q < 0) continue;
          FaceRule& r = L.faceRules[q];
          if (t.kind == G_COPY) {
            r = FaceRule{(int)cellOf(L, t.src, g - IV(t.shift[0], t.shift[1], t.shift[2])), FR_COPY};
          } else if (t.kind == G_BC) {
            r = FaceRule{0, FR_BC};
          } else if (t.kind == G_NEU) {
            r = FaceRule{0, FR_NEU};
          } else if (t.kind == G_CFLIN) {
            r = FaceRule{0, FR_CFLIN};
          } else if (t.kind == G_CFQUAD) {
            int e[3] = {0, 0, 0};
            e[t.dir] = -2 * t.side;
            r = FaceRule{(int)cellOf(L, t.dst, IV(i + e[0], j + e[1], k + e[2])), FR_CFQUAD};
          }
        }
  });
}

// The colour-1 cells ((i+j+k) odd) with at least one face ghost filled by an
// exchange copy, per box in x-fastest order (DeferredCell).
void buildDeferred(LevelPlan& L) {
  std::vector<std::vector<DeferredCell>> per(L.grids.size());
  parallelItems(L.grids.size(), [&](size_t b) {
    const Box& bx = L.grids[b];
    const int nx = bx.size(0), ny = bx.size(1);
    // Only face cells can qualify: walk the six faces (cells on an edge come
    // up on two or three of them, hence the sort and unique below).
    std::vector<int> qs;
    for (int d = 0; d < 3; ++d) {
      const int t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
      for (int s = 0; s < 2; ++s) {
        const FaceRule* r = &L.faceRules[L.faceOff[6 * b + 2 * d + s]];
        for (int v = bx.lo[t1], q = 0; v <= bx.hi[t1]; ++v)
          for (int u = bx.lo[t0]; u <= bx.hi[t0]; ++u, ++q) {
            IV p;
            p[d] = s ? bx.hi[d] : bx.lo[d];
            p[t0] = u;
            p[t1] = v;
            if (((p[0] + p[1] + p[2]) & 1) == 0 || r[q].kind != FR_COPY) continue;
            qs.push_back((p[0] - bx.lo[0]) + nx * ((p[1] - bx.lo[1]) + ny * (p[2] - bx.lo[2])));
          }
      }
    }
    std::sort(qs.begin(), qs.end());
    qs.erase(std::unique(qs.begin(), qs.end()), qs.end());
    for (int q : qs) per[b].push_back(DeferredCell{(int)b, q});
  });
  L.deferred.clear();
  for (auto& v : per) L.deferred.insert(L.deferred.end(), v.begin(), v.end());
}

// Per-chunk face ghosts of the colour passes: for colour c, the ghost cells
// of parity 1 - c that the cells of each colour-c chunk read, each as the
// ghost-fill entry (GhostCell) of its face rule, grouped by chunk.  Every face
// ghost is read by exactly one cell (the valid cell next to it), so the
// groups are disjoint; FR_FAB faces have no fill and no entry.
void buildChunkGhosts(LevelPlan& L) {
  const size_t nb = L.grids.size();
  for (int c = 0; c < 2; ++c) {
    std::vector<std::vector<std::pair<int, GhostCell>>> per(nb);
    parallelItems(nb, [&](size_t b) {
      const Box& bx = L.grids[b];
      const int half = (bx.size(0) + 1) / 2, ny = bx.size(1);
      std::vector<std::pair<int, GhostCell>>& out = per[b];
      for (int d = 0; d < 3; ++d) {
        const int t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
        for (int s = 0; s < 2; ++s) {
          const FaceRule* r = &L.faceRules[L.faceOff[6 * b + 2 * d + s]];
          for (int v = bx.lo[t1], q = 0; v <= bx.hi[t1]; ++v)
            for (int u = bx.lo[t0]; u <= bx.hi[t0]; ++u, ++q) {
              IV p;
              p[d] = s ? bx.hi[d] : bx.lo[d];
              p[t0] = u;
              p[t1] = v;
              if (((p[0] + p[1] + p[2]) & 1) != c || r[q].kind == FR_FAB) continue;
              IV g = p;
              g[d] += s ? 1 : -1;
              const int dst = (int)cellOf(L, (int)b, g), adj = (int)cellOf(L, (int)b, p);
              GhostCell e{dst, 0, 0};
              switch (r[q].kind) {
                case FR_COPY: e.s1 = r[q].src, e.s2 = -1; break;
                case FR_BC: e.s1 = adj, e.s2 = -2; break;
                case FR_NEU: e.s1 = adj, e.s2 = -1; break;
                case FR_CFLIN: e.s1 = adj, e.s2 = -3; break;
                default: e.s1 = adj, e.s2 = r[q].src; break;  // FR_CFQUAD
              }
              const int par = (bx.lo[0] + p[1] + p[2] + c) & 1;
              const int idx = ((p[1] - bx.lo[1]) + ny * (p[2] - bx.lo[2])) * half + (p[0] - bx.lo[0] - par) / 2;
              out.push_back({idx, e});
            }
        }
      }
      std::stable_sort(out.begin(), out.end(),
                       [](const std::pair<int, GhostCell>& x, const std::pair<int, GhostCell>& y) {
                         return x.first / CHUNK < y.first / CHUNK;
                       });
    });
    std::vector<GhostCell>& cells = L.chunkGhost[c];
    std::vector<int>& start = L.chunkGhostStart[c];
    cells.clear();
    start.assign(1, 0);
    for (size_t b = 0; b < nb; ++b) {
      const Box& bx = L.grids[b];
      const int64_t n = (int64_t)bx.size(1) * bx.size(2) * ((bx.size(0) + 1) / 2);
      size_t at = 0;
      for (int64_t ch = 0; ch * CHUNK < n; ++ch) {
        while (at < per[b].size() && per[b][at].first / CHUNK == ch) cells.push_back(per[b][at++].second);
        start.push_back((int)cells.size());
      }
      if (at != per[b].size()) throw std::logic_error("cmg: chunk ghost outside its box");
    }
    if (start.size() != L.chunksColor[c].size() + 1) throw std::logic_error("cmg: chunk ghost count mismatch");
  }
}

std::vector<int> blockTasks(const std::vector<int>& start) {
  std::vector<int> bt;
  if (start.size() < 2) return bt;
  const int ntask = (int)start.size() - 1, ncell = start.back();
  int t = 0;
  for (int64_t c = 0; c < ncell; c += GHOST_PER_BLOCK) {
    while (start[t + 1] <= c) ++t;
    bt.push_back(t);
  }
  bt.push_back(ntask - 1);
  return bt;
}

void buildLevel(LevelPlan& L, const Layout& grids, const Box& domain, double dx, double dxCrse, const int* bc,
                const bool* periodic) {
  L.grids = grids;
  L.index.build(L.grids.boxes);
  L.domain = domain;
  L.dx = dx;
  L.dxCrse = dxCrse;
  L.boxes.clear();
  int64_t off = 0;
  for (size_t b = 0; b < grids.size(); ++b) {
    const Box& bx = grids[b];
    BoxDesc d;
    for (int k = 0; k < 3; ++k) {
      d.lo[k] = bx.lo[k];
      d.hi[k] = bx.hi[k];
    }
    d.px = (bx.size(0) + 3) & ~1;  // nx + 2 rounded up to even
    d.py = bx.size(1) + 2;
    d.off = off;
    d.half = (int64_t)d.px * d.py * (bx.size(2) + 2) / 2;
    {
      // dividends: cell numbers of the box (plus the 256 threads of a
      // chunk's tail) and row numbers (nx ... cells per row)
      const int64_t nx = bx.size(0), ny = bx.size(1), nz = bx.size(2), half = (nx + 1) / 2;
      const int64_t qmax = nx * ny * nz + CHUNK;
      d.mNx = divMagic((int)nx, qmax);
      d.mHalf = divMagic((int)half, qmax);
      d.mNy = divMagic((int)ny, qmax);
    }
    off += 2 * d.half;
    L.boxes.push_back(d);
  }
  L.nelem = off;

  // Exchange items (Copier::exchangeDefine + trimEdges) and the physical
  // boundary faces (face ghosts outside the domain): homogeneous Dirichlet, or
  // homogeneous Neumann where bc[2 * dir + (side > 0)] is 1.
  L.ghost.clear();
  for (const Motion& m : exchangePlan(grids, domain, periodic)) {
    GhostTask t{G_COPY, m.to, m.from, 0, 0, {}, {}, {}};
    for (int k = 0; k < 3; ++k) t.shift[k] = m.toRegion.lo[k] - m.fromRegion.lo[k];
    for (int k = 0; k < 3; ++k) {
      t.lo[k] = m.toRegion.lo[k];
      t.hi[k] = m.toRegion.hi[k];
    }
    L.ghost.push_back(t);
  }
  for (size_t b = 0; b < grids.size(); ++b) {
    if (domain.contains(grids[b].grow(1))) continue;
    for (int d = 0; d < 3; ++d)
      for (int side = -1; side <= 1; side += 2) {
        if (periodic && periodic[d]) continue;  // filled from the periodic image
        Box g = grids[b].adjCell(d, side, 1);
        if (domain.contains(g)) continue;
        GhostTask t{bc && bc[2 * d + (side > 0)] == 1 ? G_NEU : G_BC, (int)b, (int)b, d, side, {}, {}, {}};
        for (int k = 0; k < 3; ++k) {
          t.lo[k] = g.lo[k];
          t.hi[k] = g.hi[k];
        }
        L.ghost.push_back(t);
      }
  }
  L.nExchBC = (int)L.ghost.size();
  // Homogeneous coarse-fine faces (AMRPoissonOp::homogeneousCFInterp,
  // AMRElliptic/AMRPoissonOp.cpp:1598-1671).  A packed face is one box; an
  // unpacked face is emitted cell by cell with the same formula.
  if (dxCrse > 0) {
    // each box's faces on a host thread, appended in box order
    std::vector<std::vector<GhostTask>> perBox(grids.size());
    parallelItems(grids.size(), [&](size_t b) {
      for (int d = 0; d < 3; ++d)
        for (int side = -1; side <= 1; side += 2) {
          CellSet s;
          if (!faceCFSet(L, grids[b], d, side, s)) continue;
          int kind = (grids[b].size(d) == 1) ? G_CFLIN : G_CFQUAD;
          Box mb = s.minBox();
          std::vector<Box> regions;
          if (mb.numPts() == s.numPts())
            regions.push_back(mb);
          else
            regions = coverByBoxes(s);
          for (const Box& r : regions) {
            GhostTask t{kind, (int)b, (int)b, d, side, {}, {}};
            for (int k = 0; k < 3; ++k) {
              t.lo[k] = r.lo[k];
              t.hi[k] = r.hi[k];
            }
            perBox[b].push_back(t);
          }
        }
    });
    for (const auto& v : perBox) L.ghost.insert(L.ghost.end(), v.begin(), v.end());
  }

  L.ghostStart.assign(1, 0);
  for (const GhostTask& t : L.ghost) {
    int64_t c = (int64_t)(t.hi[0] - t.lo[0] + 1) * (t.hi[1] - t.lo[1] + 1) * (t.hi[2] - t.lo[2] + 1);
    L.ghostStart.push_back(L.ghostStart.back() + (int)c);
  }
  L.ghostBlock = blockTasks(L.ghostStart);
  L.faceRules.clear();
  L.faceOff.clear();
  if (grids.numCells() <= kFaceRulesEagerCells) buildFaceRules(L);
  if (L.nelem >= ((int64_t)1 << 31)) throw std::runtime_error("cmg: level too large for 32-bit ghost indices");
  // Flat lists: per parity the exchange and boundary tasks, then the
  // coarse-fine ones, each task's cells of that parity in k, j, i order.
  // Counts first, then every task fills its own range on host threads.
  const size_t ntask = L.ghost.size();
  auto parityCount = [](const GhostTask& t, int par) {
    int64_t n = 0;
    const int nx = t.hi[0] - t.lo[0] + 1;
    for (int k = t.lo[2]; k <= t.hi[2]; ++k)
      for (int j = t.lo[1]; j <= t.hi[1]; ++j) {
        const int first = ((t.lo[0] + j + k) & 1) == par ? 0 : 1;  // offset of the row's first cell of parity par
        n += nx > first ? (nx - first + 1) / 2 : 0;
      }
    return n;
  };
  std::vector<int64_t> start(2 * ntask + 1, 0), count(2 * ntask, 0);
  parallelItems(2 * ntask, [&](size_t q) { count[q] = parityCount(L.ghost[q % ntask], (int)(q / ntask)); });
  {
    int64_t pos = 0;
    for (int par = 0; par < 2; ++par) {
      L.gcStart[par] = (int)pos;
      for (size_t t = 0; t < ntask; ++t) {
        if (t == (size_t)L.nExchBC) L.gcExch[par] = (int)(pos - L.gcStart[par]);
        start[par * ntask + t] = pos;
        pos += count[par * ntask + t];
      }
      if (ntask <= (size_t)L.nExchBC) L.gcExch[par] = (int)(pos - L.gcStart[par]);
      L.gcCF[par] = (int)(pos - L.gcStart[par] - L.gcExch[par]);
    }
    start[2 * ntask] = pos;
    L.gcells.resize((size_t)pos);  // every entry is written below
  }
  // Along a row the cells of one parity are two apart in x, so each of their
  // indices (and their sources', shifted by a fixed offset) is the previous
  // one plus 1 (cellIndex: same colour half, colour slot + 1).
  auto emit = [&](const GhostTask& t, int par, int64_t at) {
    const BoxDesc& db = L.boxes[t.dst];
    int e[3] = {0, 0, 0};
    if (t.kind != G_COPY) e[t.dir] = -t.side;
    const int s2fixed = t.kind == G_NEU ? -1 : t.kind == G_BC ? -2 : t.kind == G_CFLIN ? -3 : 0;
    for (int k = t.lo[2]; k <= t.hi[2]; ++k)
      for (int j = t.lo[1]; j <= t.hi[1]; ++j) {
        const int i0 = t.lo[0] + ((t.lo[0] + j + k + par) & 1);  // the row's first cell of parity par
        if (i0 > t.hi[0]) continue;
        const int n = (t.hi[0] - i0) / 2 + 1;
        const int d0 = (int)cellIndex(db, i0, j, k);
        int a0, b0 = -1, bstep = 0;
        if (t.kind == G_COPY) {
          a0 = (int)cellIndex(L.boxes[t.src], i0 - t.shift[0], j - t.shift[1], k - t.shift[2]);
        } else {
          a0 = (int)cellIndex(db, i0 + e[0], j + e[1], k + e[2]);
          if (s2fixed) {
            b0 = s2fixed;
          } else {
            b0 = (int)cellIndex(db, i0 + 2 * e[0], j + 2 * e[1], k + 2 * e[2]);
            bstep = 1;
          }
        }
        GhostCell* g = &L.gcells[at];
        for (int m = 0; m < n; ++m) {
          g[m].dst = d0 + m;
          g[m].s1 = a0 + m;
          g[m].s2 = b0 + bstep * m;
        }
        at += n;
      }
    if (at != start[par * ntask + (&t - L.ghost.data()) + 1] && (size_t)(&t - L.ghost.data()) + 1 < ntask)
      throw std::logic_error("cmg: ghost-cell count mismatch");
  };
  parallelItems(2 * ntask, [&](size_t q) {
    const int par = (int)(q / ntask);
    const size_t t = q % ntask;
    emit(L.ghost[t], par, start[q]);
  });
  L.slotStart.assign(1, 0);
  for (const GhostTask& t : L.ghost)
    L.slotStart.push_back(L.slotStart.back() + (int)colourSlots(t.lo, t.hi, parityAxis(t.lo, t.hi)));
  L.slotBlock = blockTasks(L.slotStart);

  L.chunksAll.clear();
  L.chunksColor[0].clear();
  L.chunksColor[1].clear();
  for (size_t b = 0; b < grids.size(); ++b) {
    const Box& bx = grids[b];
    chunkCounts(L.chunksAll, (int)b, bx.numPts());
    int64_t rows = (int64_t)bx.size(1) * bx.size(2);
    int64_t half = (bx.size(0) + 1) / 2;
    chunkCounts(L.chunksColor[0], (int)b, rows * half);
    chunkCounts(L.chunksColor[1], (int)b, rows * half);
  }
  // The prefill variant's per-chunk lists are built when the relaxation
  // tuner asks for them (ensureChunkGhosts).
}

bool ensureChunkGhosts(LevelPlan& L) {
  // Only where that variant can win (latency-bound levels): on larger levels
  // the separate fill is as fast, and the lists would add as much host work
  // and memory as the fill lists.
  if (!L.chunkGhostStart[0].empty() || L.grids.size() == 0 || L.grids.numCells() > kPrefillMaxCells) return false;
  ensureFaceRules(L);  // the per-chunk lists are made from the face rules
  buildChunkGhosts(L);
  return true;
}

int ownerOf(const LevelPlan& L, const IV& p) {
  for (size_t b = 0; b < L.grids.size(); ++b) {
    const Box& bx = L.grids[b];
    if (bx.lo[0] > p[0]) break;
    if (bx.contains(p)) return (int)b;
  }
  return -1;
}

// Cell -> box lookup through a bucket grid whose bucket edge is the largest
// power of two (<= 16) that every box corner is aligned to, so each bucket
// lies in at most one box.
struct OwnerIndex {
  const LevelPlan* L;
  int B = 1, sh = 0;  // block edge B = 2^sh
  IV org, n;
  std::vector<int> own;
  explicit OwnerIndex(const LevelPlan& lp) : L(&lp) {
    B = 16;
    for (const Box& b : lp.grids.boxes)
      for (int d = 0; d < 3; ++d)
        while (B > 1 && ((b.lo[d] % B) != 0 || ((b.hi[d] + 1) % B) != 0)) B /= 2;
    while ((1 << sh) < B) ++sh;
    Box dom = lp.domain;
    for (int d = 0; d < 3; ++d) {
      org[d] = floordiv(dom.lo[d], B);
      n[d] = floordiv(dom.hi[d], B) - org[d] + 1;
    }
    own.assign((size_t)n[0] * n[1] * n[2], -1);
    for (size_t k = 0; k < lp.grids.size(); ++k) {
      Box c = lp.grids[k].coarsen(B);
      for (int z = c.lo[2]; z <= c.hi[2]; ++z)
        for (int y = c.lo[1]; y <= c.hi[1]; ++y)
          for (int x = c.lo[0]; x <= c.hi[0]; ++x) own[slot(IV(x, y, z))] = (int)k;
    }
  }
  size_t slot(const IV& q) const {
    return (size_t)(q[0] - org[0]) + (size_t)n[0] * ((size_t)(q[1] - org[1]) + (size_t)n[1] * (q[2] - org[2]));
  }
  // floor(p / B) by an arithmetic shift (also for negative p)
  int find(const IV& p) const {
    IV q(p[0] >> sh, p[1] >> sh, p[2] >> sh);
    for (int d = 0; d < 3; ++d)
      if (q[d] < org[d] || q[d] >= org[d] + n[d]) return -1;
    return own[slot(q)];
  }
  int64_t cell(const IV& p) const {
    int b = find(p);
    if (b < 0) throw std::runtime_error("cmg: coarse cell outside the coarse level");
    return cellOf(*L, b, p);
  }
};

}  // namespace cmg

namespace cmg {

namespace {

// Merged (cell, weight) list with the reference's accumulate semantics
// (AMRTools/DerivStencil.cpp:79-105: equal cells add their weights).
struct Sten {
  bool defined = false;
  std::vector<IV> iv;
  std::vector<double> w;
  void acc(const IV& p, double wt) {
    defined = true;
    for (size_t i = 0; i < iv.size(); ++i)
      if (iv[i] == p) {
        w[i] += wt;
        return;
      }
    iv.push_back(p);
    w.push_back(wt);
  }
};

struct CoarseStencils {
  bool drop = false;
  Sten mixed, first[2], second[2];
};

// QuadCFStencil::buildStencils (AMRTools/QuadCFStencil.cpp:662-920) for one
// irregular coarse cell.  t[0] < t[1] are the tangential directions.
void buildIrregular(const IV& iv, const int t[2], const CellSet& good, CoarseStencils& cs) {
  // Mixed derivative: average of the one-sided 2x2 quadrant stencils that lie
  // in the good set, tested in the reference's order.  Each quadrant with low
  // corner L carries -1 at L and L+e1+e2, +1 at L+e1 and L+e2.
  const IV e1 = IV::basis(t[0]), e2 = IV::basis(t[1]);
  const IV los[4] = {iv - e1, iv, iv - e2, iv - e1 - e2};
  int nmixed = 0;
  for (int q = 0; q < 4; ++q) {
    Box qb(los[q], los[q] + e1 + e2);
    if (!good.containsBox(qb)) continue;
    ++nmixed;
    for (int a2 = 0; a2 < 2; ++a2)
      for (int a1 = 0; a1 < 2; ++a1) {
        IV p = los[q];
        p[t[0]] += a1;
        p[t[1]] += a2;
        cs.mixed.acc(p, (a1 == a2) ? -1.0 : 1.0);
      }
  }
  if (nmixed > 0) {
    double rn = nmixed;
    for (double& w : cs.mixed.w) w /= rn;
  }
  cs.drop = (nmixed == 0);
}

void buildIrregularDir(const IV& iv, int ivec, int dir, const CellSet& good, CoarseStencils& cs) {
  if (cs.drop) return;
  const IV e = IV::basis(dir);
  Box bsten = Box(iv, iv).grow(dir, 1);
  Sten& s2 = cs.second[ivec];
  Sten& s1 = cs.first[ivec];
  if (good.containsBox(bsten)) {
    s2.acc(iv - e, 1.0);
    s2.acc(iv, -2.0);
    s2.acc(iv + e, 1.0);
    s1.acc(iv - e, -0.5);
    s1.acc(iv, 0.0);
    s1.acc(iv + e, 0.5);
    return;
  }
  Box bshift = bsten.shift(dir, 1);
  if (good.containsBox(bshift)) {
    s2.acc(iv, 1.0);
    s2.acc(iv + e, -2.0);
    s2.acc(iv + e + e, 1.0);
    s1.acc(iv, -3.0 / 2.0);
    s1.acc(iv + e, 4.0 / 2.0);
    s1.acc(iv + e + e, -1.0 / 2.0);
    return;
  }
  bshift = bshift.shift(dir, -2);
  if (good.containsBox(bshift)) {
    s2.acc(iv - e - e, 1.0);
    s2.acc(iv - e, -2.0);
    s2.acc(iv, 1.0);
    s1.acc(iv - e - e, 1.0 / 2.0);
    s1.acc(iv - e, -4.0 / 2.0);
    s1.acc(iv, 3.0 / 2.0);
    return;
  }
  cs.drop = true;
  if (good.contains(iv + e)) {
    s1.acc(iv, -1.0);
    s1.acc(iv + e, 1.0);
  } else if (good.contains(iv - e)) {
    s1.acc(iv - e, -1.0);
    s1.acc(iv, 1.0);
  } else {
    s1.acc(iv, 0.0);
  }
}

}  // namespace

// Tables of one fine box: CFCoarse pool starts relative to its own pool,
// CFFine coarse indices relative to its own CFCoarse list.
struct QuadCFPart {
  std::vector<CFCoarse> coarse;
  std::vector<CFFine> fine;
  std::vector<double> w;
  std::vector<int64_t> off;
};

void buildQuadCFBox(const LevelPlan& F, const LevelPlan& C, const OwnerIndex& owner, const Layout& cfine,
                    const BoxIndex& cfineIndex, size_t fb, QuadCFPart& out) {
  std::vector<int> hits;
  const double dxf = F.dx;
  const double dxc = 2 * dxf;
  auto pushCells = [&](const IV* cells, size_t n, const double* w) {
    int start = (int)out.off.size();
    for (size_t i = 0; i < n; ++i) {
      out.off.push_back(owner.cell(cells[i]));
      out.w.push_back(w ? w[i] : 0.0);
    }
    return start;
  };
  auto pushPool = [&](const std::vector<IV>& cells, const std::vector<double>* w) {
    return pushCells(cells.data(), cells.size(), w ? w->data() : nullptr);
  };
  const Box& fbox = F.grids[fb];
  for (int d = 0; d < 3; ++d) {
    int t[2], it = 0;
    for (int k = 0; k < 3; ++k)
      if (k != d) t[it++] = k;
    for (int side = -1; side <= 1; side += 2) {
      CellSet fineIVS;
      if (!faceCFSet(F, fbox, d, side, fineIVS)) continue;
      // CFStencil::define (AMRTools/CFStencil.cpp:240-326) starts from the
      // face layer as a dense IntVectSet and removes the fine boxes cell by
      // cell, which leaves the set's cached minBox at the whole face layer:
      // the face is "packed" (Fortran PHISTAR / QUADINTERP arithmetic) only
      // when no cell was removed, and its packed box is the face layer.
      // A face partly covered by another fine box takes the C++ form even
      // where its remaining cells form a box.
      const Box faceLayer = fbox.adjCell(d, side, 1) & F.domain;
      Box packedBox = faceLayer;
      bool packed = (faceLayer.numPts() == fineIVS.numPts());
      CellSet base = fineIVS.coarsen(2);
      base.intersect(C.domain);
      // Good set: coarse cells of the widened face slab that are valid on
      // the coarse level and not under the fine level
      // (QuadCFStencil::define, AMRTools/QuadCFStencil.cpp:500-660).
      Box cgrid = fbox.coarsen(2);
      Box g2 = cgrid.adjCell(d, side, 1), g1 = g2;
      for (int k = 0; k < 2; ++k) {
        g2 = g2.grow(t[k], 2);
        g1 = g1.grow(t[k], 1);
      }
      g2 = g2 & C.domain;
      g1 = g1 & C.domain;
      CellSet good(g2, false);
      C.index.query(C.grids.boxes, g2, hits);
      for (int k : hits) good.set(C.grids[k], true);
      cfineIndex.query(cfine.boxes, g2, hits);
      for (int k : hits) good.subtract(cfine[k]);
      CellSet standard = good;
      standard.intersect(g1);
      standard = standard.erode(t[0]).erode(t[1]);
      // Irregular stencils for base cells outside the standard set.
      // CFCoarse entry of each base cell (dense over the base set's box)
      std::vector<int> coarseIndex((size_t)base.dom.numPts(), -1);
      std::vector<IV> baseCells = base.cells();
      std::vector<CoarseStencils> irr(baseCells.size());
      for (size_t i = 0; i < baseCells.size(); ++i)
        if (!standard.contains(baseCells[i])) buildIrregular(baseCells[i], t, good, irr[i]);
      for (int ivec = 0; ivec < 2; ++ivec)
        for (size_t i = 0; i < baseCells.size(); ++i)
          if (!standard.contains(baseCells[i])) buildIrregularDir(baseCells[i], ivec, t[ivec], good, irr[i]);
      for (size_t i = 0; i < baseCells.size(); ++i) {
        const IV& c = baseCells[i];
        CFCoarse e;
        e.cc = owner.cell(c);
        if (standard.contains(c)) {
          for (int k = 0; k < 2; ++k) {
            IV ek = IV::basis(t[k]);
            const IV d1[2] = {c - ek, c + ek}, d2[3] = {c - ek, c + ek, c};
            e.d1[k] = CFDeriv{1, 2, pushCells(d1, 2, nullptr)};
            e.d2[k] = CFDeriv{1, 3, pushCells(d2, 3, nullptr)};
          }
          // computeMixedDerivative: basex = e(t[0]), basey = e(t[1]).
          IV bx = IV::basis(t[0]), by = IV::basis(t[1]);
          const IV mx[4] = {c + bx + by, c - bx + by, c + bx - by, c - bx - by};
          e.mx = CFDeriv{1, 4, pushCells(mx, 4, nullptr)};
        } else {
          const CoarseStencils& cs = irr[i];
          for (int k = 0; k < 2; ++k) {
            e.d1[k] = CFDeriv{2, (int)cs.first[k].iv.size(), pushPool(cs.first[k].iv, &cs.first[k].w)};
            if (cs.drop)
              e.d2[k] = CFDeriv{0, 0, 0};
            else
              e.d2[k] = CFDeriv{2, (int)cs.second[k].iv.size(), pushPool(cs.second[k].iv, &cs.second[k].w)};
          }
          if (cs.drop)
            e.mx = CFDeriv{0, 0, 0};
          else
            e.mx = CFDeriv{2, (int)cs.mixed.iv.size(), pushPool(cs.mixed.iv, &cs.mixed.w)};
        }
        coarseIndex[base.at(c)] = (int)out.coarse.size();
        out.coarse.push_back(e);
      }
      // Fine ghost cells.  Packed faces follow the Fortran PHISTAR index
      // shift (QuadCFInterp.cpp:680-712, QuadCFInterpF.ChF:50-126).
      IV shift = packedBox.lo;
      shift[d] += side;
      for (const IV& f : fineIVS.cells()) {
        IV c(floordiv(f[0], 2), floordiv(f[1], 2), floordiv(f[2], 2));
        CFFine ff;
        ff.g = cellOf(F, (int)fb, f);
        ff.pb = cellOf(F, (int)fb, f - IV::basis(d, side));
        ff.pa = cellOf(F, (int)fb, f - IV::basis(d, 2 * side));
        ff.coarse = coarseIndex[base.at(c)];
        if (ff.coarse < 0) throw std::runtime_error("cmg: fine ghost without coarse stencil");
        ff.packed = packed ? 1 : 0;
        double xs[2];
        for (int k = 0; k < 2; ++k) {
          int you = t[k];
          if (packed) {
            int ir = f[you] - shift[you];
            int ic = ir / 2;
            double xf = (ir + 0.5) * dxf;
            double xc = (ic + 0.5) * dxc;
            xs[k] = xf - xc;
          } else {
            double xf = (f[you] + 0.5) * dxf;
            double xc = (c[you] + 0.5) * dxc;
            xs[k] = xf - xc;
          }
        }
        ff.x1 = xs[0];
        ff.x2 = xs[1];
        out.fine.push_back(ff);
      }
    }
  }
}

// The fine boxes are independent: built on host threads, then concatenated in
// box order with their pool and coarse-entry indices shifted (the same tables
// as one pass over the boxes).
void buildQuadCF(LevelPlan& F, const LevelPlan& C) {
  F.cfCoarse.clear();
  F.cfFine.clear();
  F.cfW.clear();
  F.cfOff.clear();
  OwnerIndex owner(C);
  Layout cfine = F.grids.coarsen(2);
  BoxIndex cfineIndex;
  cfineIndex.build(cfine.boxes);
  const size_t nb = F.grids.size();
  std::vector<QuadCFPart> parts(nb);
  parallelItems(nb, [&](size_t fb) { buildQuadCFBox(F, C, owner, cfine, cfineIndex, fb, parts[fb]); });
  // Concatenation: every part's ranges from prefix sums, then the parts
  // copied (and their indices shifted) on host threads.
  std::vector<size_t> c0(nb + 1, 0), f0(nb + 1, 0), p0(nb + 1, 0);
  for (size_t fb = 0; fb < nb; ++fb) {
    c0[fb + 1] = c0[fb] + parts[fb].coarse.size();
    f0[fb + 1] = f0[fb] + parts[fb].fine.size();
    p0[fb + 1] = p0[fb] + parts[fb].off.size();
  }
  F.cfCoarse.resize(c0[nb]);
  F.cfFine.resize(f0[nb]);
  F.cfW.resize(p0[nb]);
  F.cfOff.resize(p0[nb]);
  parallelItems(nb, [&](size_t fb) {
    QuadCFPart& p = parts[fb];
    const int coarseBase = (int)c0[fb], poolBase = (int)p0[fb];
    for (size_t i = 0; i < p.coarse.size(); ++i) {
      CFCoarse e = p.coarse[i];
      for (int k = 0; k < 2; ++k) {
        if (e.d1[k].kind) e.d1[k].start += poolBase;
        if (e.d2[k].kind) e.d2[k].start += poolBase;
      }
      if (e.mx.kind) e.mx.start += poolBase;
      F.cfCoarse[c0[fb] + i] = e;
    }
    for (size_t i = 0; i < p.fine.size(); ++i) {
      CFFine f = p.fine[i];
      f.coarse += coarseBase;
      F.cfFine[f0[fb] + i] = f;
    }
    std::copy(p.w.begin(), p.w.end(), F.cfW.begin() + p0[fb]);
    std::copy(p.off.begin(), p.off.end(), F.cfOff.begin() + p0[fb]);
    p = QuadCFPart();
  });
}

}  // namespace cmg

namespace cmg {

void buildCoarseFine(LevelPlan& F, LevelPlan& C) {
  // Copier from the coarsened fine layout to the coarse layout
  // (AMRPoissonOp::buildCopier, AMRElliptic/AMRPoissonOp.cpp:474-483); the
  // same items drive restriction, prolongation and zeroCovered.
  Layout cfine = F.grids.coarsen(2);
  F.toCoarse.clear();
  F.toCoarseChunksC.clear();
  F.toCoarseChunksF.clear();
  C.zeroCovered.clear();
  for (const Motion& m : copyPlan(cfine, C.grids)) {
    CoarseFineItem it;
    it.cbox = m.to;
    it.fbox = m.from;
    for (int k = 0; k < 3; ++k) {
      it.lo[k] = m.toRegion.lo[k];
      it.hi[k] = m.toRegion.hi[k];
    }
    int idx = (int)F.toCoarse.size();
    F.toCoarse.push_back(it);
    chunkCounts(F.toCoarseChunksC, idx, m.toRegion.numPts());
    chunkCounts(F.toCoarseChunksF, idx, 8 * m.toRegion.numPts());
    GhostTask z{G_ZERO, m.to, m.to, 0, 0, {}, {}};
    for (int k = 0; k < 3; ++k) {
      z.lo[k] = m.toRegion.lo[k];
      z.hi[k] = m.toRegion.hi[k];
    }
    C.zeroCovered.push_back(z);
  }
  C.zeroStart.assign(1, 0);
  for (const GhostTask& t : C.zeroCovered)
    C.zeroStart.push_back(C.zeroStart.back() +
                          (t.hi[0] - t.lo[0] + 1) * (t.hi[1] - t.lo[1] + 1) * (t.hi[2] - t.lo[2] + 1));
  C.zeroBlock = blockTasks(C.zeroStart);
}

void buildReflux(LevelPlan& C, const LevelPlan& F, bool vc) {
  // LevelFluxRegister::define / incrementCoarse / incrementFine / reflux
  // (AMRTools/LevelFluxRegister.cpp:101-262, 372-586, 649-670) reduced to the
  // uncovered coarse cells they change, with every addition kept in the
  // reference's order.
  C.rfCells.clear();
  C.rfCoarse.clear();
  C.rfFine.clear();
  Layout cfine = F.grids.coarsen(2);
  BoxIndex cfineIndex;
  cfineIndex.build(cfine.boxes);
  // Coarse boxes are independent: each builds its cells with pool starts
  // relative to its own pools on a host thread; the parts are concatenated
  // in box order (the same tables as one pass over the boxes).
  struct Part {
    std::vector<RefluxCell> cells;
    std::vector<RefluxCoarseTerm> co;
    std::vector<RefluxFineGroup> fi;
  };
  std::vector<Part> parts(C.grids.size());
  parallelItems(C.grids.size(), [&](size_t cb) {
    Part& out = parts[cb];
    const Box& cbox = C.grids[cb];
    // coarsened fine boxes next to this coarse box, in fine box order, and
    // the cells of this box they cover
    std::vector<int> hits;
    cfineIndex.query(cfine.boxes, cbox.grow(1), hits);
    if (hits.empty()) return;
    const std::vector<size_t> near(hits.begin(), hits.end());
    CellSet covered(cbox, false);
    for (size_t f : near) covered.set(cfine[f], true);
    // Per coarse cell of this box (first-touch order): its coarse terms and
    // fine groups.
    std::vector<int> slotOf((size_t)cbox.numPts(), -1);
    std::vector<IV> order;
    std::vector<std::vector<RefluxCoarseTerm>> terms;
    std::vector<std::vector<RefluxFineGroup>> groups;
    auto slot = [&](const IV& c) -> int {
      size_t q = (size_t)(c[0] - cbox.lo[0]) +
                 (size_t)cbox.size(0) * ((size_t)(c[1] - cbox.lo[1]) + (size_t)cbox.size(1) * (c[2] - cbox.lo[2]));
      if (slotOf[q] < 0) {
        slotOf[q] = (int)order.size();
        order.push_back(c);
        terms.emplace_back();
        groups.emplace_back();
      }
      return slotOf[q];
    };
    // Coarse terms, in incrementCoarse order: direction, then low/high side.
    for (int d = 0; d < 3; ++d)
      for (int side = -1; side <= 1; side += 2)
        for (size_t f : near) {
          Box loc = cfine[f].adjCell(d, side, 1) & cbox;
          if (loc.empty()) continue;
          for (int k = loc.lo[2]; k <= loc.hi[2]; ++k)
            for (int j = loc.lo[1]; j <= loc.hi[1]; ++j)
              for (int i = loc.lo[0]; i <= loc.hi[0]; ++i) {
                IV c(i, j, k);
                if (covered.contains(c)) continue;
                RefluxCoarseTerm t;
                IV e = IV::basis(d);
                IV hi = (side < 0) ? c + e : c;
                IV lo = (side < 0) ? c : c - e;
                t.hi = cellOf(C, (int)cb, hi);
                t.lo = cellOf(C, (int)cb, lo);
                t.bface = vc ? t.hi : -1;
                t.dir = d;
                t.sgn = (side < 0) ? 1.0 : -1.0;
                terms[slot(c)].push_back(t);
              }
        }
    // Fine groups, in copyTo order: fine box index.
    for (size_t f : near) {
      const Box& fbox = F.grids[f];
      for (int d = 0; d < 3; ++d)
        for (int side = -1; side <= 1; side += 2) {
          Box loc = cfine[f].adjCell(d, side, 1) & cbox;
          if (loc.empty()) continue;
          for (int k = loc.lo[2]; k <= loc.hi[2]; ++k)
            for (int j = loc.lo[1]; j <= loc.hi[1]; ++j)
              for (int i = loc.lo[0]; i <= loc.hi[0]; ++i) {
                IV c(i, j, k);
                if (covered.contains(c)) continue;
                RefluxFineGroup g;
                g.dir = d;
                g.scale = ((side < 0) ? -1.0 : 1.0) * 1.0 / 4.0;
                Box ghosts = Box(c, c).refine(2) & fbox.adjCell(d, side, 1);
                int n = 0;
                for (int z = ghosts.lo[2]; z <= ghosts.hi[2]; ++z)
                  for (int y = ghosts.lo[1]; y <= ghosts.hi[1]; ++y)
                    for (int x = ghosts.lo[0]; x <= ghosts.hi[0]; ++x) {
                      IV gcell(x, y, z);
                      IV v = gcell - IV::basis(d, side);
                      IV hi = (side < 0) ? v : gcell;
                      IV lo = (side < 0) ? gcell : v;
                      g.hi[n] = cellOf(F, (int)f, hi);
                      g.lo[n] = cellOf(F, (int)f, lo);
                      g.bface[n] = vc ? g.hi[n] : -1;
                      ++n;
                    }
                if (n != 4) throw std::runtime_error("cmg: fine face group is not 2x2");
                groups[slot(c)].push_back(g);
              }
        }
    }
    for (size_t q = 0; q < order.size(); ++q) {
      RefluxCell rc;
      rc.c = cellOf(C, (int)cb, order[q]);
      rc.nco = (int)terms[q].size();
      rc.nfi = (int)groups[q].size();
      rc.start = (int)out.co.size();
      rc.fstart = (int)out.fi.size();
      for (auto& t : terms[q]) out.co.push_back(t);
      for (auto& g : groups[q]) out.fi.push_back(g);
      out.cells.push_back(rc);
    }
  });
  // Concatenation from prefix sums, the parts copied on host threads.
  const size_t np = parts.size();
  std::vector<size_t> n0(np + 1, 0), t0(np + 1, 0), g0(np + 1, 0);
  for (size_t k = 0; k < np; ++k) {
    n0[k + 1] = n0[k] + parts[k].cells.size();
    t0[k + 1] = t0[k] + parts[k].co.size();
    g0[k + 1] = g0[k] + parts[k].fi.size();
  }
  C.rfCells.resize(n0[np]);
  C.rfCoarse.resize(t0[np]);
  C.rfFine.resize(g0[np]);
  parallelItems(np, [&](size_t k) {
    Part& p = parts[k];
    for (size_t i = 0; i < p.cells.size(); ++i) {
      RefluxCell rc = p.cells[i];
      rc.start += (int)t0[k];
      rc.fstart += (int)g0[k];
      C.rfCells[n0[k] + i] = rc;
    }
    std::copy(p.co.begin(), p.co.end(), C.rfCoarse.begin() + t0[k]);
    std::copy(p.fi.begin(), p.fi.end(), C.rfFine.begin() + g0[k]);
    p = Part();
  });
}

void buildBottom(const LevelPlan& L, BottomPlan& B) {
  B = BottomPlan();
  std::unordered_map<int64_t, int> slot;  // FAB element -> slot
  const size_t nbox = L.boxes.size();
  B.boxStart.assign(nbox + 1, 0);
  for (size_t b = 0; b < nbox; ++b) {
    const Box& bx = L.grids[b];
    B.boxStart[b] = (int)B.fab.size();
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
      for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
        for (int i = bx.lo[0]; i <= bx.hi[0]; ++i) {
          int64_t e = cellIndex(L.boxes[b], i, j, k);
          slot[e] = (int)B.fab.size();
          B.fab.push_back((int)e);
        }
  }
  B.boxStart[nbox] = (int)B.fab.size();
  B.nv = (int)B.fab.size();
  B.nb.resize(6 * (size_t)B.nv);
  static const int dirs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  for (size_t b = 0; b < nbox; ++b) {
    const Box& bx = L.grids[b];
    for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
      for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
        for (int i = bx.lo[0]; i <= bx.hi[0]; ++i) {
          int q = slot[cellIndex(L.boxes[b], i, j, k)];
          B.color[((i + j + k) & 1)].push_back(q);
          for (int d = 0; d < 6; ++d) {
            int64_t e = cellIndex(L.boxes[b], i + dirs[d][0], j + dirs[d][1], k + dirs[d][2]);
            auto it = slot.find(e);
            if (it == slot.end()) {
              it = slot.emplace(e, (int)B.fab.size()).first;
              B.fab.push_back((int)e);
            }
            B.nb[6 * (size_t)q + d] = it->second;
          }
        }
  }
  B.ng = (int)B.fab.size() - B.nv;
  B.gsrc.assign(B.ng, 0);
  B.gkind.assign(B.ng, 2);
  // Ghost tasks of the level (exchange copies, then Dirichlet faces), in
  // task order so that a slot written twice keeps the last writer.
  for (const GhostTask& t : L.ghost) {
    const BoxDesc& db = L.boxes[t.dst];
    for (int k = t.lo[2]; k <= t.hi[2]; ++k)
      for (int j = t.lo[1]; j <= t.hi[1]; ++j)
        for (int i = t.lo[0]; i <= t.hi[0]; ++i) {
          auto it = slot.find(cellIndex(db, i, j, k));
          if (it == slot.end() || it->second < B.nv) continue;
          const int g = it->second - B.nv;
          int64_t src;
          if (t.kind == G_COPY) {
            src = cellIndex(L.boxes[t.src], i - t.shift[0], j - t.shift[1], k - t.shift[2]);
            B.gkind[g] = 0;
          } else if (t.kind == G_BC || t.kind == G_NEU) {
            int e[3] = {0, 0, 0};
            e[t.dir] = -t.side;
            src = cellIndex(db, i + e[0], j + e[1], k + e[2]);
            B.gkind[g] = t.kind == G_BC ? 1 : 0;  // Neumann: a copy of the adjacent cell
          } else {
            throw std::runtime_error("cmg: coarse-fine ghost task on the bottom level");
          }
          auto s2 = slot.find(src);
          if (s2 == slot.end() || s2->second >= B.nv) throw std::runtime_error("cmg: bottom ghost source not valid");
          B.gsrc[g] = s2->second;
        }
  }
  // Every face ghost the stencil reads has a source (level 0 covers its
  // domain), so the solve reads the source directly.
  B.nbv.resize(B.nb.size());
  for (size_t i = 0; i < B.nb.size(); ++i) {
    const int n = B.nb[i];
    if (n < B.nv) {
      B.nbv[i] = n;
      continue;
    }
    const int g = n - B.nv;
    if (B.gkind[g] == 2) throw std::runtime_error("cmg: bottom level face ghost with no source");
    B.nbv[i] = B.gkind[g] == 0 ? B.gsrc[g] : -(B.gsrc[g] + 1);
  }
}

}  // namespace cmg

namespace cmg {

// ------------------------------------------------------------------ forests
// A forest level is the disjoint union of the same level of several
// hierarchies: their boxes one hierarchy after the other, each hierarchy's
// FABs in one contiguous element range.  Every table of a LevelPlan refers to
// boxes, elements, chunks or pool entries of its own level (or of the next
// coarser or finer level), so the union is the concatenation of the parts
// with those indices shifted; the hierarchies never share a cell, and every
// kernel over the union does, box by box, what it does over each part.
void mergeLevels(const std::vector<const LevelPlan*>& parts, const std::vector<int64_t>& elemOff,
                 const std::vector<int>& boxOff, const std::vector<int64_t>* coarseElemOff,
                 const std::vector<int>* coarseBoxOff, const std::vector<int64_t>* fineElemOff, LevelPlan& out) {
  const size_t K = parts.size();
  if (K == 0) throw std::invalid_argument("cmg: empty forest");
  const LevelPlan& p0 = *parts[0];
  out = LevelPlan();
  out.domain = p0.domain;
  out.dx = p0.dx;
  out.dxCrse = p0.dxCrse;
  auto shiftCell = [](GhostCell g, int64_t eo) {
    g.dst += (int)eo;
    g.s1 += (int)eo;
    if (g.s2 >= 0) g.s2 += (int)eo;
    return g;
  };
  auto shiftTask = [](GhostTask t, int bo) {
    t.dst += bo;
    t.src += bo;
    return t;
  };
  // boxes, grids, elements, chunks
  for (size_t k = 0; k < K; ++k) {
    const LevelPlan& p = *parts[k];
    if (p.dx != p0.dx || p.dxCrse != p0.dxCrse) throw std::invalid_argument("cmg: forest levels differ in dx");
    for (BoxDesc d : p.boxes) {
      d.off += elemOff[k];
      out.boxes.push_back(d);
    }
    out.grids.boxes.insert(out.grids.boxes.end(), p.grids.boxes.begin(), p.grids.boxes.end());
    out.nelem += p.nelem;
    for (Chunk c : p.chunksAll) out.chunksAll.push_back(Chunk{c.box + boxOff[k], c.start});
    for (int c = 0; c < 2; ++c)
      for (Chunk ch : p.chunksColor[c]) out.chunksColor[c].push_back(Chunk{ch.box + boxOff[k], ch.start});
    for (DeferredCell d : p.deferred) out.deferred.push_back(DeferredCell{d.box + boxOff[k], d.q});
  }
  if (out.nelem >= ((int64_t)1 << 31)) throw std::runtime_error("cmg: forest level too large for 32-bit indices");
  for (size_t k = 0; k < K; ++k) {
    out.hierStart.push_back(elemOff[k]);
    out.boxHier.insert(out.boxHier.end(), parts[k]->boxes.size(), (int)k);
  }
  out.hierStart.push_back(out.nelem);
  // ghost tasks: every part's exchange and boundary tasks, then every part's
  // coarse-fine tasks (the order the fills rely on)
  for (int pass = 0; pass < 2; ++pass)
    for (size_t k = 0; k < K; ++k) {
      const LevelPlan& p = *parts[k];
      const size_t a = pass == 0 ? 0 : (size_t)p.nExchBC, b = pass == 0 ? (size_t)p.nExchBC : p.ghost.size();
      for (size_t t = a; t < b; ++t) out.ghost.push_back(shiftTask(p.ghost[t], boxOff[k]));
      if (pass == 0) out.nExchBC += p.nExchBC;
    }
  out.ghostStart.assign(1, 0);
  out.slotStart.assign(1, 0);
  for (const GhostTask& t : out.ghost) {
    const int64_t c = (int64_t)(t.hi[0] - t.lo[0] + 1) * (t.hi[1] - t.lo[1] + 1) * (t.hi[2] - t.lo[2] + 1);
    out.ghostStart.push_back(out.ghostStart.back() + (int)c);
    out.slotStart.push_back(out.slotStart.back() + (int)colourSlots(t.lo, t.hi, parityAxis(t.lo, t.hi)));
  }
  out.ghostBlock = blockTasks(out.ghostStart);
  out.slotBlock = blockTasks(out.slotStart);
  // flat ghost cells: per parity all exchange+boundary parts, then all CF parts
  for (int par = 0; par < 2; ++par) {
    out.gcStart[par] = (int)out.gcells.size();
    for (int cf = 0; cf < 2; ++cf)
      for (size_t k = 0; k < K; ++k) {
        const LevelPlan& p = *parts[k];
        const int a = p.gcStart[par] + (cf ? p.gcExch[par] : 0);
        const int n = cf ? p.gcCF[par] : p.gcExch[par];
        for (int q = a; q < a + n; ++q) out.gcells.push_back(shiftCell(p.gcells[q], elemOff[k]));
        (cf ? out.gcCF[par] : out.gcExch[par]) += n;
      }
  }
  // face rules, per-chunk ghosts (each kept only when every part has them;
  // face rules missing here are built on the merged plan when asked for)
  bool chunkLists = true, rules = true;
  for (size_t k = 0; k < K; ++k) chunkLists = chunkLists && !parts[k]->chunkGhostStart[0].empty();
  for (size_t k = 0; k < K; ++k) rules = rules && (!parts[k]->faceOff.empty() || parts[k]->grids.size() == 0);
  for (size_t k = 0; k < K; ++k) {
    const LevelPlan& p = *parts[k];
    const int rbase = (int)out.faceRules.size();
    for (FaceRule r : p.faceRules) {
      if (!rules) break;
      if (r.kind == FR_COPY || r.kind == FR_CFQUAD || r.kind == FR_FAB) r.src += (int)elemOff[k];
      out.faceRules.push_back(r);
    }
    for (size_t q = 0; rules && q + 1 < p.faceOff.size(); ++q) out.faceOff.push_back(p.faceOff[q] + rbase);
    for (int c = 0; c < 2 && chunkLists; ++c) {
      const int gbase = (int)out.chunkGhost[c].size();
      for (const GhostCell& g : p.chunkGhost[c]) out.chunkGhost[c].push_back(shiftCell(g, elemOff[k]));
      for (size_t q = 0; q + 1 < p.chunkGhostStart[c].size(); ++q)
        out.chunkGhostStart[c].push_back(p.chunkGhostStart[c][q] + gbase);
    }
  }
  if (rules) out.faceOff.push_back((int)out.faceRules.size());
  for (int c = 0; c < 2 && chunkLists; ++c) out.chunkGhostStart[c].push_back((int)out.chunkGhost[c].size());
  // zeroing of the cells under the finer level
  for (size_t k = 0; k < K; ++k)
    for (const GhostTask& t : parts[k]->zeroCovered) out.zeroCovered.push_back(shiftTask(t, boxOff[k]));
  out.zeroStart.assign(1, 0);
  for (const GhostTask& t : out.zeroCovered)
    out.zeroStart.push_back(out.zeroStart.back() +
                            (t.hi[0] - t.lo[0] + 1) * (t.hi[1] - t.lo[1] + 1) * (t.hi[2] - t.lo[2] + 1));
  out.zeroBlock = blockTasks(out.zeroStart);
  // coarse-fine interpolation and coarse/fine maps (coarser level indices)
  if (coarseElemOff) {
    for (size_t k = 0; k < K; ++k) {
      const LevelPlan& p = *parts[k];
      const int64_t eoC = (*coarseElemOff)[k];
      const int coarseBase = (int)out.cfCoarse.size(), poolBase = (int)out.cfOff.size();
      for (CFCoarse e : p.cfCoarse) {
        e.cc += eoC;
        for (int q = 0; q < 2; ++q) {
          if (e.d1[q].kind) e.d1[q].start += poolBase;
          if (e.d2[q].kind) e.d2[q].start += poolBase;
        }
        if (e.mx.kind) e.mx.start += poolBase;
        out.cfCoarse.push_back(e);
      }
      for (CFFine f : p.cfFine) {
        f.g += elemOff[k];
        f.pa += elemOff[k];
        f.pb += elemOff[k];
        f.coarse += coarseBase;
        out.cfFine.push_back(f);
      }
      out.cfW.insert(out.cfW.end(), p.cfW.begin(), p.cfW.end());
      for (int64_t o : p.cfOff) out.cfOff.push_back(o + eoC);
      const int itemBase = (int)out.toCoarse.size();
      for (CoarseFineItem it : p.toCoarse) {
        it.cbox += (*coarseBoxOff)[k];
        it.fbox += boxOff[k];
        out.toCoarse.push_back(it);
      }
      for (Chunk c : p.toCoarseChunksF) out.toCoarseChunksF.push_back(Chunk{c.box + itemBase, c.start});
      for (Chunk c : p.toCoarseChunksC) out.toCoarseChunksC.push_back(Chunk{c.box + itemBase, c.start});
    }
  }
  // flux-register correction from the finer level (finer level indices)
  if (fineElemOff) {
    for (size_t k = 0; k < K; ++k) {
      const LevelPlan& p = *parts[k];
      const int64_t eoF = (*fineElemOff)[k];
      const int cbase = (int)out.rfCoarse.size(), fbase = (int)out.rfFine.size();
      for (RefluxCell rc : p.rfCells) {
        rc.c += elemOff[k];
        rc.start += cbase;
        rc.fstart += fbase;
        out.rfCells.push_back(rc);
      }
      for (RefluxCoarseTerm t : p.rfCoarse) {
        t.hi += elemOff[k];
        t.lo += elemOff[k];
        if (t.bface >= 0) t.bface += elemOff[k];
        out.rfCoarse.push_back(t);
      }
      for (RefluxFineGroup g : p.rfFine) {
        for (int q = 0; q < 4; ++q) {
          g.hi[q] += eoF;
          g.lo[q] += eoF;
          if (g.bface[q] >= 0) g.bface[q] += eoF;
        }
        out.rfFine.push_back(g);
      }
    }
  }
}

}  // namespace cmg
