// ORACLE — test infrastructure only.  Never linked into the product.
//
// Runs the reference's FineInterp (lib/src/AMRTools/FineInterp.cpp:
// define, interpToFine with the default PCInterp boundary limit type, or
// pwcinterpToFine) on the seeded synthetic hierarchies (problem.H): level
// `level` is filled from level `level` - 1.  The coarse data are the seeded
// right-hand side of that level, or the values of the file given as
// coarse=<path> (float64, per box in layout order, valid cells x-fastest).
//
// Usage: cmg_oracle_fineinterp key=value ... out=<prefix>
//   n0 levels maxbox block fill seed thresh boxfile (as cmg_oracle)
//   level=1 pwc=0 coarse=<path> repeat=1 (timed interpolations; the last
//   one's output is written)
// Writes <prefix>.json (boxes of both levels) and <prefix>.bin (the fine
// level's valid cells, per box in layout order, x fastest).

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "FineInterp.H"
#include "problem.H"

static std::map<std::string, std::string> g_args;
static double argd(const char* k, double d) {
  auto it = g_args.find(k);
  return it == g_args.end() ? d : std::atof(it->second.c_str());
}
static int argi(const char* k, int d) {
  auto it = g_args.find(k);
  return it == g_args.end() ? d : std::atoi(it->second.c_str());
}

static void dumpBoxes(FILE* js, const DisjointBoxLayout& g) {
  std::fprintf(js, "[");
  bool first = true;
  for (LayoutIterator lit = g.layoutIterator(); lit.ok(); ++lit) {
    const Box& b = g[lit];
    std::fprintf(js, "%s[%d,%d,%d,%d,%d,%d]", first ? "" : ",", b.smallEnd(0), b.smallEnd(1), b.smallEnd(2),
                 b.bigEnd(0), b.bigEnd(1), b.bigEnd(2));
    first = false;
  }
  std::fprintf(js, "]");
}

int main(int argc, char** argv) {
  for (int a = 1; a < argc; ++a) {
    const char* eq = std::strchr(argv[a], '=');
    if (eq) g_args[std::string(argv[a], eq - argv[a])] = std::string(eq + 1);
  }
  OracleProblem P;
  P.n0 = argi("n0", 32);
  P.numLevels = argi("levels", 2);
  P.maxBox = argi("maxbox", 32);
  P.blockFactor = argi("block", 8);
  P.fillRatio = argd("fill", 0.75);
  P.seed = (unsigned long long)argd("seed", 20261203.0);
  P.thresh = argd("thresh", 0.1);
  if (g_args.count("boxfile")) P.boxfile = g_args["boxfile"];
  const int level = argi("level", 1);
  const bool pwc = argi("pwc", 0) != 0;
  const int repeat = argi("repeat", 1);
  const std::string out = g_args.count("out") ? g_args["out"] : std::string("fineinterp_out");
  if (buildProblem(P) != 0) return 2;
  if (level < 1 || level > P.finest) {
    std::fprintf(stderr, "level %d outside 1..%d\n", level, P.finest);
    return 2;
  }
  const DisjointBoxLayout& cg = P.grids[level - 1];
  const DisjointBoxLayout& fg = P.grids[level];

  LDF coarse(cg, 1, IntVect::Unit), fine(fg, 1, IntVect::Unit);
  for (DataIterator dit = cg.dataIterator(); dit.ok(); ++dit) {
    coarse[dit()].setVal(0.0);
    coarse[dit()].copy((*P.rhs[level - 1])[dit()], cg[dit()]);
  }
  if (g_args.count("coarse")) {
    FILE* in = std::fopen(g_args["coarse"].c_str(), "rb");
    if (!in) return 2;
    for (LayoutIterator lit = cg.layoutIterator(); lit.ok(); ++lit) {
      const Box& b = cg[lit];
      FArrayBox& fab = coarse[DataIndex(lit())];
      for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
        for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
          for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) {
            double v;
            if (std::fread(&v, sizeof(double), 1, in) != 1) return 2;
            fab(IntVect(i, j, k), 0) = v;
          }
    }
    std::fclose(in);
  }
  for (DataIterator dit = fg.dataIterator(); dit.ok(); ++dit) fine[dit()].setVal(0.0);

  FineInterp fi(fg, 1, 2, P.domains[level]);
  const auto t0 = std::chrono::steady_clock::now();
  for (int r = 0; r < repeat; ++r) {
    if (pwc)
      fi.pwcinterpToFine(fine, coarse);
    else
      fi.interpToFine(fine, coarse);
  }
  const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() / repeat;

  FILE* js = std::fopen((out + ".json").c_str(), "w");
  std::fprintf(js, "{\"level\": %d, \"pwc\": %d, \"coarse_boxes\": ", level, pwc ? 1 : 0);
  dumpBoxes(js, cg);
  std::fprintf(js, ", \"fine_boxes\": ");
  dumpBoxes(js, fg);
  std::fprintf(js, "}\n");
  std::fclose(js);
  FILE* bin = std::fopen((out + ".bin").c_str(), "wb");
  for (LayoutIterator lit = fg.layoutIterator(); lit.ok(); ++lit) {
    const Box& b = fg[lit];
    const FArrayBox& fab = fine[DataIndex(lit())];
    for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
      for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
        for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) {
          double v = fab(IntVect(i, j, k), 0);
          std::fwrite(&v, sizeof(double), 1, bin);
        }
  }
  std::fclose(bin);
  std::printf("fineinterp: level=%d pwc=%d coarse boxes=%d fine boxes=%d fine cells=%ld seconds_per_call=%.6f\n",
              level, pwc ? 1 : 0, (int)cg.size(), (int)fg.size(), (long)fg.numCells(), seconds);
  return 0;
}
