// Grid generation on the host: MeshRefine::regrid with BRMeshRefine's
// Berger-Rigoutsos clustering (reference BoxTools/MeshRefine.cpp,
// BoxTools/BRMeshRefine.cpp), proper-nesting mode 1, every direction refined,
// non-periodic domains, and the example drivers' tagging loop on top.  The
// box sets are identical to the reference's (the tests compare them with the
// reference's own output); the order of boxes within a level is the sorted
// layout order.
#ifndef CMG_MESHREFINE_H
#define CMG_MESHREFINE_H

#include <cstdint>
#include <vector>

#include "geom.H"
#include "synthetic.H"

namespace cmg {

// Cell set over a box with O(1) box-containment queries (summed-volume
// table): the proper nesting domain of one level.
struct NestingSet {
  Box dom;
  std::vector<int64_t> sum;  // (nx+1)(ny+1)(nz+1) prefix counts
  void build(const CellSet& s);
  bool containsBox(const Box& b) const;
};

class MeshRefiner {
 public:
  // MeshRefine::define (MeshRefine.cpp:330-373).
  MeshRefiner(const Box& baseDomain, const std::vector<int>& refRatios, double fillRatio, int blockFactor,
              int bufferSize, int maxSize);
  // MeshRefine::regrid (MeshRefine.cpp:438-729).  tags[l]: tagged cells of
  // level l in its own index space (modified).  Returns the new finest level.
  int regrid(std::vector<std::vector<Box>>& newMeshes, std::vector<CellSet>& tags, int baseLevel, int topLevel,
             const std::vector<std::vector<Box>>& oldMeshes) const;
  // BRMeshRefine::makeBoxes (BRMeshRefine.cpp:213-308) on a list of tagged
  // cells (consumed).
  void makeBoxes(std::vector<Box>& mesh, std::vector<IV>& tags, const NestingSet& pnd, const Box& domain,
                 int maxBoxSize, int totalBufferSize) const;

 private:
  std::vector<int> nRef_, blockFactors_;
  std::vector<Box> domains_;
  double fillRatio_;
  int blockFactor_, bufferSize_, maxSize_;
  void makeBoxesRec(std::vector<Box>& mesh, IV* begin, IV* end, const NestingSet& pnd, const Box& domain,
                    int maxBoxSize, int totalBufferSize) const;
};

// Computes the grown, domain-clipped tags of one level that levelTags in
// meshrefine.cpp computes on the host (used to move that pass to a device).
struct LevelTagger {
  virtual ~LevelTagger() {}
  virtual void tags(const std::vector<Box>& grids, const Box& domain, double dx, const cmg_synth::Bumps& bumps,
                    double thresh, CellSet& out) = 0;
};

// The example drivers' hierarchy (oracle/driver.cpp, after
// releasedExamples/AMRPoisson/execCell/poissonSolve.cpp:296-317 and
// execVariableCoefficient/VClocalFuncs.cpp:398-480): base level by
// domainSplit of [0, n0-1]^3, then passes that tag |rhs| > thresh*max|rhs|
// (seeded Gaussian bumps) on every level, grow the tags by one cell and
// regrid with buffer 2, one new level per pass, up to numLevels levels.
// Returns the sorted box list of every level.  The tags of a level whose
// grids did not change since the previous pass are reused.  tagger, when
// given, computes the tags instead of the host.
std::vector<std::vector<Box>> syntheticHierarchy(int n0, int numLevels, int maxBox, int blockFactor, double fillRatio,
                                                 uint64_t seed, double thresh, LevelTagger* tagger = nullptr);

}  // namespace cmg

#endif
