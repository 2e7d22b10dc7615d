// Device-side tagging for grid generation.  The example drivers tag the
// cells of a level whose |rhs| exceeds thresh * max|rhs| over the level, grow
// every tag by one cell and clip it to the level's domain
// (releasedExamples/AMRPoisson/execVariableCoefficient/VClocalFuncs.cpp:586-624,
// with the strict comparison of the oracle's driver), then hand the tag set to
// MeshRefine::regrid.  Evaluating the seeded right-hand side at every cell of
// the level is the data-parallel part: this tagger runs it, the max-reduction,
// the threshold and the one-cell growth on the device, and copies the grown
// tag map of the domain back into a CellSet for the host's Berger-Rigoutsos.
//
// The right-hand side is evaluated with the CUDA math library's exp (at most
// 1 ulp from the host's), so a cell whose |rhs| lies within a few ulps of the
// threshold could in principle be tagged differently from the host tagger;
// the box lists are compared with the host path's on every test case.
#ifndef CMG_TAGGING_H
#define CMG_TAGGING_H

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "meshrefine.H"

namespace cmg {

class DeviceTagger : public LevelTagger {
 public:
  // Work buffers are allocated on first use, grow as needed and are owned by
  // the tagger; all work is issued on stream s of the current device.
  explicit DeviceTagger(cudaStream_t s = nullptr);
  ~DeviceTagger() override;
  DeviceTagger(const DeviceTagger&) = delete;
  DeviceTagger& operator=(const DeviceTagger&) = delete;
  void tags(const std::vector<Box>& grids, const Box& domain, double dx, const cmg_synth::Bumps& bumps,
            double thresh, CellSet& out) override;

 private:
  cudaStream_t s_;
  void* cells_ = nullptr;  // box and chunk tables
  size_t cellsBytes_ = 0;
  double* vals_ = nullptr;  // |rhs| per valid cell
  size_t valsCount_ = 0;
  uint8_t* map_[2] = {nullptr, nullptr};  // domain tag maps (ping-pong for the growth)
  size_t mapBytes_ = 0;
  unsigned long long* dMax_ = nullptr;
};

}  // namespace cmg

#endif
