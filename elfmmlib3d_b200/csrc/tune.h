// tune.h -- the autotuner (internal header; tune.cu).
//
// A knob is a choice between equivalent implementations of one stage of a
// pass (for now: the FP32 translations of the M2M, M2L and L2L stages on
// the tensor cores or on the CUDA cores).  The choice depends on the
// problem's shape, so it is made per key (knob, expansion order, leaf
// capacity, expansion columns per box, precision, plan kind) from timings of
// the real passes: the first passes of a key run every candidate (twice
// each, the faster time kept), later ones the fastest.  Decided keys are
// kept for the process and, with ELFMM3D_TUNE_FILE set, in that file (read
// at the first use, a line appended per decision) for later processes.
#pragma once
#include <string>
#include <vector>

namespace efmm {

struct TuneKey {
  int knob, p, nbox, C, prec, kind;
  bool operator<(const TuneKey& o) const;
  bool operator==(const TuneKey& o) const;
};

constexpr int TUNE_VISITS = 2;  // timed runs of each candidate before deciding

// Candidate to run now for key k among ncand (0 .. ncand - 1).
int tune_pick(const TuneKey& k, int ncand);
// The decided candidate, or fallback while undecided (no exploration: for
// passes captured into a CUDA graph, which record no stage times).
int tune_best(const TuneKey& k, int fallback);
// A timed run of candidate cand for key k (stage milliseconds).
void tune_report(const TuneKey& k, int ncand, int cand, float ms);
// Forget every key (the file is not touched).
void tune_reset();
// One line per key: "knob p nbox C prec kind decided ms0 ms1 ..." (decided
// -1 while exploring; ms of an untried candidate -1).
std::vector<std::string> tune_dump();

}  // namespace efmm
