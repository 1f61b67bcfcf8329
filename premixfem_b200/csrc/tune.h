// Launch-configuration autotuner.
//
// Kernels whose launch shape has more than one reasonable value (tile rows of
// the network convolutions, threads per subdomain of the level-1 solves and of
// the level-2 restriction / prolongation) ask the tuner for a candidate index
// under a key made of the kernel, the problem shape and the device name.  The
// first time a key is seen every candidate is launched once to warm up and
// then `reps` times between CUDA events on the launching stream; the fastest
// wins and is remembered for the life of the process.  Every candidate must be
// a pure function of its inputs (or write scratch buffers), so that timing it
// leaves the results unchanged.
//
// PMF_AUTOTUNE=0 in the environment (or -pmf_autotune 0) turns tuning off:
// candidate 0, the built-in default, is used.  PMF_TUNE_FILE=<path> keeps the
// table across processes (read on first use, rewritten after each new key).
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>

namespace pmf {

// Index of the candidate to use for `key` (0 .. ncand-1).  `launch(c)` issues
// candidate c on `st` and returns false when c does not apply to this shape.
int tune_choose(const std::string& key, int ncand, const std::function<bool(int)>& launch, cudaStream_t st,
                int reps = 3);
// Online form for kernels that change their data and run once per step of a
// loop (the lock-step eigensolver phases): tune_online_pick returns the
// candidate to launch now -- each candidate in turn until all have run once,
// then the fastest -- and the caller reports the measured time per unit of
// work (e.g. per active subdomain) with tune_online_report.  Every launch is
// a real step of the computation, so nothing is run twice.
int tune_online_pick(const std::string& key, int ncand);
void tune_online_report(const std::string& key, int ncand, int cand, float us_per_unit);
// Turn tuning on or off for the whole process (the solver option -pmf_autotune).
void tune_set_enabled(bool on);
bool tune_enabled();
// The device part of the keys ("NVIDIA B200" ...).
const std::string& tune_device();
// The table as JSON: {"key": {"choice": c, "us": [t0, t1, ...]}, ...}
std::string tune_report();

}  // namespace pmf
