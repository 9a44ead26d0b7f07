// hhg_pulse_prep.hpp -- per-pulse preparation shared with the allocation-free
// entry point (hhg_noalloc.cu): model variant, staged-interpolant degree,
// the device pulse record and the accumulated interval ends of one pulse.
#pragma once

#include <vector>

#include "../../include/hhg_gpu.h"
#include "hhg_device.cuh"

namespace hhg_prep {

// Magnus-4 substeps per measurement interval accepted by every entry point
// (a larger count would run a persistent launch for minutes to hours).
constexpr int kMaxMagnusSubsteps = 4096;
inline bool magnus_substeps_ok(int n) { return n >= 1 && n <= kMaxMagnusSubsteps; }

struct PulsePrep {
    int model = 0;   // hhg::Model
    int nf = 0;      // staged pulse functions
    int degree = 0;  // staged interpolant degree, -1 if the intervals are too coarse
    hhg::PulseDev pulse{};
    std::vector<double> tgrid;  // n_measurements + 1 accumulated interval ends
};

// Validates sys/pulse like hhg_plan_create and fills `out`; the offsets
// inside out.pulse (coef/part/j) are left at 0 and items at 0.
hhg_status prepare_pulse(const hhg_system_desc *sys, const hhg_pulse_desc *pulse, PulsePrep &out);

}  // namespace hhg_prep
