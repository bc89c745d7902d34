// efsi_diag.cuh — device reductions of the cavity drivers' diagnostics (host side).
#pragma once

#include <algorithm>

#include "efsi_common.cuh"

namespace efsi {

// Totals written by launch_diagnostics, in order:
//   [0, kDiagSums)                      sums: phase mass, x and y moments, perimeter proxy,
//                                       mixed-layer measure, kinetic energy, area-weighted
//                                       div^2, volume, out-of-bounds count, then per tensor
//                                       region (global, core, interface, tail): cells, area,
//                                       area*|det-1|, area*stress, non-SPD count
//   [kDiagSums, +kDiagMaxes)            maxima: -min phi, max phi, max speed, max |div|,
//                                       max |U|, max |V|, then per region: -min det, max det,
//                                       max |det-1|, -min lambda, max lambda, max stress
//   [kDiagSums+kDiagMaxes, +kDiagSums2) second pass: phi-weighted xx, yy, xy moments about
//                                       the centroid, Rc[8], Rs[8]
constexpr int kDiagSums = 29, kDiagMaxes = 30, kDiagSums2 = 19;
constexpr int kDiagTotals = kDiagSums + kDiagMaxes + kDiagSums2;

void launch_diagnostics(const Params& P, const efsi_diag_config& cfg, const double* U, const double* V,
                        const double* phi, const double* sxx, const double* syy, const double* sxy,
                        const RedSlot& r1, const RedSlot& r2, const RedSlot& r3, double* tot, int max_blocks,
                        cudaStream_t s);

}  // namespace efsi
