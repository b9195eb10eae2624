/*
 * The constant-mode residuals of the compensated single-precision form (FDTD_FP32_COMPENSATED).
 *
 * That form steps the pressure p_n and its increment d_n = p_n - p_(n-1). Writing p_(n-1) =
 * p_n - d_n into the reference's updates (interior fdtd.hpp:242-288, special rows
 * fdtd.hpp:860-881 of naelolaiz/acoustic-spaces) leaves every neighbour as a difference
 * (p_m - p_n) and one term in p_n alone, whose coefficient is what the update does to a constant
 * pressure at rest: zero when the stored coefficients hold it still, a rounding's worth
 * otherwise. These are those coefficients, worked out in double from the stored floats:
 *   interior   centre + sum(weights) - 2            (with a speed field: sum(weights) - total,
 *                                                     each cell's scale multiplying it)
 *   special k  coef_inv * (coef_a - coef_b + sum of the row's link weights) - 1
 * Plain C, shared by the device library's set-up and the oracle, so that both step the same
 * coefficients.
 */
#ifndef FDTD_COMPENSATED_H
#define FDTD_COMPENSATED_H

#include "../../include/fdtd_b200.h"

static inline void fdtd_compensated_residuals(const fdtd_layout *L, float *interior, float *row) {
    double weights = 0.0;
    for (uint32_t k = 0; k < L->weight_count; ++k) weights += (double)L->weights[k];
    *interior = L->scaled ? (float)(weights - (double)L->total) : (float)((double)L->centre + weights - 2.0);
    for (uint64_t k = 0; k < L->special_count; ++k) {
        double links = 0.0;
        for (uint64_t l = L->link_start[k]; l < L->link_start[k + 1]; ++l) links += (double)L->link_weight[l];
        const double kept = (double)L->coef_a[k] - (double)L->coef_b[k] + links;
        row[k] = (float)((double)L->coef_inv[k] * kept - 1.0);
    }
}

#endif
