/*
 * ORACLE / TEST INFRASTRUCTURE ONLY — the checker, never the product. Only tests, the smoke
 * check and the benchmark's CPU-baseline leg load it.
 *
 * A plain-C restatement of acoustic-spaces' WaveSolver::run (cpp/include/acoustic_spaces/
 * fdtd.hpp:786-904 of naelolaiz/acoustic-spaces) over the grid's layout (fdtd.hpp:727-782), in
 * the reference's order of operations:
 *   record     fdtd.hpp:3525-3533   probes before the step, summed in double
 *   interior   fdtd.hpp:242-288     7- and 19-point updates, with and without a speed field
 *   special    fdtd.hpp:860-881     links, branch states, coef_a/coef_b/coef_inv, source
 *   layer      fdtd.hpp:2242-2264   split-field matched layer
 *   swap       fdtd.hpp:884-885, parity swap at the end fdtd.hpp:900-903
 * ORACLE_FP32 flushes subnormal results to zero as the reference does (FlushDenormals,
 * fdtd.hpp:316-336) and equals the reference bit for bit; ORACLE_FP64 steps the same layout in
 * double (every stored coefficient promoted, no flush): the FP64 oracle. ORACLE_FP32C is no
 * restatement: it steps the same scheme in this project's compensated single precision
 * (FDTD_FP32_COMPENSATED), operation for operation as the GPU does, as that mode's checker.
 * Parity of this restatement is pinned against the reference's own run() (compiled from its
 * unmodified headers, oracle/_ref) by the tests and by the golden fixtures under tests/golden.
 */
#ifndef FDTD_ORACLE_H
#define FDTD_ORACLE_H

#include <stdint.h>

#include "../include/fdtd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_FP32 0
#define ORACLE_FP64 1
#define ORACLE_FP32C 2 /* the GPU's FDTD_FP32_COMPENSATED, its checker */

typedef struct oracle_solver oracle_solver;

int oracle_create(const fdtd_layout *layout, int precision, oracle_solver **out);
int oracle_run(oracle_solver *solver, const float *signal, uint64_t steps, double *out);
int oracle_reset(oracle_solver *solver);
void oracle_destroy(oracle_solver *solver);
/* Same buffers and order as fdtd_read_state (include/fdtd_b200.h). */
int oracle_read_state(const oracle_solver *solver, void *current, void *previous,
                      void *branch_current, void *branch_previous, void *layer_state);
const char *oracle_error(void);
/* The host threads a run of a large grid steps on (the host's cores, or ORACLE_THREADS). */
int oracle_threads(void);
/* The current (which 0) or previous (1) pressure level between runs, nx*ny*nz elements: the
   slab tests read and write its planes. */
void *oracle_level(oracle_solver *solver, int which);

#ifdef __cplusplus
}
#endif

#endif
