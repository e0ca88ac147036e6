/* Tangent-linear restatement of the reference sinksim time step (portable numerics), for gradient checks only.
 *
 * TEST INFRASTRUCTURE. Only tests/ and bench.py's CPU baseline may load this code, and only as the checker of the
 * CUDA adjoint; the sinksim_b200 package never links or calls it.
 *
 * It is the step of sinksim_oracle.c (itself pinned bit for bit to the reference's golden traces) restated over a
 * forward-mode dual number: every value is computed with exactly the operations of the portable step, in the same
 * order (so the value part is bit-identical to the oracle and takes the same branches), and carries the derivatives
 * of that value with respect to up to SST_MAX_PARAMS parameters through the same operations. The parameters enter
 * through connection areas: sst_seed_area(c, p, g) says d area[c] / d theta[p] = g. The result is the FP64
 * tangent-linear derivative of the trajectory along the branch path the forward run takes, the reference gradient
 * that a hand-written adjoint must reproduce.
 *
 * The reference has no gradients (docs/adr/0001-single-source-cpp-kernel.md:25-26); the derivative rules used for
 * the non-smooth pieces (min/max and clamps follow the branch taken; the minimum of a node's segment bottoms follows
 * the segment the reference's reduction tree selects) are stated beside the code.
 */
#ifndef SINKSIM_TANGENT_H
#define SINKSIM_TANGENT_H

#include <stdint.h>

#include "sinksim_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SST_MAX_PARAMS 10

typedef struct sst_engine sst_engine;

/* Portable numerics only (double precision, tree order). Starts at the compiled initial state. */
sst_engine* sst_create(const sso_ship* ship, const sso_sim* sim);
void sst_destroy(sst_engine* e);
/* Connection fields (values). enabled < 0, area NaN or tOn NaN leave that field as it is. */
void sst_set_connection(sst_engine* e, int32_t c, int enabled, double area, double tOn);
/* d area[c] / d theta[p] = g (0 <= p < SST_MAX_PARAMS). */
void sst_seed_area(sst_engine* e, int32_t c, int32_t p, double g);
void sst_step(sst_engine* e, int64_t n);
/* The state record (the trace layout of sso_get_record) and its tangents: d[p * recSize + k]. */
void sst_get_record(const sst_engine* e, double* rec, double* d);
/* Readouts (t, trimDeg, listDeg, waterT, inflowTpm, draftF, draftA) and their tangents d[p * 7 + k]. */
void sst_readouts(const sst_engine* e, double* r7, double* d);
int sst_foundered(const sst_engine* e);

#ifdef __cplusplus
}
#endif

#endif
