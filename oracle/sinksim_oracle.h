/* CPU restatement of the reference sinksim time step, for parity testing only.
 *
 * TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline may load this code, and
 * only as the checker of the CUDA path; the sinksim_b200 package never links or calls it.
 *
 * It restates, in plain C, the reference's kernel::step<PortableMath, Order::Tree> ("portable" numerics) and
 * kernel::step<PortableMath, Order::TreeMixed> ("portable32") (engine/include/sinksim/kernel/step.hpp:41-54),
 * operation for operation, and counts the work it does (columns clipped, node passes, segment visits, weir pow
 * calls) so that the algorithmic cost of a step can be stated exactly. sin, cos and pow are the vendored fdlibm 5.3
 * (third_party/fdlibm of the reference, compiled by oracle/Makefile), the bit reference of the portable math.
 *
 * Parity is pinned: tests/test_oracle.py holds this restatement to the reference's golden traces
 * (data/golden/titanic64/titanic.portable*.trace.json, reduced in tests/golden/) at tolerance 0 and to the
 * reference engine itself (oracle/_ref/libsinksim_ref.so) on synthetic hulls.
 */
#ifndef SINKSIM_ORACLE_H
#define SINKSIM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Arrays of a compiled ship and a compiled sim (docs/FORMATS.md of the reference). The oracle copies them. */
typedef struct {
  int32_t ncol, nseg, nnode;
  const double *x, *y, *dxdy, *zlo, *zhi;
  const int32_t* segCol;
  const double *segA, *segE;
  const double *mu, *vmax, *amin, *aov;
  const int32_t *segStart, *segCount;
} sso_ship;

typedef struct {
  double rho, g, dt;
  int32_t ngroup;
  const int32_t *gStart, *gCount, *gNodes;
  const uint8_t* gMode;
  const double *gpx, *gpy, *gpz;
  double gMargin;
  int32_t nconn;
  const int32_t *ca, *cb;
  const uint8_t* law;
  const double *cx, *cy, *cz, *area, *coef;
  const uint8_t* en;
  const double* tOn;
  const int32_t *skipGroup, *monitor;
  int32_t nmon;
  double monThreshold;
  int32_t nmark;
  const double *mkx, *mky, *mkz;
  const uint8_t* mkWhen;
  double hullTopBelow, pitchAbsAbove, buoyancyBelow, minT;
  /* ms, KG, g0x, g0y, g0z, XO, YO, mh0, Ith0, Iph0, cDz, cDth, cDph, qz, qth, qph */
  double body[16];
  double xFP, xAP;
  /* initial state: t, zO, pitch, roll, vz, wth, wph; per node vol, level, cx, cy, cz */
  double state0[7];
  const double *vol0, *level0, *cx0, *cy0, *cz0;
} sso_sim;

typedef struct {
  int64_t steps, columns, passes, segVisits, segWet, colWet, weirPow, orifice, weir, newton;
} sso_counters;

typedef struct sso_engine sso_engine;

/* mixed = 0: portable (double precision tree order); 1: portable32 (single-precision partials). */
sso_engine* sso_create(const sso_ship* ship, const sso_sim* sim, int mixed);
void sso_destroy(sso_engine* e);
/* Back to the compiled initial state with buoyancy evaluated (the reference Simulation constructor). */
void sso_reset(sso_engine* e);
void sso_set_connection(sso_engine* e, int32_t c, int enabled, double area, double tOn);
void sso_step(sso_engine* e, int64_t n);
/* Trace record: t, zO, pitch, roll, vz, wth, wph, inflow, Vb, hullTop, then vol, level, cx, cy, cz per node. */
void sso_get_record(const sso_engine* e, double* rec);
/* Restart from a record; events are cleared (Simulation::restore, engine/src/simulation.cpp:92-101). */
void sso_restore(sso_engine* e, const double* rec);
/* t, trimDeg, listDeg, waterT, inflowTpm, draftF, draftA (kernel/readouts.hpp:20-36). */
void sso_readouts(const sso_engine* e, double* r7);
/* Events as (t, id, kind) triples; returns the count. */
int sso_events(const sso_engine* e, double* out, int cap);
int sso_foundered(const sso_engine* e, double* founderT);
void sso_counters_get(const sso_engine* e, sso_counters* c);
/* Last step's flow per connection. */
void sso_flows(const sso_engine* e, double* q);

/* Hooks for the adjoint's test harness: pass(user, node, k, rec) after the k-th node pass of a node in a step's level
 * solve, rec = (level, vol, dv, mx, my, mz, zmin, zmax); solved(user) once the step's levels are solved, when
 * sso_solved_state reads the solved volumes, levels, areas, centroids, extent tops, merge flags, the step's pose
 * (R00 .. R22, tx, ty, tz, cth, 1 / R22) and buoyancy (V, x, y, z). */
typedef void (*sso_pass_hook)(void* user, int32_t node, int32_t k, const double* rec);
typedef void (*sso_solved_hook)(void* user);
void sso_set_hooks(sso_engine* e, sso_pass_hook pass, sso_solved_hook solved, void* user);
void sso_solved_state(const sso_engine* e, double* volS, double* levelS, double* areaS, double* cxS, double* cyS, double* czS, double* zmaxS,
                      int32_t* merged, double* pose14, double* buoy4);

/* The branch digest, for finite-difference checks of gradients: from sso_digest_start on, every discrete decision
 * of every step (per node pass the numbers of wet and partial segments, the Newton or bisection branch of every
 * level update, a flow that is zero or limited, a volume clipped at 0 or at its cap, an angle at its clamp) goes into
 * one FNV-1a hash. Two runs with the same digest took the same branch path: their difference is the derivative's. */
void sso_digest_start(sso_engine* e);
uint64_t sso_digest(const sso_engine* e);

#ifdef __cplusplus
}
#endif

#endif
