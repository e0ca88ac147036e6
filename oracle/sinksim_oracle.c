/* CPU restatement of the reference sinksim time step (portable and portable32 numerics), for parity testing only.
 * TEST INFRASTRUCTURE: see sinksim_oracle.h. Citations are to files of the reference repository.
 *
 * Compiled with -ffp-contract=off -fno-fast-math -fexcess-precision=standard, the reference's strict floating-point
 * flags (cmake/StrictFloatingPoint.cmake:12-17): every + and * below rounds once, in the order written.
 */
#include "sinksim_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* fdlibm 5.3 with fdlibm_ prefixes (third_party/fdlibm/fdlibm_api.h of the reference). */
double fdlibm_sin(double);
double fdlibm_cos(double);
double fdlibm_pow(double, double);

/* Scheme v1 constants (engine/include/sinksim/kernel/scheme.hpp:11-28). */
#define EMPTY_VOLUME 1e-6
#define FULL_FRACTION (1.0 - 1e-7)
#define LIMITER_SHARE 0.5
#define ORIFICE_HEAD_FLOOR 0.01
#define WEIR_COEFFICIENT (2.0 / 3.0)
#define WEIR_EXPONENT 1.5
#define VILLEMONTE_EXPONENT 0.385
#define NEWTON_FAST 6
#define SLOPE_MIN 1e-9
#define CENTROID_MIN_VOLUME 1e-9
#define NO_HEAD (-1e9)
#define NO_HEAD_TEST (-1e8)
#define PITCH_CLAMP 1.35
#define ROLL_CLAMP 1.4
#define PI_ 3.141592653589793

/* Math.max / Math.min of JavaScript for ordinary numbers: the first argument wins ties (kernel/math.hpp:29-30). */
static double jmax(double a, double b) { return (b > a) ? b : a; }
static double jmin(double a, double b) { return (b < a) ? b : a; }

typedef struct { double R00, R01, R02, R10, R11, R12, R20, R21, R22, tx, ty, tz, cth; } Pose;
typedef struct { double V, x, y, z, top; } Buoy;
typedef struct { double vol, dv, mx, my, mz, zmin, zmax; } Pass;
typedef struct { double V, Mx, My, Mz, top; } HPart;
typedef struct { float V, Mx, My, Mz, top; } HPartF;
typedef struct { float vol, dv, mx, my, mz, zmin, zmax; } PPartF;

struct sso_engine {
  int mixed;
  /* ship */
  int32_t ncol, nseg, nn;
  double *x, *y, *dxdy, *zlo, *zhi, *segA, *segE, *mu, *vmax, *amin, *aov;
  int32_t *segCol, *segStart, *segCount;
  /* sim */
  double rho, g, sq2g, dt;
  int32_t ng, nc, nmon, nmark;
  int32_t *gStart, *gCount, *gNodes;
  uint8_t* gMode;
  double *gpx, *gpy, *gpz, gMargin;
  int32_t *ca, *cb, *skip, *mon;
  uint8_t *law, *en;
  double *cx, *cy, *cz, *area, *coef, *tOn;
  double monThreshold;
  double *mkx, *mky, *mkz;
  uint8_t* mkWhen;
  double hullTopBelow, pitchAbsAbove, buoyancyBelow, minT;
  double ms, g0x, g0y, g0z, XO, YO, mh0, Ith0, Iph0, cDz, cDth, cDph, qz, qth, qph;
  double xFP, xAP;
  double st0[7];
  double *vol0, *level0, *cxs0, *cys0, *czs0;
  /* incidence (engine/src/model.cpp:26-56) */
  int32_t *incStart, *incCount, *incConn, *sea, nsea;
  uint8_t* incSide;
  /* state */
  double t, zO, pitch, roll, vz, wth, wph;
  double *vol, *level, *wcx, *wcy, *wcz;
  /* scratch */
  double *areaN, *zminN, *zmaxN, *hEff, *aEff, *acc, *excess, *q, *dV, *over;
  int32_t* deg;
  uint8_t* merged;
  Pass* passes;
  /* outputs */
  double inflow, Vb, hullTop, mw, bx, by, bz;
  /* events */
  int evCap, evCount;
  double* evT;
  int32_t* evId;
  int32_t* evKind;
  double *overT, *markT;
  int foundered;
  double founderT;
  sso_counters cnt;
  /* the adjoint harness's hooks (tests only): every node pass, and the moment the levels are solved */
  sso_pass_hook passHook;
  sso_solved_hook solvedHook;
  void* hookUser;
  int32_t* passSlot;
  double lastPose[14], lastBuoy[4];
  /* the branch digest (tests only, on while digestOn): FNV-1a over every discrete decision of every step */
  int digestOn;
  uint64_t digest;
};

/* Adds one decision code to the branch digest. */
static void decide(sso_engine* e, uint64_t code) {
  if (!e->digestOn) return;
  for (int k = 0; k < 8; ++k) { e->digest ^= (code >> (8 * k)) & 0xffu; e->digest *= 1099511628211ULL; }
}

#define DUP(dst, src, n, T)                                   \
  do {                                                        \
    size_t bytes_ = (size_t)(n) * sizeof(T) + 8;              \
    (dst) = (T*)malloc(bytes_);                               \
    if ((n) > 0) memcpy((dst), (src), (size_t)(n) * sizeof(T)); \
  } while (0)
#define ZERO(dst, n, T) ((dst) = (T*)calloc((size_t)(n) + 1, sizeof(T)))

/* ------------------------------------------------------------------ pose (kernel/frame.hpp:9-21) */
static Pose pose_at(const sso_engine* e, double zO, double th, double ph) {
  const double cth = fdlibm_cos(th), sth = fdlibm_sin(th), cph = fdlibm_cos(ph), sph = fdlibm_sin(ph);
  Pose F;
  F.R00 = cth; F.R01 = sth * sph; F.R02 = sth * cph;
  F.R10 = 0;   F.R11 = cph;       F.R12 = -sph;
  F.R20 = -sth; F.R21 = cth * sph; F.R22 = cth * cph;
  F.tx = e->XO - (F.R00 * e->g0x + F.R01 * e->g0y + F.R02 * e->g0z);
  F.ty = e->YO - (F.R10 * e->g0x + F.R11 * e->g0y + F.R12 * e->g0z);
  F.tz = zO - (F.R20 * e->g0x + F.R21 * e->g0y + F.R22 * e->g0z);
  F.cth = cth;
  return F;
}
static double wz_of(const Pose* F, double x, double y, double z) { return F->R20 * x + F->R21 * y + F->R22 * z + F->tz; }

/* ------------------------------------------------------------------ buoyancy (kernel/reduce.hpp:39-49, hydro.hpp:241-258) */
static void hcombine(HPart* a, const HPart* b) {
  a->V += b->V; a->Mx += b->Mx; a->My += b->My; a->Mz += b->Mz;
  if (b->top > a->top) a->top = b->top;
}
static void hcombine_f(HPartF* a, const HPartF* b) {
  a->V += b->V; a->Mx += b->Mx; a->My += b->My; a->Mz += b->Mz;
  if (b->top > a->top) a->top = b->top;
}

static Buoy buoyancy(sso_engine* e, const Pose* F) {
  HPart warps[8];
  if (!e->mixed) {
    const double iR = 1 / F->R22;
    for (int w = 0; w < 8; ++w) {
      HPart lane[32];
      for (int l = 0; l < 32; ++l) {
        HPart p = {0, 0, 0, 0, -1e9};
        for (int32_t i = w * 32 + l; i < e->ncol; i += 256) {
          const double x = e->x[i], y = e->y[i], lo = e->zlo[i], hi = e->zhi[i];
          const double base = F->R20 * x + F->R21 * y + F->tz;
          const double wt = base + F->R22 * hi;
          e->cnt.columns++;
          if (wt > p.top) p.top = wt;
          const double zp = -base * iR;
          if (zp <= lo) continue;
          e->cnt.colWet++;
          const double s = zp >= hi ? hi - lo : zp - lo;
          const double v = e->dxdy[i] * s;
          p.V += v; p.Mx += v * x; p.My += v * y; p.Mz += v * (lo + 0.5 * s);
        }
        lane[l] = p;
      }
      for (int off = 16; off > 0; off >>= 1)
        for (int l = 0; l < off; ++l) hcombine(&lane[l], &lane[l + off]);
      warps[w] = lane[0];
    }
  } else {
    const float R20 = (float)F->R20, R21 = (float)F->R21, R22 = (float)F->R22, tz = (float)F->tz;
    const float iR = 1.0f / R22;
    for (int w = 0; w < 8; ++w) {
      HPartF lane[32];
      for (int l = 0; l < 32; ++l) {
        HPartF p = {0.0f, 0.0f, 0.0f, 0.0f, -1e9f};
        for (int32_t i = w * 32 + l; i < e->ncol; i += 256) {
          const float x = (float)e->x[i], y = (float)e->y[i], lo = (float)e->zlo[i], hi = (float)e->zhi[i];
          const float base = R20 * x + R21 * y + tz;
          const float wt = base + R22 * hi;
          e->cnt.columns++;
          if (wt > p.top) p.top = wt;
          const float zp = -base * iR;
          if (zp <= lo) continue;
          e->cnt.colWet++;
          const float s = zp >= hi ? hi - lo : zp - lo;
          const float v = (float)e->dxdy[i] * s;
          p.V += v; p.Mx += v * x; p.My += v * y; p.Mz += v * (lo + 0.5f * s);
        }
        lane[l] = p;
      }
      for (int off = 16; off > 0; off >>= 1)
        for (int l = 0; l < off; ++l) hcombine_f(&lane[l], &lane[l + off]);
      warps[w].V = (double)lane[0].V; warps[w].Mx = (double)lane[0].Mx; warps[w].My = (double)lane[0].My;
      warps[w].Mz = (double)lane[0].Mz; warps[w].top = (double)lane[0].top;
    }
  }
  HPart tot = warps[0];
  for (int w = 1; w < 8; ++w) hcombine(&tot, &warps[w]);
  Buoy b;
  b.V = tot.V;
  b.x = tot.V > 0 ? tot.Mx / tot.V : 0;
  b.y = tot.V > 0 ? tot.My / tot.V : 0;
  b.z = tot.V > 0 ? tot.Mz / tot.V : 0;
  b.top = tot.top;
  return b;
}

/* ------------------------------------------------------------------ node pass (kernel/reduce.hpp:52-71, hydro.hpp:295-349) */
static void pcombine(Pass* a, const Pass* b) {
  a->vol += b->vol; a->dv += b->dv; a->mx += b->mx; a->my += b->my; a->mz += b->mz;
  if (b->zmin < a->zmin) a->zmin = b->zmin;
  if (b->zmax > a->zmax) a->zmax = b->zmax;
}
static void pcombine_f(PPartF* a, const PPartF* b) {
  a->vol += b->vol; a->dv += b->dv; a->mx += b->mx; a->my += b->my; a->mz += b->mz;
  if (b->zmin < a->zmin) a->zmin = b->zmin;
  if (b->zmax > a->zmax) a->zmax = b->zmax;
}

static Pass node_pass(sso_engine* e, const Pose* F, int32_t n, double h) {
  const int32_t s0 = e->segStart[n], s1 = s0 + e->segCount[n];
  const double iR = 1 / F->R22;
  Pass tot;
  e->cnt.passes++;
  if (!e->mixed) {
    Pass lane[32];
    for (int l = 0; l < 32; ++l) {
      Pass p = {0, 0, 0, 0, 0, 1e9, -1e9};
      for (int32_t j = s0 + l; j < s1; j += 32) {
        const int32_t i = e->segCol[j];
        const double x = e->x[i], y = e->y[i], a = e->segA[j], b = e->segE[j];
        const double base = F->R20 * x + F->R21 * y + F->tz;
        const double wa = base + F->R22 * a, wb = base + F->R22 * b;
        e->cnt.segVisits++;
        if (wa < p.zmin) p.zmin = wa;
        if (wb > p.zmax) p.zmax = wb;
        const double zp = (h - base) * iR;
        if (zp <= a) continue;
        e->cnt.segWet++;
        const double A = e->dxdy[i];
        double L;
        if (zp >= b) {
          L = b - a;
        } else {
          L = zp - a;
          p.dv += A;
        }
        const double v = A * L;
        p.vol += v; p.mx += v * x; p.my += v * y; p.mz += v * (a + 0.5 * L);
      }
      lane[l] = p;
    }
    for (int off = 16; off > 0; off >>= 1)
      for (int l = 0; l < off; ++l) pcombine(&lane[l], &lane[l + off]);
    tot = lane[0];
  } else {
    const float R20 = (float)F->R20, R21 = (float)F->R21, R22 = (float)F->R22, tz = (float)F->tz;
    const float fiR = 1.0f / R22;
    const float hf = (float)h;
    PPartF lane[32];
    for (int l = 0; l < 32; ++l) {
      PPartF p = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1e9f, -1e9f};
      for (int32_t j = s0 + l; j < s1; j += 32) {
        const int32_t i = e->segCol[j];
        const float x = (float)e->x[i], y = (float)e->y[i], a = (float)e->segA[j], b = (float)e->segE[j];
        const float base = R20 * x + R21 * y + tz;
        const float wa = base + R22 * a, wb = base + R22 * b;
        e->cnt.segVisits++;
        if (wa < p.zmin) p.zmin = wa;
        if (wb > p.zmax) p.zmax = wb;
        const float zp = (hf - base) * fiR;
        if (zp <= a) continue;
        e->cnt.segWet++;
        const float A = (float)e->dxdy[i];
        float L;
        if (zp >= b) {
          L = b - a;
        } else {
          L = zp - a;
          p.dv += A;
        }
        const float v = A * L;
        p.vol += v; p.mx += v * x; p.my += v * y; p.mz += v * (a + 0.5f * L);
      }
      lane[l] = p;
    }
    for (int off = 16; off > 0; off >>= 1)
      for (int l = 0; l < off; ++l) pcombine_f(&lane[l], &lane[l + off]);
    tot.vol = lane[0].vol; tot.dv = lane[0].dv; tot.mx = lane[0].mx; tot.my = lane[0].my; tot.mz = lane[0].mz;
    tot.zmin = lane[0].zmin; tot.zmax = lane[0].zmax;
  }
  const double mu = e->mu[n];
  Pass r;
  r.vol = tot.vol * mu;
  r.dv = tot.dv * mu * iR;
  r.mx = tot.mx * mu; r.my = tot.my * mu; r.mz = tot.mz * mu;
  r.zmin = tot.zmin; r.zmax = tot.zmax;
  if (e->digestOn) {
    /* which segments the level cuts (their count per lane tree is the regime of the pass), and which segment is the
       extent's bottom and top, as the numbers of partial segments and the extent's value bits do not say: count them */
    int64_t partial = 0, wet = 0;
    for (int32_t j = s0; j < s1; ++j) {
      const int32_t i = e->segCol[j];
      const double base = F->R20 * e->x[i] + F->R21 * e->y[i] + F->tz;
      const double zp = (h - base) * iR;
      if (zp > e->segA[j]) { ++wet; if (zp < e->segE[j]) ++partial; }
    }
    decide(e, (uint64_t)n << 40 ^ (uint64_t)wet << 20 ^ (uint64_t)partial);
  }
  if (e->passHook) {
    const double rec[8] = {h, r.vol, r.dv, r.mx, r.my, r.mz, r.zmin, r.zmax};
    e->passHook(e->hookUser, n, e->passSlot[n]++, rec);
  }
  return r;
}

/* ------------------------------------------------------------------ levels (kernel/levels.hpp:13-188) */
static void set_centroid(sso_engine* e, int32_t n, const Pass* p) {
  if (p->vol > CENTROID_MIN_VOLUME) { e->wcx[n] = p->mx / p->vol; e->wcy[n] = p->my / p->vol; e->wcz[n] = p->mz / p->vol; }
}

static void solve_single(sso_engine* e, const Pose* F, int32_t n) {
  const double V = e->vol[n], Vmax = e->vmax[n];
  double h = e->level[n];
  Pass p = node_pass(e, F, n, h);
  const double lo = p.zmin, hi = p.zmax;
  e->zminN[n] = lo; e->zmaxN[n] = hi;
  if (V <= EMPTY_VOLUME) { e->level[n] = lo; e->areaN[n] = 0; return; }
  if (V >= Vmax * FULL_FRACTION) {
    p = node_pass(e, F, n, hi);
    e->level[n] = hi + jmax(0.0, V - Vmax) / e->aov[n];
    e->areaN[n] = e->aov[n];
    set_centroid(e, n, &p);
    return;
  }
  if (h < lo || h > hi) {
    h = jmin(hi, jmax(lo, h));
    p = node_pass(e, F, n, h);
  }
  const double tol = jmax(1e-3 * Vmax, 0.5);
  double a = lo, b = hi;
  for (int it = 0; it < NEWTON_FAST; ++it) {
    const double err = p.vol - V;
    if (fabs(err) < tol) break;
    e->cnt.newton++;
    if (err > 0) b = h; else a = h;
    double hn = p.dv > SLOPE_MIN ? h - err / p.dv : 0.5 * (a + b);
    if (!(hn > a && hn < b)) hn = 0.5 * (a + b);
    decide(e, 0x60000000u + (uint64_t)n * 4 + (err > 0 ? 1u : 0u) + (hn == 0.5 * (a + b) ? 2u : 0u));
    h = hn;
    p = node_pass(e, F, n, h);
  }
  e->level[n] = h; e->areaN[n] = p.dv;
  set_centroid(e, n, &p);
}

static void solve_group(sso_engine* e, const Pose* F, const int32_t* m, int32_t N) {
  Pass* P = e->passes;
  double V = 0, Vmax = 0;
  for (int32_t k = 0; k < N; ++k) { V += e->vol[m[k]]; Vmax += e->vmax[m[k]]; }
  int allWet = 1;
  int32_t firstWet = -1;
  for (int32_t k = 0; k < N; ++k) {
    if (e->vol[m[k]] > 0) { if (firstWet < 0) firstWet = k; }
    else allWet = 0;
  }
  double h;
  if (allWet) {
    double s = 0;
    for (int32_t k = 0; k < N; ++k) s += e->level[m[k]];
    h = s / (double)N;
  } else {
    h = e->level[m[firstWet >= 0 ? firstWet : N - 1]];
  }
  for (int32_t k = 0; k < N; ++k) P[k] = node_pass(e, F, m[k], h);
  for (int32_t k = 0; k < N; ++k) { e->zminN[m[k]] = P[k].zmin; e->zmaxN[m[k]] = P[k].zmax; }
  double lo = P[0].zmin, hi = P[0].zmax;
  for (int32_t k = 1; k < N; ++k) { if (P[k].zmin < lo) lo = P[k].zmin; if (P[k].zmax > hi) hi = P[k].zmax; }

  if (V <= EMPTY_VOLUME) {
    for (int32_t k = 0; k < N; ++k) { e->vol[m[k]] = 0; e->level[m[k]] = P[k].zmin; e->areaN[m[k]] = 0; }
    return;
  }
  if (V >= Vmax * FULL_FRACTION) {
    const double over = jmax(0.0, V - Vmax);
    double aSum = 0;
    for (int32_t k = 0; k < N; ++k) aSum += e->aov[m[k]];
    const double dh = over / aSum;
    double assigned = 0;
    for (int32_t k = 0; k < N - 1; ++k) {
      const double v = e->vmax[m[k]] + dh * e->aov[m[k]];
      e->vol[m[k]] = v;
      assigned += v;
    }
    e->vol[m[N - 1]] = V - assigned;
    for (int32_t k = 0; k < N; ++k) {
      P[k] = node_pass(e, F, m[k], hi);
      e->level[m[k]] = hi + dh; e->areaN[m[k]] = e->aov[m[k]];
      set_centroid(e, m[k], &P[k]);
    }
    return;
  }
  if (!(h >= lo && h <= hi)) {
    h = jmin(hi, jmax(lo, h));
    for (int32_t k = 0; k < N; ++k) P[k] = node_pass(e, F, m[k], h);
  }
  const double tol = jmax(1e-3 * Vmax, 0.5);
  double a = lo, b = hi;
  for (int it = 0; it < NEWTON_FAST; ++it) {
    double sum = 0;
    for (int32_t k = 0; k < N; ++k) sum += P[k].vol;
    const double err = sum - V;
    if (fabs(err) < tol) break;
    e->cnt.newton++;
    if (err > 0) b = h; else a = h;
    double dv = 0;
    for (int32_t k = 0; k < N; ++k) dv += P[k].dv;
    double hn = dv > SLOPE_MIN ? h - err / dv : 0.5 * (a + b);
    if (!(hn > a && hn < b)) hn = 0.5 * (a + b);
    decide(e, 0x70000000u + (uint64_t)m[0] * 4 + (err > 0 ? 1u : 0u) + (hn == 0.5 * (a + b) ? 2u : 0u));
    h = hn;
    for (int32_t k = 0; k < N; ++k) P[k] = node_pass(e, F, m[k], h);
  }
  double tot = 0;
  for (int32_t k = 0; k < N; ++k) tot += P[k].vol;
  double assigned = 0;
  for (int32_t k = 0; k < N - 1; ++k) {
    double v = tot > 0 ? V * P[k].vol / tot : V / (double)N;
    if (v > e->vmax[m[k]]) v = e->vmax[m[k]];
    e->vol[m[k]] = v;
    assigned += v;
  }
  const double vmaxLast = e->vmax[m[N - 1]];
  if (V - assigned > vmaxLast) {
    const double need = V - vmaxLast;
    double capped = 0;
    for (int32_t k = N - 2; k >= 0; --k) {
      double prior = 0;
      for (int32_t j = 0; j < k; ++j) prior += e->vol[m[j]];
      const double v = (need - capped) - prior;
      if (v > e->vmax[m[k]] && k > 0) {
        e->vol[m[k]] = e->vmax[m[k]];
        capped += e->vmax[m[k]];
        continue;
      }
      e->vol[m[k]] = v;
      break;
    }
    assigned = 0;
    for (int32_t k = 0; k < N - 1; ++k) assigned += e->vol[m[k]];
  }
  e->vol[m[N - 1]] = V - assigned;
  for (int32_t k = 0; k < N; ++k) {
    e->level[m[k]] = h; e->areaN[m[k]] = P[k].dv;
    set_centroid(e, m[k], &P[k]);
  }
}

static void solve_levels(sso_engine* e, const Pose* F) {
  for (int32_t g = 0; g < e->ng; ++g) {
    const int32_t N = e->gCount[g];
    const int32_t* m = e->gNodes + e->gStart[g];
    int merged = 0;
    if (N >= 2) {
      if (e->gMode[g] == 1) {
        merged = 1;
      } else if (e->gMode[g] == 2) {
        const double zMw = wz_of(F, e->gpx[g], e->gpy[g], e->gpz[g]);
        merged = 1;
        for (int32_t k = 0; k < N; ++k)
          if (!(e->vol[m[k]] > EMPTY_VOLUME && e->level[m[k]] > zMw + e->gMargin)) { merged = 0; break; }
      }
    }
    e->merged[g] = (uint8_t)merged;
    if (merged) solve_group(e, F, m, N);
    else for (int32_t k = 0; k < N; ++k) solve_single(e, F, m[k]);
  }
}

/* ------------------------------------------------------------------ flows (kernel/flows.hpp:15-118) */
static double flow(sso_engine* e, const Pose* F, int32_t c) {
  if (!e->en[c] || e->tOn[c] > e->t) { e->q[c] = 0; return 0; }
  if (e->skip[c] >= 0 && e->merged[e->skip[c]]) { e->q[c] = 0; return 0; }
  const int32_t a = e->ca[c], b = e->cb[c];
  const double zo = F->R20 * e->cx[c] + F->R21 * e->cy[c] + F->R22 * e->cz[c] + F->tz;
  const double ha = a < 0 ? 0.0 : e->hEff[a], hbv = e->hEff[b];
  const double Ha = ha > zo ? ha - zo : 0.0, Hb = hbv > zo ? hbv - zo : 0.0;
  double q = 0;
  if (e->law[c] == 0) {
    e->cnt.orifice++;
    const double d = Ha - Hb;
    if (d != 0) q = e->coef[c] * e->area[c] * e->sq2g * d / sqrt(jmax(fabs(d), ORIFICE_HEAD_FLOOR));
  } else {
    e->cnt.weir++;
    const double H1 = Ha > Hb ? Ha : Hb;
    if (H1 > 0) {
      const double H2 = Ha > Hb ? Hb : Ha;
      double f = 1;
      if (H2 > 0) {
        const double r = H2 / H1;
        e->cnt.weirPow += 2;
        f = fdlibm_pow(jmax(0.0, 1 - fdlibm_pow(r, WEIR_EXPONENT)), VILLEMONTE_EXPONENT);
      }
      q = e->coef[c] * e->area[c] * WEIR_COEFFICIENT * e->sq2g * H1 * sqrt(H1) * f * (Ha >= Hb ? 1.0 : -1.0);
    }
  }
  if (q == 0) { e->q[c] = 0; decide(e, 0x10000000u + (uint64_t)c); return 0; }
  double dV = q * e->dt;
  const int32_t src = dV > 0 ? a : b, dst = dV > 0 ? b : a;
  const double hs = src < 0 ? 0.0 : e->hEff[src];
  const double hd = dst < 0 ? 0.0 : e->hEff[dst];
  const double inv = (src < 0 ? 0.0 : 1 / e->aEff[src]) + (dst < 0 ? 0.0 : 1 / e->aEff[dst]);
  const int32_t degRef = src < 0 ? e->deg[dst] : (dst < 0 ? e->deg[src] : (e->deg[src] > e->deg[dst] ? e->deg[src] : e->deg[dst]));
  const double share = LIMITER_SHARE / (double)(degRef > 1 ? degRef : 1);
  double lim = inv > 0 ? share * (hs - jmax(hd, zo)) / inv : fabs(dV);
  decide(e, 0x20000000u + (uint64_t)c * 8 + (lim < 0 ? 1u : 0u) + (fabs(dV) > (lim < 0 ? 0 : lim) ? 2u : 0u) + (dV > 0 ? 4u : 0u));
  if (lim < 0) lim = 0;
  if (fabs(dV) > lim) dV = dV > 0 ? lim : -lim;
  e->q[c] = dV / e->dt;
  return dV;
}

static double flows_and_volumes(sso_engine* e, const Pose* F) {
  const int32_t NN = e->nn;
  for (int32_t n = 0; n < NN; ++n) {
    e->hEff[n] = e->vol[n] > EMPTY_VOLUME ? e->level[n] : NO_HEAD;
    e->aEff[n] = e->vol[n] >= e->vmax[n] ? e->aov[n] : jmax(e->areaN[n], e->amin[n]);
  }
  for (int32_t n = 0; n < NN; ++n) {
    int32_t d = 0;
    for (int32_t k = e->incStart[n]; k < e->incStart[n] + e->incCount[n]; ++k) {
      const int32_t c = e->incConn[k];
      if (!e->en[c]) continue;
      const int32_t a = e->ca[c], b = e->cb[c];
      if (a >= 0 && e->hEff[a] < NO_HEAD_TEST && e->hEff[b] < NO_HEAD_TEST) continue;
      ++d;
    }
    e->deg[n] = d;
  }
  for (int32_t c = 0; c < e->nc; ++c) e->dV[c] = flow(e, F, c);
  for (int32_t n = 0; n < NN; ++n) {
    double a = 0;
    for (int32_t k = e->incStart[n]; k < e->incStart[n] + e->incCount[n]; ++k) {
      const double d = e->dV[e->incConn[k]];
      a = e->incSide[k] ? a + d : a - d;
    }
    e->acc[n] = a;
  }
  double seaIn = 0;
  for (int32_t k = 0; k < e->nsea; ++k) seaIn += e->dV[e->sea[k]];
  for (int32_t n = 0; n < NN; ++n) {
    double v = e->vol[n] + e->acc[n];
    if (v < 0) { v = 0; decide(e, 0x30000000u + (uint64_t)n); }
    const double vm = e->vmax[n];
    double excess = 0;
    if (v > vm) {
      const double head = jmax(0.0, -e->zmaxN[n]);
      const double cap = vm + e->aov[n] * head;
      if (v > cap) { excess = v - cap; v = cap; decide(e, 0x40000000u + (uint64_t)n); }
    }
    e->excess[n] = excess;
    e->vol[n] = v;
  }
  for (int32_t n = 0; n < NN; ++n)
    if (e->excess[n] > 0) seaIn -= e->excess[n];
  return seaIn;
}

/* ------------------------------------------------------------------ body and events (kernel/body.hpp, events.hpp) */
static void push_event(sso_engine* e, double t, int32_t id, int32_t kind) {
  if (e->evCount < e->evCap) {
    e->evT[e->evCount] = t; e->evId[e->evCount] = id; e->evKind[e->evCount] = kind;
    e->evCount++;
  }
}

static void body_and_events(sso_engine* e, const Pose* F, const Buoy* hb) {
  const double W = e->rho * e->g;
  const double Fb = W * hb->V;
  const double bxw = F->R00 * hb->x + F->R01 * hb->y + F->R02 * hb->z + F->tx;
  const double byw = F->R10 * hb->x + F->R11 * hb->y + F->R12 * hb->z + F->ty;
  double tauX = (byw - e->YO) * Fb, tauY = -(bxw - e->XO) * Fb;
  double Fz = Fb - e->g * e->ms;
  double mw = 0, Iw_p = 0, Iw_r = 0;
  for (int32_t n = 0; n < e->nn; ++n) {
    const double V = e->vol[n];
    if (V <= 0) continue;
    const double x = e->wcx[n], y = e->wcy[n], z = e->wcz[n];
    const double wx = F->R00 * x + F->R01 * y + F->R02 * z + F->tx - e->XO;
    const double wy = F->R10 * x + F->R11 * y + F->R12 * z + F->ty - e->YO;
    const double wz = F->R20 * x + F->R21 * y + F->R22 * z + F->tz - e->zO;
    const double f = -W * V;
    tauX += wy * f; tauY -= wx * f; Fz += f;
    const double m = e->rho * V;
    mw += m;
    Iw_p += m * (wx * wx + wz * wz);
    Iw_r += m * (wy * wy + wz * wz);
  }
  const double Mth = tauY, Mph = tauX * F->cth;
  /* integrate (body.hpp:42-57) */
  const double dt = e->dt;
  const double mh = e->mh0 + mw;
  const double Ith = e->Ith0 + Iw_p, Iph = e->Iph0 + Iw_r;
  const double az = (Fz - e->cDz * e->vz - e->qz * fabs(e->vz) * e->vz) / mh;
  const double ath = (Mth - e->cDth * e->wth - e->qth * fabs(e->wth) * e->wth) / Ith;
  const double aph = (Mph - e->cDph * e->wph - e->qph * fabs(e->wph) * e->wph) / Iph;
  e->vz += az * dt; e->wth += ath * dt; e->wph += aph * dt;
  e->zO += e->vz * dt; e->pitch += e->wth * dt; e->roll += e->wph * dt;
  decide(e, 0x50000000u + (uint64_t)(e->pitch > PITCH_CLAMP) + 2u * (uint64_t)(e->pitch < -PITCH_CLAMP) + 4u * (uint64_t)(e->roll > ROLL_CLAMP) +
                8u * (uint64_t)(e->roll < -ROLL_CLAMP));
  if (e->pitch > PITCH_CLAMP) { e->pitch = PITCH_CLAMP; e->wth = 0; }
  if (e->pitch < -PITCH_CLAMP) { e->pitch = -PITCH_CLAMP; e->wth = 0; }
  if (e->roll > ROLL_CLAMP) { e->roll = ROLL_CLAMP; e->wph = 0; }
  if (e->roll < -ROLL_CLAMP) { e->roll = -ROLL_CLAMP; e->wph = 0; }
  e->t += dt;
  e->Vb = hb->V; e->hullTop = hb->top; e->mw = mw;
  e->bx = hb->x; e->by = hb->y; e->bz = hb->z;
  /* events (events.hpp:11-38) */
  for (int32_t m = 0; m < e->nmon; ++m) e->over[m] = 0;
  for (int32_t c = 0; c < e->nc; ++c)
    if (e->mon[c] >= 0 && e->q[c] > 0) e->over[e->mon[c]] += e->q[c];
  for (int32_t m = 0; m < e->nmon; ++m)
    if (e->over[m] > e->monThreshold && e->overT[m] < 0) { e->overT[m] = e->t; push_event(e, e->t, m, 0); }
  for (int32_t i = 0; i < e->nmark; ++i) {
    if (e->markT[i] >= 0) continue;
    const double wz = wz_of(F, e->mkx[i], e->mky[i], e->mkz[i]);
    const int under = e->mkWhen[i] == 0;
    if ((under && wz < 0) || (!under && wz > 0)) { e->markT[i] = e->t; push_event(e, e->t, i, 1); }
  }
  if (!e->foundered && (e->hullTop < e->hullTopBelow || fabs(e->pitch) > e->pitchAbsAbove ||
                        (e->Vb < e->buoyancyBelow && e->t > e->minT))) {
    e->foundered = 1;
    e->founderT = e->t;
    push_event(e, e->t, -1, 2);
  }
}

/* ------------------------------------------------------------------ one step (kernel/step.hpp:41-54) */
static void step_once(sso_engine* e) {
  const Pose F = pose_at(e, e->zO, e->pitch, e->roll);
  const Buoy hb = buoyancy(e, &F);
  if (e->passHook) {
    const double p[14] = {F.R00, F.R01, F.R02, F.R10, F.R11, F.R12, F.R20, F.R21, F.R22, F.tx, F.ty, F.tz, F.cth, 1 / F.R22};
    memcpy(e->lastPose, p, sizeof p);
    e->lastBuoy[0] = hb.V; e->lastBuoy[1] = hb.x; e->lastBuoy[2] = hb.y; e->lastBuoy[3] = hb.z;
    for (int32_t n = 0; n < e->nn; ++n) e->passSlot[n] = 0;
  }
  solve_levels(e, &F);
  if (e->solvedHook) e->solvedHook(e->hookUser);
  const double seaIn = flows_and_volumes(e, &F);
  e->inflow = seaIn / e->dt;
  body_and_events(e, &F, &hb);
  e->cnt.steps++;
}

static void evaluate_hydro(sso_engine* e) {
  const Pose F = pose_at(e, e->zO, e->pitch, e->roll);
  const Buoy hb = buoyancy(e, &F);
  e->inflow = 0;
  e->Vb = hb.V; e->hullTop = hb.top;
  e->bx = hb.x; e->by = hb.y; e->bz = hb.z;
  double mw = 0;
  for (int32_t n = 0; n < e->nn; ++n) mw += e->rho * e->vol[n];
  e->mw = mw;
}

static void clear_events(sso_engine* e) {
  e->evCount = 0;
  e->foundered = 0;
  e->founderT = -1;
  for (int32_t m = 0; m < e->nmon; ++m) e->overT[m] = -1;
  for (int32_t i = 0; i < e->nmark; ++i) e->markT[i] = -1;
}

/* ------------------------------------------------------------------ public API */
sso_engine* sso_create(const sso_ship* S, const sso_sim* M, int mixed) {
  sso_engine* e = (sso_engine*)calloc(1, sizeof(sso_engine));
  e->mixed = mixed;
  e->ncol = S->ncol; e->nseg = S->nseg; e->nn = S->nnode;
  DUP(e->x, S->x, S->ncol, double); DUP(e->y, S->y, S->ncol, double); DUP(e->dxdy, S->dxdy, S->ncol, double);
  DUP(e->zlo, S->zlo, S->ncol, double); DUP(e->zhi, S->zhi, S->ncol, double);
  DUP(e->segCol, S->segCol, S->nseg, int32_t); DUP(e->segA, S->segA, S->nseg, double); DUP(e->segE, S->segE, S->nseg, double);
  DUP(e->mu, S->mu, S->nnode, double); DUP(e->vmax, S->vmax, S->nnode, double); DUP(e->amin, S->amin, S->nnode, double);
  DUP(e->aov, S->aov, S->nnode, double); DUP(e->segStart, S->segStart, S->nnode, int32_t); DUP(e->segCount, S->segCount, S->nnode, int32_t);

  e->rho = M->rho; e->g = M->g; e->sq2g = sqrt(2 * M->g); e->dt = M->dt;
  e->ng = M->ngroup;
  DUP(e->gStart, M->gStart, M->ngroup, int32_t); DUP(e->gCount, M->gCount, M->ngroup, int32_t);
  int32_t members = 0, maxGroup = 1;
  for (int32_t g = 0; g < M->ngroup; ++g) {
    if (M->gStart[g] + M->gCount[g] > members) members = M->gStart[g] + M->gCount[g];
    if (M->gCount[g] > maxGroup) maxGroup = M->gCount[g];
  }
  DUP(e->gNodes, M->gNodes, members, int32_t); DUP(e->gMode, M->gMode, M->ngroup, uint8_t);
  DUP(e->gpx, M->gpx, M->ngroup, double); DUP(e->gpy, M->gpy, M->ngroup, double); DUP(e->gpz, M->gpz, M->ngroup, double);
  e->gMargin = M->gMargin;
  e->nc = M->nconn;
  DUP(e->ca, M->ca, M->nconn, int32_t); DUP(e->cb, M->cb, M->nconn, int32_t); DUP(e->law, M->law, M->nconn, uint8_t);
  DUP(e->cx, M->cx, M->nconn, double); DUP(e->cy, M->cy, M->nconn, double); DUP(e->cz, M->cz, M->nconn, double);
  DUP(e->area, M->area, M->nconn, double); DUP(e->coef, M->coef, M->nconn, double); DUP(e->en, M->en, M->nconn, uint8_t);
  DUP(e->tOn, M->tOn, M->nconn, double); DUP(e->skip, M->skipGroup, M->nconn, int32_t); DUP(e->mon, M->monitor, M->nconn, int32_t);
  e->nmon = M->nmon; e->monThreshold = M->monThreshold;
  e->nmark = M->nmark;
  DUP(e->mkx, M->mkx, M->nmark, double); DUP(e->mky, M->mky, M->nmark, double); DUP(e->mkz, M->mkz, M->nmark, double);
  DUP(e->mkWhen, M->mkWhen, M->nmark, uint8_t);
  e->hullTopBelow = M->hullTopBelow; e->pitchAbsAbove = M->pitchAbsAbove; e->buoyancyBelow = M->buoyancyBelow; e->minT = M->minT;
  e->ms = M->body[0]; e->g0x = M->body[2]; e->g0y = M->body[3]; e->g0z = M->body[4]; e->XO = M->body[5]; e->YO = M->body[6];
  e->mh0 = M->body[7]; e->Ith0 = M->body[8]; e->Iph0 = M->body[9]; e->cDz = M->body[10]; e->cDth = M->body[11]; e->cDph = M->body[12];
  e->qz = M->body[13]; e->qth = M->body[14]; e->qph = M->body[15];
  e->xFP = M->xFP; e->xAP = M->xAP;
  memcpy(e->st0, M->state0, sizeof e->st0);
  DUP(e->vol0, M->vol0, S->nnode, double); DUP(e->level0, M->level0, S->nnode, double);
  DUP(e->cxs0, M->cx0, S->nnode, double); DUP(e->cys0, M->cy0, S->nnode, double); DUP(e->czs0, M->cz0, S->nnode, double);

  /* incidence: per node its connections in increasing order, side 1 at the b end; the sea list (model.cpp:26-56) */
  const int32_t NN = e->nn;
  ZERO(e->incCount, NN, int32_t); ZERO(e->incStart, NN, int32_t);
  for (int32_t c = 0; c < e->nc; ++c) { if (e->ca[c] >= 0) e->incCount[e->ca[c]]++; e->incCount[e->cb[c]]++; }
  int32_t total = 0;
  for (int32_t n = 0; n < NN; ++n) { e->incStart[n] = total; total += e->incCount[n]; }
  ZERO(e->incConn, total, int32_t); ZERO(e->incSide, total, uint8_t); ZERO(e->sea, e->nc, int32_t);
  int32_t* fill;
  ZERO(fill, NN, int32_t);
  e->nsea = 0;
  for (int32_t c = 0; c < e->nc; ++c) {
    if (e->ca[c] >= 0) {
      const int32_t k = e->incStart[e->ca[c]] + fill[e->ca[c]]++;
      e->incConn[k] = c; e->incSide[k] = 0;
    } else {
      e->sea[e->nsea++] = c;
    }
    const int32_t k = e->incStart[e->cb[c]] + fill[e->cb[c]]++;
    e->incConn[k] = c; e->incSide[k] = 1;
  }
  free(fill);

  ZERO(e->vol, NN, double); ZERO(e->level, NN, double); ZERO(e->wcx, NN, double); ZERO(e->wcy, NN, double); ZERO(e->wcz, NN, double);
  ZERO(e->areaN, NN, double); ZERO(e->zminN, NN, double); ZERO(e->zmaxN, NN, double); ZERO(e->hEff, NN, double);
  ZERO(e->aEff, NN, double); ZERO(e->acc, NN, double); ZERO(e->excess, NN, double); ZERO(e->deg, NN, int32_t);
  ZERO(e->q, e->nc, double); ZERO(e->dV, e->nc, double); ZERO(e->over, e->nmon, double);
  ZERO(e->merged, e->ng, uint8_t); ZERO(e->passes, maxGroup, Pass);
  ZERO(e->passSlot, NN, int32_t);
  e->evCap = e->nmon + e->nmark + 1;
  ZERO(e->evT, e->evCap, double); ZERO(e->evId, e->evCap, int32_t); ZERO(e->evKind, e->evCap, int32_t);
  ZERO(e->overT, e->nmon, double); ZERO(e->markT, e->nmark, double);
  sso_reset(e);
  return e;
}

void sso_reset(sso_engine* e) {
  e->t = e->st0[0]; e->zO = e->st0[1]; e->pitch = e->st0[2]; e->roll = e->st0[3];
  e->vz = e->st0[4]; e->wth = e->st0[5]; e->wph = e->st0[6];
  for (int32_t n = 0; n < e->nn; ++n) {
    e->vol[n] = e->vol0[n]; e->level[n] = e->level0[n];
    e->wcx[n] = e->cxs0[n]; e->wcy[n] = e->cys0[n]; e->wcz[n] = e->czs0[n];
    e->areaN[n] = 0;
  }
  for (int32_t c = 0; c < e->nc; ++c) { e->q[c] = 0; e->dV[c] = 0; }
  for (int32_t g = 0; g < e->ng; ++g) e->merged[g] = 0;
  clear_events(e);
  evaluate_hydro(e);
}

void sso_destroy(sso_engine* e) {
  if (!e) return;
  void* bufs[] = {e->x, e->y, e->dxdy, e->zlo, e->zhi, e->segA, e->segE, e->mu, e->vmax, e->amin, e->aov, e->segCol, e->segStart,
                  e->segCount, e->gStart, e->gCount, e->gNodes, e->gMode, e->gpx, e->gpy, e->gpz, e->ca, e->cb, e->skip, e->mon,
                  e->law, e->en, e->cx, e->cy, e->cz, e->area, e->coef, e->tOn, e->mkx, e->mky, e->mkz, e->mkWhen, e->vol0,
                  e->level0, e->cxs0, e->cys0, e->czs0, e->incStart, e->incCount, e->incConn, e->sea, e->incSide, e->vol,
                  e->level, e->wcx, e->wcy, e->wcz, e->areaN, e->zminN, e->zmaxN, e->hEff, e->aEff, e->acc, e->excess, e->q,
                  e->dV, e->over, e->deg, e->merged, e->passes, e->evT, e->evId, e->evKind, e->overT, e->markT,
                  e->passSlot};
  for (size_t i = 0; i < sizeof bufs / sizeof bufs[0]; ++i) free(bufs[i]);
  free(e);
}

void sso_set_connection(sso_engine* e, int32_t c, int enabled, double area, double tOn) {
  if (c < 0 || c >= e->nc) return;
  if (enabled >= 0) e->en[c] = (uint8_t)(enabled != 0);
  if (!isnan(area)) e->area[c] = area;
  if (!isnan(tOn)) e->tOn[c] = tOn;
}

void sso_step(sso_engine* e, int64_t n) {
  for (int64_t i = 0; i < n; ++i) step_once(e);
}

void sso_get_record(const sso_engine* e, double* r) {
  const int32_t N = e->nn;
  r[0] = e->t; r[1] = e->zO; r[2] = e->pitch; r[3] = e->roll; r[4] = e->vz; r[5] = e->wth; r[6] = e->wph;
  r[7] = e->inflow; r[8] = e->Vb; r[9] = e->hullTop;
  for (int32_t n = 0; n < N; ++n) {
    r[10 + n] = e->vol[n]; r[10 + N + n] = e->level[n];
    r[10 + 2 * N + n] = e->wcx[n]; r[10 + 3 * N + n] = e->wcy[n]; r[10 + 4 * N + n] = e->wcz[n];
  }
}

void sso_restore(sso_engine* e, const double* r) {
  const int32_t N = e->nn;
  e->t = r[0]; e->zO = r[1]; e->pitch = r[2]; e->roll = r[3]; e->vz = r[4]; e->wth = r[5]; e->wph = r[6];
  for (int32_t n = 0; n < N; ++n) {
    e->vol[n] = r[10 + n]; e->level[n] = r[10 + N + n];
    e->wcx[n] = r[10 + 2 * N + n]; e->wcy[n] = r[10 + 3 * N + n]; e->wcz[n] = r[10 + 4 * N + n];
  }
  clear_events(e);
}

void sso_readouts(const sso_engine* e, double* r7) {
  const Pose F = pose_at(e, e->zO, e->pitch, e->roll);
  r7[0] = e->t;
  r7[1] = e->pitch * 180 / PI_;
  r7[2] = e->roll * 180 / PI_;
  double water = 0;
  for (int32_t n = 0; n < e->nn; ++n) water += e->vol[n];
  r7[3] = water * e->rho / 1000;
  r7[4] = e->inflow * e->rho / 1000 * 60;
  r7[5] = -wz_of(&F, e->xFP, 0, 0);
  r7[6] = -wz_of(&F, e->xAP, 0, 0);
}

int sso_events(const sso_engine* e, double* out, int cap) {
  for (int i = 0; i < e->evCount && i < cap; ++i) { out[3 * i] = e->evT[i]; out[3 * i + 1] = e->evId[i]; out[3 * i + 2] = e->evKind[i]; }
  return e->evCount;
}

int sso_foundered(const sso_engine* e, double* founderT) {
  *founderT = e->founderT;
  return e->foundered;
}

void sso_counters_get(const sso_engine* e, sso_counters* c) { *c = e->cnt; }

void sso_flows(const sso_engine* e, double* q) { memcpy(q, e->q, (size_t)e->nc * sizeof(double)); }

void sso_set_hooks(sso_engine* e, sso_pass_hook pass, sso_solved_hook solved, void* user) {
  e->passHook = pass;
  e->solvedHook = solved;
  e->hookUser = user;
}

void sso_solved_state(const sso_engine* e, double* volS, double* levelS, double* areaS, double* cxS, double* cyS, double* czS, double* zmaxS,
                      int32_t* merged, double* pose14, double* buoy4) {
  for (int32_t n = 0; n < e->nn; ++n) {
    volS[n] = e->vol[n]; levelS[n] = e->level[n]; areaS[n] = e->areaN[n];
    cxS[n] = e->wcx[n]; cyS[n] = e->wcy[n]; czS[n] = e->wcz[n]; zmaxS[n] = e->zmaxN[n];
  }
  for (int32_t g = 0; g < e->ng; ++g) merged[g] = e->merged[g];
  memcpy(pose14, e->lastPose, sizeof e->lastPose);
  memcpy(buoy4, e->lastBuoy, sizeof e->lastBuoy);
}

void sso_digest_start(sso_engine* e) {
  e->digestOn = 1;
  e->digest = 14695981039346656037ULL;
}

uint64_t sso_digest(const sso_engine* e) { return e->digest; }
