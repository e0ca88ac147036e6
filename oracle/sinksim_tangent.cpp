// Tangent-linear restatement of the portable step over forward-mode dual numbers. TEST INFRASTRUCTURE: see
// sinksim_tangent.h. Every value operation below is the operation of sinksim_oracle.c (and so of the reference's
// kernel::step<PortableMath, Order::Tree>, engine/include/sinksim/kernel/step.hpp:41-54) in the same order; compiled
// with the reference's strict floating-point flags, the value parts equal the oracle's bits.
#include "sinksim_tangent.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

extern "C" {
double fdlibm_sin(double);
double fdlibm_cos(double);
double fdlibm_pow(double, double);
}

namespace {

constexpr int P = SST_MAX_PARAMS;

// ------------------------------------------------------------------------------------------- the dual number
struct D {
  double v;
  double d[P];
  D() : v(0) { std::memset(d, 0, sizeof d); }
  D(double x) : v(x) { std::memset(d, 0, sizeof d); }  // NOLINT: constants lift implicitly
};

inline D operator+(const D& a, const D& b) { D r(a.v + b.v); for (int p = 0; p < P; ++p) r.d[p] = a.d[p] + b.d[p]; return r; }
inline D operator-(const D& a, const D& b) { D r(a.v - b.v); for (int p = 0; p < P; ++p) r.d[p] = a.d[p] - b.d[p]; return r; }
inline D operator-(const D& a) { D r(-a.v); for (int p = 0; p < P; ++p) r.d[p] = -a.d[p]; return r; }
inline D operator*(const D& a, const D& b) {
  D r(a.v * b.v);
  for (int p = 0; p < P; ++p) r.d[p] = a.d[p] * b.v + a.v * b.d[p];
  return r;
}
inline D operator/(const D& a, const D& b) {
  D r(a.v / b.v);
  for (int p = 0; p < P; ++p) r.d[p] = (a.d[p] - r.v * b.d[p]) / b.v;
  return r;
}
inline D& operator+=(D& a, const D& b) { a = a + b; return a; }
inline D& operator-=(D& a, const D& b) { a = a - b; return a; }
inline bool operator<(const D& a, const D& b) { return a.v < b.v; }
inline bool operator>(const D& a, const D& b) { return a.v > b.v; }
inline bool operator<=(const D& a, const D& b) { return a.v <= b.v; }
inline bool operator>=(const D& a, const D& b) { return a.v >= b.v; }
inline bool operator!=(const D& a, const D& b) { return a.v != b.v; }

// chain rule with a given derivative f'(x)
inline D apply(double fx, double dfx, const D& x) {
  D r(fx);
  for (int p = 0; p < P; ++p) r.d[p] = dfx * x.d[p];
  return r;
}
inline D dsqrt(const D& x) { const double s = std::sqrt(x.v); return apply(s, s > 0 ? 0.5 / s : 0.0, x); }
inline D dfabs(const D& x) { return x.v < 0 ? -x : x; }
inline D dsin(const D& x) { return apply(fdlibm_sin(x.v), fdlibm_cos(x.v), x); }
inline D dcos(const D& x) { return apply(fdlibm_cos(x.v), -fdlibm_sin(x.v), x); }
// x^y for a constant y: y x^(y-1) = y x^y / x; at x = 0 the derivative is taken as 0 (the adjoint does the same)
inline D dpow(const D& x, double y) {
  const double f = fdlibm_pow(x.v, y);
  return apply(f, x.v != 0 ? y * f / x.v : 0.0, x);
}
// JavaScript Math.max / Math.min: the first argument wins ties (kernel/math.hpp:29-30); the derivative follows the pick
inline D jmax(const D& a, const D& b) { return (b > a) ? b : a; }
inline D jmin(const D& a, const D& b) { return (b < a) ? b : a; }

constexpr double EMPTY_VOLUME = 1e-6, FULL_FRACTION = 1.0 - 1e-7, LIMITER_SHARE = 0.5, ORIFICE_HEAD_FLOOR = 0.01;
constexpr double WEIR_COEFFICIENT = 2.0 / 3.0, WEIR_EXPONENT = 1.5, VILLEMONTE_EXPONENT = 0.385, SLOPE_MIN = 1e-9;
constexpr double CENTROID_MIN_VOLUME = 1e-9, NO_HEAD = -1e9, NO_HEAD_TEST = -1e8, PITCH_CLAMP = 1.35, ROLL_CLAMP = 1.4;
constexpr double PI_ = 3.141592653589793;
constexpr int NEWTON_FAST = 6;

struct Pose { D R00, R01, R02, R10, R11, R12, R20, R21, R22, tx, ty, tz, cth; };
struct Buoy { D V, x, y, z, top; };
struct Pass { D vol, dv, mx, my, mz, zmin, zmax; };

}  // namespace

struct sst_engine {
  // ship
  int32_t ncol, nseg, nn;
  std::vector<double> x, y, dxdy, zlo, zhi, segA, segE, mu, vmax, amin, aov;
  std::vector<int32_t> segCol, segStart, segCount;
  // sim
  double rho, g, sq2g, dt;
  int32_t ng, nc;
  std::vector<int32_t> gStart, gCount, gNodes, ca, cb, skip;
  std::vector<uint8_t> gMode, law, en;
  std::vector<double> gpx, gpy, gpz, kx, ky, kz, coef, tOn;
  double gMargin;
  double hullTopBelow, pitchAbsAbove, buoyancyBelow, minT;
  double ms, g0x, g0y, g0z, XO, YO, mh0, Ith0, Iph0, cDz, cDth, cDph, qz, qth, qph, xFP, xAP;
  std::vector<int32_t> incStart, incCount, incConn, sea;
  std::vector<uint8_t> incSide;
  // parameters: the areas, with their tangents
  std::vector<D> area;
  // state
  double t;
  D zO, pitch, roll, vz, wth, wph;
  std::vector<D> vol, level, wcx, wcy, wcz;
  // scratch
  std::vector<D> areaN, zmaxN, hEff, aEff, dV;
  std::vector<int32_t> deg;
  std::vector<uint8_t> merged;
  std::vector<Pass> passes;
  D inflow;
  int foundered;
};

namespace {

Pose pose_at(const sst_engine* e, const D& zO, const D& th, const D& ph) {
  const D cth = dcos(th), sth = dsin(th), cph = dcos(ph), sph = dsin(ph);
  Pose F;
  F.R00 = cth; F.R01 = sth * sph; F.R02 = sth * cph;
  F.R10 = D(0); F.R11 = cph; F.R12 = -sph;
  F.R20 = -sth; F.R21 = cth * sph; F.R22 = cth * cph;
  F.tx = D(e->XO) - (F.R00 * e->g0x + F.R01 * e->g0y + F.R02 * e->g0z);
  F.ty = D(e->YO) - (F.R10 * e->g0x + F.R11 * e->g0y + F.R12 * e->g0z);
  F.tz = zO - (F.R20 * e->g0x + F.R21 * e->g0y + F.R22 * e->g0z);
  F.cth = cth;
  return F;
}

D wz_of(const Pose& F, double x, double y, double z) { return F.R20 * x + F.R21 * y + F.R22 * z + F.tz; }

// Buoyancy in the GPU's order: 256 partials (partial p sums columns p, p + 256, ...), the halving tree per 32, the
// eight results in order (kernel/reduce.hpp:39-49, hydro.hpp:241-258).
Buoy buoyancy(const sst_engine* e, const Pose& F) {
  const D iR = D(1) / F.R22;
  D V[8], Mx[8], My[8], Mz[8], top[8];
  for (int w = 0; w < 8; ++w) {
    D lV[32], lMx[32], lMy[32], lMz[32], lTop[32];
    for (int l = 0; l < 32; ++l) {
      D pV(0), pMx(0), pMy(0), pMz(0), pTop(-1e9);
      for (int32_t i = w * 32 + l; i < e->ncol; i += 256) {
        const double x = e->x[i], y = e->y[i], lo = e->zlo[i], hi = e->zhi[i];
        const D base = F.R20 * x + F.R21 * y + F.tz;
        const D wt = base + F.R22 * hi;
        if (wt > pTop) pTop = wt;
        const D zp = -base * iR;
        if (zp <= D(lo)) continue;
        const D s = zp >= D(hi) ? D(hi - lo) : zp - lo;
        const D v = D(e->dxdy[i]) * s;
        pV += v; pMx += v * x; pMy += v * y; pMz += v * (D(lo) + D(0.5) * s);
      }
      lV[l] = pV; lMx[l] = pMx; lMy[l] = pMy; lMz[l] = pMz; lTop[l] = pTop;
    }
    for (int off = 16; off > 0; off >>= 1)
      for (int l = 0; l < off; ++l) {
        lV[l] += lV[l + off]; lMx[l] += lMx[l + off]; lMy[l] += lMy[l + off]; lMz[l] += lMz[l + off];
        if (lTop[l + off] > lTop[l]) lTop[l] = lTop[l + off];
      }
    V[w] = lV[0]; Mx[w] = lMx[0]; My[w] = lMy[0]; Mz[w] = lMz[0]; top[w] = lTop[0];
  }
  for (int w = 1; w < 8; ++w) {
    V[0] += V[w]; Mx[0] += Mx[w]; My[0] += My[w]; Mz[0] += Mz[w];
    if (top[w] > top[0]) top[0] = top[w];
  }
  Buoy b;
  b.V = V[0];
  b.x = V[0] > D(0) ? Mx[0] / V[0] : D(0);
  b.y = V[0] > D(0) ? My[0] / V[0] : D(0);
  b.z = V[0] > D(0) ? Mz[0] / V[0] : D(0);
  b.top = top[0];
  return b;
}

// Node pass in the tree order (kernel/reduce.hpp:52-71, hydro.hpp:295-316). The minimum and maximum carry the
// derivative of the segment the tree selects: within a lane the first strict improvement, in the tree the lower
// lane on ties, as the value comparisons already do.
Pass node_pass(const sst_engine* e, const Pose& F, int32_t n, const D& h) {
  const int32_t s0 = e->segStart[n], s1 = s0 + e->segCount[n];
  const D iR = D(1) / F.R22;
  Pass lane[32];
  for (int l = 0; l < 32; ++l) {
    Pass p;
    p.vol = D(0); p.dv = D(0); p.mx = D(0); p.my = D(0); p.mz = D(0); p.zmin = D(1e9); p.zmax = D(-1e9);
    for (int32_t j = s0 + l; j < s1; j += 32) {
      const int32_t i = e->segCol[j];
      const double x = e->x[i], y = e->y[i], a = e->segA[j], b = e->segE[j];
      const D base = F.R20 * x + F.R21 * y + F.tz;
      const D wa = base + F.R22 * a, wb = base + F.R22 * b;
      if (wa < p.zmin) p.zmin = wa;
      if (wb > p.zmax) p.zmax = wb;
      const D zp = (h - base) * iR;
      if (zp <= D(a)) continue;
      const double A = e->dxdy[i];
      D L;
      if (zp >= D(b)) {
        L = D(b - a);
      } else {
        L = zp - a;
        p.dv += D(A);
      }
      const D v = D(A) * L;
      p.vol += v; p.mx += v * x; p.my += v * y; p.mz += v * (D(a) + D(0.5) * L);
    }
    lane[l] = p;
  }
  for (int off = 16; off > 0; off >>= 1)
    for (int l = 0; l < off; ++l) {
      Pass& a = lane[l];
      const Pass& b = lane[l + off];
      a.vol += b.vol; a.dv += b.dv; a.mx += b.mx; a.my += b.my; a.mz += b.mz;
      if (b.zmin < a.zmin) a.zmin = b.zmin;
      if (b.zmax > a.zmax) a.zmax = b.zmax;
    }
  const double mu = e->mu[n];
  Pass r;
  r.vol = lane[0].vol * mu;
  r.dv = lane[0].dv * mu * iR;
  r.mx = lane[0].mx * mu; r.my = lane[0].my * mu; r.mz = lane[0].mz * mu;
  r.zmin = lane[0].zmin; r.zmax = lane[0].zmax;
  return r;
}

void set_centroid(sst_engine* e, int32_t n, const Pass& p) {
  if (p.vol > D(CENTROID_MIN_VOLUME)) { e->wcx[n] = p.mx / p.vol; e->wcy[n] = p.my / p.vol; e->wcz[n] = p.mz / p.vol; }
}

// kernel/levels.hpp:13-49
void solve_single(sst_engine* e, const Pose& F, int32_t n) {
  const D V = e->vol[n];
  const double Vmax = e->vmax[n];
  D h = e->level[n];
  Pass p = node_pass(e, F, n, h);
  const D lo = p.zmin, hi = p.zmax;
  e->zmaxN[n] = hi;
  if (V <= D(EMPTY_VOLUME)) { e->level[n] = lo; e->areaN[n] = D(0); return; }
  if (V >= D(Vmax * FULL_FRACTION)) {
    p = node_pass(e, F, n, hi);
    e->level[n] = hi + jmax(D(0.0), V - Vmax) / e->aov[n];
    e->areaN[n] = D(e->aov[n]);
    set_centroid(e, n, p);
    return;
  }
  if (h < lo || h > hi) {
    h = jmin(hi, jmax(lo, h));
    p = node_pass(e, F, n, h);
  }
  const double tol = (0.5 > 1e-3 * Vmax) ? 0.5 : 1e-3 * Vmax;  // jmax(1e-3 Vmax, 0.5)
  D a = lo, b = hi;
  for (int it = 0; it < NEWTON_FAST; ++it) {
    const D err = p.vol - V;
    if (std::fabs(err.v) < tol) break;
    if (err > D(0)) b = h; else a = h;
    D hn = p.dv > D(SLOPE_MIN) ? h - err / p.dv : D(0.5) * (a + b);
    if (!(hn > a && hn < b)) hn = D(0.5) * (a + b);
    h = hn;
    p = node_pass(e, F, n, h);
  }
  e->level[n] = h; e->areaN[n] = p.dv;
  set_centroid(e, n, p);
}

// kernel/levels.hpp:54-162
void solve_group(sst_engine* e, const Pose& F, const int32_t* m, int32_t N) {
  Pass* Pp = e->passes.data();
  D V(0);
  double Vmax = 0;
  for (int32_t k = 0; k < N; ++k) { V += e->vol[m[k]]; Vmax += e->vmax[m[k]]; }
  bool allWet = true;
  int32_t firstWet = -1;
  for (int32_t k = 0; k < N; ++k) {
    if (e->vol[m[k]] > D(0)) { if (firstWet < 0) firstWet = k; }
    else allWet = false;
  }
  D h;
  if (allWet) {
    D s(0);
    for (int32_t k = 0; k < N; ++k) s += e->level[m[k]];
    h = s / D(static_cast<double>(N));
  } else {
    h = e->level[m[firstWet >= 0 ? firstWet : N - 1]];
  }
  for (int32_t k = 0; k < N; ++k) Pp[k] = node_pass(e, F, m[k], h);
  for (int32_t k = 0; k < N; ++k) e->zmaxN[m[k]] = Pp[k].zmax;
  D lo = Pp[0].zmin, hi = Pp[0].zmax;
  for (int32_t k = 1; k < N; ++k) { if (Pp[k].zmin < lo) lo = Pp[k].zmin; if (Pp[k].zmax > hi) hi = Pp[k].zmax; }
  if (V <= D(EMPTY_VOLUME)) {
    for (int32_t k = 0; k < N; ++k) { e->vol[m[k]] = D(0); e->level[m[k]] = Pp[k].zmin; e->areaN[m[k]] = D(0); }
    return;
  }
  if (V >= D(Vmax * FULL_FRACTION)) {
    const D over = jmax(D(0.0), V - Vmax);
    double aSum = 0;
    for (int32_t k = 0; k < N; ++k) aSum += e->aov[m[k]];
    const D dh = over / aSum;
    D assigned(0);
    for (int32_t k = 0; k < N - 1; ++k) {
      const D v = D(e->vmax[m[k]]) + dh * e->aov[m[k]];
      e->vol[m[k]] = v;
      assigned += v;
    }
    e->vol[m[N - 1]] = V - assigned;
    for (int32_t k = 0; k < N; ++k) {
      Pp[k] = node_pass(e, F, m[k], hi);
      e->level[m[k]] = hi + dh; e->areaN[m[k]] = D(e->aov[m[k]]);
      set_centroid(e, m[k], Pp[k]);
    }
    return;
  }
  if (!(h >= lo && h <= hi)) {
    h = jmin(hi, jmax(lo, h));
    for (int32_t k = 0; k < N; ++k) Pp[k] = node_pass(e, F, m[k], h);
  }
  const double tol = (0.5 > 1e-3 * Vmax) ? 0.5 : 1e-3 * Vmax;  // jmax(1e-3 Vmax, 0.5)
  D a = lo, b = hi;
  for (int it = 0; it < NEWTON_FAST; ++it) {
    D sum(0);
    for (int32_t k = 0; k < N; ++k) sum += Pp[k].vol;
    const D err = sum - V;
    if (std::fabs(err.v) < tol) break;
    if (err > D(0)) b = h; else a = h;
    D dv(0);
    for (int32_t k = 0; k < N; ++k) dv += Pp[k].dv;
    D hn = dv > D(SLOPE_MIN) ? h - err / dv : D(0.5) * (a + b);
    if (!(hn > a && hn < b)) hn = D(0.5) * (a + b);
    h = hn;
    for (int32_t k = 0; k < N; ++k) Pp[k] = node_pass(e, F, m[k], h);
  }
  D tot(0);
  for (int32_t k = 0; k < N; ++k) tot += Pp[k].vol;
  D assigned(0);
  for (int32_t k = 0; k < N - 1; ++k) {
    D v = tot > D(0) ? V * Pp[k].vol / tot : V / D(static_cast<double>(N));
    if (v > D(e->vmax[m[k]])) v = D(e->vmax[m[k]]);
    e->vol[m[k]] = v;
    assigned += v;
  }
  const double vmaxLast = e->vmax[m[N - 1]];
  if (V - assigned > D(vmaxLast)) {
    const D need = V - vmaxLast;
    D capped(0);
    for (int32_t k = N - 2; k >= 0; --k) {
      D prior(0);
      for (int32_t j = 0; j < k; ++j) prior += e->vol[m[j]];
      const D v = (need - capped) - prior;
      if (v > D(e->vmax[m[k]]) && k > 0) {
        e->vol[m[k]] = D(e->vmax[m[k]]);
        capped += D(e->vmax[m[k]]);
        continue;
      }
      e->vol[m[k]] = v;
      break;
    }
    assigned = D(0);
    for (int32_t k = 0; k < N - 1; ++k) assigned += e->vol[m[k]];
  }
  e->vol[m[N - 1]] = V - assigned;
  for (int32_t k = 0; k < N; ++k) {
    e->level[m[k]] = h; e->areaN[m[k]] = Pp[k].dv;
    set_centroid(e, m[k], Pp[k]);
  }
}

void solve_levels(sst_engine* e, const Pose& F) {
  for (int32_t g = 0; g < e->ng; ++g) {
    const int32_t N = e->gCount[g];
    const int32_t* m = e->gNodes.data() + e->gStart[g];
    bool merged = false;
    if (N >= 2) {
      if (e->gMode[g] == 1) {
        merged = true;
      } else if (e->gMode[g] == 2) {
        const D zMw = wz_of(F, e->gpx[g], e->gpy[g], e->gpz[g]);
        merged = true;
        for (int32_t k = 0; k < N; ++k)
          if (!(e->vol[m[k]] > D(EMPTY_VOLUME) && e->level[m[k]] > zMw + e->gMargin)) { merged = false; break; }
      }
    }
    e->merged[g] = merged ? 1 : 0;
    if (merged) solve_group(e, F, m, N);
    else for (int32_t k = 0; k < N; ++k) solve_single(e, F, m[k]);
  }
}

// kernel/flows.hpp:38-78
D flow(sst_engine* e, const Pose& F, int32_t c) {
  if (!e->en[c] || e->tOn[c] > e->t) return D(0);
  if (e->skip[c] >= 0 && e->merged[e->skip[c]]) return D(0);
  const int32_t a = e->ca[c], b = e->cb[c];
  const D zo = F.R20 * e->kx[c] + F.R21 * e->ky[c] + F.R22 * e->kz[c] + F.tz;
  const D ha = a < 0 ? D(0.0) : e->hEff[a], hbv = e->hEff[b];
  const D Ha = ha > zo ? ha - zo : D(0.0), Hb = hbv > zo ? hbv - zo : D(0.0);
  D q(0);
  if (e->law[c] == 0) {
    const D d = Ha - Hb;
    if (d != D(0)) q = D(e->coef[c]) * e->area[c] * e->sq2g * d / dsqrt(jmax(dfabs(d), D(ORIFICE_HEAD_FLOOR)));
  } else {
    const D H1 = Ha > Hb ? Ha : Hb;
    if (H1 > D(0)) {
      const D H2 = Ha > Hb ? Hb : Ha;
      D f(1);
      if (H2 > D(0)) {
        const D r = H2 / H1;
        f = dpow(jmax(D(0.0), D(1) - dpow(r, WEIR_EXPONENT)), VILLEMONTE_EXPONENT);
      }
      q = D(e->coef[c]) * e->area[c] * WEIR_COEFFICIENT * e->sq2g * H1 * dsqrt(H1) * f * D(Ha >= Hb ? 1.0 : -1.0);
    }
  }
  if (q.v == 0) return D(0);
  D dV = q * e->dt;
  const int32_t src = dV > D(0) ? a : b, dst = dV > D(0) ? b : a;
  const D hs = src < 0 ? D(0.0) : e->hEff[src];
  const D hd = dst < 0 ? D(0.0) : e->hEff[dst];
  const D inv = (src < 0 ? D(0.0) : D(1) / e->aEff[src]) + (dst < 0 ? D(0.0) : D(1) / e->aEff[dst]);
  const int32_t degRef = src < 0 ? e->deg[dst] : (dst < 0 ? e->deg[src] : (e->deg[src] > e->deg[dst] ? e->deg[src] : e->deg[dst]));
  const double share = LIMITER_SHARE / static_cast<double>(degRef > 1 ? degRef : 1);
  D lim = inv > D(0) ? D(share) * (hs - jmax(hd, zo)) / inv : dfabs(dV);
  if (lim < D(0)) lim = D(0);
  if (dfabs(dV) > lim) dV = dV > D(0) ? lim : -lim;
  return dV;
}

D flows_and_volumes(sst_engine* e, const Pose& F) {
  const int32_t NN = e->nn;
  for (int32_t n = 0; n < NN; ++n) {
    e->hEff[n] = e->vol[n] > D(EMPTY_VOLUME) ? e->level[n] : D(NO_HEAD);
    e->aEff[n] = e->vol[n] >= D(e->vmax[n]) ? D(e->aov[n]) : jmax(e->areaN[n], D(e->amin[n]));
  }
  for (int32_t n = 0; n < NN; ++n) {
    int32_t d = 0;
    for (int32_t k = e->incStart[n]; k < e->incStart[n] + e->incCount[n]; ++k) {
      const int32_t c = e->incConn[k];
      if (!e->en[c]) continue;
      const int32_t a = e->ca[c], b = e->cb[c];
      if (a >= 0 && e->hEff[a].v < NO_HEAD_TEST && e->hEff[b].v < NO_HEAD_TEST) continue;
      ++d;
    }
    e->deg[n] = d;
  }
  for (int32_t c = 0; c < e->nc; ++c) e->dV[c] = flow(e, F, c);
  std::vector<D> acc(NN);
  for (int32_t n = 0; n < NN; ++n) {
    D a(0);
    for (int32_t k = e->incStart[n]; k < e->incStart[n] + e->incCount[n]; ++k) {
      const D& d = e->dV[e->incConn[k]];
      a = e->incSide[k] ? a + d : a - d;
    }
    acc[n] = a;
  }
  D seaIn(0);
  for (int32_t k = 0; k < static_cast<int32_t>(e->sea.size()); ++k) seaIn += e->dV[e->sea[k]];
  std::vector<D> excess(NN);
  for (int32_t n = 0; n < NN; ++n) {
    D v = e->vol[n] + acc[n];
    if (v < D(0)) v = D(0);
    const double vm = e->vmax[n];
    D ex(0);
    if (v > D(vm)) {
      const D head = jmax(D(0.0), -e->zmaxN[n]);
      const D cap = D(vm) + D(e->aov[n]) * head;
      if (v > cap) { ex = v - cap; v = cap; }
    }
    excess[n] = ex;
    e->vol[n] = v;
  }
  for (int32_t n = 0; n < NN; ++n)
    if (excess[n] > D(0)) seaIn -= excess[n];
  return seaIn;
}

void body(sst_engine* e, const Pose& F, const Buoy& hb) {
  const double W = e->rho * e->g;
  const D Fb = hb.V * W;
  const D bxw = F.R00 * hb.x + F.R01 * hb.y + F.R02 * hb.z + F.tx;
  const D byw = F.R10 * hb.x + F.R11 * hb.y + F.R12 * hb.z + F.ty;
  D tauX = (byw - e->YO) * Fb, tauY = -(bxw - e->XO) * Fb;
  D Fz = Fb - e->g * e->ms;
  D mw(0), Iw_p(0), Iw_r(0);
  for (int32_t n = 0; n < e->nn; ++n) {
    const D V = e->vol[n];
    if (V <= D(0)) continue;
    const D x = e->wcx[n], y = e->wcy[n], z = e->wcz[n];
    const D wx = F.R00 * x + F.R01 * y + F.R02 * z + F.tx - e->XO;
    const D wy = F.R10 * x + F.R11 * y + F.R12 * z + F.ty - e->YO;
    const D wz = F.R20 * x + F.R21 * y + F.R22 * z + F.tz - e->zO;
    const D f = D(-W) * V;
    tauX += wy * f; tauY -= wx * f; Fz += f;
    const D m = D(e->rho) * V;
    mw += m;
    Iw_p += m * (wx * wx + wz * wz);
    Iw_r += m * (wy * wy + wz * wz);
  }
  const D Mth = tauY, Mph = tauX * F.cth;
  const double dt = e->dt;
  const D mh = D(e->mh0) + mw;
  const D Ith = D(e->Ith0) + Iw_p, Iph = D(e->Iph0) + Iw_r;
  const D az = (Fz - D(e->cDz) * e->vz - D(e->qz) * dfabs(e->vz) * e->vz) / mh;
  const D ath = (Mth - D(e->cDth) * e->wth - D(e->qth) * dfabs(e->wth) * e->wth) / Ith;
  const D aph = (Mph - D(e->cDph) * e->wph - D(e->qph) * dfabs(e->wph) * e->wph) / Iph;
  e->vz += az * dt; e->wth += ath * dt; e->wph += aph * dt;
  e->zO += e->vz * dt; e->pitch += e->wth * dt; e->roll += e->wph * dt;
  if (e->pitch > D(PITCH_CLAMP)) { e->pitch = D(PITCH_CLAMP); e->wth = D(0); }
  if (e->pitch < D(-PITCH_CLAMP)) { e->pitch = D(-PITCH_CLAMP); e->wth = D(0); }
  if (e->roll > D(ROLL_CLAMP)) { e->roll = D(ROLL_CLAMP); e->wph = D(0); }
  if (e->roll < D(-ROLL_CLAMP)) { e->roll = D(-ROLL_CLAMP); e->wph = D(0); }
  e->t += dt;
  if (!e->foundered && (hb.top.v < e->hullTopBelow || std::fabs(e->pitch.v) > e->pitchAbsAbove ||
                        (hb.V.v < e->buoyancyBelow && e->t > e->minT)))
    e->foundered = 1;
}

void step_once(sst_engine* e) {
  const Pose F = pose_at(e, e->zO, e->pitch, e->roll);
  const Buoy hb = buoyancy(e, F);
  solve_levels(e, F);
  const D seaIn = flows_and_volumes(e, F);
  e->inflow = seaIn / D(e->dt);
  body(e, F, hb);
}

template <class T>
std::vector<T> copy_of(const T* p, int64_t n) {
  return p && n > 0 ? std::vector<T>(p, p + n) : std::vector<T>(static_cast<std::size_t>(n > 0 ? n : 0));
}

}  // namespace

extern "C" {

sst_engine* sst_create(const sso_ship* S, const sso_sim* M) {
  auto* e = new sst_engine();
  e->ncol = S->ncol; e->nseg = S->nseg; e->nn = S->nnode;
  e->x = copy_of(S->x, S->ncol); e->y = copy_of(S->y, S->ncol); e->dxdy = copy_of(S->dxdy, S->ncol);
  e->zlo = copy_of(S->zlo, S->ncol); e->zhi = copy_of(S->zhi, S->ncol);
  e->segCol = copy_of(S->segCol, S->nseg); e->segA = copy_of(S->segA, S->nseg); e->segE = copy_of(S->segE, S->nseg);
  e->mu = copy_of(S->mu, S->nnode); e->vmax = copy_of(S->vmax, S->nnode); e->amin = copy_of(S->amin, S->nnode);
  e->aov = copy_of(S->aov, S->nnode); e->segStart = copy_of(S->segStart, S->nnode); e->segCount = copy_of(S->segCount, S->nnode);
  e->rho = M->rho; e->g = M->g; e->sq2g = std::sqrt(2 * M->g); e->dt = M->dt;
  e->ng = M->ngroup;
  e->gStart = copy_of(M->gStart, M->ngroup); e->gCount = copy_of(M->gCount, M->ngroup);
  int32_t members = 0, maxGroup = 1;
  for (int32_t g = 0; g < M->ngroup; ++g) {
    members = std::max(members, M->gStart[g] + M->gCount[g]);
    maxGroup = std::max(maxGroup, M->gCount[g]);
  }
  e->gNodes = copy_of(M->gNodes, members); e->gMode = copy_of(M->gMode, M->ngroup);
  e->gpx = copy_of(M->gpx, M->ngroup); e->gpy = copy_of(M->gpy, M->ngroup); e->gpz = copy_of(M->gpz, M->ngroup);
  e->gMargin = M->gMargin;
  e->nc = M->nconn;
  e->ca = copy_of(M->ca, M->nconn); e->cb = copy_of(M->cb, M->nconn); e->law = copy_of(M->law, M->nconn);
  e->kx = copy_of(M->cx, M->nconn); e->ky = copy_of(M->cy, M->nconn); e->kz = copy_of(M->cz, M->nconn);
  e->coef = copy_of(M->coef, M->nconn); e->en = copy_of(M->en, M->nconn); e->tOn = copy_of(M->tOn, M->nconn);
  e->skip = copy_of(M->skipGroup, M->nconn);
  e->area.resize(static_cast<std::size_t>(M->nconn));
  for (int32_t c = 0; c < M->nconn; ++c) e->area[c] = D(M->area[c]);
  e->hullTopBelow = M->hullTopBelow; e->pitchAbsAbove = M->pitchAbsAbove; e->buoyancyBelow = M->buoyancyBelow; e->minT = M->minT;
  e->ms = M->body[0]; e->g0x = M->body[2]; e->g0y = M->body[3]; e->g0z = M->body[4]; e->XO = M->body[5]; e->YO = M->body[6];
  e->mh0 = M->body[7]; e->Ith0 = M->body[8]; e->Iph0 = M->body[9]; e->cDz = M->body[10]; e->cDth = M->body[11]; e->cDph = M->body[12];
  e->qz = M->body[13]; e->qth = M->body[14]; e->qph = M->body[15];
  e->xFP = M->xFP; e->xAP = M->xAP;
  // incidence: per node its connections in increasing order, side 1 at the b end; the sea list (model.cpp:26-56)
  const int32_t NN = e->nn;
  e->incCount.assign(NN, 0);
  for (int32_t c = 0; c < e->nc; ++c) { if (e->ca[c] >= 0) e->incCount[e->ca[c]]++; e->incCount[e->cb[c]]++; }
  e->incStart.assign(NN, 0);
  int32_t total = 0;
  for (int32_t n = 0; n < NN; ++n) { e->incStart[n] = total; total += e->incCount[n]; }
  e->incConn.assign(total, 0); e->incSide.assign(total, 0);
  std::vector<int32_t> fill(NN, 0);
  for (int32_t c = 0; c < e->nc; ++c) {
    if (e->ca[c] >= 0) {
      const int32_t k = e->incStart[e->ca[c]] + fill[e->ca[c]]++;
      e->incConn[k] = c; e->incSide[k] = 0;
    } else {
      e->sea.push_back(c);
    }
    const int32_t k = e->incStart[e->cb[c]] + fill[e->cb[c]]++;
    e->incConn[k] = c; e->incSide[k] = 1;
  }
  e->t = M->state0[0];
  e->zO = D(M->state0[1]); e->pitch = D(M->state0[2]); e->roll = D(M->state0[3]);
  e->vz = D(M->state0[4]); e->wth = D(M->state0[5]); e->wph = D(M->state0[6]);
  e->vol.resize(NN); e->level.resize(NN); e->wcx.resize(NN); e->wcy.resize(NN); e->wcz.resize(NN);
  for (int32_t n = 0; n < NN; ++n) {
    e->vol[n] = D(M->vol0[n]); e->level[n] = D(M->level0[n]);
    e->wcx[n] = D(M->cx0[n]); e->wcy[n] = D(M->cy0[n]); e->wcz[n] = D(M->cz0[n]);
  }
  e->areaN.assign(NN, D(0)); e->zmaxN.assign(NN, D(0)); e->hEff.assign(NN, D(0)); e->aEff.assign(NN, D(0));
  e->dV.assign(e->nc, D(0)); e->deg.assign(NN, 0); e->merged.assign(e->ng, 0); e->passes.resize(maxGroup);
  e->inflow = D(0);
  e->foundered = 0;
  return e;
}

void sst_destroy(sst_engine* e) { delete e; }

void sst_set_connection(sst_engine* e, int32_t c, int enabled, double area, double tOn) {
  if (c < 0 || c >= e->nc) return;
  if (enabled >= 0) e->en[c] = static_cast<uint8_t>(enabled != 0);
  if (!std::isnan(area)) e->area[c].v = area;
  if (!std::isnan(tOn)) e->tOn[c] = tOn;
}

void sst_seed_area(sst_engine* e, int32_t c, int32_t p, double g) {
  if (c < 0 || c >= e->nc || p < 0 || p >= P) return;
  e->area[c].d[p] = g;
}

void sst_step(sst_engine* e, int64_t n) {
  for (int64_t i = 0; i < n; ++i) step_once(e);
}

void sst_get_record(const sst_engine* e, double* r, double* d) {
  const int32_t N = e->nn, R = 10 + 5 * N;
  const D zero(0);
  const D* vals[7] = {&zero, &e->zO, &e->pitch, &e->roll, &e->vz, &e->wth, &e->wph};
  for (int k = 0; k < R; ++k) {
    const D* v;
    if (k < 7) v = vals[k];
    else if (k < 10) v = k == 7 ? &e->inflow : &zero;
    else {
      const int32_t j = k - 10, f = j / N, n = j % N;
      v = f == 0 ? &e->vol[n] : f == 1 ? &e->level[n] : f == 2 ? &e->wcx[n] : f == 3 ? &e->wcy[n] : &e->wcz[n];
    }
    r[k] = k == 0 ? e->t : v->v;
    if (d)
      for (int p = 0; p < P; ++p) d[p * R + k] = k == 0 ? 0.0 : v->d[p];
  }
}

void sst_readouts(const sst_engine* e, double* r7, double* d) {
  const Pose F = pose_at(e, e->zO, e->pitch, e->roll);
  D water(0);
  for (int32_t n = 0; n < e->nn; ++n) water += e->vol[n];
  const D out[7] = {D(e->t), e->pitch * 180.0 / D(PI_), e->roll * 180.0 / D(PI_), water * e->rho / D(1000.0),
                    e->inflow * e->rho / D(1000.0) * 60.0, -wz_of(F, e->xFP, 0, 0), -wz_of(F, e->xAP, 0, 0)};
  for (int k = 0; k < 7; ++k) {
    r7[k] = out[k].v;
    if (d)
      for (int p = 0; p < P; ++p) d[p * 7 + k] = out[k].d[p];
  }
}

int sst_foundered(const sst_engine* e) { return e->foundered; }

}  // extern "C"
