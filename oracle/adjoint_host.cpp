// The adjoint's host harness: TEST INFRASTRUCTURE. It runs the product's reverse step (sinksim_b200/csrc/
// adjoint_step.cuh, host-and-device code) on the CPU with a one-thread team, on tapes recorded by the C restatement of
// the forward step (sinksim_oracle.c), so that the reverse logic can be held to the tangent-linear restatement
// (sinksim_tangent.cpp) without a GPU. The sinksim_b200 package never links or calls it; the GPU adjoint kernel runs
// the same reverse code on the device.
#include <cmath>
#include <cstring>
#include <vector>

#include "sinksim_oracle.h"
#include "../sinksim_b200/csrc/adjoint_step.cuh"

namespace {

using namespace ssb;
using namespace ssb::adj;

// A team of one thread: every loop runs serially, every reduction is the identity.
struct HostTeam {
  int rank = 0, size = 1, warp = 0, nwarps = 1, lane = 0, width = 1;
  void sync() const {}
  void add_int(int* p, int v) const { *p += v; }
  void reduce(double*, int, double*) const {}
};

// The compiled model in the kernel's layout, in host memory.
struct HostModel {
  std::vector<double2> colXY, colLH, segXY, segLH;
  std::vector<double> colA, segAr, mu, vmax, amin, aov, gpx, gpy, gpz, kx, ky, kz, coef;
  std::vector<std::int32_t> segStart, segCount, gStart, gCount, gNodes, ca, cb, skip, incStart, incCount, incConn, sea;
  std::vector<std::uint8_t> gMode, law, incSide;
  DevModel dm{};

  HostModel(const sso_ship* S, const sso_sim* M) {
    const int nc = S->ncol, ns = S->nseg, nn = S->nnode;
    for (int i = 0; i < nc; ++i) {
      colXY.push_back(double2{S->x[i], S->y[i]});
      colLH.push_back(double2{S->zlo[i], S->zhi[i]});
      colA.push_back(S->dxdy[i]);
    }
    for (int j = 0; j < ns; ++j) {
      const int c = S->segCol[j];
      segXY.push_back(double2{S->x[c], S->y[c]});
      segLH.push_back(double2{S->segA[j], S->segE[j]});
      segAr.push_back(S->dxdy[c]);
    }
    mu.assign(S->mu, S->mu + nn); vmax.assign(S->vmax, S->vmax + nn); amin.assign(S->amin, S->amin + nn); aov.assign(S->aov, S->aov + nn);
    segStart.assign(S->segStart, S->segStart + nn); segCount.assign(S->segCount, S->segCount + nn);
    const int ng = M->ngroup;
    gStart.assign(M->gStart, M->gStart + ng); gCount.assign(M->gCount, M->gCount + ng); gMode.assign(M->gMode, M->gMode + ng);
    gpx.assign(M->gpx, M->gpx + ng); gpy.assign(M->gpy, M->gpy + ng); gpz.assign(M->gpz, M->gpz + ng);
    int members = 0, maxGroup = 1;
    for (int g = 0; g < ng; ++g) { members = std::max(members, gStart[g] + gCount[g]); maxGroup = std::max(maxGroup, gCount[g]); }
    gNodes.assign(M->gNodes, M->gNodes + members);
    const int k = M->nconn;
    ca.assign(M->ca, M->ca + k); cb.assign(M->cb, M->cb + k); skip.assign(M->skipGroup, M->skipGroup + k); law.assign(M->law, M->law + k);
    kx.assign(M->cx, M->cx + k); ky.assign(M->cy, M->cy + k); kz.assign(M->cz, M->cz + k); coef.assign(M->coef, M->coef + k);
    incCount.assign(nn, 0);
    for (int c = 0; c < k; ++c) { if (ca[c] >= 0) incCount[ca[c]]++; incCount[cb[c]]++; }
    incStart.assign(nn, 0);
    int total = 0;
    for (int n = 0; n < nn; ++n) { incStart[n] = total; total += incCount[n]; }
    incConn.assign(total, 0); incSide.assign(total, 0);
    std::vector<int> fill(nn, 0);
    for (int c = 0; c < k; ++c) {
      if (ca[c] >= 0) { const int q = incStart[ca[c]] + fill[ca[c]]++; incConn[q] = c; incSide[q] = 0; }
      else sea.push_back(c);
      const int q = incStart[cb[c]] + fill[cb[c]]++;
      incConn[q] = c; incSide[q] = 1;
    }
    DevModel& d = dm;
    d.ncol = nc; d.colXY = colXY.data(); d.colLH = colLH.data(); d.colA = colA.data();
    d.nseg = ns; d.segXY = segXY.data(); d.segLH = segLH.data(); d.segAr = segAr.data();
    d.nn = nn; d.mu = mu.data(); d.vmax = vmax.data(); d.amin = amin.data(); d.aov = aov.data();
    d.segStart = segStart.data(); d.segCount = segCount.data();
    d.ng = ng; d.gStart = gStart.data(); d.gCount = gCount.data(); d.gNodes = gNodes.data(); d.gMode = gMode.data();
    d.gpx = gpx.data(); d.gpy = gpy.data(); d.gpz = gpz.data(); d.gMargin = M->gMargin; d.maxGroup = maxGroup;
    d.nc = k; d.ca = ca.data(); d.cb = cb.data(); d.skip = skip.data(); d.law = law.data();
    d.kx = kx.data(); d.ky = ky.data(); d.kz = kz.data(); d.coef = coef.data();
    d.incStart = incStart.data(); d.incCount = incCount.data(); d.incConn = incConn.data(); d.incSide = incSide.data();
    d.nsea = static_cast<int>(sea.size()); d.sea = sea.data();
    d.rho = M->rho; d.g = M->g; d.sq2g = std::sqrt(2 * M->g); d.dt = M->dt;
    d.ms = M->body[0]; d.g0x = M->body[2]; d.g0y = M->body[3]; d.g0z = M->body[4]; d.XO = M->body[5]; d.YO = M->body[6];
    d.mh0 = M->body[7]; d.Ith0 = M->body[8]; d.Iph0 = M->body[9]; d.cDz = M->body[10]; d.cDth = M->body[11]; d.cDph = M->body[12];
    d.qz = M->body[13]; d.qth = M->body[14]; d.qph = M->body[15];
    d.xFP = M->xFP; d.xAP = M->xAP;
  }
};

// The recorder: one tape per step, filled by the oracle's hooks.
struct Recorder {
  sso_engine* e;
  TapeLayout L;
  int nn, ng;
  std::vector<unsigned char>* cur = nullptr;
  static void on_pass(void* user, int32_t n, int32_t k, const double* rec) {
    auto* r = static_cast<Recorder*>(user);
    Tape t = tape_at(r->cur->data(), r->L);
    if (k < kMaxPasses) std::memcpy(t.pass(n, k), rec, kPassFields * sizeof(double));
    t.i[r->L.npass + n] = k + 1;
  }
  static void on_solved(void* user) {
    auto* r = static_cast<Recorder*>(user);
    Tape t = tape_at(r->cur->data(), r->L);
    std::vector<std::int32_t> merged(static_cast<std::size_t>(r->ng));
    sso_solved_state(r->e, t.d + r->L.volS, t.d + r->L.levelS, t.d + r->L.areaS, t.d + r->L.cxS, t.d + r->L.cyS, t.d + r->L.czS,
                     t.d + r->L.zmaxS, merged.data(), t.d + r->L.pose, t.d + r->L.buoy);
    for (int g = 0; g < r->ng; ++g) t.i[r->L.merged + g] = merged[g];
  }
};

}  // namespace

extern "C" {

/* Objective and gradient with respect to every connection area, by the reverse sweep on the CPU.
 *
 * One instance of the model with the given connection fields, `steps` steps from the compiled initial state. The
 * objective is sum_k (trim(s_k) - trim_k)^2 + (heave(s_k) - heave_k)^2 over the states after sample_step[k] steps
 * (trim in degrees, heave the mean of the forward and aft drafts). grad receives d objective / d area[c] for every
 * connection. Returns 0, or the adjoint's error bits. */
int ssa_gradient(const sso_ship* ship, const sso_sim* sim, const uint8_t* en, const double* area, const double* tOn, int64_t steps,
                 int32_t nsamples, const int64_t* sampleStep, const double* trimT, const double* heaveT, double* J, double* grad) {
  HostModel hm(ship, sim);
  const DevModel& M = hm.dm;
  const int nn = M.nn, nc = M.nc, ng = M.ng;
  sso_engine* e = sso_create(ship, sim, 0);
  for (int c = 0; c < nc; ++c) sso_set_connection(e, c, en[c], area[c], tOn[c]);
  Recorder rec{e, tape_layout(nn, ng), nn, ng};
  sso_set_hooks(e, &Recorder::on_pass, &Recorder::on_solved, &rec);
  std::vector<std::vector<unsigned char>> tapes(static_cast<std::size_t>(steps));
  const int R = 10 + 5 * nn;
  std::vector<double> r(static_cast<std::size_t>(R));
  std::vector<double> state(static_cast<std::size_t>(steps + 1) * 7);
  auto keep_state = [&](int64_t s) {
    sso_get_record(e, r.data());
    for (int k = 0; k < 7; ++k) state[static_cast<std::size_t>(s) * 7 + k] = r[k];
  };
  keep_state(0);
  for (int64_t s = 0; s < steps; ++s) {
    auto& tp = tapes[static_cast<std::size_t>(s)];
    tp.assign(rec.L.bytes, 0);
    Tape t = tape_at(tp.data(), rec.L);
    sso_get_record(e, r.data());
    for (int k = 0; k < 7; ++k) t.d[rec.L.scal + k] = r[k];
    for (int n = 0; n < nn; ++n) {
      t.d[rec.L.volIn + n] = r[10 + n]; t.d[rec.L.levelIn + n] = r[10 + nn + n];
      t.d[rec.L.cxIn + n] = r[10 + 2 * nn + n]; t.d[rec.L.cyIn + n] = r[10 + 3 * nn + n]; t.d[rec.L.czIn + n] = r[10 + 4 * nn + n];
    }
    rec.cur = &tp;
    sso_step(e, 1);
    keep_state(s + 1);
  }
  sso_set_hooks(e, nullptr, nullptr, nullptr);
  // the objective at the sample states
  auto pose_at_state = [&](int64_t s) {
    const double* q = &state[static_cast<std::size_t>(s) * 7];
    return pose_of(M, q[1], q[2], q[3]);
  };
  double obj = 0;
  std::vector<double> aTrim(static_cast<std::size_t>(nsamples)), aHeave(static_cast<std::size_t>(nsamples));
  for (int k = 0; k < nsamples; ++k) {
    const int64_t s = sampleStep[k] < steps ? sampleStep[k] : steps;
    double tr, hv;
    trim_heave(M, pose_at_state(s), state[static_cast<std::size_t>(s) * 7 + 2], tr, hv);
    obj += (tr - trimT[k]) * (tr - trimT[k]) + (hv - heaveT[k]) * (hv - heaveT[k]);
    aTrim[k] = 2 * (tr - trimT[k]);
    aHeave[k] = 2 * (hv - heaveT[k]);
  }
  *J = obj;
  // the reverse sweep, last step first
  std::vector<double> aVol(nn, 0), aLevel(nn, 0), aCx(nn, 0), aCy(nn, 0), aCz(nn, 0);
  AdjState a{aVol.data(), aLevel.data(), aCx.data(), aCy.data(), aCz.data()};
  double aSc[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> hEff(nn), aEff(nn), dV(nc), volPost(nn), w[9], fa[4], red(32);
  for (auto& v : w) v.assign(nn, 0);
  for (auto& v : fa) v.assign(nc, 0);
  std::vector<int> deg(nn);
  std::vector<std::int32_t> clip(nn);
  UnitWork unitWork{};
  std::vector<std::uint8_t> plain(nn);
  std::vector<std::int32_t> units(nn + 1), nunits(1);
  std::vector<double> pw(2 * static_cast<std::size_t>(nc));
  std::vector<Replay> replays(static_cast<std::size_t>(nn));
  RevSlot S{hEff.data(), aEff.data(), dV.data(), volPost.data(), deg.data(), clip.data(), w[0].data(), w[1].data(), w[2].data(), w[3].data(),
            w[4].data(), w[5].data(), w[6].data(), w[7].data(), w[8].data(), fa[0].data(), fa[1].data(), fa[2].data(), fa[3].data(), red.data(),
            &unitWork, plain.data(), units.data(), nunits.data(), pw.data(), replays.data()};
  for (int c = 0; c < nc; ++c) grad[c] = 0;
  auto add_samples = [&](int64_t s) {
    for (int k = 0; k < nsamples; ++k) {
      const int64_t sk = sampleStep[k] < steps ? sampleStep[k] : steps;
      if (sk != s) continue;
      const PoseD F = pose_at_state(s);
      AdjPose aP;
      zero(aP);
      trim_heave_reverse(M, aTrim[k], aHeave[k], aP, aSc[1]);
      pose_reverse(M, F, aP, aSc[0], aSc[1], aSc[2]);
    }
  };
  HostTeam team;
  int err = 0;
  add_samples(steps);
  for (int64_t s = steps - 1; s >= 0; --s) {
    Tape t = tape_at(tapes[static_cast<std::size_t>(s)].data(), rec.L);
    reverse_step(team, M, t, en, area, tOn, S, a, aSc, grad, &err);
    add_samples(s);
  }
  sso_destroy(e);
  return err;
}

}  // extern "C"
