// The adjoint kernel: the gradient of a trajectory objective with respect to every connection area, for a batch of
// instances, by a hand-written discrete adjoint of the time step with checkpoints (no counterpart in the reference,
// which has no gradients: docs/adr/0001-single-source-cpp-kernel.md:25-26).
//
// A persistent grid of teams (W warps each, one instance at a time from a work queue), per instance:
//   1. forward: the instance runs from its initial state to tMax or its founder, exactly as the batch kernel steps it
//      (the same team_step, so the same bits), keeping the state every K steps (a checkpoint: t, pose, rates and every
//      node's volume, level and centroid, FP64) and the objective's readouts at the sample times. With the tape hooks
//      on (tapeForward), every step's tape (every node pass of the level solve, the solved levels, pose and buoyancy)
//      goes to shared memory and from there, packed, into the team's ring of step records in global memory;
//   2. reverse: segment by segment, last first. A segment whose records the ring still holds is reversed from them;
//      any other is recomputed from its checkpoint with the tape hooks on, into the ring, first. Each step's record is
//      unpacked into shared memory and reversed (adjoint_step.cuh), adding the objective's adjoint at the sample
//      states.
// Memory per team: the checkpoints of one run and the ring; the adjoint of the state lives in shared memory. When the
// ring holds a whole run (the usual case: a packed record is about 12 KB on a 64-node model) nothing is recomputed;
// with a ring of K records every segment is recomputed once, which costs one more forward pass.
//
// The objective: J = sum_k (trim(s_k) - trim*_k)^2 + (heave(s_k) - heave*_k)^2, trim in degrees and heave the mean of
// the forward and aft drafts, where s_k is the state at which a readout curve recorded every sample time would take its
// record (the first step start with t >= t_k; the final state for a run that stopped before t_k).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "adjoint_kernel.h"
#include "adjoint_step.cuh"
#include "warp_step.cuh"

namespace ssb {

namespace {

using adj::AdjPose;
using adj::PoseD;

template <int W>
struct AdjTeam {
  int rank, size, warp, nwarps, lane, width, bar;
  __device__ __forceinline__ void sync() const {
    if constexpr (W == 1) __syncwarp();
    else asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(W * 32) : "memory");
  }
  __device__ __forceinline__ void add_int(int* p, int v) const { atomicAdd(p, v); }
  // team-wide sums of K values (K <= 16), every thread receives them: each warp's sums in shared memory, then lane k
  // of every warp adds value k over the warps (in warp order) and the lanes pass the K totals round by shuffles
  __device__ __forceinline__ void reduce(double* v, int K, double* red) const {
    for (int k = 0; k < K; ++k) {
      double x = v[k];
      for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
      if (lane == 0) red[warp * 16 + k] = x;
    }
    sync();
    double s = 0;
    if (lane < K)
      for (int w = 0; w < nwarps; ++w) s += red[w * 16 + lane];
    for (int k = 0; k < K; ++k) v[k] = __shfl_sync(0xffffffffu, s, k);
    sync();
  }
};

// The tape hooks of the forward step (NoTape's counterpart): one lane of a level lane group writes each node pass, the
// team writes the solved state, the pose and the buoyancy result.
struct GpuTape {
  adj::Tape t;
  __device__ __forceinline__ void pass(int n, int k, double h, const PassR& p, const LevelLanes& L) const {
    if (L.sub != 0) return;
    if (k < adj::kMaxPasses) {
      double* r = t.pass(n, k);
      r[0] = h; r[1] = p.vol; r[2] = p.dv; r[3] = p.mx; r[4] = p.my; r[5] = p.mz; r[6] = p.zmin; r[7] = p.zmax;
    }
    t.i[t.L.npass + n] = k + 1;
  }
  template <int W>
  __device__ __forceinline__ void solved(const DevModel& M, const Slot& S, const Team<W>& T) const {
    const adj::TapeLayout& L = t.L;
    for (int n = T.rank; n < M.nn; n += 32 * W) {
      t.d[L.volS + n] = S.vol[n]; t.d[L.levelS + n] = S.level[n]; t.d[L.areaS + n] = S.area[n];
      t.d[L.cxS + n] = S.cx[n]; t.d[L.cyS + n] = S.cy[n]; t.d[L.czS + n] = S.cz[n]; t.d[L.zmaxS + n] = S.zmax[n];
    }
    for (int g = T.rank; g < M.ng; g += 32 * W) t.i[L.merged + g] = S.merged[g];
    if (T.leader()) {
      const Pose& F = *S.pose;
      const double p[14] = {F.R00, F.R01, F.R02, F.R10, F.R11, F.R12, F.R20, F.R21, F.R22, F.tx, F.ty, F.tz, F.cth, F.iR};
      for (int k = 0; k < 14; ++k) t.d[L.pose + k] = p[k];
      const Buoy& b = *S.buoy;
      t.d[L.buoy] = b.V; t.d[L.buoy + 1] = b.x; t.d[L.buoy + 2] = b.y; t.d[L.buoy + 3] = b.z;
    }
  }
};

// Instance fields for team_step: the connection fields of the instance; events go nowhere (the adjoint runs keep no
// event log: the founder flag, which ends a run, is kept in registers by team_step itself).
struct AdjInst {
  const std::uint8_t* en_;
  const double *area_, *tOn_;
  double* sink;  // per team: evCap + nmon + nmark doubles that absorb the event bookkeeping
  std::int32_t* isink;
  int nmon;
  __device__ __forceinline__ const std::uint8_t* en() const { return en_; }
  __device__ __forceinline__ const double* area() const { return area_; }
  __device__ __forceinline__ const double* tOn() const { return tOn_; }
  __device__ __forceinline__ double* evT() const { return sink; }
  __device__ __forceinline__ std::int32_t* evId() const { return isink; }
  __device__ __forceinline__ std::int32_t* evKind() const { return isink; }
  __device__ __forceinline__ double* overT() const { return sink; }
  __device__ __forceinline__ double* markT() const { return sink + nmon; }
};

// Per-team shared memory: the forward slot, then the reverse's arrays.
struct AdjSmem {
  unsigned char* raw;   // one packed step record (stageRecords), or null
  adj::RevSlot rs;
  adj::AdjState as;
  double* grad;      // [nc]
  double* sampleS;   // [nsamples] state index of each sample (as doubles)
  unsigned char* tape;  // one step's tape: written by the step's hooks, or unpacked from its record for its reverse
  std::int32_t* poff;   // [nn + 1] first pass record of each node in a packed record, then their total
};

__device__ __forceinline__ AdjSmem carve_adjoint(unsigned char* base, const AdjLayout& A) {
  AdjSmem m;
  auto d = [&](std::uint32_t off) { return reinterpret_cast<double*>(base + off); };
  m.rs.hEff = d(A.hEff); m.rs.aEff = d(A.aEff); m.rs.dV = d(A.dV); m.rs.volPost = d(A.volPost);
  m.rs.deg = reinterpret_cast<int*>(base + A.deg);
  m.rs.clip = reinterpret_cast<std::int32_t*>(base + A.clip);
  m.rs.aVolPost = d(A.aVolPost); m.rs.aCxs = d(A.aCxs); m.rs.aCys = d(A.aCys); m.rs.aCzs = d(A.aCzs); m.rs.aVs = d(A.aVs);
  m.rs.aAcc = d(A.aAcc); m.rs.aZmx = d(A.aZmx); m.rs.aLs = d(A.aLs); m.rs.aAs = d(A.aAs);
  m.rs.faHA = d(A.faHA); m.rs.faHB = d(A.faHB); m.rs.faAA = d(A.faAA); m.rs.faAB = d(A.faAB);
  m.rs.red = d(A.red);
  m.rs.work = reinterpret_cast<adj::UnitWork*>(base + A.work);
  m.rs.plain = base + A.plain;
  m.rs.units = reinterpret_cast<std::int32_t*>(base + A.units);
  m.rs.nunits = reinterpret_cast<std::int32_t*>(base + A.nunits);
  m.rs.pw = d(A.pw);
  m.rs.replays = reinterpret_cast<adj::Replay*>(base + A.replays);
  m.as.aVol = d(A.aVol); m.as.aLevel = d(A.aLevel); m.as.aCx = d(A.aCx); m.as.aCy = d(A.aCy); m.as.aCz = d(A.aCz);
  m.grad = d(A.grad);
  m.sampleS = d(A.sampleS);
  m.tape = base + A.tape;
  m.raw = A.raw ? base + A.raw : nullptr;
  m.poff = reinterpret_cast<std::int32_t*>(base + A.poff);
  return m;
}

// A checkpoint: t, zO, pitch, roll, vz, wth, wph, then vol, level, cx, cy, cz per node.
template <int W>
__device__ __forceinline__ void save_state(double* c, const SimRegs& R, const Slot& S, int nn, const Team<W>& T) {
  if (T.leader()) { c[0] = R.t; c[1] = R.zO; c[2] = R.pitch; c[3] = R.roll; c[4] = R.vz; c[5] = R.wth; c[6] = R.wph; }
  for (int n = T.rank; n < nn; n += 32 * W) {
    c[7 + n] = S.vol[n]; c[7 + nn + n] = S.level[n]; c[7 + 2 * nn + n] = S.cx[n]; c[7 + 3 * nn + n] = S.cy[n]; c[7 + 4 * nn + n] = S.cz[n];
  }
}

// Loads a state into the team's registers and slot, with the step's scratch cleared (as the batch kernel does when it
// claims an instance).
template <int W>
__device__ __forceinline__ void load_state(const double* c, SimRegs& R, Slot& S, const DevModel& M, const Team<W>& T) {
  R.t = c[0]; R.zO = c[1]; R.pitch = c[2]; R.roll = c[3]; R.vz = c[4]; R.wth = c[5]; R.wph = c[6];
  R.calm = 0; R.inflow = 0; R.Vb = 0; R.hullTop = 0; R.mw = 0; R.bx = 0; R.by = 0; R.bz = 0;
  R.foundered = 0; R.founderT = -1;
  R.evCount = M.evCap;  // no event is recorded
  const int nn = M.nn;
  for (int n = T.rank; n < nn; n += 32 * W) {
    S.vol[n] = c[7 + n]; S.level[n] = c[7 + nn + n]; S.cx[n] = c[7 + 2 * nn + n]; S.cy[n] = c[7 + 3 * nn + n]; S.cz[n] = c[7 + 4 * nn + n];
    S.area[n] = 0; S.zmax[n] = 0; S.hEff[n] = 0; S.aEff[n] = 0; S.acc[n] = 0; S.deg[n] = 0;
  }
  for (int g = T.rank; g < M.ng; g += 32 * W) S.merged[g] = 0;
  for (int c2 = T.rank; c2 < M.nc; c2 += 32 * W) { S.dV[c2] = 0; S.q[c2] = 0; }
  T.sync();
}

// A packed step record: the tape's int32 (pass counts, merged flags), each node's first pass record in the packed
// order and their total (nn + 1 int32; padded to 8 bytes), the tape's doubles up to the pass records, then only the
// pass records the step used, node by node (min(count, kMaxPasses) per node), the whole rounded up to 16 bytes. The
// pass records dominate the unpacked tape (kMaxPasses slots per node), and a node takes about 1.2 passes per step, so a
// record is about a third of the tape; the stored offsets let its reader place every pass without a scan.
__host__ __device__ __forceinline__ std::size_t record_ints_bytes(const adj::TapeLayout& L, int nn) {
  return ((L.ints + static_cast<std::size_t>(nn) + 1) * sizeof(std::int32_t) + 7) & ~static_cast<std::size_t>(7);
}

__host__ __device__ __forceinline__ std::size_t record_bytes(const adj::TapeLayout& L, int nn, int records) {
  return (record_ints_bytes(L, nn) + (L.passes + static_cast<std::size_t>(records) * adj::kPassFields) * sizeof(double) + 15) &
         ~static_cast<std::size_t>(15);
}

// poff[n] = the first pass record of node n in the packed order, poff[nn] = their total (warp 0 scans the counts).
template <int W>
__device__ __forceinline__ void pass_offsets(const std::int32_t* npass, int nn, std::int32_t* poff, const Team<W>& T) {
  if (T.warp == 0) {
    int carry = 0;
    for (int base = 0; base < nn; base += 32) {
      const int n = base + T.lane;
      const int v = n < nn ? min(npass[n], adj::kMaxPasses) : 0;
      int x = v;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (T.lane >= o) x += y;
      }
      if (n < nn) poff[n] = carry + x - v;
      carry += __shfl_sync(0xffffffffu, x, 31);
    }
    if (T.lane == 0) poff[nn] = carry;
  }
  T.sync();
}

// Packs the step's tape (shared memory) into dst (global); returns the record's bytes. Every thread of the team calls
// it; the tape may be overwritten once it returns.
template <int W>
__device__ __forceinline__ std::size_t store_record(const adj::Tape& tp, int nn, std::int32_t* poff, unsigned char* dst, const Team<W>& T) {
  const adj::TapeLayout& L = tp.L;
  pass_offsets(tp.i + L.npass, nn, poff, T);
  std::int32_t* di = reinterpret_cast<std::int32_t*>(dst);
  for (std::size_t i = T.rank; i < L.ints; i += 32 * W) di[i] = tp.i[i];
  for (int n = T.rank; n <= nn; n += 32 * W) di[L.ints + n] = poff[n];
  double* dd = reinterpret_cast<double*>(dst + record_ints_bytes(L, nn));
  for (std::size_t i = T.rank; i < L.passes; i += 32 * W) dd[i] = tp.d[i];
  constexpr int kPerNode = adj::kMaxPasses * adj::kPassFields;
  for (int i = T.rank; i < nn * kPerNode; i += 32 * W) {
    const int n = i / kPerNode, k = (i / adj::kPassFields) % adj::kMaxPasses, f = i % adj::kPassFields;
    if (k < tp.i[L.npass + n]) dd[L.passes + static_cast<std::size_t>(poff[n] + k) * adj::kPassFields + f] = tp.d[L.passes + i];
  }
  const std::size_t bytes = record_bytes(L, nn, poff[nn]);
  T.sync();
  return bytes;
}

// Unpacks a record (global) into the step's tape in shared memory, in one round of loads and one barrier: the pass
// records go to their slots by the record's own offsets; slots the step did not use are left as they are (the replay
// reads only the used ones).
template <int W>
__device__ __forceinline__ void load_record(const unsigned char* src, const adj::Tape& tp, int nn, const Team<W>& T) {
  const adj::TapeLayout& L = tp.L;
  const std::int32_t* si = reinterpret_cast<const std::int32_t*>(src);
  const std::int32_t* soff = si + L.ints;
  for (std::size_t i = T.rank; i < L.ints; i += 32 * W) tp.i[i] = si[i];
  const double* sd = reinterpret_cast<const double*>(src + record_ints_bytes(L, nn));
  for (std::size_t i = T.rank; i < L.passes; i += 32 * W) tp.d[i] = sd[i];
  constexpr int kPerNode = adj::kMaxPasses * adj::kPassFields;
  for (int i = T.rank; i < nn * kPerNode; i += 32 * W) {
    const int n = i / kPerNode, k = (i / adj::kPassFields) % adj::kMaxPasses, f = i % adj::kPassFields;
    if (k < si[L.npass + n]) tp.d[L.passes + i] = sd[L.passes + static_cast<std::size_t>(soff[n] + k) * adj::kPassFields + f];
  }
  T.sync();
}

// The step's inputs into its tape, before the step: the scalars and every node's state, pass counts cleared.
template <int W>
__device__ __forceinline__ void tape_inputs(const adj::Tape& tp, const SimRegs& R, const Slot& S, int nn, const Team<W>& T) {
  const adj::TapeLayout& L = tp.L;
  if (T.leader()) {
    tp.d[L.scal] = R.t; tp.d[L.scal + 1] = R.zO; tp.d[L.scal + 2] = R.pitch; tp.d[L.scal + 3] = R.roll;
    tp.d[L.scal + 4] = R.vz; tp.d[L.scal + 5] = R.wth; tp.d[L.scal + 6] = R.wph;
  }
  for (int n = T.rank; n < nn; n += 32 * W) {
    tp.d[L.volIn + n] = S.vol[n]; tp.d[L.levelIn + n] = S.level[n];
    tp.d[L.cxIn + n] = S.cx[n]; tp.d[L.cyIn + n] = S.cy[n]; tp.d[L.czIn + n] = S.cz[n];
    tp.i[L.npass + n] = 0;
  }
  T.sync();
}

// The ring: a record at virtual offset v sits at v mod cap; a record that would run past the end starts the next lap
// instead. After the last write at virtual end E the ring holds exactly the records at offsets >= E - cap.
__device__ __forceinline__ long long ring_place(long long v, std::size_t cap, std::size_t maxRecord) {
  const long long c = static_cast<long long>(cap);
  if (v % c + static_cast<long long>(maxRecord) > c) v = (v / c + 1) * c;
  return v;
}

__device__ __forceinline__ long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return static_cast<long long>(t);
}

// The objective's adjoint at the state with scalars (zO, pitch, roll): every thread adds the same values.
__device__ __forceinline__ void add_sample_adjoint(const DevModel& M, double zO, double th, double ph, double aTrim, double aHeave, double* aSc) {
  const PoseD F = adj::pose_of(M, zO, th, ph);
  AdjPose aP;
  adj::zero(aP);
  adj::trim_heave_reverse(M, aTrim, aHeave, aP, aSc[1]);
  adj::pose_reverse(M, F, aP, aSc[0], aSc[1], aSc[2]);
}

template <int W>
__global__ void __launch_bounds__(W * 32) adjoint_batch(DevModel M, AdjRun B, SlotLayout SL, AdjLayout AL) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int team = blockIdx.x;
  Team<W> T;
  T.warp = threadIdx.x >> 5;
  T.lane = threadIdx.x & 31;
  T.rank = threadIdx.x;
  T.bar = 1;
  AdjTeam<W> AT{T.rank, 32 * W, T.warp, W, T.lane, 32, 1};
  Slot S = carve_slot(smem, SL);
  AdjSmem A = carve_adjoint(smem + SL.bytes, AL);
  const adj::TapeLayout TL = adj::tape_layout(M.nn, M.ng);
  const std::size_t recMax = record_bytes(TL, M.nn, M.nn * adj::kMaxPasses);
  const std::size_t recSize = 7 + 5 * static_cast<std::size_t>(M.nn);
  double* const ckpt = B.ckpt + static_cast<std::size_t>(team) * B.maxCkpt * recSize;
  unsigned char* const ring = B.arena + static_cast<std::size_t>(team) * B.arenaBytes;
  long long* const off = B.stepOff + static_cast<std::size_t>(team) * (B.maxSteps + 1);
  std::int32_t* const rb = B.recBytes + static_cast<std::size_t>(team) * (B.maxSteps + 1);
  double* const sink = B.sink + static_cast<std::size_t>(team) * (M.evCap + M.nmon + M.nmark + 1);
  std::int32_t* const isink = B.isink + static_cast<std::size_t>(team) * (M.evCap + 1);
  const adj::Tape sp = adj::tape_at(A.tape, TL);
  const int NS = B.nsamples;
  for (;;) {
    if (T.leader()) {
      const int q = atomicAdd(B.queue, 1);
      S.misc[0] = B.order == nullptr || q >= B.count ? q : B.order[q];
      S.misc[2] = W * (32 / kLevelLanes<false>);  // the level solve's group counter for the first step (team_step resets it)
    }
    T.sync();
    const int inst = S.misc[0];
    T.sync();
    if (inst >= B.count) return;
    const long long tStart = global_ns();
    long long tRecompute = 0, tReverse = 0, nRecomputed = 0;
    const std::size_t ic = static_cast<std::size_t>(inst) * M.nc;
    const AdjInst I{B.en + ic, B.area + ic, B.tOn + ic, sink, isink, M.nmon};
    // the event bookkeeping sinks: overflow and mark times set (nothing fires), so events never write
    for (int k = T.rank; k < M.nmon + M.nmark + 1; k += 32 * W) sink[k] = 1.0;
    SimRegs R;
    {
      // the instance's initial state
      const std::size_t in = static_cast<std::size_t>(inst) * M.nn;
      double* c = ckpt;  // checkpoint 0 is the initial state
      if (T.leader())
        for (int k = 0; k < 7; ++k) c[k] = B.st0[static_cast<std::size_t>(inst) * 7 + k];
      for (int n = T.rank; n < M.nn; n += 32 * W) {
        c[7 + n] = B.vol0[in + n]; c[7 + M.nn + n] = B.level0[in + n];
        c[7 + 2 * M.nn + n] = B.cx0[in + n]; c[7 + 3 * M.nn + n] = B.cy0[in + n]; c[7 + 4 * M.nn + n] = B.cz0[in + n];
      }
      __threadfence_block();
      T.sync();
      load_state(c, R, S, M, T);
    }
    // ---- 1. forward with checkpoints, the objective's samples and (tapeForward) every step's record
    Pose& F = *S.pose;
    F = make_pose(M, R.zO, R.pitch, R.roll);
    const double* trimT = B.trimT + static_cast<std::size_t>(inst) * NS;
    const double* heaveT = B.heaveT + static_cast<std::size_t>(inst) * NS;
    double J = 0;
    int k = 0;
    long long s = 0, v = 0;
    for (;; ++s) {
      if (s % B.K == 0 && s > 0) {
        save_state(ckpt + static_cast<std::size_t>(s / B.K) * recSize, R, S, M.nn, T);
        T.sync();
      }
      if (R.foundered || R.t >= B.tMax || s >= B.maxSteps) break;
      while (k < NS && R.t >= B.sampleT[k]) {
        double tr, hv;
        adj::trim_heave(M, PoseD{F.R00, F.R01, F.R02, F.R10, F.R11, F.R12, F.R20, F.R21, F.R22, F.tx, F.ty, F.tz, F.cth, F.iR}, R.pitch, tr, hv);
        J += (tr - trimT[k]) * (tr - trimT[k]) + (hv - heaveT[k]) * (hv - heaveT[k]);
        if (T.leader()) {
          B.trim[static_cast<std::size_t>(inst) * NS + k] = tr; B.heave[static_cast<std::size_t>(inst) * NS + k] = hv;
          A.sampleS[k] = static_cast<double>(s);
        }
        ++k;
      }
      if (B.tapeForward) {
        tape_inputs(sp, R, S, M.nn, T);
        team_step<false, W>(M, F, R, S, I, T, GpuTape{sp});
        T.sync();
        v = ring_place(v, B.arenaBytes, recMax);
        if (T.leader()) off[s] = v;
        const std::size_t bytes = store_record(sp, M.nn, A.poff, ring + v % static_cast<long long>(B.arenaBytes), T);
        if (T.leader()) rb[s] = static_cast<std::int32_t>(bytes);
        v += static_cast<long long>(bytes);
      } else {
        team_step<false, W>(M, F, R, S, I, T);
      }
      F = make_pose(M, R.zO, R.pitch, R.roll);
    }
    const long long S_end = s;
    // the ring holds the records at virtual offsets >= v - cap: a segment is reversed from the ring when its first
    // step's record is among them
    const long long kept = B.tapeForward ? v - static_cast<long long>(B.arenaBytes) : LLONG_MAX;
    const double zE = R.zO, thE = R.pitch, phE = R.roll;
    for (; k < NS; ++k) {
      double tr, hv;
      adj::trim_heave(M, PoseD{F.R00, F.R01, F.R02, F.R10, F.R11, F.R12, F.R20, F.R21, F.R22, F.tx, F.ty, F.tz, F.cth, F.iR}, R.pitch, tr, hv);
      J += (tr - trimT[k]) * (tr - trimT[k]) + (hv - heaveT[k]) * (hv - heaveT[k]);
      if (T.leader()) {
        B.trim[static_cast<std::size_t>(inst) * NS + k] = tr; B.heave[static_cast<std::size_t>(inst) * NS + k] = hv;
        A.sampleS[k] = static_cast<double>(S_end);
      }
    }
    __threadfence_block();
    T.sync();
    const long long tForward = global_ns() - tStart;
    // ---- 2. reverse
    double aSc[6] = {0, 0, 0, 0, 0, 0};
    for (int n = T.rank; n < M.nn; n += 32 * W) { A.as.aVol[n] = 0; A.as.aLevel[n] = 0; A.as.aCx[n] = 0; A.as.aCy[n] = 0; A.as.aCz[n] = 0; }
    for (int c = T.rank; c < M.nc; c += 32 * W) A.grad[c] = 0;
    T.sync();
    // the samples at the final state (the objective's values of the trim and heave, recomputed from the outputs)
    for (int q = 0; q < NS; ++q)
      if (static_cast<long long>(A.sampleS[q]) == S_end) {
        const double tr = B.trim[static_cast<std::size_t>(inst) * NS + q], hv = B.heave[static_cast<std::size_t>(inst) * NS + q];
        add_sample_adjoint(M, zE, thE, phE, 2 * (tr - trimT[q]), 2 * (hv - heaveT[q]), aSc);
      }
    int err = 0;
    const long long nseg = (S_end + B.K - 1) / B.K;
    for (long long g = nseg - 1; g >= 0; --g) {
      const long long s0 = g * B.K, s1 = (s0 + B.K < S_end) ? s0 + B.K : S_end;
      const long long tSeg = global_ns();
      if (!(B.tapeForward && off[s0] >= kept)) {
        // recompute the segment from its checkpoint into the ring (every later segment has been reversed already, so
        // the whole ring is free; it holds K records of the largest size)
        load_state(ckpt + static_cast<std::size_t>(g) * recSize, R, S, M, T);
        F = make_pose(M, R.zO, R.pitch, R.roll);
        long long w = 0;
        nRecomputed += s1 - s0;
        for (long long st = s0; st < s1; ++st) {
          tape_inputs(sp, R, S, M.nn, T);
          team_step<false, W>(M, F, R, S, I, T, GpuTape{sp});
          T.sync();
          if (T.leader()) off[st] = w;
          const std::size_t bytes = store_record(sp, M.nn, A.poff, ring + w, T);
          if (T.leader()) rb[st] = static_cast<std::int32_t>(bytes);
          w += static_cast<long long>(bytes);
          F = make_pose(M, R.zO, R.pitch, R.roll);
        }
      }
      __threadfence_block();
      T.sync();
      const long long tRev = global_ns();
      tRecompute += tRev - tSeg;
      bool staged = false;  // the record of step st is in the raw buffer (copied while step st + 1 was reversed)
      for (long long st = s1 - 1; st >= s0; --st) {
        if (staged) {
          asm volatile("cp.async.wait_all;" ::: "memory");  // this thread's copies; the barrier makes all of them visible
          T.sync();
          load_record(A.raw, sp, M.nn, T);
        } else {
          load_record(ring + off[st] % static_cast<long long>(B.arenaBytes), sp, M.nn, T);
        }
        staged = false;
        if (st > s0) {
          const unsigned char* next = ring + off[st - 1] % static_cast<long long>(B.arenaBytes);
          if (B.stageRecords) {
            // the next step's record (the one before this) into shared memory while this one is reversed: 16-byte
            // asynchronous copies spread over the team (records and the buffer are 16-byte aligned, their sizes whole
            // numbers of 16 bytes)
            const int chunks = rb[st - 1] / 16;
            for (int k = T.rank; k < chunks; k += 32 * W) {
              const auto dst = static_cast<unsigned>(__cvta_generic_to_shared(A.raw + 16 * k));
              asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(next + 16 * k) : "memory");
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
            staged = true;
          } else if (T.leader()) {
            // or at least into L2
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(next), "r"(static_cast<unsigned>(rb[st - 1])) : "memory");
          }
        }
        adj::reverse_step(AT, M, sp, I.en(), I.area(), I.tOn(), A.rs, A.as, aSc, A.grad, &err);
        for (int q = 0; q < NS; ++q)
          if (static_cast<long long>(A.sampleS[q]) == st) {
            const double tr = B.trim[static_cast<std::size_t>(inst) * NS + q], hv = B.heave[static_cast<std::size_t>(inst) * NS + q];
            add_sample_adjoint(M, sp.d[TL.scal + 1], sp.d[TL.scal + 2], sp.d[TL.scal + 3], 2 * (tr - trimT[q]), 2 * (hv - heaveT[q]), aSc);
          }
        T.sync();
      }
      tReverse += global_ns() - tRev;
    }
    T.sync();
    for (int c = T.rank; c < M.nc; c += 32 * W) B.grad[ic + c] = A.grad[c];
    if (err) atomicOr(B.error + inst, err);
    if (T.leader()) {
      B.J[inst] = J; B.steps[inst] = S_end;
      B.phaseNs[3 * static_cast<std::size_t>(inst)] = tForward;
      B.phaseNs[3 * static_cast<std::size_t>(inst) + 1] = tRecompute;
      B.phaseNs[3 * static_cast<std::size_t>(inst) + 2] = tReverse;
      B.recomputed[inst] = nRecomputed;
    }
    T.sync();
  }
}

}  // namespace

AdjLayout adjoint_layout(int nn, int nc, int ng, int nsamples, int W, bool withRaw) {
  AdjLayout A{};
  std::uint32_t off = 0;
  auto take16 = [&](std::size_t bytes) {
    const std::uint32_t at = off;
    off = static_cast<std::uint32_t>((off + bytes + 15) & ~static_cast<std::size_t>(15));
    return at;
  };
  const std::size_t N = sizeof(double) * static_cast<std::size_t>(std::max(nn, 1));
  const std::size_t C = sizeof(double) * static_cast<std::size_t>(std::max(nc, 1));
  A.hEff = take16(N); A.aEff = take16(N); A.dV = take16(C); A.volPost = take16(N);
  A.deg = take16(sizeof(int) * static_cast<std::size_t>(std::max(nn, 1)));
  A.clip = take16(sizeof(std::int32_t) * static_cast<std::size_t>(std::max(nn, 1)));
  A.aVolPost = take16(N); A.aCxs = take16(N); A.aCys = take16(N); A.aCzs = take16(N); A.aVs = take16(N); A.aAcc = take16(N);
  A.aZmx = take16(N); A.aLs = take16(N); A.aAs = take16(N);
  A.faHA = take16(C); A.faHB = take16(C); A.faAA = take16(C); A.faAB = take16(C);
  A.red = take16(sizeof(double) * 16 * static_cast<std::size_t>(W));
  A.work = take16(sizeof(adj::UnitWork) * static_cast<std::size_t>(W));
  A.plain = take16(static_cast<std::size_t>(std::max(nn, 1)));
  A.units = take16(sizeof(std::int32_t) * static_cast<std::size_t>(std::max(nn, 1)));
  A.nunits = take16(sizeof(std::int32_t));
  A.pw = take16(2 * C);
  A.replays = take16(sizeof(adj::Replay) * static_cast<std::size_t>(std::max(nn, 1)));
  A.raw = withRaw ? take16(record_bytes(adj::tape_layout(nn, ng), nn, nn * adj::kMaxPasses)) : 0;
  A.aVol = take16(N); A.aLevel = take16(N); A.aCx = take16(N); A.aCy = take16(N); A.aCz = take16(N);
  A.grad = take16(C);
  A.sampleS = take16(sizeof(double) * static_cast<std::size_t>(std::max(nsamples, 1)));
  A.tape = take16(adj::tape_layout(nn, ng).bytes);
  A.poff = take16(sizeof(std::int32_t) * (static_cast<std::size_t>(std::max(nn, 1)) + 1));
  A.bytes = off;
  return A;
}

std::size_t adjoint_tape_bytes(int nn, int ng) { return record_bytes(adj::tape_layout(nn, ng), nn, nn * adj::kMaxPasses); }
std::size_t adjoint_record_bytes(int nn, int ng, int passRecords) { return record_bytes(adj::tape_layout(nn, ng), nn, passRecords); }

cudaError_t configure_adjoint_kernel(int W, std::size_t smem) {
  const int b = static_cast<int>(smem);
  switch (W) {
    case 4: return cudaFuncSetAttribute(adjoint_batch<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    case 8: return cudaFuncSetAttribute(adjoint_batch<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    case 16: return cudaFuncSetAttribute(adjoint_batch<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  }
  return cudaErrorInvalidValue;
}

cudaError_t adjoint_occupancy(int W, std::size_t smem, int* blocksPerSM) {
  switch (W) {
    case 4: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, adjoint_batch<4>, 4 * 32, smem);
    case 8: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, adjoint_batch<8>, 8 * 32, smem);
    case 16: return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSM, adjoint_batch<16>, 16 * 32, smem);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_adjoint_kernel(int W, const DevModel& M, const AdjRun& B, const SlotLayout& SL, const AdjLayout& AL, int teams,
                                  cudaStream_t stream) {
  const std::size_t smem = static_cast<std::size_t>(SL.bytes) + AL.bytes;
  switch (W) {
    case 4: adjoint_batch<4><<<teams, 4 * 32, smem, stream>>>(M, B, SL, AL); break;
    case 8: adjoint_batch<8><<<teams, 8 * 32, smem, stream>>>(M, B, SL, AL); break;
    case 16: adjoint_batch<16><<<teams, 16 * 32, smem, stream>>>(M, B, SL, AL); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace ssb
