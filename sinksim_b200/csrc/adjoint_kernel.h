// Host-side entry points of the adjoint kernel (adjoint_kernel.cu): the gradient of a trajectory objective with
// respect to every connection area, by a discrete adjoint with checkpoints.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "device_model.h"

namespace ssb {

// One adjoint launch: per instance its connection fields, initial state and objective targets in; the objective, its
// gradient and the run's length out; per team its checkpoints, tape and event sinks.
struct AdjRun {
  std::int32_t count;
  const std::uint8_t* en;                       // [count x nc]
  const double *area, *tOn;                     // [count x nc]
  const double* st0;                            // [count x 7]: t, zO, pitch, roll, vz, wth, wph
  const double *vol0, *level0, *cx0, *cy0, *cz0;  // [count x nn]
  double tMax;
  long long maxSteps;                           // bound on a run's steps (sizes the checkpoints)
  std::int32_t nsamples;
  const double* sampleT;                        // [nsamples] ascending
  const double *trimT, *heaveT;                 // [count x nsamples] targets
  double *trim, *heave;                         // [count x nsamples] the run's values at the samples
  double* J;                                    // [count]
  double* grad;                                 // [count x nc] d J / d area
  long long* steps;                             // [count]
  std::int32_t* error;                          // [count] adjoint error bits (adj::AdjointError), zeroed by the host
  std::int32_t* queue;                          // work-queue head, zeroed by the host
  const std::int32_t* order;                    // [count] or null: queue position k claims instance order[k]
  std::int32_t K;                               // steps between checkpoints
  std::int32_t maxCkpt;                         // checkpoints per team
  double* ckpt;                                 // [teams x maxCkpt x (7 + 5 nn)]
  // Per team a ring of packed step records (adjoint_kernel.cu: store_record) of arenaBytes bytes, at least K records of
  // the largest size, and the virtual offset of every step's record ([teams x (maxSteps + 1)]). With tapeForward the
  // forward run records every step, and the reverse recomputes only the segments the ring no longer holds.
  unsigned char* arena;
  std::size_t arenaBytes;
  long long* stepOff;
  std::int32_t* recBytes;                       // [teams x (maxSteps + 1)] each step record's bytes
  std::int32_t tapeForward;
  std::int32_t stageRecords;                    // 1: the layout has a raw record buffer (AdjLayout::raw): the reverse
                                                // copies the next step's record into it while it reverses this one
  double* sink;                                 // [teams x (evCap + nmon + nmark + 1)]
  std::int32_t* isink;                          // [teams x (evCap + 1)]
  long long* phaseNs;                           // [count x 3] the team's time on the instance (globaltimer ns):
                                                // forward, recomputation of the segments, reverse steps
  long long* recomputed;                        // [count] steps recomputed from checkpoints
};

// Byte offsets of a team's reverse arrays in shared memory, after its forward slot.
struct AdjLayout {
  std::uint32_t hEff, aEff, dV, volPost, deg, clip, aVolPost, aCxs, aCys, aCzs, aVs, aAcc, aZmx, aLs, aAs, faHA, faHB, faAA, faAB, red, work, plain, units, nunits, pw, replays, raw;
  std::uint32_t aVol, aLevel, aCx, aCy, aCz, grad, sampleS, tape, poff, bytes;
};

// withRaw: room for one packed step record of the largest size (the reverse's asynchronous copy of the next record)
AdjLayout adjoint_layout(int nn, int nc, int ng, int nsamples, int teamWarps, bool withRaw = false);
std::size_t adjoint_tape_bytes(int nn, int ng);  // the largest packed step record
std::size_t adjoint_record_bytes(int nn, int ng, int passRecords);  // a packed step record holding passRecords passes
cudaError_t configure_adjoint_kernel(int teamWarps, std::size_t smem);
cudaError_t adjoint_occupancy(int teamWarps, std::size_t smem, int* blocksPerSM);
cudaError_t launch_adjoint_kernel(int teamWarps, const DevModel& M, const AdjRun& run, const SlotLayout& slot, const AdjLayout& layout, int teams,
                                  cudaStream_t stream);

}  // namespace ssb
