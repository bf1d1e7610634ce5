// Batched stirred-tank runner: many tanks of different sizes advanced in
// lockstep, one launch per kernel family per step for all of them.
//
// Reference: the sweep runs its cases one after another, each through the
// full runner loop (crates/lbm-cli/src/sweep.rs:47-106, runner.rs:1079-1129).
// Here every case keeps its own device state (an Engine); a batch holds a
// device table of per-case descriptors (the case's HydroParams, its IBM
// arguments, force slots and per-step series) and launches
//
//   side stream:  prep -> (interp -> spread -> diag) x sweeps -> commit -> forced cells
//   main stream:  full-grid sweep of every case (lean TRT kernel)
//   join:         cached-field refresh (fprev = fcur)
//
// per step, each over the concatenation of all cases' cells, slots or
// markers. A block never straddles two cases: each family has a table of
// per-case block offsets, and a block finds its case by binary search. The
// per-case IBM early exit, the diagnostics reduction (last block of the
// case) and the step counters are per case, so every case follows exactly
// the sequence it would follow alone.
#pragma once
#include "hydro_lean.cuh"
#include "ibm.cuh"

namespace lbmb {

constexpr int BATCH_BLOCK = 128;
static_assert(BATCH_BLOCK == LEAN_BLOCK && BATCH_BLOCK == IBM_BLOCK, "one block size for every family");

struct BatchCase {
  HydroParams<float> hp;
  uint32_t n;  // cells
  int nx, ny, nz;
  const int64_t* slot_cell;  // forced cells (= force slots)
  int64_t nslots;
  Vec4<float>* fcur;
  Vec4<float>* fprev;
  IbmArgs ibm;
  double gx, gy, gz;
  double* series_torque;  // per step
  int64_t* counter;
};

// Case of block b: the last c with off[c] <= b (off has ncase + 1 entries).
__device__ __forceinline__ int batch_case(const int32_t* off, int ncase, int b) {
  int lo = 0, hi = ncase;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(off + mid) <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <int Q, class S, bool ODD, int MINB>
__global__ void __launch_bounds__(BATCH_BLOCK, MINB)
    batch_hydro_kernel(const BatchCase* cs, const int32_t* off, int ncase) {
  const int k = batch_case(off, ncase, blockIdx.x);
  const BatchCase& b = cs[k];
  const uint32_t c = uint32_t(int(blockIdx.x) - __ldg(off + k)) * BATCH_BLOCK + threadIdx.x;
  if (c >= b.n) return;
  lean_cell<Q, S, ODD>(b.hp, c);
}

template <int Q, class S, bool ODD>
static __global__ void __launch_bounds__(BATCH_BLOCK) batch_cells_kernel(const BatchCase* cs, const int32_t* off, int ncase) {
  const int k = batch_case(off, ncase, blockIdx.x);
  const BatchCase& b = cs[k];
  const int64_t i = int64_t(int(blockIdx.x) - __ldg(off + k)) * BATCH_BLOCK + threadIdx.x;
  if (i >= b.nslots) return;
  forced_cell<Q, S, COLL_TRT, ODD>(b.hp, uint32_t(b.slot_cell[i]));
}

// u_now over the slots; the runner clears the force field before the IBM,
// so the field at call time is zero and the new field starts from zero.
template <int Q, class S>
static __global__ void __launch_bounds__(BATCH_BLOCK)
    batch_prep_kernel(const BatchCase* cs, const int32_t* off, int ncase, int parity) {
  const int k = batch_case(off, ncase, blockIdx.x);
  const BatchCase& b = cs[k];
  const int64_t i = int64_t(int(blockIdx.x) - __ldg(off + k)) * BATCH_BLOCK + threadIdx.x;
  ibm_prep_body<Q, S>(b.ibm, i, static_cast<const S*>(b.hp.f), int64_t(b.hp.plane), b.slot_cell, b.hp.flags,
                      b.hp.nbr, b.nx, b.ny, b.nz, parity, b.fcur, 0, b.gx, b.gy, b.gz);
  if (i < b.ibm.ns) b.fcur[b.ibm.bslot[i]] = Vec4<float>{0.f, 0.f, 0.f, 0.f};
}

static __global__ void __launch_bounds__(BATCH_BLOCK)
    batch_interp_kernel(const BatchCase* cs, const int32_t* off, int ncase, int sweep) {
  const int k = batch_case(off, ncase, blockIdx.x);
  const BatchCase& b = cs[k];
  ibm_interp_body(b.ibm, int64_t(int(blockIdx.x) - __ldg(off + k)) * BATCH_BLOCK + threadIdx.x, sweep);
}

static __global__ void __launch_bounds__(BATCH_BLOCK) batch_spread_kernel(const BatchCase* cs, const int32_t* off, int ncase) {
  const int k = batch_case(off, ncase, blockIdx.x);
  ibm_spread_body(cs[k].ibm, int(blockIdx.x) - __ldg(off + k));
}

static __global__ void __launch_bounds__(BATCH_BLOCK)
    batch_diag_kernel(const BatchCase* cs, const int32_t* off_m, const int32_t* off_s, int ncase, int sweep) {
  const int k = batch_case(off_m, ncase, blockIdx.x);
  const int b0 = __ldg(off_m + k), nblk = __ldg(off_m + k + 1) - b0;
  const int nblk_spread = __ldg(off_s + k + 1) - __ldg(off_s + k);
  ibm_diag_body(cs[k].ibm, sweep, nblk_spread, unsigned(int(blockIdx.x) - b0), unsigned(nblk));
}

static __global__ void __launch_bounds__(BATCH_BLOCK) batch_commit_kernel(const BatchCase* cs, const int32_t* off, int ncase) {
  const int k = batch_case(off, ncase, blockIdx.x);
  const BatchCase& b = cs[k];
  ibm_commit_body<float>(b.ibm, int64_t(int(blockIdx.x) - __ldg(off + k)) * BATCH_BLOCK + threadIdx.x, b.fcur,
                         b.series_torque, nullptr, nullptr, b.counter);
}

static __global__ void __launch_bounds__(BATCH_BLOCK) batch_fprev_kernel(const BatchCase* cs, const int32_t* off, int ncase) {
  const int k = batch_case(off, ncase, blockIdx.x);
  const BatchCase& b = cs[k];
  const int64_t i = int64_t(int(blockIdx.x) - __ldg(off + k)) * BATCH_BLOCK + threadIdx.x;
  if (i < b.nslots) b.fprev[i] = b.fcur[i];
}

}  // namespace lbmb
