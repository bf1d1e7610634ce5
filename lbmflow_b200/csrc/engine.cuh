#pragma once
// Device engine behind include/lbmb.h: device memory, launch sequencing and
// CUDA graphs for one (lattice, storage) pair. Each pair is instantiated in
// its own translation unit (engine_q*_*.cu); solver.cu holds validation and
// the C ABI.
//
// Reference boundary: trait Backend<L, T> (crates/lbm-core/src/backend.rs:
// 126-363) driven by Solver<L, T, B, H> (crates/lbm-core/src/solver.rs:
// 1503-1541). One engine owns one device state; the C entry points at the
// end of this file translate exceptions into status codes.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/lbmb.h"
#include "checkpoint.hpp"
#include "aux.cuh"
#include "hydro.cuh"
#include "hydro_tma.cuh"
#include "hydro_async.cuh"
#include "hydro_pair.cuh"
#include "hydro_tile.cuh"
#include "hydro_lean.cuh"
#include "hydro_window.cuh"
#include "batch.cuh"
#include "adjoint.cuh"
#include "ibm.cuh"
#include "scalar.cuh"
#include "stress.cuh"

namespace lbmb {

extern thread_local std::string g_last_error;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess)                                                                      \
      throw ::lbmb::Error(e_ == cudaErrorMemoryAllocation ? LBMB_ERR_NOMEM : LBMB_ERR_CUDA,     \
                          std::string(#x) + ": " + cudaGetErrorString(e_));                     \
  } while (0)

inline void invalid(const std::string& m) { throw Error(LBMB_ERR_INVALID, m); }

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t k) {
    release();
    if (k == 0) k = 1;
    CK(cudaMalloc(&p, k * sizeof(T)));
    n = k;
  }
  void upload(const T* h, size_t k, cudaStream_t st) {
    if (k > n) alloc(k);
    if (k) CK(cudaMemcpyAsync(p, h, k * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  void upload(const std::vector<T>& v, cudaStream_t st) { upload(v.data(), v.size(), st); }
};

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

struct BodyState {
  int64_t nm = 0;
  std::vector<double> pos, weight;
  double center[3] = {0, 0, 0}, omega[3] = {0, 0, 0};
  double scale = 1.0;
  int radius = 0;  // radius the device stencils were built for (0: none)
  DevBuf<double> d_pos, d_weight, st_w, st_cks, cs_w, imp, mob, rmf, part_spread, part_diag;
  DevBuf<int32_t> st_off, st_slot, bslot, cs_off, cs_marker;
  int64_t ns = 0;
  bool empty_stencil = false;
};

template <class A>
struct ScalarStateT {
  std::string name;
  int q = 7;
  double diffusivity = 0.0;
  int parity = 0;
  int64_t hplane = 0;
  DevBuf<A> h;
  DevBuf<double> part, stats;
};

// Type-erased batch of engines advanced in lockstep (batch.cuh).
struct BatchBase {
  virtual ~BatchBase() = default;
  virtual void run(int64_t steps, double* torque, double* device_ms) = 0;
  virtual void autotune(int steps, int32_t* even, int32_t* odd, double* best_ms) = 0;
};

// Type-erased engine interface.
struct EngineBase {
  virtual ~EngineBase() = default;
  virtual void step(int64_t n) = 0;
  virtual void stage_in(const double* f) = 0;
  virtual void stage_out(double* f) = 0;
  virtual void init_fields(const double* rho, const double* u) = 0;
  virtual void read_moments(double* rho, double* ux, double* uy, double* uz) = 0;
  virtual void reduce_all(double out[5]) = 0;
  virtual void clear_force_field() = 0;
  virtual void get_force_field(double* out) = 0;
  virtual void ibm_set_body(int b, const double* pos, const double* w, int64_t n, const double* c,
                            const double* om) = 0;
  virtual void ibm_apply(int b, const lbmb_ibm_config& cfg, lbmb_ibm_diag* diag) = 0;
  virtual void runner_step(int b, const double* pos, const double* w, int64_t n, const double* c,
                           const double* om, const lbmb_ibm_config& cfg, lbmb_ibm_diag* diag) = 0;
  virtual int enable_scalar(int q, double d) = 0;
  virtual void set_scalar(int k, const double* c) = 0;
  virtual void get_scalar(int k, double* c) = 0;
  virtual void run_impeller(int b, const lbmb_ibm_config& cfg, int64_t steps, int k, int64_t probe_every,
                            double* torque, double* ff, double* cv, int32_t* iters) = 0;
  virtual void run_status(int64_t* executed, int32_t* diverged) = 0;
  virtual void set_wait_limit(long long cycles) = 0;
  // What this handle's current configuration allows: the adjoint and the
  // batched runner (the checks lbmb_adjoint_torque / lbmb_batch_create make).
  virtual void allows(int32_t* adjoint, int32_t* batch) const = 0;
  virtual void sync() = 0;
  virtual void timing(double* total_ms, double* hydro_ms, int64_t* launches) = 0;
  virtual void set_sweep_kernel(int kind) = 0;
  virtual int sweep_kernel() const = 0;
  virtual void set_sweep_variant(int even, int odd) = 0;
  virtual void autotune_sweep(int steps, lbmb_autotune_result* out, int32_t* trial_desc, double* trial_ms,
                              int capacity) = 0;
  virtual void adjoint_torque(const lbmb_ibm_config& cfg, const lbmb_adjoint_config& ac, lbmb_adjoint_result* out,
                              double* dJ_dpos, double* torque) = 0;
  // A batch over `all` (this engine's type for every entry), one body each.
  virtual BatchBase* make_batch(const std::vector<EngineBase*>& all, const int32_t* bodies,
                                const lbmb_ibm_config& cfg) = 0;
  virtual int64_t cells() const = 0;
  virtual void strain_rate(double* s6, double* gamma) = 0;
  virtual void set_omega_field(const double* omega) = 0;
  virtual void velocity_gradient(double* g9) = 0;
  virtual void wale_update(double tau_eff_max, double* nu_t, lbmb_wale_diag* diag) = 0;
  virtual void scalar_oxygen(int k, const OxygenSourceArgs& a, double* sum, lbmb_oxygen_diag* diag,
                             int64_t* active) = 0;
  virtual void stress_field(double dx, double dt, double mu, double* s6, double* gamma, double* viscous) = 0;
  virtual void stress_summary(double dx, double dt, double mu, double t_gamma, double t_tau, lbmb_percentiles* pg,
                              lbmb_percentiles* pt, double* device_ms) = 0;
  virtual void wall_shear(double dx, double dt, double rho, double mu, lbmb_wall_shear* out, int64_t capacity,
                          int64_t* count) = 0;
  virtual int q() const = 0;
  virtual const std::vector<uint8_t>& solid() const = 0;
  // Checkpoint/restart in the reference's v3 format (checkpoint.hpp):
  // Solver::save and Solver::restore.
  virtual void checkpoint_save(const std::string& dir) = 0;
  virtual void checkpoint_restore(const std::string& dir) = 0;
  virtual void set_scalar_name(int k, const std::string& name) = 0;
  virtual const lbmb_config& config() const = 0;
  uint64_t time = 0;              // Solver::time: hydro steps taken
  std::vector<double> wall_u_in;  // creation wall velocities (n x 3; empty: zero)
  bool has_qoi = false;           // QoiCheckpointState carried opaque
  std::string qoi_json;
  double last_total_ms = 0.0, last_hydro_ms = 0.0;
  int64_t last_hydro_launches = 0;
};

template <int Q, class S>
struct Engine final : EngineBase {
  using A = typename Codec<S>::A;
  lbmb_config cfg;
  int nx, ny, nz;
  int64_t n, plane;
  int coll;  // COLL_TRT or COLL_CM
  double omega_p, omega_m;
  cudaStream_t st = nullptr, st2 = nullptr;  // main stream, high-priority IBM stream
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_fork = nullptr, ev_join = nullptr;
  // device state
  DevBuf<S> f_alloc;     // populations with a guard margin on both sides
  S* fp = nullptr;       // first element of plane 0
  int64_t margin = 0;    // guard elements before plane 0 and after the last plane
  DevBuf<uint8_t> flags;
  DevBuf<uint32_t> nbr;
  DevBuf<Vec4<A>> wall_u;
  DevBuf<int32_t> fslot;
  int parity = 0;
  // force slots
  int64_t nslots = 0, slot_cap = 0;
  std::vector<int32_t> fslot_h;  // per cell, -1 = none
  std::vector<int64_t> slot_cell_h;
  DevBuf<int64_t> slot_cell;
  DevBuf<Vec4<A>> fprev, fcur;
  DevBuf<double> s_rho, s_unow, s_du, s_spread;
  bool field_present = false;
  bool fprev_stale = false;
  // IBM
  std::vector<std::unique_ptr<BodyState>> bodies;
  DevBuf<IbmDiagDev> d_diag;
  DevBuf<int> d_err;  // device error flag (bounded waits)
  DevBuf<int> d_flag;  // scratch flag of clear_force_field
  int sm_count = 148;
  int64_t ntiles = 0;
  bool rows_aligned = false;
  int kernel_mode = 2;  // lbmb_sweep_kind
  // tile-pipelined sweep: tiles holding a non-solid cell, window offsets
  DevBuf<int32_t> tile_list;
  int n_tiles_active = 0;
  // pair sweep: 64-cell tiles holding a non-solid cell
  DevBuf<uint32_t> pair_list;
  int n_pair_tiles = 0;
  TileDirs tile_dirs[2];
  int tile_grid[2] = {0, 0};
  // persistent window-kernel grid per (parity, concurrent with the IBM chain)
  int window_grid[4] = {0, 0, 0, 0};
  int tma_grid[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // persistent cp.async grid per (parity, collision, concurrent with the IBM chain)
  int async_grid[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // reductions
  DevBuf<double> red_part, red_out;
  int red_blocks = 0;
  // host mirrors
  std::vector<uint8_t> solid_h, flags_h;
  std::vector<double> init_rho_h, init_u_h;
  // device copy of init_u_h (the velocity the scalar equilibrium uses on
  // solid cells), refreshed when init_u_h changes
  DevBuf<double> d_init_u;
  bool d_init_u_ok = false;
  const double* init_u_dev() {
    if (!d_init_u_ok) {
      d_init_u.upload(init_u_h, st);
      d_init_u_ok = true;
    }
    return d_init_u.p;
  }
  // scalars
  std::vector<std::unique_ptr<ScalarStateT<A>>> scalars;
  // graphs
  cudaGraphExec_t step_graph = nullptr;
  int step_graph_len = 0;

  Engine(const lbmb_config& c, const uint8_t* solid, const double* wu) : cfg(c) {
    nx = c.dims[0];
    ny = c.dims[1];
    nz = c.dims[2];
    n = int64_t(nx) * ny * nz;
    plane = ceil_div(n, 64) * 64;
    if (int64_t(Q) * plane >= (int64_t(1) << 31))
      throw Error(LBMB_ERR_UNSUPPORTED, "grid too large: Q x cells must stay below 2^31 element offsets");
    coll = c.collision == LBMB_CENTRAL_MOMENT ? COLL_CM : COLL_TRT;
    double tau = 3.0 * c.nu + 0.5;
    omega_p = 1.0 / tau;
    omega_m = omega_p;
    if (c.collision == LBMB_TRT) omega_m = 1.0 / (c.magic / (tau - 0.5) + 0.5);  // params.rs:205-217
    CK(cudaSetDevice(c.device));
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    {
      int lo = 0, hi = 0;
      CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
      CK(cudaStreamCreateWithPriority(&st2, cudaStreamNonBlocking, hi));
    }
    CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_diag, cudaEventDisableTiming));
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    solid_h.assign(size_t(n), 0);
    if (solid)
      for (int64_t i = 0; i < n; ++i) solid_h[i] = solid[i] ? 1 : 0;
    if (wu) wall_u_in.assign(wu, wu + 3 * n);
    build_flags(wu);
    // Guard margin: shifted TMA windows of the odd step reach up to
    // nx*ny + nx + 1 cells (+ alignment slack and one tile) beyond a plane.
    // Plane Q is the pair sweep's scratch plane (stores of inactive cells).
    margin = ceil_div(int64_t(nx) * ny + nx + 2 + 2 * TMA_TILE + 128, 64) * 64;
    f_alloc.alloc(size_t(Q + 1) * plane + 2 * size_t(margin));
    CK(cudaMemsetAsync(f_alloc.p, 0, (size_t(Q + 1) * plane + 2 * size_t(margin)) * sizeof(S), st));
    fp = f_alloc.p + margin;
    fslot_h.assign(size_t(n), -1);
    fslot.alloc(size_t(n));
    CK(cudaMemsetAsync(fslot.p, 0xff, size_t(n) * sizeof(int32_t), st));
    grow_slots(64);
    d_diag.alloc(1);
    d_err.alloc(1);
    CK(cudaMemsetAsync(d_err.p, 0, sizeof(int), st));
    d_flag.alloc(1);
    CK(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, c.device));
    ntiles = ceil_div(n, TMA_TILE);
    rows_aligned = (nx % TmaWin<S>::PAD == 0) && ((int64_t(nx) * ny) % TmaWin<S>::PAD == 0);
    // default sweep: the lean kernel where it applies (TRT/BGK, fp32/16-bit
    // storage, no uniform force), else cp.async (4/8-byte storage), the
    // window kernel (16-bit storage) or direct loads (uniform force)
    if (sizeof(S) < 4) kernel_mode = window_ok() ? LBMB_SWEEP_WINDOW : LBMB_SWEEP_DIRECT;
    if (lean_ok(coll)) kernel_mode = LBMB_SWEEP_LEAN;
    red_blocks = int(std::min<int64_t>(ceil_div(n, RED_BLOCK), 1184));
    red_part.alloc(size_t(red_blocks) * 5);
    red_out.alloc(8);
    init_rho_h.assign(size_t(n), 1.0);
    init_u_h.assign(size_t(3 * n), 0.0);
    CK(cudaStreamSynchronize(st));
  }

  ~Engine() override {
    if (step_graph) cudaGraphExecDestroy(step_graph);
    for (auto& e : apply_cache) cudaGraphExecDestroy(e.exec);
    for (auto& e : fused_cache) cudaGraphExecDestroy(e.exec);
    for (auto& g : run_graphs)
      if (g) cudaGraphExecDestroy(g);
    if (st) cudaStreamSynchronize(st);
    bodies.clear();
    scalars.clear();
    if (st2) cudaStreamSynchronize(st2);
    if (h_diag) cudaFreeHost(h_diag);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_diag) cudaEventDestroy(ev_diag);
    if (st2) cudaStreamDestroy(st2);
    if (st) cudaStreamDestroy(st);
  }

  int64_t cells() const override { return n; }
  int q() const override { return Q; }
  const std::vector<uint8_t>& solid() const override { return solid_h; }

  int64_t idx(int x, int y, int z) const { return (int64_t(z) * ny + y) * nx + x; }

  // Cell flags, solid-neighbour masks and wall velocities.
  void build_flags(const double* wu) {
    flags_h.assign(size_t(n), 0);
    std::vector<uint32_t> nb(size_t(n), 0u);
    std::vector<Vec4<A>> w(size_t(n), Vec4<A>{A(0), A(0), A(0), A(0)});
    if (wu)
      for (int64_t i = 0; i < n; ++i) w[i] = Vec4<A>{A(wu[3 * i]), A(wu[3 * i + 1]), A(wu[3 * i + 2]), A(0)};
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const int64_t c = idx(x, y, z);
          if (solid_h[c]) {
            flags_h[c] = F_SOLID;
            continue;
          }
          uint32_t m = 0;
          bool moving = false;
          for (int q = 1; q < Q; ++q) {
            int xx = x + Lat<Q>::cx(q), yy = y + Lat<Q>::cy(q), zz = z + Lat<Q>::cz(q);
            xx = (xx + nx) % nx;
            yy = (yy + ny) % ny;
            zz = (zz + nz) % nz;
            const int64_t s = idx(xx, yy, zz);
            if (solid_h[s]) {
              m |= 1u << q;
              if (w[s].x != A(0) || w[s].y != A(0) || w[s].z != A(0)) moving = true;
            }
          }
          uint8_t fl = 0;
          if (m) fl |= F_BOUNDARY;
          if (moving) fl |= F_MOVING;
          if (cfg.free_slip_top && z == nz - 2) {
            fl |= F_SLIP | F_BOUNDARY;
            m |= NBR_SLIP;
          }
          if ((cfg.periodic[0] && (x == 0 || x == nx - 1)) || (cfg.periodic[1] && (y == 0 || y == ny - 1)) ||
              (cfg.periodic[2] && (z == 0 || z == nz - 1)))
            fl |= F_WRAP;
          flags_h[c] = fl;
          nb[c] = m;
        }
    flags.upload(flags_h, st);
    nbr.upload(nb, st);
    wall_u.upload(w, st);
    CK(cudaStreamSynchronize(st));
    build_tiles();
  }

  void invalidate_graphs() {
    if (step_graph) {
      CK(cudaGraphExecDestroy(step_graph));
      step_graph = nullptr;
    }
    for (auto& e : apply_cache) CK(cudaGraphExecDestroy(e.exec));
    apply_cache.clear();
    drop_fused_graphs();
    drop_run_graphs();
  }

  // Grow the force-slot arrays, keeping content.
  void grow_slots(int64_t need) {
    if (need <= slot_cap) return;
    int64_t cap = std::max<int64_t>(need, slot_cap * 2);
    auto grow = [&](auto& buf, size_t elems_old, size_t elems_new) {
      using E = std::remove_reference_t<decltype(*buf.p)>;
      E* old = buf.p;
      size_t old_n = buf.n;
      buf.p = nullptr;
      buf.n = 0;
      buf.alloc(elems_new);
      CK(cudaMemsetAsync(buf.p, 0, elems_new * sizeof(E), st));
      if (old) {
        CK(cudaMemcpyAsync(buf.p, old, std::min(elems_old, old_n) * sizeof(E), cudaMemcpyDeviceToDevice, st));
        CK(cudaStreamSynchronize(st));
        cudaFree(old);
      }
    };
    grow(slot_cell, size_t(slot_cap), size_t(cap));
    grow(fprev, size_t(slot_cap), size_t(cap));
    grow(fcur, size_t(slot_cap), size_t(cap));
    grow(s_rho, size_t(slot_cap), size_t(cap));
    grow(s_unow, size_t(3 * slot_cap), size_t(3 * cap));
    grow(s_du, size_t(3 * slot_cap), size_t(3 * cap));
    grow(s_spread, size_t(3 * slot_cap), size_t(3 * cap));
    slot_cap = cap;
    invalidate_graphs();
  }

  // Force slots of the given cells, appending a slot (and the F_FORCED
  // flag) for each cell that has none yet; returns the slot of every entry.
  std::vector<int32_t> ensure_slots(const std::vector<int64_t>& cells) {
    std::vector<int32_t> out(cells.size());
    int64_t need = nslots;
    for (int64_t c : cells)
      if (fslot_h[c] < 0) {
        fslot_h[c] = -2;  // mark new
        ++need;
      }
    grow_slots(need);
    std::vector<int64_t> new_cells;
    for (size_t k = 0; k < cells.size(); ++k) {
      const int64_t c = cells[k];
      if (fslot_h[c] == -2) {
        fslot_h[c] = int32_t(nslots + int64_t(new_cells.size()));
        new_cells.push_back(c);
      }
      out[k] = fslot_h[c];
    }
    if (!new_cells.empty()) {
      for (size_t i = 0; i < new_cells.size(); ++i) {
        slot_cell_h.push_back(new_cells[i]);
        flags_h[new_cells[i]] |= F_FORCED;
      }
      CK(cudaMemcpyAsync(slot_cell.p + nslots, new_cells.data(), new_cells.size() * sizeof(int64_t),
                         cudaMemcpyHostToDevice, st));
      nslots += int64_t(new_cells.size());
      if (new_cells.size() > 4096) {
        // many cells: upload the whole slot map and flag array
        CK(cudaMemcpyAsync(fslot.p, fslot_h.data(), size_t(n) * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(flags.p, flags_h.data(), size_t(n), cudaMemcpyHostToDevice, st));
      } else {
        for (size_t i = 0; i < new_cells.size(); ++i) {
          CK(cudaMemcpyAsync(fslot.p + new_cells[i], &fslot_h[new_cells[i]], sizeof(int32_t),
                             cudaMemcpyHostToDevice, st));
          CK(cudaMemcpyAsync(flags.p + new_cells[i], &flags_h[new_cells[i]], 1, cudaMemcpyHostToDevice, st));
        }
      }
      CK(cudaStreamSynchronize(st));
      invalidate_graphs();
    }
    return out;
  }

  HydroParams<A> hydro_params() {
    HydroParams<A> p;
    p.f = fp;
    p.plane = uint32_t(plane);
    p.nxy = nx * ny;
    p.flags = flags.p;
    p.nbr = nbr.p;
    p.wall_u = wall_u.p;
    p.fslot = fslot.p;
    p.fprev = fprev.p;
    p.fcur = fcur.p;
    p.nx = nx;
    p.ny = ny;
    p.nz = nz;
    p.omega_p = A(omega_p);
    p.omega_m = A(omega_m);
    p.cp = A(1.0 - omega_p / 2.0);
    p.cm = A(1.0 - omega_m / 2.0);
    p.omega_shear = A(cfg.omega_shear);
    const double cs = cfg.smagorinsky_cs;
    p.les_c = A(cs > 0.0 ? 18.0 * std::sqrt(2.0) * cs * cs : 0.0);
    p.tau0 = A(cfg.collision == LBMB_CENTRAL_MOMENT ? 1.0 / cfg.omega_shear : 3.0 * cfg.nu + 0.5);
    p.magic = A(cfg.collision == LBMB_TRT ? cfg.magic : 0.0);
    p.gx = A(cfg.force[0]);
    p.gy = A(cfg.force[1]);
    p.gz = A(cfg.force[2]);
    p.uniform_force = (p.gx != A(0) || p.gy != A(0) || p.gz != A(0)) ? 1 : 0;
    return p;
  }

  // TMA-staged sweep (persistent grid sized by the occupancy API).
  template <int COLL, bool ODD, bool RA>
  void launch_tma(const HydroParams<A>& p, cudaStream_t s) {
    auto kern = hydro_tma_kernel<Q, S, COLL, ODD, RA>;
    const size_t smem = tma_smem_bytes<Q, S>();
    const int slot = (ODD ? 1 : 0) + (RA ? 2 : 0) + (COLL == COLL_CM ? 4 : 0);
    if (tma_grid[slot] == 0) {
      CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      int per_sm = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TMA_TILE, smem));
      tma_grid[slot] = int(std::max<int64_t>(1, std::min<int64_t>(ntiles, int64_t(sm_count) * std::max(per_sm, 1))));
    }
    kern<<<unsigned(tma_grid[slot]), TMA_TILE, smem, s>>>(p, n, int(ntiles), d_err.p, omega_ptr(), wait_limit);
    CK(cudaGetLastError());
  }

  // Per-thread cp.async pipeline (persistent grid). `concurrent`: the sweep
  // of a runner step, running while the IBM chain runs on the side stream;
  // its grid leaves async_reserve block slots free for that chain.
  template <int COLL, bool ODD, int MINB, int STAGES>
  void launch_async_mb(const HydroParams<A>& p, cudaStream_t s, bool concurrent) {
    auto kern = hydro_async_kernel<Q, S, COLL, ODD, STAGES, MINB>;
    const size_t smem = async_smem_bytes<Q, S, STAGES>();
    const int slot = (ODD ? 1 : 0) + (COLL == COLL_CM ? 2 : 0) + (concurrent ? 4 : 0);
    if (async_grid[slot] == 0) {
      CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      int per_sm = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ASYNC_TILE, smem));
      const int64_t slots = int64_t(sm_count) * std::max(per_sm, 1) - (concurrent ? async_reserve : 0);
      async_grid[slot] = int(std::max<int64_t>(1, std::min<int64_t>(ntiles, slots)));
    }
    kern<<<unsigned(async_grid[slot]), ASYNC_TILE, smem, s>>>(p, n, int(ntiles));
    CK(cudaGetLastError());
  }
  template <int COLL, bool ODD>
  void launch_async(const HydroParams<A>& p, cudaStream_t s, bool concurrent) {
    if constexpr (std::is_same<A, float>::value) {
      switch (async_minb[ODD]) {
        case 5: launch_async_mb<COLL, ODD, 5, 3>(p, s, concurrent); return;
        case 6: launch_async_mb<COLL, ODD, 6, 2>(p, s, concurrent); return;
        default: break;
      }
    }
    launch_async_mb<COLL, ODD, HydroOccupancy<A>::MIN_BLOCKS, 3>(p, s, concurrent);
  }

  void set_sweep_kernel(int kind) override {
    const bool wide = sizeof(S) >= 4;
    const bool pair = std::is_same<A, float>::value && nx % 2 == 0 && !has_uniform_force();
    if (omega_on && !omega_kind_ok(kind))
      throw Error(LBMB_ERR_UNSUPPORTED, "with a relaxation field the sweep runs on direct, bulk or window kernels");
    if (kind == LBMB_SWEEP_ASYNC && !wide)
      throw Error(LBMB_ERR_UNSUPPORTED, "the cp.async sweep needs 4- or 8-byte population storage");
    if ((kind == LBMB_SWEEP_PAIR || kind == LBMB_SWEEP_TILE) && !pair)
      throw Error(LBMB_ERR_UNSUPPORTED,
                  "the pair sweep needs fp32/fp16/bf16 storage, even nx and no uniform body force");
    if (kind == LBMB_SWEEP_WINDOW && !window_ok())
      throw Error(LBMB_ERR_UNSUPPORTED, "the window sweep needs fp32/fp16/bf16 storage and no uniform body force");
    if (kind == LBMB_SWEEP_LEAN && !lean_ok(coll))
      throw Error(LBMB_ERR_UNSUPPORTED, "the lean sweep needs TRT/BGK, fp32/fp16/bf16 storage and no uniform body force");
    kernel_mode = kind;
    invalidate_graphs();
  }
  int sweep_kernel() const override { return kernel_mode; }
  // Register budget of the fp32 cp.async sweep per parity, as resident
  // blocks per SM (4 = 128 registers with a 3-tile ring, 5 = 96 with 3,
  // 6 = 80 with 2); the persistent grid fills every resident slot.
  int async_minb[2] = {4, 4};
  // Block slots the persistent cp.async grid of a runner step leaves free
  // (out of sm_count x blocks per SM): the latency-bound IBM chain on the
  // side stream runs in them while the sweep is resident, instead of
  // waiting for the whole sweep (128^3 central-moment tank on B200: 227 ->
  // 192 us per runner step with 32).
  const int async_reserve = 32;

  void set_sweep_variant(int even, int odd) override {
    if (kernel_mode == LBMB_SWEEP_ASYNC) {
      auto ok = [](int v) { return v >= 4 && v <= 6; };
      if (!ok(even) || !ok(odd))
        throw Error(LBMB_ERR_INVALID, "sweep variant: cp.async resident blocks per SM must be 4, 5 or 6");
      if (!std::is_same<A, float>::value && (even != 4 || odd != 4))
        throw Error(LBMB_ERR_UNSUPPORTED, "sweep variant: the fp64 cp.async sweep has one register budget (4)");
      async_minb[0] = even;
      async_minb[1] = odd;
      for (int& g : async_grid) g = 0;
      invalidate_graphs();
      return;
    }
    if (kernel_mode == LBMB_SWEEP_PAIR) {
      auto ok = [](int v) { return (v >= 3 && v <= 5) || (v >= PAIR_STAGED + 3 && v <= PAIR_STAGED + 5); };
      if (!ok(even) || !ok(odd))
        throw Error(LBMB_ERR_INVALID,
                    "sweep variant: pair resident blocks per SM must be 3, 4 or 5 (+10: cp.async-staged)");
      pair_minb[0] = even;
      pair_minb[1] = odd;
      prepare_pair_variant();
      invalidate_graphs();
      return;
    }
    if (kernel_mode == LBMB_SWEEP_WINDOW) {
      auto ok = [](int v) { return v >= 2 && v <= 4; };
      if (!ok(even) || !ok(odd))
        throw Error(LBMB_ERR_INVALID, "sweep variant: window resident blocks per SM must be 2, 3 or 4");
      window_minb[0] = even;
      window_minb[1] = odd;
      for (int& g : window_grid) g = 0;
      invalidate_graphs();
      return;
    }
    auto ok = [](int v) { return v >= 6 && v <= 10; };
    if (!ok(even) || !ok(odd)) throw Error(LBMB_ERR_INVALID, "sweep variant: resident blocks per SM must be 6..10");
    lean_minb[0] = even;
    lean_minb[1] = odd;
    invalidate_graphs();
  }
  bool has_uniform_force() const { return cfg.force[0] != 0.0 || cfg.force[1] != 0.0 || cfg.force[2] != 0.0; }

  bool window_ok() const { return std::is_same<A, float>::value && !has_uniform_force(); }

  bool lean_ok(int coll_kind) const {
    return std::is_same<A, float>::value && coll_kind == COLL_TRT && !has_uniform_force();
  }

  // Register budget of the lean sweep per parity (resident blocks per SM:
  // 10 = 48 registers, 9 = 56, 8 = 64, 7 = 72, 6 = 80); set by
  // lbmb_set_sweep_variant.
  int lean_minb[2] = {8, 6};

  template <bool ODD, int MINB>
  void launch_lean_mb(const HydroParams<A>& p, cudaStream_t s) {
    if constexpr (std::is_same<A, float>::value) {
      hydro_lean_kernel<Q, S, ODD, MINB><<<unsigned(ceil_div(n, LEAN_BLOCK)), LEAN_BLOCK, 0, s>>>(p, uint32_t(n));
      CK(cudaGetLastError());
    }
  }

  template <bool ODD>
  void launch_lean(const HydroParams<A>& p, cudaStream_t s) {
    switch (lean_minb[ODD]) {
      case 6: launch_lean_mb<ODD, 6>(p, s); break;
      case 7: launch_lean_mb<ODD, 7>(p, s); break;
      case 9: launch_lean_mb<ODD, 9>(p, s); break;
      case 10: launch_lean_mb<ODD, 10>(p, s); break;
      default: launch_lean_mb<ODD, 8>(p, s); break;
    }
  }

  // Whether the two-cells-per-thread kernel covers this sweep.
  bool pair_ok(const HydroParams<A>& p, int) const {
    return std::is_same<A, float>::value && !p.uniform_force && nx % 2 == 0 && !omega_on &&
           int64_t(Q + 1) * plane < (int64_t(1) << 31);
  }

  // Tile list and window offsets of the tile-pipelined sweep.
  void build_tiles() {
    const int64_t nt = ceil_div(n, TILE_CELLS);
    std::vector<int32_t> list;
    for (int64_t t = 0; t < nt; ++t) {
      bool any = false;
      for (int64_t c = t * TILE_CELLS; c < std::min<int64_t>(n, (t + 1) * TILE_CELLS) && !any; ++c)
        any = !(flags_h[size_t(c)] & F_SOLID);
      if (any) list.push_back(int32_t(t));
    }
    {
      // 64-cell warp tiles of the pair sweep holding a non-solid cell,
      // marked TILE_BND when one of them has a solid neighbour
      const int64_t np = ceil_div(n, PAIR_TILE);
      std::vector<uint32_t> pl_;
      for (int64_t t = 0; t < np; ++t) {
        bool any = false, bnd = false;
        for (int64_t c = t * PAIR_TILE; c < std::min<int64_t>(n, (t + 1) * PAIR_TILE); ++c) {
          const uint8_t fl = flags_h[size_t(c)];
          if (fl & F_SOLID) continue;
          any = true;
          bnd = bnd || (fl & F_BOUNDARY);
        }
        if (any) pl_.push_back(uint32_t(t) | (bnd ? TILE_BND : 0u));
      }
      n_pair_tiles = int(pl_.size());
      pair_list.alloc(pl_.size());
      if (!pl_.empty())
        CK(cudaMemcpyAsync(pair_list.p, pl_.data(), pl_.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    }
    n_tiles_active = int(list.size());
    tile_list.alloc(list.size());
    if (!list.empty())
      CK(cudaMemcpyAsync(tile_list.p, list.data(), list.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    using L = Lat<Q>;
    const int64_t E = 16 / int64_t(sizeof(S));
    for (int q = 0; q < Q; ++q) {
      tile_dirs[0].ws[q] = int32_t(int64_t(q) * plane);
      tile_dirs[0].r[q] = 0;
      const int64_t d = int64_t(L::cx(q)) + int64_t(L::cy(q)) * nx + int64_t(L::cz(q)) * nx * ny;
      const int64_t start = int64_t(opp(q)) * plane - d;  // >= 0: plane >= n > |d|
      tile_dirs[1].r[q] = int32_t(start % E);
      tile_dirs[1].ws[q] = int32_t(start - start % E);
    }
    CK(cudaStreamSynchronize(st));
  }

  // Register budget of the window kernel per parity, as resident blocks of
  // TILE_CELLS threads per SM (2 = 128 registers, 3 = 80, 4 = 64; ring
  // depth from window_stages); 0 = the default for the collision (CM 2,
  // TRT 3).
  int window_minb[2] = {0, 0};

  template <int COLL, bool ODD, int MINB>
  void launch_window_mb(const HydroParams<A>& p, cudaStream_t s, bool concurrent) {
    if constexpr (std::is_same<A, float>::value && (COLL == COLL_TRT || Q == 27)) {
      constexpr int STAGES = window_stages<Q, S, MINB>();
      auto kern = hydro_window_kernel<Q, S, ODD, STAGES, COLL, MINB>;
      const size_t smem = window_smem_bytes<Q, S, STAGES>();
      const int slot = (ODD ? 1 : 0) + (concurrent ? 2 : 0);
      if (window_grid[slot] == 0) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TILE_CELLS, smem));
        // in a runner step, leave the same thread slots free for the IBM
        // chain as the cp.async grid does
        const int64_t reserve = concurrent ? int64_t(async_reserve) * ASYNC_TILE / TILE_CELLS : 0;
        const int64_t slots = int64_t(sm_count) * std::max(per_sm, 1) - reserve;
        window_grid[slot] = int(std::max<int64_t>(1, std::min<int64_t>(n_tiles_active, slots)));
      }
      if (n_tiles_active == 0) return;
      kern<<<unsigned(window_grid[slot]), TILE_CELLS, smem, s>>>(p, tile_list.p, n_tiles_active, tile_dirs[ODD],
                                                                 omega_ptr());
      CK(cudaGetLastError());
    }
  }
  template <int COLL, bool ODD>
  void launch_window(const HydroParams<A>& p, cudaStream_t s, bool concurrent) {
    const int mb = window_minb[ODD] ? window_minb[ODD] : (COLL == COLL_CM ? 2 : 3);
    switch (mb) {
      case 2: launch_window_mb<COLL, ODD, 2>(p, s, concurrent); break;
      case 4: launch_window_mb<COLL, ODD, 4>(p, s, concurrent); break;
      default: launch_window_mb<COLL, ODD, 3>(p, s, concurrent); break;
    }
  }

  template <bool ODD, int COLL>
  void launch_tile(const HydroParams<A>& p, cudaStream_t s) {
    if constexpr (std::is_same<A, float>::value && (COLL == COLL_TRT || Q == 27)) {
      constexpr int STAGES = 3;
      auto kern = hydro_tile_kernel<Q, S, ODD, STAGES, COLL>;
      const size_t smem = tile_smem_bytes<Q, S, STAGES>();
      if (tile_grid[ODD] == 0) {
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TILE_THREADS, smem));
        tile_grid[ODD] = int(std::max<int64_t>(1, std::min<int64_t>(n_tiles_active, int64_t(sm_count) * std::max(per_sm, 1))));
      }
      if (n_tiles_active == 0) return;
      kern<<<unsigned(tile_grid[ODD]), TILE_THREADS, smem, s>>>(p, tile_list.p, n_tiles_active, tile_dirs[ODD]);
      CK(cudaGetLastError());
    }
  }

  // Pair sweep launch variant per parity: resident 128-thread blocks per SM
  // the registers are sized for (3 = 168 registers, 4 = 128, 5 = 96), plus
  // PAIR_STAGED for the cp.async-staged form (its shared memory may allow
  // fewer blocks).
  static constexpr int PAIR_STAGED = 10;
  int pair_minb[2] = {4, 4};
  // Resident blocks per SM of a staged pair kernel (shared memory attribute
  // set on first use; called before any capture by set_sweep_variant and the
  // autotuner's eager trials).
  template <bool ODD, int COLL, int MINB>
  int pair_staged_per_sm() {
    static int per_sm = -1;
    if constexpr (std::is_same<A, float>::value && (COLL == COLL_TRT || Q == 27)) {
      if (per_sm < 0) {
        auto kern = hydro_pair_kernel<Q, S, ODD, MINB, COLL, true>;
        const size_t smem = pair_staged_smem_bytes<Q>();
        CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        int b = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, PAIR_BLOCK, smem));
        per_sm = std::max(b, 1);
      }
    }
    return per_sm;
  }
  template <bool ODD, int COLL, int MINB, bool STAGED>
  void launch_pair_mb(const HydroParams<A>& p, cudaStream_t s, bool concurrent) {
    if constexpr (std::is_same<A, float>::value && (COLL == COLL_TRT || Q == 27)) {
      if (n_pair_tiles == 0) return;
      // persistent warps: every resident block slot, less async_reserve in
      // the sweep of a runner step, where the IBM chain runs beside it
      const int64_t need = ceil_div(n_pair_tiles, PAIR_BLOCK / 32);
      const int resident = STAGED ? std::min(MINB, pair_staged_per_sm<ODD, COLL, MINB>()) : MINB;
      const int64_t slots = int64_t(sm_count) * resident - (concurrent ? async_reserve : 0);
      const unsigned blocks = unsigned(std::max<int64_t>(1, std::min(need, slots)));
      const size_t smem = STAGED ? pair_staged_smem_bytes<Q>() : 0;
      hydro_pair_kernel<Q, S, ODD, MINB, COLL, STAGED><<<blocks, PAIR_BLOCK, smem, s>>>(p, pair_list.p, n_pair_tiles,
                                                                                         uint32_t(n));
      CK(cudaGetLastError());
    }
  }
  template <bool ODD, int COLL>
  void launch_pair(const HydroParams<A>& p, cudaStream_t s, bool concurrent) {
    switch (pair_minb[ODD]) {
      case 3: launch_pair_mb<ODD, COLL, 3, false>(p, s, concurrent); return;
      case 5: launch_pair_mb<ODD, COLL, 5, false>(p, s, concurrent); return;
      case PAIR_STAGED + 3: launch_pair_mb<ODD, COLL, 3, true>(p, s, concurrent); return;
      case PAIR_STAGED + 4: launch_pair_mb<ODD, COLL, 4, true>(p, s, concurrent); return;
      case PAIR_STAGED + 5: launch_pair_mb<ODD, COLL, 5, true>(p, s, concurrent); return;
      default: launch_pair_mb<ODD, COLL, 4, false>(p, s, concurrent); return;
    }
  }
  // Shared-memory setup of the staged pair kernels a variant names.
  void prepare_pair_variant() {
    auto one = [&](auto odd_tag, int v) {
      constexpr bool ODD = decltype(odd_tag)::value;
      auto per_coll = [&](auto coll_tag) {
        constexpr int COLL = decltype(coll_tag)::value;
        if (v == PAIR_STAGED + 3) pair_staged_per_sm<ODD, COLL, 3>();
        if (v == PAIR_STAGED + 4) pair_staged_per_sm<ODD, COLL, 4>();
        if (v == PAIR_STAGED + 5) pair_staged_per_sm<ODD, COLL, 5>();
      };
      if (coll == COLL_CM) per_coll(std::integral_constant<int, COLL_CM>{});
      else per_coll(std::integral_constant<int, COLL_TRT>{});
    };
    one(std::false_type{}, pair_minb[0]);
    one(std::true_type{}, pair_minb[1]);
  }

  template <int COLL, bool ODD>
  void launch_hydro_t(const HydroParams<A>& p, cudaStream_t s, bool main_grid, bool cells) {
    if (main_grid) {
      if (kernel_mode == LBMB_SWEEP_PAIR && pair_ok(p, COLL)) {
        launch_pair<ODD, COLL>(p, s, !cells);
      } else if (kernel_mode == LBMB_SWEEP_WINDOW && window_ok() && !p.uniform_force) {
        launch_window<COLL, ODD>(p, s, !cells);
      } else if (kernel_mode == LBMB_SWEEP_TILE && pair_ok(p, COLL)) {
        launch_tile<ODD, COLL>(p, s);
      } else if (kernel_mode == LBMB_SWEEP_LEAN && lean_ok(COLL) && !p.uniform_force) {
        launch_lean<ODD>(p, s);

      } else if (!p.uniform_force && kernel_mode == 1) {
        if (rows_aligned) launch_tma<COLL, ODD, true>(p, s);
        else launch_tma<COLL, ODD, false>(p, s);
      } else if (!p.uniform_force && kernel_mode == 2) {
        if constexpr (sizeof(S) >= 4) launch_async<COLL, ODD>(p, s, !cells);
      } else {
        const int bx = nx >= 128 ? 128 : int(ceil_div(nx, 32) * 32);
        dim3 block(bx), grid(unsigned(ceil_div(nx, bx)), unsigned(ny), unsigned(nz));
        if (p.uniform_force)
          hydro_aa_kernel<Q, S, COLL, ODD, true><<<grid, block, 0, s>>>(p, omega_ptr());
        else
          hydro_aa_kernel<Q, S, COLL, ODD, false><<<grid, block, 0, s>>>(p, omega_ptr());
        CK(cudaGetLastError());
      }
    }
    if (cells && !p.uniform_force && nslots > 0) {
      hydro_cells_kernel<Q, S, COLL, ODD><<<unsigned(ceil_div(nslots, 128)), 128, 0, s>>>(p, slot_cell.p, nslots,
                                                                                          omega_ptr());
      CK(cudaGetLastError());
    }
  }

  // Bound on every mbarrier wait of the bulk-copy sweeps, in SM cycles
  // (lbmb_set_wait_limit); a negative value runs the timeout self-test.
  long long wait_limit = WAIT_LIMIT_DEFAULT;
  void set_wait_limit(long long cycles) override { wait_limit = cycles == 0 ? WAIT_LIMIT_DEFAULT : cycles; }

  // Raise (and clear) a device-side error reported by a bounded wait.
  void check_device_error() {
    int e = 0;
    CK(cudaMemcpy(&e, d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
      CK(cudaMemset(d_err.p, 0, sizeof(int)));
      throw Error(LBMB_ERR_CUDA, "device wait timed out (bulk copy did not complete)");
    }
  }

  // One hydro step of the given parity: the full-grid sweep and (without a
  // uniform force) the forced-cell sweep.
  void launch_hydro(int par, cudaStream_t s = nullptr, bool main_grid = true, bool cells = true) {
    if (!s) s = st;
    HydroParams<A> p = hydro_params();
    if constexpr (Q == 27) {
      if (coll == COLL_CM) {
        if (par == 0) launch_hydro_t<COLL_CM, false>(p, s, main_grid, cells);
        else launch_hydro_t<COLL_CM, true>(p, s, main_grid, cells);
        return;
      }
    }
    if (par == 0) launch_hydro_t<COLL_TRT, false>(p, s, main_grid, cells);
    else launch_hydro_t<COLL_TRT, true>(p, s, main_grid, cells);
  }

  // One full step on the stream: hydro, the cached-moment field refresh,
  // then the scalars (which read the moments of the new state).
  void enqueue_step() {
    if (nslots > 0 && !has_uniform_force()) {
      // forced cells on the side stream beside the full-grid sweep of the
      // others (disjoint AA slots), as in the runner step
      CK(cudaEventRecord(ev_fork, st));
      CK(cudaStreamWaitEvent(st2, ev_fork, 0));
      launch_hydro(parity, st2, false, true);
      launch_hydro(parity, st, true, false);
      // the cached-moment field refresh follows the forced cells on the side
      // stream (the full-grid sweep reads neither field)
      if (fprev_stale) {
        CK(cudaMemcpyAsync(fprev.p, fcur.p, size_t(nslots) * sizeof(Vec4<A>), cudaMemcpyDeviceToDevice, st2));
        fprev_stale = false;
      }
      CK(cudaEventRecord(ev_join, st2));
      CK(cudaStreamWaitEvent(st, ev_join, 0));
    } else {
      launch_hydro(parity);
    }
    parity ^= 1;
    if (fprev_stale) {
      CK(cudaMemcpyAsync(fprev.p, fcur.p, size_t(nslots) * sizeof(Vec4<A>), cudaMemcpyDeviceToDevice, st));
      fprev_stale = false;
    }
    for (auto& sc : scalars) scalar_step(*sc);
  }

  ScalarParams<A> scalar_params(ScalarStateT<A>& sc) {
    ScalarParams<A> p;
    p.h = sc.h.p;
    p.hplane = sc.hplane;
    p.f = fp;
    p.plane = plane;
    p.flags = flags.p;
    p.nbr = nbr.p;
    p.fslot = fslot.p;
    p.fprev = fprev.p;
    p.nx = nx;
    p.ny = ny;
    p.nz = nz;
    p.hparity = parity;
    p.omega = A(1.0 / ((sc.q == 7 ? Lat<7>::INV_CS2 : Lat<Q>::INV_CS2) * sc.diffusivity + 0.5));
    p.gx = A(cfg.force[0]);
    p.gy = A(cfg.force[1]);
    p.gz = A(cfg.force[2]);
    return p;
  }

  void scalar_step(ScalarStateT<A>& sc) {
    ScalarParams<A> p = scalar_params(sc);
    const int bx = nx >= 128 ? 128 : int(ceil_div(nx, 32) * 32);
    dim3 block(bx), grid(unsigned(ceil_div(nx, bx)), unsigned(ny), unsigned(nz));
    if (sc.q == 7) {
      if (sc.parity == 0) scalar_step_kernel<7, Q, S, false><<<grid, block, 0, st>>>(p);
      else scalar_step_kernel<7, Q, S, true><<<grid, block, 0, st>>>(p);
    } else {
      if (sc.parity == 0) scalar_step_kernel<Q, Q, S, false><<<grid, block, 0, st>>>(p);
      else scalar_step_kernel<Q, Q, S, true><<<grid, block, 0, st>>>(p);
    }
    CK(cudaGetLastError());
    sc.parity ^= 1;
  }

  void step(int64_t steps) override {
    CK(cudaEventRecord(ev0, st));
    int64_t launches = 0;
    int64_t done = 0;
    const int G = 32;
    // Graph replay for long runs: needs parity 0 at the start, no pending
    // force-field refresh and no scalars (whose steps are launched per step).
    while (steps - done >= G && scalars.empty()) {
      if (parity != 0 || fprev_stale) {
        enqueue_step();
        ++done;
        ++launches;
        continue;
      }
      if (!step_graph) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < G; ++i) enqueue_step();
        CK(cudaStreamEndCapture(st, &g));
        CK(cudaGraphInstantiate(&step_graph, g, 0));
        CK(cudaGraphDestroy(g));
        step_graph_len = G;
        parity = 0;  // G is even
      }
      CK(cudaGraphLaunch(step_graph, st));
      done += G;
      launches += G;
    }
    for (; done < steps; ++done) {
      enqueue_step();
      ++launches;
    }
    CK(cudaEventRecord(ev1, st));
    // Asynchronous: the call returns once the work is queued (every other
    // entry point runs on the same stream, and the ones that return data
    // synchronize). The device time is resolved when it is asked for. The
    // bulk-copy kernel is the only one that can raise a device error flag,
    // so its steps are checked at once.
    pending_launches = launches;
    timing_pending = true;
    time += uint64_t(steps);
    if (kernel_mode == LBMB_SWEEP_BULK) {
      CK(cudaEventSynchronize(ev1));
      check_device_error();
    }
  }

  bool timing_pending = false;
  int64_t pending_launches = 0;

  void timing(double* total_ms, double* hydro_ms, int64_t* launches) override {
    if (timing_pending) {
      CK(cudaEventSynchronize(ev1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ev0, ev1));
      last_total_ms = ms;
      last_hydro_ms = ms;
      last_hydro_launches = pending_launches;
      timing_pending = false;
    }
    if (total_ms) *total_ms = last_total_ms;
    if (hydro_ms) *hydro_ms = last_hydro_ms;
    if (launches) *launches = last_hydro_launches;
  }

  void sync() override {
    CK(cudaStreamSynchronize(st));
    check_device_error();
  }

  // Sweep autotuner: times every kernel kind (and, for the lean kernel,
  // every register budget) that can run this configuration on the solver's
  // own grid, keeps the fastest, and leaves the state untouched (the
  // populations and parity are saved before the trials and restored after).
  void autotune_sweep(int steps, lbmb_autotune_result* out, int32_t* trial_desc, double* trial_ms,
                      int capacity) override {
    if (steps < 2) throw Error(LBMB_ERR_INVALID, "autotune: steps per trial must be >= 2");
    steps += steps & 1;  // whole even/odd pairs
    struct Cand {
      int kind, ev, od;
    };
    std::vector<Cand> cands;
    const bool wide = sizeof(S) >= 4;
    const bool is_f = std::is_same<A, float>::value;
    const bool uf = has_uniform_force();
    cands.push_back({LBMB_SWEEP_DIRECT, 0, 0});
    if (wide && !uf) {
      if (is_f) {
        for (int ev = 4; ev <= 6; ++ev)
          for (int od = 4; od <= 6; ++od) cands.push_back({LBMB_SWEEP_ASYNC, ev, od});
      } else {
        cands.push_back({LBMB_SWEEP_ASYNC, 4, 4});
      }
    }
    if (!uf) cands.push_back({LBMB_SWEEP_BULK, 0, 0});
    if (is_f && nx % 2 == 0 && !uf && !omega_on) {
      for (int ev : {3, 4, 5, PAIR_STAGED + 3, PAIR_STAGED + 4, PAIR_STAGED + 5})
        for (int od : {3, 4, 5, PAIR_STAGED + 3, PAIR_STAGED + 4, PAIR_STAGED + 5})
          cands.push_back({LBMB_SWEEP_PAIR, ev, od});
      cands.push_back({LBMB_SWEEP_TILE, 0, 0});
    }
    if (window_ok()) {
      const int hi = coll == COLL_CM ? 3 : 4;
      for (int ev = 2; ev <= hi; ++ev)
        for (int od = 2; od <= hi; ++od) cands.push_back({LBMB_SWEEP_WINDOW, ev, od});
    }
    if (lean_ok(coll))
      for (int ev = 10; ev >= 6; --ev)
        for (int od = 9; od >= 6; --od) cands.push_back({LBMB_SWEEP_LEAN, ev, od});
    if (omega_on) {
      std::vector<Cand> keep;
      for (const Cand& cd : cands)
        if (omega_kind_ok(cd.kind)) keep.push_back(cd);
      cands.swap(keep);
    }
    const int kind0 = kernel_mode, ev0_ = lean_minb[0], od0 = lean_minb[1];
    const int ae0 = async_minb[0], ao0 = async_minb[1];
    const int we0 = window_minb[0], wo0 = window_minb[1];
    const int pe0 = pair_minb[0], po0 = pair_minb[1];
    const int par0 = parity;
    const size_t fbytes = f_alloc.n * sizeof(S);
    DevBuf<S> save;
    save.alloc(f_alloc.n);
    CK(cudaMemcpyAsync(save.p, f_alloc.p, fbytes, cudaMemcpyDeviceToDevice, st));
    invalidate_graphs();
    auto trial = [&](const Cand& cd) {
      kernel_mode = cd.kind;
      if (cd.kind == LBMB_SWEEP_LEAN) {
        lean_minb[0] = cd.ev;
        lean_minb[1] = cd.od;
      }
      if (cd.kind == LBMB_SWEEP_ASYNC) {
        async_minb[0] = cd.ev;
        async_minb[1] = cd.od;
        for (int& g : async_grid) g = 0;
      }
      if (cd.kind == LBMB_SWEEP_WINDOW) {
        window_minb[0] = cd.ev;
        window_minb[1] = cd.od;
        for (int& g : window_grid) g = 0;
      }
      if (cd.kind == LBMB_SWEEP_PAIR) {
        pair_minb[0] = cd.ev;
        pair_minb[1] = cd.od;
        prepare_pair_variant();
      }
      // each trial step runs as a plain step does: with force slots, the
      // forced cells on the side stream beside the full-grid sweep
      auto trial_step = [&](int par) {
        if (nslots > 0 && !has_uniform_force()) {
          CK(cudaEventRecord(ev_fork, st));
          CK(cudaStreamWaitEvent(st2, ev_fork, 0));
          launch_hydro(par, st2, false, true);
          launch_hydro(par, st, true, false);
          CK(cudaEventRecord(ev_join, st2));
          CK(cudaStreamWaitEvent(st, ev_join, 0));
        } else {
          launch_hydro(par);
        }
      };
      for (int i = 0; i < 2; ++i) trial_step(i);  // warm-up (first launches set up grids)
      CK(cudaEventRecord(ev0, st));
      for (int i = 0; i < steps; ++i) trial_step(i & 1);
      CK(cudaEventRecord(ev1, st));
      CK(cudaEventSynchronize(ev1));
      check_device_error();
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ev0, ev1));
      return double(ms) / steps;
    };
    const double t_default = trial(kind0 == LBMB_SWEEP_ASYNC    ? Cand{kind0, ae0, ao0}
                                   : kind0 == LBMB_SWEEP_WINDOW ? Cand{kind0, we0, wo0}
                                   : kind0 == LBMB_SWEEP_PAIR   ? Cand{kind0, pe0, po0}
                                                                : Cand{kind0, ev0_, od0});
    int best = -1;
    double best_ms = 0.0;
    for (size_t i = 0; i < cands.size(); ++i) {
      const double t = trial(cands[i]);
      if (int(i) < capacity) {
        if (trial_desc) {
          trial_desc[3 * i + 0] = cands[i].kind;
          trial_desc[3 * i + 1] = cands[i].ev;
          trial_desc[3 * i + 2] = cands[i].od;
        }
        if (trial_ms) trial_ms[i] = t;
      }
      if (best < 0 || t < best_ms) {
        best = int(i);
        best_ms = t;
      }
    }
    kernel_mode = cands[best].kind;
    if (kernel_mode == LBMB_SWEEP_LEAN) {
      lean_minb[0] = cands[best].ev;
      lean_minb[1] = cands[best].od;
    } else {
      lean_minb[0] = ev0_;
      lean_minb[1] = od0;
    }
    if (kernel_mode == LBMB_SWEEP_ASYNC) {
      async_minb[0] = cands[best].ev;
      async_minb[1] = cands[best].od;
    } else {
      async_minb[0] = ae0;
      async_minb[1] = ao0;
    }
    if (kernel_mode == LBMB_SWEEP_WINDOW) {
      window_minb[0] = cands[best].ev;
      window_minb[1] = cands[best].od;
    } else {
      window_minb[0] = we0;
      window_minb[1] = wo0;
    }
    if (kernel_mode == LBMB_SWEEP_PAIR) {
      pair_minb[0] = cands[best].ev;
      pair_minb[1] = cands[best].od;
    } else {
      pair_minb[0] = pe0;
      pair_minb[1] = po0;
    }
    for (int& g : async_grid) g = 0;
    for (int& g : window_grid) g = 0;
    CK(cudaMemcpyAsync(f_alloc.p, save.p, fbytes, cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    parity = par0;
    invalidate_graphs();
    if (out) {
      out->kind = kernel_mode;
      const int* mb = kernel_mode == LBMB_SWEEP_ASYNC    ? async_minb
                      : kernel_mode == LBMB_SWEEP_WINDOW ? window_minb
                      : kernel_mode == LBMB_SWEEP_PAIR   ? pair_minb
                                                         : lean_minb;
      out->even_blocks_per_sm = mb[0];
      out->odd_blocks_per_sm = mb[1];
      out->n_trials = int32_t(cands.size());
      out->best_ms_per_step = best_ms;
      out->default_ms_per_step = t_default;
    }
  }

  void stage_in(const double* fin) override {
    DevBuf<double> tmp;
    tmp.upload(fin, size_t(Q) * n, st);
    stage_in_kernel<Q, S><<<unsigned(ceil_div(n, 256)), 256, 0, st>>>(fp, plane, tmp.p, n);
    CK(cudaGetLastError());
    parity = 0;
    // Moments refresh: the cached moments now include the current field.
    if (nslots)
      CK(cudaMemcpyAsync(fprev.p, fcur.p, size_t(nslots) * sizeof(Vec4<A>), cudaMemcpyDeviceToDevice, st));
    fprev_stale = false;
    CK(cudaStreamSynchronize(st));
    invalidate_graphs();
  }

  void stage_out(double* fout) override {
    DevBuf<double> tmp;
    tmp.alloc(size_t(Q) * n);
    stage_out_kernel<Q, S><<<unsigned(ceil_div(n, 128)), 128, 0, st>>>(fp, plane, flags.p, nbr.p, nx, ny, nz,
                                                                       parity, tmp.p, n);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(fout, tmp.p, size_t(Q) * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }

  // Solver::init_with (solver.rs:2474-2605) on the host, in the arithmetic
  // precision, then staged in.
  void init_fields(const double* r_in, const double* u_in) override {
    using L = Lat<Q>;
    std::vector<double> fh(size_t(Q) * n);
    const A three = A(3), half = A(0.5), f45 = A(4.5), f15 = A(1.5);
    const A tau = A(3.0 * cfg.nu + 0.5);
    const bool per[3] = {cfg.periodic[0] != 0, cfg.periodic[1] != 0, cfg.periodic[2] != 0};
    const int dims[3] = {nx, ny, nz};
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const int64_t c = idx(x, y, z);
          const A r = A(r_in[c]);
          const A u[3] = {A(u_in[3 * c]), A(u_in[3 * c + 1]), A(u_in[3 * c + 2])};
          const A usq = (u[0] * u[0] + u[1] * u[1]) + u[2] * u[2];
          const A drho = r - A(1);
          A fq[Q];
          for (int q = 0; q < Q; ++q) {
            const A cu = (A(L::cx(q)) * u[0] + A(L::cy(q)) * u[1]) + A(L::cz(q)) * u[2];
            fq[q] = A(L::w(q)) * (drho + r * (three * cu + f45 * cu * cu - f15 * usq));
          }
          if (!solid_h[c]) {
            auto sample = [&](int a, int dl, A out[3]) -> bool {
              int g[3] = {x, y, z};
              g[a] += dl;
              if (g[a] < 0 || g[a] >= dims[a]) {
                if (per[a]) g[a] = (g[a] + dims[a]) % dims[a];
                else return false;
              }
              const int64_t gi = idx(g[0], g[1], g[2]);
              if (solid_h[gi]) return false;
              for (int k = 0; k < 3; ++k) out[k] = A(u_in[3 * gi + k]);
              return true;
            };
            A grad[3][3] = {};
            for (int a = 0; a < 3; ++a) {
              A pv[3] = {A(0), A(0), A(0)}, mv[3] = {A(0), A(0), A(0)};
              const bool hp = sample(a, 1, pv), hm = sample(a, -1, mv);
              for (int b = 0; b < 3; ++b) {
                if (hp && hm) grad[a][b] = (pv[b] - mv[b]) * half;
                else if (hp) grad[a][b] = pv[b] - u[b];
                else if (hm) grad[a][b] = u[b] - mv[b];
                else grad[a][b] = A(0);
              }
            }
            const A div = (grad[0][0] + grad[1][1]) + grad[2][2];
            for (int q = 0; q < Q; ++q) {
              const A cq[3] = {A(L::cx(q)), A(L::cy(q)), A(L::cz(q))};
              A ccgu = cq[0] * cq[0] * grad[0][0];
              for (int a = 0; a < 3; ++a)
                for (int b = a; b < 3; ++b) {
                  if (a == 0 && b == 0) continue;
                  if (a == b) ccgu = ccgu + cq[a] * cq[a] * grad[a][a];
                  else ccgu = ccgu + cq[a] * cq[b] * (grad[a][b] + grad[b][a]);
                }
              const A fneq = -A(L::w(q)) * r * tau * (three * ccgu - div);
              fq[q] = fq[q] + fneq;
            }
          }
          for (int q = 0; q < Q; ++q) fh[size_t(q) * n + c] = double(fq[q]);
          init_rho_h[c] = double(r);
          for (int k = 0; k < 3; ++k) init_u_h[3 * c + k] = double(u[k]);
          d_init_u_ok = false;
        }
    stage_in(fh.data());
  }

  void read_moments(double* rho, double* ux, double* uy, double* uz) override {
    DevBuf<double> d;
    d.alloc(size_t(4) * n);
    moments_kernel<Q, S><<<unsigned(ceil_div(n, 128)), 128, 0, st>>>(
        fp, plane, flags.p, nbr.p, nx, ny, nz, parity, fslot.p, fprev.p, A(cfg.force[0]), A(cfg.force[1]),
        A(cfg.force[2]), d.p, d.p + n, d.p + 2 * n, d.p + 3 * n, n);
    CK(cudaGetLastError());
    std::vector<double> h(size_t(4) * n);
    CK(cudaMemcpyAsync(h.data(), d.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int64_t c = 0; c < n; ++c) {
      const bool s = solid_h[c] != 0;
      if (rho) rho[c] = s ? init_rho_h[c] : h[c];
      if (ux) ux[c] = s ? init_u_h[3 * c] : h[n + c];
      if (uy) uy[c] = s ? init_u_h[3 * c + 1] : h[2 * n + c];
      if (uz) uz[c] = s ? init_u_h[3 * c + 2] : h[3 * n + c];
    }
  }

  void reduce_all(double out[5]) override {
    reduce_kernel<Q, S><<<red_blocks, RED_BLOCK, 0, st>>>(fp, plane, flags.p, nbr.p, nx, ny, nz, parity,
                                                         fslot.p, fcur.p, double(A(cfg.force[0])),
                                                         double(A(cfg.force[1])), double(A(cfg.force[2])),
                                                         n, red_part.p);
    CK(cudaGetLastError());
    reduce_finish_kernel<<<1, 32, 0, st>>>(red_part.p, red_blocks, 5, red_out.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, red_out.p, 5 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }

  // The device part of clear_force_field with no refresh pending: zero the
  // current field, and the cached-moments field too when the cleared field
  // was uniform.
  void enqueue_clear_device(cudaStream_t s_ = nullptr) {
    if (!nslots) return;
    cudaStream_t s = s_ ? s_ : st;
    const unsigned g = unsigned(std::min<int64_t>(ceil_div(nslots, 256), int64_t(4) * sm_count));
    CK(cudaMemsetAsync(d_flag.p, 0, sizeof(int), s));
    field_uniform_kernel<A><<<g, 256, 0, s>>>(fcur.p, nslots, nslots == n ? 1 : 0, d_flag.p);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(fcur.p, 0, size_t(nslots) * sizeof(Vec4<A>), s));
    field_zero_if_uniform_kernel<A><<<g, 256, 0, s>>>(fprev.p, nslots, d_flag.p);
    CK(cudaGetLastError());
  }

  // Solver::clear_body_force_field (solver.rs:2805-2822): a uniform field
  // (all cells equal) refreshes the cached moments without it; otherwise
  // the cached moments keep the old field until the next step.
  void clear_force_field() override {
    if (!field_present) return;
    if (!fprev_stale) {
      // No refresh pending, so the host state ends the same whether the
      // field was uniform or not: the check and the conditional reset of
      // the cached-moments field run on the device, without a host sync.
      field_present = false;
      enqueue_clear_device();
      return;
    }
    bool uniform = true;
    if (nslots > 0) {
      std::vector<Vec4<A>> h(static_cast<size_t>(nslots));
      CK(cudaMemcpyAsync(h.data(), fcur.p, h.size() * sizeof(Vec4<A>), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      const Vec4<A> base = (nslots == n) ? h[0] : Vec4<A>{A(0), A(0), A(0), A(0)};
      for (auto& v : h)
        if (!(v.x == base.x && v.y == base.y && v.z == base.z)) uniform = false;
    }
    field_present = false;
    if (nslots) CK(cudaMemsetAsync(fcur.p, 0, size_t(nslots) * sizeof(Vec4<A>), st));
    if (uniform) {
      if (nslots) CK(cudaMemsetAsync(fprev.p, 0, size_t(nslots) * sizeof(Vec4<A>), st));
      fprev_stale = false;
    }
    CK(cudaStreamSynchronize(st));
  }

  // ---- shear-rate and stress QOIs (stress.cuh) ---------------------------
  StrainArgs<S> strain_args() {
    StrainArgs<S> a;
    a.fb = fp;
    a.pl = plane;
    a.flags = flags.p;
    a.nbr = nbr.p;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.parity = parity;
    a.fslot = fslot.p;
    a.fprev = fprev.p;
    a.fcur = fcur.p;
    a.field_present = field_present ? 1 : 0;
    a.gx = A(cfg.force[0]);
    a.gy = A(cfg.force[1]);
    a.gz = A(cfg.force[2]);
    a.tau_eff = A(1.0 / omega_p);
    return a;
  }

  void strain_rate(double* s6, double* gamma) override {
    DevBuf<double> d6, dg;
    if (s6) d6.alloc(size_t(6) * n);
    if (gamma) dg.alloc(size_t(n));
    strain_rate_kernel<Q, S><<<unsigned(ceil_div(n, 128)), 128, 0, st>>>(strain_args(), s6 ? d6.p : nullptr,
                                                                        gamma ? dg.p : nullptr, n);
    CK(cudaGetLastError());
    if (s6) CK(cudaMemcpyAsync(s6, d6.p, size_t(6) * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (gamma) CK(cudaMemcpyAsync(gamma, dg.p, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }

  // ---- per-cell relaxation field and WALE (les.rs) -------------------------
  DevBuf<A> omega_dev;
  bool omega_on = false;
  const A* omega_ptr() const { return omega_on ? omega_dev.p : nullptr; }

  // Kinds that take the field: direct loads, bulk copies and the window
  // kernel (the tuned cp.async, lean, pair and tile kernels keep their
  // uniform-rate code; a per-cell rate cost the cp.async central-moment
  // kernel 14% on B200 even when unused).
  bool omega_kind_ok(int kind) const {
    return kind == LBMB_SWEEP_DIRECT || kind == LBMB_SWEEP_BULK || kind == LBMB_SWEEP_WINDOW;
  }
  void omega_install() {
    if (cfg.smagorinsky_cs > 0.0)
      throw Error(LBMB_ERR_UNSUPPORTED, "a relaxation field and the Smagorinsky option cannot be combined");
    omega_on = true;
    if (!omega_kind_ok(kernel_mode)) kernel_mode = window_ok() ? LBMB_SWEEP_WINDOW : LBMB_SWEEP_DIRECT;
    invalidate_graphs();
  }

  void set_omega_field(const double* omega) override {
    if (!omega) {
      omega_on = false;
      invalidate_graphs();
      return;
    }
    for (int64_t c = 0; c < n; ++c)
      if (!std::isfinite(omega[c])) invalid("omega field values must be finite");
    std::vector<A> h(static_cast<size_t>(n));
    for (int64_t c = 0; c < n; ++c) h[size_t(c)] = A(omega[c]);
    if (omega_dev.n != size_t(n)) omega_dev.alloc(size_t(n));
    CK(cudaMemcpyAsync(omega_dev.p, h.data(), h.size() * sizeof(A), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    omega_install();
  }

  void velocity_gradient(double* g9) override {
    DevBuf<double> u3, dg;
    velocity_moments(u3);
    dg.alloc(size_t(9) * n);
    wale_kernel<Q, S><<<unsigned(ceil_div(n, 128)), 128, 0, st>>>(
        strain_args(), u3.p, wall_u.p, cfg.periodic[0], cfg.periodic[1], cfg.periodic[2], A(cfg.nu), 0, A(0), dg.p,
        nullptr, nullptr, nullptr, nullptr, n);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(g9, dg.p, size_t(9) * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }

  // WaleLes::update (les.rs:120-211): nu_t and the omega+ field, installed
  // for the next collision without leaving the device.
  void wale_update(double tau_eff_max, double* nu_t, lbmb_wale_diag* diag) override {
    if (cfg.smagorinsky_cs > 0.0)
      throw Error(LBMB_ERR_UNSUPPORTED, "WALE and the Smagorinsky option cannot be combined");
    const bool clip = !std::isnan(tau_eff_max);
    const A nu0 = A(cfg.nu);
    const A tau0 = A(0.5) + A(3.0) * nu0;
    A nu_t_max = A(0);
    if (clip) {
      if (!(std::isfinite(tau_eff_max) && tau_eff_max > 0.5)) invalid("tau_eff_max must be finite and greater than 0.5");
      if (A(tau_eff_max) < tau0) invalid("tau_eff_max must be at least the laminar tau for this solver");
      nu_t_max = (A(tau_eff_max) - tau0) / A(3.0);
    }
    DevBuf<double> u3, dnu;
    DevBuf<unsigned long long> cnt;
    cnt.alloc(2);
    CK(cudaMemsetAsync(cnt.p, 0, 2 * sizeof(unsigned long long), st));
    velocity_moments(u3);
    if (nu_t) dnu.alloc(size_t(n));
    if (omega_dev.n != size_t(n)) omega_dev.alloc(size_t(n));
    wale_kernel<Q, S><<<unsigned(ceil_div(n, 128)), 128, 0, st>>>(
        strain_args(), u3.p, wall_u.p, cfg.periodic[0], cfg.periodic[1], cfg.periodic[2], nu0, clip ? 1 : 0,
        nu_t_max, nullptr, nu_t ? dnu.p : nullptr, omega_dev.p, cnt.p, cnt.p + 1, n);
    CK(cudaGetLastError());
    unsigned long long hc[2] = {0, 0};
    CK(cudaMemcpyAsync(hc, cnt.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
    if (nu_t) CK(cudaMemcpyAsync(nu_t, dnu.p, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    omega_install();
    if (diag) {
      double mx = 0.0;
      std::memcpy(&mx, &hc[1], sizeof(double));
      diag->clipped_cells = int64_t(hc[0]);
      diag->clipped_fraction = n == 0 ? 0.0 : double(A(double(hc[0])) / A(double(n)));
      diag->max_nu_t_before_clipping = mx;
      diag->tau_eff_max = clip ? tau_eff_max : std::nan("");
      diag->nu_t_max = clip ? double(nu_t_max) : std::nan("");
    }
  }

  // cached velocity moments (lattice units) into u3 = [ux | uy | uz]
  void velocity_moments(DevBuf<double>& u3) {
    u3.alloc(size_t(3) * n);
    moments_kernel<Q, S><<<unsigned(ceil_div(n, 128)), 128, 0, st>>>(
        fp, plane, flags.p, nbr.p, nx, ny, nz, parity, fslot.p, fprev.p, A(cfg.force[0]), A(cfg.force[1]),
        A(cfg.force[2]), nullptr, u3.p, u3.p + n, u3.p + 2 * n, n);
    CK(cudaGetLastError());
  }
  static void check_si(double dx, double dt, double mu) {
    if (!(std::isfinite(dx) && dx > 0.0)) invalid("stress: dx_m must be finite and positive");
    if (!(std::isfinite(dt) && dt > 0.0)) invalid("stress: dt_s must be finite and positive");
    if (!(std::isfinite(mu) && mu > 0.0)) invalid("stress: mu_pa_s must be finite and positive");
  }

  void stress_field(double dx, double dt, double mu, double* s6, double* gamma, double* viscous) override {
    check_si(dx, dt, mu);
    DevBuf<double> u3, d6, dg, dv;
    velocity_moments(u3);
    if (s6) d6.alloc(size_t(6) * n);
    if (gamma) dg.alloc(size_t(n));
    if (viscous) dv.alloc(size_t(n));
    stress_field_kernel<<<unsigned(ceil_div(n, 128)), 128, 0, st>>>(
        u3.p, u3.p + n, u3.p + 2 * n, flags.p, nx, ny, nz, dx, dx / dt, mu, s6 ? d6.p : nullptr,
        gamma ? dg.p : nullptr, viscous ? dv.p : nullptr, nullptr, nullptr, n);
    CK(cudaGetLastError());
    if (s6) CK(cudaMemcpyAsync(s6, d6.p, size_t(6) * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (gamma) CK(cudaMemcpyAsync(gamma, dg.p, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (viscous) CK(cudaMemcpyAsync(viscous, dv.p, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }

  // runner.rs:1648-1690: percentile summaries of gamma_dot and mu gamma_dot
  // over the fluid cells (thresholds: NaN for none).
  void stress_summary(double dx, double dt, double mu, double t_gamma, double t_tau, lbmb_percentiles* pg,
                      lbmb_percentiles* pt, double* device_ms) override {
    check_si(dx, dt, mu);
    DevBuf<double> u3, key, sorted;
    DevBuf<unsigned long long> cnt;
    cnt.alloc(3);
    key.alloc(size_t(n));
    sorted.alloc(size_t(n));
    size_t tmp_bytes = 0;
    CK(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, key.p, sorted.p, int(n), 0, 64, st));
    DevBuf<unsigned char> tmp;
    tmp.alloc(std::max<size_t>(tmp_bytes, 1));
    CK(cudaMemsetAsync(cnt.p, 0, 3 * sizeof(unsigned long long), st));
    CK(cudaEventRecord(ev0, st));
    velocity_moments(u3);
    stress_field_kernel<<<unsigned(ceil_div(n, 128)), 128, 0, st>>>(u3.p, u3.p + n, u3.p + 2 * n, flags.p, nx, ny,
                                                                    nz, dx, dx / dt, mu, nullptr, nullptr, nullptr,
                                                                    key.p, cnt.p, n);
    CK(cudaGetLastError());
    CK(cub::DeviceRadixSort::SortKeys(tmp.p, tmp_bytes, key.p, sorted.p, int(n), 0, 64, st));
    unsigned long long k = 0;
    CK(cudaMemcpyAsync(&k, cnt.p, sizeof(k), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const bool hg = std::isfinite(t_gamma), ht = std::isfinite(t_tau);
    if (k > 0) {
      const unsigned g = unsigned(ceil_div(int64_t(k), 128));
      if (hg) count_above_kernel<<<g, 128, 0, st>>>(sorted.p, int64_t(k), 1.0, t_gamma, cnt.p + 1);
      if (ht) count_above_kernel<<<g, 128, 0, st>>>(sorted.p, int64_t(k), mu, t_tau, cnt.p + 2);
      CK(cudaGetLastError());
    }
    CK(cudaEventRecord(ev1, st));
    unsigned long long above[2] = {0, 0};
    CK(cudaMemcpyAsync(above, cnt.p + 1, sizeof(above), cudaMemcpyDeviceToHost, st));
    CK(cudaEventSynchronize(ev1));
    CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    if (device_ms) *device_ms = ms;
    // percentile_sorted (stress.rs:296-309) on ranks read back one by one
    auto at = [&](int64_t i) {
      double v = 0.0;
      CK(cudaMemcpy(&v, sorted.p + i, sizeof(double), cudaMemcpyDeviceToHost));
      return v;
    };
    auto fill = [&](lbmb_percentiles* o, double scale, bool has_t, unsigned long long nab) {
      if (!o) return;
      *o = lbmb_percentiles{};
      o->count = int64_t(k);
      o->valid = k > 0 ? 1 : 0;
      o->fraction_above_threshold = std::nan("");
      if (k == 0) return;
      auto pct = [&](double p) {
        if (k == 1) return scale * at(0);
        const double rank = p * double(k - 1);
        const int64_t lo = int64_t(std::floor(rank)), hi = int64_t(std::ceil(rank));
        if (lo == hi) return scale * at(lo);
        const double t = rank - double(lo);
        return (scale * at(lo)) * (1.0 - t) + (scale * at(hi)) * t;
      };
      o->p50 = pct(0.50);
      o->p90 = pct(0.90);
      o->p95 = pct(0.95);
      o->p99 = pct(0.99);
      o->max = scale * at(int64_t(k) - 1);
      if (has_t) o->fraction_above_threshold = double(nab) / double(k);
    };
    fill(pg, 1.0, hg, above[0]);
    fill(pt, mu, ht, above[1]);
  }

  void wall_shear(double dx, double dt, double rho, double mu, lbmb_wall_shear* out, int64_t capacity,
                  int64_t* count) override {
    check_si(dx, dt, mu);
    if (!(std::isfinite(rho) && rho > 0.0)) invalid("wall shear: rho_kg_m3 must be finite and positive");
    DevBuf<double> u3, tau, yp, up, nrm, vals;
    DevBuf<uint8_t> flag;
    DevBuf<int64_t> idx, sel;
    DevBuf<int> nsel;
    velocity_moments(u3);
    tau.alloc(size_t(n));
    yp.alloc(size_t(n));
    up.alloc(size_t(n));
    nrm.alloc(size_t(3) * n);
    flag.alloc(size_t(n));
    idx.alloc(size_t(n));
    sel.alloc(size_t(n));
    nsel.alloc(1);
    const unsigned g = unsigned(ceil_div(n, 128));
    wall_shear_kernel<A><<<g, 128, 0, st>>>(u3.p, u3.p + n, u3.p + 2 * n, flags.p, wall_u.p, nx, ny, nz, dx, dx / dt,
                                            rho, mu, flag.p, tau.p, yp.p, up.p, nrm.p, n);
    iota_kernel<<<g, 128, 0, st>>>(idx.p, n);
    CK(cudaGetLastError());
    size_t tmp_bytes = 0;
    CK(cub::DeviceSelect::Flagged(nullptr, tmp_bytes, idx.p, flag.p, sel.p, nsel.p, int(n), st));
    DevBuf<unsigned char> tmp;
    tmp.alloc(std::max<size_t>(tmp_bytes, 1));
    CK(cub::DeviceSelect::Flagged(tmp.p, tmp_bytes, idx.p, flag.p, sel.p, nsel.p, int(n), st));
    int m = 0;
    CK(cudaMemcpyAsync(&m, nsel.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (count) *count = m;
    const int64_t k = std::min<int64_t>(m, std::max<int64_t>(capacity, 0));
    if (!out || k == 0) return;
    vals.alloc(size_t(7) * k);
    gather_wall_kernel<<<unsigned(ceil_div(k, 128)), 128, 0, st>>>(sel.p, k, tau.p, yp.p, up.p, nrm.p, vals.p);
    CK(cudaGetLastError());
    std::vector<int64_t> hi(static_cast<size_t>(k));
    std::vector<double> hv(static_cast<size_t>(7 * k));
    CK(cudaMemcpyAsync(hi.data(), sel.p, size_t(k) * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hv.data(), vals.p, size_t(7) * k * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int64_t i = 0; i < k; ++i) {
      lbmb_wall_shear& w = out[i];
      w.cell_index = hi[size_t(i)];
      w.tau_w_pa = hv[size_t(7 * i)];
      w.y_plus = hv[size_t(7 * i + 1)];
      w.u_parallel_m_s = hv[size_t(7 * i + 2)];
      w.y_m = 0.5 * dx;
      for (int a = 0; a < 3; ++a) w.normal[a] = hv[size_t(7 * i + 3 + a)];
    }
  }

  void get_force_field(double* out) override {
    std::fill(out, out + 3 * n, 0.0);
    if (!field_present || nslots == 0) return;
    std::vector<Vec4<A>> h(static_cast<size_t>(nslots));
    CK(cudaMemcpyAsync(h.data(), fcur.p, h.size() * sizeof(Vec4<A>), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int64_t s = 0; s < nslots; ++s) {
      const int64_t c = slot_cell_h[s];
      out[3 * c] = double(h[s].x);
      out[3 * c + 1] = double(h[s].y);
      out[3 * c + 2] = double(h[s].z);
    }
  }

  // ---- IBM -------------------------------------------------------------
  void ibm_set_body(int b, const double* pos, const double* w, int64_t nm, const double* c,
                    const double* om) override {
    set_body(b, pos, w, nm, c, om, st);
  }
  // up: the stream of the marker upload when the marker set is unchanged.
  void set_body(int b, const double* pos, const double* w, int64_t nm, const double* c, const double* om,
                cudaStream_t up) {
    if (b < 0 || b > 64) invalid("IBM body slot out of range");
    if (nm <= 0) invalid("IBM body must contain at least one marker");
    for (int a = 0; a < 3; ++a)
      if (!std::isfinite(c[a]) || !std::isfinite(om[a])) invalid("IBM center and omega must be finite");
    if (int(bodies.size()) <= b) bodies.resize(size_t(b) + 1);
    // The runner passes the same marker set every step: when the markers are
    // unchanged (and so already checked) the stencils and device arrays
    // stay; only the rotation (centre, angular velocity and the slip scale)
    // is refreshed.
    BodyState* old = bodies[size_t(b)].get();
    const bool unchanged = old && old->nm == nm &&
                           std::memcmp(old->pos.data(), pos, size_t(3 * nm) * sizeof(double)) == 0 &&
                           std::memcmp(old->weight.data(), w, size_t(nm) * sizeof(double)) == 0;
    if (!unchanged)
      for (int64_t m = 0; m < nm; ++m) {
        for (int a = 0; a < 3; ++a)
          if (!std::isfinite(pos[3 * m + a]))
            invalid("IBM marker must have finite position and positive finite weight");
        if (!(std::isfinite(w[m]) && w[m] > 0.0))
          invalid("IBM marker must have finite position and positive finite weight");
      }
    if (old) {
      if (unchanged) {
        // the marker arrays are still copied, so the device always holds
        // what the caller passed (an asynchronous copy of the same bytes)
        CK(cudaMemcpyAsync(old->d_pos.p, pos, size_t(3 * nm) * sizeof(double), cudaMemcpyHostToDevice, up));
        CK(cudaMemcpyAsync(old->d_weight.p, w, size_t(nm) * sizeof(double), cudaMemcpyHostToDevice, up));
        bool same = true;
        for (int a = 0; a < 3; ++a) same = same && old->center[a] == c[a] && old->omega[a] == om[a];
        if (same) return;
        for (int a = 0; a < 3; ++a) {
          old->center[a] = c[a];
          old->omega[a] = om[a];
        }
        old->scale = body_scale(pos, nm, c, om);
        invalidate_graphs();
        return;
      }
    }
    auto bs = std::make_unique<BodyState>();
    bs->nm = nm;
    bs->pos.assign(pos, pos + 3 * nm);
    bs->weight.assign(w, w + nm);
    for (int a = 0; a < 3; ++a) {
      bs->center[a] = c[a];
      bs->omega[a] = om[a];
    }
    bs->scale = body_scale(pos, nm, c, om);
    bs->d_pos.upload(bs->pos, st);
    bs->d_weight.upload(bs->weight, st);
    bs->imp.alloc(size_t(3 * nm));
    bs->mob.alloc(size_t(nm));
    bs->rmf.alloc(size_t(3 * nm));
    bs->part_diag.alloc(size_t(9 * ceil_div(nm, IBM_BLOCK)));
    CK(cudaStreamSynchronize(st));
    bodies[b] = std::move(bs);
    invalidate_graphs();
  }

  // scale = max(max |Omega x r|, 1) (solver.rs:3090-3094)
  static double body_scale(const double* pos, int64_t nm, const double* c, const double* om) {
    double mt = 0.0;
    for (int64_t m = 0; m < nm; ++m) {
      const double r[3] = {pos[3 * m] - c[0], pos[3 * m + 1] - c[1], pos[3 * m + 2] - c[2]};
      const double t[3] = {om[1] * r[2] - om[2] * r[1], om[2] * r[0] - om[0] * r[2], om[0] * r[1] - om[1] * r[0]};
      mt = std::max(mt, std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]));
    }
    return std::max(mt, 1.0);
  }

  static double linear_kernel(double r) { return std::max(1.0 - r, 0.0); }
  static double quadratic_kernel(double r) {
    if (r < 0.5) return 0.75 - r * r;
    if (r < 1.5) return 0.5 * (1.5 - r) * (1.5 - r);
    return 0.0;
  }

  // Marker stencils (rotating_ibm.rs:163-210) -> device CSR both ways.
  void build_stencils(BodyState& B, int radius) {
    const int dims[3] = {nx, ny, nz};
    std::vector<int32_t> st_off(size_t(B.nm) + 1, 0);
    std::vector<int64_t> st_cell;
    std::vector<double> st_w;
    for (int64_t m = 0; m < B.nm; ++m) {
      std::vector<std::pair<int, double>> ax[3];
      for (int a = 0; a < 3; ++a) {
        const double p = B.pos[3 * m + a];
        const long lo = long(std::floor(p)) - radius + 1, hi = long(std::floor(p)) + radius;
        for (long i = lo; i <= hi; ++i) {
          if (i < 0 || i >= dims[a]) continue;
          const double r = std::fabs(p - double(i));
          const double w = radius == 1 ? linear_kernel(r) : quadratic_kernel(r);
          if (w != 0.0) ax[a].push_back({int(i), w});
        }
      }
      if (ax[0].empty() || ax[1].empty() || ax[2].empty()) invalid("IBM marker stencil is outside the domain");
      for (auto& px : ax[0])
        for (auto& py : ax[1])
          for (auto& pz : ax[2]) {
            const int64_t c = idx(px.first, py.first, pz.first);
            if (solid_h[c]) continue;
            st_cell.push_back(c);
            st_w.push_back(px.second * py.second * pz.second);
          }
      st_off[m + 1] = int32_t(st_cell.size());
    }
    // global slots for the cells (appended, never removed)
    const std::vector<int32_t> st_slot = ensure_slots(st_cell);
    // body slots and reverse CSR in marker order
    std::vector<int32_t> local(size_t(nslots), -1);
    std::vector<int32_t> bslot;
    for (size_t k = 0; k < st_slot.size(); ++k)
      if (local[st_slot[k]] < 0) {
        local[st_slot[k]] = int32_t(bslot.size());
        bslot.push_back(st_slot[k]);
      }
    const int64_t ns = int64_t(bslot.size());
    std::vector<int32_t> cs_off(size_t(ns) + 1, 0);
    for (size_t k = 0; k < st_slot.size(); ++k) cs_off[local[st_slot[k]] + 1]++;
    for (int64_t i = 0; i < ns; ++i) cs_off[i + 1] += cs_off[i];
    std::vector<int32_t> fill(cs_off.begin(), cs_off.end() - 1);
    std::vector<int32_t> cs_marker(st_slot.size());
    std::vector<double> cs_w(st_slot.size());
    std::vector<double> cks(size_t(ns), 0.0);
    for (int64_t m = 0; m < B.nm; ++m)
      for (int32_t k = st_off[m]; k < st_off[m + 1]; ++k) {
        const int32_t l = local[st_slot[k]];
        cs_marker[fill[l]] = int32_t(m);
        cs_w[fill[l]] = st_w[k];
        fill[l]++;
        cks[l] += st_w[k];  // cell_kernel_sum in marker order (solver.rs:3107-3116)
      }
    std::vector<double> st_cks(st_slot.size());
    for (size_t k = 0; k < st_slot.size(); ++k) st_cks[k] = cks[local[st_slot[k]]];
    B.st_off.upload(st_off, st);
    B.st_slot.upload(st_slot, st);
    B.st_w.upload(st_w, st);
    B.st_cks.upload(st_cks, st);
    B.bslot.upload(bslot, st);
    B.cs_off.upload(cs_off, st);
    B.cs_marker.upload(cs_marker, st);
    B.cs_w.upload(cs_w, st);
    B.ns = ns;
    B.part_spread.alloc(size_t(3 * std::max<int64_t>(1, ceil_div(ns, IBM_BLOCK))));
    B.radius = radius;
    CK(cudaStreamSynchronize(st));
  }

  IbmArgs ibm_args(BodyState& B, const lbmb_ibm_config& c) {
    IbmArgs a;
    a.nm = B.nm;
    a.pos = B.d_pos.p;
    a.weight = B.d_weight.p;
    a.st_off = B.st_off.p;
    a.st_slot = B.st_slot.p;
    a.st_w = B.st_w.p;
    a.st_cks = B.st_cks.p;
    a.ns = B.ns;
    a.bslot = B.bslot.p;
    a.cs_off = B.cs_off.p;
    a.cs_marker = B.cs_marker.p;
    a.cs_w = B.cs_w.p;
    a.rho = s_rho.p;
    a.u_now = s_unow.p;
    a.du = s_du.p;
    a.spread = s_spread.p;
    a.imp = B.imp.p;
    a.mob = B.mob.p;
    a.rmf = B.rmf.p;
    a.part_spread = B.part_spread.p;
    a.part_diag = B.part_diag.p;
    a.diag = d_diag.p;
    for (int k = 0; k < 3; ++k) {
      a.center[k] = B.center[k];
      a.omega[k] = B.omega[k];
    }
    a.scale = B.scale;
    a.relax = c.relaxation;
    a.tol = c.slip_tolerance;
    return a;
  }

  BodyState& body_for(int b, const lbmb_ibm_config& c) {
    if (c.max_iterations <= 0) invalid("IBM max_iterations must be positive");
    if (!(c.slip_tolerance >= 0.0 && std::isfinite(c.slip_tolerance)))
      invalid("IBM slip_tolerance must be finite and non-negative");
    if (!(c.relaxation > 0.0 && c.relaxation <= 1.0 && std::isfinite(c.relaxation)))
      invalid("IBM relaxation must be finite and in (0, 1]");
    if (c.kernel_radius != 1 && c.kernel_radius != 2) invalid("IBM kernel radius must be 1 or 2");
    if (b < 0 || b >= int(bodies.size()) || !bodies[b]) throw Error(LBMB_ERR_STATE, "IBM body not set");
    BodyState& B = *bodies[b];
    if (B.radius != c.kernel_radius) build_stencils(B, c.kernel_radius);
    return B;
  }

  // Device sequence of one apply_rotating_ibm call (no host sync).
  // Where the adjoint keeps the IBM intermediates of one step: rho, u_now
  // (per slot), mobility (per marker), du at the start of each sweep (per
  // slot) and each sweep's impulse (per marker).
  struct IbmSave {
    double *rho, *u, *mob, *du, *imp;
    size_t ns3, nm;
  };

  void enqueue_ibm(BodyState& B, const lbmb_ibm_config& c, double* s_torque, double* s_ff, int32_t* s_it,
                   int64_t* counter, bool field_at_call, cudaStream_t s_ = nullptr, const IbmSave* sv = nullptr) {
    cudaStream_t sx = s_ ? s_ : st;
    IbmArgs a = ibm_args(B, c);
    const unsigned gs = unsigned(std::max<int64_t>(1, ceil_div(B.ns, IBM_BLOCK)));
    const unsigned gm = unsigned(std::max<int64_t>(1, ceil_div(B.nm, IBM_BLOCK)));
    const uint8_t* fl = flags.p;
    const uint32_t* nb = nbr.p;
    const Vec4<A>* fc = fcur.p;
    launch_pdl(ibm_prep_kernel<Q, S>, gs, sx, a, static_cast<const S*>(fp), plane,
               static_cast<const int64_t*>(slot_cell.p), fl, nb, nx, ny, nz, parity, fc, field_at_call ? 1 : 0,
               double(A(cfg.force[0])), double(A(cfg.force[1])), double(A(cfg.force[2])));
    for (int s = 0; s < c.max_iterations; ++s) {
      if (sv && nslots)
        CK(cudaMemcpyAsync(sv->du + size_t(s) * sv->ns3 * 3, s_du.p, size_t(nslots) * 3 * sizeof(double),
                           cudaMemcpyDeviceToDevice, sx));
      launch_pdl(ibm_interp_kernel, gm, sx, a, s);
      if (sv && B.nm)
        CK(cudaMemcpyAsync(sv->imp + size_t(s) * sv->nm * 3, B.imp.p, size_t(B.nm) * 3 * sizeof(double),
                           cudaMemcpyDeviceToDevice, sx));
      launch_pdl(ibm_spread_kernel, gs, sx, a);
      launch_pdl(ibm_diag_kernel, gm, sx, a, s, int(gs));
    }
    if (sv) {
      if (nslots) {
        CK(cudaMemcpyAsync(sv->rho, s_rho.p, size_t(nslots) * sizeof(double), cudaMemcpyDeviceToDevice, sx));
        CK(cudaMemcpyAsync(sv->u, s_unow.p, size_t(nslots) * 3 * sizeof(double), cudaMemcpyDeviceToDevice, sx));
      }
      if (B.nm) CK(cudaMemcpyAsync(sv->mob, B.mob.p, size_t(B.nm) * sizeof(double), cudaMemcpyDeviceToDevice, sx));
    }
    CK(cudaGetLastError());
    launch_pdl(ibm_commit_kernel<A>, gs, sx, a, fcur.p, s_torque, s_ff, s_it, counter);
  }

  // One IBM-chain kernel of IBM_BLOCK threads with programmatic stream
  // serialization (the kernel waits for its predecessor with pdl_wait).
  template <class... KArgs, class... Args>
  void launch_pdl(void (*kernel)(KArgs...), unsigned grid, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(grid);
    lc.blockDim = dim3(IBM_BLOCK);
    lc.dynamicSmemBytes = 0;
    lc.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    CK(cudaLaunchKernelEx(&lc, kernel, static_cast<KArgs>(args)...));
  }

  // The IBM launch sequence of apply_rotating_ibm, captured once and
  // replayed while every kernel argument is unchanged (the key holds all of
  // them): one graph launch instead of 2 + 3 x sweeps kernel launches.
  struct ApplyKey {
    IbmArgs a;
    const void* f;
    const void* slots;
    const void* field;
    int64_t parity, field_at_call, sweeps;
    double force[3];
  };
  // Instantiated IBM graphs by key. A runner alternates between the two AA
  // parities (and a caller may alternate bodies), so a single cached graph
  // would be captured and instantiated again on every call.
  struct ApplyEntry {
    ApplyKey key;
    cudaGraphExec_t exec;
  };
  std::vector<ApplyEntry> apply_cache;
  static constexpr size_t APPLY_CACHE = 8;

  // The instantiated IBM graph of one apply (captured on the main stream at
  // first use; launched on either stream).
  cudaGraphExec_t apply_exec(BodyState& B, const lbmb_ibm_config& c) {
    ApplyKey k;
    std::memset(&k, 0, sizeof(k));
    k.a = ibm_args(B, c);
    k.f = fp;
    k.slots = slot_cell.p;
    k.field = fcur.p;
    k.parity = parity;
    k.field_at_call = field_present ? 1 : 0;
    k.sweeps = c.max_iterations;
    for (int i = 0; i < 3; ++i) k.force[i] = cfg.force[i];
    cudaGraphExec_t exec = nullptr;
    for (auto& e : apply_cache)
      if (std::memcmp(&k, &e.key, sizeof(k)) == 0) exec = e.exec;
    if (!exec) {
      if (apply_cache.size() >= APPLY_CACHE) {
        CK(cudaGraphExecDestroy(apply_cache.front().exec));
        apply_cache.erase(apply_cache.begin());
      }
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      enqueue_ibm(B, c, nullptr, nullptr, nullptr, nullptr, field_present);
      CK(cudaStreamEndCapture(st, &g));
      CK(cudaGraphInstantiate(&exec, g, 0));
      CK(cudaGraphDestroy(g));
      apply_cache.push_back({k, exec});
    }
    return exec;
  }

  void ibm_apply(int b, const lbmb_ibm_config& c, lbmb_ibm_diag* out) override {
    BodyState& B = body_for(b, c);
    CK(cudaGraphLaunch(apply_exec(B, c), st));
    field_present = true;
    fprev_stale = true;
    IbmDiagDev d;
    CK(cudaMemcpyAsync(&d, d_diag.p, sizeof(d), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    diag_out(d, out);
  }

  // Pinned host copy of the IBM diagnostics (runner_step) and the event
  // that marks its arrival.
  IbmDiagDev* h_diag = nullptr;
  cudaEvent_t ev_diag = nullptr;

  // One iteration of the runner loop with the caller's marker set
  // (runner.rs:1080-1085: clear_body_force_field, apply the marker set,
  // step): the marker upload and the clear on the main stream, then the IBM
  // apply, its diagnostics copy and the forced cells on the side stream
  // beside the full-grid sweep (disjoint AA slots, as in run_impeller); the
  // host waits for the diagnostics only. Same device operations and results
  // as the four calls lbmb_clear_body_force_field, lbmb_ibm_set_body,
  // lbmb_apply_rotating_ibm and lbmb_step(1).
  // Instantiated device sequences of runner_step in the steady state (a
  // field present, no refresh pending, no scalars), one per key (IBM
  // arguments and AA parity): the clear, the fork, the sweep, the IBM, the
  // diagnostics copy, the forced cells, the refresh and the join in one
  // graph launch.
  struct FusedEntry {
    ApplyKey key;
    cudaGraphExec_t exec;
  };
  std::vector<FusedEntry> fused_cache;

  void drop_fused_graphs() {
    for (auto& e : fused_cache) CK(cudaGraphExecDestroy(e.exec));
    fused_cache.clear();
  }

  // The step's device work: the clear (captured form), fork, the full-grid
  // sweep on the main stream and on the side stream the IBM apply, the
  // diagnostics copy, the forced cells and the refresh; join. (Measured: the
  // clear and the marker upload on the side stream instead made the
  // per-call loop 6% slower.)
  void enqueue_runner_step(BodyState& B, const lbmb_ibm_config& c, bool captured) {
    if (captured) enqueue_clear_device();
    CK(cudaEventRecord(ev_fork, st));
    CK(cudaStreamWaitEvent(st2, ev_fork, 0));
    launch_hydro(parity, st, true, false);
    enqueue_ibm(B, c, nullptr, nullptr, nullptr, nullptr, false, st2);
    CK(cudaMemcpyAsync(h_diag, d_diag.p, sizeof(IbmDiagDev), cudaMemcpyDeviceToHost, st2));
    // inside a graph, an external record node: the host waits on it
    CK(cudaEventRecordWithFlags(ev_diag, st2, captured ? cudaEventRecordExternal : cudaEventRecordDefault));
    launch_hydro(parity, st2, false, true);
    if (nslots) CK(cudaMemcpyAsync(fprev.p, fcur.p, size_t(nslots) * sizeof(Vec4<A>), cudaMemcpyDeviceToDevice, st2));
    CK(cudaEventRecord(ev_join, st2));
    CK(cudaStreamWaitEvent(st, ev_join, 0));
  }

  void runner_step(int b, const double* pos, const double* w, int64_t nm, const double* c, const double* om,
                   const lbmb_ibm_config& cfg_ibm, lbmb_ibm_diag* out) override {
    if (has_uniform_force()) throw Error(LBMB_ERR_UNSUPPORTED, "runner step: a uniform body force is set");
    set_body(b, pos, w, nm, c, om, st);
    BodyState& B = body_for(b, cfg_ibm);
    if (!h_diag) CK(cudaMallocHost(&h_diag, sizeof(IbmDiagDev)));
    const bool steady = field_present && !fprev_stale && scalars.empty();
    if (steady) {
      ApplyKey k;
      std::memset(&k, 0, sizeof(k));
      k.a = ibm_args(B, cfg_ibm);
      k.f = fp;
      k.slots = slot_cell.p;
      k.field = fcur.p;
      k.parity = parity;
      k.sweeps = cfg_ibm.max_iterations;
      cudaGraphExec_t exec = nullptr;
      for (auto& e : fused_cache)
        if (std::memcmp(&k, &e.key, sizeof(k)) == 0) exec = e.exec;
      if (!exec) {
        if (fused_cache.size() >= 4) {
          CK(cudaGraphExecDestroy(fused_cache.front().exec));
          fused_cache.erase(fused_cache.begin());
        }
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        enqueue_runner_step(B, cfg_ibm, true);
        CK(cudaStreamEndCapture(st, &g));
        CK(cudaGraphInstantiate(&exec, g, 0));
        CK(cudaGraphDestroy(g));
        fused_cache.push_back({k, exec});
      }
      CK(cudaEventRecord(ev0, st));
      CK(cudaGraphLaunch(exec, st));
    } else {
      clear_force_field();  // may synchronise (a refresh pending)
      CK(cudaEventRecord(ev0, st));
      enqueue_runner_step(B, cfg_ibm, false);
    }
    field_present = true;
    fprev_stale = false;
    parity ^= 1;
    for (auto& sc : scalars) scalar_step(*sc);
    CK(cudaEventRecord(ev1, st));
    pending_launches = 1;
    timing_pending = true;
    time += 1;
    if (kernel_mode == LBMB_SWEEP_BULK) {
      CK(cudaStreamSynchronize(st));
      check_device_error();
    } else {
      // The call returns once the diagnostics are on the host, while the
      // sweep may still run (as lbmb_step returns once its work is queued):
      // the host's next call overlaps it. Entry points that return data
      // synchronise the stream.
      CK(cudaEventSynchronize(ev_diag));
    }
    diag_out(*h_diag, out);
  }

  static void diag_out(const IbmDiagDev& d, lbmb_ibm_diag* out) {
    if (out) {
      out->iterations = d.iterations;
      out->slip_max = d.slip_max;
      out->slip_rms = d.slip_rms;
      out->slip_max_rel = d.slip_max_rel;
      out->slip_rms_rel = d.slip_rms_rel;
      for (int k = 0; k < 3; ++k) {
        out->torque[k] = d.torque[k];
        out->fluid_force[k] = d.fluid_force[k];
        out->marker_force[k] = d.marker_force[k];
      }
      out->momentum_error_rel = d.momentum_error_rel;
    }
  }

  // ---- scalars ----------------------------------------------------------
  int enable_scalar(int q, double d) override {
    if (!(std::isfinite(d) && d > 0.0)) invalid("scalar diffusivity must be finite > 0");
    if (q != 7 && q != Q) invalid("scalar lattice must be D3Q7 or the hydro lattice");
    auto sc = std::make_unique<ScalarStateT<A>>();
    sc->name = "scalar" + std::to_string(scalars.size());
    sc->q = q;
    sc->diffusivity = d;
    sc->hplane = plane;
    sc->h.alloc(size_t(q) * plane);
    CK(cudaMemsetAsync(sc->h.p, 0, size_t(q) * plane * sizeof(A), st));
    sc->part.alloc(size_t(red_blocks));
    sc->stats.alloc(4);
    CK(cudaStreamSynchronize(st));
    scalars.push_back(std::move(sc));
    invalidate_graphs();
    return int(scalars.size()) - 1;
  }
  ScalarStateT<A>& scalar(int k) {
    if (k < 0 || k >= int(scalars.size())) throw Error(LBMB_ERR_STATE, "scalar distribution not enabled");
    return *scalars[k];
  }
  void set_scalar(int k, const double* c) override {
    auto& sc = scalar(k);
    DevBuf<double> dc;
    dc.upload(c, size_t(n), st);
    ScalarParams<A> p = scalar_params(sc);
    const unsigned g = unsigned(ceil_div(n, 128));
    if (sc.q == 7) scalar_set_kernel<7, Q, S><<<g, 128, 0, st>>>(p, dc.p, init_u_dev(), n);
    else scalar_set_kernel<Q, Q, S><<<g, 128, 0, st>>>(p, dc.p, init_u_dev(), n);
    CK(cudaGetLastError());
    sc.parity = 0;
    CK(cudaStreamSynchronize(st));
  }
  void get_scalar(int k, double* c) override {
    auto& sc = scalar(k);
    DevBuf<double> dc;
    dc.alloc(size_t(n));
    const unsigned g = unsigned(ceil_div(n, 128));
    if (sc.q == 7)
      scalar_gather_kernel<7, A><<<g, 128, 0, st>>>(sc.h.p, sc.hplane, flags.p, nbr.p, nx, ny, nz, sc.parity, dc.p, n);
    else
      scalar_gather_kernel<Q, A><<<g, 128, 0, st>>>(sc.h.p, sc.hplane, flags.p, nbr.p, nx, ny, nz, sc.parity, dc.p, n);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c, dc.p, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  // ---- checkpoint/restart (Solver::save / restore, solver.rs:4536-5066) ----
  const lbmb_config& config() const override { return cfg; }
  void set_scalar_name(int k, const std::string& name) override {
    if (name.empty() || name.size() > 63) invalid("scalar name must have 1 to 63 bytes");
    scalar(k).name = name;
  }
  // Pinned host staging of checkpoint images (kept between calls).
  struct PinBuf {
    char* p = nullptr;
    size_t n = 0;
    PinBuf() = default;
    PinBuf(const PinBuf&) = delete;
    PinBuf& operator=(const PinBuf&) = delete;
    ~PinBuf() {
      if (p) cudaFreeHost(p);
    }
    char* ensure(size_t b) {
      if (b > n) {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        CK(cudaHostAlloc(reinterpret_cast<void**>(&p), b, cudaHostAllocDefault));
        n = b;
      }
      return p;
    }
  };
  PinBuf ckpt_pin;
  // file dtype of the populations: f64 storage writes "f64", the rest "f32"
  using FileT = typename std::conditional<std::is_same<S, double>::value, double, float>::type;

  // Solver::save (solver.rs:4536-4724): the device packs the padded
  // population and scalar planes in the file's type, one copy brings them to
  // pinned memory, and the writer hashes them while a second thread writes
  // the rank file.
  void checkpoint_save(const std::string& dir) override {
    const ckpt::Spec sp = ckpt::spec_of(cfg);
    const size_t w = sizeof(FileT);
    const int64_t np = int64_t(ckpt::padded_cells(sp));
    size_t total = size_t(Q) * size_t(np) * w;
    for (auto& sc : scalars) total += size_t(sc->q) * size_t(np) * w;
    DevBuf<char> img;
    img.alloc(total);
    char* pin = ckpt_pin.ensure(total);
    const unsigned g = unsigned(ceil_div(np, 256));
    pack_padded_kernel<Q, S, FileT><<<g, 256, 0, st>>>(fp, plane, flags.p, nbr.p, nx, ny, nz, parity,
                                                      reinterpret_cast<FileT*>(img.p), np);
    CK(cudaGetLastError());
    size_t off = size_t(Q) * size_t(np) * w;
    std::vector<size_t> soff;
    for (auto& scp : scalars) {
      ScalarStateT<A>& sc = *scp;
      FileT* out = reinterpret_cast<FileT*>(img.p + off);
      if (sc.q == 7)
        scalar_pack_padded_kernel<7, A, FileT><<<g, 256, 0, st>>>(sc.h.p, sc.hplane, flags.p, nbr.p, nx, ny, nz,
                                                                   sc.parity, out, np);
      else
        scalar_pack_padded_kernel<Q, A, FileT><<<g, 256, 0, st>>>(sc.h.p, sc.hplane, flags.p, nbr.p, nx, ny, nz,
                                                                   sc.parity, out, np);
      CK(cudaGetLastError());
      soff.push_back(off);
      off += size_t(sc.q) * size_t(np) * w;
    }
    CK(cudaMemcpyAsync(pin, img.p, total, cudaMemcpyDeviceToHost, st));
    // moments (solid cells carried), force field, concentrations
    std::vector<double> mom(size_t(4) * size_t(n));
    read_moments(mom.data(), mom.data() + n, mom.data() + 2 * n, mom.data() + 3 * n);
    std::vector<double> ff;
    if (field_present) {
      ff.resize(size_t(3) * size_t(n));
      get_force_field(ff.data());
    }
    std::vector<std::vector<double>> conc(scalars.size());
    for (size_t k = 0; k < scalars.size(); ++k) {
      conc[k].resize(size_t(n));
      get_scalar(int(k), conc[k].data());
    }
    CK(cudaStreamSynchronize(st));
    std::vector<std::string> keep;
    keep.reserve(8 + 4 * scalars.size());
    auto piece = [&](std::string b) {
      keep.push_back(std::move(b));
      return ckpt::Piece{keep.back().data(), keep.back().size()};
    };
    auto reals = [&](const std::vector<double>& v) {
      std::string b;
      ckpt::append_reals(b, v.data(), v.size(), sp.f64);
      return piece(std::move(b));
    };
    std::vector<ckpt::SectionOut> secs;
    secs.push_back({ckpt::SEC_F_PRIMARY, {ckpt::Piece{pin, uint64_t(Q) * uint64_t(np) * w}}});
    secs.push_back({ckpt::SEC_STALE_STASH, {ckpt::Piece{nullptr, uint64_t(Q) * uint64_t(np) * w}}});
    secs.push_back({ckpt::SEC_MOMENTS, {reals(mom)}});
    secs.push_back({ckpt::SEC_SOLID, {piece(ckpt::solid_section(sp, solid_h.data()))}});
    if (field_present) secs.push_back({ckpt::SEC_FORCE_FIELD, {reals(ff)}});
    if (!scalars.empty()) {
      ckpt::SectionOut sec{ckpt::SEC_SCALAR_FIELDS, {}};
      std::string count;
      const uint32_t cnt = uint32_t(scalars.size());
      count.append(reinterpret_cast<const char*>(&cnt), 4);
      sec.pieces.push_back(piece(std::move(count)));
      for (size_t k = 0; k < scalars.size(); ++k) {
        const ScalarStateT<A>& sc = *scalars[k];
        const uint64_t hl = uint64_t(sc.q) * uint64_t(np);
        sec.pieces.push_back(piece(ckpt::scalar_head(sc.name, sc.diffusivity, hl)));
        sec.pieces.push_back(ckpt::Piece{pin + soff[k], hl * w});
        for (const ckpt::Piece& p : ckpt::scalar_tail(sc.q, np, n, w))
          sec.pieces.push_back(p.data ? piece(std::string(p.data, size_t(p.len))) : p);
        sec.pieces.push_back(reals(conc[k]));
      }
      secs.push_back(std::move(sec));
    }
    if (has_qoi) secs.push_back({ckpt::SEC_QOI_ACCUMULATORS, {piece(qoi_json)}});
    ckpt::write(dir, sp, time, secs, solid_h.data(), wall_u_in.empty() ? nullptr : wall_u_in.data(), has_qoi);
  }

  // Solver::restore (solver.rs:4739-5060): the rank file is mapped and
  // hashed in place; after every check the padded planes go to the device in
  // one copy each and are unpacked into the parity-0 layout.
  void checkpoint_restore(const std::string& dir) override {
    const ckpt::Spec sp = ckpt::spec_of(cfg);
    const size_t w = sizeof(FileT);
    const int64_t np = int64_t(ckpt::padded_cells(sp));
    const ckpt::View v = ckpt::read(dir, sp, solid_h.data(), wall_u_in.empty() ? nullptr : wall_u_in.data());
    // the scalars of the file replace the solver's: checked before anything
    // is installed
    if (scalars.size() > v.scalars.size())
      throw ckpt::Failure("CKPT_SCENARIO_MISMATCH",
                          "solver has " + std::to_string(scalars.size()) + " scalar distributions, checkpoint has " +
                              std::to_string(v.scalars.size()));
    for (size_t k = 0; k < v.scalars.size(); ++k) {
      const int q = v.scalars[k].q;
      if (k < scalars.size() && scalars[k]->q != q)
        throw ckpt::Failure("CKPT_SCENARIO_MISMATCH", "scalar " + std::to_string(k) + " lattice differs: checkpoint D3Q" +
                                                          std::to_string(q) + ", solver D3Q" +
                                                          std::to_string(scalars[k]->q));
      if (!(std::isfinite(v.scalars[k].diffusivity) && v.scalars[k].diffusivity > 0.0))
        throw ckpt::Failure("CKPT_PAYLOAD_CORRUPT", "scalar diffusivity must be finite > 0");
      if (v.scalars[k].name.empty() || v.scalars[k].name.size() > 63)
        throw ckpt::Failure("CKPT_PAYLOAD_CORRUPT", "scalar name must have 1 to 63 bytes");
    }
    std::vector<double> mom(size_t(4) * size_t(n));
    ckpt::reals_to_double(v.moments, mom.size(), sp.f64, mom.data());
    std::vector<double> ff;
    if (v.force_field) {
      ff.resize(size_t(3) * size_t(n));
      ckpt::reals_to_double(v.force_field, ff.size(), sp.f64, ff.data());
    }
    size_t total = size_t(Q) * size_t(np) * w;
    for (const auto& x : v.scalars) total += size_t(x.q) * size_t(np) * w;
    DevBuf<char> img;
    img.alloc(total);
    sync();
    CK(cudaMemcpyAsync(img.p, v.f, size_t(Q) * size_t(np) * w, cudaMemcpyHostToDevice, st));
    size_t off = size_t(Q) * size_t(np) * w;
    std::vector<size_t> soff;
    for (const auto& x : v.scalars) {
      CK(cudaMemcpyAsync(img.p + off, x.h, size_t(x.q) * size_t(np) * w, cudaMemcpyHostToDevice, st));
      soff.push_back(off);
      off += size_t(x.q) * size_t(np) * w;
    }
    const unsigned g = unsigned(ceil_div(n, 256));
    unpack_padded_kernel<Q, S, FileT><<<g, 256, 0, st>>>(fp, plane, reinterpret_cast<const FileT*>(img.p), nx, ny,
                                                        nz, n);
    CK(cudaGetLastError());
    parity = 0;
    install_force_field(v.force_field ? ff.data() : nullptr);
    for (int64_t c = 0; c < n; ++c)
      if (solid_h[c]) {
        init_rho_h[c] = mom[size_t(c)];
        for (int k = 0; k < 3; ++k) init_u_h[size_t(3 * c + k)] = mom[size_t((k + 1) * n + c)];
      }
    d_init_u_ok = false;
    for (size_t k = 0; k < v.scalars.size(); ++k) {
      const ckpt::ScalarView& x = v.scalars[k];
      if (k >= scalars.size()) enable_scalar(x.q, x.diffusivity);
      ScalarStateT<A>& sc = *scalars[k];
      sc.diffusivity = x.diffusivity;
      sc.name = x.name;
      scalar_unpack_padded_kernel<A, FileT><<<g, 256, 0, st>>>(
          sc.h.p, sc.hplane, reinterpret_cast<const FileT*>(img.p + soff[k]), sc.q, nx, ny, nz, n);
      CK(cudaGetLastError());
      sc.parity = 0;
    }
    CK(cudaStreamSynchronize(st));
    time = v.step;
    has_qoi = v.has_qoi;
    qoi_json = v.qoi_json;
    invalidate_graphs();
  }

  // Body-force field of a checkpoint: slots for the fluid cells with a
  // nonzero force, the values in both the applied field and the field inside
  // the cached moments (null: no field).
  void install_force_field(const double* ff) {
    if (ff) {
      std::vector<int64_t> cells;
      for (int64_t c = 0; c < n; ++c)
        if (!solid_h[c] && fslot_h[c] < 0 && (ff[3 * c] != 0.0 || ff[3 * c + 1] != 0.0 || ff[3 * c + 2] != 0.0))
          cells.push_back(c);
      ensure_slots(cells);
    }
    if (nslots) {
      std::vector<Vec4<A>> hv(size_t(nslots), Vec4<A>{A(0), A(0), A(0), A(0)});
      if (ff)
        for (int64_t k = 0; k < nslots; ++k) {
          const int64_t c = slot_cell_h[size_t(k)];
          hv[size_t(k)] = Vec4<A>{A(ff[3 * c]), A(ff[3 * c + 1]), A(ff[3 * c + 2]), A(0)};
        }
      CK(cudaMemcpyAsync(fcur.p, hv.data(), hv.size() * sizeof(Vec4<A>), cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(fprev.p, hv.data(), hv.size() * sizeof(Vec4<A>), cudaMemcpyHostToDevice, st));
      CK(cudaStreamSynchronize(st));
    }
    field_present = ff != nullptr;
    fprev_stale = false;
    invalidate_graphs();
  }
  // Oxygen transfer / uptake on scalar k (the gather -> host source ->
  // set composition of the reference, on the device). a's arrays are host
  // pointers (n values each, or null); *sum = the source integral.
  void scalar_oxygen(int k, const OxygenSourceArgs& a0, double* sum, lbmb_oxygen_diag* diag,
                     int64_t* active) override {
    auto& sc = scalar(k);
    OxygenSourceArgs a = a0;
    DevBuf<double> dc, cs, ar, vo, de, part;
    DevBuf<int> err;
    DevBuf<unsigned long long> cnt;
    if (a0.cstar) cs.upload(a0.cstar, size_t(n), st);
    if (a0.area) ar.upload(a0.area, size_t(n), st);
    if (a0.vol) vo.upload(a0.vol, size_t(n), st);
    if (a0.density) de.upload(a0.density, size_t(n), st);
    a.cstar = a0.cstar ? cs.p : nullptr;
    a.area = a0.area ? ar.p : nullptr;
    a.vol = a0.vol ? vo.p : nullptr;
    a.density = a0.density ? de.p : nullptr;
    dc.alloc(size_t(n));
    const unsigned g = unsigned(ceil_div(n, 128));
    if (sc.q == 7)
      scalar_gather_kernel<7, A><<<g, 128, 0, st>>>(sc.h.p, sc.hplane, flags.p, nbr.p, nx, ny, nz, sc.parity, dc.p, n);
    else
      scalar_gather_kernel<Q, A><<<g, 128, 0, st>>>(sc.h.p, sc.hplane, flags.p, nbr.p, nx, ny, nz, sc.parity, dc.p, n);
    const int64_t nb = ceil_div(n, OXY_BLOCK);
    part.alloc(size_t(2 * nb));
    err.alloc(1);
    cnt.alloc(2);
    CK(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    CK(cudaMemsetAsync(cnt.p, 0, 2 * sizeof(unsigned long long), st));
    oxygen_source_kernel<<<unsigned(nb), OXY_BLOCK, 0, st>>>(dc.p, a, err.p, part.p, cnt.p, n);
    CK(cudaGetLastError());
    int e = 0;
    unsigned long long hc[2] = {0, 0};
    std::vector<double> hp(static_cast<size_t>(2 * nb));
    CK(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hc, cnt.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hp.data(), part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (e & 1) invalid("cell volume must be finite and positive");
    if (e & 2) invalid("oxygen transfer source inputs must be finite (C_L, C*, area density >= 0)");
    if (e & 4) invalid("oxygen concentration must be finite and non-negative before the uptake");
    if (e & 8) invalid("cell density must be finite and non-negative");
    double s = 0.0, mn = INFINITY;
    for (int64_t b = 0; b < nb; ++b) {
      s += hp[size_t(2 * b)];
      if (hp[size_t(2 * b + 1)] < mn) mn = hp[size_t(2 * b + 1)];
    }
    if (sum) *sum = s;
    if (active) *active = int64_t(hc[0]);
    if (diag) {
      diag->clipped_cells = int64_t(hc[1]);
      diag->clipped_fraction = n == 0 ? 0.0 : double(hc[1]) / double(n);
      diag->min_before_clip = std::isfinite(mn) ? mn : 0.0;
    }
    // set_scalar_concentration: equilibrium of the new C at the current u
    ScalarParams<A> p = scalar_params(sc);
    if (sc.q == 7) scalar_set_kernel<7, Q, S><<<g, 128, 0, st>>>(p, dc.p, init_u_dev(), n);
    else scalar_set_kernel<Q, Q, S><<<g, 128, 0, st>>>(p, dc.p, init_u_dev(), n);
    CK(cudaGetLastError());
    sc.parity = 0;
    CK(cudaStreamSynchronize(st));
  }

  // Device CV of a scalar into *out (two deterministic passes).
  void enqueue_cv(ScalarStateT<A>& sc, double* out, double nfluid) {
    for (int pass = 0; pass < 2; ++pass) {
      if (sc.q == 7)
        scalar_cv_kernel<7, A><<<red_blocks, RED_BLOCK, 0, st>>>(sc.h.p, sc.hplane, flags.p, nbr.p, nx, ny, nz,
                                                                  sc.parity, n, pass, sc.stats.p, nfluid, sc.part.p);
      else
        scalar_cv_kernel<Q, A><<<red_blocks, RED_BLOCK, 0, st>>>(sc.h.p, sc.hplane, flags.p, nbr.p, nx, ny, nz,
                                                                  sc.parity, n, pass, sc.stats.p, nfluid, sc.part.p);
      scalar_cv_finish_kernel<<<1, 32, 0, st>>>(sc.part.p, red_blocks, pass, sc.stats.p, nfluid, out);
    }
    CK(cudaGetLastError());
  }

  // ---- runner loop ------------------------------------------------------
  // Series buffers of the runner (torque, fluid force, IBM iterations, CV,
  // step counter), kept on the handle and grown only when a longer run needs
  // them: the captured runner graph writes into them, so it stays valid from
  // one call to the next.
  DevBuf<double> run_torque, run_ff, run_cv;
  DevBuf<int32_t> run_it;
  DevBuf<int64_t> run_counter;
  int64_t run_cap = 0;
  // The instantiated runner graph (RUN_G steps from parity 0) and what it
  // was captured with: the IBM launch arguments, the body, the probed scalar
  // and the parity of every scalar at the graph's first step. Sweep kernel,
  // geometry, slots and scalar set changes destroy it (invalidate_graphs).
  static constexpr int64_t RUN_G = 16;
  struct RunKey {
    ApplyKey apply;
    int32_t body;
    int32_t nscal;
    const void* sc_h[8];
    int32_t sc_par[8];
  };
  RunKey run_key;
  // graphs of 16, 8, 4 and 2 steps (index 0..3) for the same key, so that a
  // span that is not a multiple of 16 replays graphs down to one step
  static constexpr int RUN_NG = 4;
  cudaGraphExec_t run_graphs[RUN_NG] = {nullptr, nullptr, nullptr, nullptr};
  bool run_graph = false;
  // Outcome of the last run_impeller call (runner.rs:1077-1129): steps
  // executed and whether the run stopped on a non-finite total mass.
  int64_t run_executed = 0;
  bool run_diverged = false;
  // The runner checks the f64 total mass after every DIVERGE_EVERY-th step
  // of a run and stops at the first non-finite value (runner.rs:1125-1128).
  static constexpr int64_t DIVERGE_EVERY = 1000;

  void drop_run_graphs() {
    for (auto& g : run_graphs)
      if (g) {
        CK(cudaGraphExecDestroy(g));
        g = nullptr;
      }
    run_graph = false;
  }

  void run_reserve(int64_t steps) {
    if (steps <= run_cap && run_counter.p) return;
    const int64_t cap = std::max<int64_t>({steps, 2 * run_cap, int64_t(1024)});
    run_torque.alloc(size_t(cap));
    run_ff.alloc(size_t(3 * cap));
    run_it.alloc(size_t(cap));
    run_cv.alloc(size_t(cap));
    run_counter.alloc(1);
    run_cap = cap;
    drop_run_graphs();
  }

  void run_impeller(int b, const lbmb_ibm_config& c, int64_t steps, int k, int64_t probe_every, double* torque,
                    double* ffo, double* cv, int32_t* iters) override {
    BodyState& B = body_for(b, c);
    if (k >= 0) scalar(k);
    if (probe_every <= 0) probe_every = 1;
    run_reserve(steps);
    run_executed = 0;
    run_diverged = false;
    CK(cudaMemsetAsync(run_counter.p, 0, sizeof(int64_t), st));
    if (k >= 0) fill_nan(run_cv.p, steps);
    int64_t launches = 0;
    auto one_step = [&](int64_t step_index) {
      // Fork: the IBM chain (clear -> direct forcing -> forced-cell hydro)
      // runs on the high-priority side stream while the full-grid sweep of
      // every other cell runs on the main stream; the two touch disjoint
      // population slots (each cell's AA read/write set is its own).
      CK(cudaEventRecord(ev_fork, st));
      CK(cudaStreamWaitEvent(st2, ev_fork, 0));
      // Solver::clear_body_force_field: the IBM field is non-uniform, so the
      // cached moments keep it (F_prev) while the new field starts at zero.
      if (nslots) CK(cudaMemsetAsync(fcur.p, 0, size_t(nslots) * sizeof(Vec4<A>), st2));
      enqueue_ibm(B, c, run_torque.p, run_ff.p, run_it.p, run_counter.p, false, st2);
      field_present = true;
      fprev_stale = true;
      launch_hydro(parity, st2, false, true);
      launch_hydro(parity, st, true, false);
      // cached-moment field refresh on the side stream behind the forced
      // cells, hidden by the full-grid sweep
      if (nslots) CK(cudaMemcpyAsync(fprev.p, fcur.p, size_t(nslots) * sizeof(Vec4<A>), cudaMemcpyDeviceToDevice, st2));
      fprev_stale = false;
      CK(cudaEventRecord(ev_join, st2));
      CK(cudaStreamWaitEvent(st, ev_join, 0));
      parity ^= 1;
      for (auto& sc : scalars) scalar_step(*sc);
      ++launches;
      if (k >= 0 && ((step_index + 1) % probe_every == 0 || step_index + 1 == steps))
        enqueue_cv(*scalars[k], run_cv.p + step_index, double(n - solid_count()));
    };
    // Graph replay of blocks of 16, 8, 4 or 2 steps (parity-aligned) when
    // no scalar is probed. The graphs are captured, instantiated and
    // uploaded before the timed region and kept for the next call while
    // their key holds.
    const bool use_graph = (k < 0) && steps - (parity ? 1 : 0) >= 2 && scalars.size() <= 8;
    if (use_graph) {
      RunKey key;
      std::memset(&key, 0, sizeof(key));
      key.apply.a = ibm_args(B, c);
      key.apply.f = fp;
      key.apply.slots = slot_cell.p;
      key.apply.field = fcur.p;
      key.apply.sweeps = c.max_iterations;
      for (int i = 0; i < 3; ++i) key.apply.force[i] = cfg.force[i];
      key.body = b;
      key.nscal = int32_t(scalars.size());
      // scalar parities at the graph's first step (hydro parity 0)
      for (size_t i = 0; i < scalars.size(); ++i) {
        key.sc_h[i] = scalars[i]->h.p;
        key.sc_par[i] = scalars[i]->parity ^ parity;
      }
      if (run_graph && std::memcmp(&key, &run_key, sizeof(key)) != 0) drop_run_graphs();
      if (!run_graph) {
        // capture from parity 0 with the scalar parities the graph will
        // start from, then put the host state back
        const int par0 = parity;
        std::vector<int> spar(scalars.size());
        for (size_t i = 0; i < scalars.size(); ++i) {
          spar[i] = scalars[i]->parity;
          scalars[i]->parity = key.sc_par[i];
        }
        const bool fpres = field_present, fstale = fprev_stale;
        for (int gi = 0; gi < RUN_NG; ++gi) {
          parity = 0;
          cudaGraph_t g;
          CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
          for (int64_t i = 0; i < (RUN_G >> gi); ++i) one_step(0);
          CK(cudaStreamEndCapture(st, &g));
          CK(cudaGraphInstantiate(&run_graphs[gi], g, 0));
          CK(cudaGraphDestroy(g));
          // upload now, so that the first replay inside a timed span does
          // not carry it
          CK(cudaGraphUpload(run_graphs[gi], st));
        }
        run_graph = true;
        parity = par0;
        for (size_t i = 0; i < scalars.size(); ++i) scalars[i]->parity = spar[i];
        field_present = fpres;
        fprev_stale = fstale;
        launches = 0;
        run_key = key;
      }
    }
    CK(cudaEventRecord(ev0, st));
    int64_t done = 0;
    while (done < steps) {
      // next divergence check after step number `check` (1-based)
      const int64_t check = (done / DIVERGE_EVERY + 1) * DIVERGE_EVERY;
      const int64_t stop = std::min(steps, check);
      while (done < stop) {
        int gi = 0;
        while (gi < RUN_NG && stop - done < (RUN_G >> gi)) ++gi;
        if (use_graph && parity == 0 && gi < RUN_NG) {
          CK(cudaGraphLaunch(run_graphs[gi], st));
          done += RUN_G >> gi;
          launches += RUN_G >> gi;
          field_present = true;
          fprev_stale = false;
        } else {
          one_step(done);
          ++done;
        }
      }
      if (done == check) {
        double r[5];
        reduce_all(r);  // synchronizes the stream
        if (!std::isfinite(r[0] + r[1])) {
          run_diverged = true;
          break;
        }
      }
    }
    run_executed = done;
    CK(cudaEventRecord(ev1, st));
    CK(cudaEventSynchronize(ev1));
    check_device_error();
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    last_total_ms = ms;
    last_hydro_ms = ms;
    last_hydro_launches = launches;
    timing_pending = false;
    // series of the executed steps; the steps a diverged run did not take
    // read NaN (iterations 0)
    const size_t ex = size_t(done), rest = size_t(steps - done);
    const double qnan = std::nan("");
    if (torque) {
      if (ex) CK(cudaMemcpy(torque, run_torque.p, ex * sizeof(double), cudaMemcpyDeviceToHost));
      std::fill(torque + ex, torque + ex + rest, qnan);
    }
    if (ffo) {
      if (ex) CK(cudaMemcpy(ffo, run_ff.p, 3 * ex * sizeof(double), cudaMemcpyDeviceToHost));
      std::fill(ffo + 3 * ex, ffo + 3 * (ex + rest), qnan);
    }
    if (iters) {
      if (ex) CK(cudaMemcpy(iters, run_it.p, ex * sizeof(int32_t), cudaMemcpyDeviceToHost));
      std::fill(iters + ex, iters + ex + rest, 0);
    }
    if (cv && k >= 0) {
      if (ex) CK(cudaMemcpy(cv, run_cv.p, ex * sizeof(double), cudaMemcpyDeviceToHost));
      std::fill(cv + ex, cv + ex + rest, qnan);
    }
    time += uint64_t(done);
    if (run_diverged)
      throw Error(LBMB_ERR_DIVERGED, "runner: non-finite total mass after step " + std::to_string(done));
  }

  void allows(int32_t* adjoint, int32_t* batch) const override {
    const bool f32 = std::is_same<A, float>::value;
    const bool trt = coll == COLL_TRT;
    *adjoint = (trt && !omega_on && !(cfg.smagorinsky_cs > 0.0) && !has_uniform_force() && scalars.empty()) ? 1 : 0;
    *batch = (trt && f32 && !has_uniform_force() && scalars.empty() && !omega_on) ? 1 : 0;
  }

  void run_status(int64_t* executed, int32_t* diverged) override {
    if (executed) *executed = run_executed;
    if (diverged) *diverged = run_diverged ? 1 : 0;
  }

  BatchBase* make_batch(const std::vector<EngineBase*>& all, const int32_t* bodies,
                        const lbmb_ibm_config& cfg) override;

  // ---- adjoint of the runner loop ------------------------------------------
  // One runner step (clear field -> IBM -> hydro of the forced cells on the
  // side stream, full-grid sweep on the main stream, field refresh), eager.
  void enqueue_runner_step(BodyState& B, const lbmb_ibm_config& c, double* s_torque, int64_t* counter,
                           const IbmSave* sv = nullptr) {
    CK(cudaEventRecord(ev_fork, st));
    CK(cudaStreamWaitEvent(st2, ev_fork, 0));
    if (nslots) CK(cudaMemsetAsync(fcur.p, 0, size_t(nslots) * sizeof(Vec4<A>), st2));
    enqueue_ibm(B, c, s_torque, nullptr, nullptr, counter, false, st2, sv);
    field_present = true;
    launch_hydro(parity, st2, false, true);
    launch_hydro(parity, st, true, false);
    CK(cudaEventRecord(ev_join, st2));
    CK(cudaStreamWaitEvent(st, ev_join, 0));
    parity ^= 1;
    if (nslots) CK(cudaMemcpyAsync(fprev.p, fcur.p, size_t(nslots) * sizeof(Vec4<A>), cudaMemcpyDeviceToDevice, st));
    fprev_stale = false;
  }

  void snapshot(S* out) {
    snapshot_kernel<Q, S><<<unsigned(ceil_div(n, 128)), 128, 0, st>>>(fp, plane, flags.p, nbr.p, nx, ny, nz, parity,
                                                                      out, n);
    CK(cudaGetLastError());
  }

  void adjoint_torque(const lbmb_ibm_config& c0, const lbmb_adjoint_config& ac, lbmb_adjoint_result* out,
                      double* dJ_dpos, double* torque_out) override {
    if (coll != COLL_TRT) throw Error(LBMB_ERR_UNSUPPORTED, "the adjoint covers TRT/BGK collision");
    if (omega_on) throw Error(LBMB_ERR_UNSUPPORTED, "the adjoint needs uniform relaxation rates (no omega field)");
    if (cfg.smagorinsky_cs > 0.0) throw Error(LBMB_ERR_UNSUPPORTED, "the adjoint needs the subgrid model off");
    if (has_uniform_force()) throw Error(LBMB_ERR_UNSUPPORTED, "the adjoint needs no uniform body force");
    if (!scalars.empty()) throw Error(LBMB_ERR_UNSUPPORTED, "the adjoint needs a solver without scalars");
    const int64_t N = ac.steps;
    if (N < 1) invalid("adjoint: steps must be >= 1");
    if (ac.window_begin < 0 || ac.window_begin >= N) invalid("adjoint: window_begin must be in [0, steps)");
    int64_t K = ac.checkpoint_every > 0 ? ac.checkpoint_every : 100;
    K += K & 1;
    // fixed sweep count: no early exit (slip tolerance 0)
    lbmb_ibm_config c = c0;
    c.slip_tolerance = 0.0;
    BodyState& B = body_for(ac.body, c);
    const int nsweep = c.max_iterations;
    const int64_t nseg = ceil_div(N, K);
    const size_t fsz = size_t(Q) * size_t(plane);
    const size_t ns3 = size_t(std::max<int64_t>(nslots, 1));
    sync();
    // ---- forward pass with checkpoints -------------------------------------
    DevBuf<S> ck_f;
    DevBuf<Vec4<A>> ck_fp;
    ck_f.alloc(size_t(nseg) * fsz);
    ck_fp.alloc(size_t(nseg) * ns3);
    DevBuf<double> d_torque;
    DevBuf<int64_t> d_counter;
    d_torque.alloc(size_t(N));
    d_counter.alloc(1);
    CK(cudaMemsetAsync(d_counter.p, 0, sizeof(int64_t), st));
    if (!field_present && nslots) CK(cudaMemsetAsync(fprev.p, 0, ns3 * sizeof(Vec4<A>), st));
    if (fprev_stale && nslots) {
      CK(cudaMemcpyAsync(fprev.p, fcur.p, ns3 * sizeof(Vec4<A>), cudaMemcpyDeviceToDevice, st));
      fprev_stale = false;
    }
    // Graph of one full segment (K steps; K even, so every segment starts
    // at the same parity and the graph replays unchanged).
    auto capture = [&](auto&& body) {
      cudaGraph_t gr;
      cudaGraphExec_t ex = nullptr;
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      body();
      CK(cudaStreamEndCapture(st, &gr));
      CK(cudaGraphInstantiate(&ex, gr, 0));
      CK(cudaGraphDestroy(gr));
      return ex;
    };
    cudaGraphExec_t g_fwd = nullptr;
    CK(cudaEventRecord(ev0, st));
    for (int64_t seg = 0; seg < nseg; ++seg) {
      const int64_t len = std::min<int64_t>(K, N - seg * K);
      snapshot(ck_f.p + size_t(seg) * fsz);
      if (nslots)
        CK(cudaMemcpyAsync(ck_fp.p + size_t(seg) * ns3, fprev.p, size_t(nslots) * sizeof(Vec4<A>),
                           cudaMemcpyDeviceToDevice, st));
      if (len == K) {
        if (!g_fwd) {
          const int par0 = parity;
          g_fwd = capture([&] {
            for (int64_t i = 0; i < K; ++i) enqueue_runner_step(B, c, d_torque.p, d_counter.p);
          });
          parity = par0;
        }
        CK(cudaGraphLaunch(g_fwd, st));
      } else {
        for (int64_t i = 0; i < len; ++i) enqueue_runner_step(B, c, d_torque.p, d_counter.p);
      }
    }
    CK(cudaEventRecord(ev1, st));
    CK(cudaEventSynchronize(ev1));
    if (g_fwd) CK(cudaGraphExecDestroy(g_fwd));
    check_device_error();
    float fwd_ms = 0.f;
    CK(cudaEventElapsedTime(&fwd_ms, ev0, ev1));
    std::vector<double> tq(static_cast<size_t>(N));
    CK(cudaMemcpy(tq.data(), d_torque.p, size_t(N) * sizeof(double), cudaMemcpyDeviceToHost));
    double J = 0.0;
    for (int64_t nn = ac.window_begin; nn < N; ++nn) J += tq[size_t(nn)];
    const double Tbar = 1.0 / double(N - ac.window_begin);
    J *= Tbar;
    // final state, restored after the backward pass
    DevBuf<S> fin_f;
    DevBuf<Vec4<A>> fin_fp;
    fin_f.alloc(f_alloc.n);
    fin_fp.alloc(ns3);
    CK(cudaMemcpyAsync(fin_f.p, f_alloc.p, f_alloc.n * sizeof(S), cudaMemcpyDeviceToDevice, st));
    if (nslots) CK(cudaMemcpyAsync(fin_fp.p, fprev.p, size_t(nslots) * sizeof(Vec4<A>), cudaMemcpyDeviceToDevice, st));
    const int fin_parity = parity;
    // ---- backward pass ----------------------------------------------------
    // Segments are processed last to first. The recomputation of segment
    // j-1 (engine streams) runs while the backward steps of segment j run on
    // two streams of their own; each side owns one of two segment buffers.
    const size_t nm = size_t(std::max<int64_t>(B.nm, 1));
    struct SegBuf {
      DevBuf<S> f;
      DevBuf<Vec4<A>> F, fp0;
      DevBuf<double> rho, u, mob, du, imp, tb;
    };
    SegBuf sbuf[2];
    for (SegBuf& b : sbuf) {
      b.f.alloc(size_t(K) * fsz);
      b.F.alloc(size_t(K) * ns3);
      b.fp0.alloc(ns3);
      b.rho.alloc(size_t(K) * ns3);
      b.u.alloc(size_t(K) * ns3 * 3);
      b.mob.alloc(size_t(K) * nm);
      b.du.alloc(size_t(K) * nsweep * ns3 * 3);
      b.imp.alloc(size_t(K) * nsweep * nm * 3);
      b.tb.alloc(size_t(K));
    }
    auto save_of = [&](SegBuf& b, int64_t i) {
      IbmSave sv;
      sv.rho = b.rho.p + size_t(i) * ns3;
      sv.u = b.u.p + size_t(i) * ns3 * 3;
      sv.mob = b.mob.p + size_t(i) * nm;
      sv.du = b.du.p + size_t(i) * nsweep * ns3 * 3;
      sv.imp = b.imp.p + size_t(i) * nsweep * nm * 3;
      sv.ns3 = ns3;
      sv.nm = nm;
      return sv;
    };
    DevBuf<A> lam0, lam1;
    lam0.alloc(fsz);
    lam1.alloc(fsz);
    CK(cudaMemsetAsync(lam0.p, 0, fsz * sizeof(A), st));
    CK(cudaMemsetAsync(lam1.p, 0, fsz * sizeof(A), st));
    DevBuf<double> mu0, mu1, Fbar, dubar, ubar, rhobar, cksbar, umbar, tbar, mobbar, xbar, grad;
    for (DevBuf<double>* b : {&mu0, &mu1, &Fbar, &dubar, &ubar}) {
      b->alloc(3 * ns3);
      CK(cudaMemsetAsync(b->p, 0, 3 * ns3 * sizeof(double), st));
    }
    for (DevBuf<double>* b : {&rhobar, &cksbar}) {
      b->alloc(ns3);
      CK(cudaMemsetAsync(b->p, 0, ns3 * sizeof(double), st));
    }
    for (DevBuf<double>* b : {&umbar, &tbar, &xbar}) {
      b->alloc(3 * nm);
      CK(cudaMemsetAsync(b->p, 0, 3 * nm * sizeof(double), st));
    }
    mobbar.alloc(nm);
    CK(cudaMemsetAsync(mobbar.p, 0, nm * sizeof(double), st));
    grad.alloc(3);
    CK(cudaMemsetAsync(grad.p, 0, 3 * sizeof(double), st));
    DevBuf<double> dummy_t;
    DevBuf<int64_t> dummy_c;
    dummy_t.alloc(size_t(K) + 1);
    dummy_c.alloc(1);
    CK(cudaStreamSynchronize(st));
    cudaStream_t sb = nullptr, sb2 = nullptr;
    cudaEvent_t e_fork = nullptr, e_join = nullptr, e_rec[2] = {nullptr, nullptr}, e_bwd[2] = {nullptr, nullptr};
    CK(cudaStreamCreateWithFlags(&sb, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&sb2, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&e_fork, &e_join, &e_rec[0], &e_rec[1], &e_bwd[0], &e_bwd[1]})
      CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    struct Cleanup {
      std::vector<cudaStream_t> ss;
      std::vector<cudaEvent_t> es;
      std::vector<cudaGraphExec_t> gs;
      ~Cleanup() {
        for (auto x : ss) cudaStreamSynchronize(x);
        for (auto g : gs)
          if (g) cudaGraphExecDestroy(g);
        for (auto e : es) cudaEventDestroy(e);
        for (auto x : ss) cudaStreamDestroy(x);
      }
    } cleanup;
    cleanup.ss = {sb, sb2};
    cleanup.es = {e_fork, e_join, e_rec[0], e_rec[1], e_bwd[0], e_bwd[1]};
    const IbmArgs a0 = ibm_args(B, c);
    const unsigned gs = unsigned(std::max<int64_t>(1, ceil_div(B.ns, IBM_BLOCK)));
    const unsigned gm = unsigned(std::max<int64_t>(1, ceil_div(B.nm, IBM_BLOCK)));
    const unsigned gc = unsigned(ceil_div(n, ADJ_BLOCK));
    // recomputation of len steps from the restored checkpoint into b
    auto recompute = [&](SegBuf& b, int64_t len) {
      CK(cudaMemsetAsync(dummy_c.p, 0, sizeof(int64_t), st));
      for (int64_t i = 0; i < len; ++i) {
        snapshot(b.f.p + size_t(i) * fsz);
        const IbmSave sv = save_of(b, i);
        enqueue_runner_step(B, c, dummy_t.p, dummy_c.p, &sv);
        if (nslots)
          CK(cudaMemcpyAsync(b.F.p + size_t(i) * ns3, fcur.p, size_t(nslots) * sizeof(Vec4<A>),
                             cudaMemcpyDeviceToDevice, st));
      }
    };
    // backward steps of a segment of len steps held in b (stream sb)
    auto backward = [&](SegBuf& b, int64_t len) {
      for (int64_t i = len - 1; i >= 0; --i) {
        const S* fn = b.f.p + size_t(i) * fsz;
        const bool even = ((len - 1 - i) & 1) == 0;
        A* lam_in = even ? lam0.p : lam1.p;
        A* lam_out = even ? lam1.p : lam0.p;
        double* mu_in = even ? mu0.p : mu1.p;
        double* mu_out = even ? mu1.p : mu0.p;
        AdjCollide<S> pc;
        pc.f = fn;
        pc.pl = plane;
        pc.flags = flags.p;
        pc.nbr = nbr.p;
        pc.wall_u = wall_u.p;
        pc.fslot = fslot.p;
        pc.F = b.F.p + size_t(i) * ns3;
        pc.Fp = i > 0 ? b.F.p + size_t(i - 1) * ns3 : b.fp0.p;
        pc.lam_in = lam_in;
        pc.lam_out = lam_out;
        pc.mu_in = mu_in;
        pc.mu_out = mu_out;
        pc.Fbar = Fbar.p;
        pc.grad = grad.p;
        pc.nx = nx;
        pc.ny = ny;
        pc.nz = nz;
        pc.op = omega_p;
        pc.om = omega_m;
        adj_collide_kernel<Q, S><<<gc, ADJ_BLOCK, 0, sb>>>(pc, n);
        CK(cudaGetLastError());
        const IbmSave sv = save_of(b, i);
        AdjIbm ab;
        ab.a = a0;
        ab.a.rho = sv.rho;
        ab.a.u_now = sv.u;
        ab.a.mob = sv.mob;
        ab.imp_k = sv.imp;
        ab.du_k = sv.du;
        ab.nslot = int64_t(ns3);
        ab.slot_cell = slot_cell.p;
        ab.nx = nx;
        ab.ny = ny;
        ab.radius = c.kernel_radius;
        ab.Fbar = Fbar.p;
        ab.dubar = dubar.p;
        ab.ubar = ubar.p;
        ab.rhobar = rhobar.p;
        ab.cksbar = cksbar.p;
        ab.umbar = umbar.p;
        ab.tbar = tbar.p;
        ab.mobbar = mobbar.p;
        ab.xbar = xbar.p;
        ab.grad = grad.p;
        ab.tbar_step = b.tb.p + i;
        for (int k = nsweep - 1; k >= 0; --k) {
          adj_ibm_marker_kernel<<<gm, ADJ_BLOCK, 0, sb>>>(ab, k);
          adj_ibm_slot_kernel<<<gs, ADJ_BLOCK, 0, sb>>>(ab, k);
        }
        adj_ibm_mob_slot_kernel<<<gs, ADJ_BLOCK, 0, sb>>>(ab);
        adj_ibm_mob_marker_kernel<<<gm, ADJ_BLOCK, 0, sb>>>(ab);
        adj_ibm_fbar_kernel<Q, A><<<gs, ADJ_BLOCK, 0, sb>>>(ab, lam_out, plane);
        CK(cudaGetLastError());
      }
    };
    auto capture_on = [&](cudaStream_t s0, auto&& body) {
      cudaGraph_t gr;
      cudaGraphExec_t ex = nullptr;
      CK(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
      body();
      CK(cudaStreamEndCapture(s0, &gr));
      CK(cudaGraphInstantiate(&ex, gr, 0));
      CK(cudaGraphDestroy(gr));
      return ex;
    };
    cudaGraphExec_t g_rec[2] = {nullptr, nullptr}, g_bwd[2] = {nullptr, nullptr};
    std::vector<double> tbh(static_cast<size_t>(nseg * K), 0.0);
    for (int64_t t = ac.window_begin; t < N; ++t) tbh[size_t(t)] = Tbar;
    bool used[2] = {false, false};
    // stage segment seg into buffer bi on the engine streams
    auto stage = [&](int64_t seg, int bi) {
      SegBuf& b = sbuf[bi];
      const int64_t len = std::min<int64_t>(K, N - seg * K);
      if (used[bi]) CK(cudaStreamWaitEvent(st, e_bwd[bi], 0));
      CK(cudaMemcpyAsync(fp, ck_f.p + size_t(seg) * fsz, fsz * sizeof(S), cudaMemcpyDeviceToDevice, st));
      if (nslots) {
        CK(cudaMemcpyAsync(fprev.p, ck_fp.p + size_t(seg) * ns3, size_t(nslots) * sizeof(Vec4<A>),
                           cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(b.fp0.p, ck_fp.p + size_t(seg) * ns3, size_t(nslots) * sizeof(Vec4<A>),
                           cudaMemcpyDeviceToDevice, st));
      }
      CK(cudaMemcpyAsync(b.tb.p, tbh.data() + size_t(seg * K), size_t(len) * sizeof(double),
                         cudaMemcpyHostToDevice, st));
      parity = 0;
      field_present = true;
      fprev_stale = false;
      if (len == K) {
        if (!g_rec[bi]) {
          g_rec[bi] = capture_on(st, [&] { recompute(b, K); });
          cleanup.gs.push_back(g_rec[bi]);
        }
        CK(cudaGraphLaunch(g_rec[bi], st));
        parity = 0;
      } else {
        recompute(b, len);
      }
      CK(cudaEventRecord(e_rec[bi], st));
      used[bi] = true;
    };
    bool lam_in_is_0 = true;
    auto run_back = [&](int64_t seg, int bi) {
      SegBuf& b = sbuf[bi];
      const int64_t len = std::min<int64_t>(K, N - seg * K);
      CK(cudaStreamWaitEvent(sb, e_rec[bi], 0));
      if (!lam_in_is_0) {
        CK(cudaMemcpyAsync(lam0.p, lam1.p, fsz * sizeof(A), cudaMemcpyDeviceToDevice, sb));
        CK(cudaMemcpyAsync(mu0.p, mu1.p, 3 * ns3 * sizeof(double), cudaMemcpyDeviceToDevice, sb));
        lam_in_is_0 = true;
      }
      if (len == K) {
        if (!g_bwd[bi]) {
          g_bwd[bi] = capture_on(sb, [&] { backward(b, K); });
          cleanup.gs.push_back(g_bwd[bi]);
        }
        CK(cudaGraphLaunch(g_bwd[bi], sb));
      } else {
        backward(b, len);
        if (len & 1) lam_in_is_0 = false;
      }
      CK(cudaEventRecord(e_bwd[bi], sb));
    };
    CK(cudaEventRecord(ev0, st));
    stage(nseg - 1, int((nseg - 1) & 1));
    for (int64_t seg = nseg - 1; seg >= 0; --seg) {
      if (seg - 1 >= 0) stage(seg - 1, int((seg - 1) & 1));
      run_back(seg, int(seg & 1));
    }
    CK(cudaStreamWaitEvent(st, e_bwd[0], 0));
    CK(cudaStreamWaitEvent(st, e_bwd[1], 0));
    CK(cudaEventRecord(ev1, st));
    CK(cudaEventSynchronize(ev1));
    check_device_error();
    float adj_ms = 0.f;
    CK(cudaEventElapsedTime(&adj_ms, ev0, ev1));
    double gh[3];
    CK(cudaMemcpy(gh, grad.p, 3 * sizeof(double), cudaMemcpyDeviceToHost));
    if (dJ_dpos && B.nm)
      CK(cudaMemcpy(dJ_dpos, xbar.p, size_t(B.nm) * 3 * sizeof(double), cudaMemcpyDeviceToHost));
    if (torque_out) std::copy(tq.begin(), tq.end(), torque_out);
    // restore the state at the end of the forward run
    CK(cudaMemcpyAsync(f_alloc.p, fin_f.p, f_alloc.n * sizeof(S), cudaMemcpyDeviceToDevice, st));
    if (nslots) CK(cudaMemcpyAsync(fprev.p, fin_fp.p, size_t(nslots) * sizeof(Vec4<A>), cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    parity = fin_parity;
    field_present = true;
    fprev_stale = false;
    invalidate_graphs();
    time += uint64_t(N);
    // d omega / d nu (params.rs:205-217): omega+ = 1/(3 nu + 1/2),
    // omega- = 1/(magic/(3 nu) + 1/2) for TRT, = omega+ for BGK
    const double nu = cfg.nu;
    const double dwp = -3.0 * omega_p * omega_p;
    const double dwm = cfg.collision == LBMB_TRT ? omega_m * omega_m * cfg.magic / (3.0 * nu * nu) : dwp;
    if (out) {
      out->J = J;
      out->dJ_domega_plus = gh[0];
      out->dJ_domega_minus = gh[1];
      out->dJ_dnu = gh[0] * dwp + gh[1] * dwm;
      out->dJ_domega_z = gh[2];
      out->forward_ms = fwd_ms;
      out->adjoint_ms = adj_ms;
      out->markers = B.nm;
    }
  }

  int64_t solid_count() const {
    int64_t s = 0;
    for (auto v : solid_h) s += v ? 1 : 0;
    return s;
  }

  void fill_nan(double* p, int64_t k) {
    std::vector<double> h(size_t(k), std::nan(""));
    CK(cudaMemcpyAsync(p, h.data(), size_t(k) * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
  }
};

// ---------------------------------------------------------------------------
// Batch of engines of one (lattice, storage) type, advanced in lockstep with
// one launch per kernel family per step (batch.cuh). The engines keep their
// own device state and must outlive the batch.
// ---------------------------------------------------------------------------
template <int Q, class S>
struct Batch final : BatchBase {
  using E = Engine<Q, S>;
  std::vector<E*> eng;
  std::vector<BodyState*> bod;
  lbmb_ibm_config cfg;
  int ncase = 0;
  int parity = 0;
  int minb[2] = {8, 8};
  cudaStream_t st = nullptr, st2 = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_fork = nullptr, ev_join = nullptr;
  std::vector<BatchCase> cases_h;
  DevBuf<BatchCase> cases;
  DevBuf<int32_t> off_cells, off_bslots, off_slots, off_markers;
  int nb_cells = 0, nb_bslots = 0, nb_slots = 0, nb_markers = 0;
  DevBuf<double> d_torque;
  DevBuf<int64_t> d_counter;

  Batch(const std::vector<EngineBase*>& all, const int32_t* bodies, const lbmb_ibm_config& c) : cfg(c) {
    if (all.empty()) invalid("batch needs at least one solver");
    for (EngineBase* b : all) {
      E* e = dynamic_cast<E*>(b);
      if (!e) invalid("batch solvers must share lattice and storage precision");
      if (!e->lean_ok(e->coll))
        throw Error(LBMB_ERR_UNSUPPORTED, "batch solvers need TRT/BGK, fp32/fp16/bf16 storage, no uniform force");
      if (!e->scalars.empty()) throw Error(LBMB_ERR_UNSUPPORTED, "batch solvers carry no scalar distributions");
      if (e->omega_on) throw Error(LBMB_ERR_UNSUPPORTED, "batch solvers carry no relaxation field");
      eng.push_back(e);
    }
    ncase = int(eng.size());
    parity = eng[0]->parity;
    for (E* e : eng) {
      if (e->parity != parity) invalid("batch solvers must be at the same step parity");
      if (e->cfg.device != eng[0]->cfg.device) invalid("batch solvers must live on one device");
    }
    CK(cudaSetDevice(eng[0]->cfg.device));
    for (int k = 0; k < ncase; ++k) {
      eng[k]->sync();
      bod.push_back(&eng[k]->body_for(bodies ? bodies[k] : 0, cfg));
    }
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int lo = 0, hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CK(cudaStreamCreateWithPriority(&st2, cudaStreamNonBlocking, hi));
    CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    std::vector<int32_t> oc(1, 0), ob(1, 0), os(1, 0), om(1, 0);
    for (int k = 0; k < ncase; ++k) {
      E* e = eng[k];
      BodyState& B = *bod[k];
      oc.push_back(oc.back() + int32_t(ceil_div(e->n, BATCH_BLOCK)));
      ob.push_back(ob.back() + int32_t(std::max<int64_t>(1, ceil_div(B.ns, BATCH_BLOCK))));
      os.push_back(os.back() + int32_t(std::max<int64_t>(1, ceil_div(e->nslots, BATCH_BLOCK))));
      om.push_back(om.back() + int32_t(std::max<int64_t>(1, ceil_div(B.nm, BATCH_BLOCK))));
    }
    nb_cells = oc.back();
    nb_bslots = ob.back();
    nb_slots = os.back();
    nb_markers = om.back();
    off_cells.upload(oc, st);
    off_bslots.upload(ob, st);
    off_slots.upload(os, st);
    off_markers.upload(om, st);
    cases_h.resize(size_t(ncase));
    for (int k = 0; k < ncase; ++k) {
      E* e = eng[k];
      BatchCase& b = cases_h[size_t(k)];
      b.hp = e->hydro_params();
      b.n = uint32_t(e->n);
      b.nx = e->nx;
      b.ny = e->ny;
      b.nz = e->nz;
      b.slot_cell = e->slot_cell.p;
      b.nslots = e->nslots;
      b.fcur = e->fcur.p;
      b.fprev = e->fprev.p;
      b.ibm = e->ibm_args(*bod[size_t(k)], cfg);
      b.gx = b.gy = b.gz = 0.0;
      b.series_torque = nullptr;
      b.counter = nullptr;
    }
    cases.upload(cases_h, st);
    CK(cudaStreamSynchronize(st));
  }

  ~Batch() override {
    if (st) cudaStreamSynchronize(st);
    if (st2) cudaStreamSynchronize(st2);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (st) cudaStreamDestroy(st);
    if (st2) cudaStreamDestroy(st2);
  }

  template <bool ODD, int MB>
  void hydro_mb() {
    batch_hydro_kernel<Q, S, ODD, MB><<<unsigned(nb_cells), BATCH_BLOCK, 0, st>>>(cases.p, off_cells.p, ncase);
  }
  template <bool ODD>
  void hydro_par() {
    switch (minb[ODD]) {
      case 6: hydro_mb<ODD, 6>(); break;
      case 7: hydro_mb<ODD, 7>(); break;
      default: hydro_mb<ODD, 8>(); break;
    }
  }
  void hydro(int par) {
    if (par) hydro_par<true>();
    else hydro_par<false>();
    CK(cudaGetLastError());
  }

  // One runner step of every case (runner.rs:1079-1129 per case).
  void one_step() {
    CK(cudaEventRecord(ev_fork, st));
    CK(cudaStreamWaitEvent(st2, ev_fork, 0));
    batch_prep_kernel<Q, S><<<unsigned(nb_bslots), BATCH_BLOCK, 0, st2>>>(cases.p, off_bslots.p, ncase, parity);
    for (int s = 0; s < cfg.max_iterations; ++s) {
      batch_interp_kernel<<<unsigned(nb_markers), BATCH_BLOCK, 0, st2>>>(cases.p, off_markers.p, ncase, s);
      batch_spread_kernel<<<unsigned(nb_bslots), BATCH_BLOCK, 0, st2>>>(cases.p, off_bslots.p, ncase);
      batch_diag_kernel<<<unsigned(nb_markers), BATCH_BLOCK, 0, st2>>>(cases.p, off_markers.p, off_bslots.p, ncase,
                                                                         s);
    }
    batch_commit_kernel<<<unsigned(nb_bslots), BATCH_BLOCK, 0, st2>>>(cases.p, off_bslots.p, ncase);
    if (parity) batch_cells_kernel<Q, S, true><<<unsigned(nb_slots), BATCH_BLOCK, 0, st2>>>(cases.p, off_slots.p, ncase);
    else batch_cells_kernel<Q, S, false><<<unsigned(nb_slots), BATCH_BLOCK, 0, st2>>>(cases.p, off_slots.p, ncase);
    CK(cudaGetLastError());
    hydro(parity);
    CK(cudaEventRecord(ev_join, st2));
    CK(cudaStreamWaitEvent(st, ev_join, 0));
    batch_fprev_kernel<<<unsigned(nb_slots), BATCH_BLOCK, 0, st>>>(cases.p, off_slots.p, ncase);
    CK(cudaGetLastError());
    parity ^= 1;
  }

  void run(int64_t steps, double* torque, double* device_ms) override {
    if (steps < 0) invalid("steps must be >= 0");
    for (E* e : eng) e->sync();
    d_torque.alloc(size_t(std::max<int64_t>(1, steps)) * size_t(ncase));
    d_counter.alloc(size_t(ncase));
    CK(cudaMemsetAsync(d_counter.p, 0, size_t(ncase) * sizeof(int64_t), st));
    for (int k = 0; k < ncase; ++k) {
      cases_h[size_t(k)].series_torque = d_torque.p + size_t(k) * size_t(std::max<int64_t>(1, steps));
      cases_h[size_t(k)].counter = d_counter.p + k;
    }
    cases.upload(cases_h, st);
    CK(cudaEventRecord(ev0, st));
    const int64_t G = 16;
    int64_t done = 0;
    if (parity != 0 && steps > 0) {
      one_step();
      ++done;
    }
    cudaGraphExec_t exec = nullptr;
    while (steps - done >= G) {
      if (!exec) {
        cudaGraph_t g;
        const int par0 = parity;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int64_t i = 0; i < G; ++i) one_step();
        CK(cudaStreamEndCapture(st, &g));
        CK(cudaGraphInstantiate(&exec, g, 0));
        CK(cudaGraphDestroy(g));
        parity = par0;
      }
      CK(cudaGraphLaunch(exec, st));
      done += G;
    }
    if (exec) CK(cudaGraphExecDestroy(exec));
    for (; done < steps; ++done) one_step();
    CK(cudaEventRecord(ev1, st));
    CK(cudaEventSynchronize(ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    if (device_ms) *device_ms = ms;
    if (torque && steps > 0)
      CK(cudaMemcpy(torque, d_torque.p, size_t(steps) * size_t(ncase) * sizeof(double), cudaMemcpyDeviceToHost));
    for (E* e : eng) {
      e->check_device_error();
      e->parity = parity;
      e->field_present = true;
      e->fprev_stale = false;
      e->invalidate_graphs();
      e->time += uint64_t(steps);
    }
  }

  // Times the batched sweep under every register budget on the cases' own
  // grids (populations saved and restored) and keeps the fastest.
  void autotune(int steps, int32_t* even, int32_t* odd, double* best_ms) override {
    if (steps < 2) invalid("autotune: steps per trial must be >= 2");
    steps += steps & 1;
    for (E* e : eng) e->sync();
    std::vector<std::unique_ptr<DevBuf<S>>> save;
    for (E* e : eng) {
      save.emplace_back(new DevBuf<S>());
      save.back()->alloc(e->f_alloc.n);
      CK(cudaMemcpyAsync(save.back()->p, e->f_alloc.p, e->f_alloc.n * sizeof(S), cudaMemcpyDeviceToDevice, st));
    }
    double bms = 0.0;
    int be = 8, bo = 8;
    for (int ev = 8; ev >= 6; --ev)
      for (int od = 8; od >= 6; --od) {
        minb[0] = ev;
        minb[1] = od;
        hydro(0);
        hydro(1);
        CK(cudaEventRecord(ev0, st));
        for (int i = 0; i < steps; ++i) hydro(i & 1);
        CK(cudaEventRecord(ev1, st));
        CK(cudaEventSynchronize(ev1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev0, ev1));
        const double t = double(ms) / steps;
        if (bms == 0.0 || t < bms) {
          bms = t;
          be = ev;
          bo = od;
        }
      }
    minb[0] = be;
    minb[1] = bo;
    for (size_t k = 0; k < eng.size(); ++k)
      CK(cudaMemcpyAsync(eng[k]->f_alloc.p, save[k]->p, eng[k]->f_alloc.n * sizeof(S), cudaMemcpyDeviceToDevice,
                         st));
    CK(cudaStreamSynchronize(st));
    if (even) *even = be;
    if (odd) *odd = bo;
    if (best_ms) *best_ms = bms;
  }
};

template <int Q, class S>
BatchBase* Engine<Q, S>::make_batch(const std::vector<EngineBase*>& all, const int32_t* bodies,
                                    const lbmb_ibm_config& c) {
  if constexpr (std::is_same<typename Codec<S>::A, float>::value) {
    return new Batch<Q, S>(all, bodies, c);
  } else {
    throw Error(LBMB_ERR_UNSUPPORTED, "batch runs need fp32/fp16/bf16 population storage");
  }
}

// Factories, one per translation unit (engine_q*_*.cu).
EngineBase* make_engine_q19_f32(const lbmb_config&, const uint8_t*, const double*);
EngineBase* make_engine_q19_f16(const lbmb_config&, const uint8_t*, const double*);
EngineBase* make_engine_q19_bf16(const lbmb_config&, const uint8_t*, const double*);
EngineBase* make_engine_q19_f64(const lbmb_config&, const uint8_t*, const double*);
EngineBase* make_engine_q27_f32(const lbmb_config&, const uint8_t*, const double*);
EngineBase* make_engine_q27_f16(const lbmb_config&, const uint8_t*, const double*);
EngineBase* make_engine_q27_bf16(const lbmb_config&, const uint8_t*, const double*);
EngineBase* make_engine_q27_f64(const lbmb_config&, const uint8_t*, const double*);

}  // namespace lbmb
