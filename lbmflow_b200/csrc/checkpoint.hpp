// Checkpoint/restart files in the reference's v3 format (host side).
//
// Layout (crates/lbm-core/src/solver.rs:29-44, 1108-1215, 4536-4724):
//   <dir>/manifest.json               pretty JSON CheckpointManifest
//   <dir>/rank_0000_part_0000.bin     one rank file per part
// rank file = "LBMKPT\0\0" | u32 format_version = 3 | u8 endian = 0 |
//   u8 dtype (0 f32, 1 f64) | u16 lattice id (319 / 327) | u16 Q | u16 D |
//   u64 n_padded | u64 n_core | u32 section count |
//   count x (u32 id, u64 offset, u64 byte_len) | payload | u64 fnv1a64(payload)
// all little-endian. Sections: 1 F_PRIMARY (Q planes over the halo-padded
// box, deviation form), 2 STALE_STASH (the ping-pong partner), 3 MOMENTS
// (rho, ux, uy, uz compact), 4 SOLID (padded u8), 5 FORCE_FIELD (compact
// x,y,z per cell), 6 SCALAR_FIELDS, 7 PHASE_FIELD, 10 QOI_ACCUMULATORS
// (JSON).
//
// This writer is the single-part, single-rank case the stirred-tank run
// uses (Solver::save, solver.rs:4715-4724). Halo cells of the padded planes
// are written as zero and the stale stash as all-zero planes: the
// reference's halo exchange rewrites every halo population streaming reads
// before it is read, and with every non-periodic face a solid rim streaming
// writes every stash slot of a fluid cell before the swap, so neither
// carries state into the next step.
#pragma once
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lbmb.h"

namespace lbmb {
namespace ckpt {

// CheckpointError (solver.rs:46-82): a stable machine code and a message.
struct Failure : std::runtime_error {
  std::string code;
  Failure(const std::string& c, const std::string& m) : std::runtime_error(c + ": " + m), code(c) {}
};

// The GlobalSpec fields that enter the scenario hash (solver.rs:881-945)
// plus the run's arithmetic type. All faces are closed; no localized
// sources or face patches exist on this path.
struct Spec {
  int q = 19;         // 19 or 27 (D = 3)
  int collision = 1;  // 0 BGK, 1 TRT, 2 central moment
  bool f64 = true;    // run dtype "f64" (else "f32")
  int dims[3] = {0, 0, 0};
  bool periodic[3] = {false, false, false};
  double nu = 0.0, magic = 0.0, omega_shear = 0.0;
  double force[3] = {0.0, 0.0, 0.0};
};

struct Scalar {
  std::string name;
  double diffusivity = 0.0;
  int q = 0;                  // scalar lattice (7 or the hydro Q)
  std::vector<double> h;      // q x n compact, ordinary (not deviation) form
  std::vector<double> conc;   // n
};

// Solver state carried by a checkpoint, compact (halo-free) arrays.
struct State {
  uint64_t step = 0;
  std::vector<double> f;        // Q x n, deviation form, logical post-stream
  std::vector<double> moments;  // 4 x n: rho, ux, uy, uz
  bool has_force_field = false;
  std::vector<double> force_field;  // n x 3
  std::vector<Scalar> scalars;
  bool has_qoi = false;
  std::string qoi_json;  // QoiCheckpointState, carried opaque
};

uint64_t fnv1a64(const void* data, size_t len, uint64_t h = 0xcbf29ce484222325ull);
uint64_t spec_hash(const Spec& s);
uint64_t decomp_hash(const Spec& s);
uint64_t mask_hash(const Spec& s, const uint8_t* solid, const double* wall_u);
std::string hash_string(uint64_t h);

// A run of payload bytes: data, or (data == nullptr) len zero bytes.
struct Piece {
  const char* data;
  uint64_t len;
};
struct SectionOut {
  uint32_t id;
  std::vector<Piece> pieces;
};
// Section ids (solver.rs:31-44).
constexpr uint32_t SEC_F_PRIMARY = 1, SEC_STALE_STASH = 2, SEC_MOMENTS = 3, SEC_SOLID = 4, SEC_FORCE_FIELD = 5,
                   SEC_SCALAR_FIELDS = 6, SEC_PHASE_FIELD = 7, SEC_QOI_ACCUMULATORS = 10;

// A scalar entry as read: h points at q padded planes, conc at n values,
// both in the file's dtype.
struct ScalarView {
  std::string name;
  double diffusivity = 0.0;
  int q = 0;
  const char* h = nullptr;
  const char* conc = nullptr;
};
// A read-only mapping of a rank file.
struct Mapping {
  const char* p = nullptr;
  size_t n = 0;
  Mapping() = default;
  Mapping(const Mapping&) = delete;
  Mapping& operator=(const Mapping&) = delete;
  ~Mapping();
};
// A validated checkpoint in memory: pointers into the mapped rank file,
// which `hold` keeps mapped.
struct View {
  std::shared_ptr<const Mapping> hold;
  uint64_t step = 0;
  const char* f = nullptr;            // Q padded planes, file dtype
  const char* moments = nullptr;      // 4 x n, file dtype
  const char* force_field = nullptr;  // n x 3, file dtype, or null
  std::vector<ScalarView> scalars;
  bool has_qoi = false;
  std::string qoi_json;
};

uint64_t padded_cells(const Spec& s);
// The SOLID section: the padded mask after the mask exchange, one byte per
// padded cell.
std::string solid_section(const Spec& s, const uint8_t* solid);
// hash of `len` zero bytes continuing h
uint64_t fnv1a64_zeros(uint64_t len, uint64_t h);
void append_reals(std::string& out, const double* v, size_t count, bool f64);
void reals_to_double(const char* p, size_t count, bool f64, double* out);
void unpad_to_double(const char* img, const Spec& s, int planes, double* out);
std::string scalar_head(const std::string& name, double diffusivity, uint64_t h_len);
std::vector<Piece> scalar_tail(int q, int64_t np, int64_t nc, uint64_t w);

// The rank file (header, section table, payload pieces, hash trailer) and
// the manifest; the payload is hashed while a second thread writes it.
void write(const std::string& dir, const Spec& s, uint64_t step, const std::vector<SectionOut>& secs,
           const uint8_t* solid, const double* wall_u, bool stats);

// Every check of the reference's restore, in its order and with its codes,
// on the mapped rank file.
View read(const std::string& dir, const Spec& s, const uint8_t* solid, const double* wall_u);

// Whether the text is one JSON object (the QOI accumulator section).
bool json_object(const std::string& text);

// Solver::save for one part: writes manifest.json and the rank file.
// solid: n bytes or null (all fluid); wall_u: n x 3 or null (zero).
void save(const std::string& dir, const Spec& s, const uint8_t* solid, const double* wall_u, const State& st);

// Solver::restore / load_into (solver.rs:4739-5066): every check runs before
// anything is returned, in the reference's order and with its codes.
State load(const std::string& dir, const Spec& s, const uint8_t* solid, const double* wall_u);

// The checkpoint Spec of a solver configuration: dtype "f64" for F64
// storage, "f32" for F32 / F16 / BF16 storage.
Spec spec_of(const lbmb_config& c);

}  // namespace ckpt
}  // namespace lbmb
