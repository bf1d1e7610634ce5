// Staged two-cells-per-thread AA collide-stream (TRT / BGK, no uniform body
// force, fp32 | fp16 | bf16 storage, even nx).
//
// The 16-bit sweeps move 2 bytes per population, so a one-cell-per-thread
// kernel issues as many instructions per byte as it moves data: element
// loads and stores, one conversion per element and the scalar collision
// fill the issue slots before HBM is busy. This kernel spends them on two
// cells at a time and takes the loads off the threads:
//
//  * one producer warp per block streams tiles of STG_CELLS consecutive
//    cells into a ring of STAGES shared-memory buffers with bulk
//    asynchronous copies (cp.async.bulk, completion on an mbarrier): one
//    16-byte-aligned window per direction (the tile kernel's windows: plane
//    q at the tile on the even step, plane opp(q) shifted by -d_q and
//    rounded down to 16 bytes on the odd step) plus the tile's flag bytes;
//  * STG_WARPS consumer warps each own 64 cells of a tile, two x-adjacent
//    cells per thread: 4-byte shared loads of both cells' populations where
//    the window pair is aligned, the packed float2 TRT collision of
//    hydro_pair.cuh (FADD2 / FMUL2 / FFMA2), one conversion per two stored
//    elements and 4-byte global stores wherever the destination pair is
//    aligned (every direction on the even step, c_x = 0 on the odd step);
//  * full / empty mbarriers per stage replace block-wide barriers, so each
//    consumer warp moves on as soon as its tile has landed.
//
// The bytes in flight per SM are bounded by the shared-memory ring (several
// tiles ahead), not by registers. By the AA ownership rule every element a
// cell uses from a window is written in this step by that cell alone, so a
// prefetched window is never stale. Cells with a solid neighbour read the
// directions coming off a wall from their own slot (global load) on the odd
// step and write the bounced populations to their own slots; cells on a
// periodic face, under the free-slip top or next to a moving wall take the
// generic path; IBM-forced cells are left to hydro_cells_kernel.
//
// Every mbarrier wait is bounded (wait_limit cycles): a wait that runs out
// sets the device error flag; the producer then waits (bounded) for the
// copies it has issued and every warp leaves. wait_limit < 0 runs the
// timeout self-test (a wait on a barrier nothing arrives at) and touches no
// population.
#pragma once
#include "hydro_pair.cuh"
#include "hydro_tile.cuh"
#include "hydro_tma.cuh"

namespace lbmb {

// Seven consumer warps and the producer make 8-warp blocks: two resident
// blocks put four warps on each SM sub-partition (128 registers a thread),
// three put six (80 registers).
constexpr int STG_WARPS = 7;
constexpr int STG_CELLS = 2 * 32 * STG_WARPS;  // 448 cells per tile
constexpr int STG_THREADS = STG_WARPS * 32 + 32;
static_assert(STG_CELLS % 16 == 0, "tile starts on a 16-byte boundary of the flag and 2-byte population arrays");

template <int Q, class S>
struct StgLayout {
  static constexpr int E = 16 / int(sizeof(S));             // elements per 16 bytes
  static constexpr int LEN = STG_CELLS + E;                 // window elements (odd step)
  static constexpr size_t WIN_BYTES = size_t(LEN) * sizeof(S);
  static constexpr size_t EVEN_BYTES = size_t(STG_CELLS) * sizeof(S);
  static constexpr size_t STAGE_BYTES = Q * WIN_BYTES + STG_CELLS;  // windows + flags
  static_assert(WIN_BYTES % 16 == 0 && STAGE_BYTES % 16 == 0, "bulk copies need 16-byte multiples");
};

template <int Q, class S, int STAGES>
constexpr size_t staged_smem_bytes() {
  return size_t(STAGES) * StgLayout<Q, S>::STAGE_BYTES + (2 * STAGES + 1) * sizeof(uint64_t);
}

// TRT collision of two cells in float2 lanes in register-lean form: the
// operator of trt_pair_collide (hydro_pair.cuh), with the pair sums
// S = f_a + f_b and differences D = f_a - f_b recomputed where they are used
// instead of being held for all pairs (the form of trt_lean_collide).
template <int Q>
__device__ __forceinline__ void trt_pair_lean(float2 (&f)[Q], const HydroParams<float>& p) {
  using L = Lat<Q>;
  constexpr int NP = (Q - 1) / 2;
  static_assert(pair_heads_positive<Q>(), "pair head convention");
  float2 drho = f[0], jx = bc2(0.f), jy = bc2(0.f), jz = bc2(0.f);
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int a = 2 * k + 1, b = a + 1;
    drho = add2(drho, add2(f[a], f[b]));
    const float2 d = sub2(f[a], f[b]);
    if (L::cx(a) == 1) jx = add2(jx, d);
    if (L::cx(a) == -1) jx = sub2(jx, d);
    if (L::cy(a) == 1) jy = add2(jy, d);
    if (L::cy(a) == -1) jy = sub2(jy, d);
    if (L::cz(a) == 1) jz = add2(jz, d);
    if (L::cz(a) == -1) jz = sub2(jz, d);
  }
  const float2 rho = add2(drho, bc2(1.f));
  const float2 inv = make_float2(rcp_fast(rho.x), rcp_fast(rho.y));
  const float2 ux = mul2(jx, inv), uy = mul2(jy, inv), uz = mul2(jz, inv);
  const float2 usq = fma2(ux, ux, fma2(uy, uy, mul2(uz, uz)));
  float2 op = bc2(p.omega_p), om = bc2(p.omega_m);
  if (p.les_c > 0.f) {
    // second moments of the pair sums, both lanes at once
    float2 s6[6] = {bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f)};
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int a = 2 * k + 1;
      const int cx = L::cx(a), cy = L::cy(a), cz = L::cz(a);
      const float2 sv = add2(f[a], f[a + 1]);
      if (cx) s6[0] = add2(s6[0], sv);
      if (cy) s6[1] = add2(s6[1], sv);
      if (cz) s6[2] = add2(s6[2], sv);
      if (cx && cy) s6[3] = cx * cy > 0 ? add2(s6[3], sv) : sub2(s6[3], sv);
      if (cx && cz) s6[4] = cx * cz > 0 ? add2(s6[4], sv) : sub2(s6[4], sv);
      if (cy && cz) s6[5] = cy * cz > 0 ? add2(s6[5], sv) : sub2(s6[5], sv);
    }
    const float sa[6] = {s6[0].x, s6[1].x, s6[2].x, s6[3].x, s6[4].x, s6[5].x};
    const float sb[6] = {s6[0].y, s6[1].y, s6[2].y, s6[3].y, s6[4].y, s6[5].y};
    const float te0 = les_tau_pair<Q>(sa, rho.x, inv.x, ux.x, uy.x, uz.x, p.les_c, p.tau0);
    const float te1 = les_tau_pair<Q>(sb, rho.y, inv.y, ux.y, uy.y, uz.y, p.les_c, p.tau0);
    op = make_float2(rcp_fast(te0), rcp_fast(te1));
    if (p.magic > 0.f) {
      const float l0 = te0 - 0.5f, l1 = te1 - 0.5f;
      om = make_float2(l0 * rcp_fast(p.magic + 0.5f * l0), l1 * rcp_fast(p.magic + 0.5f * l1));
    } else {
      om = op;
    }
  }
  const float2 base = fma2(mul2(rho, bc2(-1.5f)), usq, drho);
  const float2 nhop = mul2(op, bc2(-0.5f)), hom = mul2(om, bc2(0.5f));
  f[0] = fma2(sub2(bc2(1.f), op), f[0], mul2(mul2(op, bc2(float(L::w(0)))), base));
  // the pairs come in weight classes (axis, face diagonal, corner) in
  // direction order; a class's coefficients are formed where it starts
  float2 oA = bc2(0.f), oB = bc2(0.f), nC = bc2(0.f);
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int a = 2 * k + 1, b = a + 1;
    if (k == 0 || wclass<Q>(a) != wclass<Q>(a - 2)) {
      const float w = float(L::w(a));
      oA = mul2(mul2(op, bc2(w)), base);
      oB = mul2(mul2(op, bc2(4.5f * w)), rho);
      nC = mul2(mul2(om, bc2(-3.f * w)), rho);
    }
    float2 cu = L::cx(a) ? ux : (L::cy(a) ? uy : uz);
    if (L::cx(a) && L::cy(a)) cu = L::cy(a) > 0 ? add2(cu, uy) : sub2(cu, uy);
    if ((L::cx(a) || L::cy(a)) && L::cz(a)) cu = L::cz(a) > 0 ? add2(cu, uz) : sub2(cu, uz);
    const float2 t = fma2(oB, mul2(cu, cu), oA);
    const float2 pn = fma2(nhop, add2(f[a], f[b]), t);          // -rp
    const float2 m = fma2(nC, cu, mul2(hom, sub2(f[a], f[b])));  // rm
    f[a] = sub2(add2(f[a], pn), m);
    f[b] = add2(add2(f[b], pn), m);
  }
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// RA: nx and nx * ny are multiples of 16 bytes of elements, so the read
// offset of every odd-step window is (-c_x) mod E, known at compile time.
template <int Q, class S, bool ODD, int STAGES, int MINB, bool RA>
__global__ void __launch_bounds__(STG_THREADS, MINB)
    hydro_staged_kernel(HydroParams<float> p, const int32_t* tiles, int ntiles, TileDirs dirs, int* err,
                        long long wait_limit) {
  using L = Lat<Q>;
  using LY = StgLayout<Q, S>;
  using IO = PairIO<S>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + size_t(STAGES) * LY::STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* never = empty + STAGES;
  __shared__ int stop;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    stop = 0;
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], STG_WARPS);
    }
    mbar_init(never, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (wait_limit < 0) {
    if (tid == 0) wait_selftest(never, wait_limit, err);
    return;
  }
  const int G = int(gridDim.x);
  S* fb = static_cast<S*>(p.f);

  if (warp == STG_WARPS) {
    // ---- producer: one lane issues every copy of the block's tiles ----
    if (lane != 0) return;
    const uint32_t wbytes = uint32_t(ODD ? LY::WIN_BYTES : LY::EVEN_BYTES);
    int issued = 0;
    for (int i = int(blockIdx.x); i < ntiles; i += G, ++issued) {
      const int s = issued % STAGES;
      if (issued >= STAGES) {
        // the consumers' release of this stage's previous round
        if (!mbar_wait_bounded(&empty[s], uint32_t(((issued / STAGES) - 1) & 1), wait_limit) ||
            *(volatile int*)&stop) {
          atomicOr(&stop, 1);
          atomicOr(err, 1);
          break;
        }
        // the consumers' shared loads of the old round before the copy engine
        // overwrites the buffer
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      unsigned char* stage = smem_raw + size_t(s) * LY::STAGE_BYTES;
      const int64_t c0 = int64_t(tiles[i]) * STG_CELLS;
      mbar_expect_tx(&full[s], uint32_t(Q) * wbytes + uint32_t(STG_CELLS));
#pragma unroll 1
      for (int q = 0; q < Q; ++q) bulk_g2s(stage + q * LY::WIN_BYTES, fb + (c0 + dirs.ws[q]), wbytes, &full[s]);
      bulk_g2s(stage + Q * LY::WIN_BYTES, p.flags + c0, uint32_t(STG_CELLS), &full[s]);
    }
    // drain: the last round of every stage has landed before the block leaves
    for (int k = issued > STAGES ? issued - STAGES : 0; k < issued; ++k)
      mbar_wait_bounded(&full[k % STAGES], uint32_t((k / STAGES) & 1), wait_limit);
    return;
  }

  // ---- consumers: two cells per thread ----
  const int nx = p.nx, nxy = p.nxy;
  const int64_t pl = int64_t(p.plane);
  // element offsets from the pair's first cell: own slot k, and slot k of
  // the neighbour x + c_k (uniform across the grid)
  auto P = [&](int k) { return int32_t(int64_t(k) * pl); };
  auto T = [&](int k) { return int32_t(int64_t(k) * pl + (L::cx(k) + L::cy(k) * nx + L::cz(k) * nxy)); };
  auto rq = [&](int q) -> int {
    if (!ODD) return 0;
    if (RA) return (-L::cx(q)) & (LY::E - 1);
    return dirs.r[q];
  };
  int it = 0;
  for (int i = int(blockIdx.x); i < ntiles; i += G, ++it) {
    const int s = it % STAGES;
    if (!mbar_wait_bounded(&full[s], uint32_t((it / STAGES) & 1), wait_limit) || *(volatile int*)&stop) {
      if (lane == 0) {
        atomicOr(&stop, 1);
        atomicOr(err, 1);
      }
      break;
    }
    const unsigned char* stage = smem_raw + size_t(s) * LY::STAGE_BYTES;
    const uint32_t c = uint32_t(tiles[i]) * STG_CELLS + 2 * tid;
    const uint32_t fl2 = *reinterpret_cast<const uint16_t*>(stage + Q * LY::WIN_BYTES + 2 * tid);
    const uint32_t fl0 = fl2 & 0xffu, fl1 = fl2 >> 8;
    const bool act0 = !(fl0 & (F_SOLID | F_FORCED)), act1 = !(fl1 & (F_SOLID | F_FORCED));
    const bool special = (fl0 | fl1) & (F_WRAP | F_SLIP | F_MOVING);
    const bool fast = (act0 || act1) && !special;
    float2 f[Q];
    if (fast) {
      const S* sb = reinterpret_cast<const S*>(stage) + 2 * tid;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const S* src = sb + q * (LY::WIN_BYTES / sizeof(S)) + rq(q);
        if (ODD && (L::cx(q) & 1)) f[q] = make_float2(IO::ld1(src), IO::ld1(src + 1));
        else f[q] = IO::ld2(src);
      }
    }
    // the stage's shared data is in registers: release it to the producer
    // before the collision
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (!(act0 || act1)) continue;
    if (special) {
      const int z = int(c / uint32_t(nxy));
      const int r = int(c - uint32_t(z) * uint32_t(nxy));
      const int y = r / nx, x = r - y * nx;
      if (act0) hydro_cell_generic<Q, S, COLL_TRT, ODD, false>(p, x, y, z, c, uint8_t(fl0));
      if (act1) hydro_cell_generic<Q, S, COLL_TRT, ODD, false>(p, x + 1, y, z, c + 1, uint8_t(fl1));
      continue;
    }
    S* cb = fb + c;
    const uint32_t mk0 = (ODD && (fl0 & F_BOUNDARY)) ? p.nbr[c] : 0u;
    const uint32_t mk1 = (ODD && (fl1 & F_BOUNDARY)) ? p.nbr[c + 1] : 0u;
    const uint32_t mk = mk0 | mk1;
    if (ODD && mk) {
      // directions coming off a wall: the cell's own slot (global)
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int o = opp(q);
        if ((mk0 >> o) & 1u) f[q].x = IO::ld1(cb + P(q));
        if ((mk1 >> o) & 1u) f[q].y = IO::ld1(cb + P(q) + 1);
      }
    }
    trt_pair_lean<Q>(f, p);
    const bool both = act0 && act1;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int o = opp(q);
      const float2 v = f[q];
      if (!ODD) {
        if (both) {
          IO::st2(cb + P(o), v);
        } else {
          if (act0) IO::st1(cb + P(o), v.x);
          if (act1) IO::st1(cb + P(o) + 1, v.y);
        }
      } else if (both && !((mk >> q) & 1u)) {
        if (L::cx(q) & 1) {
          IO::st1(cb + T(q), v.x);
          IO::st1(cb + T(q) + 1, v.y);
        } else {
          IO::st2(cb + T(q), v);
        }
      } else {
        const bool w0 = (mk0 >> q) & 1u, w1 = (mk1 >> q) & 1u;
        if (act0) IO::st1(cb + (w0 ? P(o) : T(q)), v.x);
        if (act1) IO::st1(cb + (w1 ? P(o) : T(q)) + 1, v.y);
      }
    }
  }
}

}  // namespace lbmb
