// The Ozaki GEMM with its group schedule a compile-time constant: included by
// tc.cu after OzFixedSched / oz_slot / GemmArgs / store_chunk.  Every index
// the issue loops use is a template argument, so the producer's loads and the
// MMA thread's product steps compile to straight-line code: a step is its
// barrier waits (only where a tile is first used), four MMAs and the commits
// of the tiles it frees.

template <int S>
constexpr OzFixedSched<S> kOzSched{};

// Group GI of the schedule, used only inside constant expressions.
#define OZG kOzSched<S>.g[GI]

// Runtime state of the MMA-issuing thread within one K block.
struct OzMmaCtx {
  uint32_t s0, par0;  // ring slot / parity of the block's first load
  uint32_t slots_u32, tmem;
  uint32_t started;  // accumulators already written in this phase
  uint64_t *full, *empty;
  volatile int *abort;
  int *status;
  uint64_t limit;    // wait bound (ns)
};

template <int S, int GI, int ST>
__device__ __forceinline__ bool oz_mma_step(OzMmaCtx &c) {
  constexpr int la = OZG.sa[ST], lb = OZG.sb[ST], acc = OZG.sacc[ST];
  constexpr bool wait_a = OZG.first_use[la] == ST, wait_b = OZG.first_use[lb] == ST;
  constexpr unsigned fr = OZG.sfree[ST];
  constexpr uint32_t TILE = 128 * 128;
  constexpr uint32_t IDESC = idesc_i8(128, 128);
  uint32_t sla, pa, slb, pb;
  oz_slot(c.s0, c.par0, la, sla, pa);
  oz_slot(c.s0, c.par0, lb, slb, pb);
  if (wait_a && !mbar_wait(&c.full[sla], pa, c.abort, c.status, QS_ETIMEOUT, c.limit)) return false;
  if (wait_b && !mbar_wait(&c.full[slb], pb, c.abort, c.status, QS_ETIMEOUT, c.limit)) return false;
  if (wait_a || wait_b) tc_fence_after();
  const uint32_t d = c.tmem + acc * 128;
  const uint64_t adesc = sw128_kmajor_desc(c.slots_u32 + sla * TILE);
  const uint64_t bdesc = sw128_kmajor_desc(c.slots_u32 + slb * TILE);
  const uint32_t first = ((c.started >> acc) & 1u) ? 1u : 0u;
#pragma unroll
  for (int j = 0; j < 4; ++j) mma_i8(d, adesc + 2 * j, bdesc + 2 * j, IDESC, j > 0 ? 1u : first);
  c.started |= 1u << acc;
#pragma unroll
  for (int l = 0; l < kOzMaxLoads; ++l)
    if ((fr >> l) & 1u) {
      uint32_t sl, pl;
      oz_slot(c.s0, c.par0, l, sl, pl);
      tc_commit(&c.empty[sl]);
    }
  return true;
}

template <int S, int GI, int... ST>
__device__ __forceinline__ bool oz_mma_steps(OzMmaCtx &c, std::integer_sequence<int, ST...>) {
  return (oz_mma_step<S, GI, ST>(c) && ...);
}

// Runtime state of the producer thread within one K block.
struct OzLoadCtx {
  uint32_t s0, par0;
  uint8_t *slots;
  const uint8_t *rowA, *rowB;  // this tile's panel rows at K block kb
  int64_t planeA, planeB;
  uint64_t *full, *empty;
  volatile int *abort;
  int *status;
  uint64_t limit;   // wait bound (ns)
  uint32_t issued;  // fills issued, in ring order (the exit drain's count)
};

template <int S, int GI, int LD>
__device__ __forceinline__ bool oz_load(OzLoadCtx &c) {
  constexpr int side = OZG.side[LD], slice = OZG.slice[LD];
  constexpr uint32_t TILE = 128 * 128;
  uint32_t slot, par;
  oz_slot(c.s0, c.par0, LD, slot, par);
  if (!mbar_wait(&c.empty[slot], par ^ 1u, c.abort, c.status, QS_ETIMEOUT, c.limit)) return false;
  mbar_arrive_expect_tx(&c.full[slot], TILE);
  const uint8_t *src = side == 0 ? c.rowA + slice * c.planeA : c.rowB + slice * c.planeB;
  bulk_g2s(c.slots + slot * TILE, src, TILE, &c.full[slot]);
  ++c.issued;
  return true;
}

template <int S, int GI, int... LD>
__device__ __forceinline__ bool oz_loads(OzLoadCtx &c, std::integer_sequence<int, LD...>) {
  return (oz_load<S, GI, LD>(c) && ...);
}

// One group (all its K segments and blocks) for the producer.
template <int S, int GI>
__device__ __forceinline__ bool oz_produce_group(const GemmArgs &a, uint32_t &L, OzLoadCtx &c,
                                                 const uint8_t *tileA, const uint8_t *tileB) {
  constexpr int NL = OZG.nloads;
  constexpr uint32_t TILE = 128 * 128;
  for (int ks = 0; ks < a.nkseg; ++ks) {
    const int kb0 = ks * a.kseg_blocks, kb1 = min(kb0 + a.kseg_blocks, a.kblocks);
    for (int kb = kb0; kb < kb1; ++kb) {
      c.s0 = L % kOzSlots;
      c.par0 = (L / kOzSlots) & 1u;
      c.rowA = tileA + (int64_t)kb * TILE;
      c.rowB = tileB + (int64_t)kb * TILE;
      if (!oz_loads<S, GI>(c, std::make_integer_sequence<int, NL>{})) return false;
      L += NL;
    }
  }
  return true;
}

// One group for the MMA thread.
template <int S, int GI>
__device__ __forceinline__ bool oz_mma_group(const GemmArgs &a, uint32_t &L, uint32_t &accpar,
                                             OzMmaCtx &c, uint64_t *acce, uint64_t *accf) {
  constexpr int NL = OZG.nloads, NS = OZG.nsteps, NACC = OZG.t1 - OZG.t0 + 1;
  for (int ks = 0; ks < a.nkseg; ++ks) {
#pragma unroll
    for (int q = 0; q < NACC; ++q)
      if (!mbar_wait(&acce[q], ((accpar >> q) & 1u) ^ 1u, c.abort, c.status, QS_ETIMEOUT, c.limit)) return false;
    tc_fence_after();
    c.started = 0;
    const int kb0 = ks * a.kseg_blocks, kb1 = min(kb0 + a.kseg_blocks, a.kblocks);
    for (int kb = kb0; kb < kb1; ++kb) {
      c.s0 = L % kOzSlots;
      c.par0 = (L / kOzSlots) & 1u;
      if (!oz_mma_steps<S, GI>(c, std::make_integer_sequence<int, NS>{})) return false;
      L += NL;
    }
#pragma unroll
    for (int q = 0; q < NACC; ++q) {
      tc_commit(&accf[q]);
      accpar ^= 1u << q;
    }
  }
  return true;
}

// One group for an epilogue thread: drain each diagonal's accumulator into
// the FP64 running sums.
template <int S, int GI>
__device__ __forceinline__ bool oz_drain_group(const GemmArgs &a, uint32_t &accpar, bool &first,
                                               double (&sum)[64], uint32_t tbase, uint64_t *accf,
                                               uint64_t *acce, int lane, volatile int *abort) {
  constexpr int NACC = OZG.t1 - OZG.t0 + 1, T0 = OZG.t0;
  for (int ks = 0; ks < a.nkseg; ++ks) {
#pragma unroll
    for (int qa = 0; qa < NACC; ++qa) {
      if (!mbar_wait(&accf[qa], (accpar >> qa) & 1u, abort, a.status, QS_ETIMEOUT, a.wait_ns)) return false;
      tc_fence_after();
      const double w = a.wdiag[T0 + qa];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        uint32_t dr[16];
        tmem_ld16(tbase + qa * 128 + 16 * c, dr);
        tmem_ld_wait();
#pragma unroll
        for (int e = 0; e < 16; ++e)
          sum[16 * c + e] = fma((double)(int32_t)dr[e], w, first ? 0.0 : sum[16 * c + e]);
      }
      first = false;
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[qa]);
      accpar ^= 1u << qa;
    }
  }
  return true;
}

// GROUPED: tiles come from the problem table gt (a grouped launch); else the
// launch is one problem, a, and gt is unused.
template <int S, bool GROUPED>
__global__ void __launch_bounds__(320, 1)
    oz_gemm_fixed_kernel(const __grid_constant__ GemmArgs a, const GemmTable gt) {
  constexpr uint32_t TILE = 128 * 128;
  constexpr int NG = kOzSched<S>.ngroups;
  // The last group (the top diagonals: most products, longest) runs first
  // in every tile, so a tile's final store overlaps the next tile's long
  // group instead of stalling the short one.
  constexpr int kG1 = NG - 1, kG2 = 0;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *slots = smem;
  uint64_t *bars = (uint64_t *)(slots + kOzSlots * TILE);
  uint64_t *full = bars, *empty = bars + kOzSlots, *accf = bars + 2 * kOzSlots, *acce = accf + 4;
  uint64_t *drainb = acce + 4;  // the MMA thread's exit drain
  uint32_t *tmem_slot = (uint32_t *)(drainb + 1);
  volatile int *abort = (volatile int *)(tmem_slot + 1);
  int64_t *s_offN = (int64_t *)(smem + kOzSlots * TILE + 1024);
  int32_t *s_expN = (int32_t *)(s_offN + 128);
  GemmArgs *s_args = reinterpret_cast<GemmArgs *>(s_expN + 128);
  static_assert(sizeof(GemmArgs) % 4 == 0 && sizeof(GemmArgs) <= 1024, "staged GemmArgs");

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kOzSlots; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 4; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 8);
    }
    mbar_init(drainb, 1);
    *abort = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int ntile_total = GROUPED ? gt.tile_start[gt.nprob] : a.mtiles * a.ntiles;

  if (warp == 0) {
    if (lane == 0) {
      uint32_t L = 0;
      OzLoadCtx c;
      c.slots = slots;
      c.full = full;
      c.empty = empty;
      c.abort = abort;
      c.status = a.status;
      c.limit = a.wait_ns;
      c.issued = 0;
      for (int tile = blockIdx.x; tile < ntile_total && !a.hold_loads; tile += gridDim.x) {
        int lt;
        const GemmArgs &P = tile_problem<GROUPED>(a, gt, tile, lt);
        int mt, nt;
        tile_coords(lt, P.mtiles, P.ntiles, P.band_m, mt, nt);
        c.planeA = P.planeA;
        c.planeB = P.planeB;
        const uint8_t *tileA = P.panelA + (int64_t)mt * P.kblocks * TILE;
        const uint8_t *tileB = P.panelB + (int64_t)nt * P.kblocks * TILE;
        if (!oz_produce_group<S, kG1>(P, L, c, tileA, tileB)) break;
        if constexpr (NG > 1)
          if (!oz_produce_group<S, kG2>(P, L, c, tileA, tileB)) break;
      }
      // No copy may still be landing in this CTA's shared memory at exit.
      drain_ring(full, kOzSlots, c.issued, a.status, a.wait_ns);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t L = 0, accpar = 0;
      OzMmaCtx c;
      c.slots_u32 = smem_u32(slots);
      c.tmem = tmem;
      c.full = full;
      c.empty = empty;
      c.abort = abort;
      c.status = a.status;
      c.limit = a.wait_ns;
      for (int tile = blockIdx.x; tile < ntile_total; tile += gridDim.x) {
        int lt;
        const GemmArgs &P = tile_problem<GROUPED>(a, gt, tile, lt);
        if (!oz_mma_group<S, kG1>(P, L, accpar, c, acce, accf)) break;
        if constexpr (NG > 1)
          if (!oz_mma_group<S, kG2>(P, L, accpar, c, acce, accf)) break;
      }
      // Every MMA this thread issued is complete before TMEM is released.
      tc_commit(drainb);
      mbar_wait_drain(drainb, 0, a.status, a.wait_ns);
    }
  } else {
    const int q = warp & 3;
    const int h = (warp - 2) >> 2;
    const int et = threadIdx.x - 64;
    const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + 64 * h;
    uint32_t accpar = 0;
    double sum[64];
    for (int tile = blockIdx.x; tile < ntile_total; tile += gridDim.x) {
      int lt;
      const GemmArgs &Pg = tile_problem<GROUPED>(a, gt, tile, lt);
      int mt, nt;
      tile_coords(lt, Pg.mtiles, Pg.ntiles, Pg.band_m, mt, nt);
      const int64_t m0 = (int64_t)mt * 128, n0 = (int64_t)nt * 128;
      named_bar_sync(1, 256);
      if (et < 128) {
        const int64_t n = n0 + et;
        s_offN[et] = n < Pg.N ? c_col(Pg, n) : 0;
        s_expN[et] = n < Pg.N ? Pg.expB[n] : 0;
      }
      if constexpr (GROUPED) {
        // The tile's problem arguments, staged for the epilogue warps.
        const int *src = reinterpret_cast<const int *>(&Pg);
        int *dst = reinterpret_cast<int *>(s_args);
        for (int w = et; w < (int)(sizeof(GemmArgs) / 4); w += 256) dst[w] = src[w];
      }
      named_bar_sync(1, 256);
      const GemmArgs &P = GROUPED ? *s_args : a;
      const int64_t i = m0 + 32 * q + lane;
      const bool row_ok = i < P.M;
      const int eA = row_ok ? P.expA[i] : 0;
      const int64_t crow = row_ok ? P.Cbase + c_row(P, i) : 0;
      const bool row_store = row_ok && eA != kNonFinite;
      if (row_store && (P.cplx != 1 || (lane & 1) == 0)) prefetch_c_row(P, crow, s_offN, 64 * h, 64, n0);
      bool first = true;
      if (!oz_drain_group<S, kG1>(P, accpar, first, sum, tbase, accf, acce, lane, abort)) break;
      if constexpr (NG > 1)
        if (!oz_drain_group<S, kG2>(P, accpar, first, sum, tbase, accf, acce, lane, abort)) break;
      // One copy of the store code per C kind for the four chunks (c is a
      // runtime index; the sums are picked with selects, not local memory).
      if (store_is_f64(P)) {
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
          double v[16];
#pragma unroll
          for (int e = 0; e < 16; ++e)
            v[e] = c == 0 ? sum[e] : c == 1 ? sum[16 + e] : c == 2 ? sum[32 + e] : sum[48 + e];
          store_chunk_f64(P, v, 4 * h + c, n0, row_store, crow, s_offN, s_expN, eA);
        }
      } else {
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
          double v[16];
#pragma unroll
          for (int e = 0; e < 16; ++e)
            v[e] = c == 0 ? sum[e] : c == 1 ? sum[16 + e] : c == 2 ? sum[32 + e] : sum[48 + e];
          store_chunk_any<double>(P, v, 4 * h + c, n0, row_store, crow, lane, s_offN, s_expN, eA);
        }
      }
    }
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}
