// The fixed-schedule Ozaki GEMM on CTA pairs (tcgen05 cta_group::2): a
// cluster of two CTAs computes a 256 x 128 tile of C.  Each CTA holds its 128
// rows of the A slice tiles and half (64 rows) of each B slice tile, so a
// CTA streams 24 KB instead of 32 KB per slice pair and the tensor cores read
// 6 KB of shared memory instead of 8 KB per 128x128x32 of work; the even CTA
// issues one M = 256 MMA for both.  Included by tc.cu after oz_fixed.cuh; it
// follows the same schedule (kOzSched), ring and epilogue.
//
// The slice tiles arrive by tiled tensor loads (cta_group::2, no multicast)
// over the packed panels seen as 2-D byte arrays (128-byte rows, the tiles
// already swizzled, so the copy is linear): both CTAs' loads complete their
// bytes on the even CTA's full barrier, which expects the pair's total.
//
// Two rings in the one-SM kernel's 208 KB: kOzRingA slots of 16 KB for A
// slice tiles and kOzRingB slots of 8 KB for B halves.  A K block of the
// long group takes 6 of each, so the next block's first B window and A tiles
// load while the current block still computes (the one-SM kernel's single
// ring of 13 is full with the block's 12 tiles).
//
// Barriers, per ring slot s (of either ring) and accumulator q:
//   full[s]  even CTA: its producer (expect_tx of both CTAs' bytes).
//   empty[s] both CTAs, arrived by the even CTA's multicast commit.
//   accf[q]  both CTAs, multicast commit after a K segment's MMAs.
//   acce[q]  even CTA: 8 epilogue warps of each CTA (16), the odd CTA's
//            remotely.
// Every wait is bounded (mbar_wait); all roles end at a cluster barrier.

constexpr uint32_t kOzHalfB = 64 * 128;  // the odd/even half of a B slice tile
constexpr int kOzRingA = 8, kOzRingB = 10;
static_assert(kOzRingA * 16384 + kOzRingB * kOzHalfB <= kOzSlots * 16384, "rings fit the one-SM slots");

// Ordinal of load LD among the same-side loads of its group, and the group's
// A and B load counts.
template <int S, int GI>
__host__ __device__ constexpr int oz2_side_ord(int LD) {
  int n = 0;
  for (int l = 0; l < LD; ++l) n += OZG.side[l] == OZG.side[LD] ? 1 : 0;
  return n;
}
template <int S, int GI>
__host__ __device__ constexpr int oz2_side_count(int side) {
  int n = 0;
  for (int l = 0; l < OZG.nloads; ++l) n += OZG.side[l] == side ? 1 : 0;
  return n;
}

// Slot and parity of the l-th load after ring position s0 (l < N).
template <int N>
__device__ __forceinline__ void ring_slot(uint32_t s0, uint32_t par0, int l, uint32_t &slot, uint32_t &par) {
  const uint32_t idx = s0 + (uint32_t)l;
  const uint32_t w = idx >= (uint32_t)N ? 1u : 0u;
  slot = idx - w * N;
  par = par0 ^ w;
}

// Ring positions of the two sides at the start of a K block.
struct Oz2Ring {
  uint32_t a0, pa, b0, pb;
};
__device__ __forceinline__ Oz2Ring oz2_ring(uint32_t LA, uint32_t LB) {
  return Oz2Ring{LA % kOzRingA, (LA / kOzRingA) & 1u, LB % kOzRingB, (LB / kOzRingB) & 1u};
}

// Runtime state of the MMA-issuing thread of a pair.
struct Oz2MmaCtx {
  Oz2Ring r;
  uint32_t slotsA_u32, slotsB_u32, tmem;
  uint32_t started;
  uint64_t *fullA, *emptyA, *fullB, *emptyB;
  volatile int *abort;
  int *status;
  uint64_t limit;  // wait bound (ns)
};

// Release load L's slot if step ST is its last use (compile-time choice).
template <int S, int GI, int ST, int L>
__device__ __forceinline__ void oz2_free(Oz2MmaCtx &c) {
  if constexpr (L < OZG.nloads && ((OZG.sfree[ST] >> L) & 1u)) {
    constexpr int ord = oz2_side_ord<S, GI>(L);
    uint32_t sl, pl;
    if constexpr (OZG.side[L] == 0) {
      ring_slot<kOzRingA>(c.r.a0, c.r.pa, ord, sl, pl);
      tc_commit_pair(&c.emptyA[sl]);
    } else {
      ring_slot<kOzRingB>(c.r.b0, c.r.pb, ord, sl, pl);
      tc_commit_pair(&c.emptyB[sl]);
    }
  }
}
template <int S, int GI, int ST, int... L>
__device__ __forceinline__ void oz2_frees(Oz2MmaCtx &c, std::integer_sequence<int, L...>) {
  (oz2_free<S, GI, ST, L>(c), ...);
}

template <int S, int GI, int ST>
__device__ __forceinline__ bool oz2_mma_step(Oz2MmaCtx &c) {
  constexpr int la = OZG.sa[ST], lb = OZG.sb[ST], acc = OZG.sacc[ST];
  constexpr bool wait_a = OZG.first_use[la] == ST, wait_b = OZG.first_use[lb] == ST;
  constexpr uint32_t IDESC = idesc_i8(256, 128);
  constexpr int oa = oz2_side_ord<S, GI>(la), ob = oz2_side_ord<S, GI>(lb);
  uint32_t sla, pa, slb, pb;
  ring_slot<kOzRingA>(c.r.a0, c.r.pa, oa, sla, pa);
  ring_slot<kOzRingB>(c.r.b0, c.r.pb, ob, slb, pb);
  if (wait_a && !mbar_wait(&c.fullA[sla], pa, c.abort, c.status, QS_ETIMEOUT, c.limit)) return false;
  if (wait_b && !mbar_wait(&c.fullB[slb], pb, c.abort, c.status, QS_ETIMEOUT, c.limit)) return false;
  if (wait_a || wait_b) tc_fence_after();
  const uint32_t d = c.tmem + acc * 128;
  const uint64_t adesc = sw128_kmajor_desc(c.slotsA_u32 + sla * 16384u);
  const uint64_t bdesc = sw128_kmajor_desc(c.slotsB_u32 + slb * kOzHalfB);
  const uint32_t first = ((c.started >> acc) & 1u) ? 1u : 0u;
#pragma unroll
  for (int j = 0; j < 4; ++j) mma_i8_pair(d, adesc + 2 * j, bdesc + 2 * j, IDESC, j > 0 ? 1u : first);
  c.started |= 1u << acc;
  oz2_frees<S, GI, ST>(c, std::make_integer_sequence<int, kOzMaxLoads>{});
  return true;
}

template <int S, int GI, int... ST>
__device__ __forceinline__ bool oz2_mma_steps(Oz2MmaCtx &c, std::integer_sequence<int, ST...>) {
  return (oz2_mma_step<S, GI, ST>(c) && ...);
}

// Runtime state of a pair producer within one K block.
struct Oz2LoadCtx {
  Oz2Ring r;
  uint8_t *slotsA, *slotsB;
  const void *tmA, *tmB;  // tensor maps of the A and B panels (kernel parameters)
  int yA, yB;             // first panel row of this CTA's tiles at K block kb
  int planeRowsA, planeRowsB;
  uint64_t *fullA, *emptyA, *fullB, *emptyB;
  uint32_t rank;
  volatile int *abort;
  int *status;
  uint64_t limit;            // wait bound (ns)
  uint32_t issuedA, issuedB;  // fills issued per ring, in ring order (the exit drain's counts)
};

template <int S, int GI, int LD>
__device__ __forceinline__ bool oz2_load(Oz2LoadCtx &c) {
  constexpr int side = OZG.side[LD], slice = OZG.slice[LD];
  constexpr int ord = oz2_side_ord<S, GI>(LD);
  constexpr uint32_t BYTES = side == 0 ? 16384u : kOzHalfB;
  uint32_t slot, par;
  if (side == 0) ring_slot<kOzRingA>(c.r.a0, c.r.pa, ord, slot, par);
  else ring_slot<kOzRingB>(c.r.b0, c.r.pb, ord, slot, par);
  uint64_t *full = side == 0 ? &c.fullA[slot] : &c.fullB[slot];
  uint64_t *empty = side == 0 ? &c.emptyA[slot] : &c.emptyB[slot];
  if (!mbar_wait(empty, par ^ 1u, c.abort, c.status, QS_ETIMEOUT, c.limit)) return false;
  if (c.rank == 0) mbar_arrive_expect_tx(full, 2 * BYTES);
  const uint32_t mbar = mapa_u32(full, 0);
  if (side == 0) {
    tma_load_2d_pair(c.slotsA + slot * 16384u, c.tmA, 0, c.yA + slice * c.planeRowsA, mbar);
    ++c.issuedA;
  } else {
    tma_load_2d_pair(c.slotsB + slot * kOzHalfB, c.tmB, 0, c.yB + slice * c.planeRowsB, mbar);
    ++c.issuedB;
  }
  return true;
}

template <int S, int GI, int... LD>
__device__ __forceinline__ bool oz2_loads(Oz2LoadCtx &c, std::integer_sequence<int, LD...>) {
  return (oz2_load<S, GI, LD>(c) && ...);
}

// One group for a producer.  rowA0/rowB0: panel row of this CTA's tile at K
// block 0 (tile-major panels: a tile's K blocks are 128 rows apart).
template <int S, int GI>
__device__ __forceinline__ bool oz2_produce_group(const GemmArgs &a, uint32_t &LA, uint32_t &LB, Oz2LoadCtx &c,
                                                  int rowA0, int rowB0) {
  constexpr int NL = OZG.nloads, NA = oz2_side_count<S, GI>(0), NB = oz2_side_count<S, GI>(1);
  for (int ks = 0; ks < a.nkseg; ++ks) {
    const int kb0 = ks * a.kseg_blocks, kb1 = min(kb0 + a.kseg_blocks, a.kblocks);
    for (int kb = kb0; kb < kb1; ++kb) {
      c.r = oz2_ring(LA, LB);
      c.yA = rowA0 + kb * 128;
      c.yB = rowB0 + kb * 128;
      if (!oz2_loads<S, GI>(c, std::make_integer_sequence<int, NL>{})) return false;
      LA += NA;
      LB += NB;
    }
  }
  return true;
}

template <int S, int GI>
__device__ __forceinline__ bool oz2_mma_group(const GemmArgs &a, uint32_t &LA, uint32_t &LB, uint32_t &accpar,
                                              Oz2MmaCtx &c, uint64_t *acce, uint64_t *accf) {
  constexpr int NS = OZG.nsteps, NACC = OZG.t1 - OZG.t0 + 1;
  constexpr int NA = oz2_side_count<S, GI>(0), NB = oz2_side_count<S, GI>(1);
  for (int ks = 0; ks < a.nkseg; ++ks) {
#pragma unroll
    for (int q = 0; q < NACC; ++q)
      if (!mbar_wait(&acce[q], ((accpar >> q) & 1u) ^ 1u, c.abort, c.status, QS_ETIMEOUT, c.limit))
        return false;
    tc_fence_after();
    c.started = 0;
    const int kb0 = ks * a.kseg_blocks, kb1 = min(kb0 + a.kseg_blocks, a.kblocks);
    for (int kb = kb0; kb < kb1; ++kb) {
      c.r = oz2_ring(LA, LB);
      if (!oz2_mma_steps<S, GI>(c, std::make_integer_sequence<int, NS>{})) return false;
      LA += NA;
      LB += NB;
    }
#pragma unroll
    for (int q = 0; q < NACC; ++q) {
      tc_commit_pair(&accf[q]);
      accpar ^= 1u << q;
    }
  }
  return true;
}

// The epilogue's drain, with the accumulator release sent to the even CTA.
template <int S, int GI>
__device__ __forceinline__ bool oz2_drain_group(const GemmArgs &a, uint32_t &accpar, bool &first,
                                                double (&sum)[64], uint32_t tbase, uint64_t *accf,
                                                uint64_t *acce, int lane, volatile int *abort, uint32_t rank) {
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
      if (lane == 0) {
        if (rank == 0) mbar_arrive(&acce[qa]);
        else mbar_arrive_cluster(&acce[qa], 0);
      }
      accpar ^= 1u << qa;
    }
  }
  return true;
}

// The even CTA's exit drain of one ring: every fill either CTA issued has
// landed.  Both CTAs' copies complete on the even CTA's full barriers, which
// the even producer arms for both halves, so per slot the two CTAs can be
// one fill apart when a wait gave up (a CTA refills a slot only after the
// MMA consumed the slot's previous fill, which needed both halves):
//  - the odd CTA one fill ahead: arm that phase for the odd half alone;
//  - this CTA one fill ahead: count the missing odd half as done;
// then wait for the slot's last phase.  issuedE / issuedO: the CTAs' fills
// in ring order; half: the bytes of one CTA's half of a fill.
__device__ __forceinline__ void oz2_drain_ring(uint64_t *full, int nslots, uint32_t issuedE, uint32_t issuedO,
                                               uint32_t half, int *status, uint64_t limit) {
  for (int s = 0; s < nslots; ++s) {
    const int fE = issuedE > (uint32_t)s ? (int)((issuedE - 1u - (uint32_t)s) / (uint32_t)nslots) : -1;
    const int fO = issuedO > (uint32_t)s ? (int)((issuedO - 1u - (uint32_t)s) / (uint32_t)nslots) : -1;
    if (fE < 0 && fO < 0) continue;
    if (fO == fE + 1) {
      if (fE >= 0 && !mbar_wait_drain(&full[s], (uint32_t)fE & 1u, status, limit)) continue;
      mbar_arrive_expect_tx(&full[s], half);
      mbar_wait_drain(&full[s], (uint32_t)fO & 1u, status, limit);
    } else if (fE == fO + 1) {
      if (fO >= 0 && !mbar_wait_drain(&full[s], (uint32_t)fO & 1u, status, limit)) continue;
      mbar_complete_tx(&full[s], half);
      mbar_wait_drain(&full[s], (uint32_t)fE & 1u, status, limit);
    } else {
      mbar_wait_drain(&full[s], (uint32_t)(fE > fO ? fE : fO) & 1u, status, limit);
    }
  }
}

// Pair tile t -> (m-pair, n-tile), in bands of band_m / 2 m-pairs: the same
// m-tiles per band as the one-SM kernel, so a wave's panels fit L2.
__device__ __forceinline__ void pair_tile_coords(int t, int mpairs, int ntiles, int band_m, int &mp, int &nt) {
  const int kBand = band_m / 2;
  const int per_band = kBand * ntiles;
  const int band = t / per_band, r = t - band * per_band;
  const int m0 = band * kBand;
  const int bm = mpairs - m0 < kBand ? mpairs - m0 : kBand;
  mp = m0 + r % bm;
  nt = r / bm;
}

// One launch: grid = 2 x clusters, cluster dims (2, 1, 1), one CTA per SM.
template <int S>
__global__ void __launch_bounds__(320, 1)
    oz_gemm_pair_kernel(const __grid_constant__ GemmArgs a, const __grid_constant__ CUtensorMap tmA,
                        const __grid_constant__ CUtensorMap tmB) {
  constexpr uint32_t TILE = 128 * 128;
  constexpr int NG = kOzSched<S>.ngroups;
  constexpr int kG1 = NG - 1, kG2 = 0;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *slotsA = smem, *slotsB = smem + kOzRingA * 16384;
  uint64_t *bars = (uint64_t *)(smem + kOzSlots * TILE);
  uint64_t *fullA = bars, *emptyA = fullA + kOzRingA, *fullB = emptyA + kOzRingA, *emptyB = fullB + kOzRingB;
  uint64_t *accf = emptyB + kOzRingB, *acce = accf + 4;
  uint64_t *drainb = acce + 4;  // the MMA's exit drain (committed to both CTAs)
  uint32_t *tmem_slot = (uint32_t *)(drainb + 1);
  volatile int *abort = (volatile int *)(tmem_slot + 1);
  uint32_t *s_issued = (uint32_t *)(tmem_slot + 2);  // [A, B] of the even CTA, [A, B] of the odd CTA
  int64_t *s_offN = (int64_t *)(smem + kOzSlots * TILE + 1024);
  int32_t *s_expN = (int32_t *)(s_offN + 128);

  const uint32_t rank = cluster_ctarank();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kOzRingA; ++s) {
      mbar_init(&fullA[s], 1);
      mbar_init(&emptyA[s], 1);
    }
    for (int s = 0; s < kOzRingB; ++s) {
      mbar_init(&fullB[s], 1);
      mbar_init(&emptyB[s], 1);
    }
    for (int b = 0; b < 4; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 16);
    }
    mbar_init(drainb, 1);
    *abort = 0;
    for (int i = 0; i < 4; ++i) s_issued[i] = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc_pair(tmem_slot, 512);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  cluster_sync();  // both CTAs' barriers and TMEM exist before any remote use
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int mpairs = (a.mtiles + 1) / 2;
  const int npair_tiles = mpairs * a.ntiles;
  const int cluster = blockIdx.x >> 1, nclusters = gridDim.x >> 1;

  if (warp == 0) {
    // The producer of each CTA.
    if (lane == 0) {
      uint32_t LA = 0, LB = 0;
      Oz2LoadCtx c;
      c.slotsA = slotsA;
      c.slotsB = slotsB;
      c.tmA = &tmA;
      c.tmB = &tmB;
      c.planeRowsA = (int)(a.planeA / 128);
      c.planeRowsB = (int)(a.planeB / 128);
      c.fullA = fullA;
      c.emptyA = emptyA;
      c.fullB = fullB;
      c.emptyB = emptyB;
      c.rank = rank;
      c.abort = abort;
      c.status = a.status;
      c.limit = a.wait_ns;
      c.issuedA = c.issuedB = 0;
      for (int pt = cluster; pt < npair_tiles && !a.hold_loads; pt += nclusters) {
        int mp, nt;
        pair_tile_coords(pt, mpairs, a.ntiles, a.band_m, mp, nt);
        const int mt = 2 * mp + (int)rank;
        const int rowA0 = mt * a.kblocks * 128;
        const int rowB0 = nt * a.kblocks * 128 + (int)rank * 64;
        bool ok = oz2_produce_group<S, kG1>(a, LA, LB, c, rowA0, rowB0);
        if constexpr (NG > 1) ok = ok && oz2_produce_group<S, kG2>(a, LA, LB, c, rowA0, rowB0);
        if (!ok) break;
      }
      // The fill counts go to the even CTA, which drains both CTAs' copies.
      if (rank == 0) {
        s_issued[0] = c.issuedA;
        s_issued[1] = c.issuedB;
      } else {
        st_cluster_u32(&s_issued[2], 0, c.issuedA);
        st_cluster_u32(&s_issued[3], 0, c.issuedB);
      }
    }
  } else if (warp == 1) {
    // The even CTA's MMA thread issues for both CTAs; the odd CTA's idles.
    if (lane == 0 && rank == 0) {
      uint32_t LA = 0, LB = 0, accpar = 0;
      Oz2MmaCtx c;
      c.slotsA_u32 = smem_u32(slotsA);
      c.slotsB_u32 = smem_u32(slotsB);
      c.tmem = tmem;
      c.fullA = fullA;
      c.emptyA = emptyA;
      c.fullB = fullB;
      c.emptyB = emptyB;
      c.abort = abort;
      c.status = a.status;
      c.limit = a.wait_ns;
      for (int pt = cluster; pt < npair_tiles; pt += nclusters) {
        if (!oz2_mma_group<S, kG1>(a, LA, LB, accpar, c, acce, accf)) break;
        if constexpr (NG > 1)
          if (!oz2_mma_group<S, kG2>(a, LA, LB, accpar, c, acce, accf)) break;
      }
      // Every MMA issued is complete (in both CTAs) before TMEM is released.
      tc_commit_pair(drainb);
    }
    if (lane == 0) mbar_wait_drain(drainb, 0, a.status, a.wait_ns);
  } else {
    const int q = warp & 3;
    const int h = (warp - 2) >> 2;
    const int et = threadIdx.x - 64;
    const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + 64 * h;
    uint32_t accpar = 0;
    double sum[64];
    for (int pt = cluster; pt < npair_tiles; pt += nclusters) {
      int mp, nt;
      pair_tile_coords(pt, mpairs, a.ntiles, a.band_m, mp, nt);
      const int mt = 2 * mp + (int)rank;
      const int64_t m0 = (int64_t)mt * 128, n0 = (int64_t)nt * 128;
      named_bar_sync(1, 256);
      if (et < 128) {
        const int64_t n = n0 + et;
        s_offN[et] = n < a.N ? c_col(a, n) : 0;
        s_expN[et] = n < a.N ? a.expB[n] : 0;
      }
      named_bar_sync(1, 256);
      const int64_t i = m0 + 32 * q + lane;
      const bool row_ok = i < a.M;
      const int eA = row_ok ? a.expA[i] : 0;
      const int64_t crow = row_ok ? a.Cbase + c_row(a, i) : 0;
      const bool row_store = row_ok && eA != kNonFinite;
      if (row_store && (a.cplx != 1 || (lane & 1) == 0)) prefetch_c_row(a, crow, s_offN, 64 * h, 64, n0);
      bool first = true;
      if (!oz2_drain_group<S, kG1>(a, accpar, first, sum, tbase, accf, acce, lane, abort, rank)) break;
      if constexpr (NG > 1)
        if (!oz2_drain_group<S, kG2>(a, accpar, first, sum, tbase, accf, acce, lane, abort, rank)) break;
      if (store_is_f64(a)) {
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
          double v[16];
#pragma unroll
          for (int e = 0; e < 16; ++e)
            v[e] = c == 0 ? sum[e] : c == 1 ? sum[16 + e] : c == 2 ? sum[32 + e] : sum[48 + e];
          store_chunk_f64(a, v, 4 * h + c, n0, row_store, crow, s_offN, s_expN, eA);
        }
      } else {
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
          double v[16];
#pragma unroll
          for (int e = 0; e < 16; ++e)
            v[e] = c == 0 ? sum[e] : c == 1 ? sum[16 + e] : c == 2 ? sum[32 + e] : sum[48 + e];
          store_chunk_any<double>(a, v, 4 * h + c, n0, row_store, crow, lane, s_offN, s_expN, eA);
        }
      }
    }
  }
  __syncwarp();
  tc_fence_before();
  cluster_sync();  // both CTAs' fill counts are in; every MMA is complete
  if (rank == 0 && warp == 0 && lane == 0) {
    oz2_drain_ring(fullA, kOzRingA, s_issued[0], s_issued[2], 16384u, a.status, a.wait_ns);
    oz2_drain_ring(fullB, kOzRingB, s_issued[1], s_issued[3], kOzHalfB, a.status, a.wait_ns);
  }
  cluster_sync();  // every copy has landed; no remote arrive is still pending
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem, 512);
  }
}
