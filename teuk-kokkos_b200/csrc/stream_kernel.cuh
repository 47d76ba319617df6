// Streaming RK stage kernel: persistent CTAs walk radial strips of band
// segments through a shared-memory ring filled by bulk asynchronous copies.
// Included by kernels.cu inside its anonymous namespace (it shares the SBP
// constant tables, the complex helpers and the FP64 MMA wrapper).
//
// Per CTA (one per SM, 512 threads):
//   warps 0-7     transform warps: stage combine u = y + c k in place,
//                 effective Q (stage-constrained reduction) and
//                 psi_t = A diag(.) S (.) on the FP64 tensor path, two warps
//                 per 4-row block (each takes half of the node tiles of the
//                 synthesis and one ell tile of the analysis);
//   warps 8-11    stencil warps: SBP derivatives, dissipation, RHS assembly
//                 and the RK update of every output row, two adjacent rows
//                 of one ell and all three fields per thread (one register
//                 window per field serves both rows).  They publish how
//                 many chunks no later work reads.
//   warps 12-15   producer warpgroup (24 registers): one thread issues the
//                 cp.async.bulk copies of each 16-row chunk of the stage
//                 inputs, of the Teukolsky row coefficients and (Kerr) of
//                 the rows' 1 / C_T node values into a
//                 4-stage ring (completion through mbarrier transaction
//                 counts) as soon as the stencil warps hand a stage back.
// The roles run concurrently on different chunks: the copies of the next
// chunks, the transforms of the current one and the stencils of the rows it
// completes overlap.  Every halo row is loaded and transformed once per
// strip.  Four warps per SM sub-partition.
//
// Every wait on an mbarrier gives up after kStreamWaitNs: the waiting role
// raises the CTA's abort flag and records an error code that the host reads
// after the step, and the other role leaves at its next wait.

constexpr int kStreamNep = 16;                              // ell lanes per row
constexpr int kStreamMaxTheta = 32;                         // nodes per row
constexpr int kStreamChunk = 16;                            // rows per copy
constexpr int kStreamStages = 4;                            // ring stages
constexpr int kStreamRing = kStreamChunk * kStreamStages;  // ring rows
constexpr int kStreamTWarps = 8;
constexpr int kStreamSWarps = 4;
constexpr int kStreamPWarps = 4;  // producer warpgroup (one thread loads)
constexpr int kStreamThreads = 32 * (kStreamTWarps + kStreamSWarps + kStreamPWarps);
constexpr int kStreamTThreads = 32 * kStreamTWarps;
constexpr int kStreamSThreads = 32 * kStreamSWarps;
constexpr int kStreamBlocks = 4;  // 4-row transform blocks per 16 rows
// Named barriers: 1 all transform warps, 2 the stencil warps, 3 + b the two
// warps of transform block b.
constexpr int kStreamBlockBar = 3;
static_assert(kStreamBlockBar + kStreamBlocks <= 16, "named barrier ids");
constexpr unsigned long long kStreamWaitNs = 2000000000ull;
static_assert(kStreamNep == kStreamMaxEll, "ell lanes");
static_assert(kStreamMaxTheta == kStreamMaxNodes, "node tiles");
static_assert(kStripMinRows >= 2 * 17, "strip edges clear of closures");
static_assert(kCoefRecord == kCoefCount, "coefficient record");
static_assert(2 * kStreamSThreads == kStreamNep * kStreamChunk,
              "one stencil thread per (row pair, ell) of a chunk");
static_assert(kStreamTWarps == 2 * kStreamBlocks, "two warps per block");
// Register split between the warpgroups (setmaxnreg): the launch gives
// every thread 128 registers; the producer warpgroup drops to 24, the
// transform warpgroups keep 128 (their MMA fragments and accumulators stay
// in registers) and the stencil warpgroup raises its count to 232 (two rows'
// terms, one 14-row window and the loads hoisted ahead of their use; from
// 184 up nothing spills, and more is faster).  128 x 24 + 256 x 128 +
// 128 x 232 = 65536 = 512 x 128, so the raise is always satisfiable; the
// launcher checks the launch allocation.
constexpr int kStreamLaunchRegs = 128;
constexpr int kStreamTRegs = 128;
constexpr int kStreamSRegs = 232;
constexpr int kStreamPRegs = 24;
constexpr int kStreamRegisterDemand =
    kStreamTThreads * kStreamTRegs + kStreamSThreads * kStreamSRegs +
    32 * kStreamPWarps * kStreamPRegs;
static_assert(kStreamRegisterDemand <= kStreamThreads * kStreamLaunchRegs,
              "register split fits the launch's registers");
// split-precision record of one segment: [synthesis h0, h1, analysis h0,
// h1][slice][lane] uint4, and 48 scales (32 node rows, 16 ell rows)
constexpr int kSplitRecord = 4 * split::kSlices * 32;
constexpr int kSplitScales = kStreamMaxTheta + kStreamNep;
constexpr int kStreamXs = 20;  // padded staging strides (bank-conflict free)
constexpr int kStreamTs = 36;

// Ring geometry of a streaming launch.  NarrowGeom: n_ell <= 16, at most 32
// nodes, 16-row chunks in a 4-stage ring that also holds the RK
// accumulator rows.  WideGeom: n_ell <= 24, at most 48 nodes (free-damped
// reduction), the same chunks and stages; three 24-lane rings of 64 rows do
// not fit in shared memory, two do: stage 4 copies the accumulator rows
// into the free X ring, stage 3's RK update reads them from global memory,
// and the transforms read the 1 / C_T node values from global memory.
struct NarrowGeom {
  static constexpr int kNep = kStreamNep;        // ell lanes per row
  static constexpr int kChunk = kStreamChunk;    // rows per copy
  static constexpr int kStages = kStreamStages;  // ring stages
  static constexpr int kRing = kStreamRing;      // ring rows
  static constexpr int kPairs = kStreamSThreads / kStreamNep;  // row pairs
  static constexpr int kNodeRec = kStreamMaxTheta;  // node-table record
  static constexpr bool kRingA = true;  // accumulator rows in the ring
};
struct WideGeom {
  static constexpr int kNep = 24;
  static constexpr int kChunk = kStreamChunk;
  static constexpr int kStages = kStreamStages;
  static constexpr int kRing = kChunk * kStages;
  static constexpr int kPairs = kStreamSThreads / kNep;  // 5 (8 threads idle)
  static constexpr int kNodeRec = 48;
  static constexpr bool kRingA = false;  // no accumulator or node-row ring
};
static_assert(2 * NarrowGeom::kPairs == NarrowGeom::kChunk, "narrow pass");
static_assert(WideGeom::kNep == kWideMaxEll && WideGeom::kNodeRec == kWideMaxNodes,
              "wide limits");

__device__ __forceinline__ unsigned smem_u32(const void* ptr) {
  return static_cast<unsigned>(__cvta_generic_to_shared(ptr));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar,
                                          const unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
               :
               : "r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];"
               :
               : "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar,
                                                      const unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :
               : "r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar,
                                              const unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// global -> shared bulk copy completing on `bar` (no multicast)
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src,
                                              const unsigned bytes,
                                              unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];"
      :
      : "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbarrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void named_sync(const int id, const int threads) {
  asm volatile("bar.sync %0, %1;" : : "r"(id), "r"(threads) : "memory");
}
// Barrier over `threads` threads of the CTA that also ANDs `pred` across
// them: every participant gets the same answer.
__device__ __forceinline__ bool named_sync_and(const int id, const int threads,
                                               const bool pred) {
  unsigned all;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(all)
      : "r"(pred ? 1u : 0u), "r"(id), "r"(threads)
      : "memory");
  return all != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the phase of `bar` with the given parity.  False when
// the CTA is aborting (this wait timed out, or another one did).
__device__ bool stream_wait(unsigned long long* bar, const unsigned parity,
                            volatile int* abort_flag, int* error,
                            const int code) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag != 0) return false;
    if (global_ns() - t0 > kStreamWaitNs) {
      *abort_flag = 1;
      if (error != nullptr) atomicExch(error, code);
      return false;
    }
  }
}

// Row range bookkeeping of one strip (rows of one segment).
struct StripGeom {
  long long seg_offset;  // complex offset of row 0 of the segment
  int segment, instance, m, ne, rs, nr, coef_row0;
  int node_row0;  // first row of the solve in this geometry's node table
  int kerr;  // the transform reads 1 / C_T node rows
  int r0, r1;  // output rows
  int s0, s1;  // input rows (with halo)
  int t0, t1;  // psi_t / effective-Q rows
  int chunks;
  int shift;  // ring row of absolute row q: (q + shift) mod ring rows
};

// Loader state, kept in shared memory (only its one thread touches it).
struct StreamLoaderState {
  StripGeom sg;  // geometry of `strip`
  const double2* src_u;  // stage input arrays of this launch
  const double2* src_x;
  const double2* src_a;
  int strip;     // strip of the next chunk to load (>= strip_count: done)
  int c;         // its chunk index within the strip
  int g;         // its global chunk index
  int prev_rs;   // row stride of the strip of chunk g - 1
};

// Shared-memory carve-up (bytes), identical on host and device.
struct StreamLayout {
  static constexpr int kRowMax = 3 * kStreamNep;  // complex per ring row
  size_t bars, loader, uring, xring, aring, pring, qring, coef, nodes, xw,
      tw, ex, total;
  __host__ __device__ explicit StreamLayout(const int sc) {
    size_t o = 0;
    bars = o;
    o += 128;  // 2 x stages mbarriers, abort flag, released-chunk count
    loader = o;
    o += (sizeof(StreamLoaderState) + 127) / 128 * 128;
    const size_t ring = static_cast<size_t>(kStreamRing) * kRowMax * 16;
    uring = o;
    o += ring;
    xring = o;
    o += ring;
    aring = o;
    o += ring;
    pring = o;
    o += static_cast<size_t>(kStreamRing) * kStreamNep * 16;
    qring = o;
    if (sc) o += static_cast<size_t>(kStreamRing) * kStreamNep * 16;
    coef = o;
    o += static_cast<size_t>(kStreamRing) * kCoefCount * 8;
    nodes = o;
    o += static_cast<size_t>(kStreamRing) * kNodeRecord * 8;
    xw = o;
    o += static_cast<size_t>(kStreamBlocks) * 16 * kStreamXs * 8;
    tw = o;
    o += static_cast<size_t>(kStreamBlocks) * 8 * kStreamTs * 8;
    ex = o;  // split precision: per block, 2 warps x 32 lanes x 2 doubles
    o += static_cast<size_t>(kStreamBlocks) * 128 * 8;
    total = o;
  }
};

template <int H, int HD, class G = NarrowGeom>
__device__ __forceinline__ StripGeom strip_geom(const StageLaunch& p,
                                                const int strip,
                                                const int first_chunk) {
  const TileDesc t = p.strips[strip];
  const SegmentDesc seg = p.segments[t.segment];
  const InstanceDesc& in = p.instances[seg.instance];
  StripGeom g;
  g.seg_offset = seg.offset;
  g.segment = t.segment;
  g.instance = seg.instance;
  g.m = seg.m;
  g.ne = seg.n_ell;
  g.rs = 3 * seg.n_ell;
  g.nr = in.nr;
  g.coef_row0 = in.coef_row0;
  g.node_row0 = G::kRingA ? in.coef_row0 : in.wide_row0;
  g.kerr = in.spin != 0.0 ? 1 : 0;
  g.r0 = t.r0;
  g.r1 = t.r1;
  g.s0 = max(0, t.r0 - H);
  g.s1 = min(g.nr, t.r1 + H);
  g.t0 = max(0, t.r0 - HD);
  g.t1 = min(g.nr, t.r1 + HD);
  g.chunks = (g.s1 - g.s0 + G::kChunk - 1) / G::kChunk;
  g.shift = first_chunk * G::kChunk - g.s0;
  return g;
}

template <class G = NarrowGeom>
__device__ __forceinline__ int ring_row(const int q, const int shift) {
  if constexpr ((G::kRing & (G::kRing - 1)) == 0) {
    return (q + shift) & (G::kRing - 1);
  } else {  // q + shift >= 0 for every row read
    return static_cast<int>(static_cast<unsigned>(q + shift) %
                            static_cast<unsigned>(G::kRing));
  }
}

// Ring rows of the consecutive rows q0, q0 + 1, ..., q0 + N - 1 (N <= ring
// rows): one modulo, then a wrap test per row.
template <class G, int N>
__device__ __forceinline__ void ring_rows(int (&rows)[N], const int q0,
                                          const int shift) {
  static_assert(N <= G::kRing, "window longer than the ring");
  if constexpr ((G::kRing & (G::kRing - 1)) == 0) {
#pragma unroll
    for (int i = 0; i < N; ++i) rows[i] = ring_row<G>(q0 + i, shift);
  } else {
    const int b = ring_row<G>(q0, shift);
#pragma unroll
    for (int i = 0; i < N; ++i) {
      rows[i] = b + i < G::kRing ? b + i : b + i - G::kRing;
    }
  }
}

// First row that is not yet computable for a stencil of half width `half`
// (closure: rows below `closure_rows` read the first `need` rows, rows in
// the last `closure_rows` read the last ones) when rows [.., avail) exist.
__device__ __forceinline__ int computable_end(const int avail, const int nr,
                                              const int half, const int need,
                                              const int closure_rows) {
  if (avail >= nr) return nr;
  if (avail < need) return 0;
  return min(avail - half, nr - closure_rows);
}

// SBP first derivative / dissipation with an accessor for absolute rows
// (closure rows included); mirrors sbp_derivative / sbp_dissipation.
template <int DISC, class Row>
__device__ __forceinline__ double2 ring_derivative(const Row& at, const int r,
                                                   const int nr) {
  using T = DiscTraits<DISC>;
  double2 acc = make_double2(0.0, 0.0);
  if (r < T::BR) {
#pragma unroll
    for (int c = 0; c < T::W; ++c) acc = cfma(c_sbp.left[DISC][r][c], at(c), acc);
  } else if (r + T::BR >= nr) {
    const int rr = nr - 1 - r;
#pragma unroll
    for (int c = 0; c < T::W; ++c) {
      acc = cfma(-c_sbp.left[DISC][rr][c], at(nr - 1 - c), acc);
    }
  } else {
#pragma unroll
    for (int k = T::HALF; k >= 1; --k) {
      acc = cfma(c_sbp.interior[DISC][k], csub(at(r + k), at(r - k)), acc);
    }
  }
  return acc;
}

template <int DISC, class Row>
__device__ __forceinline__ double2 ring_dissipation(const Row& at, const int r,
                                                    const int nr) {
  using T = DiscTraits<DISC>;
  double2 acc = make_double2(0.0, 0.0);
  if (r < T::SPECIAL) {
    for (int j = 0; j <= r + T::P; ++j) {
      acc = cfma(c_sbp.diss_left[DISC][r][j], at(j), acc);
    }
  } else if (r >= nr - T::SPECIAL) {
    const int rr = nr - 1 - r;
    for (int j = 0; j <= rr + T::P; ++j) {
      acc = cfma(c_sbp.diss_left[DISC][rr][j], at(nr - 1 - j), acc);
    }
  } else {
    acc = cscale(c_sbp.diss_interior[DISC][0], at(r));
#pragma unroll
    for (int k = 1; k <= T::P; ++k) {
      acc = cfma(c_sbp.diss_interior[DISC][k], cadd(at(r + k), at(r - k)), acc);
    }
  }
  return acc;
}

// Closure rows straight from a ring column: the first K rows (r < BR) or
// the last K rows (r >= nr - BR) of the radial line, K = SPECIAL + P (the
// widest closure stencil).  Two partial sums halve the dependency chain;
// table entries beyond a row's stencil are zero.
template <int DISC, class G = NarrowGeom>
__device__ __forceinline__ double2 edge_derivative(const double2* column,
                                                   const int r, const int nr,
                                                   const int shift,
                                                   const int stride) {
  using T = DiscTraits<DISC>;
  double2 a0 = make_double2(0.0, 0.0), a1 = a0;
  int rows[T::W];  // ring rows of the first / last W rows of the line
  if (r < T::BR) {
    ring_rows<G>(rows, 0, shift);
#pragma unroll
    for (int c = 0; c < T::W; ++c) {
      const double2 v = column[rows[c] * stride];
      if (c & 1) a1 = cfma(c_sbp.left[DISC][r][c], v, a1);
      else a0 = cfma(c_sbp.left[DISC][r][c], v, a0);
    }
  } else {
    const int rr = nr - 1 - r;
    ring_rows<G>(rows, nr - T::W, shift);
#pragma unroll
    for (int c = 0; c < T::W; ++c) {
      const double2 v = column[rows[T::W - 1 - c] * stride];  // row nr - 1 - c
      if (c & 1) a1 = cfma(-c_sbp.left[DISC][rr][c], v, a1);
      else a0 = cfma(-c_sbp.left[DISC][rr][c], v, a0);
    }
  }
  return cadd(a0, a1);
}

template <int DISC, class G = NarrowGeom>
__device__ __forceinline__ double2 edge_dissipation(const double2* column,
                                                    const int r, const int nr,
                                                    const int shift,
                                                    const int stride) {
  using T = DiscTraits<DISC>;
  constexpr int K = T::SPECIAL + T::P;
  double2 a0 = make_double2(0.0, 0.0), a1 = a0;
  const bool left = r < T::SPECIAL;
  const int rr = left ? r : nr - 1 - r;
  int rows[K];  // ring rows of the first / last K rows of the line
  ring_rows<G>(rows, left ? 0 : nr - K, shift);
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const double2 v = column[rows[left ? j : K - 1 - j] * stride];
    if (j & 1) a1 = cfma(c_sbp.diss_left[DISC][rr][j], v, a1);
    else a0 = cfma(c_sbp.diss_left[DISC][rr][j], v, a0);
  }
  return cadd(a0, a1);
}

// ------------------------------------------------------------- loader
// Issues the bulk copies of the CTA's chunk sequence (strips blockIdx.x,
// blockIdx.x + gridDim.x, ...; chunks of kStreamChunk rows each), one
// chunk per free ring stage.  Run by one thread.
template <int H, int HD, class G = NarrowGeom>
__device__ void loader_init(const StageLaunch& p, StreamLoaderState& L) {
  L.src_x = nullptr;
  L.src_a = nullptr;
  switch (p.stage) {
    case kStage2: L.src_u = p.y; L.src_x = p.kA; break;
    case kStage3: L.src_u = p.kB; L.src_x = p.y; L.src_a = p.acc; break;
    case kStage4: L.src_u = p.kA; L.src_a = p.acc; break;
    default: L.src_u = p.y; break;  // stage 1 and the RHS-only evaluation
  }
  L.strip = blockIdx.x;
  L.c = 0;
  L.g = 0;
  L.prev_rs = -1;
  if (L.strip < p.strip_count) L.sg = strip_geom<H, HD, G>(p, L.strip, 0);
}

// Load chunks while ring stages are free.  `released` = chunks handed back
// so far.  A strip with another row stride starts only on an empty ring
// (its rows would overlap the live stages' rows otherwise).
template <int H, int HD, class G = NarrowGeom>
__device__ void loader_pump(const StageLaunch& p, StreamLoaderState& state,
                            unsigned long long* full, double2* U, double2* X,
                            double2* A, double* CF, double* NI,
                            const int released) {
  if (state.strip >= p.strip_count || state.g >= released + G::kStages) {
    return;
  }
  // Every reader of a released stage finished before the release was
  // published; order those accesses before the copies' writes.
  __threadfence_block();
  fence_proxy_async_smem();
  StreamLoaderState L = state;
  while (L.strip < p.strip_count && L.g < released + G::kStages) {
    const StripGeom& sg = L.sg;
    if (L.c == 0 && L.prev_rs >= 0 && sg.rs != L.prev_rs && released < L.g) {
      break;
    }
    const int s = L.g % G::kStages;
    const int a0 = sg.s0 + L.c * G::kChunk;
    const int a1 = min(sg.s1, a0 + G::kChunk);
    const unsigned row_bytes = static_cast<unsigned>(sg.rs) * 16u;
    const unsigned bytes_u = static_cast<unsigned>(a1 - a0) * row_bytes;
    const unsigned bytes_x = L.src_x != nullptr ? bytes_u : 0u;
    const int o0 = max(a0, sg.r0), o1 = min(a1, sg.r1);
    // the accumulator rows of the outputs: into the A ring, or (WideGeom,
    // stage 4, where the X ring is free) into the X ring
    const bool a_rows =
        L.src_a != nullptr && o1 > o0 && (G::kRingA || p.stage == kStage4);
    const unsigned bytes_a =
        a_rows ? static_cast<unsigned>(o1 - o0) * row_bytes : 0u;
    const unsigned bytes_c =
        static_cast<unsigned>(a1 - a0) * kCoefCount * sizeof(double);
    const unsigned bytes_n = (G::kRingA && sg.kerr)
        ? static_cast<unsigned>(a1 - a0) * G::kNodeRec * sizeof(double)
        : 0u;
    const bool withheld = L.g == p.withhold_chunk && p.stage == kStage1 &&
                          blockIdx.x == 0;  // failure-detection test hook
    if (!withheld) {
      mbar_arrive_expect_tx(&full[s],
                            bytes_u + bytes_x + bytes_a + bytes_c + bytes_n);
      const long long gsrc = sg.seg_offset + static_cast<long long>(a0) * sg.rs;
      const int ra0 = ring_row<G>(a0, sg.shift);
      bulk_copy_g2s(U + ra0 * sg.rs, L.src_u + gsrc, bytes_u, &full[s]);
      if (bytes_x != 0u) {
        bulk_copy_g2s(X + ra0 * sg.rs, L.src_x + gsrc, bytes_x, &full[s]);
      }
      if (bytes_a != 0u) {
        bulk_copy_g2s((G::kRingA ? A : X) + ring_row<G>(o0, sg.shift) * sg.rs,
                      L.src_a + sg.seg_offset + static_cast<long long>(o0) * sg.rs,
                      bytes_a, &full[s]);
      }
      bulk_copy_g2s(CF + ra0 * kCoefCount,
                    p.coef_table +
                        static_cast<long long>(sg.coef_row0 + a0) * kCoefCount,
                    bytes_c, &full[s]);
      if (bytes_n != 0u) {
        bulk_copy_g2s(NI + ra0 * G::kNodeRec,
                      p.node_table + static_cast<long long>(sg.node_row0 + a0) *
                                         G::kNodeRec,
                      bytes_n, &full[s]);
      }
    }
    L.prev_rs = sg.rs;
    ++L.g;
    if (++L.c == sg.chunks) {
      L.c = 0;
      L.strip += gridDim.x;
      if (L.strip < p.strip_count) L.sg = strip_geom<H, HD, G>(p, L.strip, L.g);
    }
  }
  state = L;
}

// After an abort: copies still in flight land before the CTA exits.
template <class G = NarrowGeom>
__device__ void loader_drain(const StreamLoaderState& L,
                             unsigned long long* full) {
  for (int back = 1; back <= G::kStages && L.g - back >= 0; ++back) {
    const int gb = L.g - back;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(&full[gb % G::kStages],
                          static_cast<unsigned>(gb / G::kStages) & 1u)) {
      if (global_ns() - t0 > kStreamWaitNs) break;
    }
  }
}

// ------------------------------------------------------------- transforms
// Node fragments of one transform warp: synthesis node tiles 2h, 2h + 1,
// analysis ell tile h.
struct PsiFragments {
  double fs[2][4];  // S(j = (2h + i) * 8 + group, l = ks * 4 + quad)
  double fa[8];     // A(l = h * 8 + group, j = ks * 4 + quad)
  double gcos[2];   // 2 s a cos(theta_j)
};

// psi_t of the 4-row block at q0 (rows >= qlim skipped): this warp's half
// of the synthesis and of the analysis.  xw / tw are the block's staging
// buffers, shared with the partner warp; named barrier `bar` (one per
// block) synchronises the block's two warps between the phases.
template <int SC>
__device__ __forceinline__ void stream_psi_half(
    const int q0, const int qlim, const int h, const StripGeom& sg,
    const double2* U, const double2* QE, const double* CF, const double* NI,
    double2* PS, double* xw, double* tw, const PsiFragments& F,
    const int mts, const int ksa, const int bar, const int lane) {
  const int quad = lane & 3;
  const int group = lane >> 2;
  const int ne = sg.ne;
  const double mm = static_cast<double>(sg.m);
  {  // stage rows 2h, 2h + 1 of the block: v1 = P + 2K Q - G psi, psi
    const int rho = 2 * h + (lane >> 4);
    const int l = lane & 15;
    const int r = q0 + rho;
    double2 v1 = make_double2(0.0, 0.0), psi = make_double2(0.0, 0.0);
    if (r < qlim && l < ne) {
      const int rr = ring_row(r, sg.shift);
      const double* cf = CF + rr * kCoefCount;
      const double2* row = U + rr * sg.rs;
      const double2 Q = SC ? QE[rr * kStreamNep + l] : row[ne + l];
      psi = row[2 * ne + l];
      v1 = csub(cadd(row[l], cscale(2.0 * cf[1], Q)),
                cmul(make_double2(cf[3], mm * cf[4]), psi));
    }
    xw[(rho * 4 + 0) * kStreamXs + l] = v1.x;
    xw[(rho * 4 + 1) * kStreamXs + l] = v1.y;
    xw[(rho * 4 + 2) * kStreamXs + l] = psi.x;
    xw[(rho * 4 + 3) * kStreamXs + l] = psi.y;
  }
  named_sync(bar, 64);
  double bx[2][4];
#pragma unroll
  for (int n = 0; n < 2; ++n) {
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      bx[n][ks] = xw[(n * 8 + group) * kStreamXs + ks * 4 + quad];
    }
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int mt = 2 * h + i;
    if (mt < mts) {
      double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          dmma(acc[n][0], acc[n][1], F.fs[i][ks], bx[n][ks]);
        }
      }
      const int j = mt * 8 + group;
      double inv[2];  // 1 / C_T(r, theta_j); zero beyond the solve's nodes
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        const int r = q0 + 2 * n + (quad >> 1);
        inv[n] = r < qlim ? NI[ring_row(r, sg.shift) * kNodeRecord + j] : 0.0;
      }
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        // lane quad 0/2 holds a_j of a row, quad 1/3 holds b_j of that row
        const double o0 = __shfl_xor_sync(0xffffffffu, acc[n][0], 1);
        const double o1 = __shfl_xor_sync(0xffffffffu, acc[n][1], 1);
        if ((quad & 1) == 0) {
          const int rho = 2 * n + (quad >> 1);
          tw[(rho * 2 + 0) * kStreamTs + j] =
              (acc[n][0] + F.gcos[i] * o1) * inv[n];
          tw[(rho * 2 + 1) * kStreamTs + j] =
              (acc[n][1] - F.gcos[i] * o0) * inv[n];
        }
      }
    }
  }
  named_sync(bar, 64);
  double c[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
  for (int ks = 0; ks < 8; ++ks) {
    if (ks < ksa) {
      const double b = tw[group * kStreamTs + ks * 4 + quad];
      dmma(c[ks & 1][0], c[ks & 1][1], F.fa[ks], b);
    }
  }
  const int l = h * 8 + group;
  const int r = q0 + quad;
  if (r < qlim && l < ne) {
    PS[ring_row(r, sg.shift) * kStreamNep + l] =
        make_double2(c[0][0] + c[1][0], c[0][1] + c[1][1]);
  }
}

// Split-precision fragments of one transform warp (split_precision.cuh):
// BF16 digits of its synthesis node tile (nodes 16h .. 16h + 15, all ell)
// and of its half of the analysis K range (all ell, nodes 16h .. 16h + 15),
// with the power-of-two scales of those matrix rows.
struct SplitFragments {
  unsigned s[split::kSlices][4];  // synthesis A operand: S(j, l)
  unsigned a[split::kSlices][4];  // analysis A operand: A(l, j)
  double node_scale[2];           // 2^(F_j - 14), j = 16h + grp, 16h + grp + 8
  double ell_scale[2];            // 2^(F_l - 14), l = grp, grp + 8
  double gcos[2];                 // 2 s a cos(theta_j), the same two nodes
};

// Split-precision digits of a B operand column held by a lane quad: the
// four values of this lane, scaled by the quad's common power of two.
__device__ __forceinline__ int split_column(const double (&v)[4],
                                            uint2 (&b)[split::kSlices]) {
  double m = fmax(fmax(fabs(v[0]), fabs(v[1])), fmax(fabs(v[2]), fabs(v[3])));
  m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 1));
  m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 2));
  const int e = split::exponent(m);
  const double down = ldexp(1.0, -e);
  float t[4][split::kSlices];
#pragma unroll
  for (int i = 0; i < 4; ++i) split::digits(v[i] * down, t[i]);
#pragma unroll
  for (int s = 0; s < split::kSlices; ++s) {
    b[s].x = split::pack(t[0][s], t[1][s]);
    b[s].y = split::pack(t[2][s], t[3][s]);
  }
  return e;
}

// The 15 digit-pair products of one m16n8k16 tile into five accumulators.
__device__ __forceinline__ void split_products(
    float (&d)[split::kSlices][4], const unsigned (&a)[split::kSlices][4],
    const uint2 (&b)[split::kSlices]) {
#pragma unroll
  for (int u = 0; u < split::kSlices; ++u) d[u][0] = d[u][1] = d[u][2] = d[u][3] = 0.0f;
#pragma unroll
  for (int s = 0; s < split::kSlices; ++s) {
#pragma unroll
    for (int t = 0; s + t < split::kSlices; ++t) split::mma_bf16(d[s + t], a[s], b[t]);
  }
}

// psi_t of the 4-row block at q0 in split precision: the same staging,
// pointwise step and outputs as stream_psi_half.  Synthesis: this warp's
// 16 nodes x 16 columns (rows x {v1, psi} x {re, im}) over K = 16 ell, two
// m16n8k16 tiles.  Analysis: all 16 ell x 8 columns over K = this warp's 16
// nodes, one tile; the two warps' partial sums are added through the
// block's exchange buffer `ex` (two parities, so no extra barrier).
template <int SC>
__device__ __forceinline__ void stream_psi_split(
    const int q0, const int qlim, const int h, const StripGeom& sg,
    const double2* U, const double2* QE, const double* CF, const double* NI,
    double2* PS, double* xw, double* tw, double* ex, const SplitFragments& F,
    const int mts, const int bar, const int lane) {
  const int quad = lane & 3;
  const int group = lane >> 2;
  const int ne = sg.ne;
  const double mm = static_cast<double>(sg.m);
  {  // stage rows 2h, 2h + 1 of the block: v1 = P + 2K Q - G psi, psi
    const int rho = 2 * h + (lane >> 4);
    const int l = lane & 15;
    const int r = q0 + rho;
    double2 v1 = make_double2(0.0, 0.0), psi = make_double2(0.0, 0.0);
    if (r < qlim && l < ne) {
      const int rr = ring_row(r, sg.shift);
      const double* cf = CF + rr * kCoefCount;
      const double2* row = U + rr * sg.rs;
      const double2 Q = SC ? QE[rr * kStreamNep + l] : row[ne + l];
      psi = row[2 * ne + l];
      v1 = csub(cadd(row[l], cscale(2.0 * cf[1], Q)),
                cmul(make_double2(cf[3], mm * cf[4]), psi));
    }
    xw[(rho * 4 + 0) * kStreamXs + l] = v1.x;
    xw[(rho * 4 + 1) * kStreamXs + l] = v1.y;
    xw[(rho * 4 + 2) * kStreamXs + l] = psi.x;
    xw[(rho * 4 + 3) * kStreamXs + l] = psi.y;
  }
  named_sync(bar, 64);
  // synthesis: acc[i][n][c] = C(node 16h + group + 8i, column n * 8 + 2 quad + c)
  double acc[2][2][2];
#pragma unroll
  for (int n = 0; n < 2; ++n) {
    double v[4];
    const double* col = xw + (n * 8 + group) * kStreamXs;
    v[0] = col[2 * quad];
    v[1] = col[2 * quad + 1];
    v[2] = col[2 * quad + 8];
    v[3] = col[2 * quad + 9];
    uint2 b[split::kSlices];
    const int e = split_column(v, b);  // scale of column n * 8 + group
    float d[split::kSlices][4];
    split_products(d, F.s, b);
    const double c0 = ldexp(1.0, __shfl_sync(0xffffffffu, e, 8 * quad));
    const double c1 = ldexp(1.0, __shfl_sync(0xffffffffu, e, 8 * quad + 4));
    acc[0][n][0] = split::recombine(d, 0) * F.node_scale[0] * c0;
    acc[0][n][1] = split::recombine(d, 1) * F.node_scale[0] * c1;
    acc[1][n][0] = split::recombine(d, 2) * F.node_scale[1] * c0;
    acc[1][n][1] = split::recombine(d, 3) * F.node_scale[1] * c1;
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int mt = 2 * h + i;
    if (mt < mts) {
      const int j = mt * 8 + group;
      double inv[2];  // 1 / C_T(r, theta_j); zero beyond the solve's nodes
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        const int r = q0 + 2 * n + (quad >> 1);
        inv[n] = r < qlim ? NI[ring_row(r, sg.shift) * kNodeRecord + j] : 0.0;
      }
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        // lane quad 0/2 holds a_j of a row, quad 1/3 holds b_j of that row
        const double o0 = __shfl_xor_sync(0xffffffffu, acc[i][n][0], 1);
        const double o1 = __shfl_xor_sync(0xffffffffu, acc[i][n][1], 1);
        if ((quad & 1) == 0) {
          const int rho = 2 * n + (quad >> 1);
          tw[(rho * 2 + 0) * kStreamTs + j] =
              (acc[i][n][0] + F.gcos[i] * o1) * inv[n];
          tw[(rho * 2 + 1) * kStreamTs + j] =
              (acc[i][n][1] - F.gcos[i] * o0) * inv[n];
        }
      }
    }
  }
  named_sync(bar, 64);
  // analysis partial: C(ell group + 8i, column 2 quad + c) over this warp's
  // nodes
  double part[4];
  {
    double v[4];
    const double* col = tw + group * kStreamTs + 16 * h;
    v[0] = col[2 * quad];
    v[1] = col[2 * quad + 1];
    v[2] = col[2 * quad + 8];
    v[3] = col[2 * quad + 9];
    uint2 b[split::kSlices];
    const int e = split_column(v, b);
    float d[split::kSlices][4];
    split_products(d, F.a, b);
    const double c0 = ldexp(1.0, __shfl_sync(0xffffffffu, e, 8 * quad));
    const double c1 = ldexp(1.0, __shfl_sync(0xffffffffu, e, 8 * quad + 4));
    part[0] = split::recombine(d, 0) * F.ell_scale[0] * c0;
    part[1] = split::recombine(d, 1) * F.ell_scale[0] * c1;
    part[2] = split::recombine(d, 2) * F.ell_scale[1] * c0;
    part[3] = split::recombine(d, 3) * F.ell_scale[1] * c1;
  }
  // warp 0 finishes ell = group, warp 1 ell = group + 8: each hands the
  // other half to its partner
  double* mine = ex + (h * 32 + lane) * 2;
  double* theirs = ex + ((1 - h) * 32 + lane) * 2;
  mine[0] = h == 0 ? part[2] : part[0];
  mine[1] = h == 0 ? part[3] : part[1];
  named_sync(bar, 64);
  const double s0 = (h == 0 ? part[0] : part[2]) + theirs[0];
  const double s1 = (h == 0 ? part[1] : part[3]) + theirs[1];
  const int l = group + 8 * h;
  const int r = q0 + quad;
  if (r < qlim && l < ne) {
    PS[ring_row(r, sg.shift) * kStreamNep + l] = make_double2(s0, s1);
  }
}

template <int DISC, int SC, int PREC, int STAGE = 0>
__device__ void stream_transform(const StageLaunch& p,
                                 unsigned long long* full,
                                 unsigned long long* ready,
                                 volatile int* abort_flag, double2* U,
                                 const double2* X, double2* PS, double2* QE,
                                 const double* CF, const double* NI,
                                 double* xw_all, double* tw_all,
                                 double* ex_all, const int tt) {
  using T = DiscTraits<DISC>;
  constexpr int P = T::P, HD = T::HALF;
  constexpr int H = SC ? (P > 2 * HD ? P : 2 * HD) : P;
  const int warp = tt >> 5, lane = tt & 31;
  const int quad = lane & 3, group = lane >> 2;
  const int blk = warp >> 1, h = warp & 1;
  double* xw = xw_all + blk * 16 * kStreamXs;
  double* tw = tw_all + blk * 8 * kStreamTs;
  // zero the nodal staging once: columns beyond a solve's nodes stay zero
  for (int i = tt; i < kStreamBlocks * 8 * kStreamTs; i += kStreamTThreads) {
    tw_all[i] = 0.0;
  }

  int g = 0;
  for (int strip = blockIdx.x; strip < p.strip_count; strip += gridDim.x) {
    const StripGeom sg = strip_geom<H, HD>(p, strip, g);
    const InstanceDesc& in = p.instances[sg.instance];
    const int nt = in.ntheta, ne = sg.ne, nr = sg.nr;
    const bool kerr = in.spin != 0.0;
    const double hdt = 0.5 * in.dt;
    const double inv_h = in.inv_spacing;
    const double mm = static_cast<double>(sg.m);
    PsiFragments F;
    SplitFragments G;
    const int mts = (nt + 7) / 8, ksa = (nt + 3) / 4;
    if (kerr && PREC == 1) {
      // digit fragments of this segment: [h][slice][lane] uint4 for the
      // synthesis, then the same for the analysis; 48 scales
      const uint4* fr = p.split_frags + static_cast<long long>(sg.segment) * kSplitRecord;
#pragma unroll
      for (int sl = 0; sl < split::kSlices; ++sl) {
        const uint4 fs = fr[(h * split::kSlices + sl) * 32 + lane];
        const uint4 fa = fr[((2 + h) * split::kSlices + sl) * 32 + lane];
        G.s[sl][0] = fs.x; G.s[sl][1] = fs.y; G.s[sl][2] = fs.z; G.s[sl][3] = fs.w;
        G.a[sl][0] = fa.x; G.a[sl][1] = fa.y; G.a[sl][2] = fa.z; G.a[sl][3] = fa.w;
      }
      const double* sc = p.split_scales + static_cast<long long>(sg.segment) * kSplitScales;
      const double sa2 = 2.0 * (static_cast<double>(kSpinWeight) * in.spin);
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int j = 16 * h + group + 8 * i;
        G.node_scale[i] = sc[j];
        G.ell_scale[i] = sc[kStreamMaxTheta + group + 8 * i];
        G.gcos[i] = j < nt ? sa2 * p.trig[in.trig_offset + nt + j] : 0.0;
      }
    } else if (kerr) {
      const SegmentDesc& seg = p.segments[sg.segment];
      const double* St = p.matrices + seg.mat_offset;  // St[l][j]
      const double* At = St + ne * nt;                 // At[j][l]
      const double sa2 = 2.0 * (static_cast<double>(kSpinWeight) * in.spin);
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int j = (2 * h + i) * 8 + group;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
          const int l = ks * 4 + quad;
          F.fs[i][ks] = (j < nt && l < ne) ? St[l * nt + j] : 0.0;
        }
        F.gcos[i] = j < nt ? sa2 * p.trig[in.trig_offset + nt + j] : 0.0;
      }
      const int l = h * 8 + group;
#pragma unroll
      for (int ks = 0; ks < 8; ++ks) {
        const int j = ks * 4 + quad;
        F.fa[ks] = (j < nt && l < ne) ? At[j * ne + l] : 0.0;
      }
    }
    int pd = sg.t0;  // psi_t rows done
    for (int c = 0; c < sg.chunks; ++c, ++g) {
      const int s = g % kStreamStages;
      const unsigned parity = static_cast<unsigned>(g / kStreamStages) & 1u;
      // every transform thread waits; all of them leave together on abort
      const bool landed = stream_wait(&full[s], parity, abort_flag, p.error, 3);
      if (!named_sync_and(1, kStreamTThreads, landed)) return;
      const int a0 = sg.s0 + c * kStreamChunk;
      const int a1 = min(sg.s1, a0 + kStreamChunk);
      // stage input u = y + dt/2 k, in place
      constexpr bool kFixed = STAGE != 0;
      const int stage = kFixed ? STAGE : p.stage;
      if (stage == kStage2 || stage == kStage3) {
        const int base = ring_row(a0, sg.shift) * sg.rs;
        const int count = (a1 - a0) * sg.rs;
        double2* u = U + base;
        const double2* x = X + base;
        if (stage == kStage2) {  // U = y, X = k1
          for (int i = tt; i < count; i += kStreamTThreads) {
            u[i] = cfma(hdt, x[i], u[i]);
          }
        } else {  // U = k2, X = y
          for (int i = tt; i < count; i += kStreamTThreads) {
            u[i] = cfma(hdt, u[i], x[i]);
          }
        }
        named_sync(1, kStreamTThreads);
      }
      int pe;
      if (SC) {
        // effective Q = D psi on rows [pd, qe)
        const int qe = min(sg.t1, computable_end(a1, nr, T::HALF, T::W, T::BR));
        const int items = max(0, qe - pd) * kStreamNep;
        for (int i = tt; i < items; i += kStreamTThreads) {
          const int r = pd + i / kStreamNep;
          const int l = i % kStreamNep;
          if (l < ne) {
            const double2* col = U + 2 * ne + l;
            const int shift = sg.shift, rs = sg.rs;
            auto at = [=](const int q) { return col[ring_row(q, shift) * rs]; };
            QE[ring_row(r, sg.shift) * kStreamNep + l] =
                cscale(inv_h, ring_derivative<DISC>(at, r, nr));
          }
        }
        named_sync(1, kStreamTThreads);
        pe = qe;
      } else {
        pe = min(sg.t1, a1);
      }
      if (pe > pd) {
        if (kerr && PREC == 1) {
          for (int q = pd; q < pe; q += 4 * kStreamBlocks) {
            stream_psi_split<SC>(q + 4 * blk, pe, h, sg, U, QE, CF, NI, PS, xw,
                                 tw, ex_all + blk * 128, G, mts,
                                 kStreamBlockBar + blk, lane);
          }
        } else if (kerr) {
          for (int q = pd; q < pe; q += 4 * kStreamBlocks) {
            stream_psi_half<SC>(q + 4 * blk, pe, h, sg, U, QE, CF, NI, PS, xw,
                                tw, F, mts, ksa, kStreamBlockBar + blk, lane);
          }
        } else {
          const int items = (pe - pd) * kStreamNep;
          for (int i = tt; i < items; i += kStreamTThreads) {
            const int r = pd + i / kStreamNep;
            const int l = i % kStreamNep;
            if (l < ne) {
              const int rr = ring_row(r, sg.shift);
              const double* cf = CF + rr * kCoefCount;
              const double2* row = U + rr * sg.rs;
              const double2 Q = SC ? QE[rr * kStreamNep + l] : row[ne + l];
              const double2 psi = row[2 * ne + l];
              const double2 num =
                  csub(cadd(row[l], cscale(2.0 * cf[1], Q)),
                       cmul(make_double2(cf[3], mm * cf[4]), psi));
              PS[rr * kStreamNep + l] = cscale(cf[9], num);
            }
          }
        }
        pd = pe;
      }
      // the combine wrote ring rows that later bulk copies overwrite
      fence_proxy_async_smem();
      mbar_arrive(&ready[s]);
    }
  }
}

// ------------------------------------------------------------- stencils
// RK update of field f of one row from the stage slope k (global stores).
// (WideGeom: with `pre` the caller loaded this entry's accumulator value
// `a_pre` ahead, else it is read from global memory here.)
// (STAGE: the stage as a compile-time constant, 0: read p.stage)
template <class G = NarrowGeom, int STAGE = 0>
__device__ __forceinline__ void stream_rk_update(
    const StageLaunch& p, const StripGeom& sg, const double2* X,
    const double2* A, const long long gi, const int ri, const double2 k,
    const double dt, const double dt6, const bool pre = false,
    const double2 a_pre = make_double2(0.0, 0.0)) {
  switch (STAGE != 0 ? STAGE : p.stage) {
    case kStage2:  // X = k1
      p.kB[gi] = k;
      p.acc[gi] = cfma(2.0, k, X[ri]);
      break;
    case kStage3: {  // X = y, A = k1 + 2 k2
      const double2 y0 = X[ri];
      const double2 a = G::kRingA ? A[ri] : (pre ? a_pre : p.acc[gi]);
      p.acc[gi] = cfma(dt6, cfma(2.0, k, a), y0);
      p.kA[gi] = cfma(dt, k, y0);
      break;
    }
    case kStage4:  // A (WideGeom: X) = y + dt/6 (k1 + 2 k2 + 2 k3)
      p.y[gi] = cfma(dt6, k, G::kRingA ? A[ri] : X[ri]);
      break;
    default:  // stage 1 and the RHS-only evaluation
      p.kA[gi] = k;
      break;
  }
}

// Interior-row terms of the Teukolsky RHS: centre values, dissipation sums
// (centre tap first, then k = P..1) and derivative sums (k = HALF..1).
// A row gets the same sums, in the same order, alone or in a pair.
struct StencilTerms {
  double2 psi, Q, pt, qe;  // qe: effective Q (stage-constrained)
  double2 spsi, sQ, sP;    // dissipation sums
  double2 dpsi, dq, dpt;   // derivative sums (dq: of Q or of the effective Q)
};

template <int DISC, int N>
__device__ __forceinline__ double2 taps_dissipation(const double2 (&w)[N],
                                                    const int c) {
  using T = DiscTraits<DISC>;
  double2 acc = cscale(c_sbp.diss_interior[DISC][0], w[c]);
#pragma unroll
  for (int k = T::P; k >= 1; --k) {
    acc = cfma(c_sbp.diss_interior[DISC][k], cadd(w[c + k], w[c - k]), acc);
  }
  return acc;
}

template <int DISC, int N>
__device__ __forceinline__ double2 taps_derivative(const double2 (&w)[N],
                                                   const int c) {
  using T = DiscTraits<DISC>;
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int k = T::HALF; k >= 1; --k) {
    acc = cfma(c_sbp.interior[DISC][k], csub(w[c + k], w[c - k]), acc);
  }
  return acc;
}

// Terms of interior rows r and r + 1: one window of 2P + 2 ring rows per
// field serves both rows (12 of the 14 rows overlap for D10-5).
template <int DISC, int SC, class G = NarrowGeom>
__device__ __forceinline__ void pair_terms(
    StencilTerms (&t)[2], const double2* cpsi, const double2* cQ,
    const double2* cP, const double2* cpt, const double2* cqe, const int r,
    const int shift, const int rs) {
  using T = DiscTraits<DISC>;
  constexpr int P = T::P, HD = T::HALF, N = 2 * P + 2, M = 2 * HD + 2;
  int rows[N];
  ring_rows<G>(rows, r - P, shift);
  {
    double2 w[N];
#pragma unroll
    for (int i = 0; i < N; ++i) w[i] = cpsi[rows[i] * rs];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      t[j].psi = w[P + j];
      t[j].spsi = taps_dissipation<DISC>(w, P + j);
      t[j].dpsi = taps_derivative<DISC>(w, P + j);
    }
  }
  {
    double2 w[N];
#pragma unroll
    for (int i = 0; i < N; ++i) w[i] = cQ[rows[i] * rs];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      t[j].Q = w[P + j];
      t[j].sQ = taps_dissipation<DISC>(w, P + j);
      if (!SC) t[j].dq = taps_derivative<DISC>(w, P + j);
    }
  }
  {
    double2 w[N];
#pragma unroll
    for (int i = 0; i < N; ++i) w[i] = cP[rows[i] * rs];
#pragma unroll
    for (int j = 0; j < 2; ++j) t[j].sP = taps_dissipation<DISC>(w, P + j);
  }
  {
    double2 w[M];
#pragma unroll
    for (int i = 0; i < M; ++i) w[i] = cpt[rows[P - HD + i] * G::kNep];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      t[j].pt = w[HD + j];
      t[j].dpt = taps_derivative<DISC>(w, HD + j);
    }
  }
  if (SC) {
    double2 w[M];
#pragma unroll
    for (int i = 0; i < M; ++i) w[i] = cqe[rows[P - HD + i] * G::kNep];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      t[j].qe = w[HD + j];
      t[j].dq = taps_derivative<DISC>(w, HD + j);
    }
  } else {
    t[0].qe = t[1].qe = make_double2(0.0, 0.0);
  }
}

// Terms of one interior row (the same sums as pair_terms gives it).
template <int DISC, int SC, class G = NarrowGeom>
__device__ __forceinline__ void row_terms(
    StencilTerms& t, const double2* cpsi, const double2* cQ,
    const double2* cP, const double2* cpt, const double2* cqe, const int r,
    const int shift, const int rs) {
  using T = DiscTraits<DISC>;
  constexpr int P = T::P, HD = T::HALF, N = 2 * P + 1, M = 2 * HD + 1;
  int rows[N];
  ring_rows<G>(rows, r - P, shift);
  {
    double2 w[N];
#pragma unroll
    for (int i = 0; i < N; ++i) w[i] = cpsi[rows[i] * rs];
    t.psi = w[P];
    t.spsi = taps_dissipation<DISC>(w, P);
    t.dpsi = taps_derivative<DISC>(w, P);
  }
  {
    double2 w[N];
#pragma unroll
    for (int i = 0; i < N; ++i) w[i] = cQ[rows[i] * rs];
    t.Q = w[P];
    t.sQ = taps_dissipation<DISC>(w, P);
    if (!SC) t.dq = taps_derivative<DISC>(w, P);
  }
  {
    double2 w[N];
#pragma unroll
    for (int i = 0; i < N; ++i) w[i] = cP[rows[i] * rs];
    t.sP = taps_dissipation<DISC>(w, P);
  }
  {
    double2 w[M];
#pragma unroll
    for (int i = 0; i < M; ++i) w[i] = cpt[rows[P - HD + i] * G::kNep];
    t.pt = w[HD];
    t.dpt = taps_derivative<DISC>(w, HD);
  }
  if (SC) {
    double2 w[M];
#pragma unroll
    for (int i = 0; i < M; ++i) w[i] = cqe[rows[P - HD + i] * G::kNep];
    t.qe = w[HD];
    t.dq = taps_derivative<DISC>(w, HD);
  } else {
    t.qe = make_double2(0.0, 0.0);
  }
}

// RHS of an interior row from its terms: psi -> D psi (constraint),
// dissipation, (c_psi + lambda) psi; psi_t -> D psi_t into Q_t, psi_t
// itself; Q -> -gamma Q, dissipation, H_R D Q + q Q with Q the evolved Q
// (free-damped) or the effective Q (stage-constrained); P -> dissipation.
template <int SC>
__device__ __forceinline__ void assemble_interior(
    const StencilTerms& t, const double* cf, const double mm,
    const double lambda, const double damping, const double inv_h,
    const double diss_scale, const bool dissipate, double2& kP, double2& kQ,
    double2& kpsi) {
  kQ = cscale(damping, cscale(inv_h, t.dpsi));
  kpsi = dissipate ? cscale(diss_scale, t.spsi) : make_double2(0.0, 0.0);
  kP = cadd(cmul(make_double2(cf[7], mm * cf[8]), t.psi),
            cscale(lambda, t.psi));
  kQ = cadd(kQ, cscale(inv_h, t.dpt));
  kpsi = cadd(kpsi, t.pt);
  kQ = csub(kQ, cscale(damping, t.Q));
  if (dissipate) kQ = cfma(diss_scale, t.sQ, kQ);
  const double2 qp = SC ? t.qe : t.Q;
  kP = cadd(kP, cadd(cscale(cf[2], cscale(inv_h, t.dq)),
                     cmul(make_double2(cf[5], mm * cf[6]), qp)));
  if (dissipate) kP = cfma(diss_scale, t.sP, kP);
}

// One thread per (output row pair, ell): all three fields of two adjacent
// rows, no exchange.
template <int DISC, int SC, class G = NarrowGeom, int STAGE = 0>
__device__ void stream_stencil(const StageLaunch& p,
                               unsigned long long* ready,
                               volatile int* abort_flag,
                               volatile int* released, const double2* U,
                               const double2* X, const double2* A,
                               const double2* PS, const double2* QE,
                               const double* CF, const int st) {
  using T = DiscTraits<DISC>;
  constexpr int P = T::P, HD = T::HALF;
  constexpr int H = SC ? (P > 2 * HD ? P : 2 * HD) : P;
  const int pair = st / G::kNep;  // row pair of a pass of 2 kPairs rows
  const int l = st % G::kNep;
  // threads beyond kPairs pairs (wide geometry) take no rows
  const bool worker = G::kPairs * G::kNep == kStreamSThreads || pair < G::kPairs;
  int g = 0;
  int published = 0;  // chunks handed back so far
  // one strip, with the dissipation switch a compile-time constant (false:
  // the CTA is aborting)
  auto run_strip = [&](const int strip, auto dissipation) -> bool {
    constexpr bool dissipate = decltype(dissipation)::value;
    const int g0 = g;
    const StripGeom sg = strip_geom<H, HD, G>(p, strip, g0);
    const InstanceDesc& in = p.instances[sg.instance];
    const int ne = sg.ne, nr = sg.nr, rs = sg.rs;
    const double inv_h = in.inv_spacing;
    const double diss_scale = in.dissipation * inv_h;
    const double damping = in.damping;
    const double dt = in.dt, dt6 = in.dt / 6.0;
    const double mm = static_cast<double>(sg.m);
    const int ell = (l < ne) ? (p.segments[sg.segment].ell_min + l) : 0;
    const double lambda = -static_cast<double>((ell - kSpinWeight) *
                                               (ell + kSpinWeight + 1));
    const double2* cP = U + l;
    const double2* cQ = U + ne + l;
    const double2* cpsi = U + 2 * ne + l;
    const double2* cpt = PS + l;
    const double2* cqe = QE + l;
    int out_done = sg.r0;
    int rel = g0;  // next chunk of this strip to hand back
    for (int c = 0; c < sg.chunks; ++c, ++g) {
      const int s = g % G::kStages;
      const bool done =
          stream_wait(&ready[s], static_cast<unsigned>(g / G::kStages) & 1u,
                      abort_flag, p.error, 4);
      if (!named_sync_and(2, kStreamSThreads, done)) return false;
      const int u_end = min(sg.s1, sg.s0 + (c + 1) * G::kChunk);
      int lim = min(sg.r1, computable_end(u_end, nr, T::P, T::SPECIAL + T::P,
                                          T::SPECIAL));
      lim = min(lim, computable_end(u_end, nr, T::HALF, T::W, T::BR));
      int pe;
      if (SC) {
        const int qe =
            min(sg.t1, computable_end(u_end, nr, T::HALF, T::W, T::BR));
        lim = min(lim, computable_end(qe, nr, T::HALF, T::W, T::BR));
        pe = qe;
      } else {
        pe = min(sg.t1, u_end);
      }
      lim = min(lim, computable_end(pe, nr, T::HALF, T::W, T::BR));
      for (int r = out_done + 2 * pair; worker && r < lim;
           r += 2 * G::kPairs) {
        if (l >= ne) continue;
        const int count = r + 1 < lim ? 2 : 1;  // rows r, r + 1 of this pass
        // RK update of row q (ring row rq) from its three slopes (pre: the
        // row's accumulator values a0, a1, a2 were loaded ahead)
        auto update_at = [&](const int q, const int rq, const double2 kP,
                             const double2 kQ, const double2 kpsi,
                             const bool pre = false,
                             const double2 a0 = make_double2(0.0, 0.0),
                             const double2 a1 = make_double2(0.0, 0.0),
                             const double2 a2 = make_double2(0.0, 0.0)) {
          const long long gi =
              sg.seg_offset + static_cast<long long>(q) * rs + l;
          const int ri = rq * rs + l;
          stream_rk_update<G, STAGE>(p, sg, X, A, gi, ri, kP, dt, dt6, pre,
                                     a0);
          stream_rk_update<G, STAGE>(p, sg, X, A, gi + ne, ri + ne, kQ, dt,
                                     dt6, pre, a1);
          stream_rk_update<G, STAGE>(p, sg, X, A, gi + 2 * ne, ri + 2 * ne,
                                     kpsi, dt, dt6, pre, a2);
        };
        auto update = [&](const int q, const double2 kP, const double2 kQ,
                          const double2 kpsi) {
          update_at(q, ring_row<G>(q, sg.shift), kP, kQ, kpsi);
        };
        if (count == 2 && r >= T::BR && r + 1 + T::BR < nr) {
          // two interior rows from one register window per field
          double2 acc_pre[2][3];  // wide: the accumulator values, loaded ahead
          const bool pre =
              !G::kRingA && (STAGE != 0 ? STAGE : p.stage) == kStage3;
          if constexpr (!G::kRingA) {
            if (pre) {
              const long long gi = sg.seg_offset + static_cast<long long>(r) * rs + l;
#pragma unroll
              for (int j = 0; j < 2; ++j) {
#pragma unroll
                for (int f = 0; f < 3; ++f) {
                  acc_pre[j][f] = __ldcs(p.acc + gi + j * rs + f * ne);
                }
              }
            }
          }
          StencilTerms t[2];
          pair_terms<DISC, SC, G>(t, cpsi, cQ, cP, cpt, cqe, r, sg.shift, rs);
          int rq[2];  // ring rows of r, r + 1
          ring_rows<G>(rq, r, sg.shift);
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            double2 kP, kQ, kpsi;
            assemble_interior<SC>(t[j], CF + rq[j] * kCoefCount, mm, lambda,
                                  damping, inv_h, diss_scale, dissipate, kP,
                                  kQ, kpsi);
            update_at(r + j, rq[j], kP, kQ, kpsi, pre, acc_pre[j][0],
                      acc_pre[j][1], acc_pre[j][2]);
          }
          continue;
        }
#pragma unroll 1
        for (int q = r; q < r + count; ++q) {
          const int rr = ring_row<G>(q, sg.shift);
          const double* cf = CF + rr * kCoefCount;
          double2 kP, kQ, kpsi;
          if (q >= T::BR && q + T::BR < nr) {
            StencilTerms t;
            row_terms<DISC, SC, G>(t, cpsi, cQ, cP, cpt, cqe, q, sg.shift, rs);
            assemble_interior<SC>(t, cf, mm, lambda, damping, inv_h,
                                  diss_scale, dissipate, kP, kQ, kpsi);
          } else {  // closure rows
            const double2 psi = cpsi[rr * rs];
            const double2 Q = cQ[rr * rs];
            kQ = cadd(cscale(damping, cscale(inv_h, edge_derivative<DISC, G>(
                                                        cpsi, q, nr, sg.shift, rs))),
                      cscale(inv_h, edge_derivative<DISC, G>(cpt, q, nr, sg.shift,
                                                             G::kNep)));
            kQ = csub(kQ, cscale(damping, Q));
            kpsi = cpt[rr * G::kNep];
            kP = cadd(cmul(make_double2(cf[7], mm * cf[8]), psi),
                      cscale(lambda, psi));
            const double2 qp = SC ? cqe[rr * G::kNep] : Q;
            const double2 dq =
                SC ? edge_derivative<DISC, G>(cqe, q, nr, sg.shift, G::kNep)
                   : edge_derivative<DISC, G>(cQ, q, nr, sg.shift, rs);
            kP = cadd(kP, cadd(cscale(cf[2], cscale(inv_h, dq)),
                               cmul(make_double2(cf[5], mm * cf[6]), qp)));
            if (dissipate) {
              kpsi = cfma(diss_scale,
                          edge_dissipation<DISC, G>(cpsi, q, nr, sg.shift, rs), kpsi);
              kQ = cfma(diss_scale,
                        edge_dissipation<DISC, G>(cQ, q, nr, sg.shift, rs), kQ);
              kP = cfma(diss_scale,
                        edge_dissipation<DISC, G>(cP, q, nr, sg.shift, rs), kP);
            }
          }
          update(q, kP, kQ, kpsi);
        }
      }
      out_done = max(out_done, lim);
      // rows below `bound` are read by no later work of this strip
      int bound;
      if (c == sg.chunks - 1) {
        bound = 1 << 30;
      } else if (out_done < T::BR) {
        bound = 0;
      } else {
        bound = min(out_done - H, nr - T::SPECIAL - T::P);
      }
      while (rel <= g &&
             min(sg.s1, sg.s0 + (rel - g0 + 1) * G::kChunk) <= bound) {
        ++rel;
      }
      if (rel > published) {  // the same decision in every stencil thread
        named_sync(2, kStreamSThreads);  // every read of those rows is done
        if (st == 0) *released = rel;
        published = rel;
      }
    }
    return true;
  };
  for (int strip = blockIdx.x; strip < p.strip_count; strip += gridDim.x) {
    const int instance = p.segments[p.strips[strip].segment].instance;
    const bool ok = p.instances[instance].dissipation > 0.0
                        ? run_strip(strip, std::true_type{})
                        : run_strip(strip, std::false_type{});
    if (!ok) return;
  }
}

// Registers per thread of the calling warpgroup: raised or lowered from
// the launch's allocation (setmaxnreg.inc only raises, .dec only lowers).
template <int N>
__device__ __forceinline__ void set_max_registers() {
  static_assert(N % 8 == 0 && N >= 24 && N <= 256, "setmaxnreg range");
  if constexpr (N > kStreamLaunchRegs) {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" : : "n"(N));
  } else {  // also at N == launch: every warpgroup sets its count
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" : : "n"(N));
  }
}

// Producer: issues every chunk's copies as soon as its stage is free.
template <int H, int HD, class G = NarrowGeom>
__device__ void stream_producer(const StageLaunch& p, StreamLoaderState& L,
                                unsigned long long* full, double2* U,
                                double2* X, double2* A, double* CF,
                                double* NI, volatile int* released,
                                volatile int* abort_flag) {
  loader_init<H, HD, G>(p, L);
  unsigned long long t_last = global_ns();
  while (L.strip < p.strip_count) {
    const int before = L.g;
    loader_pump<H, HD, G>(p, L, full, U, X, A, CF, NI, *released);
    if (L.g != before) {
      t_last = global_ns();
      continue;
    }
    if (*abort_flag != 0) break;
    if (global_ns() - t_last > kStreamWaitNs) {
      *abort_flag = 1;
      if (p.error != nullptr) atomicExch(p.error, 5);
      break;
    }
    __nanosleep(128);
  }
  if (*abort_flag != 0) loader_drain<G>(L, full);
}

// STAGE: p.stage as a compile-time constant (the RK update's branch).
template <int DISC, int SC, int PREC, int STAGE>
__global__ void __launch_bounds__(kStreamThreads, 1)
    stream_stage_kernel(const StageLaunch p) {
  extern __shared__ __align__(128) unsigned char stream_smem[];
  const StreamLayout Ls(SC);
  unsigned long long* full =
      reinterpret_cast<unsigned long long*>(stream_smem + Ls.bars);
  unsigned long long* ready = full + kStreamStages;
  volatile int* abort_flag =
      reinterpret_cast<volatile int*>(ready + kStreamStages);
  volatile int* released = abort_flag + 1;  // chunks the stencils are done with
  StreamLoaderState& loader =
      *reinterpret_cast<StreamLoaderState*>(stream_smem + Ls.loader);
  double2* U = reinterpret_cast<double2*>(stream_smem + Ls.uring);
  double2* X = reinterpret_cast<double2*>(stream_smem + Ls.xring);
  double2* A = reinterpret_cast<double2*>(stream_smem + Ls.aring);
  double2* PS = reinterpret_cast<double2*>(stream_smem + Ls.pring);
  double2* QE = reinterpret_cast<double2*>(stream_smem + Ls.qring);
  double* CF = reinterpret_cast<double*>(stream_smem + Ls.coef);
  double* NI = reinterpret_cast<double*>(stream_smem + Ls.nodes);
  double* xw = reinterpret_cast<double*>(stream_smem + Ls.xw);
  double* tw = reinterpret_cast<double*>(stream_smem + Ls.tw);
  double* ex = reinterpret_cast<double*>(stream_smem + Ls.ex);
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < kStreamStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&ready[s], kStreamTThreads);
    }
    *abort_flag = 0;
    *released = 0;
    fence_mbarrier_init();
  }
  __syncthreads();
  using T = DiscTraits<DISC>;
  constexpr int H = SC ? (T::P > 2 * T::HALF ? T::P : 2 * T::HALF) : T::P;
  if (tid < kStreamTThreads) {
    set_max_registers<kStreamTRegs>();
    stream_transform<DISC, SC, PREC, STAGE>(p, full, ready, abort_flag, U, X,
                                            PS, QE, CF, NI, xw, tw, ex, tid);
  } else if (tid < kStreamTThreads + kStreamSThreads) {
    set_max_registers<kStreamSRegs>();
    stream_stencil<DISC, SC, NarrowGeom, STAGE>(p, ready, abort_flag, released,
                                                U, X, A, PS, QE, CF,
                                                tid - kStreamTThreads);
  } else {
    set_max_registers<kStreamPRegs>();
    if (tid == kStreamTThreads + kStreamSThreads) {
      stream_producer<H, T::HALF>(p, loader, full, U, X, A, CF, NI, released,
                                  abort_flag);
    }
  }
}

// ------------------------------------------------------------- wide bands
// The streaming kernel for bands of up to 24 ell and 48 nodes (free-damped
// reduction, FP64 transforms).  Same roles, chunks and waits as above, with
// the WideGeom ring (no accumulator or node-row ring): two transform warps
// share each 4-row block (three node tiles of the synthesis each, from
// fragments in registers; half of the analysis K steps each, from a
// shared-memory copy of the band's analysis matrix, partial sums added
// through `ex`); the stencil warps run the same stencil role with 24 ell
// lanes (five row pairs per pass).
constexpr int kWideXs = 36;  // staging strides of the wide transforms
constexpr int kWideTs = 52;
constexpr int kWideBlocks = kStreamBlocks;  // 4-row blocks per chunk
// Register split as in the narrow kernel.
constexpr int kWideTRegs = kStreamTRegs;
constexpr int kWideSRegs = kStreamSRegs;
constexpr int kWidePRegs = kStreamPRegs;
static_assert(kWidePRegs * 128 + kWideTRegs * 256 + kWideSRegs * 128 <=
                  kStreamThreads * kStreamLaunchRegs,
              "wide register split");
// Named barriers as in the narrow kernel.

struct WideLayout {
  size_t bars, loader, uring, xring, pring, coef, xw, tw, ex, amat, total;
  __host__ __device__ WideLayout() {
    size_t o = 0;
    bars = o;
    o += 128;  // 2 x 6 mbarriers, abort flag, released-chunk count
    loader = o;
    o += (sizeof(StreamLoaderState) + 127) / 128 * 128;
    const size_t ring =
        static_cast<size_t>(WideGeom::kRing) * 3 * WideGeom::kNep * 16;
    uring = o;
    o += ring;
    xring = o;
    o += ring;
    pring = o;
    o += static_cast<size_t>(WideGeom::kRing) * WideGeom::kNep * 16;
    coef = o;
    o += static_cast<size_t>(WideGeom::kRing) * kCoefCount * 8;
    xw = o;
    o += static_cast<size_t>(kWideBlocks) * 16 * kWideXs * 8;
    tw = o;
    o += static_cast<size_t>(kWideBlocks) * 8 * kWideTs * 8;
    ex = o;  // per block: one warp's analysis sums, 3 tiles x 2 x 32 lanes
    o += static_cast<size_t>(kWideBlocks) * 6 * 32 * 8;
    amat = o;  // A(l, j) of the strip's band, [l][j]
    o += static_cast<size_t>(WideGeom::kNep) * kWideTs * 8;
    total = o;
  }
};
static_assert(2 * WideGeom::kStages * 8 + 8 <= 128, "barrier area");
static_assert(2 * static_cast<size_t>(WideGeom::kRing) * 3 * WideGeom::kNep * 16 +
                      static_cast<size_t>(WideGeom::kRing) *
                          (WideGeom::kNep * 16 + kCoefCount * 8) +
                      static_cast<size_t>(kWideBlocks) *
                          (16 * kWideXs + 8 * kWideTs + 6 * 32) * 8 +
                      static_cast<size_t>(WideGeom::kNep) * kWideTs * 8 + 512 <=
                  227 * 1024,
              "wide shared memory");

// Synthesis fragments of one wide transform warp (h = 0, 1 of its block):
// node tiles h, h + 2, h + 4 over all 24 ell.  Its analysis covers all
// three ell tiles over the K steps h, h + 2, ..., h + 10 (nodes 4 k ..
// 4 k + 3), with the A operand read from the group's copy of A(l, j) in
// shared memory.  Interleaving splits any node count evenly between the
// two warps.
struct PsiWideFragments {
  double fs[3][6];  // S(j = (h + 2 i) * 8 + group, l = ks * 4 + quad)
  double gcos[3];   // 2 s a cos(theta_j), j = (h + 2 i) * 8 + group
};

// psi_t of the 4-row block at q0 (rows >= qlim skipped), this warp's share;
// the block's two warps synchronise on named barrier `bar`.
__device__ __forceinline__ void stream_psi_wide(
    const int q0, const int qlim, const int h, const StripGeom& sg,
    const double2* U, const double* CF, const double* node_rows, double2* PS,
    double* xw, double* tw, double* ex, const double* am,
    const PsiWideFragments& F, const int mts, const int ksa, const int bar,
    const int lane) {
  using G = WideGeom;
  const int quad = lane & 3;
  const int group = lane >> 2;
  const int ne = sg.ne;
  const double mm = static_cast<double>(sg.m);
  // 1 / C_T(r, theta_j) of this lane's outputs of the synthesis, loaded
  // first so the loads overlap the staging and the MMAs; zero beyond the
  // solve's nodes and the block's rows
  double inv[3][2];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int n = 0; n < 2; ++n) {
      const int r = q0 + 2 * n + (quad >> 1);
      const int j = (h + 2 * i) * 8 + group;
      inv[i][n] = (h + 2 * i < mts && r < qlim)
                      ? __ldg(node_rows + static_cast<long long>(r) * G::kNodeRec + j)
                      : 0.0;
    }
  }
  // stage the block's rows: v1 = P + 2K Q - G psi, psi (4 rows x 24 lanes
  // over the block's 64 threads)
  for (int it = h * 32 + lane; it < 4 * G::kNep; it += 64) {
    const int rho = it / G::kNep;
    const int l = it - rho * G::kNep;
    const int r = q0 + rho;
    double2 v1 = make_double2(0.0, 0.0), psi = make_double2(0.0, 0.0);
    if (r < qlim && l < ne) {
      const int rr = ring_row<G>(r, sg.shift);
      const double* cf = CF + rr * kCoefCount;
      const double2* row = U + rr * sg.rs;
      const double2 Q = row[ne + l];
      psi = row[2 * ne + l];
      v1 = csub(cadd(row[l], cscale(2.0 * cf[1], Q)),
                cmul(make_double2(cf[3], mm * cf[4]), psi));
    }
    xw[(rho * 4 + 0) * kWideXs + l] = v1.x;
    xw[(rho * 4 + 1) * kWideXs + l] = v1.y;
    xw[(rho * 4 + 2) * kWideXs + l] = psi.x;
    xw[(rho * 4 + 3) * kWideXs + l] = psi.y;
  }
  named_sync(bar, 64);
  {
    double bx[2][6];
#pragma unroll
    for (int n = 0; n < 2; ++n) {
#pragma unroll
      for (int ks = 0; ks < 6; ++ks) {
        bx[n][ks] = xw[(n * 8 + group) * kWideXs + ks * 4 + quad];
      }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int mt = h + 2 * i;
      if (mt < mts) {
        double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
        for (int ks = 0; ks < 6; ++ks) {
#pragma unroll
          for (int n = 0; n < 2; ++n) {
            dmma(acc[n][0], acc[n][1], F.fs[i][ks], bx[n][ks]);
          }
        }
        const int j = mt * 8 + group;
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          // lane quad 0/2 holds a_j of a row, quad 1/3 holds b_j of that row
          const double o0 = __shfl_xor_sync(0xffffffffu, acc[n][0], 1);
          const double o1 = __shfl_xor_sync(0xffffffffu, acc[n][1], 1);
          if ((quad & 1) == 0) {
            const int rho = 2 * n + (quad >> 1);
            tw[(rho * 2 + 0) * kWideTs + j] =
                (acc[n][0] + F.gcos[i] * o1) * inv[i][n];
            tw[(rho * 2 + 1) * kWideTs + j] =
                (acc[n][1] - F.gcos[i] * o0) * inv[i][n];
          }
        }
      }
    }
  }
  named_sync(bar, 64);
  double c[3][2][2];
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    c[t][0][0] = c[t][0][1] = c[t][1][0] = c[t][1][1] = 0.0;
  }
#pragma unroll
  for (int ks = 0; ks < 6; ++ks) {
    const int kg = 2 * ks + h;
    if (kg < ksa) {
      const double b = tw[group * kWideTs + kg * 4 + quad];
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const double a = am[(t * 8 + group) * kWideTs + kg * 4 + quad];
        dmma(c[t][ks & 1][0], c[t][ks & 1][1], a, b);
      }
    }
  }
  double sum[3][2];
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    sum[t][0] = c[t][0][0] + c[t][1][0];
    sum[t][1] = c[t][0][1] + c[t][1][1];
  }
  if (h == 1) {
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      ex[(t * 2 + 0) * 32 + lane] = sum[t][0];
      ex[(t * 2 + 1) * 32 + lane] = sum[t][1];
    }
  }
  named_sync(bar, 64);
  if (h == 0) {  // even K steps (this warp) + odd K steps (the partner)
    const int r = q0 + quad;
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const int l = t * 8 + group;
      if (r < qlim && l < ne) {
        PS[ring_row<G>(r, sg.shift) * G::kNep + l] =
            make_double2(sum[t][0] + ex[(t * 2 + 0) * 32 + lane],
                         sum[t][1] + ex[(t * 2 + 1) * 32 + lane]);
      }
    }
  }
}

template <int DISC, int STAGE = 0>
__device__ void stream_transform_wide(const StageLaunch& p,
                                      unsigned long long* full,
                                      unsigned long long* ready,
                                      volatile int* abort_flag, double2* U,
                                      const double2* X, double2* PS,
                                      const double* CF, double* xw_all,
                                      double* tw_all, double* ex_all,
                                      double* am, const int tt) {
  using G = WideGeom;
  using T = DiscTraits<DISC>;
  constexpr int HD = T::HALF, H = T::P;
  const int warp = tt >> 5, lane = tt & 31;
  const int quad = lane & 3, group = lane >> 2;
  const int blk = warp >> 1, h = warp & 1;
  double* xw = xw_all + blk * 16 * kWideXs;
  double* tw = tw_all + blk * 8 * kWideTs;
  double* ex = ex_all + blk * 6 * 32;
  // zero the nodal staging once (ordered by the first barrier below):
  // columns beyond a solve's nodes stay zero
  for (int i = tt; i < kWideBlocks * 8 * kWideTs; i += kStreamTThreads) {
    tw_all[i] = 0.0;
  }
  int g = 0;
  for (int strip = blockIdx.x; strip < p.strip_count; strip += gridDim.x) {
    const StripGeom sg = strip_geom<H, HD, G>(p, strip, g);
    const InstanceDesc& in = p.instances[sg.instance];
    const int nt = in.ntheta, ne = sg.ne;
    const bool kerr = in.spin != 0.0;
    const double hdt = 0.5 * in.dt;
    const double mm = static_cast<double>(sg.m);
    const double* node_rows =
        p.node_table + static_cast<long long>(sg.node_row0) * G::kNodeRec;
    PsiWideFragments F;
    const int mts = (nt + 7) / 8, ksa = (nt + 3) / 4;
    if (kerr) {
      const SegmentDesc& seg = p.segments[sg.segment];
      const double* St = p.matrices + seg.mat_offset;  // St[l][j]
      const double* At = St + ne * nt;                 // At[j][l]
      const double sa2 = 2.0 * (static_cast<double>(kSpinWeight) * in.spin);
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const int j = (h + 2 * i) * 8 + group;
#pragma unroll
        for (int ks = 0; ks < 6; ++ks) {
          const int l = ks * 4 + quad;
          F.fs[i][ks] = (j < nt && l < ne) ? St[l * nt + j] : 0.0;
        }
        F.gcos[i] = j < nt ? sa2 * p.trig[in.trig_offset + nt + j] : 0.0;
      }
      // the shared copy of A(l, j): every block of the previous strip has
      // finished reading the old one
      named_sync(1, kStreamTThreads);
      for (int i = tt; i < G::kNep * kWideTs; i += kStreamTThreads) {
        const int l = i / kWideTs;
        const int j = i - l * kWideTs;
        am[i] = (j < nt && l < ne) ? At[j * ne + l] : 0.0;
      }
      named_sync(1, kStreamTThreads);
    }
    for (int c = 0; c < sg.chunks; ++c, ++g) {
      const int s = g % G::kStages;
      const unsigned parity = static_cast<unsigned>(g / G::kStages) & 1u;
      const bool landed = stream_wait(&full[s], parity, abort_flag, p.error, 3);
      if (!named_sync_and(1, kStreamTThreads, landed)) return;
      const int a0 = sg.s0 + c * G::kChunk;
      const int a1 = min(sg.s1, a0 + G::kChunk);
      const int stage = STAGE != 0 ? STAGE : p.stage;
      if (stage == kStage2 || stage == kStage3) {  // u = y + dt/2 k
        const int base = ring_row<G>(a0, sg.shift) * sg.rs;
        const int count = (a1 - a0) * sg.rs;  // rows never wrap in a chunk
        double2* u = U + base;
        const double2* x = X + base;
        if (stage == kStage2) {  // U = y, X = k1
          for (int i = tt; i < count; i += kStreamTThreads) {
            u[i] = cfma(hdt, x[i], u[i]);
          }
        } else {  // U = k2, X = y
          for (int i = tt; i < count; i += kStreamTThreads) {
            u[i] = cfma(hdt, u[i], x[i]);
          }
        }
        named_sync(1, kStreamTThreads);
      }
      // psi_t of the chunk's rows (free-damped: pointwise in r)
      const int q_lo = max(a0, sg.t0), q_hi = min(a1, sg.t1);
      if (q_hi > q_lo) {
        if (kerr) {
          for (int q = q_lo; q < q_hi; q += 4 * kWideBlocks) {
            stream_psi_wide(q + 4 * blk, q_hi, h, sg, U, CF, node_rows, PS, xw,
                            tw, ex, am, F, mts, ksa, kStreamBlockBar + blk,
                            lane);
          }
        } else {
          const int items = (q_hi - q_lo) * G::kNep;
          for (int i = tt; i < items; i += kStreamTThreads) {
            const int r = q_lo + i / G::kNep;
            const int l = i % G::kNep;
            if (l < ne) {
              const int rr = ring_row<G>(r, sg.shift);
              const double* cf = CF + rr * kCoefCount;
              const double2* row = U + rr * sg.rs;
              const double2 Q = row[ne + l];
              const double2 psi = row[2 * ne + l];
              const double2 num =
                  csub(cadd(row[l], cscale(2.0 * cf[1], Q)),
                       cmul(make_double2(cf[3], mm * cf[4]), psi));
              PS[rr * G::kNep + l] = cscale(cf[9], num);
            }
          }
        }
      }
      // the combine wrote ring rows that later bulk copies overwrite
      fence_proxy_async_smem();
      mbar_arrive(&ready[s]);
    }
  }
}

// STAGE: p.stage as a compile-time constant.
template <int DISC, int STAGE>
__global__ void __launch_bounds__(kStreamThreads, 1)
    stream_wide_kernel(const StageLaunch p) {
  using G = WideGeom;
  using T = DiscTraits<DISC>;
  extern __shared__ __align__(128) unsigned char stream_smem[];
  const WideLayout Ls;
  unsigned long long* full =
      reinterpret_cast<unsigned long long*>(stream_smem + Ls.bars);
  unsigned long long* ready = full + G::kStages;
  volatile int* abort_flag =
      reinterpret_cast<volatile int*>(ready + G::kStages);
  volatile int* released = abort_flag + 1;
  StreamLoaderState& loader =
      *reinterpret_cast<StreamLoaderState*>(stream_smem + Ls.loader);
  double2* U = reinterpret_cast<double2*>(stream_smem + Ls.uring);
  double2* X = reinterpret_cast<double2*>(stream_smem + Ls.xring);
  double2* PS = reinterpret_cast<double2*>(stream_smem + Ls.pring);
  double* CF = reinterpret_cast<double*>(stream_smem + Ls.coef);
  double* xw = reinterpret_cast<double*>(stream_smem + Ls.xw);
  double* tw = reinterpret_cast<double*>(stream_smem + Ls.tw);
  double* ex = reinterpret_cast<double*>(stream_smem + Ls.ex);
  double* am = reinterpret_cast<double*>(stream_smem + Ls.amat);
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < G::kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&ready[s], kStreamTThreads);
    }
    *abort_flag = 0;
    *released = 0;
    fence_mbarrier_init();
  }
  __syncthreads();
  if (tid < kStreamTThreads) {
    set_max_registers<kWideTRegs>();
    stream_transform_wide<DISC, STAGE>(p, full, ready, abort_flag, U, X, PS,
                                       CF, xw, tw, ex, am, tid);
  } else if (tid < kStreamTThreads + kStreamSThreads) {
    set_max_registers<kWideSRegs>();
    // no accumulator ring (the RK update reads it from global memory) and
    // no effective-Q ring (free-damped only)
    stream_stencil<DISC, 0, G, STAGE>(p, ready, abort_flag, released, U, X,
                                      nullptr, PS, PS, CF, tid - kStreamTThreads);
  } else {
    set_max_registers<kWidePRegs>();
    if (tid == kStreamTThreads + kStreamSThreads) {
      // no node rows to copy (the transforms read them from global memory)
      stream_producer<T::P, T::HALF, G>(p, loader, full, U, X, nullptr, CF,
                                        nullptr, released, abort_flag);
    }
  }
}

// Teukolsky row coefficients of one solve (m = 1 for entries 4, 6, 8) and
// the inverse of C_T(r, theta_j) = C_T0(r) - a^2 sin^2(theta_j) on its
// nodes (the diagonal of the implicit ell-coupling, A diag(1/C_T) S).
__global__ void coefficient_table_kernel(const InstanceDesc* instance,
                                         const double* trig, const int nr,
                                         double* out, double* node_out,
                                         const int node_record) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nr) return;
  const InstanceDesc in = *instance;
  double cf[kCoefCount];
  row_coefficients(in, 1, r, cf);
  if (out != nullptr) {
#pragma unroll
    for (int k = 0; k < kCoefCount; ++k) out[r * kCoefCount + k] = cf[k];
  }
  const double a2 = in.spin * in.spin;
  double* inv = node_out + static_cast<long long>(r) * node_record;
  for (int j = 0; j < node_record; ++j) {
    double v = 0.0;
    if (j < in.ntheta) {
      const double s = trig[in.trig_offset + j];
      v = 1.0 / __dsub_rn(cf[0], __dmul_rn(__dmul_rn(a2, s), s));
    }
    inv[j] = v;
  }
}
