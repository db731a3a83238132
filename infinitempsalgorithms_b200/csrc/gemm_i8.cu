// Split-precision complex GEMM on the 5th-generation tensor cores (tcgen05, kind::i8).
//
// Scheme (Ozaki splitting with power-of-two scaling).  Each complex row i of
// op(A) gets a scale r_i = 2^e >= max_k max(|Re|,|Im|) and each complex column j of
// op(B) a scale c_j; the scaled values x / scale lie in (-1, 1) and are cut into
// `s` int8 slices x = scale * sum_t a_t 2^-7(t+1) (truncating, |a_t| <= 127).  The
// complex product is carried by a real GEMM of the expanded operands
//     At (2M x 2K): rows (i, re/im), cols (k, re/im) = [[Re, -Im], [Im, Re]]
//     Bt (N x 2K):  rows j,            cols (k, re/im) = [Re b_kj, Im b_kj]
// so that row 2i+p of At Bt^T is (Re, Im)[p] of c_ij.  For every diagonal
// d = ta + tb < s the slice pairs are summed *exactly* in an int32 TMEM
// accumulator (the K extent is chunked so no sum can overflow), and the
// epilogue adds r_i c_j 2^-7(d+2) acc to the FP64 output.  Truncation error per
// element is below 2^-7s of the row/column scale.
//
// GEMM kernel: persistent, one CTA per SM, warp-specialised, 128 x BN output tiles.
// K runs outermost: one pipeline stage holds a 64-byte K block of *every* slice
// plane of both operands, and the MMA thread issues all slice pairs (ta, tb) with
// ta + tb < s for it, each diagonal d = ta + tb into its own int32 TMEM
// accumulator (s x BN columns per tile).  Every byte brought into shared memory
// thus feeds (s + 1) / 2 MMAs on average instead of one, which is what keeps the
// tensor pipe fed from L2.
// Tile width: an M=128 MMA reads its A tile (4 KB per K=32) and B tile (BN x 32 B)
// from shared memory, whose 128 B/clk per SM feed the int8 pipe's ~7.7k MAC/clk only
// when BN >= ~115.  BN = 128 is used for s <= 4 (s x 128 TMEM columns still fit the
// 512 of an SM), 96 for s = 5 and 80 for s = 6 (480 columns), 64 beyond.
//   warp 0: TMA producer (cp.async.bulk.tensor, 64B swizzle, 2-8 stages by s)
//   warp 1: TMEM allocator + single-thread tcgen05.mma issuer (M=128, N=BN, K=32)
//   warps 2-9: epilogue, tcgen05.ld 32x32b, two warps per TMEM lane quarter, each
//           owning BN/2 columns in chunks of 32, 16 or 8; a thread sums its row's chunk over
//           all diagonals in FP64 registers and writes it (adds it, for the later
//           K groups of a tile).  When two tiles' accumulators fit in TMEM the
//           epilogue of one tile overlaps the MMAs of the next.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>

#include "imps_internal.h"
#include "split_gemm.h"

namespace imps {
namespace {

constexpr int BM = 128;          // tile rows (real rows of At)
constexpr int BN_MAX = 128;      // widest tile (rows of Bt); B planes are padded to it
constexpr int KB = 64;           // K bytes per pipeline stage (one 64B swizzle row)
constexpr int KPAD = 128;        // K padding of the slice planes (the slicing kernels' tile)
constexpr int MAX_STAGES = 8;
constexpr int MAX_BUF = 4;       // tile accumulator buffers in TMEM
constexpr int EPI_WARPS = 8;     // two warps per TMEM lane quarter, each owning BN/2 columns
constexpr int A_TILE = BM * KB;  // 8 KB per slice
constexpr int STAGE_BUDGET = 216 * 1024;
constexpr int BAR_BYTES = 512;
constexpr int NTHREADS = 32 * (2 + EPI_WARPS);
constexpr long long DRAIN_CYCLES = 2000000000LL;  // ~1 s at 1.9 GHz: bound of the error-path drains

// tile width for a slice count: the widest multiple of 16 (at most 128) whose s
// diagonals fit the 512 TMEM columns of an SM
__host__ __device__ constexpr int bn_for(int s) {
  return (s >= 1 && s <= 4) ? 128 : (s == 5 ? 96 : (s == 6 ? 80 : 64));
}
__host__ __device__ constexpr int stages_for(int s, int bn) {
  return (STAGE_BUDGET / (s * (A_TILE + bn * KB))) < MAX_STAGES ? (STAGE_BUDGET / (s * (A_TILE + bn * KB)))
                                                                 : MAX_STAGES;
}
__host__ __device__ constexpr int bufs_for(int s, int bn) {
  return (512 / (s * bn)) < MAX_BUF ? (512 / (s * bn)) : MAX_BUF;
}
__host__ constexpr int smem_bytes_for(int s, int bn) {
  return stages_for(s, bn) * s * (A_TILE + bn * KB) + 1024 + BAR_BYTES;
}
__host__ constexpr int max_smem_bytes() {
  int m = 0;
  for (int s = 1; s <= 8; ++s) m = smem_bytes_for(s, bn_for(s)) > m ? smem_bytes_for(s, bn_for(s)) : m;
  for (int s = 1; s <= 8; ++s) m = smem_bytes_for(s, 64) > m ? smem_bytes_for(s, 64) : m;
  return m;
}
static_assert(max_smem_bytes() <= 227 * 1024, "pipeline does not fit in shared memory");
static_assert(bufs_for(4, 128) >= 1 && bufs_for(8, 64) >= 1, "every diagonal of a tile fits in TMEM");
static_assert(stages_for(4, 128) >= 2, "at least double buffering at 4 slices, 128 columns");
static_assert(stages_for(8, 64) >= 2, "at least double buffering at 8 slices");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: returns false (and raises the error flag) after `limit` cycles.  The
// fast path only polls the barrier; the clock is also read on the first unsuccessful
// poll (so a bound shorter than a poll round trips at once) and the global error
// flag with the clock every 256 unsuccessful polls, so a completed phase is seen
// without extra memory latency.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* err, long long limit) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  unsigned spins = 0;
  while (!mbar_try(bar, parity)) {
    ++spins;
    if (spins == 1u) {
      if (clock64() - t0 > limit) {
        atomicExch((int*)err, 1);
        return false;
      }
      continue;
    }
    if ((spins & 255u) != 0u) continue;
    if (*err) return false;
    if (clock64() - t0 > limit) {
      atomicExch((int*)err, 1);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// UMMA shared-memory descriptor: K-major, 64B swizzle, 8-row groups 512 B apart.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
  d |= (uint64_t)1 << 16;                           // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;                  // stride byte offset: 8 rows x 64 B
  d |= (uint64_t)1 << 46;                           // descriptor version (sm100)
  d |= (uint64_t)4 << 61;                           // SWIZZLE_64B
  return d;
}

// instruction descriptor: kind::i8, s8 x s8 -> s32, both K-major, M = 128, N = BN
template <int BN>
__host__ __device__ constexpr uint32_t make_idesc() {
  return (2u << 4)                 // D format: s32
         | (1u << 7)               // A format: s8
         | (1u << 10)              // B format: s8
         | ((uint32_t)(BN >> 3) << 17)
         | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int32_t* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
// CW columns of this warp's 32 TMEM lanes, one register per column
template <int CW>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, int32_t* r) {
  if constexpr (CW == 32) tmem_ld32(taddr, r);
  else if constexpr (CW == 16) tmem_ld16(taddr, r);
  else tmem_ld8(taddr, r);
}

struct GemmArgs {
  int num_m, num_n;          // tiles
  int n_fast;                // raster: 1 -> consecutive tiles walk N (A is the larger operand)
  int kblocks;               // K blocks of KB bytes per slice plane
  int nst;                   // pipeline stages (by s)
  int nbuf;                  // tile accumulator buffers in TMEM (by s)
  int s;                     // slice diagonals d = 0 .. s-1
  double2* C;                // complex output
  int64_t ldc;
  int Mc, Nc;                // valid complex rows / cols
  const double* row_scale;   // per complex row of op(A)
  const double* col_scale;   // per complex col of op(B)
  double alpha;
  int accumulate;            // 0: C = result, 1: C += result
  int* err;
  long long wait_cycles;     // bound of each pipeline wait (SM clock cycles)
};

// Accumulation groups of one tile: K range [kb0, kb1) of every slice pair; the
// largest diagonal sums s pairs of products <= 127^2, so a group stays below 2^31.
struct GroupIter {
  const GemmArgs* g;
  int kb0 = 0;
  __device__ explicit GroupIter(const GemmArgs* a) : g(a) {}
  __device__ bool valid() const { return kb0 < g->kblocks; }
  __device__ int chunk() const { return max(1, (int)(2147483647.0 / (16129.0 * g->s * KB))); }
  __device__ int kb1() const { return min(g->kblocks, kb0 + chunk()); }
  __device__ void next() { kb0 += chunk(); }
};

__device__ __forceinline__ void tile_coords(const GemmArgs& g, int t, int& mb, int& nb) {
  if (g.n_fast) { nb = t % g.num_n; mb = t / g.num_n; }
  else { mb = t % g.num_m; nb = t / g.num_m; }
}

// Issues the slice-pair MMAs of one stage: for every diagonal d and pair (ta, d - ta),
// two K=32 MMAs into the diagonal's accumulator.  With a compile-time slice count the
// loops unroll into a straight run of MMAs on precomputed descriptors, so one thread
// keeps up with the tensor pipe.
template <int SC, int BN>
__device__ __forceinline__ void issue_stage(int S, uint64_t da, uint64_t db, uint32_t dt0, uint32_t idesc, bool fresh) {
  constexpr int B_TILE = BN * KB;
  const int s = SC > 0 ? SC : S;
#pragma unroll
  for (int d = 0; d < (SC > 0 ? SC : 8); ++d) {
    if (d >= s) break;
    const uint32_t dtmem = dt0 + (uint32_t)(d * BN);
#pragma unroll
    for (int ta = 0; ta <= d; ++ta) {
      const int tb = d - ta;
#pragma unroll
      for (int kk = 0; kk < KB / 32; ++kk) {
        // start-address field counts 16-byte units
        const uint64_t a = da + (uint64_t)((ta * A_TILE + kk * 32) >> 4);
        const uint64_t b = db + (uint64_t)((tb * B_TILE + kk * 32) >> 4);
        umma_i8(dtmem, a, b, idesc, (fresh && ta == 0 && kk == 0) ? 0u : 1u);
      }
    }
  }
}

template <int SC, int BN>
__global__ void __launch_bounds__(NTHREADS, 1)
    k_gemm_i8(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, const GemmArgs g) {
  constexpr int B_TILE = BN * KB;
  static_assert(BN % 16 == 0 && BN >= 64 && BN <= BN_MAX, "MMA N is a multiple of 16; half tiles of >= 32 columns");
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int S = SC > 0 ? SC : g.s, NST = g.nst, NBUF = g.nbuf;
  const int stage_bytes = S * (A_TILE + B_TILE);  // [A slices][B slices]
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + NST * stage_bytes);
  uint64_t* full = bars;                                  // [MAX_STAGES]
  uint64_t* empty = bars + MAX_STAGES;                    // [MAX_STAGES]
  uint64_t* tfull = bars + 2 * MAX_STAGES;                // [MAX_BUF]
  uint64_t* tempty = bars + 2 * MAX_STAGES + MAX_BUF;     // [MAX_BUF]
  uint64_t* drain = bars + 2 * MAX_STAGES + 2 * MAX_BUF;  // MMA drain on the error path
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * MAX_STAGES + 2 * MAX_BUF + 1);
  volatile int* err = g.err;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int st = 0; st < NST; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], 1);
    }
    for (int a = 0; a < NBUF; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], EPI_WARPS);  // one arrival per epilogue warp
    }
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int ntiles = g.num_m * g.num_n;

  if (warp == 0) {
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      bool ok = true;
      int issued[MAX_STAGES];  // parity of the last load issued into each stage (-1: none)
      for (int s2 = 0; s2 < MAX_STAGES; ++s2) issued[s2] = -1;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        int mb, nb;
        tile_coords(g, t, mb, nb);
        for (int kb = 0; kb < g.kblocks && ok; ++kb) {
          ok = mbar_wait(&empty[stage], phase ^ 1, err, g.wait_cycles);
          if (!ok) break;
          uint8_t* base = smem + stage * stage_bytes;
          mbar_expect_tx(&full[stage], (uint32_t)stage_bytes);
          for (int sl = 0; sl < S; ++sl) {
            tma_load_3d(base + sl * A_TILE, &mapA, &full[stage], kb * KB, mb * BM, sl);
            tma_load_3d(base + S * A_TILE + sl * B_TILE, &mapB, &full[stage], kb * KB, nb * BN, sl);
          }
          issued[stage] = (int)phase;
          if (++stage == NST) { stage = 0; phase ^= 1; }
        }
      }
      // every issued copy must land before the CTA may exit (bounded)
      for (int s2 = 0; s2 < NST; ++s2) {
        if (issued[s2] < 0) continue;
        long long t0 = clock64();
        while (!mbar_try(&full[s2], (uint32_t)issued[s2]) && clock64() - t0 < DRAIN_CYCLES) {
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = make_idesc<BN>();
      int stage = 0;
      uint32_t phase = 0;
      int grp = 0;  // accumulation-group counter (selects the TMEM buffer)
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        for (GroupIter gi(&g); gi.valid() && ok; gi.next(), ++grp) {
          const int buf = grp % NBUF;
          ok = mbar_wait(&tempty[buf], ((grp / NBUF) & 1) ^ 1, err, g.wait_cycles);
          if (!ok) break;
          tc_fence_after();
          const int kb1 = gi.kb1();
          for (int kb = gi.kb0; kb < kb1 && ok; ++kb) {
            ok = mbar_wait(&full[stage], phase, err, g.wait_cycles);
            if (!ok) break;
            tc_fence_after();
            const uint32_t a0 = smem_u32(smem + stage * stage_bytes);
            const uint32_t b0 = a0 + S * A_TILE;
            issue_stage<SC, BN>(S, make_desc(a0), make_desc(b0), tmem_base + (uint32_t)(buf * S * BN), idesc,
                            kb == gi.kb0);
            umma_commit(&empty[stage]);  // frees the smem stage when these MMAs retire
            if (++stage == NST) { stage = 0; phase ^= 1; }
          }
          if (!ok) break;
          umma_commit(&tfull[buf]);
        }
      }
      // all MMAs issued by this thread retire before TMEM is released (bounded)
      umma_commit(drain);
      long long t0 = clock64();
      while (!mbar_try(drain, 0) && clock64() - t0 < DRAIN_CYCLES) {
      }
    }
  } else {
    // epilogue warps 2..9: TMEM lane quarter q = warp % 4, column half h
    constexpr int HC = BN / 2;   // columns per epilogue thread
    constexpr int CW = (HC % 32 == 0) ? 32 : ((HC % 16 == 0) ? 16 : 8);  // columns per tcgen05.ld
    constexpr int NCH = HC / CW; // chunks (one tcgen05.ld each per diagonal)
    static_assert(HC % CW == 0, "half tile is a whole number of chunks");
    const int q = warp & 3;
    const int h = (warp - 2) / 4;
    const int row = q * 32 + lane;  // tile row == TMEM lane
    double* Cd = reinterpret_cast<double*>(g.C);
    if constexpr (NCH == 1) {
      // one chunk per thread: the row's FP64 sums are kept over all K groups of the
      // tile and written once
      int grp = 0;
      for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int mb, nb;
        tile_coords(g, t, mb, nb);
        double part[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) part[j] = 0.0;
        bool ok = true;
        for (GroupIter gi(&g); gi.valid(); gi.next(), ++grp) {
          const int buf = grp % NBUF;
          if (!mbar_wait(&tfull[buf], (grp / NBUF) & 1, err, g.wait_cycles)) { ok = false; break; }
          tc_fence_after();
          for (int d = 0; d < S; ++d) {
            const double w = ldexp(1.0, -7 * (d + 2));
            int32_t r[32];
            tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)((buf * S + d) * BN + h * HC), r);
#pragma unroll
            for (int j = 0; j < 32; ++j) part[j] = fma((double)r[j], w, part[j]);
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&tempty[buf]);
        }
        if (!ok) break;
        const int rr = mb * BM + row;              // real row of At
        const int ci = rr >> 1, part_im = rr & 1;  // complex row, re/im
        if (ci < g.Mc) {
          const double rs = g.row_scale[ci] * g.alpha;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int cj = nb * BN + h * HC + j;
            if (cj < g.Nc) {
              const double v = part[j] * rs * __ldg(&g.col_scale[cj]);
              double* p = Cd + 2 * ((int64_t)ci + g.ldc * cj) + part_im;
              *p = g.accumulate ? (*p + v) : v;
            }
          }
        }
      }
    } else {
      int grp = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        int mb, nb;
        tile_coords(g, t, mb, nb);
        const int rr = mb * BM + row;              // real row of At
        const int ci = rr >> 1, part_im = rr & 1;  // complex row, re/im
        const double rs = (ci < g.Mc) ? g.row_scale[ci] * g.alpha : 0.0;
        bool first = true;  // first K group of the tile writes (or adds, when accumulating)
        for (GroupIter gi(&g); gi.valid(); gi.next(), ++grp) {
          const int buf = grp % NBUF;
          if (!mbar_wait(&tfull[buf], (grp / NBUF) & 1, err, g.wait_cycles)) { ok = false; break; }
          tc_fence_after();
#pragma unroll 1
          for (int ch = 0; ch < NCH; ++ch) {
            // FP64 sum of this thread's CW columns over all slice diagonals of the group
            double part[CW];
#pragma unroll
            for (int j = 0; j < CW; ++j) part[j] = 0.0;
#pragma unroll 1
            for (int d = 0; d < S; ++d) {
              const double w = ldexp(1.0, -7 * (d + 2));
              int32_t r[CW];
              tmem_ld<CW>(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)((buf * S + d) * BN + h * HC + ch * CW), r);
#pragma unroll
              for (int j = 0; j < CW; ++j) part[j] = fma((double)r[j], w, part[j]);
            }
            if (ch == NCH - 1) {
              // every column of this buffer has been read: hand it back to the MMA thread
              tc_fence_before();
              __syncwarp();
              if (lane == 0) mbar_arrive(&tempty[buf]);
            }
            if (ci < g.Mc) {
              const bool add = g.accumulate || !first;
#pragma unroll
              for (int j = 0; j < CW; ++j) {
                const int cj = nb * BN + h * HC + ch * CW + j;
                if (cj < g.Nc) {
                  const double v = part[j] * rs * __ldg(&g.col_scale[cj]);
                  double* p = Cd + 2 * ((int64_t)ci + g.ldc * cj) + part_im;
                  *p = add ? (*p + v) : v;
                }
              }
            }
          }
          first = false;
        }
      }
    }
  }
  // TMEM is released only after every MMA of this CTA retired (epilogue saw all
  // groups, or the MMA thread drained on the error path)
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem_base));
  }
}

// ---------------------------------------------------------------------------
// Slicing kernels (memory bound)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

// per complex row i of op(A) (opA N: A[i + lda k]) -> atomicMax of max(|re|,|im|) bits
__global__ void k_rowmax_colmajor(int M, int K, const double2* __restrict__ A, int64_t lda, int kchunk,
                                  unsigned long long* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const int k0 = blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
  double m = 0.0;
  for (int k = k0; k < k1; ++k) {
    double2 v = A[i + lda * k];
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
  }
  atomicMax(&out[i], dbits(m));
}
// per "contiguous line" l (A[k + ld l], k < K): max over k (warp per line)
__global__ void k_linemax_contig(int L, int K, const double2* __restrict__ A, int64_t ld,
                                 unsigned long long* __restrict__ out) {
  const int l = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (l >= L) return;
  double m = 0.0;
  for (int k = lane; k < K; k += 32) {
    double2 v = A[k + ld * l];
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) out[l] = dbits(m);
}
// column max of a row-major-strided view: out[j] = max_k |B[j + ld k]|  (thread per j, chunked k)
__global__ void k_colmax_strided(int Ncol, int K, const double2* __restrict__ B, int64_t ld, int kchunk,
                                 unsigned long long* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Ncol) return;
  const int k0 = blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
  double m = 0.0;
  for (int k = k0; k < k1; ++k) {
    double2 v = B[j + ld * k];
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
  }
  atomicMax(&out[j], dbits(m));
}

// max bits -> scale 2^e > max, and its inverse (exact powers of two)
__global__ void k_scales(int n, const unsigned long long* __restrict__ mx, double* __restrict__ scale,
                         double* __restrict__ inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double m = __longlong_as_double((long long)mx[i]);
  if (!(m > 0.0) || !isfinite(m)) {
    scale[i] = 0.0;
    inv[i] = 0.0;
    return;
  }
  int e;
  frexp(m, &e);  // m = f 2^e, f in [0.5, 1)  =>  m < 2^e
  scale[i] = ldexp(1.0, e);
  inv[i] = ldexp(1.0, -e);
}

__device__ __forceinline__ void slice_value(double x, int s, int8_t* out) {
  // x in (-1, 1): the s leading base-128 digits of x, truncated toward zero, each with
  // the sign of x (x = sum_t out[t] 128^-(t+1) + r, |r| < 128^-s).  x 2^(7s) is exact
  // (a power-of-two scaling below 2^56), so its integer part carries all s digits.
  const double y = ldexp(x, 7 * s);
  const long long n = (fabs(y) < 9.0e18) ? (long long)y : 0;  // non-finite input: zero slices
  const long long a = n < 0 ? -n : n;
  for (int t = 0; t < s; ++t) {
    const int dg = (int)((a >> (7 * (s - 1 - t))) & 127);
    out[t] = (int8_t)(n < 0 ? -dg : dg);
  }
}

// Split op(A) into expanded K-major planes.  A block covers 32 complex rows x 64
// complex k of the *padded* extent (so no separate zero fill is needed); each
// thread slices 4 consecutive complex k and stores 8 bytes into each of the two
// expanded rows per plane.
// opA == 0: A[i + lda k] (transposed through shared memory), opA == 2: conj(A[k + lda i]).
template <int OPA>
__global__ void __launch_bounds__(256) k_split_a(int M, int K, const double2* __restrict__ A, int64_t lda,
                                                 const double* __restrict__ inv, int s, int8_t* __restrict__ out,
                                                 int64_t Kp, int64_t plane) {
  __shared__ double2 tile[32][65];
  const int i0 = blockIdx.y * 32, k0 = blockIdx.x * 64;
  const int tid = threadIdx.x;
  if (OPA == 0) {
    const int tx = tid & 31, ty = tid >> 5;
    for (int r = ty; r < 64; r += 8) {
      const int i = i0 + tx, k = k0 + r;
      tile[tx][r] = (i < M && k < K) ? A[i + lda * k] : make_double2(0.0, 0.0);
    }
  } else {
    const int kx = tid & 63, iy = tid >> 6;
    for (int r = iy; r < 32; r += 4) {
      const int i = i0 + r, k = k0 + kx;
      double2 v = (i < M && k < K) ? A[k + lda * i] : make_double2(0.0, 0.0);
      v.y = -v.y;
      tile[r][kx] = v;
    }
  }
  __syncthreads();
  for (int item = tid; item < 32 * 16; item += 256) {
    const int il = item >> 4, kq = item & 15;
    const int i = i0 + il;
    const double sc = (i < M) ? inv[i] : 0.0;
    int8_t re[4][8], im[4][8];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double2 v = tile[il][4 * kq + c];
      slice_value(v.x * sc, s, re[c]);
      slice_value(v.y * sc, s, im[c]);
    }
    int8_t* p0 = out + (int64_t)(2 * i) * Kp + 2 * (k0 + 4 * kq);
    for (int t = 0; t < s; ++t) {
      // row 2i: (Re, -Im) pairs; row 2i+1: (Im, Re) pairs
      uint32_t lo0 = 0, hi0 = 0, lo1 = 0, hi1 = 0;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        lo0 |= ((uint32_t)(uint8_t)re[c][t] | ((uint32_t)(uint8_t)(int8_t)(-im[c][t]) << 8)) << (16 * c);
        hi0 |= ((uint32_t)(uint8_t)re[c + 2][t] | ((uint32_t)(uint8_t)(int8_t)(-im[c + 2][t]) << 8)) << (16 * c);
        lo1 |= ((uint32_t)(uint8_t)im[c][t] | ((uint32_t)(uint8_t)re[c][t] << 8)) << (16 * c);
        hi1 |= ((uint32_t)(uint8_t)im[c + 2][t] | ((uint32_t)(uint8_t)re[c + 2][t] << 8)) << (16 * c);
      }
      *reinterpret_cast<uint2*>(p0 + plane * t) = make_uint2(lo0, hi0);
      *reinterpret_cast<uint2*>(p0 + plane * t + Kp) = make_uint2(lo1, hi1);
    }
  }
}

// Split op(B) (K x N complex) into K-major planes Bt[j][2k + p], same tiling over
// the padded extent; 8-byte stores of 4 consecutive complex k.
// opB == 0: B[k + ldb j] (contiguous in k); opB == 2: conj(B[j + ldb k]) (tile transpose).
template <int OPB>
__global__ void __launch_bounds__(256) k_split_b(int K, int N, const double2* __restrict__ B, int64_t ldb,
                                                 const double* __restrict__ inv, int s, int8_t* __restrict__ out,
                                                 int64_t Kp, int64_t plane) {
  __shared__ double2 tile[32][65];
  const int j0 = blockIdx.y * 32, k0 = blockIdx.x * 64;
  const int tid = threadIdx.x;
  if (OPB == 0) {
    const int kx = tid & 63, jy = tid >> 6;
    for (int r = jy; r < 32; r += 4) {
      const int j = j0 + r, k = k0 + kx;
      tile[r][kx] = (k < K && j < N) ? B[k + ldb * j] : make_double2(0.0, 0.0);
    }
  } else {
    const int tx = tid & 31, ty = tid >> 5;
    for (int r = ty; r < 64; r += 8) {
      const int j = j0 + tx, k = k0 + r;
      double2 v = (k < K && j < N) ? B[j + ldb * k] : make_double2(0.0, 0.0);
      v.y = -v.y;
      tile[tx][r] = v;
    }
  }
  __syncthreads();
  for (int item = tid; item < 32 * 16; item += 256) {
    const int jl = item >> 4, kq = item & 15;
    const int j = j0 + jl;
    const double sc = (j < N) ? inv[j] : 0.0;
    int8_t re[4][8], im[4][8];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double2 v = tile[jl][4 * kq + c];
      slice_value(v.x * sc, s, re[c]);
      slice_value(v.y * sc, s, im[c]);
    }
    int8_t* p0 = out + (int64_t)j * Kp + 2 * (k0 + 4 * kq);
    for (int t = 0; t < s; ++t) {
      uint32_t lo = 0, hi = 0;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        lo |= ((uint32_t)(uint8_t)re[c][t] | ((uint32_t)(uint8_t)im[c][t] << 8)) << (16 * c);
        hi |= ((uint32_t)(uint8_t)re[c + 2][t] | ((uint32_t)(uint8_t)im[c + 2][t] << 8)) << (16 * c);
      }
      *reinterpret_cast<uint2*>(p0 + plane * t) = make_uint2(lo, hi);
    }
  }
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  // resolved once per process; contexts on several host threads may race here
  static std::mutex mu;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    IMPS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    IMPS_REQUIRE(p && q == cudaDriverEntryPointSuccess, IMPS_CUDA_ERROR, "cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 3D map over int8 planes: dims (Kp bytes, rows, planes), box (KB, box_rows, 1), 64B swizzle
CUtensorMap make_map(const int8_t* base, int64_t Kp, int64_t rows, int planes, int box_rows) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  cuuint64_t dims[3] = {(cuuint64_t)Kp, (cuuint64_t)rows, (cuuint64_t)planes};
  cuuint64_t strides[2] = {(cuuint64_t)Kp, (cuuint64_t)(Kp * rows)};
  cuuint32_t box[3] = {(cuuint32_t)KB, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = get_encode()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t*>(base), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  IMPS_REQUIRE(r == CUDA_SUCCESS, IMPS_CUDA_ERROR, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

}  // namespace

// ---------------------------------------------------------------------------
void split_operand_a(Context* ctx, SplitOperand& S, Op op, int M, int K, const dcplx* A, int64_t lda, int s) {
  IMPS_REQUIRE(op == OP_N || op == OP_C, IMPS_INVALID_ARG, "split: op T is not supported");
  IMPS_REQUIRE(s >= 1 && s <= 8, IMPS_INVALID_ARG, "split: 1..8 slices");
  S.rows = M;
  S.K = K;
  S.s = s;
  S.Rp = round_up(2 * (int64_t)M, BM);
  S.Kp = round_up(2 * (int64_t)K, KPAD);
  const size_t plane = (size_t)S.Rp * S.Kp;
  S.data.ensure(plane * s);
  S.scale.ensure((size_t)M * sizeof(double));
  S.inv.ensure((size_t)M * sizeof(double));
  S.mx.ensure((size_t)M * sizeof(unsigned long long));
  ScopedTimer tm(ctx, "split_slice", 16.0 * M * K + (double)plane * s);
  IMPS_CUDA(cudaMemsetAsync(S.mx.ptr, 0, (size_t)M * 8, ctx->stream));
  auto* mx = static_cast<unsigned long long*>(S.mx.ptr);
  if (op == OP_N) {
    const int kchunk = 64;
    dim3 g((M + 127) / 128, (K + kchunk - 1) / kchunk);
    k_rowmax_colmajor<<<g, 128, 0, ctx->stream>>>(M, K, A, lda, kchunk, mx);
  } else {
    k_linemax_contig<<<(M + 7) / 8, 256, 0, ctx->stream>>>(M, K, A, lda, mx);
  }
  k_scales<<<(M + 255) / 256, 256, 0, ctx->stream>>>(M, mx, S.scale.d(), S.inv.d());
  // grid over the padded extent: Kp / 2 complex columns, Rp / 2 complex rows
  dim3 g2((unsigned)(S.Kp / 2 / 64), (unsigned)(S.Rp / 2 / 32));
  if (op == OP_N)
    k_split_a<0><<<g2, 256, 0, ctx->stream>>>(M, K, A, lda, S.inv.d(), s, static_cast<int8_t*>(S.data.ptr), S.Kp, plane);
  else
    k_split_a<2><<<g2, 256, 0, ctx->stream>>>(M, K, A, lda, S.inv.d(), s, static_cast<int8_t*>(S.data.ptr), S.Kp, plane);
  ctx->n_kernels += 5;
  IMPS_CUDA(cudaPeekAtLastError());
}

void split_operand_b(Context* ctx, SplitOperand& S, Op op, int K, int N, const dcplx* B, int64_t ldb, int s) {
  IMPS_REQUIRE(op == OP_N || op == OP_C, IMPS_INVALID_ARG, "split: op T is not supported");
  IMPS_REQUIRE(s >= 1 && s <= 8, IMPS_INVALID_ARG, "split: 1..8 slices");
  S.rows = N;
  S.K = K;
  S.s = s;
  S.Rp = round_up(N, BN_MAX);  // every B box (64 or 128 rows) lies inside the planes
  S.Kp = round_up(2 * (int64_t)K, KPAD);
  const size_t plane = (size_t)S.Rp * S.Kp;
  S.data.ensure(plane * s);
  S.scale.ensure((size_t)N * sizeof(double));
  S.inv.ensure((size_t)N * sizeof(double));
  S.mx.ensure((size_t)N * sizeof(unsigned long long));
  ScopedTimer tm(ctx, "split_slice", 16.0 * K * N + (double)plane * s);
  IMPS_CUDA(cudaMemsetAsync(S.mx.ptr, 0, (size_t)N * 8, ctx->stream));
  auto* mx = static_cast<unsigned long long*>(S.mx.ptr);
  if (op == OP_N) {
    k_linemax_contig<<<(N + 7) / 8, 256, 0, ctx->stream>>>(N, K, B, ldb, mx);
  } else {
    const int kchunk = 64;
    dim3 g((N + 127) / 128, (K + kchunk - 1) / kchunk);
    k_colmax_strided<<<g, 128, 0, ctx->stream>>>(N, K, B, ldb, kchunk, mx);
  }
  k_scales<<<(N + 255) / 256, 256, 0, ctx->stream>>>(N, mx, S.scale.d(), S.inv.d());
  dim3 g2((unsigned)(S.Kp / 2 / 64), (unsigned)(S.Rp / 32));
  if (op == OP_N)
    k_split_b<0><<<g2, 256, 0, ctx->stream>>>(K, N, B, ldb, S.inv.d(), s, static_cast<int8_t*>(S.data.ptr), S.Kp, plane);
  else
    k_split_b<2><<<g2, 256, 0, ctx->stream>>>(K, N, B, ldb, S.inv.d(), s, static_cast<int8_t*>(S.data.ptr), S.Kp, plane);
  ctx->n_kernels += 5;
  IMPS_CUDA(cudaPeekAtLastError());
}

void split_gemm(Context* ctx, const SplitOperand& A, const SplitOperand& B, int s, double alpha, bool accumulate,
                dcplx* C, int64_t ldc) {
  IMPS_REQUIRE(A.K == B.K && A.Kp == B.Kp, IMPS_DIM_MISMATCH, "split_gemm: inner dimensions differ");
  IMPS_REQUIRE(s >= 1 && s <= A.s && s <= B.s && s <= 8, IMPS_INVALID_ARG, "split_gemm: bad slice count");
  // the shared-memory opt-in is per device; setting it again is harmless
  static std::atomic<uint64_t> attr_devices{0};
  const uint64_t bit = 1ull << (ctx->device & 63);
  if (!(attr_devices.load() & bit)) {
    for (auto k : {k_gemm_i8<0, 64>, k_gemm_i8<5, 96>, k_gemm_i8<6, 80>, k_gemm_i8<2, 128>, k_gemm_i8<3, 128>,
                   k_gemm_i8<4, 128>})
      IMPS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem_bytes()));
    attr_devices.fetch_or(bit);
  }
  // tile width by slice count (TMEM holds s x BN columns): 128 for 2..4 slices, 96 for 5,
  // 80 for 6, 64 otherwise.  The B planes are padded to 128 rows; a 96- or 80-row box
  // that reaches past them reads TMA's zero fill (and still delivers its full byte count).
  const int bn = (s >= 2 && s <= 6) ? bn_for(s) : 64;
  const CUtensorMap mapA = make_map(static_cast<const int8_t*>(A.data.ptr), A.Kp, A.Rp, A.s, BM);
  const CUtensorMap mapB = make_map(static_cast<const int8_t*>(B.data.ptr), B.Kp, B.Rp, B.s, bn);
  GemmArgs g;
  g.num_m = (int)(A.Rp / BM);
  g.num_n = (B.rows + bn - 1) / bn;
  // stream the larger operand once: consecutive CTAs share its tile and walk the other
  g.n_fast = (A.Rp * A.s >= B.Rp * B.s) ? 1 : 0;
  g.kblocks = (int)(A.Kp / KB);
  g.s = s;
  g.nst = stages_for(s, bn);
  g.nbuf = bufs_for(s, bn);
  g.C = C;
  g.ldc = ldc;
  g.Mc = A.rows;
  g.Nc = B.rows;
  g.row_scale = A.scale.d();
  g.col_scale = B.scale.d();
  g.alpha = alpha;
  g.accumulate = accumulate ? 1 : 0;
  g.err = ctx->err_dev;
  g.wait_cycles = ctx->wait_cycles;
  const int ntiles = g.num_m * g.num_n;
  const int grid = std::max(1, std::min(ntiles, ctx->num_sms));
  const int smem = smem_bytes_for(s, bn);
  {
    ScopedTimer tm(ctx, "gemm_split",
                   2.0 * (double)A.Rp * (double)g.num_n * bn * (double)A.Kp * (double)(s * (s + 1) / 2));
    switch (s) {
      case 2: k_gemm_i8<2, 128><<<grid, NTHREADS, smem, ctx->stream>>>(mapA, mapB, g); break;
      case 3: k_gemm_i8<3, 128><<<grid, NTHREADS, smem, ctx->stream>>>(mapA, mapB, g); break;
      case 4: k_gemm_i8<4, 128><<<grid, NTHREADS, smem, ctx->stream>>>(mapA, mapB, g); break;
      case 5: k_gemm_i8<5, 96><<<grid, NTHREADS, smem, ctx->stream>>>(mapA, mapB, g); break;
      case 6: k_gemm_i8<6, 80><<<grid, NTHREADS, smem, ctx->stream>>>(mapA, mapB, g); break;
      default: k_gemm_i8<0, 64><<<grid, NTHREADS, smem, ctx->stream>>>(mapA, mapB, g); break;
    }
    ctx->n_kernels++;
    ctx->n_gemm++;
    IMPS_CUDA(cudaPeekAtLastError());
  }
  ctx->split_launches++;
  ctx->split_alg_flops += 8.0 * (double)A.rows * (double)B.rows * (double)A.K;
  ctx->split_exec_ops += 2.0 * (double)A.Rp * (double)g.num_n * bn * (double)A.Kp * (double)(s * (s + 1) / 2);
  // the error flag is read at the context's next host synchronisation
  ctx->err_armed = true;
}

}  // namespace imps
