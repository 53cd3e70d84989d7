// mixed_gemm.cu -- the lambda_t contraction of the number-count integral on
// the sm_100a tensor cores (tcgen05.mma, accumulators in TMEM).
//
// The lognormal MOR density exp(-(l_t - mu_kq)^2 / 2 s^2) has
// mu_kq = alpha_k + beta_q (mass and redshift parts add), so with centred
// delta_t = l_t - L, a_k = alpha_k - A0, b_q = beta_q - B0 (L = A0 + B0)
//   exp(-(l_t - mu_kq)^2 / 2s^2) = F(t,k) G(t,q) H(k,q)
//   F = exp(-(delta_t - a_k)^2 / 2s^2)        (<= 1)
//   G = exp(delta_t b_q / s^2)                (|exponent| <~ 20)
//   H = exp(-(a_k b_q + b_q^2/2) / s^2)       (folded into the epilogue)
// and the sum over lambda_t becomes, for every point, the dense product
//   D[k, (i,q)] = sum_t F(t,k) * [u_t K_i(t,q) G(t,q)]
// of shape (n_m) x (n_lam_bins n_z) x (n_lam_t): 256 x 512 x 256 at the
// 4x-density grid.  Both operands are generated on the fly from the point's
// factor vectors (FP32, MUFU ex2), split into bf16 hi + lo, and contracted as
// three bf16 MMAs (hi*hi + hi*lo + lo*hi) with FP32 accumulation in TMEM.
// The epilogue multiplies by Y(k,q) = n(M_k,z_q) H(k,q) / (sqrt(2pi) s D_kq)
// and contracts z_t with the FP32 weights C_j(q) = v_q dV Omega K_j(q) into
// FP64 mass weights W_ij(k) (and the Sigma_crit-weighted W^gamma_ij(k)).
//
// One launch covers the points of every grid: a planner kernel orders the
// points by the cost of their grid's tiles and a persistent CTA per SM walks
// the (point, 128-row lnM tile, richness-bin group) tiles in that order:
// warps 1-16 generate the operand u_t K_i G(t, q) into a shared-memory ring
// of up to 8 stages (filled two stages at a time), warp 26 streams the
// matching F(t, k) blocks (written by the prep kernels) by bulk copies, one
// per pair of stages, warp 0 issues the MMAs of a pair of stages into one of
// two TMEM accumulators, warps 17-24 drain the other; full/empty mbarriers
// (empty signalled by tcgen05.commit) order the rings and the accumulators,
// and every wait is bounded.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "engine_internal.h"
#include "host_common.h"

namespace y3b {

namespace {

__device__ __forceinline__ uint32_t
smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor, K-major, no swizzle: 8-row x 16-byte core
// matrices; lbo = byte distance between the two K-adjacent core matrices,
// sbo = byte distance between 8-row groups; version 1 (sm_100) at bit 46.
__device__ __forceinline__ uint64_t
umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor, kind::f16: D = F32 (bits 4-5), A = B = BF16
// (bits 7-9, 10-12), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__device__ __forceinline__ uint32_t
umma_idesc_bf16(int M, int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void
umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
  asm volatile(
    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
    "l"(a), "l"(b), "r"(idesc), "r"(acc)
    : "memory");
}

__device__ __forceinline__ void
umma_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                 mbar)
               : "memory");
}

__device__ __forceinline__ void
tmem_alloc(uint32_t dst_smem, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void
tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void
tc_fence_before()
{
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void
tc_fence_after()
{
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void
fence_proxy_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void
mbar_init(uint32_t addr, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

// try_wait with a suspend-time hint: the waiting thread sleeps in hardware
// until the phase completes or ~1 ms passes, instead of spinning on issue
// slots the producer warps need.
__device__ __forceinline__ bool
mbar_try_wait(uint32_t addr, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
    "selp.u32 %0, 1, 0, p;\n\t}\n"
    : "=r"(ok)
    : "r"(addr), "r"(parity), "r"(1000000u)
    : "memory");
  return ok != 0;
}

// 32 lanes x 8 columns of FP32 from TMEM, issued without waiting: the
// registers are valid only after tmem_ld_wait on the same array.
__device__ __forceinline__ void
tmem_ld8_issue(uint32_t taddr, uint32_t* r)
{
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

// Waits for the thread's outstanding TMEM loads; the array's registers are
// operands, so no use of them moves above the wait.
__device__ __forceinline__ void
tmem_ld_wait(uint32_t* r)
{
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7])
               :
               : "memory");
}

constexpr long long kWaitBudget = 2000000000LL;  // SM cycles (~1 s)
constexpr int kMmaWarp = 0;        // issues tcgen05.mma
constexpr int kAWarp0 = 1;         // warps 1..16: A((i, q), t), thread -> (q, k half, bin)
constexpr int kAWarps = 16;
constexpr int kProdWarps = kAWarps;
constexpr int kEpiWarp0 = 17;      // warps 17..24 drain TMEM (warp w reads lanes 32 (w % 4)..)
constexpr int kEpiWarps = 8;
constexpr int kLoadWarp = 25;      // stages the next tile's factor vectors in shared memory
constexpr int kFLoadWarp = 26;     // copies the F(t, k) blocks of each pair of stages (prep kernel output)
constexpr int kThreads = 32 * 27;  // 864
constexpr int kStageK = 16;        // lam_t nodes per pipeline stage (one MMA k-step)
constexpr int kMaxStages = 8;      // depth of the A ring (tuned), at most 8
constexpr int kMaxFStages = 16;    // F ring in stages (even: slots of two): what shared memory leaves
constexpr int kAccCols = 256;      // TMEM columns per accumulator buffer (2 buffers)
constexpr uint32_t kFPlane = kGemmRows * kStageK * 2;        // one bf16 plane of F: 4 KB
constexpr uint32_t kAPlane = kAccCols * kStageK * 2;         // one bf16 plane of A: 8 KB
constexpr uint32_t kStageBytes = 2 * kAPlane;               // A ring stage, hi + lo: 16 KB
constexpr uint32_t kLboF = kGemmRows * 16;                   // K-adjacent core matrices of F

__device__ __forceinline__ void
mbar_arrive(uint32_t addr)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
}

// Non-suspending probe of an mbarrier phase (the MMA thread polls: it has
// nothing else to do and must react at once).
__device__ __forceinline__ bool
mbar_test(uint32_t addr, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
    "selp.u32 %0, 1, 0, p;\n\t}\n"
    : "=r"(ok)
    : "r"(addr), "r"(parity)
    : "memory");
  return ok != 0;
}

// Bounded polling wait for the MMA thread; gives up when another warp aborts.
__device__ __forceinline__ bool
mbar_poll_or_abort(uint32_t addr, uint32_t parity, volatile int* abort_flag)
{
  long long t0 = clock64();
  while (!mbar_test(addr, parity)) {
    if (*abort_flag) return false;
    if (clock64() - t0 > kWaitBudget) {
      *abort_flag = 1;
      return false;
    }
  }
  return true;
}

// Bounded wait that also gives up as soon as another warp has aborted.
__device__ __forceinline__ bool
mbar_wait_or_abort(uint32_t addr, uint32_t parity, volatile int* abort_flag)
{
  long long t0 = clock64();
  while (!mbar_try_wait(addr, parity)) {
    if (*abort_flag) return false;
    if (clock64() - t0 > kWaitBudget) {
      *abort_flag = 1;
      return false;
    }
  }
  return true;
}

// Named barrier over `count` threads (the epilogue group).
__device__ __forceinline__ void
group_sync(int id, int count)
{
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Warp-uniform bounded wait (lane 0 polls briefly, then suspends; the warp
// follows).
__device__ __forceinline__ bool
warp_wait(uint32_t addr, uint32_t parity, volatile int* abort_flag, int lane)
{
  int ok = 1;
  if (lane == 0) {
    bool done = false;
    for (int i = 0; i < 64 && !done; ++i) done = mbar_test(addr, parity);
    if (!done) ok = mbar_wait_or_abort(addr, parity, abort_flag);
  }
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

// Position in the operand ring: stage s and the parity of its current use.
struct RingPos {
  int s = 0;
  uint32_t ph = 0;
  __device__ __forceinline__ void next(int n)
  {
    if (++s == n) {
      s = 0;
      ph ^= 1u;
    }
  }
};

// Untiled bulk copy global -> shared completing on mbarrier `mbar` (16-byte
// aligned addresses, size a multiple of 16).
__device__ __forceinline__ void
bulk_g2s(void* dst, const void* src, uint32_t bytes, uint32_t mbar)
{
  asm volatile(
    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
      smem_u32(dst)),
    "l"(src), "r"(bytes), "r"(mbar)
    : "memory");
}

// Tile t of the launch: tile_list[t] = (point << 8) | local tile, local
// tiles of a point with the richness-bin groups varying fastest; the tile's
// lam_t stage window (first | end << 16) is win_tile[point][local].
__host__ __device__ inline int
vec_slot_floats(int nz_max, int ntp_max, int uk_max)
{
  return 4 + kGemmRows + nz_max + ntp_max + uk_max;
}

// Eight columns of a row's accumulator: times Y(k, q) (Y stored
// [z / 2][row][2], one 8-byte load per z pair), contracted with the z-bin
// weights four z nodes per load into packed FP32x2 partial sums (even and
// odd z nodes side by side).
template <int NJ, bool SHEAR>
__device__ __forceinline__ void
epi_chunk8(const uint32_t* r, int qc, const float2* __restrict__ Ys2, int rl,
           const float* __restrict__ CN_s, const float* __restrict__ CG_s, int n_z, float2* pN,
           float2* pG)
{
#pragma unroll
  for (int u = 0; u < 8; u += 4) {
    const int q = qc + u;
    const float2 y01 = Ys2[(q >> 1) * kGemmRows + rl];
    const float2 y23 = Ys2[((q >> 1) + 1) * kGemmRows + rl];
    const float2 e0 = __fmul2_rn(make_float2(__uint_as_float(r[u]), __uint_as_float(r[u + 1])), y01);
    const float2 e1 =
      __fmul2_rn(make_float2(__uint_as_float(r[u + 2]), __uint_as_float(r[u + 3])), y23);
#pragma unroll
    for (int jj = 0; jj < NJ; ++jj) {
      const float4 c = *reinterpret_cast<const float4*>(CN_s + jj * n_z + q);
      pN[jj] = __ffma2_rn(make_float2(c.x, c.y), e0, pN[jj]);
      pN[jj] = __ffma2_rn(make_float2(c.z, c.w), e1, pN[jj]);
      if (SHEAR) {
        const float4 g = *reinterpret_cast<const float4*>(CG_s + jj * n_z + q);
        pG[jj] = __ffma2_rn(make_float2(g.x, g.y), e0, pG[jj]);
        pG[jj] = __ffma2_rn(make_float2(g.z, g.w), e1, pG[jj]);
      }
    }
  }
}

struct Tile {
  int p, mtile, bg;
  int kc_lo, kc_hi;  // lam_t stages of the tile's window (pairs)
  const GridDev* G;
};

__device__ __forceinline__ Tile
decode_tile(int t, const int* __restrict__ tile_list, const int* __restrict__ win_tile,
            int win_stride, const PointDev* __restrict__ pts, const GridDev* __restrict__ grids)
{
  const int v = __ldg(tile_list + t);
  Tile T;
  T.p = v >> 8;
  const int local = v & 255;
  const int w = __ldg(win_tile + (size_t)T.p * win_stride + local);
  T.G = grids + pts[T.p].grid;
  const int n_bg = T.G->n_bg;
  T.bg = local % n_bg;
  T.mtile = local / n_bg;
  T.kc_lo = w & 0xFFFF;
  T.kc_hi = w >> 16;
  return T;
}

// Exclusive prefix sum over the 1024 threads of a block; *total = the sum.
__device__ __forceinline__ int
block_excl_scan(int v, int* sh, int* total)
{
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    const int y = sh[lane];
    int z = y;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= o) z += u;
    }
    sh[lane] = z - y;
    if (lane == 31) sh[32] = z;
  }
  __syncthreads();
  const int r = sh[w] + x - v;
  *total = sh[32];
  __syncthreads();
  return r;
}

}  // namespace

// Orders the points by the cost of their grid's tiles (most expensive grid
// first, stable inside a grid) and writes the tiles of the launch in that
// order: tile_start[i] = tiles of order[0..i), tile_start[n] = all tiles,
// tile_list[t] = (point << 8) | tile inside the point, and adds the stage
// count of the full lam_t range to stage_count[1] (the contraction adds the
// stages it issues to stage_count[0]; both are zeroed once per evaluation
// call, so the chunks of one call accumulate).  One block of 1024
// threads, each owning a contiguous chunk of points.  Points whose grid is
// not in the mask are put last with no tiles.
__global__ void __launch_bounds__(1024)
tile_plan_kernel(const GridDev* __restrict__ grids, int n_grids, int grid_mask,
                 const PointDev* __restrict__ pts, int n, int* __restrict__ order,
                 int* __restrict__ tile_start, int* __restrict__ tile_list,
                 int* __restrict__ stage_count)
{
  __shared__ int sh[33];
  const int C = (n + 1023) / 1024;
  const int b = min(n, (int)threadIdx.x * C), e = min(n, b + C);
  int base = 0;
  for (int r = 0; r <= n_grids; ++r) {  // r == n_grids: points outside the mask
    int c = 0;
    for (int i = b; i < e; ++i) {
      const int g = pts[i].grid;
      const int key = grid_in_mask(grid_mask, g) ? grids[g].cost_rank : n_grids;
      c += key == r;
    }
    int tot;
    int pos = base + block_excl_scan(c, sh, &tot);
    for (int i = b; i < e; ++i) {
      const int g = pts[i].grid;
      const int key = grid_in_mask(grid_mask, g) ? grids[g].cost_rank : n_grids;
      if (key == r) order[pos++] = i;
    }
    base += tot;
  }
  __syncthreads();
  int c = 0;
  for (int i = b; i < e; ++i) {
    const int g = pts[order[i]].grid;
    c += grid_in_mask(grid_mask, g) ? grids[g].tiles_pp : 0;
  }
  int tot;
  int off = block_excl_scan(c, sh, &tot);
  int dn = 0;  // stages of the full lam_t range, this thread's tiles
  for (int i = b; i < e; ++i) {
    tile_start[i] = off;
    const int p = order[i], g = pts[p].grid;
    const int nt = grid_in_mask(grid_mask, g) ? grids[g].tiles_pp : 0;
    for (int l = 0; l < nt; ++l) tile_list[off + l] = (p << 8) | l;
    if (nt) dn += nt * (grids[g].n_t_pad / kStageK);
    off += nt;
  }
  if (threadIdx.x == 0) tile_start[n] = tot;
  int dn_tot;
  block_excl_scan(dn, sh, &dn_tot);
  if (threadIdx.x == 0) stage_count[1] += dn_tot;
}

// Persistent contraction: one CTA per SM walks the launch's tiles (point,
// 128-row lnM tile, richness-bin group), points of every grid in one launch,
// most expensive grid first.  A tile's accumulator is nIc n_z <= 256 TMEM
// columns; two buffers let the epilogue of tile j overlap the MMAs of tile
// j+1.  Roles: warp 0 issues the MMAs; warps 1-8 generate F and warps 9-16
// generate A into an n_stages-deep shared-memory ring (full/empty mbarriers,
// empty signalled by tcgen05.commit), each thread reading its point's factor
// vectors straight from global memory, so no producer waits on another;
// warps 17-24 read TMEM, apply Y(k,q) and the z-bin weights and write
// W_ij(k) in FP64.  The tile's block of Y (n_z rows of 128 lnM values,
// contiguous in the tile-blocked layout) is brought into shared memory by one
// bulk async copy issued while the tile's MMAs run.
template <int NJ, bool SHEAR>
__global__ void __launch_bounds__(kThreads, 1)
contract_kernel(const GridDev* __restrict__ grids, const PointDev* __restrict__ pts,
                const int* __restrict__ tile_start, const int* __restrict__ tile_list,
                const int* __restrict__ win_tile, int win_stride, int* __restrict__ stage_count,
                int n_points, int nz_max, int ntp_max, int uk_max, int n_stages,
                int n_fstages, const uint8_t* __restrict__ fbuf, size_t f_stride,
                const float* __restrict__ s32, double* __restrict__ Wout,
                double* __restrict__ Wgout, int w_stride, int* status)
{
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n_tiles = __ldg(tile_start + n_points);
  const int nst = n_stages, nfs = n_fstages;
  const int nfp = nfs / 2;  // F ring slots: one pair of stages (16 KB) each
  uint8_t* fring = smem + nst * kStageBytes;                          // [nfs][8 KB]
  float* Ys = reinterpret_cast<float*>(fring + nfs * kFStageBytes);  // [n_z][128]
  float* CN_s = Ys + (size_t)nz_max * kGemmRows;
  float* CG_s = CN_s + NJ * nz_max;
  // Two slots of per-tile factor vectors: scal[4] | a[128] | b[nz_max] |
  // delta[ntp_max] | u_t K_i(t)[uk_max] (all 16-byte aligned).
  const int vec_floats = vec_slot_floats(nz_max, ntp_max, uk_max);
  float* vec_s = CG_s + NJ * nz_max;
  uint32_t ctl = nst * kStageBytes + nfs * kFStageBytes +
                 4u * ((uint32_t)nz_max * kGemmRows + 2u * NJ * nz_max + 2u * vec_floats);
  ctl = (ctl + 15u) & ~15u;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + ctl);
  uint64_t* empty = full + kMaxStages;
  uint64_t* acc_full = empty + kMaxStages;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* ybar = acc_empty + 2;
  uint64_t* vec_full = ybar + 1;
  uint64_t* vec_empty = vec_full + 2;
  uint64_t* fbar = vec_empty + 2;         // F ring: block landed
  uint64_t* fempty = fbar + kMaxFStages;  // F ring: MMAs done with the block
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fempty + kMaxFStages);
  volatile int* abort_s = reinterpret_cast<volatile int*>(tmem_slot + 1);
  // Per vector slot, the decoded tile the loader staged: point, lnM tile,
  // richness-bin group, window [kc_lo, kc_hi), grid index.
  int* tinfo_s = reinterpret_cast<int*>(tmem_slot + 4);

  // Zero the operand ring once: columns a tile does not write stay finite.
  for (uint32_t i = tid * 16u; i < nst * kStageBytes; i += kThreads * 16u)
    *reinterpret_cast<uint4*>(smem + i) = make_uint4(0u, 0u, 0u, 0u);
  fence_proxy_async_smem();  // the zeros come before the tensor core's reads and the copies
  if (warp == kMmaWarp) tmem_alloc(smem_u32(tmem_slot), 2 * kAccCols);
  if (tid == 0) {
    for (int i = 0; i < nst; ++i) {
      mbar_init(smem_u32(&full[i]), kProdWarps);
      mbar_init(smem_u32(&empty[i]), 1);
    }
    for (int i = 0; i < nfp; ++i) {
      mbar_init(smem_u32(&fbar[i]), 1);
      mbar_init(smem_u32(&fempty[i]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&acc_full[b]), 1);
      mbar_init(smem_u32(&acc_empty[b]), kEpiWarps);
    }
    mbar_init(smem_u32(ybar), 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&vec_full[b]), 1);
      mbar_init(smem_u32(&vec_empty[b]), kProdWarps);
    }
    *abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kMmaWarp) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      RingPos rp, rf;
      int j = 0, last_stage = -1, last_parity = 0, issued_stages = 0;
      for (int t = blockIdx.x; t < n_tiles && !*abort_s; t += gridDim.x) {
        const Tile T = decode_tile(t, tile_list, win_tile, win_stride, pts, grids);
        const int ncp = T.G->ncp_c;
        const int buf = j & 1;
        if (j >= 2 && !mbar_poll_or_abort(smem_u32(&acc_empty[buf]), ((j >> 1) - 1) & 1, abort_s))
          break;
        tc_fence_after();
        const uint32_t dacc = tmem + (uint32_t)(buf * kAccCols);
        const uint32_t idesc = umma_idesc_bf16(kGemmRows, ncp);
        const uint32_t lboA = (uint32_t)ncp * 16u;
        bool broke = false;
        // Stages in pairs (a window's count is even), as the producers fill
        // them: one wait on the pair's second full barrier (each producer
        // warp arrives on the first before the second) and one on its F
        // block pair, six MMAs, and one commit per ring slot.
        for (int kc = T.kc_lo; kc < T.kc_hi; kc += 2, rf.next(nfp)) {
          const int s0 = rp.s;
          rp.next(nst);
          const int s1 = rp.s;
          const uint32_t ph1 = rp.ph;
          rp.next(nst);
          const int f = rf.s;
          if (!mbar_poll_or_abort(smem_u32(&full[s1]), ph1, abort_s) ||
              !mbar_poll_or_abort(smem_u32(&fbar[f]), rf.ph, abort_s)) {
            broke = true;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const uint32_t fh = smem_u32(fring + (2 * f + h) * kFStageBytes), fl = fh + kFPlane;
            const uint32_t ah = smem_u32(smem + (h ? s1 : s0) * kStageBytes), al = ah + kAPlane;
            const uint64_t dfh = umma_desc(fh, kLboF, 128), dfl = umma_desc(fl, kLboF, 128);
            const uint64_t dah = umma_desc(ah, lboA, 128), dal = umma_desc(al, lboA, 128);
            umma_bf16(dacc, dfh, dah, idesc, (kc + h) != T.kc_lo);
            umma_bf16(dacc, dfh, dal, idesc, 1u);
            umma_bf16(dacc, dfl, dah, idesc, 1u);
            umma_commit(smem_u32(&empty[h ? s1 : s0]));
          }
          umma_commit(smem_u32(&fempty[f]));
          last_stage = s1;
          last_parity = (int)ph1;
        }
        if (broke) break;
        umma_commit(smem_u32(&acc_full[buf]));  // tile j's accumulator is complete
        issued_stages += T.kc_hi - T.kc_lo;
        ++j;
      }
      atomicAdd(stage_count, issued_stages);
      // Leave only when every issued MMA has completed (bounded).
      if (last_stage >= 0) {
        long long t0 = clock64();
        while (!mbar_try_wait(smem_u32(&empty[last_stage]), last_parity))
          if (clock64() - t0 > kWaitBudget) {
            *abort_s = 1;
            break;
          }
      }
    }
    __syncwarp();
  } else if (warp < kEpiWarp0) {
    // ---------------- A((i, q), t) = u_t K_i(t, q) 2^(delta_t b_q c2) ----------------
    const int a = tid - kAWarp0 * 32;
    int chunk = 0, jt = 0;
    RingPos rp;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++jt) {
      const int slot = jt & 1;
      const float* vs = vec_s + slot * vec_floats;
      if (!warp_wait(smem_u32(&vec_full[slot]), (jt >> 1) & 1, abort_s, lane)) continue;
      __syncwarp();  // orders lane 0's acquire before every lane's reads
      // The tile as the loader decoded it (no global-memory chain here).
      const int* ti = tinfo_s + 8 * slot;
      Tile T;
      T.p = ti[0];
      T.mtile = ti[1];
      T.bg = ti[2];
      T.kc_lo = ti[3];
      T.kc_hi = ti[4];
      T.G = grids + ti[5];
      const GridDev* G = T.G;
      const int n_z = G->n_z, ntp = G->n_t_pad;
      const int i0 = T.bg * G->nIc, nIh = min(G->nIc, G->nI - i0);
      const float c2 = vs[1];
      const float* dsm = vs + 132 + nz_max;
      // This thread's item: z node q, half g of the stage's 16 lam_t nodes,
      // the stage(s) h of the pair (hs = 2 groups of threads take one stage
      // each when 4 n_z <= 512, else each thread takes both), and bpt
      // richness bins, the fewest that let the 2 hs n_z ceil(nIh / bpt)
      // items fit the 512 threads.  G(t, q) = 2^(delta_t b_q c2) does not
      // depend on the bin: it is evaluated once per (q, t) and scaled by
      // u_t K_i(t) for each of the thread's bins.
      const int hs = n_z <= 128 ? 2 : 1;
      int bpt = 1;
      while (bpt < nIh && 2 * hs * n_z * ((nIh + bpt - 1) / bpt) > kProdWarps * 32) ++bpt;
      const int nsub = (nIh + bpt - 1) / bpt;
      const int q = a % n_z, rest = a / n_z;
      const int g = rest & 1, h0 = hs == 2 ? (rest >> 1) & 1 : 0;
      const int sub = hs == 2 ? rest >> 2 : rest >> 1;
      const int il0 = sub * bpt, nb = max(0, min(bpt, nIh - il0));
      const bool active = sub < nsub && nb > 0;
      const float bq = active ? vs[4 + kGemmRows + q] * c2 : 0.f;
      const float2 bq2 = make_float2(bq, bq);
      // u_t K_i(t): the staged copy when P(lam_o | lam_t) has no z dependence,
      // else the per-(i, q) rows in global memory.
      const bool uks = G->uk_zindep != 0 && nIh * ntp <= uk_max;
      const uint32_t lboA = (uint32_t)G->ncp_c * 16u;
      for (int kc = T.kc_lo; kc < T.kc_hi; kc += 2, chunk += 2) {
        int sp2[2];
        uint32_t ph2[2];
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          sp2[hh] = rp.s;
          ph2[hh] = rp.ph;
          rp.next(nst);
        }
        if (chunk >= nst && !warp_wait(smem_u32(&empty[sp2[0]]), ph2[0] ^ 1u, abort_s, lane))
          continue;
        if (chunk + 1 >= nst && !warp_wait(smem_u32(&empty[sp2[1]]), ph2[1] ^ 1u, abort_s, lane))
          continue;
        if (*abort_s) continue;
        for (int h = h0; active && h < (hs == 2 ? h0 + 1 : 2); ++h) {
          const int t0 = (kc + h) * kStageK + g * 8;
          const float4 d0 = *reinterpret_cast<const float4*>(dsm + t0);
          const float4 d1 = *reinterpret_cast<const float4*>(dsm + t0 + 4);
          const float2 dd[4] = {make_float2(d0.x, d0.y), make_float2(d0.z, d0.w),
                                make_float2(d1.x, d1.y), make_float2(d1.z, d1.w)};
          float2 gq[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float2 x = __fmul2_rn(dd[u], bq2);
            gq[u] = make_float2(fast_exp2(x.x), fast_exp2(x.y));
          }
          uint8_t* Ah = smem + sp2[h] * kStageBytes + (uint32_t)g * lboA;
          for (int b = 0; b < nb; ++b) {
            const int il = il0 + b;
            float4 u0, u1;
            if (uks) {
              const float* uksm = dsm + ntp_max + il * ntp;
              u0 = *reinterpret_cast<const float4*>(uksm + t0);
              u1 = *reinterpret_cast<const float4*>(uksm + t0 + 4);
            } else {
              const float* __restrict__ ukg = G->UK + ((size_t)((i0 + il) * n_z + q)) * ntp;
              u0 = __ldg(reinterpret_cast<const float4*>(ukg + t0));
              u1 = __ldg(reinterpret_cast<const float4*>(ukg + t0 + 4));
            }
            const float2 uu[4] = {make_float2(u0.x, u0.y), make_float2(u0.z, u0.w),
                                  make_float2(u1.x, u1.y), make_float2(u1.z, u1.w)};
            float2 v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = __fmul2_rn(uu[u], gq[u]);
            uint8_t* Ahi = Ah + (uint32_t)(il * n_z + q) * 16u;
            store_split8(Ahi, Ahi + kAPlane, v);
          }
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(smem_u32(&full[sp2[0]]));
          mbar_arrive(smem_u32(&full[sp2[1]]));
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&vec_empty[slot]));  // done with this slot
    }
  } else if (warp == kLoadWarp) {
    // ---------------- per-tile factor vectors, one tile ahead ----------------
    if (lane == 0) {
      int j = 0, issued = -1;
      for (int t = blockIdx.x; t < n_tiles && !*abort_s; t += gridDim.x, ++j) {
        const int slot = j & 1;
        if (j >= 2 && !mbar_wait_or_abort(smem_u32(&vec_empty[slot]), ((j >> 1) - 1) & 1, abort_s))
          break;
        const Tile T = decode_tile(t, tile_list, win_tile, win_stride, pts, grids);
        const GridDev* G = T.G;
        const int n_z = G->n_z, ntp = G->n_t_pad;
        const int i0 = T.bg * G->nIc, nIh = min(G->nIc, G->nI - i0);
        const bool uks = G->uk_zindep != 0 && nIh * ntp <= uk_max;
        const float* sp = s32 + (size_t)T.p * G->s32_stride;
        float* vs = vec_s + slot * vec_floats;
        const uint32_t bytes = 4u * (4 + n_z + ntp + (uks ? nIh * ntp : 0));
        const uint32_t vb = smem_u32(&vec_full[slot]);
        int* ti = tinfo_s + 8 * slot;  // published by the arrive below (release)
        ti[0] = T.p;
        ti[1] = T.mtile;
        ti[2] = T.bg;
        ti[3] = T.kc_lo;
        ti[4] = T.kc_hi;
        ti[5] = (int)(T.G - grids);
        fence_proxy_async_smem();  // the producers' reads of this slot come first
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(vb),
                     "r"(bytes)
                     : "memory");
        bulk_g2s(vs, sp + G->f_scal, 16u, vb);
        bulk_g2s(vs + 4 + kGemmRows, sp + G->f_b, 4u * n_z, vb);
        bulk_g2s(vs + 132 + nz_max, sp + G->f_delta, 4u * ntp, vb);
        if (uks)
          for (int il = 0; il < nIh; ++il)
            bulk_g2s(vs + 132 + nz_max + ntp_max + il * ntp,
                     G->UK + (size_t)(i0 + il) * n_z * ntp, 4u * ntp, vb);
        issued = j;
      }
      // Copies still in flight (after an abort) must land before the CTA's
      // shared memory is released: wait for the last two issued (bounded).
      for (int jj = max(0, issued - 1); jj <= issued; ++jj) {
        long long t0 = clock64();
        while (!mbar_try_wait(smem_u32(&vec_full[jj & 1]), (jj >> 1) & 1) &&
               clock64() - t0 < kWaitBudget) {
        }
      }
    }
    __syncwarp();
  } else if (warp == kFLoadWarp) {
    // ---------------- F(t, k) blocks, one bulk copy per pair of stages ----------------
    if (lane == 0) {
      RingPos rp;
      int chunk = 0;
      uint32_t issued = 0, last_ph = 0;  // per slot: copy issued, parity of its last use
      for (int t = blockIdx.x; t < n_tiles && !*abort_s; t += gridDim.x) {
        const Tile T = decode_tile(t, tile_list, win_tile, win_stride, pts, grids);
        const int nk = T.G->n_t_pad / kStageK;
        const uint8_t* src =
          fbuf + (size_t)T.p * f_stride + (size_t)T.mtile * nk * kFStageBytes;
        // Warm L2 with the next tile's F blocks while this tile streams.
        if (t + (int)gridDim.x < n_tiles) {
          const Tile Tn = decode_tile(t + gridDim.x, tile_list, win_tile, win_stride, pts, grids);
          const int nkn = Tn.G->n_t_pad / kStageK;
          const uint8_t* nsrc =
            fbuf + (size_t)Tn.p * f_stride + (size_t)Tn.mtile * nkn * kFStageBytes;
          for (int kc = Tn.kc_lo; kc < Tn.kc_hi; kc += 2)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(
                           nsrc + (size_t)kc * kFStageBytes),
                         "r"((uint32_t)(2 * kFStageBytes))
                         : "memory");
        }
        bool broke = false;
        for (int kc = T.kc_lo; kc < T.kc_hi; kc += 2, ++chunk, rp.next(nfp)) {
          const int s = rp.s;
          if (chunk >= nfp && !mbar_poll_or_abort(smem_u32(&fempty[s]), rp.ph ^ 1u, abort_s)) {
            broke = true;
            break;
          }
          const uint32_t fb = smem_u32(&fbar[s]);
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                       "r"((uint32_t)(2 * kFStageBytes))
                       : "memory");
          bulk_g2s(fring + 2 * s * kFStageBytes, src + (size_t)kc * kFStageBytes,
                   2 * kFStageBytes, fb);
          issued |= 1u << s;
          last_ph = (last_ph & ~(1u << s)) | (rp.ph << s);
        }
        if (broke) break;
      }
      // No copy may still be in flight when the CTA's shared memory is
      // released: wait for the last one issued into every slot (bounded).
      for (int s = 0; s < nfp; ++s) {
        if (!((issued >> s) & 1u)) continue;
        long long t0 = clock64();
        while (!mbar_try_wait(smem_u32(&fbar[s]), (last_ph >> s) & 1u) &&
               clock64() - t0 < kWaitBudget) {
        }
      }
    }
    __syncwarp();
  } else {
    // ---------------- epilogue ----------------
    const int etid = tid - kEpiWarp0 * 32;
    constexpr int kE = kEpiWarps * 32;
    const int lq = warp & 3;                  // TMEM lane quarter of this warp
    const int eg = (warp - kEpiWarp0) >> 2;   // which half of the bins
    constexpr int kEG = kEpiWarps / 4;
    const uint32_t lane_base = (uint32_t)(lq * 32) << 16;
    int j = 0, y_pending = 0;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
      const Tile T = decode_tile(t, tile_list, win_tile, win_stride, pts, grids);
      const GridDev* G = T.G;
      const int n_z = G->n_z, n_m = G->n_m, nI = G->nI, nB = G->nB;
      const int i0 = T.bg * G->nIc, nIh = min(G->nIc, nI - i0);
      const float* __restrict__ sp = s32 + (size_t)T.p * G->s32_stride;
      group_sync(2, kE);  // the previous tile's Y and weights are no longer read
      if (warp == kEpiWarp0 && !*abort_s) {
        // Y rows q of this tile: 128 lnM values each, one bulk copy per row.
        const uint32_t yb = smem_u32(ybar);
        if (lane == 0) {
          fence_proxy_async_smem();
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(yb),
                       "r"((uint32_t)n_z * kGemmRows * 4u)
                       : "memory");
        }
        __syncwarp();
        // Y is stored tile-blocked ([lnM tile][z][128 rows]): one copy.
        if (lane == 0)
          bulk_g2s(Ys, sp + G->f_Yt + (size_t)T.mtile * n_z * kGemmRows,
                   (uint32_t)n_z * kGemmRows * 4u, yb);
        y_pending = 1;
      }
      for (int u = etid; u < NJ * n_z; u += kE) {
        CN_s[u] = sp[G->f_CN + u];
        if (SHEAR) CG_s[u] = sp[G->f_CG + u];
      }
      group_sync(2, kE);
      const int buf = j & 1;
      ++j;
      if (!warp_wait(smem_u32(&acc_full[buf]), ((j - 1) >> 1) & 1, abort_s, lane)) continue;
      if (!warp_wait(smem_u32(ybar), (j - 1) & 1, abort_s, lane)) continue;
      y_pending = 0;
      tc_fence_after();
      const int rl = lq * 32 + lane;  // row inside the tile
      const float2* Ys2 = reinterpret_cast<const float2*>(Ys);
      const int row = T.mtile * kGemmRows + rl;
      const bool valid = row < n_m;
      const uint32_t tbase = tmem + lane_base + (uint32_t)(buf * kAccCols);
      for (int il = eg; il < nIh; il += kEG) {
        const int i = i0 + il;
        double accN[NJ], accG[NJ];
#pragma unroll
        for (int jj = 0; jj < NJ; ++jj) accN[jj] = accG[jj] = 0.0;
        // Two register sets: the TMEM load of the next 8 columns is in
        // flight while the current ones are contracted.  Every 16 columns
        // the FP32 partial sums are added in FP64 (n_z is a multiple of 16).
        const uint32_t tb = tbase + (uint32_t)(il * n_z);
        uint32_t ra[8], rb[8];
        tmem_ld8_issue(tb, ra);
        tmem_ld_wait(ra);
        for (int qc = 0; qc < n_z; qc += 16) {
          float2 pN[NJ], pG[NJ];
#pragma unroll
          for (int jj = 0; jj < NJ; ++jj) pN[jj] = pG[jj] = make_float2(0.f, 0.f);
          tmem_ld8_issue(tb + (uint32_t)(qc + 8), rb);
          epi_chunk8<NJ, SHEAR>(ra, qc, Ys2, rl, CN_s, CG_s, n_z, pN, pG);
          tmem_ld_wait(rb);
          const bool more = qc + 16 < n_z;  // warp-uniform
          if (more) tmem_ld8_issue(tb + (uint32_t)(qc + 16), ra);
          epi_chunk8<NJ, SHEAR>(rb, qc + 8, Ys2, rl, CN_s, CG_s, n_z, pN, pG);
#pragma unroll
          for (int jj = 0; jj < NJ; ++jj) {
            accN[jj] += (double)pN[jj].x + (double)pN[jj].y;
            if (SHEAR) accG[jj] += (double)pG[jj].x + (double)pG[jj].y;
          }
          if (more) tmem_ld_wait(ra);
        }
        if (valid) {
#pragma unroll
          for (int jj = 0; jj < NJ; ++jj) {
            const size_t o = ((size_t)T.p * nB + i + nI * jj) * w_stride + row;
            Wout[o] = accN[jj];
            if (SHEAR) Wgout[o] = accG[jj];
          }
        }
      }
      // Release this accumulator buffer to the MMA warp.
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acc_empty[buf]));
    }
    // After an abort a Y copy may still be in flight: wait for it (bounded)
    // before the CTA's shared memory is released.
    if (warp == kEpiWarp0 && y_pending && lane == 0) {
      long long t0 = clock64();
      while (!mbar_try_wait(smem_u32(ybar), (j - 1) & 1) && clock64() - t0 < kWaitBudget) {
      }
    }
  }
  __syncthreads();
  if (*abort_s && tid == 0) set_err(status, kDevTimeout);
  if (warp == kMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * kAccCols);
  }
}

// Shared memory of the contraction without its F ring, with `stages` A stages.
static size_t
contract_smem_base(int stages, const ContractShape& c)
{
  size_t b = (size_t)stages * kStageBytes +
             4u * ((size_t)c.nz_max * kGemmRows + 2u * c.nJ * c.nz_max +
                   2u * vec_slot_floats(c.nz_max, c.ntp_max, c.uk_max));
  b = (b + 15) & ~size_t(15);
  return b + 8 * (2 * kMaxStages + 2 * kMaxFStages + 9) + 16 + 2 * 8 * 4;
}

// F ring depth in stages that fits next to `stages` A stages (even, <= 16).
int
contract_fstages(int stages, const ContractShape& c)
{
  const size_t base = contract_smem_base(stages, c), cap = 227 * 1024;
  if (base >= cap) return 0;
  return (int)std::min<size_t>(kMaxFStages, (cap - base) / kFStageBytes) & ~1;
}

static size_t
contract_smem_at(int stages, const ContractShape& c)
{
  return contract_smem_base(stages, c) + (size_t)contract_fstages(stages, c) * kFStageBytes;
}

// Default A ring depth: the deepest (<= 8) that leaves at least 4 F stages;
// 0 if not even 2 A stages do.
int
contract_stages(const ContractShape& c)
{
  for (int st = kMaxStages; st >= 2; --st)
    if (contract_fstages(st, c) >= 4) return st;
  return 0;
}

size_t
contract_smem_bytes(const ContractShape& c)
{
  size_t m = 0;
  for (int st = 2; st <= kMaxStages; ++st)
    if (contract_fstages(st, c) >= 4) m = std::max(m, contract_smem_at(st, c));
  return m ? m : (size_t)-1;
}

template <int NJ, bool SHEAR>
static int
set_attr_nj(size_t smem)
{
  Y3B_CUDA(cudaFuncSetAttribute(contract_kernel<NJ, SHEAR>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return Y3B_OK;
}

template <int NJ, bool SHEAR>
static int
launch_nj(const ContractLaunch& L, size_t smem)
{
  auto k = contract_kernel<NJ, SHEAR>;
  const int blocks = (int)std::min<long long>(std::max<long long>(L.max_tiles, 1), L.n_ctas);
  k<<<blocks, kThreads, smem, L.stream>>>(L.grids, L.pts, L.tile_start, L.tile_list, L.win_tile,
                                          L.win_stride, L.stage_count, L.n_points,
                                          L.shape.nz_max, L.shape.ntp_max, L.shape.uk_max,
                                          L.stages, contract_fstages(L.stages, L.shape), L.fbuf,
                                          L.f_stride, L.s32, L.W, L.Wg,
                                          L.w_stride, L.status);
  count_launch();
  return cuda_status(cudaGetLastError(), "contract_kernel");
}

template <bool SHEAR>
static int
launch_shear(const ContractLaunch& L, size_t smem)
{
  switch (L.shape.nJ) {
    case 1: return launch_nj<1, SHEAR>(L, smem);
    case 2: return launch_nj<2, SHEAR>(L, smem);
    case 3: return launch_nj<3, SHEAR>(L, smem);
    case 4: return launch_nj<4, SHEAR>(L, smem);
    case 5: return launch_nj<5, SHEAR>(L, smem);
    case 6: return launch_nj<6, SHEAR>(L, smem);
    case 7: return launch_nj<7, SHEAR>(L, smem);
    case 8: return launch_nj<8, SHEAR>(L, smem);
    default:
      set_error("contract: n_z_bins must be 1..8");
      return Y3B_ERR_UNSUPPORTED;
  }
}

int
contract_prepare(const ContractShape& c)
{
  const size_t smem = contract_smem_bytes(c);
  if (smem == (size_t)-1) {
    set_error("contract: the grids need more shared memory than one CTA has");
    return Y3B_ERR_UNSUPPORTED;
  }
  switch (c.nJ) {
#define Y3B_ATTR(n) \
  case n: Y3B_TRY((set_attr_nj<n, false>(smem))); return set_attr_nj<n, true>(smem);
    Y3B_ATTR(1) Y3B_ATTR(2) Y3B_ATTR(3) Y3B_ATTR(4) Y3B_ATTR(5) Y3B_ATTR(6) Y3B_ATTR(7)
    Y3B_ATTR(8)
#undef Y3B_ATTR
    default:
      set_error("contract: n_z_bins must be 1..8");
      return Y3B_ERR_UNSUPPORTED;
  }
}

int
contract_check(const ContractLaunch& L)
{
  if (L.stages < 2 || L.stages > kMaxStages || contract_fstages(L.stages, L.shape) < 4 ||
      L.n_ctas < 1) {
    set_error("contract: ring depth %d outside [2, %d] or no CTAs", L.stages,
              contract_stages(L.shape));
    return Y3B_ERR_INVALID;
  }
  return Y3B_OK;
}

int
launch_plan(const ContractLaunch& L)
{
  tile_plan_kernel<<<1, 1024, 0, L.plan_stream>>>(L.grids, L.n_grids, L.grid_mask, L.pts,
                                                  L.n_points, L.order, L.tile_start, L.tile_list,
                                                  L.stage_count);
  count_launch();
  return cuda_status(cudaGetLastError(), "tile_plan_kernel");
}

int
launch_contract(const ContractLaunch& L)
{
  Y3B_TRY(contract_check(L));
  const size_t smem = contract_smem_at(L.stages, L.shape);
  return L.shear ? launch_shear<true>(L, smem) : launch_shear<false>(L, smem);
}

}  // namespace y3b
