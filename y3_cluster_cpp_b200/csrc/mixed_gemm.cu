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
// A persistent CTA per SM walks the (point, 128-row lnM tile, richness-bin
// group) tiles: warps 1-11 generate operands into a 4-stage shared-memory
// ring, warp 0 issues the MMAs into one of two TMEM accumulators, warps 12-15
// drain the other; full/empty mbarriers (empty signalled by tcgen05.commit)
// order the ring and the accumulators, and every wait is bounded.
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

// 32 lanes x 16 columns of FP32 from TMEM.
__device__ __forceinline__ void
tmem_ld16(uint32_t taddr, float* v)
{
  uint32_t r[16];
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
    "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
      "=r"(r[14]), "=r"(r[15])
    : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Split 8 FP32 values into bf16 hi + lo and store one 16-byte core-matrix
// row of each.
__device__ __forceinline__ void
store_split8(uint8_t* hi, uint8_t* lo, const float* v)
{
  uint32_t h[4], l[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    __nv_bfloat162 hb = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
    float2 hf = __bfloat1622float2(hb);
    __nv_bfloat162 lb = __floats2bfloat162_rn(v[2 * k] - hf.x, v[2 * k + 1] - hf.y);
    h[k] = *reinterpret_cast<uint32_t*>(&hb);
    l[k] = *reinterpret_cast<uint32_t*>(&lb);
  }
  *reinterpret_cast<uint4*>(hi) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(lo) = make_uint4(l[0], l[1], l[2], l[3]);
}

constexpr long long kWaitBudget = 2000000000LL;  // SM cycles (~1 s)
constexpr int kMmaWarp = 0;        // issues tcgen05.mma
constexpr int kProdWarp0 = 1;      // warps 1..8 generate operands (one F and one A item each)
constexpr int kProdWarps = 8;
constexpr int kEpiWarp0 = 9;       // warps 9..16 drain TMEM (warp w reads lanes 32 (w % 4)..)
constexpr int kEpiWarps = 8;
constexpr int kThreads = 32 * (1 + kProdWarps + kEpiWarps);  // 544
constexpr int kStageK = 16;        // lam_t nodes per pipeline stage (one MMA k-step)
constexpr int kStages = 4;
constexpr int kAccCols = 256;      // TMEM columns per accumulator buffer (2 buffers)

__host__ __device__ inline uint32_t
stage_bytes(int ncp)
{
  return 2u * kGemmRows * kStageK * 2u + 2u * (uint32_t)ncp * kStageK * 2u;
}

// shared memory: stage ring | producer floats | epilogue floats | control
__host__ __device__ inline uint32_t
prod_floats(int n_z, int n_t_pad, int nIc)
{
  return kGemmRows + n_z + n_t_pad + nIc * n_t_pad;
}

__host__ __device__ inline uint32_t
epi_floats(int n_z, int nJ)
{
  return 2 * nJ * n_z;
}

__device__ __forceinline__ void
mbar_arrive(uint32_t addr)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
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

// Named barrier over `count` threads (the producer or the epilogue group).
__device__ __forceinline__ void
group_sync(int id, int count)
{
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Warp-uniform bounded wait (lane 0 polls, the warp follows).
__device__ __forceinline__ bool
warp_wait(uint32_t addr, uint32_t parity, volatile int* abort_flag, int lane)
{
  int ok = 1;
  if (lane == 0) ok = mbar_wait_or_abort(addr, parity, abort_flag);
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

struct TileIdx {
  int p, mtile, bg;
};

__device__ __forceinline__ TileIdx
tile_of(int t, int n_mt, int n_bg)
{
  TileIdx r;
  r.bg = t % n_bg;
  t /= n_bg;
  r.mtile = t % n_mt;
  r.p = t / n_mt;
  return r;
}

}  // namespace

// Persistent kernel: one CTA per SM loops over tiles (point, 128-row lnM
// tile, richness-bin group).  A tile's accumulator is nIc n_z <= 256 TMEM
// columns; two buffers let the epilogue of tile j overlap the MMAs of tile
// j+1.  Roles: warp 0 issues MMAs; warps 1-11 fill a 4-stage shared-memory
// ring (full/empty mbarriers, empty signalled by tcgen05.commit); warps 12-15
// read TMEM, apply Y(k,q) and the z-bin weights and write W_ij(k) in FP64.
template <int NJ, bool SHEAR>
__global__ void __launch_bounds__(kThreads, 1)
mixed_gemm_kernel(const GridDev* __restrict__ grids, const PointDev* __restrict__ pts,
                  int n_points, int grid_id, const float* __restrict__ s32,
                  double* __restrict__ Wout, double* __restrict__ Wgout, int w_stride,
                  int* status)
{
  const GridDev* Gp = grids + grid_id;
  const int n_m = Gp->n_m, n_z = Gp->n_z, n_t_pad = Gp->n_t_pad, nI = Gp->nI, nB = Gp->nB;
  const int nIc = Gp->nIc, ncp = Gp->ncp_c, n_m_pad = Gp->n_m_pad, n_bg = Gp->n_bg;
  const int n_mt = n_m_pad / kGemmRows;
  const int n_tiles = n_points * n_mt * n_bg;
  const bool uk_smem = Gp->uk_zindep != 0;
  const float* __restrict__ UK = Gp->UK;
  const size_t s32_stride = Gp->s32_stride;
  const size_t f_a = Gp->f_a, f_b = Gp->f_b, f_delta = Gp->f_delta, f_scal = Gp->f_scal;
  const size_t f_CN = Gp->f_CN, f_CG = Gp->f_CG, f_Yt = Gp->f_Yt;
  const int nk = n_t_pad / kStageK;
  const uint32_t SB = stage_bytes(ncp);
  const uint32_t lboA = (uint32_t)ncp * 16u;
  const uint32_t lboF = kGemmRows * 16u;

  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float* a_s = reinterpret_cast<float*>(smem + kStages * SB);
  float* b_s = a_s + kGemmRows;
  float* d_s = b_s + n_z;
  float* UK_s = d_s + n_t_pad;
  float* CN_s = a_s + prod_floats(n_z, n_t_pad, nIc);
  float* CG_s = CN_s + NJ * n_z;
  uint32_t ctl = kStages * SB + 4u * (prod_floats(n_z, n_t_pad, nIc) + epi_floats(n_z, NJ));
  ctl = (ctl + 15u) & ~15u;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + ctl);
  uint64_t* empty = full + kStages;
  uint64_t* acc_full = empty + kStages;
  uint64_t* acc_empty = acc_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  volatile int* abort_s = reinterpret_cast<volatile int*>(tmem_slot + 1);

  // Zero the operand ring once: padded rows/columns stay zero throughout.
  for (uint32_t i = tid * 16u; i < kStages * SB; i += kThreads * 16u)
    *reinterpret_cast<uint4*>(smem + i) = make_uint4(0u, 0u, 0u, 0u);
  if (warp == kMmaWarp) tmem_alloc(smem_u32(tmem_slot), 2 * kAccCols);
  if (tid == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(smem_u32(&full[i]), kProdWarps);
      mbar_init(smem_u32(&empty[i]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&acc_full[b]), 1);
      mbar_init(smem_u32(&acc_empty[b]), kEpiWarps);
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
      int chunk = 0, j = 0, last_stage = -1, last_parity = 0;
      for (int t = blockIdx.x; t < n_tiles && !*abort_s; t += gridDim.x) {
        const TileIdx ti = tile_of(t, n_mt, n_bg);
        if (pts[ti.p].grid != grid_id || ti.bg * nIc >= nI) continue;
        const int buf = j & 1;
        if (j >= 2 && !mbar_wait_or_abort(smem_u32(&acc_empty[buf]), ((j >> 1) - 1) & 1, abort_s))
          break;
        tc_fence_after();
        const uint32_t dacc = tmem + (uint32_t)(buf * kAccCols);
        bool broke = false;
        for (int kc = 0; kc < nk; ++kc, ++chunk) {
          const int s = chunk % kStages;
          if (!mbar_wait_or_abort(smem_u32(&full[s]), (chunk / kStages) & 1, abort_s)) {
            broke = true;
            break;
          }
          tc_fence_after();
          const uint32_t fh = smem_u32(smem + s * SB), fl = fh + lboF * 2;
          const uint32_t ah = fl + lboF * 2, al = ah + lboA * 2;
          const uint64_t dfh = umma_desc(fh, lboF, 128), dfl = umma_desc(fl, lboF, 128);
          const uint32_t idesc = umma_idesc_bf16(kGemmRows, ncp);
          const uint64_t dah = umma_desc(ah, lboA, 128), dal = umma_desc(al, lboA, 128);
          umma_bf16(dacc, dfh, dah, idesc, kc != 0);
          umma_bf16(dacc, dfh, dal, idesc, 1u);
          umma_bf16(dacc, dfl, dah, idesc, 1u);
          umma_commit(smem_u32(&empty[s]));
          last_stage = s;
          last_parity = (chunk / kStages) & 1;
        }
        if (broke) break;
        umma_commit(smem_u32(&acc_full[buf]));  // tile j's accumulator is complete
        ++j;
      }
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
    // ---------------- operand producers ----------------
    const int ptid = tid - kProdWarp0 * 32;
    constexpr int kP = kProdWarps * 32;
    int chunk = 0, last_grid_loaded = 0;
    // Every producer runs every tile iteration (named barriers stay matched);
    // after an abort the waits return at once and the work is skipped.
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
      const TileIdx ti = tile_of(t, n_mt, n_bg);
      if (pts[ti.p].grid != grid_id || ti.bg * nIc >= nI) continue;
      const int i0 = ti.bg * nIc, nIh = min(nIc, nI - i0);
      const float* __restrict__ sp = s32 + (size_t)ti.p * s32_stride;
      // Per-tile vectors (all producers have finished the previous tile's
      // generation before they are overwritten).
      group_sync(1, kP);
      const float c1 = sp[f_scal], c2 = sp[f_scal + 1];
      const float sc1 = sqrtf(c1);
      for (int m = ptid; m < kGemmRows; m += kP) {
        const int row = ti.mtile * kGemmRows + m;
        a_s[m] = row < n_m ? sp[f_a + row] * sc1 : 0.f;
      }
      for (int q = ptid; q < n_z; q += kP) b_s[q] = sp[f_b + q] * c2;
      for (int u = ptid; u < n_t_pad; u += kP) d_s[u] = sp[f_delta + u] * sc1;
      if (uk_smem && (last_grid_loaded == 0 || last_grid_loaded != i0 + 1)) {
        for (int u = ptid; u < nIh * n_t_pad; u += kP) {
          const int il = u / n_t_pad, tt = u - il * n_t_pad;
          UK_s[u] = UK[((size_t)(i0 + il) * n_z) * n_t_pad + tt];  // the q = 0 slice
        }
        last_grid_loaded = i0 + 1;
      }
      group_sync(1, kP);
      const float inv_sc1 = 1.0f / sc1;
      for (int kc = 0; kc < nk; ++kc, ++chunk) {
        const int s = chunk % kStages;
        if (chunk >= kStages &&
            !warp_wait(smem_u32(&empty[s]), ((chunk / kStages) - 1) & 1, abort_s, lane))
          continue;
        if (*abort_s) continue;
        uint8_t* st = smem + s * SB;
        uint8_t* Fhi = st;
        uint8_t* Flo = st + lboF * 2;
        uint8_t* Ahi = Flo + lboF * 2;
        uint8_t* Alo = Ahi + lboA * 2;
        // F(t, k) = 2^-((delta_t - a_k) sqrt(c1))^2: thread -> (row m, kgroup g).
        {
          const int m = ptid & (kGemmRows - 1), g = ptid >> 7;
          const int t0 = kc * kStageK + g * 8;
          const float am = a_s[m];
          const float4 d0 = *reinterpret_cast<const float4*>(d_s + t0);
          const float4 d1 = *reinterpret_cast<const float4*>(d_s + t0 + 4);
          const float dd[8] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
          float v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const float d = dd[u] - am;
            v[u] = fast_exp2(-d * d);
          }
          if (ti.mtile * kGemmRows + m >= n_m) {
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = 0.f;
          }
          store_split8(Fhi + g * lboF + m * 16, Flo + g * lboF + m * 16, v);
        }
        // A((i, q), t) = u_t K_i(t, q) 2^(delta_t c2 b_q): thread -> (q, kgroup).
        for (int ia = ptid; ia < 2 * n_z; ia += kP) {
          const int g = ia >= n_z ? 1 : 0;
          const int q = ia - g * n_z;
          const int t0 = kc * kStageK + g * 8;
          const float bq = b_s[q] * inv_sc1;  // d_s carries sqrt(c1)
          const float4 d0 = *reinterpret_cast<const float4*>(d_s + t0);
          const float4 d1 = *reinterpret_cast<const float4*>(d_s + t0 + 4);
          const float dd[8] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
          float gq[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) gq[u] = fast_exp2(dd[u] * bq);
          for (int il = 0; il < nIh; ++il) {
            float4 u0, u1;
            if (uk_smem) {
              const float4* uk = reinterpret_cast<const float4*>(UK_s + il * n_t_pad + t0);
              u0 = uk[0];
              u1 = uk[1];
            } else {
              const float4* uk = reinterpret_cast<const float4*>(
                UK + ((size_t)((i0 + il) * n_z + q)) * n_t_pad + t0);
              u0 = __ldg(uk);
              u1 = __ldg(uk + 1);
            }
            float v[8] = {u0.x * gq[0], u0.y * gq[1], u0.z * gq[2], u0.w * gq[3],
                          u1.x * gq[4], u1.y * gq[5], u1.z * gq[6], u1.w * gq[7]};
            const int row = il * n_z + q;
            store_split8(Ahi + g * lboA + row * 16, Alo + g * lboA + row * 16, v);
          }
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&full[s]));
      }
    }
  } else {
    // ---------------- epilogue ----------------
    const int etid = tid - kEpiWarp0 * 32;
    constexpr int kE = kEpiWarps * 32;
    const int lq = warp & 3;                  // TMEM lane quarter of this warp
    const int eg = (warp - kEpiWarp0) >> 2;   // which half of the bins
    constexpr int kEG = kEpiWarps / 4;
    const uint32_t lane_base = (uint32_t)(lq * 32) << 16;
    int j = 0;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
      const TileIdx ti = tile_of(t, n_mt, n_bg);
      if (pts[ti.p].grid != grid_id || ti.bg * nIc >= nI) continue;
      const int i0 = ti.bg * nIc, nIh = min(nIc, nI - i0);
      const float* __restrict__ sp = s32 + (size_t)ti.p * s32_stride;
      group_sync(2, kE);
      for (int u = etid; u < NJ * n_z; u += kE) {
        CN_s[u] = sp[f_CN + u];
        if (SHEAR) CG_s[u] = sp[f_CG + u];
      }
      group_sync(2, kE);
      const int buf = j & 1;
      ++j;
      if (!warp_wait(smem_u32(&acc_full[buf]), ((j - 1) >> 1) & 1, abort_s, lane)) continue;
      tc_fence_after();
      const int row = ti.mtile * kGemmRows + lq * 32 + lane;
      const bool valid = row < n_m;
      const float* __restrict__ Yr = sp + f_Yt + (valid ? row : 0);
      const uint32_t tbase = tmem + lane_base + (uint32_t)(buf * kAccCols);
      for (int il = eg; il < nIh; il += kEG) {
        const int i = i0 + il;
        double accN[NJ], accG[NJ];
#pragma unroll
        for (int jj = 0; jj < NJ; ++jj) accN[jj] = accG[jj] = 0.0;
        for (int qc = 0; qc < n_z; qc += 16) {
          float v[16];
          tmem_ld16(tbase + (uint32_t)(il * n_z + qc), v);
          float pN[NJ], pG[NJ];
#pragma unroll
          for (int jj = 0; jj < NJ; ++jj) pN[jj] = pG[jj] = 0.f;
          const float* __restrict__ yq = Yr + (size_t)qc * n_m_pad;
#pragma unroll
          for (int u = 0; u < 16; ++u) {
            const int q = qc + u;
            const float e = v[u] * __ldg(yq + (size_t)u * n_m_pad);
#pragma unroll
            for (int jj = 0; jj < NJ; ++jj) {
              pN[jj] = fmaf(CN_s[jj * n_z + q], e, pN[jj]);
              if (SHEAR) pG[jj] = fmaf(CG_s[jj * n_z + q], e, pG[jj]);
            }
          }
#pragma unroll
          for (int jj = 0; jj < NJ; ++jj) {
            accN[jj] += (double)pN[jj];
            if (SHEAR) accG[jj] += (double)pG[jj];
          }
        }
        if (valid) {
#pragma unroll
          for (int jj = 0; jj < NJ; ++jj) {
            const size_t o = ((size_t)ti.p * nB + i + nI * jj) * w_stride + row;
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
  }
  __syncthreads();
  if (*abort_s && tid == 0) set_err(status, kDevTimeout);
  if (warp == kMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * kAccCols);
  }
}

size_t
mixed_gemm_smem_bytes(int ncp, int n_z, int n_t_pad, int nJ, int nIc)
{
  size_t b = kStages * (size_t)stage_bytes(ncp) +
             4u * (prod_floats(n_z, n_t_pad, nIc) + epi_floats(n_z, nJ));
  b = (b + 15) & ~size_t(15);
  return b + 8 * (2 * kStages + 4) + 16;
}

template <int NJ, bool SHEAR>
static int
launch_nj(const MixedLaunch& L, size_t smem)
{
  auto k = mixed_gemm_kernel<NJ, SHEAR>;
  Y3B_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const GridDev& g = *L.g_host;
  int dev = 0, n_sm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  const long long tiles = (long long)L.n_points * (g.n_m_pad / kGemmRows) * g.n_bg;
  const int blocks = (int)std::min<long long>(tiles, n_sm);
  k<<<blocks, kThreads, smem, L.stream>>>(L.grids, L.pts, L.n_points, L.grid_id, L.s32, L.W,
                                          L.Wg, L.w_stride, L.status);
  count_launch();
  return cuda_status(cudaGetLastError(), "mixed_gemm_kernel");
}

template <bool SHEAR>
static int
launch_shear(const MixedLaunch& L, size_t smem)
{
  switch (L.g_host->nJ) {
    case 1: return launch_nj<1, SHEAR>(L, smem);
    case 2: return launch_nj<2, SHEAR>(L, smem);
    case 3: return launch_nj<3, SHEAR>(L, smem);
    case 4: return launch_nj<4, SHEAR>(L, smem);
    case 5: return launch_nj<5, SHEAR>(L, smem);
    case 6: return launch_nj<6, SHEAR>(L, smem);
    case 7: return launch_nj<7, SHEAR>(L, smem);
    case 8: return launch_nj<8, SHEAR>(L, smem);
    default:
      set_error("mixed_gemm: n_z_bins must be 1..8");
      return Y3B_ERR_UNSUPPORTED;
  }
}

int
launch_mixed_gemm(const MixedLaunch& L)
{
  const GridDev& g = *L.g_host;
  size_t smem = mixed_gemm_smem_bytes(g.ncp_c, g.n_z, g.n_t_pad, g.nJ, g.nIc);
  return L.shear ? launch_shear<true>(L, smem) : launch_shear<false>(L, smem);
}

}  // namespace y3b
