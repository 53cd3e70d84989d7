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
// One CTA per (point, 128-row lnM tile); 256 threads generate operands into a
// two-stage shared-memory ring while thread 0 issues the MMAs; completion is
// tracked with tcgen05.commit -> mbarrier, every wait is bounded.
#include <cuda_bf16.h>

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

__device__ __forceinline__ bool
mbar_try_wait(uint32_t addr, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
    "selp.u32 %0, 1, 0, p;\n\t}\n"
    : "=r"(ok)
    : "r"(addr), "r"(parity)
    : "memory");
  return ok != 0;
}

// Bounded wait: gives up after `budget` SM cycles (about a second).
__device__ __forceinline__ bool
mbar_wait_bounded(uint32_t addr, uint32_t parity, long long budget)
{
  long long t0 = clock64();
  while (!mbar_try_wait(addr, parity)) {
    if (clock64() - t0 > budget) return false;
  }
  return true;
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

struct GemmDims {
  int n_m, n_z, n_t_pad, nI, nJ, nB, n_m_pad, ncp;
};

__host__ __device__ inline uint32_t
stage_bytes(int ncp)
{
  return 2u * kGemmRows * kKChunk * 2u + 2u * (uint32_t)ncp * kKChunk * 2u;
}

__host__ __device__ inline uint32_t
vec_offset(int ncp)
{
  return 2u * stage_bytes(ncp);
}

// floats after the stages: a[128] | b[n_z] | delta[n_t_pad] | CN[nJ n_z] | CG[nJ n_z]
__host__ __device__ inline uint32_t
vec_floats(int n_z, int n_t_pad, int nJ)
{
  return kGemmRows + n_z + n_t_pad + 2 * nJ * n_z;
}

}  // namespace

__global__ void __launch_bounds__(256, 1)
mixed_gemm_kernel(const GridDev* __restrict__ grids, const PointDev* __restrict__ pts,
                  int grid_id, const float* __restrict__ s32, double* __restrict__ Wout,
                  double* __restrict__ Wgout, int w_stride, int* status)
{
  const int p = blockIdx.y;
  if (pts[p].grid != grid_id) return;  // whole CTA, before any barrier/TMEM use
  const GridDev& G = grids[grid_id];
  const int mtile = blockIdx.x;
  const int n_m = G.n_m, n_z = G.n_z, n_t_pad = G.n_t_pad, nI = G.nI, nJ = G.nJ, nB = G.nB;
  const int n_m_pad = G.n_m_pad, ncp = G.n_cols_pad;
  if (mtile * kGemmRows >= n_m) return;

  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t SB = stage_bytes(ncp);
  float* a_s = reinterpret_cast<float*>(smem + vec_offset(ncp));
  float* b_s = a_s + kGemmRows;
  float* d_s = b_s + n_z;
  float* CN_s = d_s + n_t_pad;
  float* CG_s = CN_s + nJ * n_z;
  uint32_t ctl_off = vec_offset(ncp) + 4u * vec_floats(n_z, n_t_pad, nJ);
  ctl_off = (ctl_off + 15u) & ~15u;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + ctl_off);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + ctl_off + 16);
  int* abort_s = reinterpret_cast<int*>(smem + ctl_off + 20);

  // Zero both operand stages: padded rows/columns stay zero for the whole run.
  for (uint32_t i = tid * 16u; i < 2u * SB; i += 256u * 16u)
    *reinterpret_cast<uint4*>(smem + i) = make_uint4(0u, 0u, 0u, 0u);
  const float* sp = s32 + (size_t)p * G.s32_stride;
  for (int m = tid; m < kGemmRows; m += 256) {
    int row = mtile * kGemmRows + m;
    a_s[m] = row < n_m ? sp[G.f_a + row] : 0.f;
  }
  for (int q = tid; q < n_z; q += 256) b_s[q] = sp[G.f_b + q];
  for (int t = tid; t < n_t_pad; t += 256) d_s[t] = sp[G.f_delta + t];
  for (int u = tid; u < nJ * n_z; u += 256) {
    CN_s[u] = sp[G.f_CN + u];
    CG_s[u] = sp[G.f_CG + u];
  }
  const float c1 = sp[G.f_scal], c2 = sp[G.f_scal + 1];
  uint32_t ncols = 32;
  while ((int)ncols < ncp) ncols <<= 1;
  if (warp == 0) tmem_alloc(smem_u32(tmem_slot), ncols);
  if (tid == 0) {
    mbar_init(smem_u32(&mbar[0]), 1);
    mbar_init(smem_u32(&mbar[1]), 1);
    *abort_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int nk = n_t_pad / kKChunk;
  const float* UK = G.UK;
  const uint32_t lboA = (uint32_t)ncp * 16u;
  int last_committed = -1;
  for (int kc = 0; kc < nk; ++kc) {
    const int s = kc & 1;
    uint8_t* st = smem + s * SB;
    uint8_t* Fhi = st;
    uint8_t* Flo = st + kGemmRows * kKChunk * 2;
    uint8_t* Ahi = st + 2 * kGemmRows * kKChunk * 2;
    uint8_t* Alo = Ahi + ncp * kKChunk * 2;
    if (kc >= 2) {
      if (!mbar_wait_bounded(smem_u32(&mbar[s]), ((kc - 2) >> 1) & 1, kWaitBudget))
        atomicExch(abort_s, 1);
    }
    __syncthreads();
    if (*abort_s) break;
    // F operand: 128 lnM rows x 32 lam_t, [kgroup][row][8].
    for (int item = tid; item < kGemmRows * 4; item += 256) {
      const int m = item & (kGemmRows - 1), g = item >> 7;
      const int t0 = kc * kKChunk + g * 8;
      const bool valid = mtile * kGemmRows + m < n_m;
      const float am = a_s[m];
      float v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        float d = d_s[t0 + u] - am;
        v[u] = valid ? exp2f(-d * d * c1) : 0.f;
      }
      store_split8(Fhi + g * (kGemmRows * 16) + m * 16, Flo + g * (kGemmRows * 16) + m * 16, v);
    }
    // A operand: (i, q) columns x 32 lam_t; G(t,q) is shared by the nI rows.
    for (int item = tid; item < n_z * 4; item += 256) {
      const int q = item % n_z, g = item / n_z;
      const int t0 = kc * kKChunk + g * 8;
      const float bq = b_s[q];
      float gq[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) gq[u] = exp2f(d_s[t0 + u] * bq * c2);
      for (int i = 0; i < nI; ++i) {
        const float4* uk =
          reinterpret_cast<const float4*>(UK + ((size_t)(i * n_z + q)) * n_t_pad + t0);
        const float4 u0 = __ldg(uk), u1 = __ldg(uk + 1);
        float v[8] = {u0.x * gq[0], u0.y * gq[1], u0.z * gq[2], u0.w * gq[3],
                      u1.x * gq[4], u1.y * gq[5], u1.z * gq[6], u1.w * gq[7]};
        const int row = i * n_z + q;
        store_split8(Ahi + g * lboA + row * 16, Alo + g * lboA + row * 16, v);
      }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < kKChunk / 16; ++ks) {
        const uint32_t fh = smem_u32(Fhi) + (2 * ks) * (kGemmRows * 16);
        const uint32_t fl = smem_u32(Flo) + (2 * ks) * (kGemmRows * 16);
        const uint64_t ah = umma_desc(fh, kGemmRows * 16, 128);
        const uint64_t al = umma_desc(fl, kGemmRows * 16, 128);
        for (int c = 0; c * 256 < ncp; ++c) {
          const int nc = min(256, ncp - c * 256);
          const uint32_t idesc = umma_idesc_bf16(kGemmRows, nc);
          const uint32_t boff = (2 * ks) * lboA + c * 256 * 16;
          const uint64_t bh = umma_desc(smem_u32(Ahi) + boff, lboA, 128);
          const uint64_t bl = umma_desc(smem_u32(Alo) + boff, lboA, 128);
          const uint32_t d = tmem + (uint32_t)(c * 256);
          umma_bf16(d, ah, bh, idesc, (kc | ks) != 0);
          umma_bf16(d, ah, bl, idesc, 1u);
          umma_bf16(d, al, bh, idesc, 1u);
        }
      }
      umma_commit(smem_u32(&mbar[s]));
    }
    last_committed = kc;
  }
  // Wait for the last committed chunk (covers every earlier MMA).
  if (last_committed >= 0) {
    if (!mbar_wait_bounded(smem_u32(&mbar[last_committed & 1]), (last_committed >> 1) & 1,
                           kWaitBudget))
      atomicExch(abort_s, 1);
  }
  __syncthreads();
  const bool aborted = *abort_s != 0;
  if (aborted && tid == 0) set_err(status, kDevTimeout);
  tc_fence_after();

  if (!aborted) {
    const int lq = warp & 3, half = warp >> 2;
    const int row = mtile * kGemmRows + lq * 32 + lane;
    const bool valid = row < n_m;
    const float* Yt = sp + G.f_Yt;
    const uint32_t lane_base = (uint32_t)(lq * 32) << 16;
    for (int i = half; i < nI; i += 2) {
      double accN[kMaxZBins], accG[kMaxZBins];
#pragma unroll
      for (int j = 0; j < kMaxZBins; ++j) accN[j] = accG[j] = 0.0;
      for (int qc = 0; qc < n_z; qc += 16) {
        float v[16];
        tmem_ld16(tmem + lane_base + (uint32_t)(i * n_z + qc), v);
        float pN[kMaxZBins], pG[kMaxZBins];
#pragma unroll
        for (int j = 0; j < kMaxZBins; ++j) pN[j] = pG[j] = 0.f;
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          const int q = qc + u;
          const float e = v[u] * (valid ? Yt[(size_t)q * n_m_pad + row] : 0.f);
#pragma unroll
          for (int j = 0; j < kMaxZBins; ++j) {
            if (j < nJ) {
              pN[j] = fmaf(CN_s[j * n_z + q], e, pN[j]);
              pG[j] = fmaf(CG_s[j * n_z + q], e, pG[j]);
            }
          }
        }
#pragma unroll
        for (int j = 0; j < kMaxZBins; ++j) {
          accN[j] += (double)pN[j];
          accG[j] += (double)pG[j];
        }
      }
      if (valid) {
        for (int j = 0; j < nJ; ++j) {
          const size_t o = ((size_t)p * nB + i + nI * j) * w_stride + row;
          Wout[o] = accN[j];
          Wgout[o] = accG[j];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, ncols);
  }
}

size_t
mixed_gemm_smem_bytes(int ncp, int n_z, int n_t_pad, int nJ)
{
  size_t b = vec_offset(ncp) + 4u * vec_floats(n_z, n_t_pad, nJ);
  b = (b + 15) & ~size_t(15);
  return b + 32;
}

int
launch_mixed_gemm(const MixedLaunch& L)
{
  const GridDev& g = *L.g_host;
  size_t smem = mixed_gemm_smem_bytes(g.n_cols_pad, g.n_z, g.n_t_pad, g.nJ);
  Y3B_CUDA(cudaFuncSetAttribute(mixed_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
  dim3 grid(g.n_m_pad / kGemmRows, L.n_points);
  mixed_gemm_kernel<<<grid, 256, smem, L.stream>>>(L.grids, L.pts, L.grid_id, L.s32, L.W, L.Wg,
                                                   L.w_stride, L.status);
  count_launch();
  return cuda_status(cudaGetLastError(), "mixed_gemm_kernel");
}

}  // namespace y3b
