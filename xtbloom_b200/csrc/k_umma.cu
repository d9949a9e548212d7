// Split-precision (3xTF32) product tiles on the fifth-generation tensor
// cores: tcgen05.mma with the accumulator in tensor memory.
//
// The split form multiplies FP64 operands as a_hi b_hi + a_hi b_lo + a_lo b_hi
// with TF32 parts (hi = TF32(a), lo = TF32(a - hi)) and FP32 accumulation, which
// carries about 22 bits of each product.  One CTA forms one 64 x 64 tile of
// C = op(A) diag(w) B of one system (the same tiling, symmetric mirroring and
// per-system precision selection as k_gemm): its 256 threads load a 32-deep
// K chunk of FP64 operands, split them and store the parts in shared memory
// in the canonical K-major layout of the tensor-core descriptors; one thread
// issues 3 x 4 MMAs (M = 128 with the tile's 64 rows in the upper half, N =
// 64, K = 8) accumulating in a 64-column TMEM allocation and commits them to
// an mbarrier; the chunk's completion releases the shared buffers.  After
// the last chunk the accumulator is read back with tcgen05.ld (warps 0, 1, 4,
// 5: rows 0-63, two column halves) and stored in FP64.
//
// Layouts (matching the sm_100 descriptor definitions of CUTLASS,
// cute/arch/mma_sm100_desc.hpp):
//  * operand tiles (A: 128 rows, B: 64 rows, both K-major, 32 K-values of
//    4 bytes): core matrices of 8 rows x 16 bytes; core matrix (row group g,
//    K quad c) at byte (8 g + c) * 128; leading-byte offset (between the two
//    K quads of one MMA) 128 B, stride-byte offset (between row groups) 1024 B;
//    no swizzle; descriptor version 1;
//  * instruction descriptor: D F32, A and B TF32, both K-major, N >> 3, M >> 4.
//
// Every wait on the mbarrier is bounded; a wait that runs out sets the
// caller's fault flag, waits once more (bounded) for the MMAs in flight and
// frees the tensor memory before the CTA returns.  The TMEM need is 64
// columns per CTA; shared memory (48 KB per CTA) admits at most four CTAs
// per SM, 256 of the SM's 512 columns, so an allocation never waits.
#include "kernels.cuh"

namespace xtb {
namespace {

constexpr int UM = 128, UN = 64, UKC = 32;   // MMA rows, tile columns, K chunk
constexpr int kTileM = 64;                   // output rows per tile (upper half of UM)
constexpr uint32_t kTmemCols = 64;
constexpr uint32_t kIdesc = (1u << 4)                          // D: F32
                            | (2u << 7) | (2u << 10)            // A, B: TF32
                            | ((uint32_t)(UN >> 3) << 17)       // N >> 3
                            | ((uint32_t)(UM >> 4) << 24);      // M >> 4

// 32-bit word offset of element (row r, k) in a K-major operand tile
__device__ __forceinline__ uint32_t kmajor(int r, int k) {
  return ((((r >> 3) * (UKC / 4) + (k >> 2)) * 128) >> 2) + (r & 7) * 4 + (k & 3);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  const uint64_t lbo = 128 >> 4, sbo = ((UKC / 4) * 128) >> 4;
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void split_tf32_parts(double x, uint32_t& hi, uint32_t& lo) {
  const float f = (float)x;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(f));
  const float r = (float)(x - (double)__uint_as_float(hi));
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem), "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

// Bounded wait for the completion of the given phase of an mbarrier.
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
  for (int i = 0; i < (1 << 22); ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace

template <bool TA, bool W>
__global__ void __launch_bounds__(256) k_gemm_umma(GemmArgs g) {
  extern __shared__ __align__(128) uint32_t usm[];
  uint32_t* Ah = usm;                 // UM x UKC
  uint32_t* Al = Ah + UM * UKC;
  uint32_t* Bh = Al + UM * UKC;       // UN x UKC
  uint32_t* Bl = Bh + UN * UKC;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const int s = g.list[blockIdx.y];
  if (g.only != nullptr && g.only[s] == 0) return;
  if (g.prec[g.prec_of != nullptr ? g.prec_of[s] : s] != 0) return;   // FP64 systems: k_gemm
  const int M = g.dm[s], N = g.dn[s], K = g.dk[s];
  const int ld = g.nao[s];
  const int tm = (M + kTileM - 1) / kTileM, tn = (N + UN - 1) / UN;
  int ti, tj;
  if (g.sym) {
    const int t = blockIdx.x;
    if (t >= tm * (tm + 1) / 2) return;
    ti = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
    while (ti * (ti + 1) / 2 > t) --ti;
    tj = t - ti * (ti + 1) / 2;
  } else {
    if ((int)blockIdx.x >= tm * tn) return;
    ti = blockIdx.x / tn;
    tj = blockIdx.x % tn;
  }
  const bool mirror = g.sym && ti != tj;
  const double* A = g.A + g.offA[s];
  const double* B = g.B + g.offB[s];
  double* C = g.C + g.offC[s];
  const double* w = W ? g.w + g.offW[s] : nullptr;
  const int i0 = ti * kTileM, j0 = tj * UN;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // rows 64..127 of the A operand stay zero
  for (int e = tid; e < (UM - kTileM) * UKC; e += 256) {
    const int r = kTileM + e / UKC, k = e % UKC;
    Ah[kmajor(r, k)] = 0u;
    Al[kmajor(r, k)] = 0u;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&tmem_slot)), "r"(kTmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t bar = smem_u32(&mbar);
  uint32_t phase = 0;
  bool late = false;
  for (int k0 = 0; k0 < K; k0 += UKC) {
    // stage the chunk: 64 x 32 of op(A) and 32 x 64 of diag(w) B, split
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + q * 256;   // 0..2047
      int ii, kk;
      double av;
      if (TA) {
        kk = e / kTileM;
        ii = e % kTileM;
        const int gk = k0 + kk, gi = i0 + ii;
        av = (gk < K && gi < M) ? A[(int64_t)gk * ld + gi] : 0.0;
      } else {
        ii = e / UKC;
        kk = e % UKC;
        const int gk = k0 + kk, gi = i0 + ii;
        av = (gk < K && gi < M) ? A[(int64_t)gi * ld + gk] : 0.0;
      }
      uint32_t hi, lo;
      split_tf32_parts(av, hi, lo);
      Ah[kmajor(ii, kk)] = hi;
      Al[kmajor(ii, kk)] = lo;
      const int kb = e / UN, jj = e % UN;
      const int gk = k0 + kb, gj = j0 + jj;
      double bv = (gk < K && gj < N) ? B[(int64_t)gk * ld + gj] : 0.0;
      if (W && gk < K) bv *= w[gk];
      split_tf32_parts(bv, hi, lo);
      Bh[kmajor(jj, kb)] = hi;
      Bl[kmajor(jj, kb)] = lo;
    }
    // the generic-proxy stores must be visible to the tensor core's reads
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int ks = 0; ks < UKC / 8; ++ks) {
        const uint32_t off = ks * 2 * 128;   // two K quads per MMA
        const uint64_t ah = smem_desc(smem_u32(Ah) + off), al = smem_desc(smem_u32(Al) + off);
        const uint64_t bh = smem_desc(smem_u32(Bh) + off), bl = smem_desc(smem_u32(Bl) + off);
        umma_tf32(tmem, al, bh, (k0 > 0 || ks > 0) ? 1u : 0u);
        umma_tf32(tmem, ah, bl, 1u);
        umma_tf32(tmem, ah, bh, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   ::"r"(bar) : "memory");
    }
    // the chunk's MMAs are complete before its buffers are rewritten
    if (!mbar_wait(bar, phase)) late = true;
    phase ^= 1u;
    late = __syncthreads_or(late);
    if (late) break;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (late) {
    if (tid == 0 && g.fault != nullptr) atomicExch(g.fault, 1);
    mbar_wait(bar, phase ^ 1u);   // once more for the MMAs in flight (bounded)
  } else {
    const int quarter = warp & 3;
    if (quarter < 2) {
      const int row = quarter * 32 + lane;
      const int col0 = (warp >> 2) * 32;
      uint32_t v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = 0u;   // an empty contraction gives zeros
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)col0;
      if (K > 0) {
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
          "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
            "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
            "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
            "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(taddr)
          : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      }
      const int gi = i0 + row;
      if (gi < M) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int gj = j0 + col0 + j;
          if (gj < N) {
            const double x = (double)__uint_as_float(v[j]);
            C[(int64_t)gi * ld + gj] = x;
            if (mirror) C[(int64_t)gj * ld + gi] = x;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
}

size_t gemm_umma_bytes() { return (size_t)(2 * UM * UKC + 2 * UN * UKC) * sizeof(uint32_t); }

// Launch over the split-precision systems of the list (the others return at
// once); the grid covers the 64 x 64 tiles of the largest system (lower ones
// when symmetric).
void launch_gemm_umma(const GemmArgs& g, bool transA, bool weighted, int tm, int count,
                      cudaStream_t stream) {
  if (count == 0 || g.prec == nullptr) return;
  const int tiles = g.sym ? tm * (tm + 1) / 2 : tm * tm;
  const dim3 grid(tiles, count);
  const size_t bytes = gemm_umma_bytes();
  if (transA && weighted) {
    allow_max_dynamic_smem(k_gemm_umma<true, true>);
    k_gemm_umma<true, true><<<grid, 256, bytes, stream>>>(g);
  } else if (transA) {
    allow_max_dynamic_smem(k_gemm_umma<true, false>);
    k_gemm_umma<true, false><<<grid, 256, bytes, stream>>>(g);
  } else if (weighted) {
    allow_max_dynamic_smem(k_gemm_umma<false, true>);
    k_gemm_umma<false, true><<<grid, 256, bytes, stream>>>(g);
  } else {
    allow_max_dynamic_smem(k_gemm_umma<false, false>);
    k_gemm_umma<false, false><<<grid, 256, bytes, stream>>>(g);
  }
}

}  // namespace xtb
