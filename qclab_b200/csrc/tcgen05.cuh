// Thin wrappers over the sm_100a tensor-core instructions (tcgen05.*) and
// mbarriers used by the tensor-memory sweep kernel.
//
// Layouts (PTX ISA, tcgen05 "matrix descriptors" and "instruction
// descriptor"):
//  * shared-memory matrix descriptor, K-major, no swizzle: 8-row x 16-byte
//    core matrices; bits [0,14) start address >> 4, [16,30) leading byte
//    offset >> 4 (stride between core matrices along K), [32,46) stride byte
//    offset >> 4 (stride between 8-row groups along M/N), bits [46,48) = 1
//    (descriptor version), layout type (bits [61,64)) 0 = no swizzle;
//  * instruction descriptor: [4,6) D format (1 = f32), [7,10) A format,
//    [10,13) B format (2 = tf32 for kind::tf32), bit 15/16 A/B major
//    (0 = K-major), [17,23) N >> 3, [24,29) M >> 4;
//  * tensor memory address: lane in bits [16,32), column in [0,16); a warp
//    reaches lanes 32 (warp % 4) .. + 31 with tcgen05.ld / tcgen05.st.
// kind::tf32 reads the top 19 bits of each 32-bit operand (the low 13
// mantissa bits are truncated), so callers split operands into exact tf32
// values first.
#pragma once

#include <cstdint>

namespace qsv {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint64_t sdesc_kmajor(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// D[tmem d] (+)= A[tmem a] * B[smem desc], one CTA, kind::tf32
__device__ __forceinline__ void mma_tf32_ts(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      ::"r"(d), "r"(a), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// Arrives on the mbarrier once every tcgen05 operation this thread issued
// before has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void bar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the phase with the given parity to complete: at most `limit`
// suspended polls of up to `hint_ns` each; gives up early when *abort is
// non-zero.  Returns false when the wait did not end with the phase
// completed.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, const volatile int* abort,
                                         int limit, uint32_t hint_ns = 1000000u) {
  const uint32_t a = smem_addr(bar);
  for (int it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(a), "r"(parity), "r"(hint_ns) : "memory");
    if (ok) return true;
    if (*abort) return false;
  }
  return false;
}

__device__ __forceinline__ void bar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void alloc(uint32_t* slot, uint32_t ncols) {  // one full warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               ::"r"(smem_addr(slot)), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t ncols) {  // the same warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes -> later reads by the tensor core
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void st_32x32b_x16(uint32_t taddr, const uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16};"
      ::"r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
        "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]),
        "r"(v[14]), "r"(v[15])
      : "memory");
}
__device__ __forceinline__ void wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void ld_32x32b_x32(uint32_t taddr, float (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]),
        "=f"(v[7]), "=f"(v[8]), "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]),
        "=f"(v[14]), "=f"(v[15]), "=f"(v[16]), "=f"(v[17]), "=f"(v[18]), "=f"(v[19]),
        "=f"(v[20]), "=f"(v[21]), "=f"(v[22]), "=f"(v[23]), "=f"(v[24]), "=f"(v[25]),
        "=f"(v[26]), "=f"(v[27]), "=f"(v[28]), "=f"(v[29]), "=f"(v[30]), "=f"(v[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// fp32 -> tf32 bit patterns with integer operations (finite inputs):
// truncation (what kind::tf32 itself does to a 32-bit operand), round to
// nearest with ties away from zero (half a tf32 unit added to the magnitude
// bits) and round to nearest with ties to even.
__device__ __forceinline__ uint32_t tf32_trunc(float x) { return __float_as_uint(x) & 0xffffe000u; }
__device__ __forceinline__ uint32_t tf32_round(float x) {
  return (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
}
__device__ __forceinline__ uint32_t tf32_round_even(float x) {
  const uint32_t u = __float_as_uint(x);
  return (u + 0xfffu + ((u >> 13) & 1u)) & 0xffffe000u;
}
// x = hi + lo with hi = tf32_trunc(x) (x - hi is exact in fp32) and lo that
// remainder rounded to tf32 (ties to even: the remainder has at most 13
// significant bits, so ties are frequent and ties away from zero would bias
// the sum): |x - hi - lo| <= 2^-21 |x|, mean error zero.
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
  hi = tf32_trunc(x);
  lo = tf32_round_even(x - __uint_as_float(hi));
}

}  // namespace tc
}  // namespace qsv
