// addchain.cuh -- multi-limb adds on the PTX carry flag (generated, do not edit).
// add_chain_cN: s[0..N) = a[0..N) + b[0..N) + cin (cin in {0,1}); returns the carry out.
#pragma once
#include <stdint.h>

namespace kira {

__device__ __forceinline__ uint32_t add_chain_c1(const uint32_t* a, const uint32_t* b,
                                                 uint32_t cin, uint32_t* s) {
  uint32_t cout;
  asm("{\n\t.reg .u32 t;\n\t"
      "add.cc.u32 t, %4, -1;\n\t"
      "addc.cc.u32 %0, %2, %3;\n\t"
      "addc.u32 %1, 0, 0;\n\t}"
      : "=&r"(s[0]), "=&r"(cout)
      : "r"(a[0]), "r"(b[0]), "r"(cin));
  return cout;
}

__device__ __forceinline__ uint32_t add_chain_c2(const uint32_t* a, const uint32_t* b,
                                                 uint32_t cin, uint32_t* s) {
  uint32_t cout;
  asm("{\n\t.reg .u32 t;\n\t"
      "add.cc.u32 t, %7, -1;\n\t"
      "addc.cc.u32 %0, %3, %4;\n\t"
      "addc.cc.u32 %1, %5, %6;\n\t"
      "addc.u32 %2, 0, 0;\n\t}"
      : "=&r"(s[0]), "=&r"(s[1]), "=&r"(cout)
      : "r"(a[0]), "r"(b[0]), "r"(a[1]), "r"(b[1]), "r"(cin));
  return cout;
}

__device__ __forceinline__ uint32_t add_chain_c3(const uint32_t* a, const uint32_t* b,
                                                 uint32_t cin, uint32_t* s) {
  uint32_t cout;
  asm("{\n\t.reg .u32 t;\n\t"
      "add.cc.u32 t, %10, -1;\n\t"
      "addc.cc.u32 %0, %4, %5;\n\t"
      "addc.cc.u32 %1, %6, %7;\n\t"
      "addc.cc.u32 %2, %8, %9;\n\t"
      "addc.u32 %3, 0, 0;\n\t}"
      : "=&r"(s[0]), "=&r"(s[1]), "=&r"(s[2]), "=&r"(cout)
      : "r"(a[0]), "r"(b[0]), "r"(a[1]), "r"(b[1]), "r"(a[2]), "r"(b[2]), "r"(cin));
  return cout;
}

__device__ __forceinline__ uint32_t add_chain_c4(const uint32_t* a, const uint32_t* b,
                                                 uint32_t cin, uint32_t* s) {
  uint32_t cout;
  asm("{\n\t.reg .u32 t;\n\t"
      "add.cc.u32 t, %13, -1;\n\t"
      "addc.cc.u32 %0, %5, %6;\n\t"
      "addc.cc.u32 %1, %7, %8;\n\t"
      "addc.cc.u32 %2, %9, %10;\n\t"
      "addc.cc.u32 %3, %11, %12;\n\t"
      "addc.u32 %4, 0, 0;\n\t}"
      : "=&r"(s[0]), "=&r"(s[1]), "=&r"(s[2]), "=&r"(s[3]), "=&r"(cout)
      : "r"(a[0]), "r"(b[0]), "r"(a[1]), "r"(b[1]), "r"(a[2]), "r"(b[2]), "r"(a[3]), "r"(b[3]), "r"(cin));
  return cout;
}

__device__ __forceinline__ uint32_t add_chain_c5(const uint32_t* a, const uint32_t* b,
                                                 uint32_t cin, uint32_t* s) {
  uint32_t cout;
  asm("{\n\t.reg .u32 t;\n\t"
      "add.cc.u32 t, %16, -1;\n\t"
      "addc.cc.u32 %0, %6, %7;\n\t"
      "addc.cc.u32 %1, %8, %9;\n\t"
      "addc.cc.u32 %2, %10, %11;\n\t"
      "addc.cc.u32 %3, %12, %13;\n\t"
      "addc.cc.u32 %4, %14, %15;\n\t"
      "addc.u32 %5, 0, 0;\n\t}"
      : "=&r"(s[0]), "=&r"(s[1]), "=&r"(s[2]), "=&r"(s[3]), "=&r"(s[4]), "=&r"(cout)
      : "r"(a[0]), "r"(b[0]), "r"(a[1]), "r"(b[1]), "r"(a[2]), "r"(b[2]), "r"(a[3]), "r"(b[3]), "r"(a[4]), "r"(b[4]), "r"(cin));
  return cout;
}

__device__ __forceinline__ uint32_t add_chain_c6(const uint32_t* a, const uint32_t* b,
                                                 uint32_t cin, uint32_t* s) {
  uint32_t cout;
  asm("{\n\t.reg .u32 t;\n\t"
      "add.cc.u32 t, %19, -1;\n\t"
      "addc.cc.u32 %0, %7, %8;\n\t"
      "addc.cc.u32 %1, %9, %10;\n\t"
      "addc.cc.u32 %2, %11, %12;\n\t"
      "addc.cc.u32 %3, %13, %14;\n\t"
      "addc.cc.u32 %4, %15, %16;\n\t"
      "addc.cc.u32 %5, %17, %18;\n\t"
      "addc.u32 %6, 0, 0;\n\t}"
      : "=&r"(s[0]), "=&r"(s[1]), "=&r"(s[2]), "=&r"(s[3]), "=&r"(s[4]), "=&r"(s[5]), "=&r"(cout)
      : "r"(a[0]), "r"(b[0]), "r"(a[1]), "r"(b[1]), "r"(a[2]), "r"(b[2]), "r"(a[3]), "r"(b[3]), "r"(a[4]), "r"(b[4]), "r"(a[5]), "r"(b[5]), "r"(cin));
  return cout;
}

__device__ __forceinline__ uint32_t add_chain_c7(const uint32_t* a, const uint32_t* b,
                                                 uint32_t cin, uint32_t* s) {
  uint32_t cout;
  asm("{\n\t.reg .u32 t;\n\t"
      "add.cc.u32 t, %22, -1;\n\t"
      "addc.cc.u32 %0, %8, %9;\n\t"
      "addc.cc.u32 %1, %10, %11;\n\t"
      "addc.cc.u32 %2, %12, %13;\n\t"
      "addc.cc.u32 %3, %14, %15;\n\t"
      "addc.cc.u32 %4, %16, %17;\n\t"
      "addc.cc.u32 %5, %18, %19;\n\t"
      "addc.cc.u32 %6, %20, %21;\n\t"
      "addc.u32 %7, 0, 0;\n\t}"
      : "=&r"(s[0]), "=&r"(s[1]), "=&r"(s[2]), "=&r"(s[3]), "=&r"(s[4]), "=&r"(s[5]), "=&r"(s[6]), "=&r"(cout)
      : "r"(a[0]), "r"(b[0]), "r"(a[1]), "r"(b[1]), "r"(a[2]), "r"(b[2]), "r"(a[3]), "r"(b[3]), "r"(a[4]), "r"(b[4]), "r"(a[5]), "r"(b[5]), "r"(a[6]), "r"(b[6]), "r"(cin));
  return cout;
}

__device__ __forceinline__ uint32_t add_chain_c8(const uint32_t* a, const uint32_t* b,
                                                 uint32_t cin, uint32_t* s) {
  uint32_t cout;
  asm("{\n\t.reg .u32 t;\n\t"
      "add.cc.u32 t, %25, -1;\n\t"
      "addc.cc.u32 %0, %9, %10;\n\t"
      "addc.cc.u32 %1, %11, %12;\n\t"
      "addc.cc.u32 %2, %13, %14;\n\t"
      "addc.cc.u32 %3, %15, %16;\n\t"
      "addc.cc.u32 %4, %17, %18;\n\t"
      "addc.cc.u32 %5, %19, %20;\n\t"
      "addc.cc.u32 %6, %21, %22;\n\t"
      "addc.cc.u32 %7, %23, %24;\n\t"
      "addc.u32 %8, 0, 0;\n\t}"
      : "=&r"(s[0]), "=&r"(s[1]), "=&r"(s[2]), "=&r"(s[3]), "=&r"(s[4]), "=&r"(s[5]), "=&r"(s[6]), "=&r"(s[7]), "=&r"(cout)
      : "r"(a[0]), "r"(b[0]), "r"(a[1]), "r"(b[1]), "r"(a[2]), "r"(b[2]), "r"(a[3]), "r"(b[3]), "r"(a[4]), "r"(b[4]), "r"(a[5]), "r"(b[5]), "r"(a[6]), "r"(b[6]), "r"(a[7]), "r"(b[7]), "r"(cin));
  return cout;
}

// s = a + b over L limbs (carry out of the top limb dropped).
template <int L>
__device__ __forceinline__ void add_chain(const uint32_t (&a)[L], const uint32_t (&b)[L],
                                         uint32_t (&s)[L]) {
  uint32_t c = 0;
#pragma unroll
  for (int k0 = 0; k0 < L; k0 += 8) {
    constexpr int kMax = 8;
    const int n = (L - k0) < kMax ? (L - k0) : kMax;
    switch (n) {
      case 1: c = add_chain_c1(a + k0, b + k0, c, s + k0); break;
      case 2: c = add_chain_c2(a + k0, b + k0, c, s + k0); break;
      case 3: c = add_chain_c3(a + k0, b + k0, c, s + k0); break;
      case 4: c = add_chain_c4(a + k0, b + k0, c, s + k0); break;
      case 5: c = add_chain_c5(a + k0, b + k0, c, s + k0); break;
      case 6: c = add_chain_c6(a + k0, b + k0, c, s + k0); break;
      case 7: c = add_chain_c7(a + k0, b + k0, c, s + k0); break;
      case 8: c = add_chain_c8(a + k0, b + k0, c, s + k0); break;
      default: break;
    }
  }
}

}  // namespace kira
