// Host build of the library's software binary64 operations, for the CPU tests that compare them
// with the machine's IEEE-754 doubles (test infrastructure; compiled by tests/test_softf64.py).
#include <cstdint>

#include "softf64.cuh"

using namespace bvhc::sf;

extern "C" void sf_eval(int op, const uint64_t* a, const uint64_t* b, uint64_t* out, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    switch (op) {
      case 0: out[i] = add(a[i], b[i]); break;
      case 1: out[i] = sub(a[i], b[i]); break;
      case 2: out[i] = mul(a[i], b[i]); break;
      case 3: out[i] = div(a[i], b[i]); break;
      case 4: out[i] = sqrt(a[i]); break;
      case 5: out[i] = (uint64_t)lt(a[i], b[i]) | ((uint64_t)le(a[i], b[i]) << 1) | ((uint64_t)eq(a[i], b[i]) << 2); break;
      case 6: out[i] = f32_bits(to_f32(a[i])); break;
      case 7: out[i] = from_f32(f32_from_bits((uint32_t)a[i])); break;
      case 8: out[i] = from_u64(a[i]); break;
      case 9: out[i] = (uint64_t)(int64_t)to_i32_trunc(a[i]); break;
      default: out[i] = 0;
    }
  }
}
