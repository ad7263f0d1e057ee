// Host-side check of the product's field arithmetic (whirlaway_b200/csrc/kb.cuh and
// poseidon2.cuh compile for the host too): Montgomery products, lazy reductions, the
// unsigned-min additions and the shortcut multiplications of the Poseidon2 internal layer,
// each against a plain modular reference. Built and run by tests/test_boundary.py.
#include <cstdio>
#include <random>
#include "poseidon2.cuh"
using namespace kb;
int main() {
  std::mt19937_64 g(1);
  long b1=0,b2=0,b3=0,b4=0,b5=0,b6=0;
  for (int it = 0; it < 100000; it++) {
    uint32_t x = g() % P, y = g() % P;
    if (add(x, y) != (uint32_t)(((uint64_t)x + y) % P)) b1++;
    if (sub(x, y) != (uint32_t)(((uint64_t)x + P - y) % P)) b2++;
    uint32_t xm = to_mont(x), ym = to_mont(y);
    if (from_mont(mul(xm, ym)) != (uint32_t)((uint64_t)x * y % P)) b3++;
    for (int i = 0; i < 16; i++) if (p2_diag_mul<16>(i, xm) != mul(xm, p2_diag<16>(i))) { if(b4<5) printf("w16 i=%d x=%u got %u want %u\n", i, xm, p2_diag_mul<16>(i, xm), mul(xm, p2_diag<16>(i))); b4++; }
    if (halve(xm) != mul(xm, inv_m(to_mont(2)))) b5++;
  }
  for (int it = 0; it < 100000; it++) {
    uint64_t acc = 0; uint32_t ref = 0;
    for (int k = 0; k < 4; k++) { uint32_t a = g() % P, b = g() % P; acc += wmul(a, b); ref = add(ref, mul(a, b)); }
    if (redc(acc) != ref) b6++;
  }
  for (int it = 0; it < 2000; it++) {
    uint32_t x = g() % P, xm = to_mont(x);
    for (int i = 0; i < 24; i++) if (p2_diag_mul<24>(i, xm) != mul(xm, p2_diag<24>(i))) b4++;
  }
  printf("add %ld sub %ld mul %ld diag %ld halve %ld redc %ld\n", b1,b2,b3,b4,b5,b6);
  return (b1 + b2 + b3 + b4 + b5 + b6) ? 1 : 0;
}
