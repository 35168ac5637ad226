// Prints the TMA box geometry of the y-column prefetches for every grid
// length the library dispatches (les_engine.cuh with_small) in FP32 and
// FP64: "<real bytes> <NS> <inverse|forward> <TC> <NB> <BR> <ok> <complex bytes>".
// Host code only; tests/test_tma_geometry.py checks the TMA's rules on it.
#include <cstdio>
#include "les_kernels.cuh"
using namespace les;
template <class T, int NS> void one() {
  constexpr int M = 3 * NS / 2;
  using C = ColCfg<M, T>;
  using BI = ColBox<T, NS, C::TC>;
  using BF = ColBox<T, M, C::TC>;
  printf("%d %d inverse %d %d %d %d %d\n", (int)sizeof(T), NS, C::TC, BI::NB, BI::BR, (int)BI::ok, (int)sizeof(cx<T>));
  printf("%d %d forward %d %d %d %d %d\n", (int)sizeof(T), NS, C::TC, BF::NB, BF::BR, (int)BF::ok, (int)sizeof(cx<T>));
}
template <class T> void all() {
  one<T, 16>(); one<T, 32>(); one<T, 64>(); one<T, 96>(); one<T, 128>();
  one<T, 192>(); one<T, 256>(); one<T, 384>(); one<T, 512>();
}
int main() {
  all<float>();
  all<double>();
  return 0;
}
