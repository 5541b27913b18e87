// Ascending sorting networks over a register array of unsigned keys.
#pragma once

#include <cstdint>

namespace fknn {

// Ascending sorting networks (comparator counts 1, 5, 19, 60,
// 185, 531 for 2..64 keys).  8 and 16 keys use published minimum-size
// networks; larger sizes sort both halves and join them with Batcher's
// odd-even merge.  Each network was checked with the 0-1 principle (all
// 2^n binary inputs for n <= 16, all pairs of sorted binary halves for the
// merges).
template <int KCAP, typename T>
__device__ __forceinline__ void cas_up(T (&L)[KCAP], int i, int j) {
  const T a = L[i], b = L[j];
  const bool sw = b < a;
  L[i] = sw ? b : a;
  L[j] = sw ? a : b;
}

template <int KCAP, int LO, int N, int R, typename T>
__device__ __forceinline__ void odd_even_merge(T (&L)[KCAP]) {
  constexpr int M = R * 2;
  if constexpr (M < N) {
    odd_even_merge<KCAP, LO, N, M>(L);
    odd_even_merge<KCAP, LO + R, N, M>(L);
#pragma unroll
    for (int i = LO + R; i + R < LO + N; i += M) cas_up<KCAP>(L, i, i + R);
  } else {
    cas_up<KCAP>(L, LO, LO + R);
  }
}

template <int KCAP, int OFF, int N, typename T>
__device__ __forceinline__ void sort_network(T (&L)[KCAP]) {
  if constexpr (N == 2) {
    cas_up<KCAP>(L, OFF, OFF + 1);
  } else if constexpr (N == 4) {
    constexpr int net[5][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}, {1, 2}};
#pragma unroll
    for (int c = 0; c < 5; ++c) cas_up<KCAP>(L, OFF + net[c][0], OFF + net[c][1]);
  } else if constexpr (N == 8) {
    constexpr int net[19][2] = {{0, 2}, {1, 3}, {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6},
                                {3, 7}, {0, 1}, {2, 3}, {4, 5}, {6, 7}, {2, 4}, {3, 5},
                                {1, 4}, {3, 6}, {1, 2}, {3, 4}, {5, 6}};
#pragma unroll
    for (int c = 0; c < 19; ++c) cas_up<KCAP>(L, OFF + net[c][0], OFF + net[c][1]);
  } else if constexpr (N == 16) {
    constexpr int net[60][2] = {
        {0, 13}, {1, 12}, {2, 15}, {3, 14}, {4, 8},  {5, 6},   {7, 11},  {9, 10},  {0, 5},
        {1, 7},  {2, 9},  {3, 4},  {6, 13}, {8, 14}, {10, 15}, {11, 12}, {0, 1},   {2, 3},
        {4, 5},  {6, 8},  {7, 9},  {10, 11}, {12, 13}, {14, 15}, {0, 2},  {1, 3},   {4, 10},
        {5, 11}, {6, 7},  {8, 9},  {12, 14}, {13, 15}, {1, 2},  {3, 12},  {4, 6},   {5, 7},
        {8, 10}, {9, 11}, {13, 14}, {1, 4}, {2, 6},   {5, 8},   {7, 10},  {9, 13},  {11, 14},
        {2, 4},  {3, 6},  {9, 12}, {11, 13}, {3, 5},  {6, 8},   {7, 9},   {10, 12}, {3, 4},
        {5, 6},  {7, 8},  {9, 10}, {11, 12}, {6, 7},  {8, 9}};
#pragma unroll
    for (int c = 0; c < 60; ++c) cas_up<KCAP>(L, OFF + net[c][0], OFF + net[c][1]);
  } else if constexpr (N > 16) {
    sort_network<KCAP, OFF, N / 2>(L);
    sort_network<KCAP, OFF + N / 2, N / 2>(L);
    odd_even_merge<KCAP, OFF, N, 1>(L);
  }
}

}  // namespace fknn
