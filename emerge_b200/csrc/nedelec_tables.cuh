// GENERATED by gen_tables.py -- do not edit.
// Closed-form Nedelec-2 (Volakis mixed) element integrals in the canonical
// (vertex-rank) frame: exact barycentric-monomial integrals divided by V.
#pragma once
namespace emg_tables {
// 1 for DoFs whose basis function carries the orientation sign (ne2, nf0, nf1)
__host__ __device__ constexpr int odd(int x) { return x >= 6 ? 1 : 0; }
template <int f, int s> struct Pair;
template <> struct Pair<0, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[0][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[0][0]); emg_mac(acc, -0.05, G[0][1]); emg_mac(acc, -0.05, G[1][0]); emg_mac(acc, 0.1, G[1][1]); }
};
template <> struct Pair<0, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[0][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][0]); emg_mac(acc, -0.05, G[0][2]); emg_mac(acc, -0.05, G[1][0]); emg_mac(acc, 0.1, G[1][2]); }
};
template <> struct Pair<0, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[0][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][0]); emg_mac(acc, -0.05, G[0][3]); emg_mac(acc, -0.05, G[1][0]); emg_mac(acc, 0.1, G[1][3]); }
};
template <> struct Pair<0, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[0][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][1]); emg_mac(acc, -0.1, G[0][2]); emg_mac(acc, -0.05, G[1][1]); emg_mac(acc, 0.05, G[1][2]); }
};
template <> struct Pair<0, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[0][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][1]); emg_mac(acc, -0.1, G[0][3]); emg_mac(acc, -0.05, G[1][1]); emg_mac(acc, 0.05, G[1][3]); }
};
template <> struct Pair<0, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][2]); emg_mac(acc, -0.05, G[0][3]); emg_mac(acc, -0.05, G[1][2]); emg_mac(acc, 0.05, G[1][3]); }
};
template <> struct Pair<0, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][0]); emg_mac(acc, 0.03333333333333333, G[1][1]); }
};
template <> struct Pair<0, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, 0.03333333333333333, G[1][2]); }
};
template <> struct Pair<0, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, 0.03333333333333333, G[1][3]); }
};
template <> struct Pair<0, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][2]); emg_mac(acc, 0.008333333333333333, G[1][1]); emg_mac(acc, 0.008333333333333333, G[1][2]); }
};
template <> struct Pair<0, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][3]); emg_mac(acc, 0.008333333333333333, G[1][1]); emg_mac(acc, 0.008333333333333333, G[1][3]); }
};
template <> struct Pair<0, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, 0.008333333333333333, G[1][2]); emg_mac(acc, 0.008333333333333333, G[1][3]); }
};
template <> struct Pair<0, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][0]); emg_mac(acc, 0.5, H[0][1]); emg_mac(acc, 1.0, H[0][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][1]); emg_mac(acc, -0.016666666666666666, G[0][2]); emg_mac(acc, -0.016666666666666666, G[1][1]); emg_mac(acc, 0.016666666666666666, G[1][2]); }
};
template <> struct Pair<0, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][0]); emg_mac(acc, 0.5, H[0][2]); emg_mac(acc, 1.0, H[0][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][1]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.016666666666666666, G[1][1]); emg_mac(acc, 0.016666666666666666, G[1][3]); }
};
template <> struct Pair<0, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][1]); emg_mac(acc, 0.5, H[0][2]); emg_mac(acc, 1.0, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][2]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.016666666666666666, G[1][2]); emg_mac(acc, 0.016666666666666666, G[1][3]); }
};
template <> struct Pair<0, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][3]); emg_mac(acc, 0.5, H[0][4]); emg_mac(acc, 1.0, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][2]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, 0.008333333333333333, G[1][3]); }
};
template <> struct Pair<0, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][0]); emg_mac(acc, 1.0, H[0][1]); emg_mac(acc, 0.5, H[0][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.016666666666666666, G[0][2]); emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, 0.016666666666666666, G[1][2]); }
};
template <> struct Pair<0, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][0]); emg_mac(acc, 1.0, H[0][2]); emg_mac(acc, 0.5, H[0][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, 0.016666666666666666, G[1][3]); }
};
template <> struct Pair<0, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][1]); emg_mac(acc, 1.0, H[0][2]); emg_mac(acc, 0.5, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, 0.016666666666666666, G[1][3]); }
};
template <> struct Pair<0, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][3]); emg_mac(acc, 1.0, H[0][4]); emg_mac(acc, 0.5, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][1]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.008333333333333333, G[1][1]); emg_mac(acc, 0.008333333333333333, G[1][3]); }
};
template <> struct Pair<1, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[1][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][0]); emg_mac(acc, -0.05, G[0][1]); emg_mac(acc, -0.05, G[2][0]); emg_mac(acc, 0.1, G[2][1]); }
};
template <> struct Pair<1, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[1][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[0][0]); emg_mac(acc, -0.05, G[0][2]); emg_mac(acc, -0.05, G[2][0]); emg_mac(acc, 0.1, G[2][2]); }
};
template <> struct Pair<1, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[1][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][0]); emg_mac(acc, -0.05, G[0][3]); emg_mac(acc, -0.05, G[2][0]); emg_mac(acc, 0.1, G[2][3]); }
};
template <> struct Pair<1, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[1][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[0][1]); emg_mac(acc, -0.05, G[0][2]); emg_mac(acc, -0.05, G[2][1]); emg_mac(acc, 0.05, G[2][2]); }
};
template <> struct Pair<1, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][1]); emg_mac(acc, -0.05, G[0][3]); emg_mac(acc, -0.05, G[2][1]); emg_mac(acc, 0.05, G[2][3]); }
};
template <> struct Pair<1, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[1][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][2]); emg_mac(acc, -0.1, G[0][3]); emg_mac(acc, -0.05, G[2][2]); emg_mac(acc, 0.05, G[2][3]); }
};
template <> struct Pair<1, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, 0.03333333333333333, G[2][1]); }
};
template <> struct Pair<1, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][0]); emg_mac(acc, 0.03333333333333333, G[2][2]); }
};
template <> struct Pair<1, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, 0.03333333333333333, G[2][3]); }
};
template <> struct Pair<1, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][1]); emg_mac(acc, 0.008333333333333333, G[2][1]); emg_mac(acc, 0.008333333333333333, G[2][2]); }
};
template <> struct Pair<1, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, 0.008333333333333333, G[2][1]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<1, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][3]); emg_mac(acc, 0.008333333333333333, G[2][2]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<1, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[1][0]); emg_mac(acc, 0.5, H[1][1]); emg_mac(acc, 1.0, H[1][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][1]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, -0.016666666666666666, G[2][1]); emg_mac(acc, 0.016666666666666666, G[2][2]); }
};
template <> struct Pair<1, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[1][0]); emg_mac(acc, 0.5, H[1][2]); emg_mac(acc, 1.0, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][1]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.016666666666666666, G[2][1]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<1, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[1][1]); emg_mac(acc, 0.5, H[1][2]); emg_mac(acc, 1.0, H[1][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][2]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.016666666666666666, G[2][2]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<1, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[1][3]); emg_mac(acc, 0.5, H[1][4]); emg_mac(acc, 1.0, H[1][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][2]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.008333333333333333, G[2][2]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<1, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[1][0]); emg_mac(acc, 1.0, H[1][1]); emg_mac(acc, 0.5, H[1][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][2]); }
};
template <> struct Pair<1, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[1][0]); emg_mac(acc, 1.0, H[1][2]); emg_mac(acc, 0.5, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<1, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[1][1]); emg_mac(acc, 1.0, H[1][2]); emg_mac(acc, 0.5, H[1][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<1, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[1][3]); emg_mac(acc, 1.0, H[1][4]); emg_mac(acc, 0.5, H[1][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][1]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<2, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[2][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][0]); emg_mac(acc, -0.05, G[0][1]); emg_mac(acc, -0.05, G[3][0]); emg_mac(acc, 0.1, G[3][1]); }
};
template <> struct Pair<2, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[2][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][0]); emg_mac(acc, -0.05, G[0][2]); emg_mac(acc, -0.05, G[3][0]); emg_mac(acc, 0.1, G[3][2]); }
};
template <> struct Pair<2, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[2][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[0][0]); emg_mac(acc, -0.05, G[0][3]); emg_mac(acc, -0.05, G[3][0]); emg_mac(acc, 0.1, G[3][3]); }
};
template <> struct Pair<2, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[0][1]); emg_mac(acc, -0.05, G[0][2]); emg_mac(acc, -0.05, G[3][1]); emg_mac(acc, 0.05, G[3][2]); }
};
template <> struct Pair<2, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[2][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[0][1]); emg_mac(acc, -0.05, G[0][3]); emg_mac(acc, -0.05, G[3][1]); emg_mac(acc, 0.05, G[3][3]); }
};
template <> struct Pair<2, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[2][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[0][2]); emg_mac(acc, -0.05, G[0][3]); emg_mac(acc, -0.05, G[3][2]); emg_mac(acc, 0.05, G[3][3]); }
};
template <> struct Pair<2, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, 0.03333333333333333, G[3][1]); }
};
template <> struct Pair<2, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, 0.03333333333333333, G[3][2]); }
};
template <> struct Pair<2, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][0]); emg_mac(acc, 0.03333333333333333, G[3][3]); }
};
template <> struct Pair<2, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, 0.008333333333333333, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<2, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][1]); emg_mac(acc, 0.008333333333333333, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<2, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][2]); emg_mac(acc, 0.008333333333333333, G[3][2]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<2, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[2][0]); emg_mac(acc, 0.5, H[2][1]); emg_mac(acc, 1.0, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][1]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, -0.016666666666666666, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<2, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[2][0]); emg_mac(acc, 0.5, H[2][2]); emg_mac(acc, 1.0, H[2][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][1]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.016666666666666666, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<2, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[2][1]); emg_mac(acc, 0.5, H[2][2]); emg_mac(acc, 1.0, H[2][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][2]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.016666666666666666, G[3][2]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<2, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[2][3]); emg_mac(acc, 0.5, H[2][4]); emg_mac(acc, 1.0, H[2][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][2]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[3][2]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<2, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[2][0]); emg_mac(acc, 1.0, H[2][1]); emg_mac(acc, 0.5, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<2, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[2][0]); emg_mac(acc, 1.0, H[2][2]); emg_mac(acc, 0.5, H[2][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<2, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[2][1]); emg_mac(acc, 1.0, H[2][2]); emg_mac(acc, 0.5, H[2][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<2, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[2][3]); emg_mac(acc, 1.0, H[2][4]); emg_mac(acc, 0.5, H[2][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][1]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<3, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[3][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[1][0]); emg_mac(acc, -0.05, G[1][1]); emg_mac(acc, -0.1, G[2][0]); emg_mac(acc, 0.05, G[2][1]); }
};
template <> struct Pair<3, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[3][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[1][0]); emg_mac(acc, -0.05, G[1][2]); emg_mac(acc, -0.05, G[2][0]); emg_mac(acc, 0.05, G[2][2]); }
};
template <> struct Pair<3, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[1][0]); emg_mac(acc, -0.05, G[1][3]); emg_mac(acc, -0.05, G[2][0]); emg_mac(acc, 0.05, G[2][3]); }
};
template <> struct Pair<3, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[3][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[1][1]); emg_mac(acc, -0.05, G[1][2]); emg_mac(acc, -0.05, G[2][1]); emg_mac(acc, 0.1, G[2][2]); }
};
template <> struct Pair<3, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[3][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[1][1]); emg_mac(acc, -0.05, G[1][3]); emg_mac(acc, -0.05, G[2][1]); emg_mac(acc, 0.1, G[2][3]); }
};
template <> struct Pair<3, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[1][2]); emg_mac(acc, -0.1, G[1][3]); emg_mac(acc, -0.05, G[2][2]); emg_mac(acc, 0.05, G[2][3]); }
};
template <> struct Pair<3, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][1]); emg_mac(acc, 0.03333333333333333, G[2][0]); }
};
template <> struct Pair<3, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][0]); emg_mac(acc, 0.008333333333333333, G[2][0]); emg_mac(acc, 0.008333333333333333, G[2][2]); }
};
template <> struct Pair<3, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, 0.008333333333333333, G[2][0]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<3, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][1]); emg_mac(acc, 0.03333333333333333, G[2][2]); }
};
template <> struct Pair<3, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, 0.03333333333333333, G[2][3]); }
};
template <> struct Pair<3, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][3]); emg_mac(acc, 0.008333333333333333, G[2][2]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<3, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[3][0]); emg_mac(acc, 0.5, H[3][1]); emg_mac(acc, 1.0, H[3][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.016666666666666666, G[2][2]); }
};
template <> struct Pair<3, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[3][0]); emg_mac(acc, 0.5, H[3][2]); emg_mac(acc, 1.0, H[3][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<3, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[3][1]); emg_mac(acc, 0.5, H[3][2]); emg_mac(acc, 1.0, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][2]); emg_mac(acc, -0.016666666666666666, G[1][3]); emg_mac(acc, -0.008333333333333333, G[2][2]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<3, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[3][3]); emg_mac(acc, 0.5, H[3][4]); emg_mac(acc, 1.0, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][2]); emg_mac(acc, -0.016666666666666666, G[1][3]); emg_mac(acc, -0.016666666666666666, G[2][2]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<3, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[3][0]); emg_mac(acc, 1.0, H[3][1]); emg_mac(acc, 0.5, H[3][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, -0.016666666666666666, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][2]); }
};
template <> struct Pair<3, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[3][0]); emg_mac(acc, 1.0, H[3][2]); emg_mac(acc, 0.5, H[3][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.016666666666666666, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<3, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[3][1]); emg_mac(acc, 1.0, H[3][2]); emg_mac(acc, 0.5, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][0]); emg_mac(acc, -0.016666666666666666, G[1][3]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<3, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[3][3]); emg_mac(acc, 1.0, H[3][4]); emg_mac(acc, 0.5, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][1]); emg_mac(acc, -0.016666666666666666, G[1][3]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<4, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[4][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[1][0]); emg_mac(acc, -0.05, G[1][1]); emg_mac(acc, -0.1, G[3][0]); emg_mac(acc, 0.05, G[3][1]); }
};
template <> struct Pair<4, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[1][0]); emg_mac(acc, -0.05, G[1][2]); emg_mac(acc, -0.05, G[3][0]); emg_mac(acc, 0.05, G[3][2]); }
};
template <> struct Pair<4, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[4][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[1][0]); emg_mac(acc, -0.05, G[1][3]); emg_mac(acc, -0.05, G[3][0]); emg_mac(acc, 0.05, G[3][3]); }
};
template <> struct Pair<4, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[4][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[1][1]); emg_mac(acc, -0.05, G[1][2]); emg_mac(acc, -0.05, G[3][1]); emg_mac(acc, 0.1, G[3][2]); }
};
template <> struct Pair<4, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[4][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[1][1]); emg_mac(acc, -0.05, G[1][3]); emg_mac(acc, -0.05, G[3][1]); emg_mac(acc, 0.1, G[3][3]); }
};
template <> struct Pair<4, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[1][2]); emg_mac(acc, -0.05, G[1][3]); emg_mac(acc, -0.05, G[3][2]); emg_mac(acc, 0.05, G[3][3]); }
};
template <> struct Pair<4, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][1]); emg_mac(acc, 0.03333333333333333, G[3][0]); }
};
template <> struct Pair<4, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, 0.008333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<4, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][0]); emg_mac(acc, 0.008333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<4, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, 0.03333333333333333, G[3][2]); }
};
template <> struct Pair<4, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][1]); emg_mac(acc, 0.03333333333333333, G[3][3]); }
};
template <> struct Pair<4, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][2]); emg_mac(acc, 0.008333333333333333, G[3][2]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<4, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[4][0]); emg_mac(acc, 0.5, H[4][1]); emg_mac(acc, 1.0, H[4][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<4, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[4][0]); emg_mac(acc, 0.5, H[4][2]); emg_mac(acc, 1.0, H[4][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<4, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[4][1]); emg_mac(acc, 0.5, H[4][2]); emg_mac(acc, 1.0, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][2]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[3][2]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<4, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[4][3]); emg_mac(acc, 0.5, H[4][4]); emg_mac(acc, 1.0, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][2]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.016666666666666666, G[3][2]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<4, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[4][0]); emg_mac(acc, 1.0, H[4][1]); emg_mac(acc, 0.5, H[4][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<4, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[4][0]); emg_mac(acc, 1.0, H[4][2]); emg_mac(acc, 0.5, H[4][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<4, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[4][1]); emg_mac(acc, 1.0, H[4][2]); emg_mac(acc, 0.5, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<4, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[4][3]); emg_mac(acc, 1.0, H[4][4]); emg_mac(acc, 0.5, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<5, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[2][0]); emg_mac(acc, -0.05, G[2][1]); emg_mac(acc, -0.05, G[3][0]); emg_mac(acc, 0.05, G[3][1]); }
};
template <> struct Pair<5, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[5][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[2][0]); emg_mac(acc, -0.05, G[2][2]); emg_mac(acc, -0.1, G[3][0]); emg_mac(acc, 0.05, G[3][2]); }
};
template <> struct Pair<5, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[5][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[2][0]); emg_mac(acc, -0.05, G[2][3]); emg_mac(acc, -0.05, G[3][0]); emg_mac(acc, 0.05, G[3][3]); }
};
template <> struct Pair<5, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.05, G[2][1]); emg_mac(acc, -0.05, G[2][2]); emg_mac(acc, -0.1, G[3][1]); emg_mac(acc, 0.05, G[3][2]); }
};
template <> struct Pair<5, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[2][1]); emg_mac(acc, -0.05, G[2][3]); emg_mac(acc, -0.05, G[3][1]); emg_mac(acc, 0.05, G[3][3]); }
};
template <> struct Pair<5, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 4.0, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.1, G[2][2]); emg_mac(acc, -0.05, G[2][3]); emg_mac(acc, -0.05, G[3][2]); emg_mac(acc, 0.1, G[3][3]); }
};
template <> struct Pair<5, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.008333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][1]); }
};
template <> struct Pair<5, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, -0.008333333333333333, G[2][2]); emg_mac(acc, 0.03333333333333333, G[3][0]); }
};
template <> struct Pair<5, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[2][0]); emg_mac(acc, 0.008333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<5, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, -0.008333333333333333, G[2][2]); emg_mac(acc, 0.03333333333333333, G[3][1]); }
};
template <> struct Pair<5, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[2][1]); emg_mac(acc, 0.008333333333333333, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<5, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[2][2]); emg_mac(acc, 0.03333333333333333, G[3][3]); }
};
template <> struct Pair<5, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[5][0]); emg_mac(acc, 0.5, H[5][1]); emg_mac(acc, 1.0, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[2][1]); emg_mac(acc, -0.008333333333333333, G[2][2]); emg_mac(acc, -0.016666666666666666, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<5, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[5][0]); emg_mac(acc, 0.5, H[5][2]); emg_mac(acc, 1.0, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][1]); emg_mac(acc, -0.008333333333333333, G[2][3]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<5, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[5][1]); emg_mac(acc, 0.5, H[5][2]); emg_mac(acc, 1.0, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][2]); emg_mac(acc, -0.008333333333333333, G[2][3]); emg_mac(acc, -0.008333333333333333, G[3][2]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<5, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[5][3]); emg_mac(acc, 0.5, H[5][4]); emg_mac(acc, 1.0, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][2]); emg_mac(acc, -0.008333333333333333, G[2][3]); emg_mac(acc, -0.008333333333333333, G[3][2]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<5, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[5][0]); emg_mac(acc, 1.0, H[5][1]); emg_mac(acc, 0.5, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[2][0]); emg_mac(acc, -0.008333333333333333, G[2][2]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<5, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[5][0]); emg_mac(acc, 1.0, H[5][2]); emg_mac(acc, 0.5, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][0]); emg_mac(acc, -0.008333333333333333, G[2][3]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<5, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[5][1]); emg_mac(acc, 1.0, H[5][2]); emg_mac(acc, 0.5, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][0]); emg_mac(acc, -0.008333333333333333, G[2][3]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<5, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[5][3]); emg_mac(acc, 1.0, H[5][4]); emg_mac(acc, 0.5, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][1]); emg_mac(acc, -0.008333333333333333, G[2][3]); emg_mac(acc, -0.016666666666666666, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<6, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][0]); emg_mac(acc, 0.03333333333333333, G[1][1]); }
};
template <> struct Pair<6, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, 0.03333333333333333, G[1][2]); }
};
template <> struct Pair<6, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, 0.03333333333333333, G[1][3]); }
};
template <> struct Pair<6, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, 0.03333333333333333, G[0][2]); emg_mac(acc, -0.008333333333333333, G[1][1]); }
};
template <> struct Pair<6, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, 0.03333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[1][1]); }
};
template <> struct Pair<6, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, 0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, 0.008333333333333333, G[1][3]); }
};
template <> struct Pair<6, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.9, H[0][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.01904761904761905, G[0][0]); emg_mac(acc, -0.004761904761904762, G[0][1]); emg_mac(acc, -0.004761904761904762, G[1][0]); emg_mac(acc, 0.01904761904761905, G[1][1]); }
};
template <> struct Pair<6, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[0][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[1][0]); emg_mac(acc, 0.016666666666666666, G[1][2]); }
};
template <> struct Pair<6, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[0][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[1][0]); emg_mac(acc, 0.016666666666666666, G[1][3]); }
};
template <> struct Pair<6, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.45, H[0][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[0][1]); emg_mac(acc, 0.016666666666666666, G[0][2]); emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, -0.002380952380952381, G[1][2]); }
};
template <> struct Pair<6, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.45, H[0][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[0][1]); emg_mac(acc, 0.016666666666666666, G[0][3]); emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, -0.002380952380952381, G[1][3]); }
};
template <> struct Pair<6, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[0][2]); emg_mac(acc, 0.0011904761904761906, G[0][3]); emg_mac(acc, 0.0011904761904761906, G[1][2]); emg_mac(acc, 0.0011904761904761906, G[1][3]); }
};
template <> struct Pair<6, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[0][1]); emg_mac(acc, 0.3, H[0][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][2]); emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.002380952380952381, G[1][2]); }
};
template <> struct Pair<6, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[0][2]); emg_mac(acc, 0.3, H[0][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][3]); emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.002380952380952381, G[1][3]); }
};
template <> struct Pair<6, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.3, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][2]); emg_mac(acc, 0.004761904761904762, G[1][3]); }
};
template <> struct Pair<6, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][2]); emg_mac(acc, 0.004761904761904762, G[0][3]); }
};
template <> struct Pair<6, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[0][1]); emg_mac(acc, 0.15, H[0][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.002380952380952381, G[0][2]); emg_mac(acc, 0.002380952380952381, G[1][2]); }
};
template <> struct Pair<6, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[0][2]); emg_mac(acc, 0.15, H[0][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.002380952380952381, G[0][3]); emg_mac(acc, 0.002380952380952381, G[1][3]); }
};
template <> struct Pair<6, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[0][0]); emg_mac(acc, -0.0011904761904761906, G[1][0]); emg_mac(acc, 0.004761904761904762, G[1][3]); }
};
template <> struct Pair<6, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[0][1]); emg_mac(acc, 0.004761904761904762, G[0][3]); emg_mac(acc, -0.0011904761904761906, G[1][1]); }
};
template <> struct Pair<7, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.03333333333333333, G[2][1]); }
};
template <> struct Pair<7, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][0]); emg_mac(acc, 0.03333333333333333, G[2][2]); }
};
template <> struct Pair<7, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.03333333333333333, G[2][3]); }
};
template <> struct Pair<7, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][1]); emg_mac(acc, 0.008333333333333333, G[0][2]); emg_mac(acc, 0.008333333333333333, G[2][2]); }
};
template <> struct Pair<7, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, 0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<7, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, 0.03333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[2][2]); }
};
template <> struct Pair<7, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[1][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][1]); emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][1]); }
};
template <> struct Pair<7, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.9, H[1][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.01904761904761905, G[0][0]); emg_mac(acc, -0.004761904761904762, G[0][2]); emg_mac(acc, -0.004761904761904762, G[2][0]); emg_mac(acc, 0.01904761904761905, G[2][2]); }
};
template <> struct Pair<7, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[1][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<7, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[1][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][1]); emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[2][1]); emg_mac(acc, 0.002380952380952381, G[2][2]); }
};
template <> struct Pair<7, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[0][1]); emg_mac(acc, 0.0011904761904761906, G[0][3]); emg_mac(acc, 0.0011904761904761906, G[2][1]); emg_mac(acc, 0.0011904761904761906, G[2][3]); }
};
template <> struct Pair<7, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.45, H[1][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, 0.016666666666666666, G[0][3]); emg_mac(acc, 0.002380952380952381, G[2][2]); emg_mac(acc, -0.002380952380952381, G[2][3]); }
};
template <> struct Pair<7, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[1][0]); emg_mac(acc, 0.3, H[1][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[0][1]); emg_mac(acc, -0.002380952380952381, G[2][1]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<7, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.3, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][1]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<7, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[1][2]); emg_mac(acc, 0.3, H[1][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][3]); emg_mac(acc, -0.004761904761904762, G[2][2]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<7, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[0][2]); emg_mac(acc, 0.004761904761904762, G[0][3]); emg_mac(acc, -0.0011904761904761906, G[2][2]); }
};
template <> struct Pair<7, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[1][0]); emg_mac(acc, 0.15, H[1][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<7, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[0][0]); emg_mac(acc, -0.0011904761904761906, G[2][0]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<7, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[1][2]); emg_mac(acc, 0.15, H[1][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.002380952380952381, G[0][3]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<7, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][1]); emg_mac(acc, 0.004761904761904762, G[0][3]); }
};
template <> struct Pair<8, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.03333333333333333, G[3][1]); }
};
template <> struct Pair<8, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.03333333333333333, G[3][2]); }
};
template <> struct Pair<8, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][0]); emg_mac(acc, 0.03333333333333333, G[3][3]); }
};
template <> struct Pair<8, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, 0.008333333333333333, G[0][2]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<8, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][1]); emg_mac(acc, 0.008333333333333333, G[0][3]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<8, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[0][2]); emg_mac(acc, 0.008333333333333333, G[0][3]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<8, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[2][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][1]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][1]); }
};
template <> struct Pair<8, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[2][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<8, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.9, H[2][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.01904761904761905, G[0][0]); emg_mac(acc, -0.004761904761904762, G[0][3]); emg_mac(acc, -0.004761904761904762, G[3][0]); emg_mac(acc, 0.01904761904761905, G[3][3]); }
};
template <> struct Pair<8, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[0][1]); emg_mac(acc, 0.0011904761904761906, G[0][2]); emg_mac(acc, 0.0011904761904761906, G[3][1]); emg_mac(acc, 0.0011904761904761906, G[3][2]); }
};
template <> struct Pair<8, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[2][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][1]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<8, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[2][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][2]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<8, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.3, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[3][1]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<8, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[2][0]); emg_mac(acc, 0.3, H[2][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[0][1]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<8, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[2][1]); emg_mac(acc, 0.3, H[2][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<8, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][2]); emg_mac(acc, 0.0011904761904761906, G[0][3]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<8, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[0][0]); emg_mac(acc, -0.0011904761904761906, G[3][0]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<8, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[2][0]); emg_mac(acc, 0.15, H[2][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<8, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[2][1]); emg_mac(acc, 0.15, H[2][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<8, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][1]); emg_mac(acc, 0.0011904761904761906, G[0][3]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<9, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][1]); emg_mac(acc, -0.03333333333333333, G[2][0]); emg_mac(acc, 0.008333333333333333, G[2][1]); }
};
template <> struct Pair<9, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][0]); emg_mac(acc, 0.008333333333333333, G[1][2]); emg_mac(acc, 0.008333333333333333, G[2][2]); }
};
template <> struct Pair<9, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, 0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<9, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][1]); emg_mac(acc, 0.03333333333333333, G[2][2]); }
};
template <> struct Pair<9, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][1]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.03333333333333333, G[2][3]); }
};
template <> struct Pair<9, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, 0.03333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[2][2]); }
};
template <> struct Pair<9, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.45, H[3][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[1][0]); emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, 0.016666666666666666, G[2][0]); emg_mac(acc, -0.002380952380952381, G[2][1]); }
};
template <> struct Pair<9, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[3][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][0]); emg_mac(acc, -0.002380952380952381, G[1][2]); emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, 0.002380952380952381, G[2][2]); }
};
template <> struct Pair<9, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[1][0]); emg_mac(acc, 0.0011904761904761906, G[1][3]); emg_mac(acc, 0.0011904761904761906, G[2][0]); emg_mac(acc, 0.0011904761904761906, G[2][3]); }
};
template <> struct Pair<9, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.9, H[3][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.01904761904761905, G[1][1]); emg_mac(acc, -0.004761904761904762, G[1][2]); emg_mac(acc, -0.004761904761904762, G[2][1]); emg_mac(acc, 0.01904761904761905, G[2][2]); }
};
template <> struct Pair<9, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[3][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[2][1]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<9, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.45, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[1][2]); emg_mac(acc, 0.016666666666666666, G[1][3]); emg_mac(acc, 0.002380952380952381, G[2][2]); emg_mac(acc, -0.002380952380952381, G[2][3]); }
};
template <> struct Pair<9, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[3][0]); emg_mac(acc, 0.15, H[3][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<9, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[1][1]); emg_mac(acc, -0.0011904761904761906, G[2][1]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<9, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[1][2]); emg_mac(acc, 0.004761904761904762, G[1][3]); emg_mac(acc, -0.0011904761904761906, G[2][2]); }
};
template <> struct Pair<9, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[3][4]); emg_mac(acc, 0.3, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][3]); emg_mac(acc, -0.004761904761904762, G[2][2]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<9, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[3][0]); emg_mac(acc, 0.3, H[3][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[1][0]); emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<9, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.3, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][0]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<9, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][0]); emg_mac(acc, 0.004761904761904762, G[1][3]); }
};
template <> struct Pair<9, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[3][4]); emg_mac(acc, 0.15, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.002380952380952381, G[1][3]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<10, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][1]); emg_mac(acc, -0.03333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][1]); }
};
template <> struct Pair<10, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][0]); emg_mac(acc, 0.008333333333333333, G[1][2]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<10, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][0]); emg_mac(acc, 0.008333333333333333, G[1][3]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<10, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[1][1]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.03333333333333333, G[3][2]); }
};
template <> struct Pair<10, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][1]); emg_mac(acc, 0.03333333333333333, G[3][3]); }
};
template <> struct Pair<10, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[1][2]); emg_mac(acc, 0.008333333333333333, G[1][3]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<10, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.45, H[4][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[1][0]); emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, 0.016666666666666666, G[3][0]); emg_mac(acc, -0.002380952380952381, G[3][1]); }
};
template <> struct Pair<10, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[1][0]); emg_mac(acc, 0.0011904761904761906, G[1][2]); emg_mac(acc, 0.0011904761904761906, G[3][0]); emg_mac(acc, 0.0011904761904761906, G[3][2]); }
};
template <> struct Pair<10, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[4][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][0]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<10, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[4][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, -0.002380952380952381, G[1][2]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<10, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.9, H[4][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.01904761904761905, G[1][1]); emg_mac(acc, -0.004761904761904762, G[1][3]); emg_mac(acc, -0.004761904761904762, G[3][1]); emg_mac(acc, 0.01904761904761905, G[3][3]); }
};
template <> struct Pair<10, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][2]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<10, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[1][1]); emg_mac(acc, -0.0011904761904761906, G[3][1]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<10, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[4][0]); emg_mac(acc, 0.15, H[4][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<10, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][2]); emg_mac(acc, 0.0011904761904761906, G[1][3]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<10, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[4][3]); emg_mac(acc, 0.3, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[1][2]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<10, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.3, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[3][0]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<10, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[4][0]); emg_mac(acc, 0.3, H[4][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[1][0]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<10, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][0]); emg_mac(acc, 0.0011904761904761906, G[1][3]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<10, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[4][3]); emg_mac(acc, 0.15, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<11, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.008333333333333333, G[2][1]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][1]); }
};
template <> struct Pair<11, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[2][2]); emg_mac(acc, -0.03333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<11, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[2][0]); emg_mac(acc, 0.008333333333333333, G[2][3]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<11, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[2][2]); emg_mac(acc, -0.03333333333333333, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<11, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[2][1]); emg_mac(acc, 0.008333333333333333, G[2][3]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<11, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.03333333333333333, G[2][2]); emg_mac(acc, 0.03333333333333333, G[3][3]); }
};
template <> struct Pair<11, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[2][0]); emg_mac(acc, 0.0011904761904761906, G[2][1]); emg_mac(acc, 0.0011904761904761906, G[3][0]); emg_mac(acc, 0.0011904761904761906, G[3][1]); }
};
template <> struct Pair<11, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.45, H[5][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, 0.002380952380952381, G[2][2]); emg_mac(acc, 0.016666666666666666, G[3][0]); emg_mac(acc, -0.002380952380952381, G[3][2]); }
};
template <> struct Pair<11, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[5][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][0]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<11, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.45, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[2][1]); emg_mac(acc, 0.002380952380952381, G[2][2]); emg_mac(acc, 0.016666666666666666, G[3][1]); emg_mac(acc, -0.002380952380952381, G[3][2]); }
};
template <> struct Pair<11, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.45, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][1]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<11, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.9, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.01904761904761905, G[2][2]); emg_mac(acc, -0.004761904761904762, G[2][3]); emg_mac(acc, -0.004761904761904762, G[3][2]); emg_mac(acc, 0.01904761904761905, G[3][3]); }
};
template <> struct Pair<11, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[2][2]); emg_mac(acc, -0.004761904761904762, G[3][1]); emg_mac(acc, 0.0011904761904761906, G[3][2]); }
};
template <> struct Pair<11, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][1]); emg_mac(acc, 0.0011904761904761906, G[2][3]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<11, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[5][1]); emg_mac(acc, 0.15, H[5][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][2]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<11, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[5][3]); emg_mac(acc, 0.15, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][2]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<11, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[2][2]); emg_mac(acc, -0.004761904761904762, G[3][0]); emg_mac(acc, 0.0011904761904761906, G[3][2]); }
};
template <> struct Pair<11, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][0]); emg_mac(acc, 0.0011904761904761906, G[2][3]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<11, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[5][1]); emg_mac(acc, 0.3, H[5][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<11, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[5][3]); emg_mac(acc, 0.3, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[2][1]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<12, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][0]); emg_mac(acc, 0.5, H[1][0]); emg_mac(acc, 1.0, H[3][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][0]); emg_mac(acc, -0.016666666666666666, G[1][1]); emg_mac(acc, -0.016666666666666666, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][1]); }
};
template <> struct Pair<12, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][1]); emg_mac(acc, 0.5, H[1][1]); emg_mac(acc, 1.0, H[3][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][0]); emg_mac(acc, -0.016666666666666666, G[1][2]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][2]); }
};
template <> struct Pair<12, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][2]); emg_mac(acc, 0.5, H[1][2]); emg_mac(acc, 1.0, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][0]); emg_mac(acc, -0.016666666666666666, G[1][3]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<12, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][3]); emg_mac(acc, 0.5, H[1][3]); emg_mac(acc, 1.0, H[3][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.016666666666666666, G[2][2]); }
};
template <> struct Pair<12, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][4]); emg_mac(acc, 0.5, H[1][4]); emg_mac(acc, 1.0, H[3][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<12, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][5]); emg_mac(acc, 0.5, H[1][5]); emg_mac(acc, 1.0, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][2]); emg_mac(acc, -0.016666666666666666, G[1][3]); emg_mac(acc, -0.008333333333333333, G[2][2]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<12, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[1][0]); emg_mac(acc, 0.3, H[3][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.002380952380952381, G[2][0]); emg_mac(acc, 0.002380952380952381, G[2][1]); }
};
template <> struct Pair<12, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[0][1]); emg_mac(acc, 0.3, H[3][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[1][0]); emg_mac(acc, -0.002380952380952381, G[1][2]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<12, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.3, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][3]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<12, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[0][3]); emg_mac(acc, 0.15, H[1][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<12, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[1][1]); emg_mac(acc, -0.0011904761904761906, G[1][3]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<12, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][3]); emg_mac(acc, 0.0011904761904761906, G[2][2]); emg_mac(acc, 0.0011904761904761906, G[2][3]); }
};
template <> struct Pair<12, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[0][0]); emg_mac(acc, -0.05, H[0][1]); emg_mac(acc, -0.1, H[0][3]); emg_mac(acc, -0.05, H[1][0]); emg_mac(acc, 0.1, H[1][1]); emg_mac(acc, 0.1, H[1][3]); emg_mac(acc, -0.1, H[3][0]); emg_mac(acc, 0.1, H[3][1]); emg_mac(acc, 0.4, H[3][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[1][1]); emg_mac(acc, -0.002380952380952381, G[1][2]); emg_mac(acc, -0.002380952380952381, G[2][1]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<12, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[0][0]); emg_mac(acc, -0.05, H[0][2]); emg_mac(acc, -0.1, H[0][4]); emg_mac(acc, -0.05, H[1][0]); emg_mac(acc, 0.1, H[1][2]); emg_mac(acc, 0.1, H[1][4]); emg_mac(acc, -0.1, H[3][0]); emg_mac(acc, 0.1, H[3][2]); emg_mac(acc, 0.4, H[3][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[2][1]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<12, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[0][1]); emg_mac(acc, -0.1, H[0][2]); emg_mac(acc, -0.1, H[0][5]); emg_mac(acc, -0.05, H[1][1]); emg_mac(acc, 0.05, H[1][2]); emg_mac(acc, 0.1, H[1][5]); emg_mac(acc, -0.1, H[3][1]); emg_mac(acc, 0.1, H[3][2]); emg_mac(acc, 0.4, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][2]); emg_mac(acc, -0.004761904761904762, G[1][3]); emg_mac(acc, -0.002380952380952381, G[2][2]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<12, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[0][3]); emg_mac(acc, -0.1, H[0][4]); emg_mac(acc, -0.1, H[0][5]); emg_mac(acc, -0.05, H[1][3]); emg_mac(acc, 0.05, H[1][4]); emg_mac(acc, 0.2, H[1][5]); emg_mac(acc, -0.1, H[3][3]); emg_mac(acc, 0.1, H[3][4]); emg_mac(acc, 0.2, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[1][2]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[2][2]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<12, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[0][0]); emg_mac(acc, -0.1, H[0][1]); emg_mac(acc, -0.05, H[0][3]); emg_mac(acc, 0.05, H[1][0]); emg_mac(acc, 0.2, H[1][1]); emg_mac(acc, 0.05, H[1][3]); emg_mac(acc, 0.1, H[3][0]); emg_mac(acc, 0.2, H[3][1]); emg_mac(acc, 0.2, H[3][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][0]); emg_mac(acc, -0.002380952380952381, G[1][2]); emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<12, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[0][0]); emg_mac(acc, -0.1, H[0][2]); emg_mac(acc, -0.05, H[0][4]); emg_mac(acc, 0.05, H[1][0]); emg_mac(acc, 0.2, H[1][2]); emg_mac(acc, 0.05, H[1][4]); emg_mac(acc, 0.1, H[3][0]); emg_mac(acc, 0.2, H[3][2]); emg_mac(acc, 0.2, H[3][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[1][0]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<12, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[0][1]); emg_mac(acc, -0.2, H[0][2]); emg_mac(acc, -0.05, H[0][5]); emg_mac(acc, 0.05, H[1][1]); emg_mac(acc, 0.1, H[1][2]); emg_mac(acc, 0.05, H[1][5]); emg_mac(acc, 0.1, H[3][1]); emg_mac(acc, 0.2, H[3][2]); emg_mac(acc, 0.2, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][0]); emg_mac(acc, -0.004761904761904762, G[1][3]); emg_mac(acc, -0.0011904761904761906, G[2][0]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<12, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[0][3]); emg_mac(acc, -0.2, H[0][4]); emg_mac(acc, -0.05, H[0][5]); emg_mac(acc, 0.05, H[1][3]); emg_mac(acc, 0.1, H[1][4]); emg_mac(acc, 0.1, H[1][5]); emg_mac(acc, 0.1, H[3][3]); emg_mac(acc, 0.2, H[3][4]); emg_mac(acc, 0.1, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.0011904761904761906, G[2][1]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<13, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][0]); emg_mac(acc, 0.5, H[2][0]); emg_mac(acc, 1.0, H[4][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][0]); emg_mac(acc, -0.016666666666666666, G[1][1]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][1]); }
};
template <> struct Pair<13, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][1]); emg_mac(acc, 0.5, H[2][1]); emg_mac(acc, 1.0, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][0]); emg_mac(acc, -0.016666666666666666, G[1][2]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<13, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][2]); emg_mac(acc, 0.5, H[2][2]); emg_mac(acc, 1.0, H[4][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][0]); emg_mac(acc, -0.016666666666666666, G[1][3]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<13, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][3]); emg_mac(acc, 0.5, H[2][3]); emg_mac(acc, 1.0, H[4][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<13, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][4]); emg_mac(acc, 0.5, H[2][4]); emg_mac(acc, 1.0, H[4][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<13, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[0][5]); emg_mac(acc, 0.5, H[2][5]); emg_mac(acc, 1.0, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][2]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[3][2]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<13, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[2][0]); emg_mac(acc, 0.3, H[4][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][1]); }
};
template <> struct Pair<13, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.3, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][2]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<13, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[0][2]); emg_mac(acc, 0.3, H[4][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[1][0]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<13, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[1][1]); emg_mac(acc, -0.0011904761904761906, G[1][2]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<13, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[0][4]); emg_mac(acc, 0.15, H[2][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<13, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][2]); emg_mac(acc, 0.0011904761904761906, G[3][2]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<13, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[0][0]); emg_mac(acc, -0.05, H[0][1]); emg_mac(acc, -0.1, H[0][3]); emg_mac(acc, -0.05, H[2][0]); emg_mac(acc, 0.1, H[2][1]); emg_mac(acc, 0.1, H[2][3]); emg_mac(acc, -0.1, H[4][0]); emg_mac(acc, 0.1, H[4][1]); emg_mac(acc, 0.4, H[4][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, -0.002380952380952381, G[1][2]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<13, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[0][0]); emg_mac(acc, -0.05, H[0][2]); emg_mac(acc, -0.1, H[0][4]); emg_mac(acc, -0.05, H[2][0]); emg_mac(acc, 0.1, H[2][2]); emg_mac(acc, 0.1, H[2][4]); emg_mac(acc, -0.1, H[4][0]); emg_mac(acc, 0.1, H[4][2]); emg_mac(acc, 0.4, H[4][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[1][1]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<13, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[0][1]); emg_mac(acc, -0.05, H[0][2]); emg_mac(acc, -0.1, H[0][5]); emg_mac(acc, -0.05, H[2][1]); emg_mac(acc, 0.05, H[2][2]); emg_mac(acc, 0.1, H[2][5]); emg_mac(acc, -0.1, H[4][1]); emg_mac(acc, 0.1, H[4][2]); emg_mac(acc, 0.4, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[1][2]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<13, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[0][3]); emg_mac(acc, -0.05, H[0][4]); emg_mac(acc, -0.1, H[0][5]); emg_mac(acc, -0.05, H[2][3]); emg_mac(acc, 0.05, H[2][4]); emg_mac(acc, 0.2, H[2][5]); emg_mac(acc, -0.1, H[4][3]); emg_mac(acc, 0.1, H[4][4]); emg_mac(acc, 0.2, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][2]); emg_mac(acc, -0.0011904761904761906, G[1][3]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<13, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[0][0]); emg_mac(acc, -0.1, H[0][1]); emg_mac(acc, -0.05, H[0][3]); emg_mac(acc, 0.05, H[2][0]); emg_mac(acc, 0.2, H[2][1]); emg_mac(acc, 0.05, H[2][3]); emg_mac(acc, 0.1, H[4][0]); emg_mac(acc, 0.2, H[4][1]); emg_mac(acc, 0.2, H[4][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[1][0]); emg_mac(acc, -0.002380952380952381, G[1][2]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<13, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[0][0]); emg_mac(acc, -0.1, H[0][2]); emg_mac(acc, -0.05, H[0][4]); emg_mac(acc, 0.05, H[2][0]); emg_mac(acc, 0.2, H[2][2]); emg_mac(acc, 0.05, H[2][4]); emg_mac(acc, 0.1, H[4][0]); emg_mac(acc, 0.2, H[4][2]); emg_mac(acc, 0.2, H[4][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][0]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<13, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[0][1]); emg_mac(acc, -0.1, H[0][2]); emg_mac(acc, -0.05, H[0][5]); emg_mac(acc, 0.05, H[2][1]); emg_mac(acc, 0.1, H[2][2]); emg_mac(acc, 0.05, H[2][5]); emg_mac(acc, 0.1, H[4][1]); emg_mac(acc, 0.2, H[4][2]); emg_mac(acc, 0.2, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][0]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.0011904761904761906, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<13, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[0][3]); emg_mac(acc, -0.1, H[0][4]); emg_mac(acc, -0.05, H[0][5]); emg_mac(acc, 0.05, H[2][3]); emg_mac(acc, 0.1, H[2][4]); emg_mac(acc, 0.1, H[2][5]); emg_mac(acc, 0.1, H[4][3]); emg_mac(acc, 0.2, H[4][4]); emg_mac(acc, 0.1, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, -0.0011904761904761906, G[1][3]); emg_mac(acc, -0.0011904761904761906, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<14, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[1][0]); emg_mac(acc, 0.5, H[2][0]); emg_mac(acc, 1.0, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[2][0]); emg_mac(acc, -0.016666666666666666, G[2][1]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][1]); }
};
template <> struct Pair<14, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[1][1]); emg_mac(acc, 0.5, H[2][1]); emg_mac(acc, 1.0, H[5][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[2][0]); emg_mac(acc, -0.016666666666666666, G[2][2]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<14, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[1][2]); emg_mac(acc, 0.5, H[2][2]); emg_mac(acc, 1.0, H[5][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][0]); emg_mac(acc, -0.016666666666666666, G[2][3]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<14, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[1][3]); emg_mac(acc, 0.5, H[2][3]); emg_mac(acc, 1.0, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[2][1]); emg_mac(acc, -0.008333333333333333, G[2][2]); emg_mac(acc, -0.016666666666666666, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<14, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[1][4]); emg_mac(acc, 0.5, H[2][4]); emg_mac(acc, 1.0, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][1]); emg_mac(acc, -0.008333333333333333, G[2][3]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<14, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[1][5]); emg_mac(acc, 0.5, H[2][5]); emg_mac(acc, 1.0, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][2]); emg_mac(acc, -0.008333333333333333, G[2][3]); emg_mac(acc, -0.008333333333333333, G[3][2]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<14, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.3, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][1]); emg_mac(acc, 0.004761904761904762, G[3][1]); }
};
template <> struct Pair<14, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[2][1]); emg_mac(acc, 0.3, H[5][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][2]); emg_mac(acc, 0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<14, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[1][2]); emg_mac(acc, 0.3, H[5][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<14, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[2][1]); emg_mac(acc, -0.0011904761904761906, G[2][2]); emg_mac(acc, 0.004761904761904762, G[3][1]); }
};
template <> struct Pair<14, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][1]); emg_mac(acc, 0.0011904761904761906, G[3][1]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<14, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[1][5]); emg_mac(acc, 0.15, H[2][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][2]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<14, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[1][0]); emg_mac(acc, -0.05, H[1][1]); emg_mac(acc, -0.1, H[1][3]); emg_mac(acc, -0.1, H[2][0]); emg_mac(acc, 0.05, H[2][1]); emg_mac(acc, 0.1, H[2][3]); emg_mac(acc, -0.1, H[5][0]); emg_mac(acc, 0.1, H[5][1]); emg_mac(acc, 0.4, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[2][1]); emg_mac(acc, -0.002380952380952381, G[2][2]); emg_mac(acc, -0.004761904761904762, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<14, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[1][0]); emg_mac(acc, -0.05, H[1][2]); emg_mac(acc, -0.1, H[1][4]); emg_mac(acc, -0.05, H[2][0]); emg_mac(acc, 0.05, H[2][2]); emg_mac(acc, 0.1, H[2][4]); emg_mac(acc, -0.1, H[5][0]); emg_mac(acc, 0.1, H[5][2]); emg_mac(acc, 0.4, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[2][1]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<14, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[1][1]); emg_mac(acc, -0.05, H[1][2]); emg_mac(acc, -0.1, H[1][5]); emg_mac(acc, -0.05, H[2][1]); emg_mac(acc, 0.1, H[2][2]); emg_mac(acc, 0.1, H[2][5]); emg_mac(acc, -0.1, H[5][1]); emg_mac(acc, 0.1, H[5][2]); emg_mac(acc, 0.4, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[2][2]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<14, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[1][3]); emg_mac(acc, -0.05, H[1][4]); emg_mac(acc, -0.1, H[1][5]); emg_mac(acc, -0.05, H[2][3]); emg_mac(acc, 0.1, H[2][4]); emg_mac(acc, 0.1, H[2][5]); emg_mac(acc, -0.1, H[5][3]); emg_mac(acc, 0.1, H[5][4]); emg_mac(acc, 0.2, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[2][2]); emg_mac(acc, -0.0011904761904761906, G[2][3]); emg_mac(acc, -0.0011904761904761906, G[3][2]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<14, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[1][0]); emg_mac(acc, -0.1, H[1][1]); emg_mac(acc, -0.05, H[1][3]); emg_mac(acc, 0.1, H[2][0]); emg_mac(acc, 0.1, H[2][1]); emg_mac(acc, 0.05, H[2][3]); emg_mac(acc, 0.1, H[5][0]); emg_mac(acc, 0.2, H[5][1]); emg_mac(acc, 0.2, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[2][0]); emg_mac(acc, -0.002380952380952381, G[2][2]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<14, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[1][0]); emg_mac(acc, -0.1, H[1][2]); emg_mac(acc, -0.05, H[1][4]); emg_mac(acc, 0.05, H[2][0]); emg_mac(acc, 0.1, H[2][2]); emg_mac(acc, 0.05, H[2][4]); emg_mac(acc, 0.1, H[5][0]); emg_mac(acc, 0.2, H[5][2]); emg_mac(acc, 0.2, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[2][0]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, -0.0011904761904761906, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<14, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[1][1]); emg_mac(acc, -0.1, H[1][2]); emg_mac(acc, -0.05, H[1][5]); emg_mac(acc, 0.05, H[2][1]); emg_mac(acc, 0.2, H[2][2]); emg_mac(acc, 0.05, H[2][5]); emg_mac(acc, 0.1, H[5][1]); emg_mac(acc, 0.2, H[5][2]); emg_mac(acc, 0.2, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[2][0]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<14, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[1][3]); emg_mac(acc, -0.1, H[1][4]); emg_mac(acc, -0.05, H[1][5]); emg_mac(acc, 0.05, H[2][3]); emg_mac(acc, 0.2, H[2][4]); emg_mac(acc, 0.05, H[2][5]); emg_mac(acc, 0.1, H[5][3]); emg_mac(acc, 0.2, H[5][4]); emg_mac(acc, 0.1, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[2][1]); emg_mac(acc, -0.0011904761904761906, G[2][3]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<15, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[3][0]); emg_mac(acc, 0.5, H[4][0]); emg_mac(acc, 1.0, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][0]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][1]); }
};
template <> struct Pair<15, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[3][1]); emg_mac(acc, 0.5, H[4][1]); emg_mac(acc, 1.0, H[5][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[2][0]); emg_mac(acc, -0.008333333333333333, G[2][2]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<15, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[3][2]); emg_mac(acc, 0.5, H[4][2]); emg_mac(acc, 1.0, H[5][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][0]); emg_mac(acc, -0.008333333333333333, G[2][3]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<15, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[3][3]); emg_mac(acc, 0.5, H[4][3]); emg_mac(acc, 1.0, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[2][1]); emg_mac(acc, -0.016666666666666666, G[2][2]); emg_mac(acc, -0.016666666666666666, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<15, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[3][4]); emg_mac(acc, 0.5, H[4][4]); emg_mac(acc, 1.0, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][1]); emg_mac(acc, -0.016666666666666666, G[2][3]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<15, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.5, H[3][5]); emg_mac(acc, 0.5, H[4][5]); emg_mac(acc, 1.0, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[2][2]); emg_mac(acc, -0.008333333333333333, G[2][3]); emg_mac(acc, -0.008333333333333333, G[3][2]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<15, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][0]); emg_mac(acc, 0.004761904761904762, G[3][0]); }
};
template <> struct Pair<15, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[2][0]); emg_mac(acc, -0.0011904761904761906, G[2][2]); emg_mac(acc, 0.004761904761904762, G[3][0]); }
};
template <> struct Pair<15, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][0]); emg_mac(acc, 0.0011904761904761906, G[3][0]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<15, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[4][3]); emg_mac(acc, 0.3, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][2]); emg_mac(acc, 0.002380952380952381, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<15, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[3][4]); emg_mac(acc, 0.3, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[2][1]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<15, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[3][5]); emg_mac(acc, 0.15, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[2][2]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<15, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[3][0]); emg_mac(acc, -0.05, H[3][1]); emg_mac(acc, -0.1, H[3][3]); emg_mac(acc, -0.1, H[4][0]); emg_mac(acc, 0.05, H[4][1]); emg_mac(acc, 0.1, H[4][3]); emg_mac(acc, -0.1, H[5][0]); emg_mac(acc, 0.2, H[5][1]); emg_mac(acc, 0.2, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[2][1]); emg_mac(acc, -0.002380952380952381, G[2][2]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<15, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[3][0]); emg_mac(acc, -0.05, H[3][2]); emg_mac(acc, -0.1, H[3][4]); emg_mac(acc, -0.05, H[4][0]); emg_mac(acc, 0.05, H[4][2]); emg_mac(acc, 0.1, H[4][4]); emg_mac(acc, -0.1, H[5][0]); emg_mac(acc, 0.2, H[5][2]); emg_mac(acc, 0.2, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[2][1]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, -0.0011904761904761906, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<15, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[3][1]); emg_mac(acc, -0.05, H[3][2]); emg_mac(acc, -0.1, H[3][5]); emg_mac(acc, -0.05, H[4][1]); emg_mac(acc, 0.1, H[4][2]); emg_mac(acc, 0.1, H[4][5]); emg_mac(acc, -0.1, H[5][1]); emg_mac(acc, 0.1, H[5][2]); emg_mac(acc, 0.2, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[2][2]); emg_mac(acc, -0.0011904761904761906, G[2][3]); emg_mac(acc, -0.0011904761904761906, G[3][2]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<15, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[3][3]); emg_mac(acc, -0.05, H[3][4]); emg_mac(acc, -0.1, H[3][5]); emg_mac(acc, -0.05, H[4][3]); emg_mac(acc, 0.1, H[4][4]); emg_mac(acc, 0.1, H[4][5]); emg_mac(acc, -0.1, H[5][3]); emg_mac(acc, 0.1, H[5][4]); emg_mac(acc, 0.4, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[2][2]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<15, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[3][0]); emg_mac(acc, -0.1, H[3][1]); emg_mac(acc, -0.05, H[3][3]); emg_mac(acc, 0.1, H[4][0]); emg_mac(acc, 0.1, H[4][1]); emg_mac(acc, 0.05, H[4][3]); emg_mac(acc, 0.1, H[5][0]); emg_mac(acc, 0.4, H[5][1]); emg_mac(acc, 0.1, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[2][0]); emg_mac(acc, -0.002380952380952381, G[2][2]); emg_mac(acc, -0.004761904761904762, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<15, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[3][0]); emg_mac(acc, -0.1, H[3][2]); emg_mac(acc, -0.05, H[3][4]); emg_mac(acc, 0.05, H[4][0]); emg_mac(acc, 0.1, H[4][2]); emg_mac(acc, 0.05, H[4][4]); emg_mac(acc, 0.1, H[5][0]); emg_mac(acc, 0.4, H[5][2]); emg_mac(acc, 0.1, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[2][0]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<15, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[3][1]); emg_mac(acc, -0.1, H[3][2]); emg_mac(acc, -0.05, H[3][5]); emg_mac(acc, 0.05, H[4][1]); emg_mac(acc, 0.2, H[4][2]); emg_mac(acc, 0.05, H[4][5]); emg_mac(acc, 0.1, H[5][1]); emg_mac(acc, 0.2, H[5][2]); emg_mac(acc, 0.1, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[2][0]); emg_mac(acc, -0.0011904761904761906, G[2][3]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<15, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[3][3]); emg_mac(acc, -0.1, H[3][4]); emg_mac(acc, -0.05, H[3][5]); emg_mac(acc, 0.05, H[4][3]); emg_mac(acc, 0.2, H[4][4]); emg_mac(acc, 0.05, H[4][5]); emg_mac(acc, 0.1, H[5][3]); emg_mac(acc, 0.2, H[5][4]); emg_mac(acc, 0.2, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[2][1]); emg_mac(acc, -0.002380952380952381, G[2][3]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<16, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][0]); emg_mac(acc, 1.0, H[1][0]); emg_mac(acc, 0.5, H[3][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, -0.016666666666666666, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][1]); }
};
template <> struct Pair<16, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][1]); emg_mac(acc, 1.0, H[1][1]); emg_mac(acc, 0.5, H[3][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][2]); }
};
template <> struct Pair<16, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][2]); emg_mac(acc, 1.0, H[1][2]); emg_mac(acc, 0.5, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[2][0]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<16, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][3]); emg_mac(acc, 1.0, H[1][3]); emg_mac(acc, 0.5, H[3][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][1]); emg_mac(acc, -0.016666666666666666, G[0][2]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.016666666666666666, G[2][2]); }
};
template <> struct Pair<16, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][4]); emg_mac(acc, 1.0, H[1][4]); emg_mac(acc, 0.5, H[3][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][1]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.008333333333333333, G[2][1]); emg_mac(acc, 0.016666666666666666, G[2][3]); }
};
template <> struct Pair<16, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][5]); emg_mac(acc, 1.0, H[1][5]); emg_mac(acc, 0.5, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][2]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.008333333333333333, G[2][2]); emg_mac(acc, 0.008333333333333333, G[2][3]); }
};
template <> struct Pair<16, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[1][0]); emg_mac(acc, 0.15, H[3][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.002380952380952381, G[2][0]); emg_mac(acc, 0.002380952380952381, G[2][1]); }
};
template <> struct Pair<16, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[0][1]); emg_mac(acc, 0.15, H[3][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<16, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[0][0]); emg_mac(acc, -0.0011904761904761906, G[0][3]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<16, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[0][3]); emg_mac(acc, 0.3, H[1][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[0][1]); emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<16, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.3, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][3]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<16, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][3]); emg_mac(acc, 0.0011904761904761906, G[2][2]); emg_mac(acc, 0.0011904761904761906, G[2][3]); }
};
template <> struct Pair<16, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[0][0]); emg_mac(acc, 0.05, H[0][1]); emg_mac(acc, 0.1, H[0][3]); emg_mac(acc, -0.1, H[1][0]); emg_mac(acc, 0.2, H[1][1]); emg_mac(acc, 0.2, H[1][3]); emg_mac(acc, -0.05, H[3][0]); emg_mac(acc, 0.05, H[3][1]); emg_mac(acc, 0.2, H[3][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][1]); emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[2][1]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<16, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[0][0]); emg_mac(acc, 0.05, H[0][2]); emg_mac(acc, 0.1, H[0][4]); emg_mac(acc, -0.1, H[1][0]); emg_mac(acc, 0.2, H[1][2]); emg_mac(acc, 0.2, H[1][4]); emg_mac(acc, -0.05, H[3][0]); emg_mac(acc, 0.05, H[3][2]); emg_mac(acc, 0.2, H[3][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[0][1]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[2][1]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<16, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[0][1]); emg_mac(acc, 0.1, H[0][2]); emg_mac(acc, 0.1, H[0][5]); emg_mac(acc, -0.1, H[1][1]); emg_mac(acc, 0.1, H[1][2]); emg_mac(acc, 0.2, H[1][5]); emg_mac(acc, -0.05, H[3][1]); emg_mac(acc, 0.05, H[3][2]); emg_mac(acc, 0.2, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[0][2]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[2][2]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<16, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[0][3]); emg_mac(acc, 0.1, H[0][4]); emg_mac(acc, 0.1, H[0][5]); emg_mac(acc, -0.1, H[1][3]); emg_mac(acc, 0.1, H[1][4]); emg_mac(acc, 0.4, H[1][5]); emg_mac(acc, -0.05, H[3][3]); emg_mac(acc, 0.05, H[3][4]); emg_mac(acc, 0.1, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][2]); emg_mac(acc, -0.004761904761904762, G[0][3]); emg_mac(acc, -0.002380952380952381, G[2][2]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<16, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[0][0]); emg_mac(acc, 0.1, H[0][1]); emg_mac(acc, 0.05, H[0][3]); emg_mac(acc, 0.1, H[1][0]); emg_mac(acc, 0.4, H[1][1]); emg_mac(acc, 0.1, H[1][3]); emg_mac(acc, 0.05, H[3][0]); emg_mac(acc, 0.1, H[3][1]); emg_mac(acc, 0.1, H[3][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, 0.004761904761904762, G[2][2]); }
};
template <> struct Pair<16, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[0][0]); emg_mac(acc, 0.1, H[0][2]); emg_mac(acc, 0.05, H[0][4]); emg_mac(acc, 0.1, H[1][0]); emg_mac(acc, 0.4, H[1][2]); emg_mac(acc, 0.1, H[1][4]); emg_mac(acc, 0.05, H[3][0]); emg_mac(acc, 0.1, H[3][2]); emg_mac(acc, 0.1, H[3][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[2][0]); emg_mac(acc, 0.004761904761904762, G[2][3]); }
};
template <> struct Pair<16, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[0][1]); emg_mac(acc, 0.2, H[0][2]); emg_mac(acc, 0.05, H[0][5]); emg_mac(acc, 0.1, H[1][1]); emg_mac(acc, 0.2, H[1][2]); emg_mac(acc, 0.1, H[1][5]); emg_mac(acc, 0.05, H[3][1]); emg_mac(acc, 0.1, H[3][2]); emg_mac(acc, 0.1, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.0011904761904761906, G[2][0]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<16, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[0][3]); emg_mac(acc, 0.2, H[0][4]); emg_mac(acc, 0.05, H[0][5]); emg_mac(acc, 0.1, H[1][3]); emg_mac(acc, 0.2, H[1][4]); emg_mac(acc, 0.2, H[1][5]); emg_mac(acc, 0.05, H[3][3]); emg_mac(acc, 0.1, H[3][4]); emg_mac(acc, 0.05, H[3][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][1]); emg_mac(acc, -0.004761904761904762, G[0][3]); emg_mac(acc, -0.0011904761904761906, G[2][1]); emg_mac(acc, 0.002380952380952381, G[2][3]); }
};
template <> struct Pair<17, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][0]); emg_mac(acc, 1.0, H[2][0]); emg_mac(acc, 0.5, H[4][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][1]); }
};
template <> struct Pair<17, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][1]); emg_mac(acc, 1.0, H[2][1]); emg_mac(acc, 0.5, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<17, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][2]); emg_mac(acc, 1.0, H[2][2]); emg_mac(acc, 0.5, H[4][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<17, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][3]); emg_mac(acc, 1.0, H[2][3]); emg_mac(acc, 0.5, H[4][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][1]); emg_mac(acc, -0.016666666666666666, G[0][2]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<17, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][4]); emg_mac(acc, 1.0, H[2][4]); emg_mac(acc, 0.5, H[4][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][1]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<17, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[0][5]); emg_mac(acc, 1.0, H[2][5]); emg_mac(acc, 0.5, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][2]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[3][2]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<17, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[2][0]); emg_mac(acc, 0.15, H[4][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][1]); }
};
template <> struct Pair<17, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[0][0]); emg_mac(acc, -0.0011904761904761906, G[0][2]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<17, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[0][2]); emg_mac(acc, 0.15, H[4][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<17, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.3, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][2]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<17, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[0][4]); emg_mac(acc, 0.3, H[2][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[0][1]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<17, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[0][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][2]); emg_mac(acc, 0.0011904761904761906, G[3][2]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<17, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[0][0]); emg_mac(acc, 0.05, H[0][1]); emg_mac(acc, 0.1, H[0][3]); emg_mac(acc, -0.1, H[2][0]); emg_mac(acc, 0.2, H[2][1]); emg_mac(acc, 0.2, H[2][3]); emg_mac(acc, -0.05, H[4][0]); emg_mac(acc, 0.05, H[4][1]); emg_mac(acc, 0.2, H[4][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.0011904761904761906, G[0][1]); emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<17, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[0][0]); emg_mac(acc, 0.05, H[0][2]); emg_mac(acc, 0.1, H[0][4]); emg_mac(acc, -0.1, H[2][0]); emg_mac(acc, 0.2, H[2][2]); emg_mac(acc, 0.2, H[2][4]); emg_mac(acc, -0.05, H[4][0]); emg_mac(acc, 0.05, H[4][2]); emg_mac(acc, 0.2, H[4][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][1]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<17, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[0][1]); emg_mac(acc, 0.05, H[0][2]); emg_mac(acc, 0.1, H[0][5]); emg_mac(acc, -0.1, H[2][1]); emg_mac(acc, 0.1, H[2][2]); emg_mac(acc, 0.2, H[2][5]); emg_mac(acc, -0.05, H[4][1]); emg_mac(acc, 0.05, H[4][2]); emg_mac(acc, 0.2, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][2]); emg_mac(acc, -0.0011904761904761906, G[0][3]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<17, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[0][3]); emg_mac(acc, 0.05, H[0][4]); emg_mac(acc, 0.1, H[0][5]); emg_mac(acc, -0.1, H[2][3]); emg_mac(acc, 0.1, H[2][4]); emg_mac(acc, 0.4, H[2][5]); emg_mac(acc, -0.05, H[4][3]); emg_mac(acc, 0.05, H[4][4]); emg_mac(acc, 0.1, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[0][2]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<17, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[0][0]); emg_mac(acc, 0.1, H[0][1]); emg_mac(acc, 0.05, H[0][3]); emg_mac(acc, 0.1, H[2][0]); emg_mac(acc, 0.4, H[2][1]); emg_mac(acc, 0.1, H[2][3]); emg_mac(acc, 0.05, H[4][0]); emg_mac(acc, 0.1, H[4][1]); emg_mac(acc, 0.1, H[4][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.004761904761904762, G[3][2]); }
};
template <> struct Pair<17, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[0][0]); emg_mac(acc, 0.1, H[0][2]); emg_mac(acc, 0.05, H[0][4]); emg_mac(acc, 0.1, H[2][0]); emg_mac(acc, 0.4, H[2][2]); emg_mac(acc, 0.1, H[2][4]); emg_mac(acc, 0.05, H[4][0]); emg_mac(acc, 0.1, H[4][2]); emg_mac(acc, 0.1, H[4][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<17, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[0][1]); emg_mac(acc, 0.1, H[0][2]); emg_mac(acc, 0.05, H[0][5]); emg_mac(acc, 0.1, H[2][1]); emg_mac(acc, 0.2, H[2][2]); emg_mac(acc, 0.1, H[2][5]); emg_mac(acc, 0.05, H[4][1]); emg_mac(acc, 0.1, H[4][2]); emg_mac(acc, 0.1, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.0011904761904761906, G[0][3]); emg_mac(acc, -0.0011904761904761906, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<17, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[0][3]); emg_mac(acc, 0.1, H[0][4]); emg_mac(acc, 0.05, H[0][5]); emg_mac(acc, 0.1, H[2][3]); emg_mac(acc, 0.2, H[2][4]); emg_mac(acc, 0.2, H[2][5]); emg_mac(acc, 0.05, H[4][3]); emg_mac(acc, 0.1, H[4][4]); emg_mac(acc, 0.05, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][1]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.0011904761904761906, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<18, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[1][0]); emg_mac(acc, 1.0, H[2][0]); emg_mac(acc, 0.5, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][1]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][1]); }
};
template <> struct Pair<18, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[1][1]); emg_mac(acc, 1.0, H[2][1]); emg_mac(acc, 0.5, H[5][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<18, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[1][2]); emg_mac(acc, 1.0, H[2][2]); emg_mac(acc, 0.5, H[5][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][0]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<18, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[1][3]); emg_mac(acc, 1.0, H[2][3]); emg_mac(acc, 0.5, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][1]); emg_mac(acc, -0.008333333333333333, G[0][2]); emg_mac(acc, -0.016666666666666666, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<18, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[1][4]); emg_mac(acc, 1.0, H[2][4]); emg_mac(acc, 0.5, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][1]); emg_mac(acc, -0.008333333333333333, G[0][3]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<18, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[1][5]); emg_mac(acc, 1.0, H[2][5]); emg_mac(acc, 0.5, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[0][2]); emg_mac(acc, -0.016666666666666666, G[0][3]); emg_mac(acc, -0.008333333333333333, G[3][2]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<18, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.15, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[0][0]); emg_mac(acc, -0.0011904761904761906, G[0][1]); emg_mac(acc, 0.004761904761904762, G[3][1]); }
};
template <> struct Pair<18, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[2][1]); emg_mac(acc, 0.15, H[5][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<18, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[1][2]); emg_mac(acc, 0.15, H[5][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][0]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<18, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[2][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][1]); emg_mac(acc, 0.004761904761904762, G[3][1]); }
};
template <> struct Pair<18, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[1][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[0][1]); emg_mac(acc, 0.0011904761904761906, G[3][1]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<18, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[1][5]); emg_mac(acc, 0.3, H[2][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<18, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[1][0]); emg_mac(acc, 0.05, H[1][1]); emg_mac(acc, 0.1, H[1][3]); emg_mac(acc, -0.2, H[2][0]); emg_mac(acc, 0.1, H[2][1]); emg_mac(acc, 0.2, H[2][3]); emg_mac(acc, -0.05, H[5][0]); emg_mac(acc, 0.05, H[5][1]); emg_mac(acc, 0.2, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][1]); emg_mac(acc, -0.0011904761904761906, G[0][2]); emg_mac(acc, -0.004761904761904762, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<18, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[1][0]); emg_mac(acc, 0.05, H[1][2]); emg_mac(acc, 0.1, H[1][4]); emg_mac(acc, -0.1, H[2][0]); emg_mac(acc, 0.1, H[2][2]); emg_mac(acc, 0.2, H[2][4]); emg_mac(acc, -0.05, H[5][0]); emg_mac(acc, 0.05, H[5][2]); emg_mac(acc, 0.2, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][1]); emg_mac(acc, -0.0011904761904761906, G[0][3]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<18, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[1][1]); emg_mac(acc, 0.05, H[1][2]); emg_mac(acc, 0.1, H[1][5]); emg_mac(acc, -0.1, H[2][1]); emg_mac(acc, 0.2, H[2][2]); emg_mac(acc, 0.2, H[2][5]); emg_mac(acc, -0.05, H[5][1]); emg_mac(acc, 0.05, H[5][2]); emg_mac(acc, 0.2, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<18, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[1][3]); emg_mac(acc, 0.05, H[1][4]); emg_mac(acc, 0.1, H[1][5]); emg_mac(acc, -0.1, H[2][3]); emg_mac(acc, 0.2, H[2][4]); emg_mac(acc, 0.2, H[2][5]); emg_mac(acc, -0.05, H[5][3]); emg_mac(acc, 0.05, H[5][4]); emg_mac(acc, 0.1, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][2]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.0011904761904761906, G[3][2]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<18, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[1][0]); emg_mac(acc, 0.1, H[1][1]); emg_mac(acc, 0.05, H[1][3]); emg_mac(acc, 0.2, H[2][0]); emg_mac(acc, 0.2, H[2][1]); emg_mac(acc, 0.1, H[2][3]); emg_mac(acc, 0.05, H[5][0]); emg_mac(acc, 0.1, H[5][1]); emg_mac(acc, 0.1, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.0011904761904761906, G[0][2]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<18, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[1][0]); emg_mac(acc, 0.1, H[1][2]); emg_mac(acc, 0.05, H[1][4]); emg_mac(acc, 0.1, H[2][0]); emg_mac(acc, 0.2, H[2][2]); emg_mac(acc, 0.1, H[2][4]); emg_mac(acc, 0.05, H[5][0]); emg_mac(acc, 0.1, H[5][2]); emg_mac(acc, 0.1, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[0][0]); emg_mac(acc, -0.0011904761904761906, G[0][3]); emg_mac(acc, -0.0011904761904761906, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<18, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[1][1]); emg_mac(acc, 0.1, H[1][2]); emg_mac(acc, 0.05, H[1][5]); emg_mac(acc, 0.1, H[2][1]); emg_mac(acc, 0.4, H[2][2]); emg_mac(acc, 0.1, H[2][5]); emg_mac(acc, 0.05, H[5][1]); emg_mac(acc, 0.1, H[5][2]); emg_mac(acc, 0.1, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[0][0]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<18, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[1][3]); emg_mac(acc, 0.1, H[1][4]); emg_mac(acc, 0.05, H[1][5]); emg_mac(acc, 0.1, H[2][3]); emg_mac(acc, 0.4, H[2][4]); emg_mac(acc, 0.1, H[2][5]); emg_mac(acc, 0.05, H[5][3]); emg_mac(acc, 0.1, H[5][4]); emg_mac(acc, 0.05, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[0][1]); emg_mac(acc, -0.002380952380952381, G[0][3]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<19, 0> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[3][0]); emg_mac(acc, 1.0, H[4][0]); emg_mac(acc, 0.5, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.008333333333333333, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][1]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][1]); }
};
template <> struct Pair<19, 1> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[3][1]); emg_mac(acc, 1.0, H[4][1]); emg_mac(acc, 0.5, H[5][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, -0.016666666666666666, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][2]); }
};
template <> struct Pair<19, 2> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[3][2]); emg_mac(acc, 1.0, H[4][2]); emg_mac(acc, 0.5, H[5][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][0]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[3][0]); emg_mac(acc, 0.008333333333333333, G[3][3]); }
};
template <> struct Pair<19, 3> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[3][3]); emg_mac(acc, 1.0, H[4][3]); emg_mac(acc, 0.5, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][2]); emg_mac(acc, -0.016666666666666666, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][2]); }
};
template <> struct Pair<19, 4> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[3][4]); emg_mac(acc, 1.0, H[4][4]); emg_mac(acc, 0.5, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][1]); emg_mac(acc, -0.008333333333333333, G[1][3]); emg_mac(acc, -0.008333333333333333, G[3][1]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<19, 5> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.5, H[3][5]); emg_mac(acc, 1.0, H[4][5]); emg_mac(acc, 0.5, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.016666666666666666, G[1][2]); emg_mac(acc, -0.016666666666666666, G[1][3]); emg_mac(acc, -0.008333333333333333, G[3][2]); emg_mac(acc, 0.016666666666666666, G[3][3]); }
};
template <> struct Pair<19, 6> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[5][0]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.0011904761904761906, G[1][0]); emg_mac(acc, -0.0011904761904761906, G[1][1]); emg_mac(acc, 0.004761904761904762, G[3][0]); }
};
template <> struct Pair<19, 7> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[4][1]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][0]); emg_mac(acc, 0.004761904761904762, G[3][0]); }
};
template <> struct Pair<19, 8> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[3][2]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][0]); emg_mac(acc, 0.0011904761904761906, G[3][0]); emg_mac(acc, 0.0011904761904761906, G[3][3]); }
};
template <> struct Pair<19, 9> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.3, H[4][3]); emg_mac(acc, 0.15, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.002380952380952381, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<19, 10> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[3][4]); emg_mac(acc, 0.15, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.004761904761904762, G[1][1]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<19, 11> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.15, H[3][5]); emg_mac(acc, 0.3, H[4][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, -0.002380952380952381, G[1][2]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<19, 12> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.05, H[3][0]); emg_mac(acc, 0.05, H[3][1]); emg_mac(acc, 0.1, H[3][3]); emg_mac(acc, -0.2, H[4][0]); emg_mac(acc, 0.1, H[4][1]); emg_mac(acc, 0.2, H[4][3]); emg_mac(acc, -0.05, H[5][0]); emg_mac(acc, 0.1, H[5][1]); emg_mac(acc, 0.1, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, -0.0011904761904761906, G[1][2]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<19, 13> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[3][0]); emg_mac(acc, 0.05, H[3][2]); emg_mac(acc, 0.1, H[3][4]); emg_mac(acc, -0.1, H[4][0]); emg_mac(acc, 0.1, H[4][2]); emg_mac(acc, 0.2, H[4][4]); emg_mac(acc, -0.05, H[5][0]); emg_mac(acc, 0.1, H[5][2]); emg_mac(acc, 0.1, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][1]); emg_mac(acc, -0.0011904761904761906, G[1][3]); emg_mac(acc, -0.0011904761904761906, G[3][1]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<19, 14> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[3][1]); emg_mac(acc, 0.05, H[3][2]); emg_mac(acc, 0.1, H[3][5]); emg_mac(acc, -0.1, H[4][1]); emg_mac(acc, 0.2, H[4][2]); emg_mac(acc, 0.2, H[4][5]); emg_mac(acc, -0.05, H[5][1]); emg_mac(acc, 0.05, H[5][2]); emg_mac(acc, 0.1, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][2]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.0011904761904761906, G[3][2]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<19, 15> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, -0.1, H[3][3]); emg_mac(acc, 0.05, H[3][4]); emg_mac(acc, 0.1, H[3][5]); emg_mac(acc, -0.1, H[4][3]); emg_mac(acc, 0.2, H[4][4]); emg_mac(acc, 0.2, H[4][5]); emg_mac(acc, -0.05, H[5][3]); emg_mac(acc, 0.05, H[5][4]); emg_mac(acc, 0.2, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][2]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[3][2]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
template <> struct Pair<19, 16> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.05, H[3][0]); emg_mac(acc, 0.1, H[3][1]); emg_mac(acc, 0.05, H[3][3]); emg_mac(acc, 0.2, H[4][0]); emg_mac(acc, 0.2, H[4][1]); emg_mac(acc, 0.1, H[4][3]); emg_mac(acc, 0.05, H[5][0]); emg_mac(acc, 0.2, H[5][1]); emg_mac(acc, 0.05, H[5][3]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][0]); emg_mac(acc, -0.0011904761904761906, G[1][2]); emg_mac(acc, -0.004761904761904762, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][2]); }
};
template <> struct Pair<19, 17> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[3][0]); emg_mac(acc, 0.1, H[3][2]); emg_mac(acc, 0.05, H[3][4]); emg_mac(acc, 0.1, H[4][0]); emg_mac(acc, 0.2, H[4][2]); emg_mac(acc, 0.1, H[4][4]); emg_mac(acc, 0.05, H[5][0]); emg_mac(acc, 0.2, H[5][2]); emg_mac(acc, 0.05, H[5][4]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.002380952380952381, G[1][0]); emg_mac(acc, -0.0011904761904761906, G[1][3]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<19, 18> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[3][1]); emg_mac(acc, 0.1, H[3][2]); emg_mac(acc, 0.05, H[3][5]); emg_mac(acc, 0.1, H[4][1]); emg_mac(acc, 0.4, H[4][2]); emg_mac(acc, 0.1, H[4][5]); emg_mac(acc, 0.05, H[5][1]); emg_mac(acc, 0.1, H[5][2]); emg_mac(acc, 0.05, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[1][0]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[3][0]); emg_mac(acc, 0.002380952380952381, G[3][3]); }
};
template <> struct Pair<19, 19> {
  template <class A, class T> __device__ __forceinline__ static void stiff(A &acc, const T &H) { emg_mac(acc, 0.1, H[3][3]); emg_mac(acc, 0.1, H[3][4]); emg_mac(acc, 0.05, H[3][5]); emg_mac(acc, 0.1, H[4][3]); emg_mac(acc, 0.4, H[4][4]); emg_mac(acc, 0.1, H[4][5]); emg_mac(acc, 0.05, H[5][3]); emg_mac(acc, 0.1, H[5][4]); emg_mac(acc, 0.1, H[5][5]); }
  template <class A, class T> __device__ __forceinline__ static void mass(A &acc, const T &G) { emg_mac(acc, 0.004761904761904762, G[1][1]); emg_mac(acc, -0.002380952380952381, G[1][3]); emg_mac(acc, -0.002380952380952381, G[3][1]); emg_mac(acc, 0.004761904761904762, G[3][3]); }
};
// total multiply-adds over the 400 ordered pairs: 2474
}  // namespace emg_tables
